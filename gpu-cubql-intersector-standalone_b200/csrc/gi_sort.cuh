// gi_sort.cuh -- device scan and LSD radix sort (8- or 10-bit digits, stable).
//
// Used by the BVH build (30-bit Morton keys, replaces the reference's CUB
// DeviceRadixSort in include/third-party/cubql/level_cut_builder.h:345-347)
// and by output ordering (64-bit (job, a, b) keys).
#pragma once
#include <cstdint>
#include <cuda_runtime.h>

#include "gi_internal.cuh"

namespace gi {

// counts kernel launches made by this library (for gi_stats.launches)
void note_launches(unsigned n);

// Programmatic dependent launch of the build's kernels.  A kernel launched by
// launch_dep may be scheduled while the kernel before it in the stream is still
// finishing; at its first statement (pdl_enter) it waits for that kernel's
// completion and memory (griddepcontrol.wait), then lets its own successor be
// scheduled (griddepcontrol.launch_dependents).  Because the wait comes first
// in every such kernel, each one starts its work after all earlier kernels of
// the stream have completed, as in a plain launch; only the launch latency of
// the next kernel overlaps the tail of the current one.  In a plain launch both
// instructions are no-ops.
__device__ __forceinline__ void pdl_enter()
{
    asm volatile("griddepcontrol.wait;" ::: "memory");
    asm volatile("griddepcontrol.launch_dependents;" ::: "memory");
}

// Launches k(args...) with programmatic stream serialisation; a launch the
// driver refuses is repeated as a plain launch.
template <class... KArgs, class... Args>
inline void launch_dep(void (*k)(KArgs...), unsigned grid, unsigned block, cudaStream_t st, Args... args)
{
    cudaLaunchConfig_t lc = {};
    lc.gridDim = dim3(grid);
    lc.blockDim = dim3(block);
    lc.dynamicSmemBytes = 0;
    lc.stream = st;
    cudaLaunchAttribute at[1];
    at[0].id = cudaLaunchAttributeProgrammaticStreamSerialization;
    at[0].val.programmaticStreamSerializationAllowed = 1;
    lc.attrs = at;
    lc.numAttrs = 1;
    if (cudaLaunchKernelEx(&lc, k, args...) != cudaSuccess) {
        (void)cudaGetLastError();
        k<<<grid, block, 0, st>>>(args...);
    }
}

constexpr int kScanThreads = 1024;
constexpr int kScanItems = 4;
constexpr int kScanTile = kScanThreads * kScanItems;

// block-wide exclusive scan of per-thread sums; returns the block total
__device__ __forceinline__ uint32_t block_exclusive_scan(uint32_t v, uint32_t* smem_warp, uint32_t* total)
{
    const int lane = threadIdx.x & 31, wid = threadIdx.x >> 5, nw = blockDim.x >> 5;
    uint32_t x = v;
#pragma unroll
    for (int o = 1; o < 32; o <<= 1) {
        uint32_t y = __shfl_up_sync(0xffffffffu, x, o);
        if (lane >= o) x += y;
    }
    if (lane == 31) smem_warp[wid] = x;
    __syncthreads();
    if (wid == 0) {
        uint32_t w = lane < nw ? smem_warp[lane] : 0u;
        uint32_t s = w;
#pragma unroll
        for (int o = 1; o < 32; o <<= 1) {
            uint32_t y = __shfl_up_sync(0xffffffffu, s, o);
            if (lane >= o) s += y;
        }
        if (lane < nw) smem_warp[lane] = s - w;
        if (lane == nw - 1) smem_warp[32] = s;
    }
    __syncthreads();
    uint32_t r = smem_warp[wid] + x - v;
    *total = smem_warp[32];
    __syncthreads();
    return r;
}

__global__ void k_scan_tiles(const uint32_t* in, uint32_t* out, uint32_t n, uint32_t* tile_sums)
{
    pdl_enter();
    __shared__ uint32_t sw[33];
    uint32_t base = blockIdx.x * kScanTile + threadIdx.x * kScanItems;
    uint32_t v[kScanItems];
    uint32_t s = 0;
#pragma unroll
    for (int k = 0; k < kScanItems; k++) {
        v[k] = (base + k < n) ? in[base + k] : 0u;
        s += v[k];
    }
    uint32_t tot;
    uint32_t ex = block_exclusive_scan(s, sw, &tot);
#pragma unroll
    for (int k = 0; k < kScanItems; k++) {
        if (base + k < n) out[base + k] = ex;
        ex += v[k];
    }
    if (threadIdx.x == 0 && tile_sums) tile_sums[blockIdx.x] = tot;
}

__global__ void k_scan_add(uint32_t* out, uint32_t n, const uint32_t* tile_offsets)
{
    pdl_enter();
    uint32_t add = tile_offsets[blockIdx.x];
    uint32_t base = blockIdx.x * kScanTile + threadIdx.x * kScanItems;
#pragma unroll
    for (int k = 0; k < kScanItems; k++)
        if (base + k < n) out[base + k] += add;
}

// exclusive scan of n uint32 (in and out may alias); temp needs scan_temp_words(n)
inline size_t scan_temp_words(size_t n)
{
    size_t t = 0;
    while (n > (size_t)kScanTile) {
        n = (n + kScanTile - 1) / kScanTile;
        t += n + 1;
    }
    return t + 1;
}
inline void scan_exclusive(const uint32_t* in, uint32_t* out, uint32_t n, uint32_t* temp, cudaStream_t st)
{
    if (n == 0) return;
    uint32_t tiles = (n + kScanTile - 1) / kScanTile;
    if (tiles == 1) {
        launch_dep(k_scan_tiles, 1, kScanThreads, st, in, out, n, (uint32_t*)nullptr);
        note_launches(1);
        return;
    }
    uint32_t* sums = temp;
    launch_dep(k_scan_tiles, tiles, kScanThreads, st, in, out, n, sums);
    scan_exclusive(sums, sums, tiles, temp + tiles + 1, st);
    launch_dep(k_scan_add, tiles, kScanThreads, st, out, n, (const uint32_t*)sums);
    note_launches(2);
}

// Exclusive scan left in two parts: out[] holds the scan within each tile of
// kScanTile words and *sums (nullptr for a single tile) the scanned tile
// totals, so that the full scan at j is out[j] + sums[j / kScanTile].  A
// consumer that adds the tile offset itself saves the add pass.
inline void scan_exclusive_split(const uint32_t* in, uint32_t* out, uint32_t n, uint32_t* temp, const uint32_t** sums,
                                 cudaStream_t st)
{
    *sums = nullptr;
    if (n == 0) return;
    uint32_t tiles = (n + kScanTile - 1) / kScanTile;
    launch_dep(k_scan_tiles, tiles, kScanThreads, st, in, out, n, tiles > 1 ? temp : (uint32_t*)nullptr);
    note_launches(1);
    if (tiles > 1) {
        scan_exclusive(temp, temp, tiles, temp + tiles + 1, st);
        *sums = temp;
    }
}

// ---------------------------------------------------------------------------
// Decoupled look-back (tile prefix sums in one pass): a status word per tile
// and slot holds a flag and a count, the tile's own aggregate first, then its
// inclusive prefix.
// ---------------------------------------------------------------------------
constexpr unsigned kFlagAgg = 1u << 30, kFlagInc = 2u << 30, kCountMask = (1u << 30) - 1u;
constexpr unsigned long long kLookbackSpins = 1ull << 22;

// Exclusive prefix of this tile over the preceding tiles, per status slot.
// Returns false if a wait ran out (the error bit is set; results are invalid).
__device__ __forceinline__ bool lookback(unsigned* status, unsigned tile, unsigned stride, unsigned own,
                                         unsigned* excl_out, unsigned* err)
{
    unsigned excl = 0;
    if (tile > 0) {
        // publish the local aggregate first so successors need not wait for our prefix
        atomicExch(status + (size_t)tile * stride, kFlagAgg | (own & kCountMask));
        unsigned t = tile - 1;
        for (;;) {
            volatile unsigned* q = status + (size_t)t * stride;
            unsigned v = *q;
            unsigned long long spins = 0;
            while ((v & ~kCountMask) == 0u) {
                if (++spins > kLookbackSpins) {
                    atomicOr(err, kErrTimeout);
                    *excl_out = 0;
                    return false;
                }
                __nanosleep(32);
                v = *q;
            }
            excl += v & kCountMask;
            if ((v & ~kCountMask) == kFlagInc || t == 0) break;
            t--;
        }
    }
    __threadfence();
    atomicExch(status + (size_t)tile * stride, kFlagInc | ((excl + own) & kCountMask));
    *excl_out = excl;
    return true;
}

// ---------------------------------------------------------------------------
// Radix sort
// ---------------------------------------------------------------------------
// 12 keys per thread: 427 tiles of 3,072 keys for a 1.3M-triangle mesh, which
// keeps more scatter warps resident per SM than 4,096-key tiles (build 0.435 ->
// 0.418 ms on B200; 10 and 14 keys per thread gave 0.427 and 0.426 ms, 8 keys
// 0.436 ms: smaller tiles pay more per-tile overhead)
constexpr int kRsThreads = 256;
constexpr int kRsItems = 12;
constexpr int kRsTile = kRsThreads * kRsItems;  // 3072
constexpr int kRsWarps = kRsThreads / 32;

template <class K, int BITS>
__global__ void __launch_bounds__(kRsThreads) k_rs_hist(const K* __restrict__ keys, uint32_t n, int shift,
                                                        uint32_t* __restrict__ counts, uint32_t ntiles)
{
    pdl_enter();
    constexpr uint32_t kDig = 1u << BITS;
    __shared__ uint32_t h[kDig];
    for (uint32_t d = threadIdx.x; d < kDig; d += kRsThreads) h[d] = 0;
    __syncthreads();
    // every load of the tile is issued before the first shared-memory atomic
    // (one round trip to memory per thread instead of one per few keys)
    uint32_t base = blockIdx.x * kRsTile;
    K kk[kRsItems];
#pragma unroll
    for (int k = 0; k < kRsItems; k++) {
        const uint32_t i = base + k * kRsThreads + threadIdx.x;
        kk[k] = i < n ? keys[i] : (K)0;
    }
#pragma unroll
    for (int k = 0; k < kRsItems; k++) {
        const uint32_t i = base + k * kRsThreads + threadIdx.x;
        if (i < n) atomicAdd(&h[(uint32_t)(kk[k] >> shift) & (kDig - 1u)], 1u);
    }
    __syncthreads();
    for (uint32_t d = threadIdx.x; d < kDig; d += kRsThreads) counts[d * ntiles + blockIdx.x] = h[d];
}

template <class K, int BITS>
__global__ void __launch_bounds__(kRsThreads) k_rs_scatter(const K* __restrict__ kin, const uint32_t* __restrict__ vin,
                                                           K* __restrict__ kout, uint32_t* __restrict__ vout, uint32_t n,
                                                           int shift, const uint32_t* __restrict__ offsets,
                                                           const uint32_t* __restrict__ tile_sums, uint32_t ntiles)
{
    pdl_enter();
    constexpr uint32_t kDig = 1u << BITS;
    __shared__ uint32_t wc[kRsWarps][kDig];
    __shared__ uint32_t tile_off[kDig];
    const int lane = threadIdx.x & 31, w = threadIdx.x >> 5;
    for (uint32_t d = lane; d < kDig; d += 32) wc[w][d] = 0;
    for (uint32_t d = threadIdx.x; d < kDig; d += kRsThreads) {
        const uint32_t j = d * ntiles + blockIdx.x;
        tile_off[d] = offsets[j] + (tile_sums ? tile_sums[j / kScanTile] : 0u);
    }
    __syncwarp();
    const uint32_t seg = blockIdx.x * kRsTile + w * 32 * kRsItems;
    K key[kRsItems];
    uint32_t val[kRsItems];
    uint32_t rank[kRsItems];
    uint32_t dig[kRsItems];
    const unsigned lt = (1u << lane) - 1u;
#pragma unroll
    for (int c = 0; c < kRsItems; c++) {
        uint32_t i = seg + c * 32 + lane;
        bool ok = i < n;
        key[c] = ok ? kin[i] : (K)0;
        val[c] = ok ? vin[i] : 0u;
        uint32_t d = ok ? ((uint32_t)(key[c] >> shift) & (kDig - 1u)) : kDig;
        dig[c] = d;
        unsigned peers = __match_any_sync(0xffffffffu, d);
        uint32_t r = 0;
        if (ok) r = wc[w][d] + __popc(peers & lt);
        rank[c] = r;
        __syncwarp();
        if (ok && (peers & lt) == 0) wc[w][d] += __popc(peers);
        __syncwarp();
    }
    __syncthreads();
    // per digit: exclusive prefix over warps
    for (uint32_t d = threadIdx.x; d < kDig; d += kRsThreads) {
        uint32_t run = 0;
        for (int q = 0; q < kRsWarps; q++) {
            uint32_t t = wc[q][d];
            wc[q][d] = run;
            run += t;
        }
    }
    __syncthreads();
#pragma unroll
    for (int c = 0; c < kRsItems; c++) {
        uint32_t d = dig[c];
        if (d < kDig) {
            uint32_t pos = tile_off[d] + wc[w][d] + rank[c];
            kout[pos] = key[c];
            vout[pos] = val[c];
        }
    }
}

// Sorts (keys, vals) by the low `bits` bits of the key in passes of BITS-bit
// digits.  The passes alternate between the two buffer pairs; on return
// (k0, v0) point to the pair that holds the result and (k1, v1) to the other
// (swapped after an odd number of passes, nothing copied).  Scratch: counts
// radix_counts_words<BITS>(n) words, scan temp.  hist0_done: the producer of the
// keys already wrote the first pass's per-tile digit counts into `counts`
// (layout of k_rs_hist: digit-major, one column per kRsTile keys).
template <class K, int BITS = 8>
void radix_sort(K*& k0, uint32_t*& v0, K*& k1, uint32_t*& v1, uint32_t n, int bits, uint32_t* counts, uint32_t* temp,
                cudaStream_t st, bool hist0_done = false)
{
    if (n <= 1) return;
    uint32_t ntiles = (n + kRsTile - 1) / kRsTile;
    int passes = (bits + BITS - 1) / BITS;
    K* ks = k0;
    uint32_t* vs = v0;
    K* kd = k1;
    uint32_t* vd = v1;
    for (int p = 0; p < passes; p++) {
        if (p > 0 || !hist0_done) {
            launch_dep(k_rs_hist<K, BITS>, ntiles, kRsThreads, st, (const K*)ks, n, BITS * p, counts, ntiles);
            note_launches(1);
        }
        const uint32_t* sums = nullptr;
        scan_exclusive_split(counts, counts, (1u << BITS) * ntiles, temp, &sums, st);
        launch_dep(k_rs_scatter<K, BITS>, ntiles, kRsThreads, st, (const K*)ks, (const uint32_t*)vs, kd, vd, n,
                   BITS * p, (const uint32_t*)counts, sums, ntiles);
        note_launches(1);
        K* tk = ks;
        ks = kd;
        kd = tk;
        uint32_t* tv = vs;
        vs = vd;
        vd = tv;
    }
    k1 = kd;
    v1 = vd;
    k0 = ks;
    v0 = vs;
}

template <int BITS = 8>
inline size_t radix_counts_words(uint32_t n)
{
    return (1ull << BITS) * ((n + kRsTile - 1) / kRsTile);
}

}  // namespace gi
