// gi_kernels.cu -- sm_100a kernels of the mesh-mesh intersector.
//
// Build (once per mesh, replaces the reference's level-cut / forest builders,
// include/third-party/cubql/level_cut_builder.h:278-364 and forest_builder.h:405-517,
// which loop on the host with a device sync per tree level):
//   k_validate -> k_tri_boxes -> k_morton -> radix sort -> k_karras -> k_leaves
//   -> k_refit (bottom-up, atomic arrival counters) -> k_depth -> scan -> k_collapse
// No host round trip between kernels.
//
// Intersect (replaces crossCheck.cu, DualTreeStep.cu, rapidDescendKernel.cu and the
// chunk loop of SingleTreeBatchIntersector.cu:170-455 in the reference):
//   k_traverse  one cooperative persistent launch: level-synchronous BVH4 x BVH4
//               traversal (16 child pairs per node pair, one half-warp each),
//               warp-aggregated appends, bounded software grid barrier between
//               levels, then the first filter stage over all leaf pairs.
//   k_exact     FP64 filter + exact integer signs for the escalated pairs.
//   k_segments  intersection sets and correctly rounded endpoints.
//   ordering    radix sort by (job, a, b) and gathers.
#include <atomic>
#include <cstdio>

#include "gi_classify.cuh"
#include "gi_launch.h"
#include "gi_sort.cuh"

namespace gi {

static std::atomic<unsigned long long> g_launches{0};
void note_launches(unsigned n)
{
    g_launches.fetch_add(n, std::memory_order_relaxed);
}
unsigned long long launch_count()
{
    return g_launches.load(std::memory_order_relaxed);
}

// ===========================================================================
// Build
// ===========================================================================
__global__ void k_validate(const double* __restrict__ V, uint32_t nv, const uint32_t* __restrict__ T, uint32_t nt,
                           unsigned* err)
{
    size_t i = blockIdx.x * (size_t)blockDim.x + threadIdx.x;
    size_t stride = (size_t)gridDim.x * blockDim.x;
    for (size_t k = i; k < 3ull * nv; k += stride) {
        double x = V[k];
        double a = fabs(x);
        if (!(a <= 0x1p100) || (x != 0.0 && a < 0x1p-100)) atomicOr(err, 2u);
    }
    for (size_t k = i; k < 3ull * nt; k += stride)
        if (T[k] >= nv) atomicOr(err, 1u);
}

__device__ __forceinline__ unsigned f2ord(float f)
{
    unsigned u = __float_as_uint(f);
    return (u & 0x80000000u) ? ~u : (u | 0x80000000u);
}
__device__ __forceinline__ float ord2f(unsigned u)
{
    return __uint_as_float((u & 0x80000000u) ? (u & 0x7fffffffu) : ~u);
}

// FP32 boxes rounded outward (so every exact triangle lies inside its box) and
// centroid bounds.  The reference rounds to nearest (src/common/utils.cu:639),
// which can drop true pairs; outward rounding keeps the candidate set a superset.
__global__ void k_tri_boxes(const double* __restrict__ V, const uint32_t* __restrict__ T, uint32_t nt,
                            float* __restrict__ box, double* __restrict__ box64, unsigned* __restrict__ cb)
{
    float cmin[3] = {INFINITY, INFINITY, INFINITY}, cmax[3] = {-INFINITY, -INFINITY, -INFINITY};
    for (uint32_t t = blockIdx.x * blockDim.x + threadIdx.x; t < nt; t += gridDim.x * blockDim.x) {
        uint32_t i0 = T[3 * (size_t)t], i1 = T[3 * (size_t)t + 1], i2 = T[3 * (size_t)t + 2];
        for (int k = 0; k < 3; k++) {
            double a = V[3 * (size_t)i0 + k], b = V[3 * (size_t)i1 + k], c = V[3 * (size_t)i2 + k];
            double lo = fmin(a, fmin(b, c)), hi = fmax(a, fmax(b, c));
            float flo = __double2float_rd(lo), fhi = __double2float_ru(hi);
            box[6 * (size_t)t + k] = flo;
            box[6 * (size_t)t + 3 + k] = fhi;
            if (box64) {
                box64[6 * (size_t)t + k] = lo;
                box64[6 * (size_t)t + 3 + k] = hi;
            }
            float cc = 0.5f * flo + 0.5f * fhi;
            cmin[k] = fminf(cmin[k], cc);
            cmax[k] = fmaxf(cmax[k], cc);
        }
    }
    for (int k = 0; k < 3; k++) {
        for (int o = 16; o > 0; o >>= 1) {
            cmin[k] = fminf(cmin[k], __shfl_xor_sync(0xffffffffu, cmin[k], o));
            cmax[k] = fmaxf(cmax[k], __shfl_xor_sync(0xffffffffu, cmax[k], o));
        }
    }
    if ((threadIdx.x & 31) == 0) {
        for (int k = 0; k < 3; k++) {
            atomicMin(&cb[k], f2ord(cmin[k]));
            atomicMax(&cb[3 + k], f2ord(cmax[k]));
        }
    }
}

__device__ __forceinline__ uint32_t spread10(uint32_t x)
{
    x &= 0x3ffu;
    x = (x | (x << 16)) & 0x030000FFu;
    x = (x | (x << 8)) & 0x0300F00Fu;
    x = (x | (x << 4)) & 0x030C30C3u;
    x = (x | (x << 2)) & 0x09249249u;
    return x;
}

__global__ void k_morton(const float* __restrict__ box, uint32_t nt, const unsigned* __restrict__ cb,
                         uint32_t* __restrict__ keys, uint32_t* __restrict__ vals)
{
    uint32_t t = blockIdx.x * blockDim.x + threadIdx.x;
    if (t >= nt) return;
    uint32_t q[3];
    for (int k = 0; k < 3; k++) {
        float lo = ord2f(cb[k]), hi = ord2f(cb[3 + k]);
        float c = 0.5f * box[6 * (size_t)t + k] + 0.5f * box[6 * (size_t)t + 3 + k];
        float ext = hi - lo;
        float f = ext > 0.0f ? (c - lo) / ext : 0.0f;
        f = fminf(fmaxf(f, 0.0f), 1.0f);
        q[k] = (uint32_t)fminf(f * 1024.0f, 1023.0f);
    }
    keys[t] = (spread10(q[0]) << 2) | (spread10(q[1]) << 1) | spread10(q[2]);
    vals[t] = t;
}

__device__ __forceinline__ int kdelta(const uint32_t* __restrict__ keys, int n, int i, int j)
{
    if (j < 0 || j >= n) return -1;
    uint32_t a = keys[i], b = keys[j];
    if (a == b) return 32 + __clz((unsigned)(i ^ j));
    return __clz(a ^ b);
}

// Karras 2012 radix-tree construction over sorted Morton keys (ties by index).
__global__ void k_karras(const uint32_t* __restrict__ keys, int n, uint2* __restrict__ child, int* __restrict__ parent)
{
    int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= n - 1) return;
    int d = (kdelta(keys, n, i, i + 1) - kdelta(keys, n, i, i - 1)) >= 0 ? 1 : -1;
    int dmin = kdelta(keys, n, i, i - d);
    int lmax = 2;
    while (kdelta(keys, n, i, i + lmax * d) > dmin) lmax <<= 1;
    int l = 0;
    for (int t = lmax >> 1; t >= 1; t >>= 1)
        if (kdelta(keys, n, i, i + (l + t) * d) > dmin) l += t;
    int j = i + l * d;
    int dnode = kdelta(keys, n, i, j);
    int s = 0, t = l;
    do {
        t = (t + 1) >> 1;
        if (kdelta(keys, n, i, i + (s + t) * d) > dnode) s += t;
    } while (t > 1);
    int gamma = i + s * d + min(d, 0);
    uint32_t left = (min(i, j) == gamma) ? (kLeaf | (uint32_t)gamma) : (uint32_t)gamma;
    uint32_t right = (max(i, j) == gamma + 1) ? (kLeaf | (uint32_t)(gamma + 1)) : (uint32_t)(gamma + 1);
    child[i] = make_uint2(left, right);
    parent[(left & kLeaf) ? (n - 1 + (int)(left & ~kLeaf)) : (int)left] = i;
    parent[(right & kLeaf) ? (n - 1 + (int)(right & ~kLeaf)) : (int)right] = i;
    if (i == 0) parent[0] = -1;
}

template <class S>
__global__ void k_leaves(const uint32_t* __restrict__ vals, uint32_t n, const uint32_t* __restrict__ T,
                         const S* __restrict__ boxOrig, S* __restrict__ leafBox, uint4* __restrict__ leafTri)
{
    uint32_t p = blockIdx.x * blockDim.x + threadIdx.x;
    if (p >= n) return;
    uint32_t tri = vals[p];
    for (int k = 0; k < 6; k++) leafBox[6 * (size_t)p + k] = boxOrig[6 * (size_t)tri + k];
    if (leafTri) leafTri[p] = make_uint4(T[3 * (size_t)tri], T[3 * (size_t)tri + 1], T[3 * (size_t)tri + 2], tri);
}

template <class S>
__device__ __forceinline__ S ldcg_s(const S* p);
template <>
__device__ __forceinline__ float ldcg_s<float>(const float* p)
{
    return __ldcg(p);
}
template <>
__device__ __forceinline__ double ldcg_s<double>(const double* p)
{
    return __ldcg(p);
}

// Bottom-up refit: the second thread to arrive at a node merges both children.
template <class S>
__global__ void k_refit(int n, const uint2* __restrict__ child, const int* __restrict__ parent,
                        const S* __restrict__ leafBox, S* nodeBox, unsigned* flags)
{
    int p = blockIdx.x * blockDim.x + threadIdx.x;
    if (p >= n) return;
    int node = parent[n - 1 + p];
    for (int guard = 0; node >= 0 && guard < n; guard++) {
        __threadfence();
        if (atomicAdd(&flags[node], 1u) == 0u) return;
        __threadfence();
        uint2 c = child[node];
        S b[6];
        for (int side = 0; side < 2; side++) {
            uint32_t r = side ? c.y : c.x;
            const S* src = (r & kLeaf) ? leafBox + 6 * (size_t)(r & ~kLeaf) : nodeBox + 6 * (size_t)r;
            for (int k = 0; k < 6; k++) {
                S v = ldcg_s<S>(src + k);
                if (side == 0) b[k] = v;
                else b[k] = (k < 3) ? (v < b[k] ? v : b[k]) : (v > b[k] ? v : b[k]);
            }
        }
        for (int k = 0; k < 6; k++) nodeBox[6 * (size_t)node + k] = b[k];
        __threadfence();
        node = parent[node];
    }
}

__global__ void k_depth(int n, const int* __restrict__ parent, uint32_t* __restrict__ even)
{
    int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= n - 1) return;
    int d = 0, x = i;
    while (x > 0 && d < n) {
        x = parent[x];
        d++;
    }
    even[i] = (d & 1) == 0;
}

template <class S, class NodeT>
__global__ void k_collapse(int n, const uint2* __restrict__ child, const uint32_t* __restrict__ even,
                           const uint32_t* __restrict__ widx, const S* __restrict__ leafBox,
                           const S* __restrict__ nodeBox, NodeT* __restrict__ nodes)
{
    int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= n - 1 || !even[i]) return;
    uint32_t slot[4];
    int ns = 0;
    uint2 c = child[i];
    uint32_t cc[2] = {c.x, c.y};
    for (int s = 0; s < 2; s++) {
        if (cc[s] & kLeaf) {
            slot[ns++] = cc[s];
        } else {
            uint2 g = child[cc[s]];
            slot[ns++] = g.x;
            slot[ns++] = g.y;
        }
    }
    NodeT out;
    for (int k = 0; k < 4; k++) {
        if (k < ns) {
            uint32_t r = slot[k];
            const S* src = (r & kLeaf) ? leafBox + 6 * (size_t)(r & ~kLeaf) : nodeBox + 6 * (size_t)r;
            out.lox[k] = src[0];
            out.loy[k] = src[1];
            out.loz[k] = src[2];
            out.hix[k] = src[3];
            out.hiy[k] = src[4];
            out.hiz[k] = src[5];
            out.child[k] = (r & kLeaf) ? r : widx[r];
        } else {
            out.lox[k] = out.loy[k] = out.loz[k] = (S)INFINITY;
            out.hix[k] = out.hiy[k] = out.hiz[k] = (S)-INFINITY;
            out.child[k] = kEmpty;
        }
    }
    for (int k = 0; k < (int)(sizeof(out.pad) / sizeof(out.pad[0])); k++) out.pad[k] = 0;
    nodes[widx[i]] = out;
}

cudaError_t launch_validate(const double* verts, uint32_t nv, const uint32_t* tris, uint32_t nt, unsigned* d_err,
                            cudaStream_t st)
{
    k_validate<<<1024, 256, 0, st>>>(verts, nv, tris, nt, d_err);
    note_launches(1);
    return cudaGetLastError();
}

#define GI_TRY(x)                                \
    do {                                         \
        cudaError_t e_ = (x);                    \
        if (e_ != cudaSuccess) return e_;        \
    } while (0)

cudaError_t build_bvh(MeshBuffers& m, bool fp64, cudaStream_t st)
{
    const uint32_t n = m.nt;
    if (n == 0) {
        m.root = kEmpty;
        m.nnodes = 0;
        return cudaSuccess;
    }
    // scratch
    float* box = nullptr;
    double* box64 = nullptr;
    unsigned* cb = nullptr;
    uint32_t *k0 = nullptr, *v0 = nullptr, *k1 = nullptr, *v1 = nullptr, *counts = nullptr, *stemp = nullptr;
    uint2* child = nullptr;
    int* parent = nullptr;
    unsigned* flags = nullptr;
    uint32_t *even = nullptr, *widx = nullptr;
    void* nodeBox = nullptr;
    size_t cw = radix_counts_words(n);
    size_t sw = scan_temp_words(cw > n ? cw : n);
    GI_TRY(cudaMallocAsync(&box, sizeof(float) * 6 * n, st));
    if (fp64) GI_TRY(cudaMallocAsync(&box64, sizeof(double) * 6 * n, st));
    GI_TRY(cudaMallocAsync(&cb, sizeof(unsigned) * 8, st));
    GI_TRY(cudaMallocAsync(&k0, sizeof(uint32_t) * n, st));
    GI_TRY(cudaMallocAsync(&v0, sizeof(uint32_t) * n, st));
    GI_TRY(cudaMallocAsync(&k1, sizeof(uint32_t) * n, st));
    GI_TRY(cudaMallocAsync(&v1, sizeof(uint32_t) * n, st));
    GI_TRY(cudaMallocAsync(&counts, sizeof(uint32_t) * cw, st));
    GI_TRY(cudaMallocAsync(&stemp, sizeof(uint32_t) * sw, st));
    unsigned cbinit[8] = {0xffffffffu, 0xffffffffu, 0xffffffffu, 0u, 0u, 0u, 0u, 0u};
    GI_TRY(cudaMemcpyAsync(cb, cbinit, sizeof(cbinit), cudaMemcpyHostToDevice, st));
    int tb = 256;
    int gb = (int)((n + tb - 1) / tb);
    k_tri_boxes<<<gb < 4096 ? gb : 4096, tb, 0, st>>>(m.verts, m.tris, n, box, box64, cb);
    k_morton<<<gb, tb, 0, st>>>(box, n, cb, k0, v0);
    radix_sort<uint32_t>(k0, v0, k1, v1, n, 30, counts, stemp, st);
    // leaves in sorted order
    if (!fp64) {
        GI_TRY(cudaMallocAsync(&m.leafBox, sizeof(float) * 6 * n, st));
        GI_TRY(cudaMallocAsync(&m.leafTri, sizeof(uint4) * n, st));
        k_leaves<float><<<gb, tb, 0, st>>>(v0, n, m.tris, box, m.leafBox, m.leafTri);
    } else {
        GI_TRY(cudaMallocAsync(&m.leafBox64, sizeof(double) * 6 * n, st));
        k_leaves<double><<<gb, tb, 0, st>>>(v0, n, m.tris, box64, m.leafBox64, nullptr);
    }
    if (n == 1) {
        m.root = kLeaf | 0u;
        m.nnodes = 0;
    } else {
        GI_TRY(cudaMallocAsync(&child, sizeof(uint2) * (n - 1), st));
        GI_TRY(cudaMallocAsync(&parent, sizeof(int) * (2 * (size_t)n - 1), st));
        GI_TRY(cudaMallocAsync(&flags, sizeof(unsigned) * (n - 1), st));
        GI_TRY(cudaMallocAsync(&even, sizeof(uint32_t) * (n - 1), st));
        GI_TRY(cudaMallocAsync(&widx, sizeof(uint32_t) * (n - 1), st));
        GI_TRY(cudaMallocAsync(&nodeBox, (fp64 ? sizeof(double) : sizeof(float)) * 6 * (n - 1), st));
        GI_TRY(cudaMemsetAsync(flags, 0, sizeof(unsigned) * (n - 1), st));
        int gi_ = (int)((n - 1 + tb - 1) / tb);
        k_karras<<<gi_, tb, 0, st>>>(k0, (int)n, child, parent);
        if (!fp64)
            k_refit<float><<<gb, tb, 0, st>>>((int)n, child, parent, m.leafBox, (float*)nodeBox, flags);
        else
            k_refit<double><<<gb, tb, 0, st>>>((int)n, child, parent, m.leafBox64, (double*)nodeBox, flags);
        k_depth<<<gi_, tb, 0, st>>>((int)n, parent, even);
        scan_exclusive(even, widx, n - 1, stemp, st);
        // number of wide nodes = widx[n-2] + even[n-2]
        uint32_t last[2];
        GI_TRY(cudaMemcpyAsync(&last[0], widx + (n - 2), sizeof(uint32_t), cudaMemcpyDeviceToHost, st));
        GI_TRY(cudaMemcpyAsync(&last[1], even + (n - 2), sizeof(uint32_t), cudaMemcpyDeviceToHost, st));
        GI_TRY(cudaStreamSynchronize(st));
        uint32_t nw = last[0] + last[1];
        if (!fp64) {
            GI_TRY(cudaMallocAsync(&m.nodes, sizeof(WNode) * (size_t)nw, st));
            k_collapse<float, WNode><<<gi_, tb, 0, st>>>((int)n, child, even, widx, m.leafBox, (float*)nodeBox,
                                                         m.nodes);
        } else {
            GI_TRY(cudaMallocAsync(&m.nodes64, sizeof(WNode64) * (size_t)nw, st));
            k_collapse<double, WNode64><<<gi_, tb, 0, st>>>((int)n, child, even, widx, m.leafBox64,
                                                            (double*)nodeBox, m.nodes64);
        }
        m.nnodes = nw;
        m.root = 0;
    }
    GI_TRY(cudaGetLastError());
    cudaFreeAsync(box, st);
    if (box64) cudaFreeAsync(box64, st);
    cudaFreeAsync(cb, st);
    cudaFreeAsync(k0, st);
    cudaFreeAsync(v0, st);
    cudaFreeAsync(k1, st);
    cudaFreeAsync(v1, st);
    cudaFreeAsync(counts, st);
    cudaFreeAsync(stemp, st);
    if (child) cudaFreeAsync(child, st);
    if (parent) cudaFreeAsync(parent, st);
    if (flags) cudaFreeAsync(flags, st);
    if (even) cudaFreeAsync(even, st);
    if (widx) cudaFreeAsync(widx, st);
    if (nodeBox) cudaFreeAsync(nodeBox, st);
    if (!fp64)
        m.bytes += sizeof(float) * 6 * (size_t)n + sizeof(uint4) * (size_t)n + sizeof(WNode) * (size_t)m.nnodes;
    else
        m.bytes += sizeof(double) * 6 * (size_t)n + sizeof(WNode64) * (size_t)m.nnodes;
    return cudaGetLastError();
}

// ===========================================================================
// Traversal
// ===========================================================================
template <class S>
struct Box {
    S lo[3], hi[3];
};

// Conservative world box of a local box under a pose:
//   centre' = Rf c + bf, half' = |Rf| h, padded by rho (|Rf|(|c| + h) + padm) + tau.
// rho = 2^-19 (FP32) / 2^-48 (FP64) covers, with a margin of >= 3x, the rounding of
// Rf and bf, of the box arithmetic, of c and h, and of the FP64 posed vertices.
__device__ __forceinline__ void world_box(const DevPose& P, Box<float>& b)
{
    float c[3], h[3];
    for (int k = 0; k < 3; k++) {
        c[k] = 0.5f * b.lo[k] + 0.5f * b.hi[k];
        h[k] = 0.5f * b.hi[k] - 0.5f * b.lo[k];
    }
    for (int r = 0; r < 3; r++) {
        float wc = P.bf[r], wh = 0.0f, mag = P.padm[r];
        for (int k = 0; k < 3; k++) {
            float a = P.Rf[3 * r + k];
            wc = fmaf(a, c[k], wc);
            wh = fmaf(fabsf(a), h[k], wh);
            mag = fmaf(fabsf(a), fabsf(c[k]) + h[k], mag);
        }
        float pad = fmaf(0x1p-19f, mag, 0x1p-120f);
        b.lo[r] = wc - wh - pad;
        b.hi[r] = wc + wh + pad;
    }
}
__device__ __forceinline__ void world_box(const DevPose& P, Box<double>& b)
{
    double c[3], h[3];
    for (int k = 0; k < 3; k++) {
        c[k] = 0.5 * b.lo[k] + 0.5 * b.hi[k];
        h[k] = 0.5 * b.hi[k] - 0.5 * b.lo[k];
    }
    for (int r = 0; r < 3; r++) {
        double wc = P.b64[r], wh = 0.0, mag = P.padm64[r];
        for (int k = 0; k < 3; k++) {
            double a = P.R[3 * r + k];
            wc = fma(a, c[k], wc);
            wh = fma(fabs(a), h[k], wh);
            mag = fma(fabs(a), fabs(c[k]) + h[k], mag);
        }
        double pad = fma(0x1p-48, mag, 0x1p-300);
        b.lo[r] = wc - wh - pad;
        b.hi[r] = wc + wh + pad;
    }
}

template <bool F64>
struct Prec;
template <>
struct Prec<false> {
    using S = float;
    using Node = WNode;
    static __device__ __forceinline__ const Node* nodes(const MeshDev& M) { return M.nodes; }
    static __device__ __forceinline__ const S* leafBox(const MeshDev& M) { return M.leafBox; }
};
template <>
struct Prec<true> {
    using S = double;
    using Node = WNode64;
    static __device__ __forceinline__ const Node* nodes(const MeshDev& M) { return M.nodes64; }
    static __device__ __forceinline__ const S* leafBox(const MeshDev& M) { return M.leafBox64; }
};

template <bool F64>
__device__ __forceinline__ bool load_child(const MeshDev& M, uint32_t ref, int i, Box<typename Prec<F64>::S>& b,
                                           uint32_t& cref)
{
    using S = typename Prec<F64>::S;
    if (ref == kEmpty) return false;
    if (ref & kLeaf) {
        if (i != 0) return false;
        const S* lb = Prec<F64>::leafBox(M) + 6 * (size_t)(ref & ~kLeaf);
        for (int k = 0; k < 3; k++) {
            b.lo[k] = __ldg(lb + k);
            b.hi[k] = __ldg(lb + 3 + k);
        }
        cref = ref;
        return true;
    }
    const typename Prec<F64>::Node* nd = Prec<F64>::nodes(M) + ref;
    cref = __ldg(&nd->child[i]);
    if (cref == kEmpty) return false;
    b.lo[0] = __ldg(&nd->lox[i]);
    b.lo[1] = __ldg(&nd->loy[i]);
    b.lo[2] = __ldg(&nd->loz[i]);
    b.hi[0] = __ldg(&nd->hix[i]);
    b.hi[1] = __ldg(&nd->hiy[i]);
    b.hi[2] = __ldg(&nd->hiz[i]);
    return true;
}

template <class S>
__device__ __forceinline__ bool overlap(const Box<S>& a, const Box<S>& b)
{
    return a.lo[0] <= b.hi[0] && b.lo[0] <= a.hi[0] && a.lo[1] <= b.hi[1] && b.lo[1] <= a.hi[1] &&
           a.lo[2] <= b.hi[2] && b.lo[2] <= a.hi[2];
}

__device__ __forceinline__ unsigned warp_append(bool pred, unsigned* counter)
{
    const unsigned lane = threadIdx.x & 31;
    unsigned m = __ballot_sync(0xffffffffu, pred);
    if (m == 0) return 0;
    unsigned leader = __ffs(m) - 1;
    unsigned base = 0;
    if (lane == leader) base = atomicAdd(counter, (unsigned)__popc(m));
    base = __shfl_sync(0xffffffffu, base, leader);
    return base + __popc(m & ((1u << lane) - 1u));
}

__device__ __forceinline__ unsigned ld_cg_u32(const unsigned* p)
{
    return __ldcg(p);
}

constexpr unsigned long long kBarrierSpins = 1ull << 22;

// Software grid barrier for a cooperative launch (all blocks co-resident).
// Every wait is bounded: after kBarrierSpins polls the block records
// kErrBarrier and continues; the kernel then drains and the host reports
// GI_ERR_TIMEOUT.
__device__ void grid_sync(Counters* C)
{
    __syncthreads();
    if (threadIdx.x == 0) {
        volatile unsigned* genp = &C->bar_gen;
        unsigned g = *genp;
        __threadfence();
        unsigned arrived = atomicAdd(&C->bar_count, 1u);
        if (arrived == gridDim.x - 1) {
            atomicExch(&C->bar_count, 0u);
            __threadfence();
            atomicAdd(&C->bar_gen, 1u);
        } else {
            unsigned long long spins = 0;
            while (*genp == g) {
                if (++spins > kBarrierSpins) {
                    atomicOr(&C->err, kErrBarrier);
                    break;
                }
                __nanosleep(100);
            }
        }
        __threadfence();
    }
    __syncthreads();
}

template <bool F64>
__device__ __forceinline__ void load_tri(const MeshDev& M, const DevPose& P, uint32_t pos, double3* out,
                                         uint32_t* tri_id)
{
    uint4 t = __ldg(M.leafTri + pos);
    out[0] = world_vertex(M.verts, t.x, P);
    out[1] = world_vertex(M.verts, t.y, P);
    out[2] = world_vertex(M.verts, t.z, P);
    *tri_id = t.w;
}

template <bool F64>
__global__ void __launch_bounds__(256) k_traverse(Bufs B)
{
    using S = typename Prec<F64>::S;
    Counters* C = B.cnt;
    const unsigned lane = threadIdx.x & 31;
    const unsigned warp = (blockIdx.x * blockDim.x + threadIdx.x) >> 5;
    const unsigned nwarps = (gridDim.x * blockDim.x) >> 5;
    const unsigned hl = lane & 15, ci = hl & 3, cj = hl >> 2, half = lane >> 4;
    unsigned long long visited = 0;
    unsigned level = 0;
    for (; level < 4096; level++) {
        const unsigned cur = level % 3, nxt = (level + 1) % 3, clr = (level + 2) % 3;
        unsigned n = ld_cg_u32(&C->front[cur]);
        if (n == 0 || ld_cg_u32(&C->overflow) || ld_cg_u32(&C->err)) break;
        if (n > B.cap_front) n = B.cap_front;
        if (blockIdx.x == 0 && threadIdx.x == 0) C->front[clr] = 0;
        const uint4* in = B.front[level & 1];
        uint4* out = B.front[(level + 1) & 1];
        for (unsigned base = warp * 2; base < n; base += nwarps * 2) {
            const unsigned e = base + half;
            const bool have = e < n;
            uint4 ent = have ? __ldcg(in + e) : make_uint4(0u, kEmpty, kEmpty, 0u);
            visited += (have && hl == 0);
            const JobDev& J = B.jobs[ent.x];
            Box<S> ba, bb;
            uint32_t ca = kEmpty, cb = kEmpty;
            bool va = have && load_child<F64>(J.A, ent.y, ci, ba, ca);
            bool vb = have && load_child<F64>(J.B, ent.z, cj, bb, cb);
            bool valid = va && vb;
            if (valid) {
                if (!J.pa.identity) world_box(J.pa, ba);
                if (!J.pb.identity) world_box(J.pb, bb);
                valid = overlap(ba, bb);
            }
            const bool isCand = valid && (ca & kLeaf) && (cb & kLeaf);
            const bool isFront = valid && !isCand;
            unsigned pf = warp_append(isFront, &C->front[nxt]);
            if (isFront) {
                if (pf < B.cap_front) out[pf] = make_uint4(ent.x, ca, cb, 0u);
                else atomicOr(&C->overflow, kOvfFrontier);
            }
            unsigned pc = warp_append(isCand, &C->cand);
            if (isCand) {
                if (pc < B.cap_cand) B.cand[pc] = make_uint4(ent.x, ca & ~kLeaf, cb & ~kLeaf, 0u);
                else atomicOr(&C->overflow, kOvfCand);
            }
        }
        grid_sync(C);
    }
    if (blockIdx.x == 0 && threadIdx.x == 0) C->levels = level;
    for (int o = 16; o > 0; o >>= 1) visited += __shfl_xor_sync(0xffffffffu, visited, o);
    if (lane == 0 && visited) atomicAdd(&C->node_pairs, visited);
    if (ld_cg_u32(&C->overflow) || ld_cg_u32(&C->err)) return;

    // ---- first filter stage over all leaf pairs ----
    unsigned nc = ld_cg_u32(&C->cand);
    if (nc > B.cap_cand) nc = B.cap_cand;
    unsigned long long decided = 0;
    for (unsigned base = warp * 32; base < nc; base += nwarps * 32) {
        const unsigned i = base + lane;
        const bool have = i < nc;
        int dec = DEC_NO;
        uint32_t ta = 0, tb = 0, job = 0;
        if (have) {
            uint4 c = __ldcg(B.cand + i);
            job = c.x;
            const JobDev& J = B.jobs[job];
            double3 P[3], Q[3];
            load_tri<F64>(J.A, J.pa, c.y, P, &ta);
            load_tri<F64>(J.B, J.pb, c.z, Q, &tb);
            if constexpr (F64) dec = classify_fast<double>(P, Q);
            else dec = classify_fast<float>(P, Q);
            decided += (dec != DEC_ESC);
        }
        const bool yes = have && dec == DEC_YES;
        const bool esc = have && dec == DEC_ESC;
        unsigned pr = warp_append(yes, &C->res);
        if (yes) {
            if (pr < B.cap_res) B.res[pr] = make_uint4(job, ta, tb, 0u);
            else atomicOr(&C->overflow, kOvfRes);
        }
        unsigned pe = warp_append(esc, &C->esc);
        if (esc) {
            if (pe < B.cap_esc) B.esc[pe] = i;
            else atomicOr(&C->overflow, kOvfEsc);
        }
    }
    for (int o = 16; o > 0; o >>= 1) decided += __shfl_xor_sync(0xffffffffu, decided, o);
    if (lane == 0 && decided) atomicAdd(&C->filter_decided, decided);
}

// ===========================================================================
// Exact stage and segments
// ===========================================================================
__global__ void __launch_bounds__(128) k_exact(Bufs B)
{
    Counters* C = B.cnt;
    const unsigned lane = threadIdx.x & 31;
    const unsigned gtid = blockIdx.x * blockDim.x + threadIdx.x;
    const unsigned nth = gridDim.x * blockDim.x;
    unsigned ne = ld_cg_u32(&C->esc);
    if (ne > B.cap_esc) ne = B.cap_esc;
    unsigned long long nexact = 0;
    for (unsigned base = gtid - lane; base < ne; base += nth) {
        const unsigned i = base + lane;
        const bool have = i < ne;
        bool yes = false;
        uint32_t ta = 0, tb = 0, job = 0;
        if (have) {
            uint4 c = __ldcg(B.cand + __ldcg(B.esc + i));
            job = c.x;
            const JobDev& J = B.jobs[job];
            double3 pts[6];
            load_tri<false>(J.A, J.pa, c.y, pts, &ta);
            load_tri<false>(J.B, J.pb, c.z, pts + 3, &tb);
            ExactSigns S{&C->err, 0ull};
            TTRes r;
            classify_exact(pts, r, S);
            yes = r.kind != KIND_NONE;
            nexact += S.nexact;
        }
        unsigned pr = warp_append(yes, &C->res);
        if (yes) {
            if (pr < B.cap_res) B.res[pr] = make_uint4(job, ta, tb, 0u);
            else atomicOr(&C->overflow, kOvfRes);
        }
    }
    for (int o = 16; o > 0; o >>= 1) nexact += __shfl_xor_sync(0xffffffffu, nexact, o);
    if (lane == 0 && nexact) atomicAdd(&C->exact_signs, nexact);
}

__device__ __forceinline__ void load_tri_orig(const MeshDev& M, const DevPose& P, uint32_t tri, double3* out)
{
    const uint32_t* t = M.tris + 3 * (size_t)tri;
    out[0] = world_vertex(M.verts, __ldg(t), P);
    out[1] = world_vertex(M.verts, __ldg(t + 1), P);
    out[2] = world_vertex(M.verts, __ldg(t + 2), P);
}

__global__ void __launch_bounds__(128) k_segments(Bufs B, uint32_t nres, double* __restrict__ segs,
                                                  uint32_t* __restrict__ nseg)
{
    Counters* C = B.cnt;
    const unsigned gtid = blockIdx.x * blockDim.x + threadIdx.x;
    const unsigned nth = gridDim.x * blockDim.x;
    for (unsigned i = gtid; i < nres; i += nth) {
        uint4 rr = __ldcg(B.res + i);
        const JobDev& J = B.jobs[rr.x];
        double3 pts[6];
        load_tri_orig(J.A, J.pa, rr.y, pts);
        load_tri_orig(J.B, J.pb, rr.z, pts + 3);
        ExactSigns S{&C->err, 0ull};
        TTRes r;
        classify_exact(pts, r, S);
        double3 q[3];
        uint32_t ns = 0;
        if (r.kind == KIND_POINT || r.kind == KIND_SEGMENT || r.kind == KIND_TRIANGLE) {
            for (int k = 0; k < r.n && k < 3; k++)
                if (!construct_point(pts, r.pt[k], q[k], &C->exact_points)) atomicOr(&C->err, kErrExactCapacity);
            double* o = segs + 18 * (size_t)i;
            if (r.kind == KIND_POINT) {
                double v[6] = {q[0].x, q[0].y, q[0].z, q[0].x, q[0].y, q[0].z};
                for (int k = 0; k < 6; k++) o[k] = v[k];
                ns = 1;
            } else if (r.kind == KIND_SEGMENT) {
                double v[6] = {q[0].x, q[0].y, q[0].z, q[1].x, q[1].y, q[1].z};
                for (int k = 0; k < 6; k++) o[k] = v[k];
                ns = 1;
            } else {
                for (int e = 0; e < 3; e++) {
                    const double3& u = q[e];
                    const double3& w = q[(e + 1) % 3];
                    double v[6] = {u.x, u.y, u.z, w.x, w.y, w.z};
                    for (int k = 0; k < 6; k++) o[6 * e + k] = v[k];
                }
                ns = 3;
            }
        }
        nseg[i] = ns;
    }
}

// ===========================================================================
// Ordering
// ===========================================================================
__global__ void k_order_keys(const uint4* __restrict__ res, uint32_t n, int bits_a, int bits_b,
                             unsigned long long* __restrict__ keys, uint32_t* __restrict__ vals)
{
    uint32_t i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= n) return;
    uint4 r = res[i];
    keys[i] = ((unsigned long long)r.x << (bits_a + bits_b)) | ((unsigned long long)r.y << bits_b) | r.z;
    vals[i] = i;
}
__global__ void k_iota(uint32_t* v, uint32_t n)
{
    uint32_t i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i < n) v[i] = i;
}

size_t scan_temp_words_host(size_t n)
{
    return scan_temp_words(n);
}

size_t order_scratch_bytes(uint32_t n)
{
    size_t cw = radix_counts_words(n);
    size_t sw = scan_temp_words(cw > n ? cw : n);
    return 2 * sizeof(unsigned long long) * (size_t)n + sizeof(uint32_t) * ((size_t)n + cw + sw) + 1024;
}

cudaError_t launch_order(const uint4* res, uint32_t n, int bits_a, int bits_b, int bits_job, bool sort,
                         uint32_t* perm_out, OrderScratch scratch, cudaStream_t st)
{
    if (n == 0) return cudaSuccess;
    int tb = 256, gb = (int)((n + tb - 1) / tb);
    if (!sort) {
        k_iota<<<gb, tb, 0, st>>>(perm_out, n);
        note_launches(1);
        return cudaGetLastError();
    }
    char* p = (char*)scratch.ptr;
    unsigned long long* k0 = (unsigned long long*)p;
    p += sizeof(unsigned long long) * (size_t)n;
    unsigned long long* k1 = (unsigned long long*)p;
    p += sizeof(unsigned long long) * (size_t)n;
    uint32_t* v1 = (uint32_t*)p;
    p += sizeof(uint32_t) * (size_t)n;
    size_t cw = radix_counts_words(n);
    uint32_t* counts = (uint32_t*)p;
    p += sizeof(uint32_t) * cw;
    uint32_t* stemp = (uint32_t*)p;
    k_order_keys<<<gb, tb, 0, st>>>(res, n, bits_a, bits_b, k0, perm_out);
    note_launches(1);
    radix_sort<unsigned long long>(k0, perm_out, k1, v1, n, bits_a + bits_b + bits_job, counts, stemp, st);
    return cudaGetLastError();
}

__global__ void k_gather_pairs(const uint4* __restrict__ res, const uint32_t* __restrict__ perm, uint32_t n,
                               const uint32_t* __restrict__ nseg, int32_t* __restrict__ pairs_out,
                               uint32_t* __restrict__ job_out, uint32_t* __restrict__ cnt_sorted)
{
    uint32_t k = blockIdx.x * blockDim.x + threadIdx.x;
    if (k >= n) return;
    uint32_t s = perm[k];
    uint4 r = res[s];
    pairs_out[2 * (size_t)k] = (int32_t)r.y;
    pairs_out[2 * (size_t)k + 1] = (int32_t)r.z;
    if (job_out) job_out[k] = r.x;
    if (cnt_sorted) cnt_sorted[k] = nseg[s];
}
__global__ void k_gather_segs(const uint32_t* __restrict__ perm, uint32_t n, const double* __restrict__ segs,
                              const uint32_t* __restrict__ nseg, const uint32_t* __restrict__ off,
                              double* __restrict__ segs_out, int32_t* __restrict__ segpair_out, uint32_t* total)
{
    uint32_t k = blockIdx.x * blockDim.x + threadIdx.x;
    if (k >= n) return;
    uint32_t s = perm[k];
    uint32_t c = nseg[s], o = off[k];
    for (uint32_t q = 0; q < c; q++) {
        for (int j = 0; j < 6; j++) segs_out[6 * (size_t)(o + q) + j] = segs[18 * (size_t)s + 6 * q + j];
        segpair_out[o + q] = (int32_t)k;
    }
    if (k == n - 1) *total = o + c;
}

cudaError_t launch_gather(const uint4* res, const uint32_t* perm, uint32_t n, const double* segs,
                          const uint32_t* nseg, int32_t* pairs_out, uint32_t* job_out, double* segs_out,
                          int32_t* segpair_out, uint32_t* seg_offsets, uint32_t* seg_scan_temp, bool want_segments,
                          uint32_t* d_total_segs, cudaStream_t st)
{
    if (n == 0) return cudaSuccess;
    int tb = 256, gb = (int)((n + tb - 1) / tb);
    k_gather_pairs<<<gb, tb, 0, st>>>(res, perm, n, nseg, pairs_out, job_out, want_segments ? seg_offsets : nullptr);
    note_launches(1);
    if (want_segments) {
        scan_exclusive(seg_offsets, seg_offsets, n, seg_scan_temp, st);
        k_gather_segs<<<gb, tb, 0, st>>>(perm, n, segs, nseg, seg_offsets, segs_out, segpair_out, d_total_segs);
        note_launches(1);
    }
    return cudaGetLastError();
}

// ===========================================================================
// Launchers
// ===========================================================================
__global__ void k_init_frontier(Bufs B)
{
    uint32_t j = blockIdx.x * blockDim.x + threadIdx.x;
    if (j >= B.njobs) return;
    const JobDev& J = B.jobs[j];
    if (J.A.nt == 0 || J.B.nt == 0) return;
    unsigned p = atomicAdd(&B.cnt->front[0], 1u);
    B.front[0][p] = make_uint4(j, J.A.root, J.B.root, 0u);
}

cudaError_t launch_init_frontier(const Bufs& b, cudaStream_t st)
{
    k_init_frontier<<<(b.njobs + 255) / 256, 256, 0, st>>>(b);
    note_launches(1);
    return cudaGetLastError();
}

cudaError_t query_launch(int device, LaunchCfg* cfg)
{
    cudaDeviceProp prop;
    GI_TRY(cudaGetDeviceProperties(&prop, device));
    cfg->sms = prop.multiProcessorCount;
    int b32 = 0, b64 = 0;
    GI_TRY(cudaOccupancyMaxActiveBlocksPerMultiprocessor(&b32, k_traverse<false>, 256, 0));
    GI_TRY(cudaOccupancyMaxActiveBlocksPerMultiprocessor(&b64, k_traverse<true>, 256, 0));
    int b = b32 < b64 ? b32 : b64;
    if (b < 1) b = 1;
    cfg->trav_blocks = b * cfg->sms;
    cfg->trav_threads = 256;
    return cudaSuccess;
}

cudaError_t launch_traverse(const Bufs& b, const LaunchCfg& cfg, int precision, cudaStream_t st)
{
    Bufs args = b;
    void* params[] = {&args};
    note_launches(1);
    if (precision == 1)
        return cudaLaunchCooperativeKernel((const void*)k_traverse<true>, dim3(cfg.trav_blocks), dim3(256), params, 0,
                                           st);
    return cudaLaunchCooperativeKernel((const void*)k_traverse<false>, dim3(cfg.trav_blocks), dim3(256), params, 0,
                                       st);
}

cudaError_t launch_exact(const Bufs& b, const LaunchCfg& cfg, cudaStream_t st)
{
    k_exact<<<cfg.sms * 4, 128, 0, st>>>(b);
    note_launches(1);
    return cudaGetLastError();
}

cudaError_t launch_segments(const Bufs& b, uint32_t nres, double* segs, uint32_t* nseg, const LaunchCfg& cfg,
                            cudaStream_t st)
{
    if (nres == 0) return cudaSuccess;
    unsigned blocks = (nres + 127) / 128;
    unsigned maxb = cfg.sms * 8;
    k_segments<<<blocks < maxb ? blocks : maxb, 128, 0, st>>>(b, nres, segs, nseg);
    note_launches(1);
    return cudaGetLastError();
}

}  // namespace gi
