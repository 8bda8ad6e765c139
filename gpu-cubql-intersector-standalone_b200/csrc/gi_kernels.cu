// gi_kernels.cu -- sm_100a kernels of the mesh-mesh intersector.
//
// Build (once per mesh, replaces the reference's level-cut / forest builders,
// include/third-party/cubql/level_cut_builder.h:278-364 and forest_builder.h:405-517,
// which loop on the host with a device sync per tree level):
//   k_validate -> k_tri_boxes -> k_morton_hist -> radix sort -> k_karras_leaves (leaves + binary tree)
//   -> k_state_tables -> k_wide_flags -> scan -> k_collapse (size-greedy 4-wide nodes,
//   topology) -> k_refit_wide (bottom-up over the wide tree, atomic arrival counters)
// One host round trip, for the wide-node count (the node array's size).
//
// Intersect (replaces crossCheck.cu, DualTreeStep.cu, rapidDescendKernel.cu and the
// chunk loop of SingleTreeBatchIntersector.cu:170-455 in the reference):
//   k_traverse  one persistent launch: seeding from the cut pairs, BVH4 x BVH4
//               traversal through warp stacks and a device work queue (16 child
//               pairs per node pair; no grid barrier), and the first filter
//               stage on the leaf pairs, run by warps without node pairs.
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

// Boxes are 6 consecutive values (lo xyz, hi xyz): 24 B for float (8-byte
// aligned), 48 B for double (16-byte aligned), moved as three 2-vectors.
template <class S>
struct Vec2Of;
template <>
struct Vec2Of<float> {
    using T = float2;
};
template <>
struct Vec2Of<double> {
    using T = double2;
};
template <class S>
__device__ __forceinline__ void load_box_cg(const S* p, S b[6])
{
    using V = typename Vec2Of<S>::T;
    const V* q = reinterpret_cast<const V*>(p);
    const V a = __ldcg(q), c = __ldcg(q + 1), d = __ldcg(q + 2);
    b[0] = a.x, b[1] = a.y, b[2] = c.x, b[3] = c.y, b[4] = d.x, b[5] = d.y;
}
template <class S>
__device__ __forceinline__ void store_box(S* p, const S b[6])
{
    using V = typename Vec2Of<S>::T;
    V* q = reinterpret_cast<V*>(p);
    q[0] = V{b[0], b[1]};
    q[1] = V{b[2], b[3]};
    q[2] = V{b[4], b[5]};
}

// FP32 boxes rounded outward (so every exact triangle lies inside its box) and
// centroid bounds.  The reference rounds to nearest (src/common/utils.cu:639),
// which can drop true pairs; outward rounding keeps the candidate set a superset.
constexpr int kTriBoxThreads = 256;
__global__ void __launch_bounds__(kTriBoxThreads, 4) k_tri_boxes(const double* __restrict__ V, uint32_t nv,
                                                              const uint32_t* __restrict__ T, uint32_t nt,
                                                              float* __restrict__ box, double* __restrict__ box64,
                                                              unsigned* __restrict__ cb)
{
    pdl_enter();
    float cmin[3] = {INFINITY, INFINITY, INFINITY}, cmax[3] = {-INFINITY, -INFINITY, -INFINITY};
    // two triangles per iteration, all their loads issued before any use
    const uint32_t stride = gridDim.x * blockDim.x;
    for (uint32_t t = blockIdx.x * blockDim.x + threadIdx.x; t < nt; t += 2 * stride) {
        const uint32_t tt[2] = {t, t + stride < nt ? t + stride : t};
        uint32_t ix[2][3];
        double v[2][9];
#pragma unroll
        for (int q = 0; q < 2; q++)
#pragma unroll
            for (int j = 0; j < 3; j++) ix[q][j] = min(T[3 * (size_t)tt[q] + j], nv - 1u);  // validated later
#pragma unroll
        for (int q = 0; q < 2; q++)
#pragma unroll
            for (int j = 0; j < 3; j++) {
                const double3 p = load_vertex(V, ix[q][j]);
                v[q][3 * j] = p.x;
                v[q][3 * j + 1] = p.y;
                v[q][3 * j + 2] = p.z;
            }
#pragma unroll
        for (int q = 0; q < 2; q++) {
            if (q == 1 && tt[1] == t) break;
            const size_t o = 6 * (size_t)tt[q];
            float fb[6];
#pragma unroll
            for (int k = 0; k < 3; k++) {
                const double a = v[q][k], b = v[q][3 + k], c = v[q][6 + k];
                const double lo = fmin(a, fmin(b, c)), hi = fmax(a, fmax(b, c));
                fb[k] = __double2float_rd(lo);
                fb[3 + k] = __double2float_ru(hi);
                if (box64) {
                    box64[o + k] = lo;
                    box64[o + 3 + k] = hi;
                }
                const float cc = 0.5f * fb[k] + 0.5f * fb[3 + k];
                cmin[k] = fminf(cmin[k], cc);
                cmax[k] = fmaxf(cmax[k], cc);
            }
            store_box(box + o, fb);
        }
    }
    // block reduction, then one set of atomics per block: per-warp atomics on
    // the same six words serialised in L2 and dominated the kernel
    __shared__ float red[kTriBoxThreads / 32][6];
    for (int k = 0; k < 3; k++) {
        for (int o = 16; o > 0; o >>= 1) {
            cmin[k] = fminf(cmin[k], __shfl_xor_sync(0xffffffffu, cmin[k], o));
            cmax[k] = fmaxf(cmax[k], __shfl_xor_sync(0xffffffffu, cmax[k], o));
        }
    }
    const int lane = threadIdx.x & 31, w = threadIdx.x >> 5;
    if (lane == 0)
        for (int k = 0; k < 3; k++) {
            red[w][k] = cmin[k];
            red[w][3 + k] = cmax[k];
        }
    __syncthreads();
    if (threadIdx.x < 6) {
        const int k = threadIdx.x;
        float v = red[0][k];
        for (int q = 1; q < kTriBoxThreads / 32; q++) v = k < 3 ? fminf(v, red[q][k]) : fmaxf(v, red[q][k]);
        if (k < 3) atomicMin(&cb[k], f2ord(v));
        else atomicMax(&cb[k], f2ord(v));
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

// Box centre coordinate c quantised to 10 bits over [lo, lo + ext].
__device__ __forceinline__ uint32_t morton_axis(float c, float lo, float ext)
{
    float f = ext > 0.0f ? (c - lo) / ext : 0.0f;
    f = fminf(fmaxf(f, 0.0f), 1.0f);
    return (uint32_t)fminf(f * 1024.0f, 1023.0f);
}

// 30-bit Morton keys of the triangles (their box centres quantised to 10 bits
// per axis over the centroid bounds cb: ordered-float min x, y, z, max x, y,
// z) with identity values, kRsTile triangles per block, and each block's counts
// of the first radix digit in the layout of k_rs_hist (digit-major, one column
// per block), so the sort's first pass needs no histogram launch.  All of a
// thread's box loads are issued before its first shared-memory atomic.
template <int BITS>
__global__ void __launch_bounds__(kRsThreads) k_morton_hist(const float* __restrict__ box, uint32_t nt,
                                                            const unsigned* __restrict__ cb,
                                                            uint32_t* __restrict__ keys, uint32_t* __restrict__ vals,
                                                            uint32_t* __restrict__ counts, uint32_t ntiles)
{
    pdl_enter();
    constexpr uint32_t kDig = 1u << BITS;
    __shared__ uint32_t h[kDig];
    for (uint32_t d = threadIdx.x; d < kDig; d += kRsThreads) h[d] = 0;
    float lo[3], ext[3];
#pragma unroll
    for (int k = 0; k < 3; k++) {
        lo[k] = ord2f(cb[k]);
        ext[k] = ord2f(cb[3 + k]) - lo[k];
    }
    const uint32_t base = blockIdx.x * kRsTile;
    uint32_t kk[kRsItems];
#pragma unroll
    for (int it = 0; it < kRsItems; it++) {
        const uint32_t t = base + it * kRsThreads + threadIdx.x;
        kk[it] = 0;
        if (t < nt) {
            const float2* b2 = reinterpret_cast<const float2*>(box + 6 * (size_t)t);
            const float2 a = b2[0], b = b2[1], c = b2[2];  // lo x, y | lo z, hi x | hi y, z
            const uint32_t qx = morton_axis(0.5f * a.x + 0.5f * b.y, lo[0], ext[0]);
            const uint32_t qy = morton_axis(0.5f * a.y + 0.5f * c.x, lo[1], ext[1]);
            const uint32_t qz = morton_axis(0.5f * b.x + 0.5f * c.y, lo[2], ext[2]);
            kk[it] = (spread10(qx) << 2) | (spread10(qy) << 1) | spread10(qz);
        }
    }
    __syncthreads();  // the histogram is cleared
#pragma unroll
    for (int it = 0; it < kRsItems; it++) {
        const uint32_t t = base + it * kRsThreads + threadIdx.x;
        if (t < nt) {
            keys[t] = kk[it];
            vals[t] = t;
            atomicAdd(&h[kk[it] & (kDig - 1u)], 1u);
        }
    }
    __syncthreads();
    for (uint32_t d = threadIdx.x; d < kDig; d += kRsThreads) counts[d * ntiles + blockIdx.x] = h[d];
}

__device__ __forceinline__ int kdelta(const uint32_t* __restrict__ keys, int n, int i, int j)
{
    if (j < 0 || j >= n) return -1;
    uint32_t a = keys[i], b = keys[j];
    if (a == b) return 32 + __clz((unsigned)(i ^ j));
    return __clz(a ^ b);
}

// Karras 2012 radix-tree construction over sorted Morton keys (ties by index),
// internal node i (i < n - 1).  child[i] = (left ref, right ref, leaves under
// left, leaves under right); parent[] of the internal children (the root's is -1).
__device__ __forceinline__ void karras_node(int i, const uint32_t* __restrict__ keys, int n, uint4* __restrict__ child,
                                            int* __restrict__ parent)
{
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
    const int lo = min(i, j), hi = max(i, j);
    child[i] = make_uint4(left, right, (uint32_t)(gamma - lo + 1), (uint32_t)(hi - gamma));
    if (!(left & kLeaf)) parent[left] = i;
    if (!(right & kLeaf)) parent[right] = i;
    if (i == 0) parent[0] = -1;
}

// Leaves in sorted order (position p < n: the box and the vertex indices of
// triangle vals[p]) and the radix tree's internal node p (p < n - 1), in one
// launch: both are gathers or searches bound by latency, so each thread has
// two independent chains in flight.
template <class S>
__global__ void k_karras_leaves(const uint32_t* __restrict__ keys, const uint32_t* __restrict__ vals, int n,
                                const uint32_t* __restrict__ T, const S* __restrict__ boxOrig,
                                S* __restrict__ leafBox, uint4* __restrict__ leafTri, uint4* __restrict__ child,
                                int* __restrict__ parent)
{
    pdl_enter();
    const int p = blockIdx.x * blockDim.x + threadIdx.x;
    if (p >= n) return;
    const uint32_t tri = vals[p];
    S b[6];
    load_box_cg(boxOrig + 6 * (size_t)tri, b);
    uint4 t4 = make_uint4(0u, 0u, 0u, 0u);
    if (leafTri) t4 = make_uint4(T[3 * (size_t)tri], T[3 * (size_t)tri + 1], T[3 * (size_t)tri + 2], tri);
    if (p < n - 1) karras_node(p, keys, n, child, parent);
    store_box(leafBox + 6 * (size_t)p, b);
    if (leafTri) leafTri[p] = t4;
}

__device__ __forceinline__ unsigned arrive_acq_rel(unsigned* f)
{
    unsigned old;
    asm volatile("atom.acq_rel.gpu.global.add.u32 %0, [%1], 1;" : "=r"(old) : "l"(f) : "memory");
    return old;
}

// ---------------------------------------------------------------------------
// Collapse of the binary radix tree into the 4-wide BVH, size-greedy.
//
// A wide node is made from a binary node r by opening r and then, twice, the
// part with the most leaves (ties: the leftmost part), as long as that part is
// an internal node; the parts stay in left-to-right order.  Each binary node is
// thus either a wide node (state W) or opened in the second (O2) or third (O3)
// step of its wide ancestor's expansion.  Opening the largest part shrinks
// the largest subtree of a wide node faster than taking grandchildren by
// depth parity does on the unbalanced trees that Morton splits give on a
// surface: on a 1.3 M-triangle sphere the pair tree of two such meshes has
// one level and a fifth of its node pairs fewer.
//
// A node's state follows from its parent's through a 3-entry table that
// depends only on the leaf counts around it (k_state_tables).  k_wide_flags
// composes the tables up the parent chain until the composition no longer
// depends on the state above (about five steps a node), so no top-down pass
// over the levels is needed.
constexpr unsigned kStW = 0u, kStO2 = 1u, kStO3 = 2u;
constexpr unsigned kErrBuild = 4u;  // error word bit: an inconsistent wide tree (not expected)

// position (0..2) of the first maximum of three counts
__device__ __forceinline__ unsigned first_max3(uint32_t a, uint32_t b, uint32_t c)
{
    unsigned k = 0;
    uint32_t m = a;
    if (b > m) {
        m = b;
        k = 1;
    }
    if (c > m) k = 2;
    return k;
}

// tab[y] bits 2s..2s+1: the state of internal node y (y >= 1) when its parent
// is in state s (s = W, O2; a child of an O3 node is always W).
__global__ void k_state_tables(int n, const uint4* __restrict__ child, const int* __restrict__ parent,
                               uint8_t* __restrict__ tab)
{
    pdl_enter();
    int y = blockIdx.x * blockDim.x + threadIdx.x;
    if (y < 1 || y >= n - 1) return;
    const int p = parent[y];
    const uint4 c = child[p];
    const bool left = c.x == (uint32_t)y;
    const uint32_t z = left ? c.y : c.x;
    const uint32_t ny = left ? c.z : c.w, nz = left ? c.w : c.z;
    // parent in W: step 2 opens the larger child (tie: the left one)
    unsigned sW;
    if (left ? ny >= nz : ny > nz) {
        sW = kStO2;
    } else {  // the sibling z (internal: nz > ny >= 2) was opened; step 3 over the three parts
        const uint4 g = child[z];
        const uint32_t n0 = g.z, n1 = g.w;
        sW = (left ? first_max3(ny, n0, n1) == 0u : first_max3(n0, n1, ny) == 2u) ? kStO3 : kStW;
    }
    // parent in O2 (opened by its own parent r): step 3 over p's children and p's sibling
    unsigned sO2 = kStW;
    const int r = parent[p];
    if (r >= 0) {
        const uint4 cr = child[r];
        const bool pleft = cr.x == (uint32_t)p;
        const uint32_t ns = pleft ? cr.w : cr.z;
        const uint32_t n0 = c.z, n1 = c.w;
        const unsigned mine = pleft ? (left ? 0u : 1u) : (left ? 1u : 2u);
        const unsigned k = pleft ? first_max3(n0, n1, ns) : first_max3(ns, n0, n1);
        sO2 = k == mine ? kStO3 : kStW;
    }
    tab[y] = (uint8_t)(sW | (sO2 << 2) | (kStW << 4));
}

// wide[i] = 1 iff binary node i becomes a wide node.
__global__ void k_wide_flags(int n, const int* __restrict__ parent, const uint8_t* __restrict__ tab,
                             uint32_t* __restrict__ wide)
{
    pdl_enter();
    int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= n - 1) return;
    if (i == 0) {
        wide[0] = 1u;
        return;
    }
    unsigned f = tab[i];  // state of i as a function of the state of the node above the chain
    int x = parent[i];
    for (int guard = 0; x > 0 && guard < n; guard++) {
        const unsigned f0 = f & 3u, f1 = (f >> 2) & 3u, f2 = (f >> 4) & 3u;
        if (f0 == f1 && f1 == f2) break;
        const unsigned t = __ldg(tab + x);
        f = ((f >> (2u * (t & 3u))) & 3u) | (((f >> (2u * ((t >> 2) & 3u))) & 3u) << 2) |
            (((f >> (2u * ((t >> 4) & 3u))) & 3u) << 4);
        x = parent[x];
    }
    wide[i] = (f & 3u) == kStW ? 1u : 0u;  // the root is a wide node
}

// Writes wide node widx[i] from binary node i: the size-greedy expansion of i
// (the same choices as k_state_tables), with the boxes of its leaf children
// (consecutive leaves: the loads of neighbouring threads share lines); the
// boxes of wide children are filled by k_refit_wide.  For each wide child it
// writes the (wide node, slot) it sits in (nodeUp; the root's is kEmpty),
// and per node kids | leaf kids << 8 (nkids) and the arrival count so far,
// its leaf kids (arrive).  An internal part that is not a wide node, or whose
// index is out of range, cannot arise; it is written as an empty slot and
// flagged in *bad rather than followed.
template <class S, class NodeT>
__global__ void k_collapse(int n, const uint4* __restrict__ child, const uint32_t* __restrict__ wide,
                           const uint32_t* __restrict__ widx, uint32_t nw, const S* __restrict__ leafBox,
                           NodeT* __restrict__ nodes, uint2* __restrict__ nodeUp, uint32_t* __restrict__ nkids,
                           unsigned* __restrict__ arrive, unsigned* __restrict__ bad)
{
    pdl_enter();
    int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= n - 1 || !wide[i]) return;
    const uint32_t wi = widx[i];
    if (wi >= nw) {
        atomicOr(bad, kErrBuild);
        return;
    }
    if (wi == 0u) nodeUp[0] = make_uint2(kEmpty, 0u);
    const uint4 c = child[i];
    uint32_t slot[4] = {c.x, c.y, kEmpty, kEmpty};
    uint32_t num[4] = {c.z, c.w, 0u, 0u};
    int ns = 2;
#pragma unroll
    for (int step = 0; step < 2; step++) {
        int b = 0;
        for (int k = 1; k < ns; k++)
            if (num[k] > num[b]) b = k;
        if (num[b] < 2u) break;
        const uint4 g = child[slot[b]];
        for (int k = ns; k > b + 1; k--) {
            slot[k] = slot[k - 1];
            num[k] = num[k - 1];
        }
        slot[b] = g.x;
        slot[b + 1] = g.y;
        num[b] = g.z;
        num[b + 1] = g.w;
        ns++;
    }
    NodeT out;
    uint32_t kids = 0, leaves = 0;
    for (int k = 0; k < 4; k++) {
        uint32_t r = k < ns ? slot[k] : kEmpty;
        if (r != kEmpty && !(r & kLeaf) && (!wide[r] || widx[r] >= nw)) {
            atomicOr(bad, kErrBuild);
            r = kEmpty;
        }
        S bx[6] = {(S)INFINITY, (S)INFINITY, (S)INFINITY, (S)-INFINITY, (S)-INFINITY, (S)-INFINITY};
        if (r == kEmpty) {
            out.child[k] = kEmpty;
        } else if (r & kLeaf) {
            load_box_cg(leafBox + 6 * (size_t)(r & ~kLeaf), bx);
            out.child[k] = r;
            kids++;
            leaves++;
        } else {
            const uint32_t cw = widx[r];
            out.child[k] = cw;
            nodeUp[cw] = make_uint2(wi, (uint32_t)k);
            kids++;
        }
        out.lox[k] = bx[0];
        out.loy[k] = bx[1];
        out.loz[k] = bx[2];
        out.hix[k] = bx[3];
        out.hiy[k] = bx[4];
        out.hiz[k] = bx[5];
    }
    for (int k = 0; k < (int)(sizeof(out.pad) / sizeof(out.pad[0])); k++) out.pad[k] = 0;
    nkids[wi] = kids | (leaves << 8);
    arrive[wi] = leaves;
    nodes[wi] = out;
}

// The six child-box fields of a wide node, read through L2 (other threads of
// the same launch wrote them): the union of its slots (empty slots hold
// +inf / -inf and change nothing).
__device__ __forceinline__ void node_union_cg(const WNode* nd, float b[6])
{
    const float4* q = reinterpret_cast<const float4*>(nd);
#pragma unroll
    for (int f = 0; f < 6; f++) {
        const float4 v = __ldcg(q + f);
        b[f] = f < 3 ? fminf(fminf(v.x, v.y), fminf(v.z, v.w)) : fmaxf(fmaxf(v.x, v.y), fmaxf(v.z, v.w));
    }
}
__device__ __forceinline__ void node_union_cg(const WNode64* nd, double b[6])
{
    const double2* q = reinterpret_cast<const double2*>(nd);
#pragma unroll
    for (int f = 0; f < 6; f++) {
        const double2 v = __ldcg(q + 2 * f), w = __ldcg(q + 2 * f + 1);
        b[f] = f < 3 ? fmin(fmin(v.x, v.y), fmin(w.x, w.y)) : fmax(fmax(v.x, v.y), fmax(w.x, w.y));
    }
}

// Bottom-up refit of the wide tree, one thread per wide node.  A node whose
// children are all leaves is complete after k_collapse: its thread takes the
// union of its slots, stores it into its slot of the node above and arrives
// there; the thread that arrives last (after the node's other children) takes
// that node's union and climbs on.  Nodes with a wide child return at once.
// The links of the node above are loaded while the arrival is in flight, so a
// level costs the slot stores, the arrival atomic and one read of the node's
// six box fields; the wide tree has about half the levels of the binary one.
template <class S, class NodeT>
__global__ void k_refit_wide(uint32_t nw, const uint2* __restrict__ nodeUp, const uint32_t* __restrict__ nkids,
                             NodeT* nodes, unsigned* arrive, unsigned* bad)
{
    pdl_enter();
    const uint32_t w0 = blockIdx.x * blockDim.x + threadIdx.x;
    if (w0 >= nw) return;
    const uint32_t k0 = nkids[w0];
    if ((k0 & 0xffu) != (k0 >> 8)) return;  // a wide child completes this node
    S b[6];
    node_union_cg(nodes + w0, b);
    uint2 up = nodeUp[w0];
    for (uint32_t guard = 0; guard < nw; guard++) {
        if (up.x == kEmpty) return;  // the root is complete
        const uint32_t w = up.x, k = up.y & 3u;
        if (w >= nw) {
            atomicOr(bad, kErrBuild);
            return;
        }
        NodeT* nd = nodes + w;
        nd->lox[k] = b[0];
        nd->loy[k] = b[1];
        nd->loz[k] = b[2];
        nd->hix[k] = b[3];
        nd->hiy[k] = b[4];
        nd->hiz[k] = b[5];
        const uint2 upn = nodeUp[w];
        const uint32_t need = nkids[w] & 0xffu;
        // release: this slot's stores before the arrival; acquire: the other slots' after it
        if (arrive_acq_rel(&arrive[w]) + 1u != need) return;
        node_union_cg(nd, b);
        up = upn;
    }
}

// Cuts of the wide BVH: the root expanded three and four times (leaves met on
// the way are kept), each entry's box from its parent's child slot.  One block
// expands a level at a time, an entry per thread, the children placed by a
// block scan, so entries keep the order of a sequential expansion.  Output:
// the depth-3 cut (at most 4^3 entries) at [0, kCutMax), the depth-4 cut (at
// most 4^4) at [kCutMax, kCutCap); ncut[0], ncut[1] their sizes.  The
// traversal starts from all pairs of two meshes' cuts.
constexpr int kCutThreads = kCut4Max;
template <class S, class NodeT>
__global__ void __launch_bounds__(kCutThreads) k_cut(const NodeT* __restrict__ nodes, const S* __restrict__ leafBox,
                                                     uint32_t root, uint32_t* __restrict__ cutRef,
                                                     S* __restrict__ cutBox, uint32_t* __restrict__ ncut)
{
    pdl_enter();
    __shared__ uint32_t r[2][kCut4Max];
    __shared__ S b[2][kCut4Max][6];
    __shared__ uint32_t sw[33];
    const unsigned tid = threadIdx.x;
    if (root & kLeaf) {
        if (tid == 0) {
            for (int c = 0; c < 2; c++) {
                const unsigned o = c ? kCutMax : 0u;
                cutRef[o] = root;
                for (int k = 0; k < 6; k++) cutBox[6 * o + k] = leafBox[6 * (size_t)(root & ~kLeaf) + k];
            }
            ncut[0] = ncut[1] = 1u;
        }
        return;
    }
    if (tid == 0) r[0][0] = root;  // the root's own box is never used: it is expanded first
    __syncthreads();
    unsigned n = 1, cur = 0;
    for (int depth = 1; depth <= 4; depth++) {
        // n <= 4^(depth-1) <= kCutThreads: one entry per thread
        const uint32_t ref = tid < n ? r[cur][tid] : kLeaf;
        const bool node = tid < n && !(ref & kLeaf);
        unsigned cnt = 0;
        if (tid < n) {
            if (!node) cnt = 1;
            else
                for (int c = 0; c < 4; c++) cnt += nodes[ref].child[c] != kEmpty;
        }
        unsigned tot;
        const unsigned ex = block_exclusive_scan(cnt, sw, &tot);
        const unsigned nx = cur ^ 1u;
        if (tid < n) {
            if (!node) {
                r[nx][ex] = ref;
                for (int k = 0; k < 6; k++) b[nx][ex][k] = b[cur][tid][k];
            } else {
                const NodeT& nd = nodes[ref];
                unsigned m = ex;
                for (int c = 0; c < 4; c++) {
                    if (nd.child[c] == kEmpty) continue;
                    r[nx][m] = nd.child[c];
                    b[nx][m][0] = nd.lox[c];
                    b[nx][m][1] = nd.loy[c];
                    b[nx][m][2] = nd.loz[c];
                    b[nx][m][3] = nd.hix[c];
                    b[nx][m][4] = nd.hiy[c];
                    b[nx][m][5] = nd.hiz[c];
                    m++;
                }
            }
        }
        __syncthreads();
        n = tot;
        cur = nx;
        if (depth >= 3) {
            const unsigned o = depth == 3 ? 0u : (unsigned)kCutMax;
            for (unsigned e = tid; e < n; e += kCutThreads) {
                cutRef[o + e] = r[cur][e];
                for (int k = 0; k < 6; k++) cutBox[6 * (o + e) + k] = b[cur][e][k];
            }
            if (tid == 0) ncut[depth - 3] = n;
        }
    }
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

cudaError_t build_bvh(MeshBuffers& m, bool fp64, unsigned* d_err, cudaMemPool_t pool, cudaStream_t st)
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
    uint4* child = nullptr;
    int* parent = nullptr;
    unsigned* arrive = nullptr;
    uint2* nodeUp = nullptr;
    uint32_t* nkids = nullptr;
    uint32_t *wide = nullptr, *widx = nullptr;
    uint8_t* tab = nullptr;
    constexpr int kMortonDigit = 10;  // 30-bit keys: three passes
    size_t cw = radix_counts_words<kMortonDigit>(n);
    size_t sw = scan_temp_words(cw > n ? cw : n);
    GI_TRY(pool_alloc(&box, sizeof(float) * 6 * n, pool, st));
    if (fp64) GI_TRY(pool_alloc(&box64, sizeof(double) * 6 * n, pool, st));
    GI_TRY(pool_alloc(&cb, sizeof(unsigned) * 8, pool, st));
    GI_TRY(pool_alloc(&k0, sizeof(uint32_t) * n, pool, st));
    GI_TRY(pool_alloc(&v0, sizeof(uint32_t) * n, pool, st));
    GI_TRY(pool_alloc(&k1, sizeof(uint32_t) * n, pool, st));
    GI_TRY(pool_alloc(&v1, sizeof(uint32_t) * n, pool, st));
    GI_TRY(pool_alloc(&counts, sizeof(uint32_t) * cw, pool, st));
    GI_TRY(pool_alloc(&stemp, sizeof(uint32_t) * sw, pool, st));
    unsigned cbinit[8] = {0xffffffffu, 0xffffffffu, 0xffffffffu, 0u, 0u, 0u, 0u, 0u};
    GI_TRY(cudaMemcpyAsync(cb, cbinit, sizeof(cbinit), cudaMemcpyHostToDevice, st));
    int tb = 256;
    int gb = (int)((n + tb - 1) / tb);
    // Kernels that follow another kernel in the stream are launched as its
    // programmatic dependents (launch_dep): each waits for its predecessor at
    // its first statement, so only the next launch's latency overlaps the tail
    // of the current kernel (0.474 -> 0.446 ms per 1.3M-triangle build on
    // B200).  The two kernels that follow a copy (k_tri_boxes after the bounds'
    // initial values, k_collapse after the wide-node count) are plain launches.
    // four resident blocks per SM, each looping: the centroid bounds take one set of atomics per block
    const int gboxes = (int)((n + 2 * kTriBoxThreads - 1) / (2 * kTriBoxThreads));
    k_tri_boxes<<<gboxes < 592 ? gboxes : 592, kTriBoxThreads, 0, st>>>(m.verts, m.nv, m.tris, n, box, box64, cb);
    const uint32_t ntiles = (n + kRsTile - 1) / kRsTile;
    launch_dep(k_morton_hist<kMortonDigit>, ntiles, kRsThreads, st, (const float*)box, n, (const unsigned*)cb, k0, v0,
               counts, ntiles);
    radix_sort<uint32_t, kMortonDigit>(k0, v0, k1, v1, n, 30, counts, stemp, st, true);
    if (n > 1) {
        GI_TRY(pool_alloc(&child, sizeof(uint4) * (n - 1), pool, st));
        GI_TRY(pool_alloc(&parent, sizeof(int) * (n - 1), pool, st));
    }
    // leaves in sorted order, and the binary radix tree
    if (!fp64) {
        GI_TRY(pool_alloc(&m.leafBox, sizeof(float) * 6 * n, pool, st));
        GI_TRY(pool_alloc(&m.leafTri, sizeof(uint4) * n, pool, st));
        launch_dep(k_karras_leaves<float>, gb, tb, st, (const uint32_t*)k0, (const uint32_t*)v0, (int)n,
                   (const uint32_t*)m.tris, (const float*)box, m.leafBox, m.leafTri, child, parent);
    } else {
        GI_TRY(pool_alloc(&m.leafBox64, sizeof(double) * 6 * n, pool, st));
        launch_dep(k_karras_leaves<double>, gb, tb, st, (const uint32_t*)k0, (const uint32_t*)v0, (int)n,
                   (const uint32_t*)m.tris, (const double*)box64, m.leafBox64, (uint4*)nullptr, child, parent);
    }
    if (n == 1) {
        m.root = kLeaf | 0u;
        m.nnodes = 0;
    } else {
        GI_TRY(pool_alloc(&wide, sizeof(uint32_t) * (n - 1), pool, st));
        GI_TRY(pool_alloc(&tab, sizeof(uint8_t) * (n - 1), pool, st));
        GI_TRY(pool_alloc(&widx, sizeof(uint32_t) * (n - 1), pool, st));
        int gi_ = (int)((n - 1 + tb - 1) / tb);
        launch_dep(k_state_tables, gi_, tb, st, (int)n, (const uint4*)child, (const int*)parent, tab);
        launch_dep(k_wide_flags, gi_, tb, st, (int)n, (const int*)parent, (const uint8_t*)tab, wide);
        scan_exclusive(wide, widx, n - 1, stemp, st);
        // number of wide nodes = widx[n-2] + wide[n-2]
        uint32_t last[2];
        GI_TRY(cudaMemcpyAsync(&last[0], widx + (n - 2), sizeof(uint32_t), cudaMemcpyDeviceToHost, st));
        GI_TRY(cudaMemcpyAsync(&last[1], wide + (n - 2), sizeof(uint32_t), cudaMemcpyDeviceToHost, st));
        GI_TRY(cudaStreamSynchronize(st));
        uint32_t nw = last[0] + last[1];
        GI_TRY(pool_alloc(&nodeUp, sizeof(uint2) * (size_t)nw, pool, st));
        GI_TRY(pool_alloc(&nkids, sizeof(uint32_t) * (size_t)nw, pool, st));
        GI_TRY(pool_alloc(&arrive, sizeof(unsigned) * (size_t)nw, pool, st));
        const int gw = (int)((nw + tb - 1) / tb);
        if (!fp64) {
            GI_TRY(pool_alloc(&m.nodes, sizeof(WNode) * (size_t)nw, pool, st));
            k_collapse<float, WNode><<<gi_, tb, 0, st>>>((int)n, child, wide, widx, nw, m.leafBox, m.nodes,
                                                         nodeUp, nkids, arrive, d_err);
            launch_dep(k_refit_wide<float, WNode>, gw, tb, st, nw, (const uint2*)nodeUp, (const uint32_t*)nkids, m.nodes,
                       arrive, d_err);
        } else {
            GI_TRY(pool_alloc(&m.nodes64, sizeof(WNode64) * (size_t)nw, pool, st));
            k_collapse<double, WNode64><<<gi_, tb, 0, st>>>((int)n, child, wide, widx, nw, m.leafBox64,
                                                            m.nodes64, nodeUp, nkids, arrive, d_err);
            launch_dep(k_refit_wide<double, WNode64>, gw, tb, st, nw, (const uint2*)nodeUp, (const uint32_t*)nkids,
                       m.nodes64, arrive, d_err);
        }
        m.nnodes = nw;
        m.root = 0;
    }
    // depth-3 and depth-4 cuts (refs and sizes shared by both precisions; boxes per
    // precision); the sizes stay on the device, where the seeding reads them
    {
        if (!m.ncuts) GI_TRY(pool_alloc(&m.ncuts, sizeof(uint32_t) * 2, pool, st));
        uint32_t* d_n = m.ncuts;
        if (!m.cutRef) GI_TRY(pool_alloc(&m.cutRef, sizeof(uint32_t) * kCutCap, pool, st));
        if (!fp64) {
            GI_TRY(pool_alloc(&m.cutBox, sizeof(float) * 6 * kCutCap, pool, st));
            launch_dep(k_cut<float, WNode>, 1, kCutThreads, st, (const WNode*)m.nodes, (const float*)m.leafBox, m.root,
                       m.cutRef, m.cutBox, d_n);
        } else {
            GI_TRY(pool_alloc(&m.cutBox64, sizeof(double) * 6 * kCutCap, pool, st));
            launch_dep(k_cut<double, WNode64>, 1, kCutThreads, st, (const WNode64*)m.nodes64,
                       (const double*)m.leafBox64, m.root, m.cutRef, m.cutBox64, d_n);
        }
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
    if (arrive) cudaFreeAsync(arrive, st);
    if (nodeUp) cudaFreeAsync(nodeUp, st);
    if (nkids) cudaFreeAsync(nkids, st);
    if (wide) cudaFreeAsync(wide, st);
    if (tab) cudaFreeAsync(tab, st);
    if (widx) cudaFreeAsync(widx, st);
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

// World box -> conservative box in the local frame of pose P (inverse map
// local = Ri*w + bi, Ri = R^T).  Same construction and bound as world_box; the
// pad also covers the error of R^T as the inverse (inv_eta <= 2^-30) and the
// FP64 rounding of the posed vertices.
__device__ __forceinline__ void local_box(const DevPose& P, Box<float>& b)
{
    float c[3], h[3];
    for (int k = 0; k < 3; k++) {
        c[k] = 0.5f * b.lo[k] + 0.5f * b.hi[k];
        h[k] = 0.5f * b.hi[k] - 0.5f * b.lo[k];
    }
    for (int r = 0; r < 3; r++) {
        float wc = P.bif[r], wh = 0.0f, mag = P.padmi[r];
        for (int k = 0; k < 3; k++) {
            float a = P.Rif[3 * r + k];
            wc = fmaf(a, c[k], wc);
            wh = fmaf(fabsf(a), h[k], wh);
            mag = fmaf(fabsf(a), fabsf(c[k]) + h[k], mag);
        }
        float pad = fmaf(0x1p-19f, mag, 0x1p-120f);
        b.lo[r] = wc - wh - pad;
        b.hi[r] = wc + wh + pad;
    }
}
__device__ __forceinline__ void local_box(const DevPose& P, Box<double>& b)
{
    double c[3], h[3];
    for (int k = 0; k < 3; k++) {
        c[k] = 0.5 * b.lo[k] + 0.5 * b.hi[k];
        h[k] = 0.5 * b.hi[k] - 0.5 * b.lo[k];
    }
    const double rel = 0x1p-48 + P.inv_eta;
    for (int r = 0; r < 3; r++) {
        double wc = P.bi64[r], wh = 0.0, mag = P.padmi64[r];
        for (int k = 0; k < 3; k++) {
            double a = P.Ri64[3 * r + k];
            wc = fma(a, c[k], wc);
            wh = fma(fabs(a), h[k], wh);
            mag = fma(fabs(a), fabs(c[k]) + h[k], mag);
        }
        double pad = fma(rel, mag, 0x1p-300);
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

// Children of a node reference in the mesh-local frame, structure of arrays
// (slot i of every array is child i).  A wide node gives up to four (one
// 128-byte line loaded as seven 16-byte vectors, or two lines for FP64); a
// leaf reference stands for itself in slot 0.  Every array is indexed by
// constants only, so the whole set lives in registers.
template <class S>
struct Kids {
    S lx[4], ly[4], lz[4], hx[4], hy[4], hz[4];
    uint32_t c[4];
};

__device__ __forceinline__ void put4(float (&d)[4], const float4& v)
{
    d[0] = v.x;
    d[1] = v.y;
    d[2] = v.z;
    d[3] = v.w;
}
__device__ __forceinline__ void put4(double (&d)[4], const double2& a, const double2& b)
{
    d[0] = a.x;
    d[1] = a.y;
    d[2] = b.x;
    d[3] = b.y;
}

__device__ __forceinline__ void load_kids(const MeshDev& M, uint32_t ref, Kids<float>& k)
{
    if (ref & kLeaf) {
        const float2* lb = reinterpret_cast<const float2*>(M.leafBox + 6 * (size_t)(ref & ~kLeaf));
        const float2 a = __ldg(lb), b = __ldg(lb + 1), c = __ldg(lb + 2);
        put4(k.lx, make_float4(a.x, 0.f, 0.f, 0.f));
        put4(k.ly, make_float4(a.y, 0.f, 0.f, 0.f));
        put4(k.lz, make_float4(b.x, 0.f, 0.f, 0.f));
        put4(k.hx, make_float4(b.y, 0.f, 0.f, 0.f));
        put4(k.hy, make_float4(c.x, 0.f, 0.f, 0.f));
        put4(k.hz, make_float4(c.y, 0.f, 0.f, 0.f));
        k.c[0] = ref;
        k.c[1] = k.c[2] = k.c[3] = kEmpty;
        return;
    }
    const float4* p = reinterpret_cast<const float4*>(M.nodes + ref);
    put4(k.lx, __ldg(p));
    put4(k.ly, __ldg(p + 1));
    put4(k.lz, __ldg(p + 2));
    put4(k.hx, __ldg(p + 3));
    put4(k.hy, __ldg(p + 4));
    put4(k.hz, __ldg(p + 5));
    const uint4 ch = __ldg(reinterpret_cast<const uint4*>(p + 6));
    k.c[0] = ch.x;
    k.c[1] = ch.y;
    k.c[2] = ch.z;
    k.c[3] = ch.w;
}
__device__ __forceinline__ void load_kids(const MeshDev& M, uint32_t ref, Kids<double>& k)
{
    if (ref & kLeaf) {
        const double2* lb = reinterpret_cast<const double2*>(M.leafBox64 + 6 * (size_t)(ref & ~kLeaf));
        const double2 a = __ldg(lb), b = __ldg(lb + 1), c = __ldg(lb + 2);
        const double2 z = make_double2(0.0, 0.0);
        put4(k.lx, make_double2(a.x, 0.0), z);
        put4(k.ly, make_double2(a.y, 0.0), z);
        put4(k.lz, make_double2(b.x, 0.0), z);
        put4(k.hx, make_double2(b.y, 0.0), z);
        put4(k.hy, make_double2(c.x, 0.0), z);
        put4(k.hz, make_double2(c.y, 0.0), z);
        k.c[0] = ref;
        k.c[1] = k.c[2] = k.c[3] = kEmpty;
        return;
    }
    const double2* p = reinterpret_cast<const double2*>(M.nodes64 + ref);
    put4(k.lx, __ldg(p), __ldg(p + 1));
    put4(k.ly, __ldg(p + 2), __ldg(p + 3));
    put4(k.lz, __ldg(p + 4), __ldg(p + 5));
    put4(k.hx, __ldg(p + 6), __ldg(p + 7));
    put4(k.hy, __ldg(p + 8), __ldg(p + 9));
    put4(k.hz, __ldg(p + 10), __ldg(p + 11));
    const uint4 ch = __ldg(reinterpret_cast<const uint4*>(p + 12));
    k.c[0] = ch.x;
    k.c[1] = ch.y;
    k.c[2] = ch.z;
    k.c[3] = ch.w;
}

// Maps the four child boxes to the world frame (same bound as world_box).
template <class S>
__device__ __forceinline__ void world_kids(const DevPose& P, Kids<S>& k)
{
#pragma unroll
    for (int i = 0; i < 4; i++) {
        Box<S> b;
        b.lo[0] = k.lx[i];
        b.lo[1] = k.ly[i];
        b.lo[2] = k.lz[i];
        b.hi[0] = k.hx[i];
        b.hi[1] = k.hy[i];
        b.hi[2] = k.hz[i];
        world_box(P, b);
        k.lx[i] = b.lo[0];
        k.ly[i] = b.lo[1];
        k.lz[i] = b.lo[2];
        k.hx[i] = b.hi[0];
        k.hy[i] = b.hi[1];
        k.hz[i] = b.hi[2];
    }
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

// Maps the four child boxes (world frame) into the local frame of pose P.
template <class S>
__device__ __forceinline__ void local_kids(const DevPose& P, Kids<S>& k)
{
#pragma unroll
    for (int i = 0; i < 4; i++) {
        Box<S> b;
        b.lo[0] = k.lx[i];
        b.lo[1] = k.ly[i];
        b.lo[2] = k.lz[i];
        b.hi[0] = k.hx[i];
        b.hi[1] = k.hy[i];
        b.hi[2] = k.hz[i];
        local_box(P, b);
        k.lx[i] = b.lo[0];
        k.ly[i] = b.lo[1];
        k.lz[i] = b.lo[2];
        k.hx[i] = b.hi[0];
        k.hy[i] = b.hi[1];
        k.hz[i] = b.hi[2];
    }
}

// 16-bit mask of the overlapping child pairs (bit 4i+j: a's child i, b's child j).
template <class S>
__device__ __forceinline__ unsigned overlap_mask(const Kids<S>& a, const Kids<S>& b)
{
    unsigned m = 0;
#pragma unroll
    for (int i = 0; i < 4; i++)
#pragma unroll
        for (int j = 0; j < 4; j++) {
            const bool ov = (a.lx[i] <= b.hx[j]) & (b.lx[j] <= a.hx[i]) & (a.ly[i] <= b.hy[j]) &
                            (b.ly[j] <= a.hy[i]) & (a.lz[i] <= b.hz[j]) & (b.lz[j] <= a.hz[i]);
            m |= (ov ? 1u : 0u) << (4 * i + j);
        }
    return m;
}

// Bit i of `x` (i < 4) spread over nibble i: the child pairs (i, *).
__device__ __forceinline__ unsigned rows4(unsigned x)
{
    return ((x & 1u) ? 0x000Fu : 0u) | ((x & 2u) ? 0x00F0u : 0u) | ((x & 4u) ? 0x0F00u : 0u) |
           ((x & 8u) ? 0xF000u : 0u);
}


// One node pair: load both nodes, map the child boxes to the world frame and
// test the 4 x 4 child pairs without branches.  fm / cm: bit 4i+j set when
// child pair (i, j) overlaps and leads to a node pair / a leaf pair.
template <bool F64>
__device__ __forceinline__ void expand_pair(const Bufs& B, const uint4& ent, unsigned& fm, unsigned& cm,
                                            uint32_t (&ca)[4], uint32_t (&cb)[4])
{
    using S = typename Prec<F64>::S;
    const JobDev& J = B.jobs[ent.x];
    Kids<S> a, b;
    load_kids(J.A, ent.y, a);
    load_kids(J.B, ent.z, b);
    if (!J.pa.identity) world_kids(J.pa, a);
    // a posed B can also be tested in its own frame (A's world boxes mapped
    // back through B's pose against B's stored boxes): the world box of a
    // rotated box is wider than the box, and each test alone is conservative.
    // It removes about a quarter of the pairs for about a third more work per
    // pair, which pays where the traversal is bound by work (batches), not by
    // the latency of its levels (one pair).
    unsigned m = 0xFFFFu;
    if (B.two_frame && J.pb.inv_ok) {
        Kids<S> al = a;
        local_kids(J.pb, al);
        m = overlap_mask(al, b);
    }
    if (!J.pb.identity) world_kids(J.pb, b);
    m &= overlap_mask(a, b);
    unsigned va = 0, vb = 0, la = 0, lb = 0;
#pragma unroll
    for (int i = 0; i < 4; i++) {
        ca[i] = a.c[i];
        cb[i] = b.c[i];
        va |= (a.c[i] != kEmpty ? 1u : 0u) << i;
        vb |= (b.c[i] != kEmpty ? 1u : 0u) << i;
        la |= ((a.c[i] & kLeaf) && a.c[i] != kEmpty ? 1u : 0u) << i;
        lb |= ((b.c[i] & kLeaf) && b.c[i] != kEmpty ? 1u : 0u) << i;
    }
    m &= rows4(va) & (vb * 0x1111u);
    const unsigned leafpair = rows4(la) & (lb * 0x1111u);
    cm = m & leafpair;
    fm = m & ~leafpair;
}

// ---------------------------------------------------------------------------
// Quad-cooperative expansion: the four lanes of a quad share one node pair and
// lane k (= lane & 3) owns child k of both nodes.  Each lane loads one child
// slot of each node (the four lanes of a quad read one 16-byte segment per
// field of the structure-of-arrays node), maps its own boxes to the world
// frame, receives B's four child boxes from its quad by width-4 shuffles and
// tests its A child against them: four tests instead of sixteen, one box
// transform instead of four, so the dependent chain of one expansion is a
// fraction of the one-lane form's.
// ---------------------------------------------------------------------------
__device__ __forceinline__ void load_kid(const MeshDev& M, uint32_t ref, unsigned k, Box<float>& b, uint32_t& c)
{
    if (ref & kLeaf) {
        if (k == 0u) {
            const float* lb = M.leafBox + 6 * (size_t)(ref & ~kLeaf);
            for (int q = 0; q < 3; q++) {
                b.lo[q] = __ldg(lb + q);
                b.hi[q] = __ldg(lb + 3 + q);
            }
            c = ref;
        } else {
            for (int q = 0; q < 3; q++) b.lo[q] = b.hi[q] = 0.0f;
            c = kEmpty;
        }
        return;
    }
    const float* p = reinterpret_cast<const float*>(M.nodes + ref);
    for (int q = 0; q < 3; q++) {
        b.lo[q] = __ldg(p + 4 * q + k);
        b.hi[q] = __ldg(p + 12 + 4 * q + k);
    }
    c = __ldg(reinterpret_cast<const uint32_t*>(p + 24) + k);
}
__device__ __forceinline__ void load_kid(const MeshDev& M, uint32_t ref, unsigned k, Box<double>& b, uint32_t& c)
{
    if (ref & kLeaf) {
        if (k == 0u) {
            const double* lb = M.leafBox64 + 6 * (size_t)(ref & ~kLeaf);
            for (int q = 0; q < 3; q++) {
                b.lo[q] = __ldg(lb + q);
                b.hi[q] = __ldg(lb + 3 + q);
            }
            c = ref;
        } else {
            for (int q = 0; q < 3; q++) b.lo[q] = b.hi[q] = 0.0;
            c = kEmpty;
        }
        return;
    }
    const double* p = reinterpret_cast<const double*>(M.nodes64 + ref);
    for (int q = 0; q < 3; q++) {
        b.lo[q] = __ldg(p + 4 * q + k);
        b.hi[q] = __ldg(p + 12 + 4 * q + k);
    }
    c = __ldg(reinterpret_cast<const uint32_t*>(p + 24) + k);
}

template <class S>
__device__ __forceinline__ void shfl_box(const Box<S>& src, Box<S>& dst, unsigned j)
{
#pragma unroll
    for (int q = 0; q < 3; q++) {
        dst.lo[q] = __shfl_sync(0xffffffffu, src.lo[q], (int)j, 4);
        dst.hi[q] = __shfl_sync(0xffffffffu, src.hi[q], (int)j, 4);
    }
}

// Called by all 32 lanes (the shuffles need them); lanes of a quad without a
// node pair pass have = false and get no children.  fm / cm: bit j set when
// (own A child, B child j) overlap and lead to a node pair / a leaf pair;
// cb[j] receives B's child refs.
template <bool F64>
__device__ __forceinline__ void expand_quad(const Bufs& B, const uint4& ent, bool have, unsigned sub, unsigned& fm,
                                            unsigned& cm, uint32_t& ca, uint32_t (&cb)[4])
{
    using S = typename Prec<F64>::S;
    const JobDev& J = B.jobs[have ? ent.x : 0u];
    Box<S> a, b;
    uint32_t mb = kEmpty;
    ca = kEmpty;
    for (int q = 0; q < 3; q++) a.lo[q] = a.hi[q] = b.lo[q] = b.hi[q] = S(0);
    if (have) {
        load_kid(J.A, ent.y, sub, a, ca);
        load_kid(J.B, ent.z, sub, b, mb);
        if (ca != kEmpty && !J.pa.identity) world_box(J.pa, a);
    }
    // optional second test in B's own frame (see expand_pair)
    unsigned m2 = 0xFu;
    if (B.two_frame) {  // uniform over the launch
        const bool twof = have && J.pb.inv_ok;
        Box<S> al = a;
        if (twof && ca != kEmpty) local_box(J.pb, al);
        m2 = 0u;
#pragma unroll
        for (int j = 0; j < 4; j++) {
            Box<S> bl;
            shfl_box(b, bl, (unsigned)j);
            if (!twof || overlap(al, bl)) m2 |= 1u << j;
        }
    }
    if (have && mb != kEmpty && !J.pb.identity) world_box(J.pb, b);
    fm = cm = 0u;
    const bool leafa = (ca & kLeaf) && ca != kEmpty;
#pragma unroll
    for (int j = 0; j < 4; j++) {
        Box<S> bj;
        shfl_box(b, bj, (unsigned)j);
        cb[j] = __shfl_sync(0xffffffffu, mb, j, 4);
        const bool ov = ca != kEmpty && cb[j] != kEmpty && ((m2 >> j) & 1u) && overlap(a, bj);
        const bool leafb = (cb[j] & kLeaf) != 0u;
        if (ov) {
            if (leafa && leafb) cm |= 1u << j;
            else fm |= 1u << j;
        }
    }
}

// ---------------------------------------------------------------------------
// Persistent BVH4 x BVH4 traversal: a small warp stack in front of a device
// work queue (no grid barrier).
//
// Each warp expands up to 32 node pairs per iteration (one per lane).  It
// keeps up to 32 of their children on its own shared-memory stack for its next
// iteration, with no global round trip, and publishes the rest to the global
// queue; leaf pairs (candidates) always go to the global candidate list, so
// the first filter stage runs on warps that have no node pair at hand.  The
// launch first seeds the queue: every overlapping pair of the two meshes'
// cut entries (depth 4 for a single pair, depth 3 for a batch) becomes a node
// pair (a leaf pair, a candidate).
//
// Slot protocol (queue and candidate list): producers reserve slots with one
// atomic per warp, write the entries and, after a release fence, store the
// call's tag in each slot's flag word.  A warp takes a ticket of 32
// consecutive slots (one atomicAdd on the head counter), polls their 32 tag
// words with acquire loads (one 128-byte line, so polling has no hot spot;
// a ready tag orders the entry's load after it) and keeps the ticket
// until all 32 slots are processed.  Only warps with empty stacks take node
// tickets, and ready queue slots come before stack entries, so queued work
// never waits behind a warp that is busy with its own.
//
// Termination: the low half of `work_cand` is the number of node pairs that
// exist, its high half the candidate slots reserved.  Seeds add to both
// before the seed count completes; an expansion adds (children - expanded
// pairs) and its candidates in one atomic, before any child is published, so
// the node-pair count never passes through zero while a node pair exists, and
// the load that reads it at zero reads the final candidate count.  Reading
// seed_done == all seed tests and then a zero node-pair count proves the
// traversal is over.  Every wait is bounded; overflow or a spent wait raises the abort
// flag.
// ---------------------------------------------------------------------------
constexpr unsigned kIdleSpins = 1u << 22;     // consecutive idle polls of one warp (~1 s)
constexpr unsigned kWarpStack = 32;           // stack capacity of a warp (both expansion forms)
constexpr int kTravThreads = 256;
constexpr int kTravWarps = kTravThreads / 32;

__device__ __forceinline__ unsigned ld_vol(const unsigned* p)
{
    return *(const volatile unsigned*)p;
}

// Release / acquire fence at GPU scope: orders entry stores before the tag
// stores that follow, and an observed tag before the entry loads that follow.
// acquire load: the loads after it see what the writer published before its
// release (fence + tag store), without waiting for this thread's own stores
__device__ __forceinline__ unsigned ld_acq(const unsigned* p)
{
    unsigned v;
    asm volatile("ld.acquire.gpu.global.u32 %0, [%1];" : "=r"(v) : "l"(p) : "memory");
    return v;
}

// Programmatic dependent launch: the launch that follows on the stream (the
// call's finish) may be scheduled now; it waits for this grid's completion and
// memory before it reads anything (wait_prior_grid).  Without such a launch
// both are no-ops.
__device__ __forceinline__ void allow_dependent_launch()
{
    asm volatile("griddepcontrol.launch_dependents;" ::: "memory");
}

__device__ __forceinline__ void wait_prior_grid()
{
    asm volatile("griddepcontrol.wait;" ::: "memory");
}

__device__ __forceinline__ void fence_acq_rel()
{
    asm volatile("fence.acq_rel.gpu;" ::: "memory");
}

__device__ __forceinline__ unsigned take_ticket(unsigned* head)
{
    unsigned b = 0;
    if ((threadIdx.x & 31) == 0) b = atomicAdd(head, 32u);
    return __shfl_sync(0xffffffffu, b, 0);
}

// Seed tests per job: every pair of the two meshes' cut entries.
__device__ __forceinline__ unsigned seed_tests_per_job(const Bufs& B)
{
    return B.deep_seed ? (unsigned)kCut4Max * kCut4Max : (unsigned)kCutMax * kCutMax;
}

// Seeds the queue: pair (i, j) of the depth-3 (or depth-4) cut entries of every job.  Warps
// claim chunks of 32 seed tests with one atomic, so only warps that run do the
// work (nothing waits for a block that never becomes resident); seed_done
// counts finished tests after their node pairs are counted in `work`.
template <bool F64>
__device__ __forceinline__ void seed_cut_pairs(const Bufs& B, unsigned total)
{
    using S = typename Prec<F64>::S;
    Counters* C = B.cnt;
    const unsigned lane = threadIdx.x & 31;
    const unsigned per_job = seed_tests_per_job(B);
    const unsigned coff = B.deep_seed ? (unsigned)kCutMax : 0u;  // the cut's first entry
    for (;;) {
        unsigned base = 0;
        if (lane == 0) base = atomicAdd(&C->seed_head, 32u);
        base = __shfl_sync(0xffffffffu, base, 0);
        if (base >= total) break;
        const unsigned g = base + lane;
        bool front = false, cand = false;
        uint32_t ra = 0, rb = 0, job = 0;
        if (g < total) {
            job = g / per_job;
            const unsigned t = g % per_job;
            const JobDev& J = B.jobs[job];
            const bool both = J.A.nt && J.B.nt;  // an empty mesh has no cut (null sizes)
            const unsigned nA = both ? __ldg(J.A.ncuts + (B.deep_seed ? 1 : 0)) : 0u;
            const unsigned nB = both ? __ldg(J.B.ncuts + (B.deep_seed ? 1 : 0)) : 0u;
            if (t < nA * nB) {
                const unsigned i = coff + t / nB, j = coff + t % nB;
                const S* ba_ = F64 ? (const S*)J.A.cutBox64 : (const S*)J.A.cutBox;
                const S* bb_ = F64 ? (const S*)J.B.cutBox64 : (const S*)J.B.cutBox;
                Box<S> ba, bb;
                for (int k = 0; k < 3; k++) {
                    ba.lo[k] = ba_[6 * i + k];
                    ba.hi[k] = ba_[6 * i + 3 + k];
                    bb.lo[k] = bb_[6 * j + k];
                    bb.hi[k] = bb_[6 * j + 3 + k];
                }
                if (!J.pa.identity) world_box(J.pa, ba);
                if (!J.pb.identity) world_box(J.pb, bb);
                if (overlap(ba, bb)) {
                    ra = J.A.cutRef[i];
                    rb = J.B.cutRef[j];
                    cand = (ra & kLeaf) && (rb & kLeaf);
                    front = !cand;
                }
            }
        }
        const unsigned nfront = __popc(__ballot_sync(0xffffffffu, front));
        unsigned pf = warp_append(front, &C->q_tail);
        if (front) {
            if (pf < B.cap_queue) B.queue[pf] = make_uint4(job, ra, rb, 0u);
            else {
                atomicOr(&C->overflow, kOvfFrontier);
                atomicExch(&C->abort_, 1u);
            }
        }
        // candidate slots and node pairs counted in one atomic, before any seed is published
        const unsigned cm = __ballot_sync(0xffffffffu, cand);
        unsigned long long old = 0;
        if (lane == 0 && (cm || nfront))
            old = atomicAdd(&C->work_cand, ((unsigned long long)__popc(cm) << 32) + nfront);
        const unsigned pc = (unsigned)(__shfl_sync(0xffffffffu, old, 0) >> 32) + __popc(cm & ((1u << lane) - 1u));
        if (cand) {
            if (pc < B.cap_cand) B.cand[pc] = make_uint4(job, ra & ~kLeaf, rb & ~kLeaf, 0u);
            else {
                atomicOr(&C->overflow, kOvfCand);
                atomicExch(&C->abort_, 1u);
            }
        }
        __syncwarp();
        fence_acq_rel();
        if (front && pf < B.cap_queue) *(volatile unsigned*)(B.qflag + pf) = B.tag;
        if (cand && pc < B.cap_cand) *(volatile unsigned*)(B.cflag + pc) = B.tag;
        __syncwarp();
        if (lane == 0) {
            fence_acq_rel();
            atomicAdd(&C->seed_done, min(32u, total - base));
        }
    }
}

// First filter stage on one candidate per lane (have = lane holds one):
// intersecting pairs go to the result list, undecided ones to the escalation
// list (one atomic per list per warp).
template <bool F64>
__device__ __forceinline__ void filter_candidates(const Bufs& B, bool have, const uint4& c,
                                                  unsigned long long& decided, unsigned long long& tested)
{
    Counters* C = B.cnt;
    int dec = DEC_NO;
    uint32_t ta = 0, tb = 0;
    unsigned pat = 0;
    if (have) {
        tested++;
        const JobDev& J = B.jobs[c.x];
        double3 P[3], Q[3];
        load_tri<F64>(J.A, J.pa, c.y, P, &ta);
        load_tri<F64>(J.B, J.pb, c.z, Q, &tb);
        if constexpr (F64) dec = classify_fast<double>(P, Q, &pat);
        else dec = classify_fast<float>(P, Q, &pat);
        decided += (dec != DEC_ESC);
    }
    const bool yes = have && dec == DEC_YES;
    const bool esc = have && dec == DEC_ESC;
    const unsigned pr = warp_append(yes, &C->res);
    if (yes) {
        if (pr < B.cap_res) B.res[pr] = make_uint4(c.x, ta, tb, pat);
        else atomicOr(&C->overflow, kOvfRes);
    }
    const unsigned pe = warp_append(esc, &C->esc);
    if (esc) {
        if (pe < B.cap_esc) B.esc[pe] = make_uint4(c.x, c.y, c.z, 0u);
        else atomicOr(&C->overflow, kOvfEsc);
    }
}

// A traversal block's counts at its end: summed over its warps in shared
// memory, then one atomic per counter for the block (every warp's own atomics
// on the same three words queued up at the end of the launch).  Every thread
// of the block must call it.
__device__ __forceinline__ void block_stats(Counters* C, unsigned long long visited, unsigned long long decided,
                                            unsigned long long tested, unsigned levels = 0u)
{
    __shared__ unsigned long long s_stats[4][kTravWarps];
    for (int o = 16; o > 0; o >>= 1) {
        visited += __shfl_xor_sync(0xffffffffu, visited, o);
        decided += __shfl_xor_sync(0xffffffffu, decided, o);
        tested += __shfl_xor_sync(0xffffffffu, tested, o);
        levels = max(levels, __shfl_xor_sync(0xffffffffu, levels, o));
    }
    const unsigned warp = threadIdx.x >> 5;
    if ((threadIdx.x & 31u) == 0u) {
        s_stats[0][warp] = visited;
        s_stats[1][warp] = decided;
        s_stats[2][warp] = tested;
        s_stats[3][warp] = levels;
    }
    __syncthreads();
    if (threadIdx.x < 4u) {
        unsigned long long t = 0;
#pragma unroll
        for (int w = 0; w < kTravWarps; w++)
            t = threadIdx.x == 3u ? max(t, s_stats[3][w]) : t + s_stats[threadIdx.x][w];
        if (threadIdx.x == 3u) {
            if (t) atomicMax(&C->levels, (unsigned)t);
        } else if (t) {
            atomicAdd(threadIdx.x == 0u ? &C->node_pairs : (threadIdx.x == 1u ? &C->filter_decided : &C->tested), t);
        }
    }
}

// QUAD selects the expansion form: one node pair per lane (32 per warp
// iteration, the form for work-bound launches) or one per quad (8 per
// iteration with a quarter of the dependent chain, the form for launches bound
// by the latency of the traversal's levels).  The host picks it per workload.
template <bool F64, bool QUAD>
__global__ void __launch_bounds__(kTravThreads, 2) k_traverse(Bufs B)
{
    constexpr unsigned kSlots = QUAD ? 8u : 32u;  // node-queue slots per ticket: one per work unit
    constexpr unsigned kStack = QUAD ? 8u : 32u;  // node pairs kept for the next iteration
    __shared__ uint4 stk[kTravWarps][kWarpStack];
    allow_dependent_launch();
    Counters* C = B.cnt;
    const unsigned lane = threadIdx.x & 31;
    uint4* S = stk[threadIdx.x >> 5];
    const unsigned seed_total = B.njobs * seed_tests_per_job(B);
    seed_cut_pairs<F64>(B, seed_total);
    unsigned long long visited = 0, decided = 0, tested = 0;
    unsigned maxlev = 0, idle = 0, backoff = 32;
    unsigned sn = 0;         // node pairs on this warp's stack (warp-uniform, <= kWarpStack)
    bool ticket = false;     // holds a node-queue ticket
    unsigned nbase = 0, npend = 0;
    unsigned cbase = take_ticket(&C->c_head);
    unsigned cpend = 0xffffffffu;  // lanes whose candidate slot is still to be processed
    unsigned iter = 0;
    for (;;) {
        ++iter;
        if (!ticket && sn == 0u) {
            unsigned b0 = 0;
            if (lane == 0) b0 = atomicAdd(&C->q_head, kSlots);
            nbase = __shfl_sync(0xffffffffu, b0, 0);
            npend = kSlots == 32u ? 0xffffffffu : (1u << kSlots) - 1u;
            ticket = true;
        }
        const unsigned unit = QUAD ? (lane >> 2) : lane;  // work unit: a quad or a lane
        const unsigned sub = QUAD ? (lane & 3u) : 0u;
        const unsigned ubit = QUAD ? 4u * unit : unit;     // the unit's first lane
        const unsigned ns = nbase + unit;  // one queue slot per unit
        const unsigned i = cbase + lane;   // one candidate slot per lane
        const bool nslot = ticket && ((npend >> unit) & 1u) && ns < B.cap_queue;
        const bool cslot = ((cpend >> lane) & 1u) && i < B.cap_cand;
        // everything this pass polls, issued together.  The abort flag is one
        // line that every warp reads, so it is read every 8th pass only; its
        // round trip overlaps the node loads of a warp that works from its stack.
        unsigned ab = 0;
        if (lane == 0 && (iter & 7u) == 0u) ab = ld_vol(&C->abort_);
        const unsigned ntag = nslot ? ld_acq(B.qflag + ns) : 0u;
        const unsigned ctag = cslot ? ld_acq(B.cflag + i) : 0u;
        const bool from_queue = nslot && ntag == B.tag;  // the same in every lane of a unit
        const unsigned qball = __ballot_sync(0xffffffffu, from_queue && sub == 0u);  // a unit's first lane: ready
        if (sn != 0u || qball != 0u) {
            idle = 0;
            backoff = 32;
            // ready queue slots first (queued work is what idle warps wait
            // for), the other units pop the stack
            const unsigned take = min(sn, kSlots - (unsigned)__popc(qball));
            const unsigned rank = unit - (unsigned)__popc(qball & ((1u << ubit) - 1u));
            const bool from_stack = !from_queue && rank < take;
            uint4 ent = make_uint4(0u, kEmpty, kEmpty, 0u);
            if (from_stack) {
                ent = S[sn - 1u - rank];
            } else if (from_queue) {
                ent = __ldcg(B.queue + ns);  // ordered after the tag's acquire load
            }
            sn -= take;
            __syncwarp();  // popped entries are read before the pushes below reuse their slots
            const bool have = from_stack || from_queue;
            if (have && sub == 0u) {
                visited++;
                maxlev = max(maxlev, ent.w);
            }
            unsigned fm = 0, cm = 0;
            uint32_t ca[4], cb[4];
            if constexpr (QUAD) {
                expand_quad<F64>(B, ent, have, sub, fm, cm, ca[0], cb);
            } else {
                if (have) expand_pair<F64>(B, ent, fm, cm, ca, cb);
            }
            // children: node pairs onto the stack (up to keep), the rest to the
            // queue; candidates to the global candidate list
            const unsigned nf = __popc(fm), nc = __popc(cm);
            unsigned incf = nf, incc = nc;
#pragma unroll
            for (int o = 1; o < 32; o <<= 1) {
                const unsigned yf = __shfl_up_sync(0xffffffffu, incf, o);
                const unsigned yc = __shfl_up_sync(0xffffffffu, incc, o);
                if (lane >= (unsigned)o) {
                    incf += yf;
                    incc += yc;
                }
            }
            const unsigned kf = __shfl_sync(0xffffffffu, incf, 31);
            const unsigned kc = __shfl_sync(0xffffffffu, incc, 31);
            const unsigned done = __popc(__ballot_sync(0xffffffffu, have && sub == 0u));
            const unsigned keep = min(kf, kStack - sn);
            unsigned qb = 0, cg = 0;
            if (lane == 31) {
                if (kf > keep) qb = atomicAdd(&C->q_tail, kf - keep);
                // candidate slots and node pairs made minus expanded in one
                // atomic, before any child is published: the node-pair count
                // reaches zero in the same update that reserves the last
                // expansion's candidate slots
                if (kc || kf != done) {
                    const unsigned long long old = atomicAdd(
                        &C->work_cand, ((unsigned long long)kc << 32) + (unsigned long long)(long long)(int)(kf - done));
                    cg = (unsigned)(old >> 32);
                }
            }
            qb = __shfl_sync(0xffffffffu, qb, 31);
            cg = __shfl_sync(0xffffffffu, cg, 31);
            const unsigned f0 = incf - nf;  // this lane's first node child in the warp's order
            const unsigned c0 = cg + incc - nc;  // this lane's first candidate slot
            {
                // child slot q: the pair (A child q / 4, B child q % 4) in the lane
                // form, (own A child, B child q) in the quad form; the unrolled
                // loop indexes the registers with constants and has no
                // data-dependent trip count
                constexpr int kQ = QUAD ? 4 : 16;
                unsigned g = f0, h = c0;
#pragma unroll
                for (int q = 0; q < kQ; q++) {
                    const uint32_t ra = QUAD ? ca[0] : ca[q >> 2], rb = QUAD ? cb[q] : cb[q & 3];
                    if ((fm >> q) & 1u) {
                        const uint4 e = make_uint4(ent.x, ra, rb, ent.w + 1u);
                        if (g < keep) {
                            S[sn + g] = e;
                        } else {
                            const unsigned sl = qb + (g - keep);
                            if (sl < B.cap_queue) B.queue[sl] = e;
                        }
                        g++;
                    }
                    if ((cm >> q) & 1u) {
                        if (h < B.cap_cand) B.cand[h] = make_uint4(ent.x, ra & ~kLeaf, rb & ~kLeaf, 0u);
                        h++;
                    }
                }
            }
            __syncwarp();  // the work count above precedes every tag store below
            const unsigned qx0 = max(f0, keep), qx1 = f0 + nf;
            if (qx0 < qx1 || nc != 0u) {
                fence_acq_rel();
                for (unsigned x = qx0; x < qx1; x++) {
                    const unsigned sl = qb + (x - keep);
                    if (sl < B.cap_queue) {
                        *(volatile unsigned*)(B.qflag + sl) = B.tag;
                    } else {
                        atomicOr(&C->overflow, kOvfFrontier);
                        atomicExch(&C->abort_, 1u);
                    }
                }
                for (unsigned x = c0; x < c0 + nc; x++) {
                    if (x < B.cap_cand) {
                        *(volatile unsigned*)(B.cflag + x) = B.tag;
                    } else {
                        atomicOr(&C->overflow, kOvfCand);
                        atomicExch(&C->abort_, 1u);
                    }
                }
            }
            __syncwarp();  // stack pushes visible to the whole warp
            sn += keep;
            if (ticket) {
                unsigned qm = qball;
                if constexpr (QUAD) {
                    qm = 0;
#pragma unroll
                    for (int q = 0; q < 8; q++) qm |= ((qball >> (4 * q)) & 1u) << q;
                }
                npend &= ~qm;
                if (npend == 0u) ticket = false;
            }
            if (__any_sync(0xffffffffu, ab != 0u)) break;
            continue;
        }
        if (__any_sync(0xffffffffu, ab != 0u)) break;
        // ---- no node pair: candidates of the candidate ticket ----
        const bool cready = cslot && ctag == B.tag;
        const unsigned cavail = __ballot_sync(0xffffffffu, cready);
        if (cavail) {
            idle = 0;
            backoff = 32;
            uint4 c = make_uint4(0u, 0u, 0u, 0u);
            if (cready) {
                c = __ldcg(B.cand + i);  // ordered after the tag's acquire load
            }
            filter_candidates<F64>(B, cready, c, decided, tested);
            cpend &= ~cavail;
            if (cpend == 0u) {
                cbase = take_ticket(&C->c_head);
                cpend = 0xffffffffu;
            }
            continue;
        }
        // ---- nothing ready: over, or wait.  Over (all seed tests done, then
        // work == 0, read in that order) means no node pair exists any more and
        // no slot will be published: the warp is done once none of its pending
        // candidate slots lies below the final candidate count.
        if ((idle & 3u) == 3u) {
            unsigned over = 0, ncand = 0;
            if (lane == 0) {
                const unsigned sd = ld_vol(&C->seed_done);
                fence_acq_rel();
                const unsigned long long wc = *(const volatile unsigned long long*)&C->work_cand;
                over = sd == seed_total && (unsigned)wc == 0u;
                ncand = min((unsigned)(wc >> 32), B.cap_cand);
            }
            over = __shfl_sync(0xffffffffu, over, 0);
            ncand = __shfl_sync(0xffffffffu, ncand, 0);
            if (over && !__any_sync(0xffffffffu, ((cpend >> lane) & 1u) && i < ncand)) break;
        }
        if (++idle > kIdleSpins) {
            if (lane == 0) {
                atomicOr(&C->err, kErrTimeout);
                atomicExch(&C->abort_, 1u);
            }
            break;
        }
        __nanosleep(backoff);
        backoff = min(backoff * 2u, 256u);
    }
    block_stats(C, visited, decided, tested, maxlev + 1u);
}

// ---------------------------------------------------------------------------
// Level-synchronous BVH4 x BVH4 traversal (one cooperative launch).
//
// In the queue traversal above, the levels' end times advance by 12-15 us while
// one warp iteration takes about 3 us: most of a level is the hand-off of node
// pairs between warps through tagged queue slots.  Here the grid moves level by
// level instead.  All node pairs of a level, and the leaf pairs the previous
// level made, are split among all warps in static chunks (warp w takes chunks
// w, w + warps, ...); the children form the next level's list; one grid barrier
// (about a microsecond) separates the levels, so a level costs one or a few warp
// iterations plus the barrier.  A level of at most `quad_below` node pairs is
// expanded in the quad form (a quarter of the dependent chain, 8 node pairs per
// warp), a wider one in the lane form (32 per warp).
//
// Level l appends its node children (low half) and its leaf pairs (high half)
// to the 64-bit counter lvl[l % 3], one atomic per warp and chunk.  The last
// block to arrive at the barrier that ends level l decides whether the
// traversal is over (no pair made, or the abort flag set: the same decision
// for every block), clears lvl[(l + 2) % 3] (last read before level l began)
// and stamps the level's end time.  Node pairs of level l live in half l % 2 of
// the queue buffer; leaf pairs are appended to the candidate list in level
// order, so level l + 1 filters candidates [snap_l, snap_l + count) with snap
// summed from the counters in every block alike.  Every barrier wait is
// bounded; a spent wait sets kErrTimeout and the abort flag and the block ends.
// ---------------------------------------------------------------------------
__device__ __forceinline__ unsigned long long globaltimer_ns()
{
    unsigned long long t;
    asm volatile("mov.u64 %0, %%globaltimer;" : "=l"(t));
    return t;
}

__device__ __forceinline__ void st_release_u32(unsigned* p, unsigned v)
{
    asm volatile("st.release.gpu.global.u32 [%0], %1;" ::"l"(p), "r"(v) : "memory");
}
__device__ __forceinline__ void st_relaxed_u32(unsigned* p, unsigned v)
{
    asm volatile("st.relaxed.gpu.global.u32 [%0], %1;" ::"l"(p), "r"(v) : "memory");
}

// Grid barrier ending level `lev` of the level-synchronous traversal, among
// `nblocks` blocks.  Returns false when the block's wait ran out (the block must
// leave the kernel).  The last block to arrive decides for every block whether
// the traversal is over, clears the counter slot that level lev + 2 will use,
// stamps the level's end time and publishes the level's candidates to the
// candidate blocks (split form); they are all written once every node block has
// arrived.  Its loads go out together and its stores are released by one
// release store of the generation word, so the barrier costs few round trips
// to L2 on its critical path.
__device__ __forceinline__ bool level_barrier(const Bufs& B, unsigned& gen, unsigned lev, unsigned nblocks,
                                              unsigned long long& v_out, bool& stop_out)
{
    __shared__ unsigned s_ok, s_stop;
    __shared__ unsigned long long s_v;
    Counters* C = B.cnt;
    __syncthreads();
    if (threadIdx.x == 0) {
        s_ok = 1u;
        // the arrival is an acquire-release atomic: it releases this block's
        // writes of the level (ordered before it by the block barrier) and, for
        // the last arriver, acquires every other block's
        const unsigned arrived = arrive_acq_rel(&C->bar_count) + 1u;
        if (arrived == nblocks) {
            // every block has arrived: the counts of this level are final
            const unsigned long long v = __ldcg(&C->lvl[lev % 3u]);
            const unsigned ab = __ldcg(&C->abort_);
            const unsigned prev = __ldcg(&C->cand_total);
            // with published candidates the levels stop when no node pair is left
            // (the filtering warps finish the candidates); otherwise when the
            // level made nothing
            const bool stop = ab != 0u || (B.publish ? (unsigned)v == 0u : v == 0ull);
            const unsigned tot = prev + (unsigned)(v >> 32);
            C->bar_count = 0u;
            C->bstop = stop ? 1u : 0u;
            C->bpub[0] = v;
            C->bpub[1] = stop ? 1ull : 0ull;
            s_v = v;
            s_stop = stop ? 1u : 0u;
            C->lvl[(lev + 2u) % 3u] = 0ull;
            C->cand_total = tot;
            atomicMax(&C->q_tail, 2u * (unsigned)v);  // both halves of the queue buffer must hold the widest level
            if (lev < (unsigned)kLevelTimes) C->level_ns[lev] = globaltimer_ns();
            if (B.publish) {
                st_relaxed_u32(&C->cand_ready, tot);
                // cand_ready is visible before the final flag
                if (stop) st_release_u32(&C->cand_final, 1u);
            }
            st_release_u32(&C->bar_gen, gen + 1u);  // releases every store above
        } else {
            unsigned spins = 0;
            while (ld_acq(&C->bar_gen) == gen) {
                if (++spins > kIdleSpins) {
                    atomicOr(&C->err, kErrTimeout);
                    atomicExch(&C->abort_, 1u);
                    s_ok = 0u;
                    break;
                }
                __nanosleep(32);
            }
            // the level's counts and the decision, published before the release
            const ulonglong2 pub = __ldcg(reinterpret_cast<const ulonglong2*>(C->bpub));
            s_v = pub.x;
            s_stop = pub.y != 0ull ? 1u : 0u;
        }
        gen++;
    }
    __syncthreads();
    v_out = s_v;
    stop_out = s_stop != 0u;
    return s_ok != 0u;
}

// Level 0: every pair of the two meshes' cut entries; overlapping pairs become
// the first level's node pairs or candidates.
template <bool F64>
__device__ __forceinline__ void seed_levels(const Bufs& B, unsigned gw, unsigned nw, uint4* front, uint32_t capL)
{
    using S = typename Prec<F64>::S;
    Counters* C = B.cnt;
    const unsigned lane = threadIdx.x & 31;
    const unsigned per_job = seed_tests_per_job(B);
    const unsigned total = B.njobs * per_job;
    const unsigned coff = B.deep_seed ? (unsigned)kCutMax : 0u;
    for (unsigned base = gw * 32u; base < total; base += nw * 32u) {
        const unsigned g = base + lane;
        bool fr = false, cand = false;
        uint32_t ra = 0, rb = 0, job = 0;
        if (g < total) {
            job = g / per_job;
            const unsigned t = g % per_job;
            const JobDev& J = B.jobs[job];
            const bool both = J.A.nt && J.B.nt;
            const unsigned nA = both ? __ldg(J.A.ncuts + (B.deep_seed ? 1 : 0)) : 0u;
            const unsigned nB = both ? __ldg(J.B.ncuts + (B.deep_seed ? 1 : 0)) : 0u;
            if (t < nA * nB) {
                const unsigned i = coff + t / nB, j = coff + t % nB;
                const S* ba_ = F64 ? (const S*)J.A.cutBox64 : (const S*)J.A.cutBox;
                const S* bb_ = F64 ? (const S*)J.B.cutBox64 : (const S*)J.B.cutBox;
                Box<S> ba, bb;
                for (int k = 0; k < 3; k++) {
                    ba.lo[k] = ba_[6 * i + k];
                    ba.hi[k] = ba_[6 * i + 3 + k];
                    bb.lo[k] = bb_[6 * j + k];
                    bb.hi[k] = bb_[6 * j + 3 + k];
                }
                if (!J.pa.identity) world_box(J.pa, ba);
                if (!J.pb.identity) world_box(J.pb, bb);
                if (overlap(ba, bb)) {
                    ra = J.A.cutRef[i];
                    rb = J.B.cutRef[j];
                    cand = (ra & kLeaf) && (rb & kLeaf);
                    fr = !cand;
                }
            }
        }
        const unsigned fb = __ballot_sync(0xffffffffu, fr), cb = __ballot_sync(0xffffffffu, cand);
        if (!(fb | cb)) continue;
        unsigned long long old = 0;
        if (lane == 0) old = atomicAdd(&C->lvl[0], ((unsigned long long)__popc(cb) << 32) + __popc(fb));
        old = __shfl_sync(0xffffffffu, old, 0);
        const unsigned lt = (1u << lane) - 1u;
        if (fr) {
            const unsigned pf = (unsigned)old + __popc(fb & lt);
            if (pf < capL) {
                front[pf] = make_uint4(job, ra, rb, 0u);
            } else {
                atomicOr(&C->overflow, kOvfFrontier);
                atomicExch(&C->abort_, 1u);
            }
        }
        if (cand) {
            const unsigned pc = (unsigned)(old >> 32) + __popc(cb & lt);
            if (pc < B.cap_cand) {
                B.cand[pc] = make_uint4(job, ra & ~kLeaf, rb & ~kLeaf, 0u);
            } else {
                atomicOr(&C->overflow, kOvfCand);
                atomicExch(&C->abort_, 1u);
            }
        }
    }
}

// Reserves the warp's children in one atomic: node pairs of the next level and
// candidates of this level.  nf / nc: this lane's counts.  Returns this lane's
// first node-pair slot (f) and first candidate slot (c).
__device__ __forceinline__ void level_reserve(const Bufs& B, unsigned lev, unsigned snap, unsigned nf, unsigned nc,
                                              unsigned& f, unsigned& c)
{
    const unsigned lane = threadIdx.x & 31;
    unsigned incf = nf, incc = nc;
#pragma unroll
    for (int o = 1; o < 32; o <<= 1) {
        const unsigned yf = __shfl_up_sync(0xffffffffu, incf, o);
        const unsigned yc = __shfl_up_sync(0xffffffffu, incc, o);
        if (lane >= (unsigned)o) {
            incf += yf;
            incc += yc;
        }
    }
    unsigned long long old = 0;
    if (lane == 31 && (incf | incc))
        old = atomicAdd(&B.cnt->lvl[lev % 3u], ((unsigned long long)incc << 32) + incf);
    old = __shfl_sync(0xffffffffu, old, 31);
    f = (unsigned)old + incf - nf;
    c = snap + (unsigned)(old >> 32) + incc - nc;
}

// Published candidates (split form).  A warp takes chunks of 32 candidates
// with one atomic and filters each once the node blocks have published it
// (every level's candidates are published by the barrier that ends it).  The
// loop is software-pipelined: the next chunk is claimed before the current one
// is filtered, and when it is already published, its candidate records and
// triangle records are loaded before the current chunk's vertices, so these
// two dependent round trips overlap the current chunk's work.  A warp leaves
// when its chunk starts at or beyond the final count.
constexpr unsigned kGone = 0xffffffffu;

// Lane 0 waits (bounded) until the chunk at `base` is published in full or no
// more candidates will come; returns the published count, or kGone.
__device__ __forceinline__ unsigned wait_published(Counters* C, unsigned base)
{
    unsigned ready = 0, spins = 0;
    for (;;) {
        ready = ld_acq(&C->cand_ready);
        if (ready >= base + 32u) return ready;
        if (ld_acq(&C->cand_final)) return ld_acq(&C->cand_ready);  // written before the final flag
        if (ld_vol(&C->abort_)) return kGone;
        if (++spins > kIdleSpins) {
            atomicOr(&C->err, kErrTimeout);
            atomicExch(&C->abort_, 1u);
            return kGone;
        }
        __nanosleep(64);
    }
}

struct PubChunk {
    uint4 c;       // candidate: job, leaf position in A, leaf position in B
    uint4 ta, tb;  // the two leaves' records: vertex indices and original triangle id
    bool have;
};

__device__ __forceinline__ PubChunk load_published(const Bufs& B, unsigned base, unsigned ready)
{
    PubChunk k;
    const unsigned i = base + (threadIdx.x & 31u);
    k.have = i < min(ready, B.cap_cand);
    k.c = k.have ? __ldcg(B.cand + i) : make_uint4(0u, 0u, 0u, 0u);
    k.ta = k.tb = make_uint4(0u, 0u, 0u, 0u);
    if (k.have) {
        const JobDev& J = B.jobs[k.c.x];
        k.ta = __ldg(J.A.leafTri + k.c.y);
        k.tb = __ldg(J.B.leafTri + k.c.z);
    }
    return k;
}

template <bool F64>
__device__ __forceinline__ void filter_loaded(const Bufs& B, const PubChunk& k, unsigned long long& decided,
                                              unsigned long long& tested)
{
    Counters* C = B.cnt;
    int dec = DEC_NO;
    unsigned pat = 0;
    if (k.have) {
        tested++;
        const JobDev& J = B.jobs[k.c.x];
        double3 P[3], Q[3];
        P[0] = world_vertex(J.A.verts, k.ta.x, J.pa);
        P[1] = world_vertex(J.A.verts, k.ta.y, J.pa);
        P[2] = world_vertex(J.A.verts, k.ta.z, J.pa);
        Q[0] = world_vertex(J.B.verts, k.tb.x, J.pb);
        Q[1] = world_vertex(J.B.verts, k.tb.y, J.pb);
        Q[2] = world_vertex(J.B.verts, k.tb.z, J.pb);
        if constexpr (F64) dec = classify_fast<double>(P, Q, &pat);
        else dec = classify_fast<float>(P, Q, &pat);
        decided += (dec != DEC_ESC);
    }
    const bool yes = k.have && dec == DEC_YES;
    const bool esc = k.have && dec == DEC_ESC;
    const unsigned pr = warp_append(yes, &C->res);
    if (yes) {
        if (pr < B.cap_res) B.res[pr] = make_uint4(k.c.x, k.ta.w, k.tb.w, pat);
        else atomicOr(&C->overflow, kOvfRes);
    }
    const unsigned pe = warp_append(esc, &C->esc);
    if (esc) {
        if (pe < B.cap_esc) B.esc[pe] = make_uint4(k.c.x, k.c.y, k.c.z, 0u);
        else atomicOr(&C->overflow, kOvfEsc);
    }
}

template <bool F64>
__device__ __forceinline__ void filter_published(const Bufs& B, unsigned long long& decided,
                                                 unsigned long long& tested)
{
    Counters* C = B.cnt;
    const unsigned lane = threadIdx.x & 31;
    unsigned base = 0, ready = 0;
    if (lane == 0) {
        base = atomicAdd(&C->c_head, 32u);
        ready = wait_published(C, base);
    }
    base = __shfl_sync(0xffffffffu, base, 0);
    ready = __shfl_sync(0xffffffffu, ready, 0);
    if (ready == kGone || base >= ready) return;
    PubChunk cur = load_published(B, base, ready);
    for (;;) {
        // the next chunk: claimed now, its records loaded now if it is published
        unsigned nbase = 0, nready = 0;
        if (lane == 0) {
            nbase = atomicAdd(&C->c_head, 32u);
            nready = ld_acq(&C->cand_ready);
        }
        nbase = __shfl_sync(0xffffffffu, nbase, 0);
        nready = __shfl_sync(0xffffffffu, nready, 0);
        const bool early = nready >= nbase + 32u;
        PubChunk nxt;
        if (early) nxt = load_published(B, nbase, nready);
        filter_loaded<F64>(B, cur, decided, tested);
        if (!early) {
            if (lane == 0) nready = wait_published(C, nbase);
            nready = __shfl_sync(0xffffffffu, nready, 0);
            if (nready == kGone || nbase >= nready) return;
            nxt = load_published(B, nbase, nready);
        }
        cur = nxt;
    }
}

template <bool F64>
__global__ void __launch_bounds__(kTravThreads, 2) k_traverse_levels(Bufs B)
{
    Counters* C = B.cnt;
    const unsigned lane = threadIdx.x & 31;
    // blocks [0, nblocks) expand node pairs; in the split form the others filter candidates
    const unsigned nblocks = gridDim.x - B.cand_blocks;
    const bool node_block = blockIdx.x < nblocks;
    const unsigned gw = (blockIdx.x * blockDim.x + threadIdx.x) >> 5;
    const unsigned nw = (nblocks * blockDim.x) >> 5;
    const uint32_t capL = B.cap_queue / 2u;
    uint4* const front0 = B.queue;
    uint4* const front1 = B.queue + capL;
    allow_dependent_launch();
    if (blockIdx.x == 0 && threadIdx.x == 0) C->t_start = globaltimer_ns();
    unsigned long long visited = 0, decided = 0, tested = 0;
    unsigned gen = 0, snap = 0, lev = 0;
    bool ovf_f = false, ovf_c = false;
    // the node blocks seed; the candidate blocks filter from the start
    if (node_block) seed_levels<F64>(B, gw, nw, front0, capL);
    else filter_published<F64>(B, decided, tested);
    for (; node_block;) {
        unsigned long long v;
        bool stop;
        if (!level_barrier(B, gen, lev, nblocks, v, stop)) return;
        if (stop) break;
        // v: the pairs made by level `lev`, expanded and filtered by level lev + 1
        const unsigned n = min((unsigned)v, capL);
        const unsigned cbase = snap, cend = min(snap + (unsigned)(v >> 32), B.cap_cand);
        snap += (unsigned)(v >> 32);
        ++lev;
        const uint4* cur = (lev & 1u) ? front0 : front1;
        uint4* nxt = (lev & 1u) ? front1 : front0;
        const bool quad = n <= B.quad_below;
        const unsigned per = quad ? 8u : 32u;
        const unsigned node_chunks = (n + per - 1u) / per;
        // published candidates are left to the filtering warps
        const unsigned chunks = node_chunks + (!B.publish && cend > cbase ? (cend - cbase + 31u) / 32u : 0u);
        for (unsigned k = gw; k < chunks; k += nw) {
            if (k < node_chunks) {
                if (quad) {
                    const unsigned unit = lane >> 2, sub = lane & 3u;
                    const unsigned idx = k * 8u + unit;
                    const bool have = idx < n;
                    const uint4 ent = have ? __ldcg(cur + idx) : make_uint4(0u, kEmpty, kEmpty, 0u);
                    visited += (have && sub == 0u) ? 1u : 0u;
                    unsigned fm = 0, cm = 0;
                    uint32_t ca = kEmpty, cb[4];
                    expand_quad<F64>(B, ent, have, sub, fm, cm, ca, cb);
                    unsigned f, c;
                    level_reserve(B, lev, snap, __popc(fm), __popc(cm), f, c);
#pragma unroll
                    for (int j = 0; j < 4; j++) {
                        if ((fm >> j) & 1u) {
                            if (f < capL) nxt[f] = make_uint4(ent.x, ca, cb[j], 0u);
                            else ovf_f = true;
                            f++;
                        }
                        if ((cm >> j) & 1u) {
                            if (c < B.cap_cand) B.cand[c] = make_uint4(ent.x, ca & ~kLeaf, cb[j] & ~kLeaf, 0u);
                            else ovf_c = true;
                            c++;
                        }
                    }
                } else {
                    const unsigned idx = k * 32u + lane;
                    const bool have = idx < n;
                    uint4 ent = make_uint4(0u, kEmpty, kEmpty, 0u);
                    unsigned fm = 0, cm = 0;
                    uint32_t ca[4], cb[4];
                    if (have) {
                        ent = __ldcg(cur + idx);
                        visited++;
                        expand_pair<F64>(B, ent, fm, cm, ca, cb);
                    }
                    unsigned f, c;
                    level_reserve(B, lev, snap, __popc(fm), __popc(cm), f, c);
                    // child slot q = 4i + j is the pair (A child i, B child j); the
                    // unrolled loop indexes the registers with constants
#pragma unroll
                    for (int q = 0; q < 16; q++) {
                        if ((fm >> q) & 1u) {
                            if (f < capL) nxt[f] = make_uint4(ent.x, ca[q >> 2], cb[q & 3], 0u);
                            else ovf_f = true;
                            f++;
                        }
                        if ((cm >> q) & 1u) {
                            if (c < B.cap_cand)
                                B.cand[c] = make_uint4(ent.x, ca[q >> 2] & ~kLeaf, cb[q & 3] & ~kLeaf, 0u);
                            else ovf_c = true;
                            c++;
                        }
                    }
                }
            } else {
                const unsigned i = cbase + (k - node_chunks) * 32u + lane;
                const bool have = i < cend;
                const uint4 cnd = have ? __ldcg(B.cand + i) : make_uint4(0u, 0u, 0u, 0u);
                filter_candidates<F64>(B, have, cnd, decided, tested);
            }
        }
        if (ovf_f || ovf_c) {
            if (ovf_f) atomicOr(&C->overflow, kOvfFrontier);
            if (ovf_c) atomicOr(&C->overflow, kOvfCand);
            atomicExch(&C->abort_, 1u);
            ovf_f = ovf_c = false;
        }
    }
    // published candidates: the node blocks are done (the last barrier published
    // every candidate and the final flag) and filter what is left
    if (node_block && B.publish) filter_published<F64>(B, decided, tested);
    block_stats(C, visited, decided, tested);
    if (blockIdx.x == 0 && threadIdx.x == 0) {
        C->levels = lev;
        C->work_cand = (unsigned long long)snap << 32;  // candidates made, for the host's retry sizing
    }
}

// ===========================================================================
// Exact stage and segments
// ===========================================================================
// Exact stage over the escalated pairs, grid-stride over the threads of the
// launch (nth a multiple of 32): intersecting pairs are appended to the results.
__device__ __forceinline__ void exact_stage(const Bufs& B, unsigned gtid, unsigned nth)
{
    Counters* C = B.cnt;
    const unsigned lane = threadIdx.x & 31;
    unsigned ne = ld_cg_u32(&C->esc);
    if (ne > B.cap_esc) ne = B.cap_esc;
    unsigned long long nexact = 0;
    for (unsigned base = gtid - lane; base < ne; base += nth) {
        const unsigned i = base + lane;
        const bool have = i < ne;
        bool yes = false;
        uint32_t ta = 0, tb = 0, job = 0;
        if (have) {
            uint4 c = __ldcg(B.esc + i);
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

__global__ void __launch_bounds__(128) k_exact(Bufs B)
{
    exact_stage(B, blockIdx.x * blockDim.x + threadIdx.x, gridDim.x * blockDim.x);
}

__device__ __forceinline__ void load_tri_orig(const MeshDev& M, const DevPose& P, uint32_t tri, double3* out)
{
    const uint32_t* t = M.tris + 3 * (size_t)tri;
    out[0] = world_vertex(M.verts, __ldg(t), P);
    out[1] = world_vertex(M.verts, __ldg(t + 1), P);
    out[2] = world_vertex(M.verts, __ldg(t + 2), P);
}

// One endpoint of a general-position segment: crossing `sel` of the pattern
// (0, 1: P's edges from its lone vertex through plane(Q); 2, 3: Q's edges from
// its lone vertex through plane(P)), fast path on values in registers, the
// exact construction when the rounding test fails.
__device__ __forceinline__ bool pattern_point(const double3* pts, int o1, int o2, int sel, double3& q,
                                              unsigned long long* exact_points)
{
    const double3 P0 = pts[0], P1 = pts[1], P2 = pts[2], Q0 = pts[3], Q1 = pts[4], Q2 = pts[5];
    const bool onP = sel < 2;
    const int lone = onP ? o1 : o2;
    // the lone vertex and the other end of the edge (the non-lone vertices in order)
    const double3 T0 = onP ? P0 : Q0, T1 = onP ? P1 : Q1, T2 = onP ? P2 : Q2;
    const double3 L = lone == 0 ? T0 : (lone == 1 ? T1 : T2);
    const int first = (sel & 1) == 0;
    const double3 E = first ? (lone == 0 ? T1 : T0) : (lone == 2 ? T1 : T2);
    const double3 U0 = onP ? Q0 : P0, U1 = onP ? Q1 : P1, U2 = onP ? Q2 : P2;
    if (construct_plane_fast(U0, U1, U2, L, E, q)) return true;
    const int other = first ? (lone == 0 ? 1 : 0) : (lone == 2 ? 1 : 2);
    const SymPt sp = onP ? sp_plane(o1, other, 3, 4, 5) : sp_plane(3 + o2, 3 + other, 0, 1, 2);
    return construct_point(pts, sp, q, exact_points);
}

// Segments of one result (up to 3, 6 doubles each, at o): their count.  A
// result that carries an endpoint pattern (decided by the first filter in
// general position) only needs its two crossings constructed; `per` threads
// (1 or 2, adjacent lanes) share it, thread `half` constructing endpoints
// half, half + per, ..  A result without a pattern is classified exactly by
// its thread with half = 0 alone (the others return 0).
__device__ __forceinline__ uint32_t result_segments(const Bufs& B, const uint4& rr, double* o, unsigned half = 0u,
                                                    unsigned per = 1u)
{
    Counters* C = B.cnt;
    const JobDev& J = B.jobs[B.njobs == 1 ? 0u : rr.x];  // one job: its loads need not wait for rr
    double3 pts[6];
    load_tri_orig(J.A, J.pa, rr.y, pts);
    load_tri_orig(J.B, J.pb, rr.z, pts + 3);
    if (rr.w & kPatValid) {
        const int o1 = (rr.w >> 1) & 3, o2 = (rr.w >> 3) & 3;
        unsigned m = ((rr.w >> 5) & 3u) | (((rr.w >> 7) & 3u) << 2);
        const int s0 = __ffs(m) - 1;
        m &= m - 1u;
        const int s1 = m ? __ffs(m) - 1 : s0;
        for (unsigned k = half; k < 2u; k += per) {
            double3 q;
            if (!pattern_point(pts, o1, o2, k ? s1 : s0, q, &C->exact_points)) atomicOr(&C->err, kErrExactCapacity);
            o[3 * k] = q.x;
            o[3 * k + 1] = q.y;
            o[3 * k + 2] = q.z;
        }
        return 1;
    }
    if (half) return 0;
    ExactSigns S{&C->err, 0ull};
    TTRes r;
    classify_exact(pts, r, S);
    double3 q[3];
    if (r.kind == KIND_POINT || r.kind == KIND_SEGMENT || r.kind == KIND_TRIANGLE) {
        for (int k = 0; k < r.n && k < 3; k++)
            if (!construct_point(pts, r.pt[k], q[k], &C->exact_points)) atomicOr(&C->err, kErrExactCapacity);
        if (r.kind == KIND_POINT) {
            double v[6] = {q[0].x, q[0].y, q[0].z, q[0].x, q[0].y, q[0].z};
            for (int k = 0; k < 6; k++) o[k] = v[k];
            return 1;
        }
        if (r.kind == KIND_SEGMENT) {
            double v[6] = {q[0].x, q[0].y, q[0].z, q[1].x, q[1].y, q[1].z};
            for (int k = 0; k < 6; k++) o[k] = v[k];
            return 1;
        }
        for (int e = 0; e < 3; e++) {
            const double3& u = q[e];
            const double3& w = q[(e + 1) % 3];
            double v[6] = {u.x, u.y, u.z, w.x, w.y, w.z};
            for (int k = 0; k < 6; k++) o[6 * e + k] = v[k];
        }
        return 3;
    }
    return 0;
}

__global__ void __launch_bounds__(128) k_segments(Bufs B, double* __restrict__ segs, uint32_t* __restrict__ nseg)
{
    Counters* C = B.cnt;
    const unsigned gtid = blockIdx.x * blockDim.x + threadIdx.x;
    const unsigned nth = gridDim.x * blockDim.x;
    if (ld_cg_u32(&C->overflow)) return;
    unsigned nres = ld_cg_u32(&C->res);
    if (nres > B.cap_res) nres = B.cap_res;
    for (unsigned i = gtid; i < nres; i += nth) nseg[i] = result_segments(B, __ldcg(B.res + i), segs + 18 * (size_t)i);
}

// ===========================================================================
// Ordering: results sorted by (job, a, b) with an LSD radix sort whose sizes
// come from the device counters (no host round trip).  One kernel builds the
// keys and the digit histograms of every pass, one scans them, and each pass
// is one scatter kernel: tiles of 4096 items take their global offset per
// digit by decoupled look-back over the preceding tiles (bounded waits).
// The gather kernel applies the permutation and places the segments, finding
// its segment offset by the same look-back.
// ===========================================================================
constexpr int kOsThreads = 256;
constexpr int kOsItems = 16;
constexpr int kOsTile = kOsThreads * kOsItems;
constexpr int kOsWarps = kOsThreads / 32;
constexpr int kOsGatherTile = 1024;

__device__ __forceinline__ unsigned res_count(const Bufs& B)
{
    if (ld_cg_u32(&B.cnt->overflow)) return 0u;
    unsigned n = ld_cg_u32(&B.cnt->res);
    return n > B.cap_res ? B.cap_res : n;
}

__device__ __forceinline__ unsigned long long order_key(const uint4& r, const OrderBufs& O)
{
    return ((unsigned long long)r.x << (O.bits_a + O.bits_b)) | ((unsigned long long)r.y << O.bits_b) | r.z;
}

// Keys, identity values and the histograms of every digit pass; the last
// block to finish scans the histograms into digit bases (and clears them for
// the next call), so no separate scan launch is needed.
__global__ void __launch_bounds__(kOsThreads) k_os_hist(Bufs B, OrderBufs O)
{
    __shared__ unsigned h[kOsMaxPasses][256];
    __shared__ uint32_t sw[33];
    __shared__ unsigned s_last;
    const unsigned n = res_count(B);
    for (int p = 0; p < O.passes; p++) h[p][threadIdx.x] = 0;
    // look-back status of every pass and of the gather starts unset
    const unsigned ntiles = (n + kOsTile - 1) / kOsTile;
    const size_t nstat = (size_t)(O.passes + 1) * O.ntiles_cap * 256;
    for (size_t k = blockIdx.x * (size_t)blockDim.x + threadIdx.x; k < nstat; k += (size_t)gridDim.x * blockDim.x) {
        const size_t t = (k / 256) % O.ntiles_cap;
        if (t < ntiles) O.status[k] = 0u;
    }
    const unsigned ngather = (n + kOsGatherTile - 1) / kOsGatherTile;
    for (unsigned k = blockIdx.x * blockDim.x + threadIdx.x; k < ngather; k += gridDim.x * blockDim.x)
        O.gstatus[k] = 0u;
    if (blockIdx.x == 0 && threadIdx.x <= (unsigned)O.passes) O.tile_ctr[threadIdx.x] = 0u;
    __syncthreads();
    for (unsigned i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x) {
        const unsigned long long key = order_key(__ldcg(B.res + i), O);
        O.keys[0][i] = key;
        O.vals[0][i] = i;
        for (int p = 0; p < O.passes; p++) atomicAdd(&h[p][(unsigned)(key >> (8 * p)) & 255u], 1u);
    }
    __syncthreads();
    for (int p = 0; p < O.passes; p++)
        if (h[p][threadIdx.x]) atomicAdd(&O.hist[p * 256 + threadIdx.x], h[p][threadIdx.x]);
    __threadfence();
    __syncthreads();
    if (threadIdx.x == 0) s_last = (atomicAdd(&O.tile_ctr[kOsMaxPasses + 1], 1u) == gridDim.x - 1) ? 1u : 0u;
    __syncthreads();
    if (!s_last) return;
    __threadfence();
    for (int p = 0; p < O.passes; p++) {
        const unsigned v = __ldcg(&O.hist[p * 256 + threadIdx.x]);
        unsigned tot;
        const unsigned ex = block_exclusive_scan(v, sw, &tot);
        O.base[p * 256 + threadIdx.x] = ex;
        O.hist[p * 256 + threadIdx.x] = 0u;
    }
    if (threadIdx.x == 0) O.tile_ctr[kOsMaxPasses + 1] = 0u;
}

__global__ void __launch_bounds__(kOsThreads) k_os_scatter(Bufs B, OrderBufs O, int pass)
{
    __shared__ unsigned wc[kOsWarps][256];
    __shared__ unsigned tile_base[256];
    __shared__ unsigned s_tile;
    const unsigned n = res_count(B);
    const unsigned ntiles = (n + kOsTile - 1) / kOsTile;
    if (threadIdx.x == 0) s_tile = atomicAdd(&O.tile_ctr[pass], 1u);
    __syncthreads();
    const unsigned tile = s_tile;
    if (tile >= ntiles) return;
    const int lane = threadIdx.x & 31, w = threadIdx.x >> 5;
    const int shift = 8 * pass;
    const unsigned long long* kin = O.keys[pass & 1];
    const uint32_t* vin = O.vals[pass & 1];
    unsigned long long* kout = O.keys[(pass + 1) & 1];
    uint32_t* vout = O.vals[(pass + 1) & 1];
    for (int d = lane; d < 256; d += 32) wc[w][d] = 0;
    __syncwarp();
    const unsigned seg = tile * kOsTile + w * 32 * kOsItems;
    unsigned long long key[kOsItems];
    uint32_t val[kOsItems], rank[kOsItems], dig[kOsItems];
    const unsigned lt = (1u << lane) - 1u;
    // all loads first (independent, in flight together), then the ranking
#pragma unroll
    for (int c = 0; c < kOsItems; c++) {
        const unsigned i = seg + c * 32 + lane;
        key[c] = i < n ? __ldcg(kin + i) : 0ull;
        val[c] = i < n ? __ldcg(vin + i) : 0u;
    }
#pragma unroll
    for (int c = 0; c < kOsItems; c++) {
        const unsigned i = seg + c * 32 + lane;
        const bool ok = i < n;
        const unsigned d = ok ? ((unsigned)(key[c] >> shift) & 255u) : 256u;
        dig[c] = d;
        const unsigned peers = __match_any_sync(0xffffffffu, d);
        rank[c] = ok ? wc[w][d] + __popc(peers & lt) : 0u;
        __syncwarp();
        if (ok && (peers & lt) == 0) wc[w][d] += __popc(peers);
        __syncwarp();
    }
    __syncthreads();
    {
        const unsigned d = threadIdx.x;
        unsigned run = 0;
        for (int q = 0; q < kOsWarps; q++) {
            const unsigned t = wc[q][d];
            wc[q][d] = run;
            run += t;
        }
        unsigned excl;
        lookback(O.status + (size_t)pass * O.ntiles_cap * 256 + d, tile, 256, run, &excl, &B.cnt->err);
        tile_base[d] = O.base[pass * 256 + d] + excl;
    }
    __syncthreads();
#pragma unroll
    for (int c = 0; c < kOsItems; c++) {
        const unsigned d = dig[c];
        if (d < 256u) {
            const unsigned pos = tile_base[d] + wc[w][d] + rank[c];
            kout[pos] = key[c];
            vout[pos] = val[c];
        }
    }
}

// sorted position k -> pairs_out[k], job_out[k]; the segments of the pair go
// to the prefix sum of the segment counts (tile look-back).  One item per
// thread, so every load of a thread is issued at once.
__global__ void __launch_bounds__(kOsGatherTile) k_os_gather(Bufs B, OrderBufs O, const double* __restrict__ segs,
                                                             const uint32_t* __restrict__ nseg, int32_t* pairs_out,
                                                             uint32_t* job_out, double* segs_out,
                                                             int32_t* segpair_out, int want_segments, int sorted)
{
    __shared__ uint32_t sw[33];
    __shared__ unsigned s_tile, s_base;
    const unsigned n = res_count(B);
    const unsigned ntiles = (n + kOsGatherTile - 1) / kOsGatherTile;
    if (threadIdx.x == 0) s_tile = atomicAdd(&O.tile_ctr[O.passes], 1u);
    __syncthreads();
    const unsigned tile = s_tile;
    if (tile >= ntiles) return;
    const unsigned k = tile * kOsGatherTile + threadIdx.x;
    const bool ok = k < n;
    const unsigned src = ok ? (sorted ? __ldcg(O.vals[O.passes & 1] + k) : k) : 0u;
    const unsigned c = (ok && want_segments) ? __ldcg(nseg + src) : 0u;
    const uint4 r = ok ? __ldcg(B.res + src) : make_uint4(0u, 0u, 0u, 0u);
    unsigned tot;
    const unsigned ex = block_exclusive_scan(c, sw, &tot);
    if (threadIdx.x == 0) {
        unsigned excl;
        lookback(O.gstatus, tile, 1, tot, &excl, &B.cnt->err);
        s_base = excl;
        if (tile == ntiles - 1) B.cnt->nseg = excl + tot;
    }
    __syncthreads();
    if (!ok) return;
    pairs_out[2 * (size_t)k] = (int32_t)r.y;
    pairs_out[2 * (size_t)k + 1] = (int32_t)r.z;
    job_out[k] = r.x;
    const unsigned off = s_base + ex;
    for (unsigned q = 0; q < c; q++) {
        const double2* sp = reinterpret_cast<const double2*>(segs + 18 * (size_t)src + 6 * q);
        double2* dp = reinterpret_cast<double2*>(segs_out + 6 * (size_t)(off + q));
        dp[0] = __ldcg(sp);
        dp[1] = __ldcg(sp + 1);
        dp[2] = __ldcg(sp + 2);
        segpair_out[off + q] = (int32_t)k;
    }
}

size_t order_scratch_bytes(uint32_t cap, int passes)
{
    size_t ntiles = (cap + kOsTile - 1) / kOsTile;
    return 2 * sizeof(unsigned long long) * (size_t)cap + 2 * sizeof(uint32_t) * (size_t)cap +
           sizeof(uint32_t) * ((size_t)(passes + 1) * ntiles * 256 + 2 * kOsMaxPasses * 256 + kOsMaxPasses + 2 +
                               (size_t)cap / kOsGatherTile + 1 + kOrderSmallBlocks + 5 * kFinParts + 2) +
           (sizeof(unsigned long long) + sizeof(uint32_t)) * ((size_t)kFinParts * kFinBucket + kFinOverflow) + 8192;
}

OrderBufs make_order_bufs(void* scratch, uint32_t cap, int bits_a, int bits_b, int bits_job)
{
    OrderBufs O;
    O.bits_a = bits_a;
    O.bits_b = bits_b;
    O.passes = (bits_a + bits_b + bits_job + 7) / 8;
    O.ntiles_cap = (cap + kOsTile - 1) / kOsTile;
    char* p = (char*)scratch;
    auto take = [&](size_t bytes) {
        char* q = p;
        p += (bytes + 255) & ~(size_t)255;
        return (void*)q;
    };
    O.keys[0] = (unsigned long long*)take(sizeof(unsigned long long) * cap);
    O.keys[1] = (unsigned long long*)take(sizeof(unsigned long long) * cap);
    O.vals[0] = (uint32_t*)take(sizeof(uint32_t) * cap);
    O.vals[1] = (uint32_t*)take(sizeof(uint32_t) * cap);
    // fixed layout (independent of the pass count of the call): the histogram
    // must stay at the same, zeroed, address from one call to the next
    O.status = (uint32_t*)take(sizeof(uint32_t) * (size_t)(kOsMaxPasses + 1) * O.ntiles_cap * 256);
    O.gstatus = (uint32_t*)take(sizeof(uint32_t) * ((size_t)cap / kOsGatherTile + 1));
    O.hist = (uint32_t*)take(sizeof(uint32_t) * kOsMaxPasses * 256);
    O.base = (uint32_t*)take(sizeof(uint32_t) * kOsMaxPasses * 256);
    O.tile_ctr = (uint32_t*)take(sizeof(uint32_t) * (kOsMaxPasses + 2));
    O.tile_tot = (uint32_t*)take(sizeof(uint32_t) * kOrderSmallBlocks);
    O.fin = (uint32_t*)take(sizeof(uint32_t) * 2 * kFinParts);
    O.fin_off = (uint32_t*)take(sizeof(uint32_t) * (3 * kFinParts + 2));
    O.fin_bkey = (unsigned long long*)take(sizeof(unsigned long long) * kFinParts * kFinBucket);
    O.fin_bval = (uint32_t*)take(sizeof(uint32_t) * kFinParts * kFinBucket);
    O.fin_okey = (unsigned long long*)take(sizeof(unsigned long long) * kFinOverflow);
    O.fin_oval = (uint32_t*)take(sizeof(uint32_t) * kFinOverflow);
    return O;
}

cudaError_t launch_order_gather(const Bufs& b, const OrderBufs& O, bool sort, const double* segs,
                                const uint32_t* nseg, int32_t* pairs_out, uint32_t* job_out, double* segs_out,
                                int32_t* segpair_out, bool want_segments, const LaunchCfg& cfg, cudaStream_t st)
{
    const unsigned tiles = O.ntiles_cap ? O.ntiles_cap : 1u;
    OrderBufs o = O;
    if (!sort) o.passes = 0;
    k_os_hist<<<cfg.sms * 2, kOsThreads, 0, st>>>(b, o);
    note_launches(1);
    if (sort) {
        for (int p = 0; p < o.passes; p++) {
            k_os_scatter<<<tiles, kOsThreads, 0, st>>>(b, o, p);
            note_launches(1);
        }
    }
    const unsigned gtiles = O.ntiles_cap * (kOsTile / kOsGatherTile);
    k_os_gather<<<gtiles, kOsGatherTile, 0, st>>>(b, o, segs, nseg, pairs_out, job_out, segs_out, segpair_out,
                                                  want_segments ? 1 : 0, sort ? 1 : 0);
    note_launches(1);
    return cudaGetLastError();
}

// ---------------------------------------------------------------------------
// Small-count ordering (up to kOrderSmallMax results) in cooperative launches:
// one, or a rank launch and a place launch when the segments are built on
// another stream in between.
//
// At a few thousand to a few tens of thousands of results the radix passes
// above are bound by launch and look-back latency, not by bytes.  Here each of
// kOrderSmallBlocks blocks sorts one run of kOrderSmallRun keys, one key per
// thread, with a bitonic network whose partner distances below 32 are warp
// shuffles (only the longer ones go through shared memory).  The (job, a, b)
// keys are unique, so the final position of a key is its rank in its own run
// plus its lower bound in every other run: each block copies all sorted runs
// into shared memory and searches them there.  A third phase gathers the pairs
// and places the segments (block scan + the preceding runs' totals).  The
// phases are separated by grid barriers; the launch is cooperative, so all
// blocks are co-resident, and every barrier wait is bounded all the same.
// ---------------------------------------------------------------------------
constexpr int kOrderSmallThreads = kOrderSmallRun;  // one key per thread
constexpr size_t kOrderSmallDyn = sizeof(unsigned long long) * kOrderSmallMax;  // all runs, phase 2

// Arrive at grid barrier `k` (1-based) of the launch; waits bounded.  On a spent
// wait the error bit is set and later barriers of the block no longer wait.
__device__ __forceinline__ void grid_barrier(unsigned* ctr, unsigned k, unsigned* err, unsigned* s_ok)
{
    __syncthreads();
    if (threadIdx.x == 0) {
        __threadfence();
        atomicAdd(ctr, 1u);
        const unsigned target = k * gridDim.x;
        unsigned long long spins = 0;
        while (*s_ok && ld_vol(ctr) < target) {
            if (++spins > kLookbackSpins) {
                atomicOr(err, kErrTimeout);
                *s_ok = 0u;
                break;
            }
            __nanosleep(64);
        }
        __threadfence();
    }
    __syncthreads();
}

__global__ void __launch_bounds__(kOrderSmallThreads, 1)
    k_order_small(Bufs B, OrderBufs O, const double* __restrict__ segs, const uint32_t* __restrict__ nseg,
                  int32_t* pairs_out, uint32_t* job_out, double* segs_out, int32_t* segpair_out, int want_segments,
                  int sorted, unsigned phases, unsigned bar0)
{
    extern __shared__ unsigned long long allk[];  // every sorted run (phase 2)
    __shared__ unsigned long long sk[kOrderSmallRun];
    __shared__ uint32_t sv[kOrderSmallRun];
    __shared__ uint32_t sw[33];
    __shared__ unsigned s_ok, s_base;
    Counters* C = B.cnt;
    const unsigned n = res_count(B);
    if (n > kOrderSmallMax) {  // same decision in every block: no barrier is reached
        if (blockIdx.x == 0 && threadIdx.x == 0) C->order_redo = kRedoCount;
        return;
    }
    if (threadIdx.x == 0) s_ok = 1u;
    const unsigned tid = threadIdx.x;
    const unsigned nruns = (n + kOrderSmallRun - 1) / kOrderSmallRun;
    const unsigned t = blockIdx.x;
    const unsigned base = t * kOrderSmallRun;
    const unsigned len = t < nruns ? min((unsigned)kOrderSmallRun, n - base) : 0u;
    uint32_t* perm = O.vals[1];
    unsigned bar = bar0;  // grid barriers already passed by an earlier launch of this call
    if (sorted && (phases & kOrderRank)) {
        // ---- phase 1: sort this block's run (padding keys sort last) ----
        unsigned long long key = tid < len ? order_key(__ldcg(B.res + base + tid), O) : ~0ull;
        uint32_t val = tid < len ? base + tid : 0xffffffffu;
        if (len > 1) {  // uniform in the block
            for (unsigned k = 2; k <= (unsigned)kOrderSmallRun; k <<= 1)
                for (unsigned j = k >> 1; j > 0; j >>= 1) {
                    unsigned long long pk;
                    uint32_t pv;
                    if (j >= 32u) {
                        __syncthreads();  // the previous stage's reads are done
                        sk[tid] = key;
                        sv[tid] = val;
                        __syncthreads();
                        pk = sk[tid ^ j];
                        pv = sv[tid ^ j];
                    } else {
                        pk = __shfl_xor_sync(0xffffffffu, key, j);
                        pv = __shfl_xor_sync(0xffffffffu, val, j);
                    }
                    // the lower index of an ascending pair (or the upper of a
                    // descending one) keeps the smaller key
                    const bool keep_min = ((tid & j) == 0u) == ((tid & k) == 0u);
                    if (keep_min ? (pk < key) : (pk > key)) {
                        key = pk;
                        val = pv;
                    }
                }
        }
        if (tid < len) O.keys[0][base + tid] = key;
        grid_barrier(&C->obar, ++bar, &C->err, &s_ok);
        // ---- phase 2: final position = own rank + lower bounds in the other runs ----
        // all runs into shared memory: every copy is issued before any is
        // waited for (asynchronous 16-byte copies through L2 only: the key
        // buffer is rewritten by every call, so no L1 copy of it may be used;
        // an odd last key is loaded the same way, through L2)
        for (unsigned c = tid; c < n / 2u; c += kOrderSmallThreads) {
            const unsigned dst = (unsigned)__cvta_generic_to_shared(allk + 2u * c);
            asm volatile("cp.async.cg.shared.global [%0], [%1], 16;\n" ::"r"(dst), "l"(O.keys[0] + 2u * c)
                         : "memory");
        }
        if ((n & 1u) && tid == 0) allk[n - 1u] = __ldcg(O.keys[0] + (n - 1u));
        asm volatile("cp.async.wait_all;\n" ::: "memory");
        __syncthreads();
        // A warp's keys are consecutive in its sorted run, so in another run
        // their lower bounds lie between those of its first and its last key.
        // Two lanes per run find that bracket (four runs at once); every lane
        // then counts the keys below its own inside the bracket, held in the
        // warp's registers and searched with shuffles, or (a bracket wider
        // than two chunks) with its own search of the bracket.
        const unsigned lane = tid & 31u, wbase = tid & ~31u;
        if (wbase < len) {  // warp-uniform
            const unsigned wlast = min(len - wbase, 32u) - 1u;  // the warp's last key
            const unsigned long long kf = __shfl_sync(0xffffffffu, key, 0);
            const unsigned long long kl = __shfl_sync(0xffffffffu, key, wlast);
            unsigned pos = tid;
            for (unsigned s0 = 0; s0 < nruns; s0 += 4) {
                // lanes 2r and 2r + 1: lower bounds of the first and last key in run s0 + r
                unsigned a = 0, b = 0;
                if (lane < 8u) {
                    const unsigned sr = s0 + (lane >> 1);
                    if (sr < nruns && sr != t) {
                        a = sr * kOrderSmallRun;
                        b = a + min((unsigned)kOrderSmallRun, n - a);
                    }
                    const unsigned long long q = (lane & 1u) ? kl : kf;
                    while (a < b) {
                        const unsigned mid = (a + b) >> 1;
                        if (allk[mid] < q) a = mid + 1u;
                        else b = mid;
                    }
                }
#pragma unroll
                for (unsigned r = 0; r < 4u; r++) {
                    const unsigned sr = s0 + r;
                    if (sr >= nruns || sr == t) continue;  // warp-uniform
                    const unsigned L = sr * kOrderSmallRun;
                    const unsigned lo = __shfl_sync(0xffffffffu, a, 2u * r);
                    const unsigned hi = __shfl_sync(0xffffffffu, a, 2u * r + 1u);
                    unsigned c = 0;
                    if (hi - lo <= 64u) {
                        for (unsigned w0 = lo; w0 < hi; w0 += 32u) {
                            const unsigned cnt = min(32u, hi - w0);
                            const unsigned long long v = lane < cnt ? allk[w0 + lane] : ~0ull;
                            unsigned first = 0, count = cnt;  // lower bound of key among v[0 .. cnt)
                            for (int st = 0; st < 6; st++) {  // 2^5 < 32 + 1 <= 2^6
                                const unsigned half = count >> 1;
                                const unsigned long long vm = __shfl_sync(0xffffffffu, v, (first + half) & 31u);
                                if (count > 0u) {
                                    if (vm < key) {
                                        first += half + 1u;
                                        count -= half + 1u;
                                    } else {
                                        count = half;
                                    }
                                }
                            }
                            c += first;
                        }
                    } else {
                        unsigned x = lo, y = hi;
                        while (x < y) {
                            const unsigned mid = (x + y) >> 1;
                            if (allk[mid] < key) x = mid + 1u;
                            else y = mid;
                        }
                        c = x - lo;
                    }
                    pos += lo - L + c;
                }
            }
            if (lane <= wlast && pos < n) perm[pos] = val;
        }
        // the placing phase reads every block's perm entries; a separate
        // placing launch is ordered after this one by the kernel boundary
        if (phases & kOrderPlace) grid_barrier(&C->obar, ++bar, &C->err, &s_ok);
    }
    if (!(phases & kOrderPlace)) return;
    // ---- phase 3: gather pairs, place segments (one sorted position per thread) ----
    const unsigned k = base + tid;
    const bool ok = tid < len;
    unsigned src = ok ? (sorted ? __ldcg(perm + k) : k) : 0u;
    if (src >= n) src = 0u;
    const unsigned cnt = (ok && want_segments) ? __ldcg(nseg + src) : 0u;
    const uint4 rr = ok ? __ldcg(B.res + src) : make_uint4(0u, 0u, 0u, 0u);
    unsigned tot;
    const unsigned ex = block_exclusive_scan(cnt, sw, &tot);
    if (tid == 0) O.tile_tot[t] = tot;
    grid_barrier(&C->obar, ++bar, &C->err, &s_ok);
    if (tid < 32u) {
        // the preceding blocks' totals, loaded by one warp at once and summed by shuffles
        static_assert(kOrderSmallBlocks <= 32, "one warp sums the block totals");
        unsigned v = tid < t ? __ldcg(O.tile_tot + tid) : 0u;
#pragma unroll
        for (int o = 16; o > 0; o >>= 1) v += __shfl_xor_sync(0xffffffffu, v, o);
        if (tid == 0) {
            s_base = v;
            if (nruns && t == nruns - 1) C->nseg = v + tot;
        }
    }
    __syncthreads();
    if (!ok) return;
    pairs_out[2 * (size_t)k] = (int32_t)rr.y;
    pairs_out[2 * (size_t)k + 1] = (int32_t)rr.z;
    job_out[k] = rr.x;
    const unsigned off = s_base + ex;
    for (unsigned e = 0; e < cnt; e++) {
        const double2* sp = reinterpret_cast<const double2*>(segs + 18 * (size_t)src + 6 * e);
        double2* dp = reinterpret_cast<double2*>(segs_out + 6 * (size_t)(off + e));
        dp[0] = __ldcg(sp);
        dp[1] = __ldcg(sp + 1);
        dp[2] = __ldcg(sp + 2);
        segpair_out[off + e] = (int32_t)k;
    }
}

cudaError_t launch_order_small(const Bufs& b, const OrderBufs& O, bool sort, const double* segs,
                               const uint32_t* nseg, int32_t* pairs_out, uint32_t* job_out, double* segs_out,
                               int32_t* segpair_out, bool want_segments, cudaStream_t st)
{
    return launch_order_small_phases(b, O, sort, segs, nseg, pairs_out, job_out, segs_out, segpair_out,
                                     want_segments, kOrderRank | kOrderPlace, st);
}

cudaError_t launch_order_small_phases(const Bufs& b, const OrderBufs& O, bool sort, const double* segs,
                                      const uint32_t* nseg, int32_t* pairs_out, uint32_t* job_out, double* segs_out,
                                      int32_t* segpair_out, bool want_segments, unsigned phases, cudaStream_t st)
{
    if (!sort) phases &= ~kOrderRank;  // nothing to rank: results keep their order
    if (!phases) return cudaSuccess;
    const size_t dyn = (phases & kOrderRank) ? kOrderSmallDyn : 0;
    // the shared-memory opt-in is a per-device function attribute: set it once per device
    static std::atomic<uint64_t> attr_done{0};
    int dev = 0;
    cudaError_t e = cudaGetDevice(&dev);
    if (e != cudaSuccess) return e;
    const uint64_t bit = dev < 64 ? (1ull << dev) : 0ull;
    if (!bit || !(attr_done.load(std::memory_order_acquire) & bit)) {
        e = cudaFuncSetAttribute((const void*)k_order_small, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                 (int)kOrderSmallDyn);
        if (e != cudaSuccess) return e;
        attr_done.fetch_or(bit, std::memory_order_acq_rel);
    }
    Bufs bb = b;
    OrderBufs oo = O;
    const double* a_segs = segs;
    const uint32_t* a_nseg = nseg;
    int ws = want_segments ? 1 : 0, so = sort ? 1 : 0;
    // a ranking launch without the placing phase passes one grid barrier; a
    // placing launch that follows it in the same call counts its barrier after it
    unsigned ph = phases, b0 = (sort && !(phases & kOrderRank)) ? 1u : 0u;
    void* args[] = {&bb, &oo, &a_segs, &a_nseg, &pairs_out, &job_out, &segs_out, &segpair_out, &ws, &so, &ph, &b0};
    e = cudaLaunchCooperativeKernel((const void*)k_order_small, dim3(kOrderSmallBlocks), dim3(kOrderSmallThreads),
                                    args, dyn, st);
    note_launches(1);
    return e;
}

// ===========================================================================
// Post-traversal work of a call in one cooperative launch (sorted output, up to
// kFinMax results, keys of at most 63 bits):
//   phase 0  the exact stage on the escalated pairs (only when there are any:
//            the count is final at launch, so every block decides alike);
//   phase 1  one result per thread, or per two adjacent threads when the grid
//            has threads enough (each then builds one of the two endpoints),
//            results spread over all blocks: its key goes into its partition
//            (the key's top kFinPartBits bits) at the slot one atomic on the
//            partition's count returns, in a fixed bucket of kFinBucket slots
//            or, beyond it, one overflow list; then its segments, whose count
//            the partition's segment count gains;
//   barrier  the block that arrives last scans the partition counts into key
//            and segment offsets and lists the partitions over kFinBucket keys
//            before it releases the others;
//   phase 2  in a partition of up to kFinBucket keys, each result's thread
//            ranks its key against the bucket (the keys are unique, so the rank
//            is the number of smaller keys) and writes its pair, job and
//            segments at their final positions; a larger partition is one
//            block's (its bucket and its overflow entries, bitonic sort in
//            shared memory).
// Every wait is bounded.  Over kFinMax results (or more results than threads),
// a partition over kFinBig keys or a full overflow list make the kernel refuse
// (Counters::order_redo, decided alike in every block).  Launched as a
// programmatic dependent of the traversal: it waits for the traversal's grid
// (griddepcontrol.wait) before anything else.
// ===========================================================================
constexpr int kFinThreads = 256;
constexpr int kFinWarps = kFinThreads / 32;
// dynamic shared memory: a big partition's keys and values, or (in the last
// block of the key phase) the partition counts
constexpr size_t kFinDyn = (sizeof(unsigned long long) + sizeof(uint32_t)) * kFinBig > 2 * sizeof(uint32_t) * kFinParts
                               ? (sizeof(unsigned long long) + sizeof(uint32_t)) * kFinBig
                               : 2 * sizeof(uint32_t) * kFinParts;
static_assert(kFinParts % (32 * kFinWarps) == 0, "whole rows of 32 partitions per warp");
static_assert(kFinBucket % 8 == 0, "a bucket is read 8 keys at a time");
static_assert(kFinMax <= (1u << 30), "a bucket value holds the result index below bit 30");

// One result at its final position: pair and job from the key, its segments
// copied from the scratch, each segment's pair index set.
__device__ __forceinline__ void fin_place(const OrderBufs& O, const FinArgs& F, unsigned long long key, unsigned idx,
                                          unsigned pos, unsigned ns, unsigned so)
{
    // (positions stay inside the arrays even after a spent barrier wait)
    if (pos >= F.cap || (size_t)so + ns > 3 * (size_t)F.cap) return;
    const unsigned long long ma = (1ull << O.bits_a) - 1ull, mb = (1ull << O.bits_b) - 1ull;
    F.pairs_out[2 * (size_t)pos] = (int32_t)((key >> O.bits_b) & ma);
    F.pairs_out[2 * (size_t)pos + 1] = (int32_t)(key & mb);
    F.job_out[pos] = (uint32_t)(key >> (O.bits_a + O.bits_b));
    for (unsigned e = 0; e < ns; e++) {
        const double2* sp = reinterpret_cast<const double2*>(F.segs + 18 * (size_t)idx + 6 * e);
        double2* dp = reinterpret_cast<double2*>(F.segs_out + 6 * (size_t)(so + e));
        dp[0] = __ldcg(sp);
        dp[1] = __ldcg(sp + 1);
        dp[2] = __ldcg(sp + 2);
        F.segpair_out[so + e] = (int32_t)pos;
    }
}

__device__ __forceinline__ void fin_stamp(Counters* C, int k)
{
    if (blockIdx.x == 0 && threadIdx.x == 0) C->fin_ns[k] = globaltimer_ns();
}

// Block end: the last block to end stamps the launch's end.
__device__ __forceinline__ void fin_end(Counters* C)
{
    __syncthreads();
    if (threadIdx.x == 0 && atomicAdd(&C->fin_done, 1u) == gridDim.x - 1u) C->fin_ns[4] = globaltimer_ns();
}

// Layout of O.fin_off: key offsets (kFinParts + 1), segment offsets (kFinParts),
// the number of big partitions, then their ids.
constexpr int kFinSoff = kFinParts + 1;
constexpr int kFinNbig = 2 * kFinParts + 1;
constexpr int kFinBigIds = 2 * kFinParts + 2;

// Run by the block that arrives last at the phase-1 barrier: the exclusive
// scans of the partition key and segment counts into O.fin_off (one warp per
// 512 partitions, 32 at a time, coalesced), the list of partitions over
// kFinBucket keys, the counts cleared for the next call, and the refusal
// decided.  Returns the refusal code (0: none).
__device__ __forceinline__ unsigned fin_scan_counts(const OrderBufs& O, Counters* C, uint32_t* sw, unsigned* s_nbig,
                                                    uint32_t* sk)
{
    constexpr int kSeg = kFinParts / kFinWarps;  // partitions per warp
    constexpr int kIt = kSeg / 32;
    const unsigned tid = threadIdx.x, lane = tid & 31u, warp = tid >> 5;
    uint32_t* const kcount = O.fin;
    uint32_t* const scount = O.fin + kFinParts;
    uint32_t* const koff = O.fin_off;
    uint32_t* const soff = O.fin_off + kFinSoff;
    const unsigned over = ld_cg_u32(&C->fin_over);
    // all counts into shared memory first (every load in flight at once), then
    // the scan reads them there
    uint32_t* const ss = sk + kFinParts;
#pragma unroll
    for (int it = 0; it < kFinParts / kFinThreads; it++) {
        const unsigned q = it * kFinThreads + tid;
        sk[q] = __ldcg(kcount + q);
        ss[q] = __ldcg(scount + q);
    }
    __syncthreads();
    const unsigned w0 = warp * kSeg;
    uint32_t kc[kIt], sc[kIt];
#pragma unroll
    for (int it = 0; it < kIt; it++) {
        kc[it] = sk[w0 + 32 * it + lane];
        sc[it] = ss[w0 + 32 * it + lane];
    }
    uint32_t tk = 0, ts = 0;
    bool too_big = false;
#pragma unroll
    for (int it = 0; it < kIt; it++) {
        tk += kc[it];
        ts += sc[it];
        too_big |= kc[it] > (uint32_t)kFinBig;
    }
    tk = __reduce_add_sync(0xffffffffu, tk);
    ts = __reduce_add_sync(0xffffffffu, ts);
    const bool any_big = __any_sync(0xffffffffu, too_big);
    if (lane == 0) {
        sw[warp] = tk;
        sw[kFinWarps + warp] = ts;
        sw[2 * kFinWarps + warp] = any_big ? 1u : 0u;
    }
    __syncthreads();
    unsigned kb = 0, sb = 0, ktot = 0, stot = 0, refuse = 0;
#pragma unroll
    for (int w = 0; w < kFinWarps; w++) {
        const unsigned a = sw[w], b = sw[kFinWarps + w];
        if ((unsigned)w < warp) {
            kb += a;
            sb += b;
        }
        ktot += a;
        stot += b;
        refuse |= sw[2 * kFinWarps + w];
    }
#pragma unroll
    for (int it = 0; it < kIt; it++) {
        const unsigned p = w0 + 32 * it + lane;
        unsigned xk = kc[it], xs = sc[it];
#pragma unroll
        for (int o = 1; o < 32; o <<= 1) {
            const unsigned yk = __shfl_up_sync(0xffffffffu, xk, o), ys = __shfl_up_sync(0xffffffffu, xs, o);
            if (lane >= (unsigned)o) {
                xk += yk;
                xs += ys;
            }
        }
        koff[p] = kb + xk - kc[it];
        soff[p] = sb + xs - sc[it];
        kb += __shfl_sync(0xffffffffu, xk, 31);
        sb += __shfl_sync(0xffffffffu, xs, 31);
        kcount[p] = 0u;
        scount[p] = 0u;
        if (kc[it] > (uint32_t)kFinBucket) {
            const unsigned at = atomicAdd(s_nbig, 1u);
            if (at < (unsigned)kFinParts) O.fin_off[kFinBigIds + at] = p;
        }
    }
    __syncthreads();
    if (tid == 0) {
        koff[kFinParts] = ktot;
        O.fin_off[kFinNbig] = *s_nbig;
        C->nseg = stot;
    }
    if (refuse || over > (unsigned)kFinOverflow) return kRedoCrowded;
    return 0u;
}

__global__ void __launch_bounds__(kFinThreads, 2) k_finish(Bufs B, OrderBufs O, FinArgs F)
{
    wait_prior_grid();  // the traversal's results are complete and visible
    extern __shared__ unsigned long long fin_dyn[];  // a big partition: kFinBig keys, then kFinBig values
    __shared__ uint32_t sw[33];
    __shared__ unsigned s_ok, s_last, s_redo, s_fill, s_nbig;
    Counters* C = B.cnt;
    const unsigned tid = threadIdx.x, lane = tid & 31u, warp = tid >> 5;
    const unsigned gtid = blockIdx.x * kFinThreads + tid, nth = gridDim.x * kFinThreads;
    if (tid == 0) {
        s_ok = 1u;
        s_nbig = 0u;
    }
    fin_stamp(C, 0);
    if (ld_cg_u32(&C->overflow)) {  // final at launch: the call reruns with larger buffers
        fin_end(C);
        return;
    }
    // ---- phase 0: exact stage ----
    if (ld_cg_u32(&C->esc)) {
        exact_stage(B, gtid, nth);
        grid_barrier(&C->obar, 1u, &C->err, &s_ok);
        if (ld_cg_u32(&C->overflow)) {  // read after the barrier: alike in every block
            fin_end(C);
            return;
        }
    }
    fin_stamp(C, 1);
    const unsigned n = ld_cg_u32(&C->res);
    if (n > kFinMax || n > nth) {  // one result per thread at most
        if (blockIdx.x == 0 && tid == 0) C->order_redo = kRedoCount;
        fin_end(C);
        return;
    }
    // ---- phase 1: this thread's result: its key into its partition, its segments ----
    // thread slots go to the warps of different blocks first (warp w of block b
    // holds slots 32 (b + w G) ..), so that a small result spreads over every
    // SM; when there are slots enough, two adjacent slots share a result (its
    // two endpoints, FP64 work that one warp per SM sub-partition would issue
    // too slowly), the first of them owning its key
    const unsigned g = 32u * (blockIdx.x + gridDim.x * warp) + lane;
    const unsigned per = 2u * n <= nth ? 2u : 1u;
    const unsigned i = g / per, half = g % per;
    const bool mine = i < n && half == 0u;
    unsigned long long key = 0;
    unsigned p = 0, ns = 0, slot = 0;
    if (i < n) {
        const uint4 rr = __ldcg(B.res + i);
        if (mine) {
            key = order_key(rr, O);
            p = (unsigned)(key >> F.shift);
            slot = atomicAdd(O.fin + p, 1u);  // waited for after the segments
        }
        if (F.want_segments) ns = result_segments(B, rr, F.segs + 18 * (size_t)i, half, per);
    }
    if (mine) {
        if (ns) atomicAdd(O.fin + kFinParts + p, ns);
        const uint32_t v = i | (ns << 30);
        if (slot < (unsigned)kFinBucket) {
            O.fin_bkey[p * kFinBucket + slot] = key;
            O.fin_bval[p * kFinBucket + slot] = v;
        } else {
            const unsigned o = atomicAdd(&C->fin_over, 1u);
            if (o < (unsigned)kFinOverflow) {
                O.fin_okey[o] = key;
                O.fin_oval[o] = v;
            }
        }
    }
    // ---- barrier: the last block to arrive scans the counts, then releases ----
    __syncthreads();
    if (tid == 0) s_last = arrive_acq_rel(&C->fbar) == gridDim.x - 1u ? 1u : 0u;
    __syncthreads();
    if (s_last) {
        if (tid == 0) C->fin_ns[2] = globaltimer_ns();
        const unsigned r = fin_scan_counts(O, C, sw, &s_nbig, reinterpret_cast<uint32_t*>(fin_dyn));
        if (tid == 0) {
            if (r) C->order_redo = r;
            s_redo = r;
            __threadfence();
            st_release_u32(&C->frel, r ? 2u : 1u);
        }
    } else if (tid == 0) {
        unsigned v = ld_acq(&C->frel);
        unsigned long long spins = 0;
        while (v == 0u) {
            if (++spins > kLookbackSpins) {
                atomicOr(&C->err, kErrTimeout);
                v = 2u;
                break;
            }
            __nanosleep(32);
            v = ld_acq(&C->frel);
        }
        s_redo = v == 2u ? 1u : 0u;
    }
    __syncthreads();
    if (s_redo) {
        fin_end(C);
        return;
    }
    fin_stamp(C, 3);
    // ---- phase 2: each result ranks itself in its partition's bucket ----
    const uint32_t* const koff = O.fin_off;
    const uint32_t* const soff = O.fin_off + kFinSoff;
    if (mine) {
        // the offsets, the bucket's first 8 keys and the segments, all at once
        const unsigned base = __ldcg(koff + p), end = __ldcg(koff + p + 1), so = __ldcg(soff + p);
        const ulonglong2* bk2 = reinterpret_cast<const ulonglong2*>(O.fin_bkey + p * kFinBucket);
        const uint4* bv4 = reinterpret_cast<const uint4*>(O.fin_bval + p * kFinBucket);
        ulonglong2 k2[4];
        uint4 v4[2];
#pragma unroll
        for (int q = 0; q < 4; q++) k2[q] = __ldcg(bk2 + q);
        v4[0] = __ldcg(bv4);
        v4[1] = __ldcg(bv4 + 1);
        double2 sg[9];
#pragma unroll
        for (int e = 0; e < 9; e++)
            if (e < 3 * (int)ns) sg[e] = __ldcg(reinterpret_cast<const double2*>(F.segs + 18 * (size_t)i) + e);
        const unsigned m = end - base;
        if (m <= (unsigned)kFinBucket) {
            unsigned rank = 0, pre = 0;
            const unsigned long long kk[8] = {k2[0].x, k2[0].y, k2[1].x, k2[1].y, k2[2].x, k2[2].y, k2[3].x, k2[3].y};
            const uint32_t vv[8] = {v4[0].x, v4[0].y, v4[0].z, v4[0].w, v4[1].x, v4[1].y, v4[1].z, v4[1].w};
#pragma unroll
            for (int j = 0; j < 8; j++)
                if ((unsigned)j < m && kk[j] < key) {
                    rank++;
                    pre += vv[j] >> 30;
                }
            for (unsigned j = 8; j < m; j++) {
                const unsigned long long kj = __ldcg(O.fin_bkey + p * kFinBucket + j);
                if (kj < key) {
                    rank++;
                    pre += __ldcg(O.fin_bval + p * kFinBucket + j) >> 30;
                }
            }
            const unsigned pos = base + rank, s0 = so + pre;
            if (pos < F.cap && (size_t)s0 + ns <= 3 * (size_t)F.cap) {
                const unsigned long long ma = (1ull << O.bits_a) - 1ull, mb = (1ull << O.bits_b) - 1ull;
                F.pairs_out[2 * (size_t)pos] = (int32_t)((key >> O.bits_b) & ma);
                F.pairs_out[2 * (size_t)pos + 1] = (int32_t)(key & mb);
                F.job_out[pos] = (uint32_t)(key >> (O.bits_a + O.bits_b));
                double2* dp = reinterpret_cast<double2*>(F.segs_out + 6 * (size_t)s0);
#pragma unroll
                for (int e = 0; e < 9; e++)
                    if (e < 3 * (int)ns) dp[e] = sg[e];
                for (unsigned e = 0; e < ns; e++) F.segpair_out[s0 + e] = (int32_t)pos;
            }
        }
    }
    // partitions over kFinBucket keys (listed by the scan): one block each,
    // whose threads gather its bucket and its overflow entries into shared
    // memory and sort them there (bitonic)
    const unsigned nbig = min(__ldcg(O.fin_off + kFinNbig), (unsigned)kFinParts);
    unsigned long long* bk = fin_dyn;
    uint32_t* bv = reinterpret_cast<uint32_t*>(fin_dyn + kFinBig);
    for (unsigned q = blockIdx.x; q < nbig; q += gridDim.x) {
        const unsigned pb = __ldcg(O.fin_off + kFinBigIds + q);
        if (pb >= (unsigned)kFinParts) continue;  // block-uniform
        const unsigned base = __ldcg(koff + pb), m = __ldcg(koff + pb + 1) - base;
        if (m <= (unsigned)kFinBucket || m > (unsigned)kFinBig) continue;
        unsigned mp = 2u * kFinBucket;
        while (mp < m) mp <<= 1;
        __syncthreads();  // the previous partition's reads are done
        for (unsigned t = tid; t < mp; t += kFinThreads) {
            bk[t] = ~0ull;  // padding sorts last
            bv[t] = 0u;
        }
        if (tid == 0) s_fill = kFinBucket;
        __syncthreads();
        if (tid < (unsigned)kFinBucket) {
            bk[tid] = __ldcg(O.fin_bkey + pb * kFinBucket + tid);
            bv[tid] = __ldcg(O.fin_bval + pb * kFinBucket + tid);
        }
        const unsigned nover = min(ld_cg_u32(&C->fin_over), (unsigned)kFinOverflow);
        for (unsigned t = tid; t < nover; t += kFinThreads) {
            const unsigned long long kt = __ldcg(O.fin_okey + t);
            if ((unsigned)(kt >> F.shift) == pb) {
                const unsigned at = atomicAdd(&s_fill, 1u);
                if (at < mp) {
                    bk[at] = kt;
                    bv[at] = __ldcg(O.fin_oval + t);
                }
            }
        }
        __syncthreads();
        for (unsigned k = 2; k <= mp; k <<= 1)
            for (unsigned j = k >> 1; j > 0; j >>= 1) {
                for (unsigned t = tid; t < mp; t += kFinThreads) {
                    const unsigned u = t ^ j;
                    if (u > t) {
                        const unsigned long long x = bk[t], y = bk[u];
                        if ((x > y) == ((t & k) == 0u)) {
                            bk[t] = y;
                            bk[u] = x;
                            const uint32_t w = bv[t];
                            bv[t] = bv[u];
                            bv[u] = w;
                        }
                    }
                }
                __syncthreads();
            }
        unsigned run = __ldcg(soff + pb);
        for (unsigned c0 = 0; c0 < m; c0 += kFinThreads) {
            const unsigned k = c0 + tid;
            const bool have = k < m;
            const uint32_t v = have ? bv[k] : 0u;
            const unsigned nsk = v >> 30;
            unsigned idx = v & ((1u << 30) - 1u);
            if (idx >= n) idx = 0u;
            unsigned tot;
            const unsigned ex = block_exclusive_scan(nsk, sw, &tot);
            if (have) fin_place(O, F, bk[k], idx, base + k, nsk, run + ex);
            run += tot;
        }
    }
    fin_end(C);
}

cudaError_t launch_finish(const Bufs& b, const OrderBufs& O, const FinArgs& F, const LaunchCfg& cfg, cudaStream_t st,
                          bool dependent)
{
    Bufs bb = b;
    OrderBufs oo = O;
    FinArgs ff = F;
    note_launches(1);
    if (dependent) {
        // cooperative, and a programmatic dependent of the traversal launched
        // just before it on the stream: its launch overlaps the traversal's end
        cudaLaunchConfig_t lc = {};
        lc.gridDim = dim3(cfg.fin_per_sm * cfg.sms);
        lc.blockDim = dim3(kFinThreads);
        lc.dynamicSmemBytes = kFinDyn;
        lc.stream = st;
        cudaLaunchAttribute at[2];
        at[0].id = cudaLaunchAttributeCooperative;
        at[0].val.cooperative = 1;
        at[1].id = cudaLaunchAttributeProgrammaticStreamSerialization;
        at[1].val.programmaticStreamSerializationAllowed = 1;
        lc.attrs = at;
        lc.numAttrs = 2;
        const cudaError_t e = cudaLaunchKernelEx(&lc, k_finish, bb, oo, ff);
        if (e == cudaSuccess) return e;
        (void)cudaGetLastError();  // refused: launch it the plain cooperative way
    }
    void* args[] = {&bb, &oo, &ff};
    return cudaLaunchCooperativeKernel((const void*)k_finish, dim3(cfg.fin_per_sm * cfg.sms), dim3(kFinThreads), args,
                                      kFinDyn, st);
}

// ===========================================================================
// Launchers
// ===========================================================================

cudaError_t query_launch(int device, LaunchCfg* cfg)
{
    cudaDeviceProp prop;
    GI_TRY(cudaGetDeviceProperties(&prop, device));
    cfg->sms = prop.multiProcessorCount;
    int n[2][2] = {}, nl[2] = {};
    GI_TRY(cudaOccupancyMaxActiveBlocksPerMultiprocessor(&nl[0], k_traverse_levels<false>, kTravThreads, 0));
    GI_TRY(cudaOccupancyMaxActiveBlocksPerMultiprocessor(&nl[1], k_traverse_levels<true>, kTravThreads, 0));
    for (int a = 0; a < 2; a++) cfg->levels_per_sm[a] = nl[a] < 1 ? 1 : (nl[a] > 2 ? 2 : nl[a]);
    int nf = 0;
    GI_TRY(cudaOccupancyMaxActiveBlocksPerMultiprocessor(&nf, k_finish, kFinThreads, kFinDyn));
    cfg->fin_per_sm = nf < 1 ? 1 : (nf > 2 ? 2 : nf);
    GI_TRY(cudaOccupancyMaxActiveBlocksPerMultiprocessor(&n[0][0], k_traverse<false, false>, kTravThreads, 0));
    GI_TRY(cudaOccupancyMaxActiveBlocksPerMultiprocessor(&n[0][1], k_traverse<false, true>, kTravThreads, 0));
    GI_TRY(cudaOccupancyMaxActiveBlocksPerMultiprocessor(&n[1][0], k_traverse<true, false>, kTravThreads, 0));
    GI_TRY(cudaOccupancyMaxActiveBlocksPerMultiprocessor(&n[1][1], k_traverse<true, true>, kTravThreads, 0));
    for (int a = 0; a < 2; a++)
        for (int q = 0; q < 2; q++) cfg->trav_per_sm[a][q] = n[a][q] < 1 ? 1 : n[a][q];
    cfg->trav_threads = kTravThreads;
    return cudaSuccess;
}

// The persistent traversal needs no co-residency (nothing waits on a block
// that has not started); the grid is at most the resident block count so
// that every warp is live from the start.
cudaError_t launch_traverse(const Bufs& b, const LaunchCfg& cfg, int precision, TravShape shape, cudaStream_t st)
{
    note_launches(1);
    const int f64 = precision == 1 ? 1 : 0, q = shape.quad ? 1 : 0;
    if (shape.levels) {
        // cooperative: the grid barriers need every block resident.  Bit 0 of the
        // shape selects the split form: a quarter of the blocks filter candidates
        // while the other three quarters expand the levels' node pairs (pose
        // stream of two 1.3M-triangle meshes on B200: 0.1065 ms of traversal against 0.1072 with a third,
        // 0.1075-0.1083 with a fifth, more with a half)
        const int grid = cfg.levels_per_sm[f64] * cfg.sms;
        Bufs bb = b;
        bb.cand_blocks = shape.one_per_sm ? (unsigned)(grid / 4) : 0u;
        bb.publish = shape.one_per_sm ? 1u : 0u;
        bb.quad_below = shape.quad ? (unsigned)((grid - (int)bb.cand_blocks) * (kTravThreads / 32) * 8) : 0u;
        void* args[] = {&bb};
        return cudaLaunchCooperativeKernel(f64 ? (const void*)k_traverse_levels<true> : (const void*)k_traverse_levels<false>,
                                           dim3(grid), dim3(kTravThreads), args, 0, st);
    }
    const int grid = (shape.one_per_sm ? 1 : cfg.trav_per_sm[f64][q]) * cfg.sms;
    if (f64) {
        if (q) k_traverse<true, true><<<grid, kTravThreads, 0, st>>>(b);
        else k_traverse<true, false><<<grid, kTravThreads, 0, st>>>(b);
    } else {
        if (q) k_traverse<false, true><<<grid, kTravThreads, 0, st>>>(b);
        else k_traverse<false, false><<<grid, kTravThreads, 0, st>>>(b);
    }
    return cudaGetLastError();
}

cudaError_t launch_exact(const Bufs& b, const LaunchCfg& cfg, cudaStream_t st)
{
    k_exact<<<cfg.sms * 4, 128, 0, st>>>(b);
    note_launches(1);
    return cudaGetLastError();
}

cudaError_t launch_segments(const Bufs& b, double* segs, uint32_t* nseg, const LaunchCfg& cfg, cudaStream_t st)
{
    k_segments<<<cfg.sms * 8, 128, 0, st>>>(b, segs, nseg);
    note_launches(1);
    return cudaGetLastError();
}

}  // namespace gi
