// gi_pairs.cu -- exact predicate cascade over an explicit list of candidate pairs.
//
// The reference evaluates candidate triangle pairs with a chain of kernels
// over a pair list (src/GPU_exact_predicates/OriginShiftedFloatPredicate.cu:7-26,
// DoublePredicate.cu:166-201, InexactBigIntFilter.cu, ExactBigIntPredicate.cu)
// and sends what stays undecided to CGAL on the CPU (src/CPU/YellowFilter.h:80-137).
// gi_classify_pairs does the same job on the device only: the first filter
// stage decides the general-position pairs, the rest are collected in a
// scratch list and decided exactly (FP64 filter, then integer arithmetic).
#include "gi_classify.cuh"
#include "gi_host.h"

namespace gi {

__device__ __forceinline__ unsigned pairs_warp_append(bool pred, unsigned* counter)
{
    const unsigned lane = threadIdx.x & 31;
    const unsigned m = __ballot_sync(0xffffffffu, pred);
    if (m == 0) return 0;
    const unsigned leader = __ffs(m) - 1;
    unsigned base = 0;
    if (lane == leader) base = atomicAdd(counter, (unsigned)__popc(m));
    base = __shfl_sync(0xffffffffu, base, leader);
    return base + __popc(m & ((1u << lane) - 1u));
}

__device__ __forceinline__ void pairs_load_tri(const MeshDev& M, const DevPose& P, uint32_t tri, double3* out)
{
    const uint32_t* t = M.tris + 3 * (size_t)tri;
    out[0] = world_vertex(M.verts, __ldg(t), P);
    out[1] = world_vertex(M.verts, __ldg(t + 1), P);
    out[2] = world_vertex(M.verts, __ldg(t + 2), P);
}

// scratch layout: [0] escalation count, [1] error bits, [64 ..) escalated pair indices
constexpr unsigned kPairsScratchHead = 64;

template <bool F64>
__global__ void __launch_bounds__(256) k_pairs_filter(JobDev J, const int32_t* __restrict__ pairs, uint32_t n,
                                                      uint8_t* __restrict__ out, unsigned* __restrict__ scratch)
{
    const unsigned lane = threadIdx.x & 31;
    const unsigned warp = (blockIdx.x * blockDim.x + threadIdx.x) >> 5;
    const unsigned nwarps = (gridDim.x * blockDim.x) >> 5;
    for (unsigned base = warp * 32; base < n; base += nwarps * 32) {
        const unsigned i = base + lane;
        int dec = DEC_NO;
        if (i < n) {
            const int32_t a = pairs[2 * (size_t)i], b = pairs[2 * (size_t)i + 1];
            if (a < 0 || b < 0 || (uint32_t)a >= J.A.nt || (uint32_t)b >= J.B.nt) {
                atomicOr(&scratch[1], 4u);
                out[i] = 0;
            } else {
                double3 P[3], Q[3];
                pairs_load_tri(J.A, J.pa, (uint32_t)a, P);
                pairs_load_tri(J.B, J.pb, (uint32_t)b, Q);
                if constexpr (F64) dec = classify_fast<double>(P, Q);
                else dec = classify_fast<float>(P, Q);
                out[i] = dec == DEC_YES ? 1 : 0;
            }
        }
        const bool esc = i < n && dec == DEC_ESC;
        const unsigned p = pairs_warp_append(esc, &scratch[0]);
        if (esc) scratch[kPairsScratchHead + p] = i;  // at most n escalations
    }
}

__global__ void __launch_bounds__(128) k_pairs_exact(JobDev J, const int32_t* __restrict__ pairs,
                                                     uint8_t* __restrict__ out, unsigned* __restrict__ scratch)
{
    const unsigned nesc = __ldcg(&scratch[0]);
    for (unsigned k = blockIdx.x * blockDim.x + threadIdx.x; k < nesc; k += gridDim.x * blockDim.x) {
        const unsigned i = __ldcg(&scratch[kPairsScratchHead + k]);
        double3 pts[6];
        pairs_load_tri(J.A, J.pa, (uint32_t)pairs[2 * (size_t)i], pts);
        pairs_load_tri(J.B, J.pb, (uint32_t)pairs[2 * (size_t)i + 1], pts + 3);
        ExactSigns S{&scratch[1], 0ull};
        TTRes r;
        classify_exact(pts, r, S);
        out[i] = r.kind != KIND_NONE ? 1 : 0;
    }
}

// Runs the cascade with `scratch` (kPairsScratchHead + n words, zeroed head)
// on stream st; returns the error bits through the host copy.
static cudaError_t run_pairs(const JobDev& J, const int32_t* d_pairs, uint32_t n, int precision, uint8_t* d_out,
                             unsigned* scratch, int sms, cudaStream_t st, unsigned* h_err)
{
    cudaError_t e = cudaMemsetAsync(scratch, 0, sizeof(unsigned) * 2, st);
    if (e != cudaSuccess) return e;
    if (n) {
        unsigned blocks = (n + 255) / 256;
        unsigned maxb = (unsigned)sms * 8;
        if (blocks > maxb) blocks = maxb;
        if (precision == GI_PREC_FP64) k_pairs_filter<true><<<blocks, 256, 0, st>>>(J, d_pairs, n, d_out, scratch);
        else k_pairs_filter<false><<<blocks, 256, 0, st>>>(J, d_pairs, n, d_out, scratch);
        k_pairs_exact<<<sms * 4, 128, 0, st>>>(J, d_pairs, d_out, scratch);
        note_launches(2);
        e = cudaGetLastError();
        if (e != cudaSuccess) return e;
    }
    e = cudaMemcpyAsync(h_err, scratch + 1, sizeof(unsigned), cudaMemcpyDeviceToHost, st);
    if (e != cudaSuccess) return e;
    return cudaStreamSynchronize(st);
}

static gi_status pairs_job(gi_ctx* c, const gi_mesh* A, const gi_pose* pa, const gi_mesh* B, const gi_pose* pb,
                           JobDev* J)
{
    gi_pose ia, ib;
    gi_pose_identity(&ia);
    gi_pose_identity(&ib);
    const gi_pose& PA = pa ? *pa : ia;
    const gi_pose& PB = pb ? *pb : ib;
    if (!pose_ok(PA) || !pose_ok(PB)) return set_err(c, GI_ERR_RANGE, "pose outside the supported domain");
    J->A = mesh_dev(A);
    J->B = mesh_dev(B);
    J->pa = make_dev_pose(PA);
    J->pb = make_dev_pose(PB);
    return GI_OK;
}

static gi_status pairs_status(gi_ctx* c, cudaError_t e, unsigned herr)
{
    if (e != cudaSuccess) return set_err(c, GI_ERR_CUDA, "classify pairs", e);
    if (herr & 4u) return set_err(c, GI_ERR_INVALID_ARG, "pair index out of range");
    if (herr & kErrExactCapacity) return set_err(c, GI_ERR_RANGE, "exact arithmetic capacity exceeded");
    return GI_OK;
}

}  // namespace gi

using namespace gi;

extern "C" gi_status gi_classify_pairs(gi_ctx* c, const gi_mesh* A, const gi_pose* pa, const gi_mesh* B,
                                       const gi_pose* pb, const int32_t* d_pairs, uint32_t npairs,
                                       int32_t precision_mode, uint8_t* d_out)
{
    if (!c || !A || !B || A->ctx != c || B->ctx != c || (npairs && (!d_pairs || !d_out))) return GI_ERR_INVALID_ARG;
    std::lock_guard<std::mutex> lk(c->mu);
    cudaSetDevice(c->device);
    JobDev J;
    gi_status s = pairs_job(c, A, pa, B, pb, &J);
    if (s != GI_OK) return s;
    unsigned* scratch = nullptr;
    cudaError_t e = pool_alloc(&scratch, sizeof(unsigned) * (kPairsScratchHead + (size_t)npairs), c->pool, c->st);
    if (e != cudaSuccess) return set_err(c, GI_ERR_OOM, "classify pairs scratch", e);
    unsigned herr = 0;
    e = run_pairs(J, d_pairs, npairs, precision_mode, d_out, scratch, c->cfg.sms, c->st, &herr);
    cudaFreeAsync(scratch, c->st);
    return pairs_status(c, e, herr);
}

// ---------------------------------------------------------------------------
// gi_classify_pairs_noalloc: the same cascade with scratch that is never
// allocated at call time.
//
// Some callers cannot allocate device memory while they run: a pose-update
// control loop that reserved its whole memory budget at start-up and must not
// grow a pool afterwards, a host framework whose caching allocator already owns
// the free HBM, or a latency-bound loop that cannot take the stall of a pool
// growing or trimming on its stream.  For them the escalation list lives in one
// fixed array in the module's device memory instead of the context's pool.
//
// Limits and rules:
//  * at most GI_NOALLOC_MAX_PAIRS pairs per call; more is rejected with
//    GI_ERR_CAPACITY before any work is queued;
//  * the array is one per device, shared by every context on that device, so
//    calls whose device work overlaps in time (two threads, or two contexts, on
//    the same device at once) race on it and their results are undefined.
//    A call blocks until its work is done, so calls made one after another
//    from the host are safe;
//  * the first call on a device looks up the array's device address (with that
//    device current) and keeps it; make that first call before any stream
//    capture begins.
//  * the two head words (escalation count, error bits) must start at zero;
//    each call clears them on its stream with a memset before the kernels.
constexpr uint32_t kNoAllocMaxPairs = GI_NOALLOC_MAX_PAIRS;
static_assert(kNoAllocMaxPairs == (1u << 20), "header limit and scratch size disagree");
static __device__ __align__(256) unsigned g_pairs_scratch[kPairsScratchHead + kNoAllocMaxPairs];  // 4 MiB + 256 B

constexpr int kNoAllocMaxDevices = 64;
static std::mutex g_noalloc_mu;
static unsigned* g_noalloc_ptr[kNoAllocMaxDevices] = {};

// Device address of g_pairs_scratch on c->device (which must be current).
static gi_status noalloc_scratch(gi_ctx* c, unsigned** out)
{
    if (c->device < 0 || c->device >= kNoAllocMaxDevices)
        return set_err(c, GI_ERR_INVALID_ARG, "device ordinal beyond the no-alloc scratch table");
    std::lock_guard<std::mutex> lk(g_noalloc_mu);
    if (!g_noalloc_ptr[c->device]) {
        unsigned* ptr = nullptr;
        cudaError_t e = cudaGetSymbolAddress((void**)&ptr, g_pairs_scratch);
        if (e != cudaSuccess || !ptr) return set_err(c, GI_ERR_CUDA, "no-alloc scratch symbol address", e);
        g_noalloc_ptr[c->device] = ptr;
    }
    *out = g_noalloc_ptr[c->device];
    return GI_OK;
}

extern "C" gi_status gi_classify_pairs_noalloc(gi_ctx* c, const gi_mesh* A, const gi_pose* pa, const gi_mesh* B,
                                               const gi_pose* pb, const int32_t* d_pairs, uint32_t npairs,
                                               int32_t precision_mode, uint8_t* d_out)
{
    if (!c || !A || !B || A->ctx != c || B->ctx != c || (npairs && (!d_pairs || !d_out))) return GI_ERR_INVALID_ARG;
    std::lock_guard<std::mutex> lk(c->mu);
    if (npairs > kNoAllocMaxPairs)
        return set_err(c, GI_ERR_CAPACITY, "npairs exceeds the fixed scratch of gi_classify_pairs_noalloc "
                                           "(at most GI_NOALLOC_MAX_PAIRS = 1048576 pairs per call)");
    cudaError_t e = cudaSetDevice(c->device);
    if (e != cudaSuccess) return set_err(c, GI_ERR_CUDA, "set device", e);
    JobDev J;
    gi_status s = pairs_job(c, A, pa, B, pb, &J);
    if (s != GI_OK) return s;
    unsigned* scratch = nullptr;
    s = noalloc_scratch(c, &scratch);
    if (s != GI_OK) return s;
    unsigned herr = 0;
    e = run_pairs(J, d_pairs, npairs, precision_mode, d_out, scratch, c->cfg.sms, c->st, &herr);
    return pairs_status(c, e, herr);
}
