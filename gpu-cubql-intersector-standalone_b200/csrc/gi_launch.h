// gi_launch.h -- host-side launchers of the kernels in gi_kernels.cu.
#pragma once
#include <cstdint>
#include <cuda_runtime.h>

#include "gi_internal.cuh"

namespace gi {

// Device arrays owned by one resident mesh.
struct MeshBuffers {
    double* verts = nullptr;
    uint32_t* tris = nullptr;
    uint4* leafTri = nullptr;
    float* leafBox = nullptr;
    WNode* nodes = nullptr;
    double* leafBox64 = nullptr;
    WNode64* nodes64 = nullptr;
    uint32_t* cutRef = nullptr;
    uint32_t* ncuts = nullptr;  // device: sizes of the depth-3 and depth-4 cuts
    float* cutBox = nullptr;
    double* cutBox64 = nullptr;
    uint32_t nv = 0, nt = 0, nnodes = 0, root = 0;
    size_t bytes = 0;
};

// Stream-ordered allocation from the context's own pool (the device's default
// pool when none is given).
inline cudaError_t pool_alloc(void** p, size_t bytes, cudaMemPool_t pool, cudaStream_t st)
{
    return pool ? cudaMallocFromPoolAsync(p, bytes, pool, st) : cudaMallocAsync(p, bytes, st);
}
template <class T>
inline cudaError_t pool_alloc(T** p, size_t bytes, cudaMemPool_t pool, cudaStream_t st)
{
    return pool_alloc(reinterpret_cast<void**>(p), bytes, pool, st);
}

// Validates indices / coordinate domain (err bit 1: bad index, 2: out of domain).
cudaError_t launch_validate(const double* verts, uint32_t nv, const uint32_t* tris, uint32_t nt, unsigned* d_err,
                            cudaStream_t st);

// Builds the 4-wide BVH (FP32 boxes) or, with fp64 = true, the FP64 node copy.
// d_err: a device word (required); bit 2 (4u) is set if the wide tree came out
// inconsistent (not expected; the kernels then skip the bad links).
cudaError_t build_bvh(MeshBuffers& m, bool fp64, unsigned* d_err, cudaMemPool_t pool, cudaStream_t st);

// Intersect launch configuration.
struct LaunchCfg {
    int sms = 0;
    int trav_per_sm[2][2] = {};  // resident traversal blocks per SM, [FP64][quad form]
    int levels_per_sm[2] = {};   // resident blocks of the level-synchronous traversal (at most 2), [FP64]
    int fin_per_sm = 1;          // resident blocks of the post-traversal launch (at most 2)
    int trav_threads = 256;
};

// Traversal shapes the tuner chooses from: the work-queue traversal or the
// level-synchronous one (bit 2); expansion form (bit 1: one node pair per quad
// of lanes; for the level-synchronous traversal, the quad form on levels of at
// most 8 node pairs per warp); bit 0: the work-queue traversal with one block
// per SM (else all resident), the level-synchronous one in its split form
// (a quarter of the blocks only filter candidates).
struct TravShape {
    bool quad = false;
    bool one_per_sm = false;
    bool levels = false;
};
constexpr int kTravShapes = 8;
inline TravShape trav_shape(int k)
{
    TravShape t;
    t.quad = (k & 2) != 0;
    t.one_per_sm = (k & 1) != 0;
    t.levels = (k & 4) != 0;
    return t;
}
cudaError_t query_launch(int device, LaunchCfg* cfg);

// Traversal + first filter stage (persistent, work queue), then the exact stage.
cudaError_t launch_traverse(const Bufs& b, const LaunchCfg& cfg, int precision, TravShape shape, cudaStream_t st);
cudaError_t launch_exact(const Bufs& b, const LaunchCfg& cfg, cudaStream_t st);
// Segments of every result (count from the device counters):
// segs[18*i ..] (up to 3 segments), nseg[i].
cudaError_t launch_segments(const Bufs& b, double* segs, uint32_t* nseg, const LaunchCfg& cfg, cudaStream_t st);

// Output ordering (radix sort by (job, a, b), sizes from the device counters)
// and the gather of pairs / jobs / segments in that order.
constexpr int kOsMaxPasses = 8;
struct OrderBufs {
    unsigned long long* keys[2];
    uint32_t* vals[2];
    uint32_t* status;    // look-back status: (passes + 1) x ntiles_cap x 256
    uint32_t* gstatus;   // look-back status of the gather tiles
    uint32_t* hist;      // kOsMaxPasses x 256 (kept zero between calls)
    uint32_t* base;      // kOsMaxPasses x 256
    uint32_t* tile_ctr;  // kOsMaxPasses + 2 (per pass, the gather, the histogram blocks)
    uint32_t* tile_tot;  // kOrderSmallBlocks: segment totals per run (small-count path)
    // one-launch finish (k_finish)
    uint32_t* fin;       // 2 x kFinParts: keys and segments per partition (zero between calls)
    uint32_t* fin_off;   // kFinParts + 1 key offsets, kFinParts segment offsets, the number of
                         // partitions over kFinBucket keys, their ids (kFinParts at most)
    unsigned long long* fin_bkey;  // kFinParts x kFinBucket: each partition's first keys
    uint32_t* fin_bval;            // ... and their result index | segment count << 30
    unsigned long long* fin_okey;  // kFinOverflow: the keys beyond a bucket
    uint32_t* fin_oval;
    uint32_t ntiles_cap;
    int passes;
    int bits_a, bits_b;
};
size_t order_scratch_bytes(uint32_t cap, int passes);
OrderBufs make_order_bufs(void* scratch, uint32_t cap, int bits_a, int bits_b, int bits_job);
cudaError_t launch_order_gather(const Bufs& b, const OrderBufs& O, bool sort, const double* segs,
                                const uint32_t* nseg, int32_t* pairs_out, uint32_t* job_out, double* segs_out,
                                int32_t* segpair_out, bool want_segments, const LaunchCfg& cfg, cudaStream_t st);
// Small-count ordering: a cooperative launch of kOrderSmallBlocks blocks,
// each sorting a run of kOrderSmallRun keys, for up to kOrderSmallMax results.
// If the call produced more, the kernel only sets Counters::order_redo and the
// caller reruns with launch_order_gather.  Keys must fit in 63 bits.
constexpr int kOrderSmallRun = 1024;
constexpr int kOrderSmallBlocks = 24;
constexpr uint32_t kOrderSmallMax = (uint32_t)kOrderSmallRun * kOrderSmallBlocks;
cudaError_t launch_order_small(const Bufs& b, const OrderBufs& O, bool sort, const double* segs,
                               const uint32_t* nseg, int32_t* pairs_out, uint32_t* job_out, double* segs_out,
                               int32_t* segpair_out, bool want_segments, cudaStream_t st);
// The same in two launches: kOrderRank (sort the runs, rank every key) needs
// only the final result list; kOrderPlace (gather the pairs, place the
// segments) needs the segments too, so the ranking can run while the segments
// are built on another stream.
constexpr unsigned kOrderRank = 1u, kOrderPlace = 2u;
cudaError_t launch_order_small_phases(const Bufs& b, const OrderBufs& O, bool sort, const double* segs,
                                      const uint32_t* nseg, int32_t* pairs_out, uint32_t* job_out, double* segs_out,
                                      int32_t* segpair_out, bool want_segments, unsigned phases, cudaStream_t st);
// Everything after the traversal in one cooperative launch, for sorted output
// of up to kFinMax results with keys of at most 63 bits: the exact stage (when
// pairs were escalated), the segments, and the ordering by partitions of the
// key's top kFinPartBits bits (one warp ranks a partition of up to kFinBucket
// keys, one block a larger one, up to kFinBig).  A call over those limits
// makes the kernel set only Counters::order_redo; the caller then reruns on
// the general path (launch_exact, launch_segments, launch_order_gather).
constexpr int kFinPartBits = 12;
constexpr int kFinParts = 1 << kFinPartBits;
constexpr int kFinBucket = 32;
constexpr int kFinOverflow = 1 << 14;
constexpr int kFinBig = 2048;
constexpr uint32_t kFinMax = 1u << 16;
struct FinArgs {
    double* segs;       // per result: up to 3 segments (scratch)
    int32_t* pairs_out;
    uint32_t* job_out;
    double* segs_out;
    int32_t* segpair_out;
    uint32_t cap;       // results the output arrays hold (segments: 3 per result)
    int want_segments;
    int shift;          // partition of a key = key >> shift
};
// dependent: launched right after the traversal on the same stream, with no
// other stream work between them (programmatic dependent launch)
cudaError_t launch_finish(const Bufs& b, const OrderBufs& O, const FinArgs& F, const LaunchCfg& cfg, cudaStream_t st,
                          bool dependent = false);

// Number of kernels launched by the launchers of this library (monotonic).
unsigned long long launch_count();
void note_launches(unsigned n);


}  // namespace gi
