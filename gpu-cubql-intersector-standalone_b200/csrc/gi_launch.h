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
    uint32_t nv = 0, nt = 0, nnodes = 0, root = 0;
    size_t bytes = 0;
};

// Validates indices / coordinate domain (err bit 1: bad index, 2: out of domain).
cudaError_t launch_validate(const double* verts, uint32_t nv, const uint32_t* tris, uint32_t nt, unsigned* d_err,
                            cudaStream_t st);

// Builds the 4-wide BVH (FP32 boxes) or, with fp64 = true, the FP64 node copy.
cudaError_t build_bvh(MeshBuffers& m, bool fp64, cudaStream_t st);

// Intersect launch configuration.
struct LaunchCfg {
    int sms = 0;
    int trav_blocks = 0;  // co-resident blocks for the cooperative traversal
    int trav_threads = 256;
};
cudaError_t query_launch(int device, LaunchCfg* cfg);

// Runs traversal + first filter stage (cooperative), then the exact stage.
cudaError_t launch_traverse(const Bufs& b, const LaunchCfg& cfg, int precision, cudaStream_t st);
cudaError_t launch_exact(const Bufs& b, const LaunchCfg& cfg, cudaStream_t st);
// Segments for res[0, nres): segs[3*i .. 3*i+2], nseg[i], kind[i].
cudaError_t launch_segments(const Bufs& b, uint32_t nres, double* segs, uint32_t* nseg, const LaunchCfg& cfg,
                            cudaStream_t st);

// Output ordering for nres results: sorted pairs (int2 per pair) and the
// permutation; per-job counts.  Scratch is taken from `scratch` (bytes).
struct OrderScratch {
    void* ptr = nullptr;
    size_t bytes = 0;
};
size_t order_scratch_bytes(uint32_t nres);
size_t scan_temp_words_host(size_t n);
cudaError_t launch_order(const uint4* res, uint32_t nres, int bits_a, int bits_b, int bits_job, bool sort,
                         uint32_t* perm_out, OrderScratch scratch, cudaStream_t st);
// Gathers pairs / segments in permutation order.
cudaError_t launch_gather(const uint4* res, const uint32_t* perm, uint32_t nres, const double* segs,
                          const uint32_t* nseg, int32_t* pairs_out, uint32_t* job_out, double* segs_out,
                          int32_t* segpair_out, uint32_t* seg_offsets, uint32_t* seg_scan_temp, bool want_segments,
                          uint32_t* d_total_segs, cudaStream_t st);

// Number of kernels launched by the launchers of this library (monotonic).
unsigned long long launch_count();

// Init of the frontier: entry i = (i, rootA_i, rootB_i) from the job array.
cudaError_t launch_init_frontier(const Bufs& b, cudaStream_t st);

}  // namespace gi
