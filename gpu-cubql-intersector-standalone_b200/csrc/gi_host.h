// gi_host.h -- host-side state behind the opaque handles of include/gi/gi.h
// (shared by the translation units that implement the C ABI).
#pragma once
#include <atomic>
#include <cstdio>
#include <mutex>
#include <string>
#include <vector>

#include "gi/gi.h"
#include "gi_launch.h"

using gi::Counters;
using gi::JobDev;
using gi::MeshBuffers;

struct gi_mesh {
    gi_ctx* ctx = nullptr;
    gi::MeshBuffers b;
    bool has64 = false;
};

struct gi_result {
    std::vector<int32_t> pairs;
    std::vector<double> segs;
    std::vector<int32_t> seg_pair;
    gi_stats stats;
};

struct gi_ctx {
    int device = 0;
    cudaStream_t st = nullptr;
    cudaMemPool_t pool = nullptr;  // stream-ordered allocations of this context
    gi::LaunchCfg cfg;
    uint64_t budget = 0;
    uint32_t flags = 0;
    std::atomic<uint64_t> mesh_bytes{0};
    std::string last_error;
    std::mutex mu;  // serialises device work of this context

    Counters* d_cnt = nullptr;
    Counters* h_cnt = nullptr;  // pinned
    JobDev* d_jobs = nullptr;
    JobDev* h_jobs = nullptr;  // pinned
    uint32_t cap_jobs = 0;
    uint4* queue = nullptr;
    unsigned* qflag = nullptr;
    uint32_t cap_front = 0, cap_qflag = 0;
    unsigned* cflag = nullptr;
    uint32_t cap_cflag = 0;
    unsigned tag = 0;
    uint4* cand = nullptr;
    uint32_t cap_cand = 0;
    uint4* res = nullptr;
    uint32_t cap_res = 0;
    uint4* esc = nullptr;
    uint32_t cap_esc = 0;
    // outputs
    double* segs = nullptr;  // 18 per result slot
    uint32_t* nseg = nullptr;
    int32_t* pairs_out = nullptr;
    uint32_t* job_out = nullptr;
    double* segs_out = nullptr;
    int32_t* segpair_out = nullptr;
    uint32_t cap_out = 0;
    uint64_t pred_pairs = 0, pred_segs = 0;  // result sizes of the previous call
    void* order_scratch = nullptr;
    size_t order_scratch_bytes = 0;
    // pinned staging for results
    void* h_stage = nullptr;
    size_t h_stage_bytes = 0;
    cudaEvent_t ev[8] = {};
};

inline gi_status set_err(gi_ctx* c, gi_status s, const char* what, cudaError_t e = cudaSuccess)
{
    if (c) {
        char buf[512];
        if (e != cudaSuccess)
            snprintf(buf, sizeof buf, "%s: %s (%s)", what, cudaGetErrorString(e), cudaGetErrorName(e));
        else
            snprintf(buf, sizeof buf, "%s", what);
        c->last_error = buf;
    }
    return s;
}

#define CK(ctx, x, what)                                                            \
    do {                                                                            \
        cudaError_t e_ = (x);                                                       \
        if (e_ != cudaSuccess) {                                                    \
            return set_err((ctx), e_ == cudaErrorMemoryAllocation ? GI_ERR_OOM : GI_ERR_CUDA, (what), e_); \
        }                                                                           \
    } while (0)


// pose checks and device views (gi_api.cu)
bool pose_ok(const gi_pose& p);
gi::DevPose make_dev_pose(const gi_pose& p);
gi::MeshDev mesh_dev(const gi_mesh* m);
