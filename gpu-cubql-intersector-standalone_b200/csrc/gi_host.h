// gi_host.h -- host-side state behind the opaque handles of include/gi/gi.h
// (shared by the translation units that implement the C ABI).
#pragma once
#include <atomic>
#include <condition_variable>
#include <cstdio>
#include <cstring>
#include <deque>
#include <map>
#include <memory>
#include <mutex>
#include <string>
#include <thread>
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
    double build_ms = 0.0;  // device time of validation + BVH build (CUDA events on the build stream)
};

// Pinned host blocks that results are copied into.  A call takes one block
// from its context's pool; the results of that call point into it (no further
// copy) and the block goes back to the pool when the last of them is freed,
// even after the context itself is gone.
// Host threads that split large memcpys into parts; the calling thread works
// on its own job too.  Several callers may copy at once (the two meshes of a
// one-shot call): each job is queued, helpers take its parts in turn.
class CopyPool {
public:
    explicit CopyPool(unsigned helpers)
    {
        for (unsigned i = 0; i < helpers; i++) th_.emplace_back([this] { work(); });
    }
    ~CopyPool()
    {
        {
            std::lock_guard<std::mutex> lk(mu_);
            stop_ = true;
        }
        cv_.notify_all();
        for (auto& t : th_) t.join();
    }
    CopyPool(const CopyPool&) = delete;
    CopyPool& operator=(const CopyPool&) = delete;

    void copy(void* dst, const void* src, size_t bytes)
    {
        constexpr size_t kPart = (size_t)1 << 20;
        Job j{static_cast<char*>(dst), static_cast<const char*>(src), bytes, kPart, (unsigned)((bytes + kPart - 1) / kPart)};
        if (j.parts <= 1 || th_.empty()) {
            std::memcpy(dst, src, bytes);
            return;
        }
        {
            std::lock_guard<std::mutex> lk(mu_);
            q_.push_back(&j);
        }
        cv_.notify_all();
        // the caller takes parts as well
        for (;;) {
            unsigned part;
            {
                std::lock_guard<std::mutex> lk(mu_);
                if (j.next >= j.parts) break;
                part = claim(&j);
            }
            run(&j, part);
            std::lock_guard<std::mutex> lk(mu_);
            j.done++;
        }
        std::unique_lock<std::mutex> lk(mu_);
        done_.wait(lk, [&] { return j.done == j.parts; });
    }

private:
    struct Job {
        char* dst;
        const char* src;
        size_t bytes, part_bytes;
        unsigned parts;
        unsigned next = 0, done = 0;  // guarded by mu_
    };
    // takes the next part of j (mu_ held); the job leaves the queue with its last part
    unsigned claim(Job* j)
    {
        const unsigned part = j->next++;
        if (j->next == j->parts)
            for (auto it = q_.begin(); it != q_.end(); ++it)
                if (*it == j) {
                    q_.erase(it);
                    break;
                }
        return part;
    }
    static void run(Job* j, unsigned part)
    {
        const size_t off = (size_t)part * j->part_bytes;
        const size_t n = j->bytes - off < j->part_bytes ? j->bytes - off : j->part_bytes;
        std::memcpy(j->dst + off, j->src + off, n);
    }
    void work()
    {
        for (;;) {
            Job* j;
            unsigned part;
            {
                std::unique_lock<std::mutex> lk(mu_);
                cv_.wait(lk, [&] { return stop_ || !q_.empty(); });
                if (stop_) return;
                j = q_.front();
                part = claim(j);
            }
            run(j, part);
            {
                // the job is not touched after this: its owner returns once done == parts
                std::lock_guard<std::mutex> lk(mu_);
                j->done++;
            }
            done_.notify_all();
        }
    }
    std::mutex mu_;
    std::condition_variable cv_, done_;
    std::deque<Job*> q_;
    std::vector<std::thread> th_;
    bool stop_ = false;
};

// Pinned chunks through which pageable host arrays are copied to the device:
// helpers fill one chunk while the DMA of the other runs.
struct Staging {
    static constexpr size_t kChunk = (size_t)4 << 20;
    void* buf[2] = {nullptr, nullptr};
    cudaEvent_t ev[2] = {nullptr, nullptr};
    bool ready = false;
    cudaError_t init()
    {
        if (ready) return cudaSuccess;
        for (int i = 0; i < 2; i++) {
            cudaError_t e = cudaMallocHost(&buf[i], kChunk);
            if (e == cudaSuccess) e = cudaEventCreateWithFlags(&ev[i], cudaEventDisableTiming);
            if (e != cudaSuccess) return e;
        }
        ready = true;
        return cudaSuccess;
    }
    void release()
    {
        for (int i = 0; i < 2; i++) {
            if (ev[i]) cudaEventSynchronize(ev[i]), cudaEventDestroy(ev[i]);
            if (buf[i]) cudaFreeHost(buf[i]);
            ev[i] = nullptr;
            buf[i] = nullptr;
        }
        ready = false;
    }
};

struct PinnedPool;
struct PinnedBuf {
    void* p = nullptr;
    size_t bytes = 0;
    std::atomic<int> refs{0};
    std::shared_ptr<PinnedPool> home;  // set while results hold the block
};
struct PinnedPool {
    std::mutex mu;
    std::vector<PinnedBuf*> free_list;
    size_t free_bytes = 0;
    // free blocks kept for reuse up to this many bytes; beyond it the smallest
    // are released.  Pinning and unpinning cost milliseconds and cudaFreeHost
    // waits for the device, so a serving loop whose round sizes vary must not
    // release and allocate blocks on every round.
    static constexpr size_t kKeepFreeBytes = (size_t)512 << 20;
    ~PinnedPool()
    {
        for (PinnedBuf* b : free_list) {
            cudaFreeHost(b->p);
            delete b;
        }
    }
    // smallest free block of at least `bytes`, or a new one (nullptr: out of pinned memory)
    PinnedBuf* get(size_t bytes)
    {
        {
            std::lock_guard<std::mutex> lk(mu);
            size_t best = free_list.size();
            for (size_t i = 0; i < free_list.size(); i++)
                if (free_list[i]->bytes >= bytes && (best == free_list.size() || free_list[i]->bytes < free_list[best]->bytes))
                    best = i;
            if (best != free_list.size()) {
                PinnedBuf* b = free_list[best];
                free_list.erase(free_list.begin() + (long)best);
                free_bytes -= b->bytes;
                return b;
            }
        }
        PinnedBuf* b = new (std::nothrow) PinnedBuf();
        if (!b) return nullptr;
        // power-of-two sizes (at least 1 MB) with at least half the request as
        // headroom: a block serves later results of similar or somewhat larger
        // size, so a result that grows a little does not pin a new block (pinning
        // takes milliseconds) in the middle of a pose stream
        size_t want = (size_t)1 << 20;
        while (want < bytes + bytes / 2) want <<= 1;
        if (cudaMallocHost(&b->p, want) != cudaSuccess) {
            delete b;
            return nullptr;
        }
        b->bytes = want;
        return b;
    }
    void put(PinnedBuf* b)
    {
        std::vector<PinnedBuf*> drop;
        {
            std::lock_guard<std::mutex> lk(mu);
            free_list.push_back(b);
            free_bytes += b->bytes;
            while (free_bytes > kKeepFreeBytes && free_list.size() > 1) {  // release the smallest
                size_t k = 0;
                for (size_t i = 1; i < free_list.size(); i++)
                    if (free_list[i]->bytes < free_list[k]->bytes) k = i;
                free_bytes -= free_list[k]->bytes;
                drop.push_back(free_list[k]);
                free_list.erase(free_list.begin() + (long)k);
            }
        }
        for (PinnedBuf* d : drop) {
            cudaFreeHost(d->p);
            delete d;
        }
    }
};
// Drops one result's hold on a block (the block returns to its pool at zero).
inline void pinned_release(PinnedBuf* b)
{
    if (!b || b->refs.fetch_sub(1) != 1) return;
    std::shared_ptr<PinnedPool> pool = std::move(b->home);
    if (pool) pool->put(b);
    else {
        cudaFreeHost(b->p);
        delete b;
    }
}

struct gi_result {
    PinnedBuf* buf = nullptr;  // storage of the arrays below (shared by the results of one call)
    const int32_t* pairs = nullptr;
    uint64_t npairs = 0;
    const double* segs = nullptr;
    const int32_t* seg_pair = nullptr;
    uint64_t nsegs = 0;
    gi_stats stats;
};

// Traversal autotuner: per workload class (precision, number of jobs, total
// triangles in factors of 4), each traversal shape is timed on the context's
// own calls (the best of kTries traversals, CUDA events on the context's
// stream); a shape whose first time is over 1.3x the best so far is not tried
// again.  After that the fastest shape is used.  Every shape gives the same
// result.
struct TravTuner {
    static constexpr int kTries = 2;
    struct Entry {
        float best[gi::kTravShapes];
        int tries[gi::kTravShapes];
        int choice = -1;
        Entry()
        {
            for (int k = 0; k < gi::kTravShapes; k++) {
                best[k] = 3.0e38f;
                tries[k] = 0;
            }
        }
    };
    std::map<uint32_t, Entry> table;
    static uint32_t key(int precision, uint32_t njobs, uint64_t tris)
    {
        const uint32_t jc = njobs <= 1 ? 0u : njobs < 16 ? 1u : njobs < 256 ? 2u : 3u;
        uint32_t lg = 0;
        while (lg < 20 && (4ull << (2 * lg)) <= tris) lg++;
        return (uint32_t)(precision & 1) | (jc << 1) | (lg << 3);
    }
    int pick(uint32_t k)
    {
        Entry& e = table[k];
        if (e.choice >= 0) return e.choice;
        for (int s = 0; s < gi::kTravShapes; s++)
            if (e.tries[s] < kTries) return s;
        int b = 0;
        for (int s = 1; s < gi::kTravShapes; s++)
            if (e.best[s] < e.best[b]) b = s;
        e.choice = b;
        return b;
    }
    void report(uint32_t k, int s, float ms)
    {
        Entry& e = table[k];
        if (e.choice >= 0 || s < 0 || s >= gi::kTravShapes) return;
        e.tries[s]++;
        if (ms < e.best[s]) e.best[s] = ms;
        float lead = 3.0e38f;
        for (int q = 0; q < gi::kTravShapes; q++)
            if (q != s && e.tries[q] > 0) lead = lead < e.best[q] ? lead : e.best[q];
        if (e.tries[s] == 1 && ms > 1.3f * lead) e.tries[s] = kTries;  // clearly slower: one try is enough
    }
};

struct gi_ctx {
    int device = 0;
    cudaStream_t st = nullptr;
    cudaStream_t st2 = nullptr;  // second mesh of a one-shot call builds here, concurrently with the first
    std::unique_ptr<CopyPool> copy_pool;  // created with the first staged upload
    std::once_flag copy_pool_once;
    Staging stage[2];                     // per upload stream (st, st2)
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
    uint32_t fin_backoff = 0;  // calls left before the one-launch finish is tried again after a refusal
    void* order_scratch = nullptr;
    size_t order_scratch_bytes = 0;
    // pinned blocks the results are copied into
    std::shared_ptr<PinnedPool> pinned = std::make_shared<PinnedPool>();
    TravTuner tuner;
    int fixed_shape = -1;  // >= 0: traversal shape forced (tests), else tuned
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
