// gi_api.cu -- C ABI (include/gi/gi.h) over the kernels in gi_kernels.cu.
//
// Host flow of gi_intersect (replaces KernelBVHController::runIntersectionPipeline,
// src/GPUIntersector/KernelBVHController.cu:603-699 in the reference, whose chunk
// loop syncs and copies to the host several times per chunk and calls CGAL on
// the CPU for undecided pairs):
//   counters reset -> frontier init -> k_traverse (cooperative) -> k_exact
//   -> one counters read-back (capacity check; buffers grow x4 and the call is
//      re-run on overflow) -> k_segments -> ordering -> copies to the host.
// No CPU fallback exists: every pair is decided on the device.
#include <algorithm>
#include <atomic>
#include <chrono>
#include <cmath>
#include <condition_variable>
#include <cstdio>
#include <cstring>
#include <deque>
#include <map>
#include <mutex>
#include <new>
#include <string>
#include <thread>
#include <vector>

#include "gi_host.h"

using namespace gi;

extern "C" const char* gi_status_string(gi_status s)
{
    switch (s) {
        case GI_OK: return "ok";
        case GI_ERR_INVALID_ARG: return "invalid argument";
        case GI_ERR_OOM: return "out of memory";
        case GI_ERR_CAPACITY: return "capacity exceeded";
        case GI_ERR_TIMEOUT: return "device wait timed out";
        case GI_ERR_CUDA: return "CUDA error";
        case GI_ERR_RANGE: return "coordinates outside the supported domain";
        case GI_ERR_NOT_READY: return "not ready";
        case GI_ERR_NO_DEVICE: return "no CUDA device";
    }
    return "unknown status";
}

extern "C" const char* gi_last_error(const gi_ctx* ctx)
{
    return ctx ? ctx->last_error.c_str() : "";
}

extern "C" gi_status gi_device_count(int32_t* n)
{
    if (!n) return GI_ERR_INVALID_ARG;
    int c = 0;
    cudaError_t e = cudaGetDeviceCount(&c);
    if (e != cudaSuccess) {
        *n = 0;
        return GI_ERR_NO_DEVICE;
    }
    *n = c;
    return GI_OK;
}

template <class T>
static cudaError_t grow(T*& p, uint32_t& cap, uint32_t need, cudaMemPool_t pool, cudaStream_t st)
{
    if (need <= cap && p) return cudaSuccess;
    if (p) cudaFreeAsync(p, st);
    p = nullptr;
    cudaError_t e = pool_alloc(&p, sizeof(T) * (size_t)need, pool, st);
    if (e == cudaSuccess) cap = need;
    else cap = 0;
    return e;
}

extern "C" gi_status gi_create(const gi_options* opts, gi_ctx** out)
{
    if (!out) return GI_ERR_INVALID_ARG;
    *out = nullptr;
    int ndev = 0;
    if (cudaGetDeviceCount(&ndev) != cudaSuccess || ndev == 0) return GI_ERR_NO_DEVICE;
    gi_ctx* c = new (std::nothrow) gi_ctx();
    if (!c) return GI_ERR_OOM;
    c->device = opts ? opts->device : 0;
    c->budget = opts ? opts->hbm_budget_bytes : 0;
    c->flags = opts ? opts->flags : 0;
    if (c->flags & GI_FLAG_FIXED_SHAPE) c->fixed_shape = (int)((c->flags >> 9) & 7u);
    if (c->device < 0 || c->device >= ndev) {
        delete c;
        return GI_ERR_INVALID_ARG;
    }
    cudaSetDevice(c->device);
    cudaError_t e = cudaStreamCreateWithFlags(&c->st, cudaStreamNonBlocking);
    if (e == cudaSuccess) e = cudaStreamCreateWithFlags(&c->st2, cudaStreamNonBlocking);
    if (e == cudaSuccess) {
        // the context's own stream-ordered pool: memory freed by one call (a
        // released mesh, a grown buffer) is reused by the next without being
        // unmapped and mapped again, up to the release threshold
        cudaMemPoolProps pp = {};
        pp.allocType = cudaMemAllocationTypePinned;
        pp.location.type = cudaMemLocationTypeDevice;
        pp.location.id = c->device;
        e = cudaMemPoolCreate(&c->pool, &pp);
        if (e == cudaSuccess) {
            uint64_t keep = c->budget ? c->budget : (16ull << 30);
            e = cudaMemPoolSetAttribute(c->pool, cudaMemPoolAttrReleaseThreshold, &keep);
        }
    }
    if (e == cudaSuccess) e = query_launch(c->device, &c->cfg);
    if (e == cudaSuccess) e = cudaMalloc(&c->d_cnt, sizeof(Counters));
    if (e == cudaSuccess) e = cudaMallocHost(&c->h_cnt, sizeof(Counters));
    for (int i = 0; i < 8 && e == cudaSuccess; i++) e = cudaEventCreate(&c->ev[i]);
    if (e != cudaSuccess) {
        gi_destroy(c);
        return e == cudaErrorMemoryAllocation ? GI_ERR_OOM : GI_ERR_NO_DEVICE;
    }
    *out = c;
    return GI_OK;
}

extern "C" gi_status gi_destroy(gi_ctx* c)
{
    if (!c) return GI_ERR_INVALID_ARG;
    cudaSetDevice(c->device);
    if (c->st) cudaStreamSynchronize(c->st);
    if (c->st2) cudaStreamSynchronize(c->st2);
    for (auto& sg : c->stage) sg.release();
    c->copy_pool.reset();
    if (c->d_cnt) cudaFree(c->d_cnt);
    if (c->d_jobs) cudaFree(c->d_jobs);
    void* pooled[] = {c->queue, c->qflag,     c->cand,         c->cflag,   c->res,
                      c->esc,   c->segs,      c->nseg,         c->pairs_out, c->job_out,
                      c->segs_out, c->segpair_out, c->order_scratch};
    for (void* p : pooled)
        if (p) cudaFreeAsync(p, c->st);
    if (c->st) cudaStreamSynchronize(c->st);
    if (c->pool) cudaMemPoolDestroy(c->pool);
    if (c->h_cnt) cudaFreeHost(c->h_cnt);
    if (c->h_jobs) cudaFreeHost(c->h_jobs);
    for (auto& e : c->ev)
        if (e) cudaEventDestroy(e);
    if (c->st) cudaStreamDestroy(c->st);
    if (c->st2) cudaStreamDestroy(c->st2);
    delete c;
    return GI_OK;
}

// ---------------------------------------------------------------------------
// Meshes
// ---------------------------------------------------------------------------
static void mesh_free(gi_ctx* c, gi_mesh* m, cudaStream_t st);

// Mesh uploads run on a given stream and report errors to a given sink, so
// that the two meshes of a one-shot call can be built from two host threads.
struct UploadSink {
    gi_ctx* c;
    std::string* msg;  // nullptr: the context's last error
    gi_status fail(gi_status s, const char* what, cudaError_t e = cudaSuccess) const
    {
        if (!msg) return set_err(c, s, what, e);
        char buf[512];
        if (e != cudaSuccess)
            snprintf(buf, sizeof buf, "%s: %s (%s)", what, cudaGetErrorString(e), cudaGetErrorName(e));
        else
            snprintf(buf, sizeof buf, "%s", what);
        *msg = buf;
        return s;
    }
    gi_status cuda(cudaError_t e, const char* what) const
    {
        return fail(e == cudaErrorMemoryAllocation ? GI_ERR_OOM : GI_ERR_CUDA, what, e);
    }
};

#define CKS(sink, x, what)                          \
    do {                                            \
        cudaError_t e_ = (x);                       \
        if (e_ != cudaSuccess) return (sink).cuda(e_, (what)); \
    } while (0)

static gi_status mesh_finish(gi_ctx* c, gi_mesh* m, gi_mesh** out, cudaStream_t st, const UploadSink& sk)
{
    // The validation result is read back with the build's last synchronisation,
    // not before it: the build reads vertex indices clamped to the array, so an
    // invalid mesh costs a wasted build but no out-of-bounds access.
    unsigned* d_err = nullptr;
    CKS(sk, pool_alloc(&d_err, sizeof(unsigned), c->pool, st), "alloc");
    CKS(sk, cudaMemsetAsync(d_err, 0, sizeof(unsigned), st), "memset");
    // device time of validation + build (the reference's buildRefitMesh*Ms);
    // events of this call only, as two meshes may build at once on two streams
    cudaEvent_t eb[2] = {nullptr, nullptr};
    bool timed = cudaEventCreate(&eb[0]) == cudaSuccess && cudaEventCreate(&eb[1]) == cudaSuccess &&
                 cudaEventRecord(eb[0], st) == cudaSuccess;
    cudaError_t e = launch_validate(m->b.verts, m->b.nv, m->b.tris, m->b.nt, d_err, st);
    if (e == cudaSuccess) e = build_bvh(m->b, false, d_err, c->pool, st);
    timed = timed && cudaEventRecord(eb[1], st) == cudaSuccess;
    unsigned herr = 0;
    // a pageable destination: the copy returns when the stream has reached it (the build is done)
    cudaError_t es = cudaMemcpyAsync(&herr, d_err, sizeof(unsigned), cudaMemcpyDeviceToHost, st);
    // on an error the stream may still hold kernels that use the mesh: drain it before freeing
    const cudaError_t es2 = cudaStreamSynchronize(st);
    if (es == cudaSuccess) es = es2;
    if (e == cudaSuccess) e = es;
    float bms = 0.0f;
    if (timed && e == cudaSuccess && cudaEventElapsedTime(&bms, eb[0], eb[1]) == cudaSuccess) m->build_ms = bms;
    for (cudaEvent_t ev : eb)
        if (ev) cudaEventDestroy(ev);
    cudaGetLastError();  // a failed event call above is not the build's error
    cudaFreeAsync(d_err, st);
    if (e != cudaSuccess) {
        mesh_free(c, m, st);
        return sk.fail(e == cudaErrorMemoryAllocation ? GI_ERR_OOM : GI_ERR_CUDA, "BVH build", e);
    }
    if (herr) {
        mesh_free(c, m, st);
        if (herr & 1u) return sk.fail(GI_ERR_INVALID_ARG, "triangle index out of range");
        if (herr & 2u) return sk.fail(GI_ERR_RANGE, "vertex coordinate outside the supported domain");
        return sk.fail(GI_ERR_CUDA, "BVH build: inconsistent wide-node collapse");
    }
    c->mesh_bytes += m->b.bytes;
    if (c->budget && c->mesh_bytes > c->budget) {
        mesh_free(c, m, st);
        return sk.fail(GI_ERR_OOM, "HBM budget exceeded by mesh upload");
    }
    *out = m;
    return GI_OK;
}

static gi_status mesh_alloc(gi_ctx* c, uint32_t nv, uint32_t nt, gi_mesh** pm, cudaStream_t st, const UploadSink& sk)
{
    if (nt && !nv) return sk.fail(GI_ERR_INVALID_ARG, "triangle index out of range");  // no vertex to index
    gi_mesh* m = new (std::nothrow) gi_mesh();
    if (!m) return GI_ERR_OOM;
    m->ctx = c;
    m->b.nv = nv;
    m->b.nt = nt;
    // 16 bytes past the last vertex: the kernels read a vertex as the two
    // aligned 16-byte vectors that hold it (load_vertex)
    size_t vb = sizeof(double) * 3 * (size_t)(nv ? nv : 1) + 16, tb = sizeof(uint32_t) * 3 * (size_t)(nt ? nt : 1);
    if (c->budget && c->mesh_bytes + vb + tb > c->budget) {
        delete m;
        return sk.fail(GI_ERR_OOM, "HBM budget exceeded by mesh upload");
    }
    cudaError_t e = pool_alloc(&m->b.verts, vb, c->pool, st);
    if (e == cudaSuccess) e = pool_alloc(&m->b.tris, tb, c->pool, st);
    if (e != cudaSuccess) {
        if (m->b.verts) cudaFreeAsync(m->b.verts, st);
        delete m;
        return sk.fail(GI_ERR_OOM, "mesh allocation", e);
    }
    m->b.bytes = vb + tb;
    *pm = m;
    return GI_OK;
}

// Host -> device copy on stream st.  Pinned sources go straight to the DMA
// engine.  A large pageable source would be staged by the CUDA driver on the
// calling thread at about a third of the link rate; instead the context's
// copy helpers fill one pinned chunk while the DMA of the previous one runs.
// Returns when the source may be reused (like a pageable cudaMemcpyAsync).
static cudaError_t h2d(gi_ctx* c, void* dst, const void* src, size_t bytes, cudaStream_t st)
{
    if (bytes < 2 * Staging::kChunk) return cudaMemcpyAsync(dst, src, bytes, cudaMemcpyHostToDevice, st);
    cudaPointerAttributes a{};
    if (cudaPointerGetAttributes(&a, src) != cudaSuccess) {
        cudaGetLastError();  // an unknown pointer is ordinary host memory
        a.type = cudaMemoryTypeUnregistered;
    }
    if (a.type != cudaMemoryTypeUnregistered)
        return cudaMemcpyAsync(dst, src, bytes, cudaMemcpyHostToDevice, st);
    Staging& sg = c->stage[st == c->st2 ? 1 : 0];
    cudaError_t e = sg.init();
    if (e != cudaSuccess) {
        cudaGetLastError();
        return cudaMemcpyAsync(dst, src, bytes, cudaMemcpyHostToDevice, st);
    }
    std::call_once(c->copy_pool_once, [c] {
        const unsigned hw = std::thread::hardware_concurrency();
        c->copy_pool.reset(new CopyPool(hw >= 16 ? 7u : hw >= 4 ? hw / 2 - 1 : 0u));
    });
    size_t k = 0;
    for (size_t off = 0; off < bytes; off += Staging::kChunk, k++) {
        const int slot = (int)(k & 1);
        const size_t n = bytes - off < Staging::kChunk ? bytes - off : Staging::kChunk;
        e = cudaEventSynchronize(sg.ev[slot]);  // the slot's previous DMA is done
        if (e != cudaSuccess) return e;
        c->copy_pool->copy(sg.buf[slot], static_cast<const char*>(src) + off, n);
        e = cudaMemcpyAsync(static_cast<char*>(dst) + off, sg.buf[slot], n, cudaMemcpyHostToDevice, st);
        if (e == cudaSuccess) e = cudaEventRecord(sg.ev[slot], st);
        if (e != cudaSuccess) return e;
    }
    return cudaSuccess;
}

// Host arrays -> device mesh with its BVH, on stream st (the caller holds c->mu).
static gi_status mesh_upload_on(gi_ctx* c, const double* verts, uint32_t nv, const uint32_t* tris, uint32_t nt,
                                gi_mesh** out, cudaStream_t st, const UploadSink& sk)
{
    gi_mesh* m = nullptr;
    gi_status s = mesh_alloc(c, nv, nt, &m, st, sk);
    if (s != GI_OK) return s;
    cudaError_t e = cudaSuccess;
    if (nv) e = h2d(c, m->b.verts, verts, sizeof(double) * 3 * (size_t)nv, st);
    if (e == cudaSuccess && nt) e = h2d(c, m->b.tris, tris, sizeof(uint32_t) * 3 * (size_t)nt, st);
    if (e != cudaSuccess) {
        cudaStreamSynchronize(st);
        mesh_free(c, m, st);
        return sk.cuda(e, "upload mesh");
    }
    return mesh_finish(c, m, out, st, sk);
}

extern "C" gi_status gi_mesh_upload(gi_ctx* c, const double* verts, uint32_t nv, const uint32_t* tris, uint32_t nt,
                                    gi_mesh** out)
{
    if (!c || !out || (nv && !verts) || (nt && !tris) || nt > 0x7fffffffu) return GI_ERR_INVALID_ARG;
    std::lock_guard<std::mutex> lk(c->mu);
    cudaSetDevice(c->device);
    return mesh_upload_on(c, verts, nv, tris, nt, out, c->st, UploadSink{c, nullptr});
}

extern "C" gi_status gi_wait_stream(gi_ctx* c, void* stream)
{
    if (!c) return GI_ERR_INVALID_ARG;
    std::lock_guard<std::mutex> lk(c->mu);
    CK(c, cudaSetDevice(c->device), "set device");
    // ev[7] is kept for this hand-off: recorded on the caller's stream, waited
    // on by the context's two streams (the wait binds the work recorded now)
    CK(c, cudaEventRecord(c->ev[7], static_cast<cudaStream_t>(stream)), "record on the caller's stream");
    CK(c, cudaStreamWaitEvent(c->st, c->ev[7], 0), "stream wait");
    CK(c, cudaStreamWaitEvent(c->st2, c->ev[7], 0), "stream wait");
    return GI_OK;
}

extern "C" gi_status gi_mesh_upload_device(gi_ctx* c, const double* d_verts, uint32_t nv, const uint32_t* d_tris,
                                           uint32_t nt, gi_mesh** out)
{
    if (!c || !out || (nv && !d_verts) || (nt && !d_tris) || nt > 0x7fffffffu) return GI_ERR_INVALID_ARG;
    std::lock_guard<std::mutex> lk(c->mu);
    cudaSetDevice(c->device);
    gi_mesh* m = nullptr;
    const UploadSink sk{c, nullptr};
    gi_status s = mesh_alloc(c, nv, nt, &m, c->st, sk);
    if (s != GI_OK) return s;
    if (nv) CK(c, cudaMemcpyAsync(m->b.verts, d_verts, sizeof(double) * 3 * (size_t)nv, cudaMemcpyDeviceToDevice,
                                  c->st), "copy vertices");
    if (nt) CK(c, cudaMemcpyAsync(m->b.tris, d_tris, sizeof(uint32_t) * 3 * (size_t)nt, cudaMemcpyDeviceToDevice,
                                  c->st), "copy triangles");
    return mesh_finish(c, m, out, c->st, sk);
}

// Frees a mesh's buffers in order on stream st (the caller holds c->mu).
static void mesh_free(gi_ctx* c, gi_mesh* m, cudaStream_t st)
{
    cudaSetDevice(c->device);
    // stream-ordered: work already queued on st still sees the mesh
    void* p[] = {m->b.verts,   m->b.tris,   m->b.leafTri, m->b.leafBox,  m->b.nodes,   m->b.leafBox64,
                 m->b.nodes64, m->b.cutRef, m->b.cutBox,  m->b.cutBox64, m->b.ncuts};
    for (void* q : p)
        if (q) cudaFreeAsync(q, st);
    if (m->b.bytes <= c->mesh_bytes) c->mesh_bytes -= m->b.bytes;
    delete m;
}

extern "C" gi_status gi_mesh_release(gi_ctx* c, gi_mesh* m)
{
    if (!c || !m || m->ctx != c) return GI_ERR_INVALID_ARG;
    std::lock_guard<std::mutex> lk(c->mu);
    mesh_free(c, m, c->st);
    return GI_OK;
}

extern "C" gi_status gi_mesh_build_ms(const gi_mesh* m, double* ms)
{
    if (!m || !ms) return GI_ERR_INVALID_ARG;
    *ms = m->build_ms;
    return GI_OK;
}

extern "C" gi_status gi_mesh_info(const gi_mesh* m, uint32_t* nv, uint32_t* nt, uint64_t* nodes, uint64_t* bytes)
{
    if (!m) return GI_ERR_INVALID_ARG;
    if (nv) *nv = m->b.nv;
    if (nt) *nt = m->b.nt;
    if (nodes) *nodes = m->b.nnodes;
    if (bytes) *bytes = m->b.bytes;
    return GI_OK;
}

// ---------------------------------------------------------------------------
// Poses (RotationTools.h:28-70)
// ---------------------------------------------------------------------------
extern "C" gi_status gi_pose_identity(gi_pose* p)
{
    if (!p) return GI_ERR_INVALID_ARG;
    memset(p, 0, sizeof *p);
    p->R[0] = p->R[4] = p->R[8] = 1.0;
    p->identity = 1;
    return GI_OK;
}

extern "C" gi_status gi_pose_from_euler_deg(const double rot[3], const double center[3], const double trans[3],
                                            gi_pose* out)
{
    if (!rot || !center || !trans || !out) return GI_ERR_INVALID_ARG;
    // R = Rz * Ry * Rx (RotationTools.h:28-53), degrees to radians with the same constant
    volatile double d2r = 3.14159265358979323846 / 180.0;
    double rx = rot[0] * d2r, ry = rot[1] * d2r, rz = rot[2] * d2r;
    double cx = cos(rx), sx = sin(rx), cy = cos(ry), sy = sin(ry), cz = cos(rz), sz = sin(rz);
    memset(out, 0, sizeof *out);
    out->R[0] = cy * cz;
    out->R[1] = sx * sy * cz - cx * sz;
    out->R[2] = cx * sy * cz + sx * sz;
    out->R[3] = cy * sz;
    out->R[4] = sx * sy * sz + cx * cz;
    out->R[5] = cx * sy * sz - sx * cz;
    out->R[6] = -sy;
    out->R[7] = sx * cy;
    out->R[8] = cx * cy;
    for (int i = 0; i < 3; i++) {
        out->center[i] = center[i];
        out->trans[i] = trans[i];
    }
    out->identity = (rot[0] == 0.0 && rot[1] == 0.0 && rot[2] == 0.0 && trans[0] == 0.0 && trans[1] == 0.0 &&
                     trans[2] == 0.0);
    return GI_OK;
}

extern "C" gi_status gi_pose_apply(const gi_pose* p, const double* v, uint64_t nv, double* out)
{
    if (!p || (nv && (!v || !out))) return GI_ERR_INVALID_ARG;
    for (uint64_t i = 0; i < nv; i++) {
        if (p->identity) {
            out[3 * i] = v[3 * i];
            out[3 * i + 1] = v[3 * i + 1];
            out[3 * i + 2] = v[3 * i + 2];
            continue;
        }
        volatile double x = v[3 * i] - p->center[0], y = v[3 * i + 1] - p->center[1], z = v[3 * i + 2] - p->center[2];
        volatile double t0 = p->R[0] * x, t1 = p->R[1] * y, t2 = p->R[2] * z;
        volatile double rx = t0 + t1;
        rx = rx + t2;
        volatile double u0 = p->R[3] * x, u1 = p->R[4] * y, u2 = p->R[5] * z;
        volatile double ry = u0 + u1;
        ry = ry + u2;
        volatile double w0 = p->R[6] * x, w1 = p->R[7] * y, w2 = p->R[8] * z;
        volatile double rz = w0 + w1;
        rz = rz + w2;
        volatile double ox = rx + p->center[0], oy = ry + p->center[1], oz = rz + p->center[2];
        out[3 * i] = ox + p->trans[0];
        out[3 * i + 1] = oy + p->trans[1];
        out[3 * i + 2] = oz + p->trans[2];
    }
    return GI_OK;
}

bool pose_ok(const gi_pose& p)
{
    if (p.identity) return true;
    for (double r : p.R)
        if (!(fabs(r) <= 16.0)) return false;
    for (int i = 0; i < 3; i++)
        if (!(fabs(p.center[i]) <= 0x1p90) || !(fabs(p.trans[i]) <= 0x1p90)) return false;
    return true;
}

DevPose make_dev_pose(const gi_pose& p)
{
    DevPose d;
    memset(&d, 0, sizeof d);
    d.identity = p.identity ? 1 : 0;
    for (int i = 0; i < 9; i++) d.R[i] = p.identity ? (i % 4 == 0 ? 1.0 : 0.0) : p.R[i];
    for (int i = 0; i < 3; i++) {
        d.C[i] = p.identity ? 0.0 : p.center[i];
        d.T[i] = p.identity ? 0.0 : p.trans[i];
    }
    for (int r = 0; r < 3; r++) {
        double rc = d.R[3 * r] * d.C[0] + d.R[3 * r + 1] * d.C[1] + d.R[3 * r + 2] * d.C[2];
        d.b64[r] = d.C[r] + d.T[r] - rc;
        double m = fabs(d.C[r]) + fabs(d.T[r]) + fabs(d.R[3 * r]) * fabs(d.C[0]) +
                   fabs(d.R[3 * r + 1]) * fabs(d.C[1]) + fabs(d.R[3 * r + 2]) * fabs(d.C[2]);
        d.padm64[r] = m * (1.0 + 0x1p-40);
        d.bf[r] = (float)d.b64[r];
        d.padm[r] = nextafterf((float)d.padm64[r], INFINITY);
    }
    for (int i = 0; i < 9; i++) d.Rf[i] = (float)d.R[i];
    // inverse map, used to test boxes in this mesh's own frame as well
    if (!d.identity) {
        double eta = 0.0;
        for (int i = 0; i < 3; i++)
            for (int j = 0; j < 3; j++) {
                double g = 0.0;
                for (int k = 0; k < 3; k++) g += d.R[3 * k + i] * d.R[3 * k + j];
                eta = std::max(eta, fabs(g - (i == j ? 1.0 : 0.0)));
            }
        d.inv_eta = eta;
        d.inv_ok = eta <= 0x1p-30 ? 1 : 0;
        for (int r = 0; r < 3; r++)
            for (int k = 0; k < 3; k++) d.Ri64[3 * r + k] = d.R[3 * k + r];
        for (int r = 0; r < 3; r++) {
            double acc = 0.0, m = fabs(d.C[r]);
            for (int k = 0; k < 3; k++) {
                acc += d.Ri64[3 * r + k] * (d.C[k] + d.T[k]);
                m += fabs(d.Ri64[3 * r + k]) * (fabs(d.C[k]) + fabs(d.T[k]));
            }
            d.bi64[r] = d.C[r] - acc;
            d.padmi64[r] = m * (1.0 + 0x1p-40);
            d.bif[r] = (float)d.bi64[r];
            d.padmi[r] = nextafterf((float)d.padmi64[r], INFINITY);
        }
        for (int i = 0; i < 9; i++) d.Rif[i] = (float)d.Ri64[i];
    }
    return d;
}

MeshDev mesh_dev(const gi_mesh* m)
{
    MeshDev d;
    d.verts = m->b.verts;
    d.tris = m->b.tris;
    d.leafTri = m->b.leafTri;
    d.leafBox = m->b.leafBox;
    d.leafBox64 = m->b.leafBox64;
    d.nodes = m->b.nodes;
    d.nodes64 = m->b.nodes64;
    d.cutRef = m->b.cutRef;
    d.cutBox = m->b.cutBox;
    d.cutBox64 = m->b.cutBox64;
    d.ncuts = m->b.ncuts;
    d.root = m->b.root;
    d.nv = m->b.nv;
    d.nt = m->b.nt;
    d.nnodes = m->b.nnodes;
    return d;
}

extern "C" gi_status gi_intersect_opts_default(gi_intersect_opts* o)
{
    if (!o) return GI_ERR_INVALID_ARG;
    o->want_segments = 1;
    o->precision_mode = GI_PREC_FP32_CASCADE;
    o->sort_output = 1;
    o->reserved = 0;
    return GI_OK;
}

static int bits_for(uint64_t n)
{
    int b = 1;
    while ((1ull << b) < n) b++;
    return b;
}

static gi_status ensure_fp64(gi_ctx* c, gi_mesh* m)
{
    if (m->has64 || m->b.nt == 0) {
        m->has64 = true;
        return GI_OK;
    }
    unsigned* d_err = nullptr;
    cudaError_t e = pool_alloc(&d_err, sizeof(unsigned), c->pool, c->st);
    if (e != cudaSuccess) return set_err(c, GI_ERR_OOM, "FP64 BVH build", e);
    unsigned herr = 0;
    e = cudaMemsetAsync(d_err, 0, sizeof(unsigned), c->st);
    if (e == cudaSuccess) e = build_bvh(m->b, true, d_err, c->pool, c->st);
    if (e == cudaSuccess) e = cudaMemcpyAsync(&herr, d_err, sizeof(unsigned), cudaMemcpyDeviceToHost, c->st);
    const cudaError_t es = cudaStreamSynchronize(c->st);
    if (e == cudaSuccess) e = es;
    cudaFreeAsync(d_err, c->st);
    if (e != cudaSuccess) return set_err(c, GI_ERR_CUDA, "FP64 BVH build", e);
    if (herr) return set_err(c, GI_ERR_CUDA, "FP64 BVH build: inconsistent wide-node collapse");
    m->has64 = true;
    return GI_OK;
}

// A pinned block of at least `need` bytes for this call's results in *buf
// (the block held so far goes back to the pool if it is too small).
static gi_status pinned_for(gi_ctx* c, PinnedBuf** buf, size_t need)
{
    if (*buf && (*buf)->bytes >= need) return GI_OK;
    if (*buf) c->pinned->put(*buf);
    *buf = c->pinned->get(need);
    return *buf ? GI_OK : set_err(c, GI_ERR_OOM, "pinned result staging");
}

// Core: runs the job list on the device and fills per-job results.
// One host synchronisation per call: every kernel takes its sizes from the
// device counters, and the results are copied back speculatively at the size
// of the previous call (a second copy follows only when the result grew).
static gi_status run_jobs(gi_ctx* c, const std::vector<JobDev>& jobs, const gi_intersect_opts& o,
                          std::vector<gi_result*>& outs)
{
    const uint32_t nj = (uint32_t)jobs.size();
    const int prec = o.precision_mode == GI_PREC_FP64 ? 1 : 0;
    const bool want_segs = o.want_segments != 0;
    const bool sort = o.sort_output != 0;
    uint64_t maxA = 1, maxB = 1, sumT = 0;
    for (const auto& j : jobs) {
        maxA = std::max<uint64_t>(maxA, j.A.nt);
        maxB = std::max<uint64_t>(maxB, j.B.nt);
        sumT += j.A.nt + j.B.nt;
    }
    int ba = bits_for(maxA), bb = bits_for(maxB), bj = nj > 1 ? bits_for(nj) : 0;
    if (ba + bb + bj > 64) return set_err(c, GI_ERR_INVALID_ARG, "batch too large for 64-bit ordering keys");
    if (nj > (1u << 19)) return set_err(c, GI_ERR_INVALID_ARG, "at most 2^19 jobs per batch");
    if (nj > c->cap_jobs) {
        if (c->d_jobs) cudaFree(c->d_jobs);
        if (c->h_jobs) cudaFreeHost(c->h_jobs);
        c->d_jobs = nullptr;
        c->h_jobs = nullptr;
        c->cap_jobs = 0;
        CK(c, cudaMalloc(&c->d_jobs, sizeof(JobDev) * nj), "jobs");
        CK(c, cudaMallocHost(&c->h_jobs, sizeof(JobDev) * nj), "jobs staging");
        c->cap_jobs = nj;
    }
    memcpy(c->h_jobs, jobs.data(), sizeof(JobDev) * nj);
    CK(c, cudaMemcpyAsync(c->d_jobs, c->h_jobs, sizeof(JobDev) * nj, cudaMemcpyHostToDevice, c->st), "jobs copy");
    const bool tiny = (c->flags & GI_FLAG_TINY_BUFFERS) != 0;
    uint32_t need_front =
        std::max<uint32_t>(c->cap_front, tiny ? 64u : (uint32_t)std::min<uint64_t>(std::max<uint64_t>(1u << 21, sumT), 1u << 26));
    uint32_t need_cand =
        std::max<uint32_t>(c->cap_cand, tiny ? 64u : (uint32_t)std::min<uint64_t>(sumT * 2 + 4096, 1u << 22));
    uint32_t need_res = std::max<uint32_t>(c->cap_res, tiny ? 64u : std::max<uint32_t>(need_cand / 4, 1u << 16));
    uint32_t need_esc = std::max<uint32_t>(c->cap_esc, tiny ? 64u : std::max<uint32_t>(need_cand / 4, 1u << 16));
    const unsigned long long launches0 = launch_count();
    Counters& H = *c->h_cnt;
    int retries = 0;
    uint32_t nres = 0, nsegs = 0;
    char* hp = nullptr;
    size_t off_jobs = 0, off_segs = 0, off_segpair = 0;
    // pinned block the results land in; returned to the pool on every early exit
    PinnedBuf* buf = nullptr;
    struct BufGuard {
        gi_ctx* c;
        PinnedBuf*& b;
        ~BufGuard()
        {
            if (b) c->pinned->put(b);
        }
    } guard{c, buf};
    // ordering path: the small cooperative one when the previous call's count says
    // the result will be small (the kernel refuses, and this loop reruns on the
    // radix path, if it is not)
    bool small_order = ba + bb + bj <= 63 && c->pred_pairs <= kOrderSmallMax - kOrderSmallMax / 4;
    // everything after the traversal in one launch: sorted output of a result
    // the previous call's count says is small enough (the kernel refuses, and
    // this loop reruns on the general path, if it is not, or if its keys crowd
    // into one partition; a refusal keeps the next calls off this path a while)
    bool fin = sort && ba + bb + bj <= 63 && c->pred_pairs <= kFinMax - kFinMax / 4 && c->fin_backoff == 0;
    if (c->fin_backoff) c->fin_backoff--;
    const int kbits = ba + bb + bj;
    const int fin_shift = kbits > kFinPartBits ? kbits - kFinPartBits : 0;
    const uint32_t tune_key = TravTuner::key(prec, nj, sumT);
    const int shape = c->fixed_shape >= 0 ? c->fixed_shape : c->tuner.pick(tune_key);
    for (;;) {
        CK(c, grow(c->queue, c->cap_front, need_front, c->pool, c->st), "node queue");
        if (c->cap_qflag < c->cap_front) {
            // fresh tag words must not match any call's tag: zero them
            CK(c, grow(c->qflag, c->cap_qflag, c->cap_front, c->pool, c->st), "node queue");
            CK(c, cudaMemsetAsync(c->qflag, 0, sizeof(unsigned) * c->cap_qflag, c->st), "node queue");
        }
        CK(c, grow(c->cand, c->cap_cand, need_cand, c->pool, c->st), "candidates");
        if (c->cap_cflag < c->cap_cand) {
            CK(c, grow(c->cflag, c->cap_cflag, c->cap_cand, c->pool, c->st), "candidates");
            CK(c, cudaMemsetAsync(c->cflag, 0, sizeof(unsigned) * c->cap_cflag, c->st), "candidates");
        }
        CK(c, grow(c->res, c->cap_res, need_res, c->pool, c->st), "results");
        CK(c, grow(c->esc, c->cap_esc, need_esc, c->pool, c->st), "escalations");
        const uint32_t cap = c->cap_res;
        if (cap > c->cap_out) {
            void* old[] = {c->segs, c->nseg, c->pairs_out, c->job_out, c->segs_out, c->segpair_out};
            for (void* p : old)
                if (p) cudaFreeAsync(p, c->st);
            c->cap_out = 0;
            CK(c, pool_alloc(&c->segs, sizeof(double) * 18 * (size_t)cap, c->pool, c->st), "segments");
            CK(c, pool_alloc(&c->nseg, sizeof(uint32_t) * cap, c->pool, c->st), "segments");
            CK(c, pool_alloc(&c->pairs_out, sizeof(int32_t) * 2 * (size_t)cap, c->pool, c->st), "pairs");
            CK(c, pool_alloc(&c->job_out, sizeof(uint32_t) * cap, c->pool, c->st), "pairs");
            CK(c, pool_alloc(&c->segs_out, sizeof(double) * 18 * (size_t)cap, c->pool, c->st), "segments");
            CK(c, pool_alloc(&c->segpair_out, sizeof(int32_t) * 3 * (size_t)cap, c->pool, c->st), "segments");
            c->cap_out = cap;
        }
        size_t osb = order_scratch_bytes(cap, kOsMaxPasses);
        if (osb > c->order_scratch_bytes) {
            if (c->order_scratch) cudaFreeAsync(c->order_scratch, c->st);
            c->order_scratch = nullptr;
            c->order_scratch_bytes = 0;
            CK(c, pool_alloc(&c->order_scratch, osb, c->pool, c->st), "order scratch");
            CK(c, cudaMemsetAsync(c->order_scratch, 0, osb, c->st), "order scratch");
            c->order_scratch_bytes = osb;
        }
        OrderBufs O = make_order_bufs(c->order_scratch, cap, ba, bb, bj);
        Bufs b;
        b.jobs = c->d_jobs;
        b.njobs = nj;
        b.queue = c->queue;
        b.qflag = c->qflag;
        b.cap_queue = std::min(c->cap_front, c->cap_qflag);
        b.cand = c->cand;
        b.cflag = c->cflag;
        b.cap_cand = std::min(c->cap_cand, c->cap_cflag);
        if (++c->tag == 0) {
            // after 2^32 calls the tags wrap: clear the tag words once
            CK(c, cudaMemsetAsync(c->qflag, 0, sizeof(unsigned) * c->cap_qflag, c->st), "node queue");
            CK(c, cudaMemsetAsync(c->cflag, 0, sizeof(unsigned) * c->cap_cflag, c->st), "candidates");
            c->tag = 1;
        }
        b.tag = c->tag;
        b.res = c->res;
        b.cap_res = c->cap_res;
        b.esc = c->esc;
        b.cap_esc = c->cap_esc;
        b.cnt = c->d_cnt;
        b.precision = prec;
        b.two_frame = nj > 1 ? 1 : 0;
        // one pair: skip the narrowest level by seeding from the depth-4 cuts
        // (up to 256 x 256 seed tests); a batch keeps the depth-3 cuts, whose
        // seed tests grow with the number of jobs
        b.deep_seed = nj == 1 ? 1 : 0;
        b.quad_below = 0u;   // set by the launcher of the level-synchronous traversal
        b.cand_blocks = 0u;
        b.publish = 0u;
        CK(c, cudaMemsetAsync(c->d_cnt, 0, sizeof(Counters), c->st), "counters");
        CK(c, cudaEventRecord(c->ev[0], c->st), "event");
        CK(c, launch_traverse(b, c->cfg, prec, trav_shape(shape), c->st), "traverse");
        // the finish follows the traversal directly (programmatic dependent
        // launch): no event between them; the general path keeps its events
        if (!fin) CK(c, cudaEventRecord(c->ev[1], c->st), "event");
        if (fin) {
            FinArgs F;
            F.segs = c->segs;
            F.pairs_out = c->pairs_out;
            F.job_out = c->job_out;
            F.segs_out = c->segs_out;
            F.segpair_out = c->segpair_out;
            F.cap = cap;
            F.want_segments = want_segs ? 1 : 0;
            F.shift = fin_shift;
            CK(c, launch_finish(b, O, F, c->cfg, c->st, true), "exact stage, segments and ordering");
        } else {
            CK(c, launch_exact(b, c->cfg, c->st), "exact stage");
            CK(c, cudaEventRecord(c->ev[2], c->st), "event");
            if (small_order && want_segs && sort) {
                // the segments are built on the second stream while the ordering
                // ranks the results; only the placing launch waits for them
                CK(c, cudaStreamWaitEvent(c->st2, c->ev[2], 0), "event");
                CK(c, launch_segments(b, c->segs, c->nseg, c->cfg, c->st2), "segments");
                CK(c, cudaEventRecord(c->ev[3], c->st2), "event");
                CK(c, launch_order_small_phases(b, O, sort, c->segs, c->nseg, c->pairs_out, c->job_out, c->segs_out,
                                                c->segpair_out, want_segs, kOrderRank, c->st),
                   "ordering");
                CK(c, cudaStreamWaitEvent(c->st, c->ev[3], 0), "event");
                CK(c, launch_order_small_phases(b, O, sort, c->segs, c->nseg, c->pairs_out, c->job_out, c->segs_out,
                                                c->segpair_out, want_segs, kOrderPlace, c->st),
                   "ordering");
            } else {
                if (want_segs) CK(c, launch_segments(b, c->segs, c->nseg, c->cfg, c->st), "segments");
                CK(c, cudaEventRecord(c->ev[3], c->st), "event");
                if (small_order)
                    CK(c, launch_order_small(b, O, sort, c->segs, c->nseg, c->pairs_out, c->job_out, c->segs_out,
                                             c->segpair_out, want_segs, c->st),
                       "ordering");
                else
                    CK(c, launch_order_gather(b, O, sort, c->segs, c->nseg, c->pairs_out, c->job_out, c->segs_out,
                                              c->segpair_out, want_segs, c->cfg, c->st),
                       "ordering");
            }
        }
        CK(c, cudaEventRecord(c->ev[4], c->st), "event");
        // speculative copy at the previous call's size
        uint32_t pp = std::min<uint32_t>(cap, (uint32_t)std::min<uint64_t>(c->pred_pairs + c->pred_pairs / 4 + 1024,
                                                                          0xffffffffu));
        uint32_t ps = want_segs ? std::min<uint32_t>(3 * cap, c->pred_segs + c->pred_segs / 4 + 1024) : 0u;
        off_jobs = sizeof(int32_t) * 2 * (size_t)pp;
        off_segs = off_jobs + (nj > 1 ? sizeof(uint32_t) * (size_t)pp : 0);
        off_segs = (off_segs + 15) & ~(size_t)15;
        off_segpair = off_segs + sizeof(double) * 6 * (size_t)ps;
        gi_status s = pinned_for(c, &buf, off_segpair + sizeof(int32_t) * (size_t)ps + 64);
        if (s != GI_OK) return s;
        hp = (char*)buf->p;
        CK(c, cudaMemcpyAsync(c->h_cnt, c->d_cnt, sizeof(Counters), cudaMemcpyDeviceToHost, c->st), "counters");
        CK(c, cudaMemcpyAsync(hp, c->pairs_out, off_jobs, cudaMemcpyDeviceToHost, c->st), "copy pairs");
        if (nj > 1)
            CK(c, cudaMemcpyAsync(hp + off_jobs, c->job_out, sizeof(uint32_t) * pp, cudaMemcpyDeviceToHost, c->st),
               "copy jobs");
        if (ps) {
            CK(c, cudaMemcpyAsync(hp + off_segs, c->segs_out, sizeof(double) * 6 * ps, cudaMemcpyDeviceToHost, c->st),
               "copy segments");
            CK(c, cudaMemcpyAsync(hp + off_segpair, c->segpair_out, sizeof(int32_t) * ps, cudaMemcpyDeviceToHost,
                                  c->st),
               "copy segments");
        }
        CK(c, cudaStreamSynchronize(c->st), "sync");
        if (H.err & kErrTimeout) {
            // a finish launch that gave up may leave partition counts behind
            if (fin) cudaMemsetAsync(O.fin, 0, sizeof(uint32_t) * 2 * kFinParts, c->st);
            return set_err(c, GI_ERR_TIMEOUT, "a bounded device wait ran out");
        }
        if (H.err & kErrExactCapacity) return set_err(c, GI_ERR_RANGE, "exact arithmetic capacity exceeded");
        if (H.overflow) {
            if (retries >= 12) return set_err(c, GI_ERR_CAPACITY, "intersection buffers stayed too small");
            retries++;
            auto g4 = [](uint32_t cur, uint32_t seen) {
                uint64_t v = std::max<uint64_t>((uint64_t)cur * 4, (uint64_t)seen + seen / 2 + 1024);
                return (uint32_t)std::min<uint64_t>(v, 0x7fffffffu);
            };
            if (H.overflow & kOvfFrontier) need_front = g4(c->cap_front, H.q_tail);
            if (H.overflow & kOvfCand) need_cand = g4(c->cap_cand, (uint32_t)(H.work_cand >> 32));
            if (H.overflow & (kOvfRes | kOvfCand)) need_res = g4(c->cap_res, H.res);
            if (H.overflow & (kOvfEsc | kOvfCand)) need_esc = g4(c->cap_esc, H.esc);
            continue;
        }
        if (H.order_redo) {
            if (fin) {
                // a refusal after the counting leaves the partition counts behind
                CK(c, cudaMemsetAsync(O.fin, 0, sizeof(uint32_t) * 2 * kFinParts, c->st), "finish counts");
                fin = false;
                if (H.order_redo == kRedoCrowded) c->fin_backoff = 64;
                if (H.res > kOrderSmallMax) small_order = false;
                continue;
            }
            if (!small_order) return set_err(c, GI_ERR_CAPACITY, "ordering path refused twice");
            small_order = false;
            continue;
        }
        nres = H.res;
        nsegs = want_segs ? H.nseg : 0;
        if (nres > pp || nsegs > ps) {
            // the result outgrew the speculative copy: copy it again at its real size
            off_jobs = sizeof(int32_t) * 2 * (size_t)nres;
            off_segs = (off_jobs + (nj > 1 ? sizeof(uint32_t) * (size_t)nres : 0) + 15) & ~(size_t)15;
            off_segpair = off_segs + sizeof(double) * 6 * (size_t)nsegs;
            s = pinned_for(c, &buf, off_segpair + sizeof(int32_t) * (size_t)nsegs + 64);
            if (s != GI_OK) return s;
            hp = (char*)buf->p;
            if (nres) CK(c, cudaMemcpyAsync(hp, c->pairs_out, off_jobs, cudaMemcpyDeviceToHost, c->st), "copy pairs");
            if (nres && nj > 1)
                CK(c, cudaMemcpyAsync(hp + off_jobs, c->job_out, sizeof(uint32_t) * nres, cudaMemcpyDeviceToHost,
                                      c->st),
                   "copy jobs");
            if (nsegs) {
                CK(c, cudaMemcpyAsync(hp + off_segs, c->segs_out, sizeof(double) * 6 * nsegs, cudaMemcpyDeviceToHost,
                                      c->st),
                   "copy segments");
                CK(c, cudaMemcpyAsync(hp + off_segpair, c->segpair_out, sizeof(int32_t) * nsegs,
                                      cudaMemcpyDeviceToHost, c->st),
                   "copy segments");
            }
            CK(c, cudaStreamSynchronize(c->st), "sync");
        }
        break;
    }
    c->pred_pairs = nres;
    c->pred_segs = nsegs;
    float ms_trav = 0, ms_exact = 0, ms_seg = 0, ms_sort = 0, ms_total = 0;
    cudaEventElapsedTime(&ms_total, c->ev[0], c->ev[4]);
    if (fin) {
        // the finish follows the traversal with no event between them: its span
        // and phases from its own timestamps (taken after it waited for the
        // traversal), the traversal the rest of the call
        const double span = H.fin_ns[4] >= H.fin_ns[0] ? 1e-6 * double(H.fin_ns[4] - H.fin_ns[0]) : 0.0;
        if (H.fin_ns[1] >= H.fin_ns[0] && H.fin_ns[2] >= H.fin_ns[1]) {
            ms_exact = (float)(1e-6 * double(H.fin_ns[1] - H.fin_ns[0]));
            ms_seg = (float)(1e-6 * double(H.fin_ns[2] - H.fin_ns[1]));
        }
        ms_trav = std::max(0.0f, ms_total - (float)span);
        ms_sort = std::max(0.0f, (float)span - ms_exact - ms_seg);
    } else {
        cudaEventElapsedTime(&ms_trav, c->ev[0], c->ev[1]);
        cudaEventElapsedTime(&ms_exact, c->ev[1], c->ev[2]);
        cudaEventElapsedTime(&ms_seg, c->ev[2], c->ev[3]);
        cudaEventElapsedTime(&ms_sort, c->ev[3], c->ev[4]);
    }
    if (c->fixed_shape < 0) c->tuner.report(tune_key, shape, ms_trav);
    // split per job (sorted by job first)
    std::vector<uint32_t> job_start(nj + 1, 0);
    if (nj == 1) {
        job_start[1] = nres;
    } else {
        const uint32_t* hj = (const uint32_t*)(hp + off_jobs);
        for (uint32_t k = 0; k < nres; k++) job_start[hj[k] + 1]++;
        for (uint32_t j = 0; j < nj; j++) job_start[j + 1] += job_start[j];
    }
    // results are views into the pinned block (no further copy); a batch's
    // segment pair indices are rebased to each job in place
    const int32_t* hpairs = (const int32_t*)hp;
    const double* hsegs = (const double*)(hp + off_segs);
    int32_t* hsegpair = (int32_t*)(hp + off_segpair);
    for (uint32_t j = 0; j < nj; j++) {
        outs[j] = new (std::nothrow) gi_result();
        if (!outs[j]) {
            for (uint32_t k = 0; k < j; k++) {
                delete outs[k];
                outs[k] = nullptr;
            }
            return set_err(c, GI_ERR_OOM, "result");
        }
    }
    buf->refs.store((int)nj);
    buf->home = c->pinned;
    size_t sp = 0;
    for (uint32_t j = 0; j < nj; j++) {
        gi_result* r = outs[j];
        r->buf = buf;
        uint32_t a = job_start[j], e = job_start[j + 1];
        r->pairs = hpairs + 2 * (size_t)a;
        r->npairs = e - a;
        size_t s0 = sp;
        if (nj == 1) sp = nsegs;  // one job: all segments are its own
        else
            while (sp < nsegs && (uint32_t)hsegpair[sp] < e) sp++;
        r->segs = hsegs + 6 * s0;
        r->seg_pair = hsegpair + s0;
        r->nsegs = sp - s0;
        if (a)
            for (size_t q = s0; q < sp; q++) hsegpair[q] -= (int32_t)a;
        gi_stats& s2 = r->stats;
        memset(&s2, 0, sizeof s2);
        s2.tris_a = jobs[j].A.nt;
        s2.tris_b = jobs[j].B.nt;
        s2.nodes_a = jobs[j].A.nnodes;
        s2.nodes_b = jobs[j].B.nnodes;
        s2.pairs = e - a;
        s2.segments = r->nsegs;
        // launch-wide counters (shared by all jobs of a batch)
        s2.node_pairs = H.node_pairs;
        s2.candidates = H.tested;
        s2.filter_decided = H.filter_decided;
        s2.escalated = H.esc;
        s2.exact_signs = H.exact_signs;
        s2.exact_points = H.exact_points;
        s2.levels = H.levels;
        s2.retries = (uint32_t)retries;
        s2.launches = (uint32_t)(launch_count() - launches0);
        s2.traverse_shape = (uint32_t)shape;
        s2.ms_traverse = ms_trav;
        s2.ms_exact = ms_exact;
        s2.ms_segments = ms_seg;
        s2.ms_sort = ms_sort;
        s2.ms_total = ms_total;
        static_assert(sizeof(s2.level_end_ms) / sizeof(double) == (size_t)kLevelTimes, "level time slots");
        if (fin && H.fin_ns[0] && H.fin_ns[4] >= H.fin_ns[0]) {
            for (int k = 0; k < 4; k++)
                s2.finish_ms[k] = H.fin_ns[k + 1] >= H.fin_ns[0] ? 1e-6 * double(H.fin_ns[k + 1] - H.fin_ns[0]) : 0.0;
            s2.finish_phases = 4;
        }
        if (trav_shape(shape).levels && H.t_start) {
            const uint32_t nl = std::min<uint32_t>(H.levels + 1u, (uint32_t)kLevelTimes);
            for (uint32_t l = 0; l < nl && H.level_ns[l] >= H.t_start; l++) {
                s2.level_end_ms[l] = 1e-6 * double(H.level_ns[l] - H.t_start);
                s2.level_times = l + 1;
            }
        }
    }
    buf = nullptr;  // now held by the results
    return GI_OK;
}

extern "C" gi_status gi_intersect(gi_ctx* c, const gi_mesh* A, const gi_pose* pa, const gi_mesh* B, const gi_pose* pb,
                                  const gi_intersect_opts* opts, gi_result** out)
{
    if (!c || !A || !B || !out || A->ctx != c || B->ctx != c) return GI_ERR_INVALID_ARG;
    gi_pair_job j;
    j.A = A;
    j.B = B;
    if (pa) j.pose_a = *pa;
    else gi_pose_identity(&j.pose_a);
    if (pb) j.pose_b = *pb;
    else gi_pose_identity(&j.pose_b);
    return gi_intersect_batch(c, &j, 1, opts, out);
}

extern "C" gi_status gi_intersect_batch(gi_ctx* c, const gi_pair_job* jobs, uint32_t nj, const gi_intersect_opts* opts,
                                        gi_result** out)
{
    if (!c || !jobs || !out || nj == 0) return GI_ERR_INVALID_ARG;
    gi_intersect_opts o;
    if (opts) o = *opts;
    else gi_intersect_opts_default(&o);
    std::lock_guard<std::mutex> lk(c->mu);
    cudaSetDevice(c->device);
    std::vector<JobDev> jd(nj);
    for (uint32_t i = 0; i < nj; i++) {
        const gi_pair_job& j = jobs[i];
        if (!j.A || !j.B || j.A->ctx != c || j.B->ctx != c) return GI_ERR_INVALID_ARG;
        if (!pose_ok(j.pose_a) || !pose_ok(j.pose_b)) return set_err(c, GI_ERR_RANGE, "pose outside the supported domain");
        if (o.precision_mode == GI_PREC_FP64) {
            gi_status s = ensure_fp64(c, const_cast<gi_mesh*>(j.A));
            if (s == GI_OK) s = ensure_fp64(c, const_cast<gi_mesh*>(j.B));
            if (s != GI_OK) return s;
        }
        jd[i].A = mesh_dev(j.A);
        jd[i].B = mesh_dev(j.B);
        jd[i].pa = make_dev_pose(j.pose_a);
        jd[i].pb = make_dev_pose(j.pose_b);
    }
    std::vector<gi_result*> outs(nj, nullptr);
    gi_status s = run_jobs(c, jd, o, outs);
    if (s != GI_OK) {
        for (auto* r : outs) delete r;
        return s;
    }
    for (uint32_t i = 0; i < nj; i++) out[i] = outs[i];
    return GI_OK;
}

extern "C" gi_status gi_intersect_oneshot(gi_ctx* c, const double* vA, uint32_t nvA, const uint32_t* tA, uint32_t ntA,
                                          const gi_pose* pa, const double* vB, uint32_t nvB, const uint32_t* tB,
                                          uint32_t ntB, const gi_pose* pb, const gi_intersect_opts* opts,
                                          gi_result** out)
{
    if (!c || !out || (nvA && !vA) || (ntA && !tA) || (nvB && !vB) || (ntB && !tB) || ntA > 0x7fffffffu ||
        ntB > 0x7fffffffu)
        return GI_ERR_INVALID_ARG;
    gi_mesh *A = nullptr, *B = nullptr;
    gi_status s;
    {
        // B is copied and built on the second stream by a helper thread while A
        // is on the context's stream: B's copy overlaps A's build and the two
        // builds overlap each other
        std::lock_guard<std::mutex> lk(c->mu);
        cudaSetDevice(c->device);
        gi_status sb = GI_OK;
        std::string msg_b;
        std::thread tb([&] {
            cudaSetDevice(c->device);
            sb = mesh_upload_on(c, vB, nvB, tB, ntB, &B, c->st2, UploadSink{c, &msg_b});
        });
        s = mesh_upload_on(c, vA, nvA, tA, ntA, &A, c->st, UploadSink{c, nullptr});
        tb.join();
        if (s == GI_OK && sb != GI_OK) {
            s = sb;
            c->last_error = msg_b;
        }
        if (s != GI_OK) {
            if (A) mesh_free(c, A, c->st);
            if (B) mesh_free(c, B, c->st);
            return s;
        }
    }
    s = gi_intersect(c, A, pa, B, pb, opts, out);
    gi_mesh_release(c, A);
    gi_mesh_release(c, B);
    return s;
}

// ---------------------------------------------------------------------------
// Results
// ---------------------------------------------------------------------------
extern "C" gi_status gi_result_pairs(const gi_result* r, const int32_t** p, uint64_t* n)
{
    if (!r || !p || !n) return GI_ERR_INVALID_ARG;
    *p = r->pairs;
    *n = r->npairs;
    return GI_OK;
}
extern "C" gi_status gi_result_segments(const gi_result* r, const double** s, const int32_t** sp, uint64_t* n)
{
    if (!r || !s || !n) return GI_ERR_INVALID_ARG;
    *s = r->segs;
    if (sp) *sp = r->seg_pair;
    *n = r->nsegs;
    return GI_OK;
}
extern "C" gi_status gi_result_stats(const gi_result* r, gi_stats* out)
{
    if (!r || !out) return GI_ERR_INVALID_ARG;
    *out = r->stats;
    return GI_OK;
}
extern "C" gi_status gi_result_free(gi_result* r)
{
    if (!r) return GI_ERR_INVALID_ARG;
    pinned_release(r->buf);
    delete r;
    return GI_OK;
}

// ---------------------------------------------------------------------------
// Serving: a host thread admits pending pose requests into device rounds.
// ---------------------------------------------------------------------------
struct gi_server {
    gi_ctx* ctx = nullptr;
    gi_server_opts opts;
    std::mutex mu;
    std::condition_variable cv, done_cv;
    struct Req {
        uint64_t ticket;
        gi_pair_job job;
    };
    std::deque<Req> pending;
    std::map<uint64_t, gi_result*> done;
    std::map<uint64_t, gi_status> failed;
    uint64_t next_ticket = 1;
    bool stop = false;
    std::thread worker;
};

static void server_loop(gi_server* s)
{
    for (;;) {
        std::vector<gi_server::Req> round;
        {
            std::unique_lock<std::mutex> lk(s->mu);
            s->cv.wait(lk, [&] { return s->stop || !s->pending.empty(); });
            if (s->stop && s->pending.empty()) return;
            uint32_t cap = s->opts.max_inflight ? s->opts.max_inflight : 256;
            while (!s->pending.empty() && round.size() < cap) {
                round.push_back(s->pending.front());
                s->pending.pop_front();
            }
        }
        std::vector<gi_pair_job> jobs(round.size());
        for (size_t i = 0; i < round.size(); i++) jobs[i] = round[i].job;
        std::vector<gi_result*> outs(round.size(), nullptr);
        gi_status st = gi_intersect_batch(s->ctx, jobs.data(), (uint32_t)jobs.size(), &s->opts.opts, outs.data());
        {
            std::lock_guard<std::mutex> lk(s->mu);
            for (size_t i = 0; i < round.size(); i++) {
                if (st == GI_OK) s->done[round[i].ticket] = outs[i];
                else s->failed[round[i].ticket] = st;
            }
        }
        s->done_cv.notify_all();
    }
}

extern "C" gi_status gi_server_start(gi_ctx* c, const gi_server_opts* opts, gi_server** out)
{
    if (!c || !out) return GI_ERR_INVALID_ARG;
    gi_server* s = new (std::nothrow) gi_server();
    if (!s) return GI_ERR_OOM;
    s->ctx = c;
    if (opts) s->opts = *opts;
    else {
        memset(&s->opts, 0, sizeof s->opts);
        gi_intersect_opts_default(&s->opts.opts);
    }
    s->worker = std::thread(server_loop, s);
    *out = s;
    return GI_OK;
}

extern "C" gi_status gi_server_submit(gi_server* s, const gi_mesh* A, const gi_pose* pa, const gi_mesh* B,
                                      const gi_pose* pb, uint64_t* ticket)
{
    if (!s || !A || !B || !ticket) return GI_ERR_INVALID_ARG;
    gi_server::Req r;
    r.job.A = A;
    r.job.B = B;
    if (pa) r.job.pose_a = *pa;
    else gi_pose_identity(&r.job.pose_a);
    if (pb) r.job.pose_b = *pb;
    else gi_pose_identity(&r.job.pose_b);
    {
        std::lock_guard<std::mutex> lk(s->mu);
        if (s->stop) return GI_ERR_INVALID_ARG;
        r.ticket = s->next_ticket++;
        s->pending.push_back(r);
        *ticket = r.ticket;
    }
    s->cv.notify_one();
    return GI_OK;
}

extern "C" gi_status gi_server_poll(gi_server* s, uint64_t ticket, gi_result** out)
{
    if (!s || !out) return GI_ERR_INVALID_ARG;
    std::lock_guard<std::mutex> lk(s->mu);
    auto it = s->done.find(ticket);
    if (it != s->done.end()) {
        *out = it->second;
        s->done.erase(it);
        return GI_OK;
    }
    auto f = s->failed.find(ticket);
    if (f != s->failed.end()) {
        gi_status st = f->second;
        s->failed.erase(f);
        return st;
    }
    return GI_ERR_NOT_READY;
}

extern "C" gi_status gi_server_wait(gi_server* s, uint64_t ticket, uint32_t timeout_ms, gi_result** out)
{
    if (!s || !out) return GI_ERR_INVALID_ARG;
    std::unique_lock<std::mutex> lk(s->mu);
    auto ready = [&] { return s->done.count(ticket) || s->failed.count(ticket); };
    if (!s->done_cv.wait_for(lk, std::chrono::milliseconds(timeout_ms), ready)) return GI_ERR_TIMEOUT;
    auto it = s->done.find(ticket);
    if (it != s->done.end()) {
        *out = it->second;
        s->done.erase(it);
        return GI_OK;
    }
    gi_status st = s->failed[ticket];
    s->failed.erase(ticket);
    return st;
}

extern "C" gi_status gi_server_stop(gi_server* s)
{
    if (!s) return GI_ERR_INVALID_ARG;
    {
        std::lock_guard<std::mutex> lk(s->mu);
        s->stop = true;
    }
    s->cv.notify_all();
    if (s->worker.joinable()) s->worker.join();
    for (auto& kv : s->done) delete kv.second;
    delete s;
    return GI_OK;
}
