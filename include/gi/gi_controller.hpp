// gi_controller.hpp -- C++ host shim over the C ABI with the reference's
// GPUIntersector interface (YuryUoL/gpu-cubql-intersector-standalone).
//
// Header-only, C++17, no CUDA compiler needed: the host code that drives the
// reference's KernelBVHController (src/GPUIntersector/KernelBVHController.h:36-95)
// and runGridForestIntersectionPipeline
// (src/GPUIntersector/StandaloneBVHPipeline.h:27-43) compiles against this
// header with the same method names and argument order and links libgi.so.
//
// Differences a caller sees:
//  * failures throw gi::Error (status + message) instead of exiting the
//    process (reference: SingleTreeBatchCommon.h:13-22) or returning silently;
//  * the CGAL mesh arguments are accepted and not used: there is no CPU
//    fallback, the device decides every pair exactly;
//  * level / leafThreshold / batchMultiplier / dual-tree step counts tune the
//    reference's level-cut BVH and are accepted and ignored (the LBVH has no
//    level cut and the traversal sizes itself);
//  * the predicate mode argument (runIntersectionPipeline's gpuDouble,
//    KernelBVHController.h:60-63; runGridForestIntersectionPipeline's
//    gpuPredicateMode) is honoured: the reference's modes 0-4
//    (apps/mainApplication.cpp:1595-1607) all begin with the float filter and
//    escalate through (simulated) double or integers to CPU CGAL, which is what
//    the FP32 cascade does on the device (float filter -> FP64 filter -> exact
//    integers), so they select GI_PREC_FP32_CASCADE; the added mode
//    kPredicateModePlainFP64 (5) selects the plain FP64 form, and any other
//    value throws gi::Error(GI_ERR_INVALID_ARG) instead of being ignored;
//  * the output int2* is malloc-owned by the callee and released by the
//    caller with std::free, as in the reference
//    (SingleTreeBatchIntersector.cu:149-167); pairs come sorted by (a, b);
//  * like the reference, construct() keeps non-owning pointers to the host
//    arrays (for reconstructGPU); the caller keeps them alive.
#ifndef GI_GI_CONTROLLER_HPP
#define GI_GI_CONTROLLER_HPP

#include <chrono>
#include <cstdlib>
#include <cstring>
#include <stdexcept>
#include <string>
#include <vector>

#include "gi.h"

#if defined(__has_include)
#if __has_include(<vector_types.h>)
#include <vector_types.h>
#define GI_HAVE_CUDA_VECTOR_TYPES 1
#endif
#endif

namespace gi {

#ifdef GI_HAVE_CUDA_VECTOR_TYPES
using vec3d = ::double3;
using tri3u = ::uint3;
using pair2i = ::int2;
#else
struct vec3d { double x, y, z; };
struct tri3u { unsigned x, y, z; };
struct pair2i { int x, y; };
#endif
static_assert(sizeof(vec3d) == 24 && sizeof(tri3u) == 12 && sizeof(pair2i) == 8, "packed xyz layouts");

class Error : public std::runtime_error {
public:
    Error(gi_status s, const std::string& what) : std::runtime_error(what), status(s) {}
    gi_status status;
};

// Point with CGAL's accessor style (p.x()), the type getCenterA/B return.
struct Point3 {
    double x_ = 0, y_ = 0, z_ = 0;
    Point3() = default;
    Point3(double x, double y, double z) : x_(x), y_(y), z_(z) {}
    double x() const { return x_; }
    double y() const { return y_; }
    double z() const { return z_; }
};

// Field names of the reference's ExecutionStats (src/common/ExecutionStats.h:12-46)
// filled from gi_stats; `detail` keeps the full record.
struct ExecutionStats {
    uint32_t meshATotalNodes = 0;
    uint32_t meshAExtractedTargets = 0;
    uint32_t meshBTotalNodes = 0;
    uint32_t meshBExtractedTargets = 0;
    uint32_t totalIntersections = 0;
    uint64_t totalPossiblePairs = 0;
    double intersectionPercentage = 0.0;
    double buildRefitMeshAMs = 0.0;
    double buildRefitMeshBMs = 0.0;
    double gpuCrossCheckEngineMs = 0.0;
    double dualTreeStepMs = 0.0;
    double parallelDfsDescentBMs = 0.0;
    double initialAllocAndCopyMs = 0.0;
    double thrustInitOverheadMs = 0.0;
    double finalCleanupSyncMs = 0.0;
    double GPUTotalTime = 0.0;
    int totalCrissCrossBatches = 0;
    uint64_t finalAabbCandidatePairs = 0;
    size_t confirmedGreenPairs = 0;   // pairs decided by the first (float) filter stage
    size_t confirmedYellowPairs = 0;  // pairs escalated to the FP64 / exact stage
    gi_stats detail{};
};

namespace detail {
inline void check(gi_status s, const gi_ctx* c, const char* what)
{
    if (s == GI_OK) return;
    std::string m = std::string(what) + ": " + gi_status_string(s);
    const char* e = c ? gi_last_error(c) : nullptr;
    if (e && *e) m += std::string(" (") + e + ")";
    throw Error(s, m);
}
template <class P>
inline void xyz(const P& p, double out[3])
{
    out[0] = static_cast<double>(p.x());
    out[1] = static_cast<double>(p.y());
    out[2] = static_cast<double>(p.z());
}
// The reference's predicate modes 0-4 and the added plain-FP64 mode -> GI_PREC_*.
constexpr int kPredicateModePlainFP64 = 5;
inline int32_t precision_for_predicate_mode(int mode)
{
    if (mode >= 0 && mode <= 4) return GI_PREC_FP32_CASCADE;
    if (mode == kPredicateModePlainFP64) return GI_PREC_FP64;
    throw Error(GI_ERR_INVALID_ARG, "predicate mode " + std::to_string(mode) +
                                        " (reference modes are 0-4; 5 selects the plain FP64 form)");
}
inline void fill(ExecutionStats& s, const gi_stats& d)
{
    s.detail = d;
    s.meshATotalNodes = static_cast<uint32_t>(d.nodes_a);
    s.meshBTotalNodes = static_cast<uint32_t>(d.nodes_b);
    s.totalIntersections = static_cast<uint32_t>(d.pairs);
    s.totalPossiblePairs = d.tris_a * d.tris_b;
    s.intersectionPercentage = s.totalPossiblePairs ? 100.0 * double(d.pairs) / double(s.totalPossiblePairs) : 0.0;
    s.gpuCrossCheckEngineMs = d.ms_traverse;
    s.dualTreeStepMs = 0.0;
    s.parallelDfsDescentBMs = 0.0;
    s.GPUTotalTime = d.ms_total;
    s.totalCrissCrossBatches = 1;
    s.finalAabbCandidatePairs = d.candidates;
    s.confirmedGreenPairs = static_cast<size_t>(d.filter_decided);
    s.confirmedYellowPairs = static_cast<size_t>(d.escalated);
}
inline double ms_since(std::chrono::steady_clock::time_point t0)
{
    return std::chrono::duration<double, std::milli>(std::chrono::steady_clock::now() - t0).count();
}
// Copies a result's pairs into a malloc'd int2 array (caller frees with std::free).
inline void take_pairs(gi_result* r, pair2i*& out, size_t& n, const gi_ctx* c)
{
    const int32_t* p = nullptr;
    uint64_t np = 0;
    check(gi_result_pairs(r, &p, &np), c, "gi_result_pairs");
    out = nullptr;
    n = static_cast<size_t>(np);
    if (np) {
        out = static_cast<pair2i*>(std::malloc(sizeof(pair2i) * np));
        if (!out) throw Error(GI_ERR_OOM, "host allocation of the pair array");
        std::memcpy(out, p, sizeof(pair2i) * np);
    }
}
}  // namespace detail

// One intersection result of the reference's segment type
// (src/CPU/MeshIntersectionCurves.h:24-29): two FP64 endpoints and the pair.
struct IntersectionSegment {
    double p0[3], p1[3];
    int faceA, faceB;
};

class KernelBVHController {
public:
    explicit KernelBVHController(int device = 0, uint64_t hbm_budget_bytes = 0, uint32_t flags = 0)
    {
        gi_options o{device, flags, hbm_budget_bytes};
        detail::check(gi_create(&o, &ctx_), nullptr, "gi_create");
    }
    ~KernelBVHController()
    {
        clearGPU();
        if (ctx_) gi_destroy(ctx_);
    }
    KernelBVHController(const KernelBVHController&) = delete;
    KernelBVHController& operator=(const KernelBVHController&) = delete;

    // KernelBVHController.h:46-51
    template <class MeshT, class PointT>
    void construct(MeshT&, MeshT&, const PointT& centerA, const PointT& centerB, const vec3d* hVertsA,
                   int numVertsA, const tri3u* hIndicesA, int numTrianglesA, int /*levelA*/, const vec3d* hVertsB,
                   int numVertsB, const tri3u* hIndicesB, int numTrianglesB, int /*levelB*/, int /*leafThreshold*/,
                   ExecutionStats& stats)
    {
        detail::xyz(centerA, cA_);
        detail::xyz(centerB, cB_);
        hA_ = {hVertsA, numVertsA, hIndicesA, numTrianglesA};
        hB_ = {hVertsB, numVertsB, hIndicesB, numTrianglesB};
        upload(stats);
    }
    // KernelBVHController.h:53-57 (centres at the origin)
    template <class MeshT>
    void construct(MeshT& a, MeshT& b, const vec3d* hVertsA, int numVertsA, const tri3u* hIndicesA,
                   int numTrianglesA, int levelA, const vec3d* hVertsB, int numVertsB, const tri3u* hIndicesB,
                   int numTrianglesB, int levelB, int leafThreshold, ExecutionStats& stats)
    {
        construct(a, b, Point3(), Point3(), hVertsA, numVertsA, hIndicesA, numTrianglesA, levelA, hVertsB,
                  numVertsB, hIndicesB, numTrianglesB, levelB, leafThreshold, stats);
    }

    // KernelBVHController.h:60-63.  The meshes stay resident; only the current
    // poses are applied, so a new pose costs one traversal and no rebuild.
    void runIntersectionPipeline(int /*batchMultiplier*/, int /*numberOfDualTreeSteps*/,
                                 int /*activateAsyncDownload*/, pair2i*& outFinalExactPairs, size_t& outFinalCount,
                                 ExecutionStats& stats, int gpuDouble)
    {
        gi_result* r = run(want_segments_, detail::precision_for_predicate_mode(gpuDouble));
        try {
            detail::take_pairs(r, outFinalExactPairs, outFinalCount, ctx_);
            keep_segments(r);
        } catch (...) {
            gi_result_free(r);
            throw;
        }
        gi_stats st{};
        gi_result_stats(r, &st);
        detail::fill(stats, st);
        gi_result_free(r);
    }

    // KernelBVHController.h:72-77.  Stores the Euler poses (degrees, about the
    // stored centres); nothing runs on the device until the next intersection.
    void setTransformBoth(vec3d rotDegA, vec3d transA, vec3d rotDegB, vec3d transB, float& timeGPU, float& timeCPU,
                          float& timeTransformVerts, float& timeAssembleTris, float& timeGenBoxes)
    {
        const auto t0 = std::chrono::steady_clock::now();
        const double ra[3] = {rotDegA.x, rotDegA.y, rotDegA.z}, ta[3] = {transA.x, transA.y, transA.z};
        const double rb[3] = {rotDegB.x, rotDegB.y, rotDegB.z}, tb[3] = {transB.x, transB.y, transB.z};
        detail::check(gi_pose_from_euler_deg(ra, cA_, ta, &poseA_), ctx_, "gi_pose_from_euler_deg");
        detail::check(gi_pose_from_euler_deg(rb, cB_, tb, &poseB_), ctx_, "gi_pose_from_euler_deg");
        std::memcpy(rotA_, ra, sizeof ra);
        std::memcpy(transA_, ta, sizeof ta);
        std::memcpy(rotB_, rb, sizeof rb);
        std::memcpy(transB_, tb, sizeof tb);
        timeGPU = timeTransformVerts = timeAssembleTris = timeGenBoxes = 0.0f;
        timeCPU = static_cast<float>(detail::ms_since(t0));
    }
    // KernelBVHController.h:80 (legacy: translate B, keep its rotation)
    void setTranslation(double xB, double yB, double zB)
    {
        float t[5];
        setTransformBoth(vec3d{rotA_[0], rotA_[1], rotA_[2]}, vec3d{transA_[0], transA_[1], transA_[2]},
                         vec3d{rotB_[0], rotB_[1], rotB_[2]}, vec3d{xB, yB, zB}, t[0], t[1], t[2], t[3], t[4]);
    }

    // KernelBVHController.h:66-69
    void cleanup() { clearGPU(); }
    void clearGPU()
    {
        if (A_) gi_mesh_release(ctx_, A_);
        if (B_) gi_mesh_release(ctx_, B_);
        A_ = B_ = nullptr;
    }
    void reconstructGPU(ExecutionStats& stats, int, int) { reconstructGPU(stats); }
    void reconstructGPU(ExecutionStats& stats)
    {
        if (!hA_.v || !hB_.v) throw Error(GI_ERR_INVALID_ARG, "reconstructGPU before construct");
        upload(stats);
    }

    Point3 getCenterA() const { return Point3(cA_[0], cA_[1], cA_[2]); }
    Point3 getCenterB() const { return Point3(cB_[0], cB_[1], cB_[2]); }
    bool isGPUAllocated() const { return A_ != nullptr && B_ != nullptr; }

    // ---- additions over the reference interface ----
    // Segments of the last runIntersectionPipeline (computeExactIntersectionCurves,
    // src/CPU/MeshIntersectionCurves.cpp:27-91, on the device).
    void setWantSegments(bool on) { want_segments_ = on; }
    const std::vector<IntersectionSegment>& lastSegments() const { return segs_; }
    gi_ctx* context() const { return ctx_; }
    const gi_mesh* meshA() const { return A_; }
    const gi_mesh* meshB() const { return B_; }
    const gi_pose& poseA() const { return poseA_; }
    const gi_pose& poseB() const { return poseB_; }

private:
    struct HostMesh {
        const vec3d* v = nullptr;
        int nv = 0;
        const tri3u* t = nullptr;
        int nt = 0;
    };

    void upload(ExecutionStats& stats)
    {
        clearGPU();
        gi_pose_identity(&poseA_);
        gi_pose_identity(&poseB_);
        auto t0 = std::chrono::steady_clock::now();
        detail::check(gi_mesh_upload(ctx_, reinterpret_cast<const double*>(hA_.v), uint32_t(hA_.nv),
                                     reinterpret_cast<const uint32_t*>(hA_.t), uint32_t(hA_.nt), &A_),
                      ctx_, "gi_mesh_upload(A)");
        stats.buildRefitMeshAMs = detail::ms_since(t0);
        t0 = std::chrono::steady_clock::now();
        detail::check(gi_mesh_upload(ctx_, reinterpret_cast<const double*>(hB_.v), uint32_t(hB_.nv),
                                     reinterpret_cast<const uint32_t*>(hB_.t), uint32_t(hB_.nt), &B_),
                      ctx_, "gi_mesh_upload(B)");
        stats.buildRefitMeshBMs = detail::ms_since(t0);
        uint32_t nv, nt;
        uint64_t nodes, bytes;
        gi_mesh_info(A_, &nv, &nt, &nodes, &bytes);
        stats.meshATotalNodes = uint32_t(nodes);
        gi_mesh_info(B_, &nv, &nt, &nodes, &bytes);
        stats.meshBTotalNodes = uint32_t(nodes);
    }

    gi_result* run(bool segments, int32_t precision)
    {
        if (!isGPUAllocated()) throw Error(GI_ERR_INVALID_ARG, "runIntersectionPipeline before construct");
        gi_intersect_opts o;
        gi_intersect_opts_default(&o);
        o.want_segments = segments ? 1 : 0;
        o.precision_mode = precision;
        gi_result* r = nullptr;
        detail::check(gi_intersect(ctx_, A_, &poseA_, B_, &poseB_, &o, &r), ctx_, "gi_intersect");
        return r;
    }

    void keep_segments(gi_result* r)
    {
        segs_.clear();
        if (!want_segments_) return;
        const double* s = nullptr;
        const int32_t* sp = nullptr;
        uint64_t n = 0;
        detail::check(gi_result_segments(r, &s, &sp, &n), ctx_, "gi_result_segments");
        const int32_t* pairs = nullptr;
        uint64_t np = 0;
        detail::check(gi_result_pairs(r, &pairs, &np), ctx_, "gi_result_pairs");
        segs_.resize(static_cast<size_t>(n));
        for (uint64_t i = 0; i < n; ++i) {
            std::memcpy(segs_[i].p0, s + 6 * i, 3 * sizeof(double));
            std::memcpy(segs_[i].p1, s + 6 * i + 3, 3 * sizeof(double));
            const uint64_t k = static_cast<uint64_t>(sp[i]);
            if (k >= np) throw Error(GI_ERR_INVALID_ARG, "segment pair index out of range");
            segs_[i].faceA = pairs[2 * k];
            segs_[i].faceB = pairs[2 * k + 1];
        }
    }

    gi_ctx* ctx_ = nullptr;
    gi_mesh* A_ = nullptr;
    gi_mesh* B_ = nullptr;
    HostMesh hA_, hB_;
    double cA_[3] = {0, 0, 0}, cB_[3] = {0, 0, 0};
    double rotA_[3] = {0, 0, 0}, transA_[3] = {0, 0, 0}, rotB_[3] = {0, 0, 0}, transB_[3] = {0, 0, 0};
    gi_pose poseA_{}, poseB_{};
    bool want_segments_ = false;
    std::vector<IntersectionSegment> segs_;
};

// StandaloneBVHPipeline.h:27-43: one-shot upload + build + intersect + release.
// The mesh arguments and the grid / batch / mode tuning values are accepted and
// not needed.  Pairs are malloc-owned by the callee, released with std::free.
template <class MeshT, class PointT>
inline void runGridForestIntersectionPipeline(MeshT&, MeshT&, const vec3d* hVertsA, int numVertsA,
                                              const tri3u* hIndicesA, int numTrianglesA, int /*maxCellSizeA*/,
                                              const vec3d* hVertsB, int numVertsB, const tri3u* hIndicesB,
                                              int numTrianglesB, int /*maxCellSizeB*/, int /*batchMultiplier*/,
                                              int /*numberOfDualTreeSteps*/, int gpuPredicateMode,
                                              int /*leafThreshold*/, ExecutionStats& stats,
                                              pair2i*& outFinalExactPairs, size_t& outFinalCount,
                                              const PointT& centerA, const PointT& centerB, vec3d rotA, vec3d transA,
                                              vec3d rotB, vec3d transB, int device = 0)
{
    gi_options o{device, 0u, 0ull};
    gi_ctx* c = nullptr;
    detail::check(gi_create(&o, &c), nullptr, "gi_create");
    gi_result* r = nullptr;
    try {
        double ca[3], cb[3];
        detail::xyz(centerA, ca);
        detail::xyz(centerB, cb);
        const double ra[3] = {rotA.x, rotA.y, rotA.z}, ta[3] = {transA.x, transA.y, transA.z};
        const double rb[3] = {rotB.x, rotB.y, rotB.z}, tb[3] = {transB.x, transB.y, transB.z};
        gi_pose pa, pb;
        detail::check(gi_pose_from_euler_deg(ra, ca, ta, &pa), c, "gi_pose_from_euler_deg");
        detail::check(gi_pose_from_euler_deg(rb, cb, tb, &pb), c, "gi_pose_from_euler_deg");
        gi_intersect_opts io;
        gi_intersect_opts_default(&io);
        io.want_segments = 0;
        io.precision_mode = detail::precision_for_predicate_mode(gpuPredicateMode);
        detail::check(gi_intersect_oneshot(c, reinterpret_cast<const double*>(hVertsA), uint32_t(numVertsA),
                                           reinterpret_cast<const uint32_t*>(hIndicesA), uint32_t(numTrianglesA),
                                           &pa, reinterpret_cast<const double*>(hVertsB), uint32_t(numVertsB),
                                           reinterpret_cast<const uint32_t*>(hIndicesB), uint32_t(numTrianglesB),
                                           &pb, &io, &r),
                      c, "gi_intersect_oneshot");
        detail::take_pairs(r, outFinalExactPairs, outFinalCount, c);
        gi_stats st{};
        gi_result_stats(r, &st);
        detail::fill(stats, st);
    } catch (...) {
        if (r) gi_result_free(r);
        gi_destroy(c);
        throw;
    }
    gi_result_free(r);
    gi_destroy(c);
}

}  // namespace gi

#endif
