// gi_suite.hpp -- seeded pose-sweep verification harness, header-only C++17
// over gi_controller.hpp: the counterpart of the reference's TestSuite
// (src/CPU/TestSuite.h:9-131, src/CPU/TestSuite.cpp:22-596).
//
// runSuite() keeps A at its base pose and perturbs B per step with the poses
// of gi_sweep_poses (the reference's std::mt19937 draws, TestSuite.cpp:
// 478-505).  Each step (evaluateStep, TestSuite.cpp:235-321) runs
//  * the ground truth: a caller-supplied exact intersector over the posed
//    vertex arrays (the reference runs CGAL's compute_face_face_intersection
//    on the transformed meshes, TestSuite.cpp:79-102);
//  * optionally a second reference of the caller's (the reference's CGAL
//    parallel run, TestSuite.cpp:104-124);
//  * the persistent controller path: setTransformBoth + runIntersectionPipeline
//    on the resident meshes (TestSuite.cpp:126-161);
//  * the one-shot path: runGridForestIntersectionPipeline on the posed arrays
//    with zero rotations and translations, as the reference calls it
//    (TestSuite.cpp:181-233);
// and compares pair sets (exact match; false positives and negatives of the
// controller path), computes the candidate yield and the surface overlap
// ratio Omega = area of the faces in the truth / total area of both meshes,
// on the unposed meshes (TestSuite.cpp:34-77).  A line per step and a
// consensus summary go to the log; the reference's three CSV files are
// written (exportToCSV, exportStandardComputeCSV, exportStandaloneComputeCSV,
// TestSuite.cpp:323-443) with its headers and 10 significant digits.
//
// Differences a caller sees:
//  * the CGAL stages are the caller's callbacks; the reference's column names
//    cgal_classic_ms / cgal_parallel_ms / cgal_parallel_match are kept for
//    them;
//  * the breakdown CSVs keep the reference's columns; stages this library
//    does not have (cross check, dual-tree steps, DFS descent, CPU narrow
//    phase, workspace clean-up) are 0, aabb_candidate_exec_ms is the fused
//    traversal + first filter, gpu_double_predicates_ms the FP64 / exact stage,
//    thrust_compaction_d2h_ms the output ordering, and orange pairs (CPU
//    fallback) are 0; columns of this library's own follow the reference's;
//  * derived file names use the extension of the file name only
//    ("out.d/run" -> "out.d/run_standard_breakdown.csv").
#ifndef GI_GI_SUITE_HPP
#define GI_GI_SUITE_HPP

#include <algorithm>
#include <chrono>
#include <cmath>
#include <cstdio>
#include <functional>
#include <ostream>
#include <string>
#include <unordered_set>
#include <utility>
#include <vector>

#include "gi_controller.hpp"

namespace gi {

// TestSuite.h:9-25
struct TestConfig {
    int numSteps = 10;
    double maxTranslation = 0.5;
    double maxRotationDeg = 15.0;
    int enableGpuPrecision = 1;  // predicate mode of the controller path (reference modes 0-4; 5 = plain FP64)
    unsigned int seed = 1337;
    std::string csvOutputPath = "benchmark_results.csv";
    bool testMainGpuPipeline = true;
    bool testStandalonePipeline = true;
    bool testCgalParallel = true;  // run the second reference, when one is given
};

// TestSuite.h:27-56
struct VerificationResult {
    int stepIndex = 0;
    vec3d rotA{}, transA{}, rotB{}, transB{};
    size_t totalPossiblePairs = 0;
    size_t groundTruthCount = 0;
    size_t candidatePairs = 0;
    double candidateYield = 0.0;
    double surfaceOverlapRatio = 0.0;

    double cgalClassicTimeMs = 0.0;  // ground truth
    double cgalParallelTimeMs = 0.0; // second reference
    size_t cgalParallelCount = 0;
    bool cgalParallelExactMatch = false;

    double gpuMainTimeMs = 0.0;
    size_t gpuMainCount = 0;
    bool gpuMainExactMatch = false;
    size_t mainFalsePositives = 0;
    size_t mainFalseNegatives = 0;
    ExecutionStats mainStats;

    double standaloneTimeMs = 0.0;
    size_t standaloneCount = 0;
    bool standaloneExactMatch = false;
    size_t standaloneFalsePositives = 0;
    size_t standaloneFalseNegatives = 0;
    ExecutionStats standaloneStats;
};

class TestSuite {
public:
    using PairList = std::vector<std::pair<int, int>>;
    // An intersector over posed vertex arrays (3 doubles per vertex, 3 indices per triangle).
    using ReferenceFn = std::function<PairList(const double* vA, uint32_t nvA, const uint32_t* tA, uint32_t ntA,
                                               const double* vB, uint32_t nvB, const uint32_t* tB, uint32_t ntB)>;

    // `ctl` has been constructed on the same host arrays (its centres are the
    // rotation centres of the poses); the arrays stay alive while the suite runs.
    TestSuite(KernelBVHController& ctl, const vec3d* vA, int nvA, const tri3u* tA, int ntA, const vec3d* vB, int nvB,
              const tri3u* tB, int ntB, ReferenceFn groundTruth, ReferenceFn cgalParallel = nullptr)
        : ctl_(ctl), A_{vA, nvA, tA, ntA}, B_{vB, nvB, tB, ntB}, truth_(std::move(groundTruth)),
          parallel_(std::move(cgalParallel))
    {
        if (!truth_) throw Error(GI_ERR_INVALID_ARG, "TestSuite needs a ground-truth intersector");
        areaA_ = face_areas(A_, totalA_);
        areaB_ = face_areas(B_, totalB_);
    }

    // TestSuite.cpp:455-596.  Returns the per-step results; all three CSVs are written.
    std::vector<VerificationResult> runSuite(const TestConfig& config, vec3d baseRotA = {}, vec3d baseTransA = {},
                                             vec3d baseRotB = {}, vec3d baseTransB = {}, std::ostream* log = nullptr)
    {
        const int n = std::max(0, config.numSteps);
        std::vector<double> rot(3 * size_t(n)), trans(3 * size_t(n));
        const double br[3] = {baseRotB.x, baseRotB.y, baseRotB.z}, bt[3] = {baseTransB.x, baseTransB.y, baseTransB.z};
        detail::check(gi_sweep_poses(config.seed, uint32_t(n), config.maxRotationDeg, config.maxTranslation, br, bt,
                                     rot.data(), trans.data()),
                      nullptr, "gi_sweep_poses");
        std::vector<VerificationResult> all;
        all.reserve(size_t(n));
        int agreed = 0;
        for (int i = 0; i < n; ++i) {
            const vec3d rotB{rot[3 * i], rot[3 * i + 1], rot[3 * i + 2]};
            const vec3d transB{trans[3 * i], trans[3 * i + 1], trans[3 * i + 2]};
            all.push_back(evaluateStep(i, baseRotA, baseTransA, rotB, transB, config));
            const bool same = coincided(all.back(), config);
            agreed += same;
            if (log) print_step(*log, all.back(), config, same);
        }
        if (log) {
            char b[160];
            *log << "  Total Steps Run          : " << n << "\n";
            std::snprintf(b, sizeof b, "  Steps with Full Consensus: %d / %d (%.1f%%)\n", agreed, n,
                          n ? 100.0 * agreed / n : 0.0);
            *log << b;
        }
        exportToCSV(config.csvOutputPath, all);
        exportStandardComputeCSV(deriveFilename(config.csvOutputPath, "_standard_breakdown"), all);
        exportStandaloneComputeCSV(deriveFilename(config.csvOutputPath, "_standalone_breakdown"), all);
        return all;
    }

    // TestSuite.cpp:235-321
    VerificationResult evaluateStep(int stepIdx, vec3d rotA, vec3d transA, vec3d rotB, vec3d transB,
                                    const TestConfig& config)
    {
        VerificationResult res;
        res.stepIndex = stepIdx;
        res.rotA = rotA;
        res.transA = transA;
        res.rotB = rotB;
        res.transB = transB;
        res.totalPossiblePairs = size_t(A_.nt) * size_t(B_.nt);

        const Point3 cA = ctl_.getCenterA(), cB = ctl_.getCenterB();
        const std::vector<double> pA = posed(A_, cA, rotA, transA), pB = posed(B_, cB, rotB, transB);
        auto call = [&](const ReferenceFn& f, double& ms) {
            const auto t0 = std::chrono::steady_clock::now();
            PairList p = f(pA.data(), uint32_t(A_.nv), reinterpret_cast<const uint32_t*>(A_.t), uint32_t(A_.nt),
                           pB.data(), uint32_t(B_.nv), reinterpret_cast<const uint32_t*>(B_.t), uint32_t(B_.nt));
            ms = detail::ms_since(t0);
            return canonical(std::move(p));
        };
        const PairList truth = call(truth_, res.cgalClassicTimeMs);
        res.groundTruthCount = truth.size();
        res.surfaceOverlapRatio = overlap_ratio(truth);

        if (config.testCgalParallel && parallel_) {
            const PairList p = call(parallel_, res.cgalParallelTimeMs);
            res.cgalParallelCount = p.size();
            res.cgalParallelExactMatch = p == truth;
        }
        if (config.testMainGpuPipeline) {
            if (!ctl_.isGPUAllocated()) ctl_.reconstructGPU(res.mainStats);
            const auto t0 = std::chrono::steady_clock::now();
            float t[5];
            ctl_.setTransformBoth(rotA, transA, rotB, transB, t[0], t[1], t[2], t[3], t[4]);
            pair2i* out = nullptr;
            size_t cnt = 0;
            ctl_.runIntersectionPipeline(1, 0, 0, out, cnt, res.mainStats, config.enableGpuPrecision);
            res.gpuMainTimeMs = detail::ms_since(t0);
            const PairList got = take(out, cnt);
            res.gpuMainCount = got.size();
            res.gpuMainExactMatch = got == truth;
            diff(got, truth, res.mainFalsePositives, res.mainFalseNegatives);
            res.candidatePairs = size_t(res.mainStats.finalAabbCandidatePairs);
        }
        if (config.testStandalonePipeline) {
            const auto t0 = std::chrono::steady_clock::now();
            pair2i* out = nullptr;
            size_t cnt = 0;
            struct NoMesh {
            } ma, mb;
            const vec3d zero{0.0, 0.0, 0.0};
            runGridForestIntersectionPipeline(ma, mb, reinterpret_cast<const vec3d*>(pA.data()), A_.nv, A_.t, A_.nt,
                                              0, reinterpret_cast<const vec3d*>(pB.data()), B_.nv, B_.t, B_.nt, 0, 1,
                                              0, config.enableGpuPrecision, 4, res.standaloneStats, out, cnt, cA, cB,
                                              zero, zero, zero, zero);
            res.standaloneTimeMs = detail::ms_since(t0);
            const PairList got = take(out, cnt);
            res.standaloneCount = got.size();
            res.standaloneExactMatch = got == truth;
            diff(got, truth, res.standaloneFalsePositives, res.standaloneFalseNegatives);
            if (!config.testMainGpuPipeline) res.candidatePairs = size_t(res.standaloneStats.finalAabbCandidatePairs);
        }
        if (res.totalPossiblePairs > 0)
            res.candidateYield = double(res.candidatePairs) / double(res.totalPossiblePairs);
        return res;
    }

    // TestSuite.cpp:323-356
    static bool exportToCSV(const std::string& path, const std::vector<VerificationResult>& results)
    {
        FILE* f = std::fopen(path.c_str(), "w");
        if (!f) return false;
        std::fputs("step,intersections,candidates,total_possible_pairs,candidate_yield,surface_overlap_omega,"
                   "hybrid_ms,hybrid_standalone_ms,cgal_classic_ms,cgal_parallel_ms,"
                   "hybrid_match,standalone_match,cgal_parallel_match\n",
                   f);
        for (const auto& r : results)
            std::fprintf(f, "%d,%zu,%zu,%zu,%.10g,%.10g,%.10g,%.10g,%.10g,%.10g,%d,%d,%d\n", r.stepIndex,
                         r.groundTruthCount, r.candidatePairs, r.totalPossiblePairs, r.candidateYield,
                         r.surfaceOverlapRatio, r.gpuMainTimeMs, r.standaloneTimeMs, r.cgalClassicTimeMs,
                         r.cgalParallelTimeMs, r.gpuMainExactMatch ? 1 : 0, r.standaloneExactMatch ? 1 : 0,
                         r.cgalParallelExactMatch ? 1 : 0);
        return std::fclose(f) == 0;
    }

    // TestSuite.cpp:358-398
    static bool exportStandardComputeCSV(const std::string& path, const std::vector<VerificationResult>& results)
    {
        FILE* f = std::fopen(path.c_str(), "w");
        if (!f) return false;
        std::fputs("step,gpu_total_ms,cross_check_engine_ms,dual_tree_step_ms,parallel_dfs_descent_ms,"
                   "preallocate_ms,assembly_phase_ms,aabb_candidate_exec_ms,gpu_float_predicates_ms,"
                   "gpu_double_predicates_ms,thrust_compaction_d2h_ms,cpu_narrow_phase_ms,"
                   "loop_workspace_cleanup_ms,explicit_cleanup_sync_ms,"
                   "confirmed_green_pairs,confirmed_yellow_pairs,confirmed_orange_pairs",
                   f);
        std::fputs(kExtraHeader, f);
        for (const auto& r : results) {
            const gi_stats& d = r.mainStats.detail;
            std::fprintf(f, "%d,%.10g,0,0,0,0,0,%.10g,0,%.10g,%.10g,0,0,0,%zu,%zu,0", r.stepIndex, d.ms_total,
                         d.ms_traverse, d.ms_exact, d.ms_sort, r.mainStats.confirmedGreenPairs,
                         r.mainStats.confirmedYellowPairs);
            extra(f, r.mainStats, r.gpuMainTimeMs);
        }
        return std::fclose(f) == 0;
    }

    // TestSuite.cpp:400-443
    static bool exportStandaloneComputeCSV(const std::string& path, const std::vector<VerificationResult>& results)
    {
        FILE* f = std::fopen(path.c_str(), "w");
        if (!f) return false;
        std::fputs("step,gpu_total_ms,raw_alloc_copy_ms,thrust_init_overhead_ms,build_refit_mesh_a_ms,"
                   "build_refit_mesh_b_ms,cross_check_engine_ms,dual_tree_step_ms,parallel_dfs_descent_ms,"
                   "preallocate_ms,assembly_phase_ms,aabb_candidate_exec_ms,gpu_float_predicates_ms,"
                   "gpu_double_predicates_ms,thrust_compaction_d2h_ms,cpu_narrow_phase_ms,loop_workspace_cleanup_ms,"
                   "explicit_cleanup_sync_ms,confirmed_green_pairs,confirmed_yellow_pairs,confirmed_orange_pairs",
                   f);
        std::fputs(kExtraHeader, f);
        for (const auto& r : results) {
            const gi_stats& d = r.standaloneStats.detail;
            std::fprintf(f, "%d,%.10g,0,0,0,0,0,0,0,0,0,%.10g,0,%.10g,%.10g,0,0,0,%zu,%zu,0", r.stepIndex,
                         d.ms_total, d.ms_traverse, d.ms_exact, d.ms_sort, r.standaloneStats.confirmedGreenPairs,
                         r.standaloneStats.confirmedYellowPairs);
            extra(f, r.standaloneStats, r.standaloneTimeMs);
        }
        return std::fclose(f) == 0;
    }

    // TestSuite.cpp:445-453, with the extension taken from the file name only
    static std::string deriveFilename(const std::string& base, const std::string& suffix)
    {
        const size_t slash = base.find_last_of("/\\");
        const size_t dot = base.find_last_of('.');
        if (dot == std::string::npos || (slash != std::string::npos && dot < slash) ||
            dot == (slash == std::string::npos ? 0 : slash + 1))
            return base + suffix + ".csv";
        return base.substr(0, dot) + suffix + ".csv";
    }

private:
    struct HostMesh {
        const vec3d* v;
        int nv;
        const tri3u* t;
        int nt;
    };

    static constexpr const char* kExtraHeader =
        ",segments_ms,call_wall_ms,candidates,node_pairs,escalated,exact_signs,exact_points,pairs,levels,launches,"
        "traverse_shape\n";

    static void extra(FILE* f, const ExecutionStats& s, double wall_ms)
    {
        const gi_stats& d = s.detail;
        std::fprintf(f, ",%.10g,%.10g,%llu,%llu,%llu,%llu,%llu,%llu,%u,%u,%u\n", d.ms_segments, wall_ms,
                     (unsigned long long)d.candidates, (unsigned long long)d.node_pairs,
                     (unsigned long long)d.escalated, (unsigned long long)d.exact_signs,
                     (unsigned long long)d.exact_points, (unsigned long long)d.pairs, d.levels, d.launches,
                     d.traverse_shape);
    }

    static std::vector<double> face_areas(const HostMesh& m, double& total)
    {
        std::vector<double> a(size_t(std::max(0, m.nt)));
        total = 0.0;
        for (int f = 0; f < m.nt; ++f) {
            const vec3d &p = m.v[m.t[f].x], &q = m.v[m.t[f].y], &r = m.v[m.t[f].z];
            const double ux = q.x - p.x, uy = q.y - p.y, uz = q.z - p.z;
            const double wx = r.x - p.x, wy = r.y - p.y, wz = r.z - p.z;
            const double cx = uy * wz - uz * wy, cy = uz * wx - ux * wz, cz = ux * wy - uy * wx;
            a[size_t(f)] = 0.5 * std::sqrt(cx * cx + cy * cy + cz * cz);
            total += a[size_t(f)];
        }
        return a;
    }

    double overlap_ratio(const PairList& truth) const
    {
        if (truth.empty() || totalA_ + totalB_ <= 0.0) return 0.0;
        std::unordered_set<int> fa, fb;
        for (const auto& p : truth) {
            fa.insert(p.first);
            fb.insert(p.second);
        }
        double s = 0.0;
        for (int f : fa)
            if (f >= 0 && f < A_.nt) s += areaA_[size_t(f)];
        for (int f : fb)
            if (f >= 0 && f < B_.nt) s += areaB_[size_t(f)];
        return s / (totalA_ + totalB_);
    }

    static std::vector<double> posed(const HostMesh& m, const Point3& c, vec3d rot, vec3d trans)
    {
        const double r[3] = {rot.x, rot.y, rot.z}, t[3] = {trans.x, trans.y, trans.z}, cc[3] = {c.x(), c.y(), c.z()};
        gi_pose p;
        detail::check(gi_pose_from_euler_deg(r, cc, t, &p), nullptr, "gi_pose_from_euler_deg");
        std::vector<double> out(3 * size_t(std::max(0, m.nv)));
        detail::check(gi_pose_apply(&p, reinterpret_cast<const double*>(m.v), uint64_t(m.nv), out.data()), nullptr,
                      "gi_pose_apply");
        return out;
    }

    static PairList canonical(PairList p)
    {
        std::sort(p.begin(), p.end());
        p.erase(std::unique(p.begin(), p.end()), p.end());
        return p;
    }

    static PairList take(pair2i* out, size_t n)
    {
        PairList p(n);
        for (size_t i = 0; i < n; ++i) p[i] = {out[i].x, out[i].y};
        std::free(out);
        return canonical(std::move(p));
    }

    // TestSuite.cpp:285-296: both lists sorted and duplicate-free
    static void diff(const PairList& got, const PairList& truth, size_t& fp, size_t& fn)
    {
        PairList tmp;
        std::set_difference(got.begin(), got.end(), truth.begin(), truth.end(), std::back_inserter(tmp));
        fp = tmp.size();
        tmp.clear();
        std::set_difference(truth.begin(), truth.end(), got.begin(), got.end(), std::back_inserter(tmp));
        fn = tmp.size();
    }

    // the reference compares counts (TestSuite.cpp:507-519); here the pair sets
    bool coincided(const VerificationResult& r, const TestConfig& c) const
    {
        bool ok = true;
        if (c.testCgalParallel && parallel_ && !r.cgalParallelExactMatch) ok = false;
        if (c.testMainGpuPipeline && !r.gpuMainExactMatch) ok = false;
        if (c.testStandalonePipeline && !r.standaloneExactMatch) ok = false;
        return ok;
    }

    void print_step(std::ostream& os, const VerificationResult& r, const TestConfig& c, bool same) const
    {
        char b[512];
        std::snprintf(b, sizeof b,
                      "test %3d:\n  [Transform A] Rot(deg)=(%.16g, %.16g, %.16g) | Trans=(%.16g, %.16g, %.16g)\n"
                      "  [Transform B] Rot(deg)=(%.16g, %.16g, %.16g) | Trans=(%.16g, %.16g, %.16g)\n",
                      r.stepIndex, r.rotA.x, r.rotA.y, r.rotA.z, r.transA.x, r.transA.y, r.transA.z, r.rotB.x,
                      r.rotB.y, r.rotB.z, r.transB.x, r.transB.y, r.transB.z);
        os << b;
        std::snprintf(b, sizeof b, "  [Results]     Truth=%4zu", r.groundTruthCount);
        os << b;
        if (c.testCgalParallel && parallel_) {
            std::snprintf(b, sizeof b, " | Parallel=%4zu", r.cgalParallelCount);
            os << b;
        }
        if (c.testMainGpuPipeline) {
            std::snprintf(b, sizeof b, " | Controller=%4zu (fp %zu, fn %zu)", r.gpuMainCount, r.mainFalsePositives,
                          r.mainFalseNegatives);
            os << b;
        }
        if (c.testStandalonePipeline) {
            std::snprintf(b, sizeof b, " | Standalone=%4zu", r.standaloneCount);
            os << b;
        }
        std::snprintf(b, sizeof b,
                      " | %s\n  [Metrics]     Omega=%.2f%% | Controller_t=%.2fms | Standalone_t=%.2fms | "
                      "Truth_t=%.2fms\n\n",
                      same ? "[ALL COINCIDED]" : "[DISTINCTIONS FOUND]", r.surfaceOverlapRatio * 100.0,
                      r.gpuMainTimeMs, r.standaloneTimeMs, r.cgalClassicTimeMs);
        os << b;
    }

    KernelBVHController& ctl_;
    HostMesh A_, B_;
    ReferenceFn truth_, parallel_;
    std::vector<double> areaA_, areaB_;
    double totalA_ = 0.0, totalB_ = 0.0;
};

}  // namespace gi

#endif
