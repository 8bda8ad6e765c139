// run_suite.cpp -- drives the pose-sweep harness gi::TestSuite
// (include/gi/gi_suite.hpp) with the exact CPU oracle as the ground truth and
// the oracle on all threads as the second reference, the way the reference's
// REPL drives TestSuite::runSuite (src/CPU/TestSuite.cpp:455-596) with CGAL.
// Test infrastructure: the oracle is the checker, never the thing measured.
//
// After the sweep, every step's pose is run once more on the controller with
// segments on and the segments are compared with the oracle's (the reference's
// curve output, src/CPU/MeshIntersectionCurves.cpp:27-91).
//
// Usage: run_suite [steps] [seed] [maxRotDeg] [maxTrans] [csv] [segments(0|1)]
// Exit status 0 iff every step matched exactly.
#include <algorithm>
#include <cmath>
#include <cstdio>
#include <cstdlib>
#include <iostream>
#include <string>
#include <vector>

#include "gi/gi_suite.hpp"

extern "C" {
#include "gi_oracle.h"
}

namespace {

struct HostMesh {
    std::vector<gi::vec3d> v;
    std::vector<gi::tri3u> t;
};

// UV sphere: 2 poles + (rings-1) rings of `seg` vertices, 2*seg*(rings-1) triangles.
HostMesh uv_sphere(int seg, int rings, double r)
{
    const double kPi = 3.14159265358979323846;
    HostMesh m;
    m.v.push_back({0.0, 0.0, r});
    for (int i = 1; i < rings; ++i) {
        const double phi = kPi * i / rings;
        for (int j = 0; j < seg; ++j) {
            const double th = 2.0 * kPi * j / seg;
            m.v.push_back({r * std::sin(phi) * std::cos(th), r * std::sin(phi) * std::sin(th), r * std::cos(phi)});
        }
    }
    m.v.push_back({0.0, 0.0, -r});
    const unsigned north = 0, south = unsigned(m.v.size() - 1);
    auto idx = [&](int i, int j) { return unsigned(1 + i * seg + (j % seg)); };
    for (int j = 0; j < seg; ++j) m.t.push_back({north, idx(0, j), idx(0, j + 1)});
    for (int i = 0; i < rings - 2; ++i)
        for (int j = 0; j < seg; ++j) {
            m.t.push_back({idx(i, j), idx(i + 1, j), idx(i, j + 1)});
            m.t.push_back({idx(i, j + 1), idx(i + 1, j), idx(i + 1, j + 1)});
        }
    for (int j = 0; j < seg; ++j) m.t.push_back({south, idx(rings - 2, j + 1), idx(rings - 2, j)});
    return m;
}

struct OracleOut {
    int32_t* pairs = nullptr;
    uint64_t npairs = 0;
    double* segs = nullptr;
    int32_t* seg_pair = nullptr;
    uint64_t nsegs = 0;
    ~OracleOut()
    {
        oc_free(pairs);
        oc_free(segs);
        oc_free(seg_pair);
    }
};

// the oracle over posed arrays (identity poses)
bool oracle_run(const double* vA, uint32_t nvA, const uint32_t* tA, uint32_t ntA, const double* vB, uint32_t nvB,
                const uint32_t* tB, uint32_t ntB, int segments, int nthreads, OracleOut& o)
{
    oc_pose id;
    oc_pose_identity(&id);
    oc_stats st;
    return oc_intersect_meshes(vA, nvA, tA, ntA, &id, vB, nvB, tB, ntB, &id, segments, nthreads, 0, &o.pairs,
                               &o.npairs, &o.segs, &o.seg_pair, &o.nsegs, &st) == 0;
}

gi::TestSuite::ReferenceFn oracle_fn(int nthreads)
{
    return [nthreads](const double* vA, uint32_t nvA, const uint32_t* tA, uint32_t ntA, const double* vB,
                      uint32_t nvB, const uint32_t* tB, uint32_t ntB) {
        OracleOut o;
        if (!oracle_run(vA, nvA, tA, ntA, vB, nvB, tB, ntB, 0, nthreads, o))
            throw gi::Error(GI_ERR_INVALID_ARG, "oracle failed");
        gi::TestSuite::PairList p(o.npairs);
        for (uint64_t k = 0; k < o.npairs; ++k) p[k] = {o.pairs[2 * k], o.pairs[2 * k + 1]};
        return p;
    };
}

using SegKey = std::vector<double>;

SegKey seg_key(const double* a, const double* b, int fa, int fb)
{
    SegKey k{double(fa), double(fb)};
    const bool sw = std::lexicographical_compare(b, b + 3, a, a + 3);
    const double* lo = sw ? b : a;
    const double* hi = sw ? a : b;
    k.insert(k.end(), lo, lo + 3);
    k.insert(k.end(), hi, hi + 3);
    return k;
}

}  // namespace

int main(int argc, char** argv)
{
    gi::TestConfig cfg;
    cfg.numSteps = argc > 1 ? std::atoi(argv[1]) : 10;
    cfg.seed = argc > 2 ? unsigned(std::strtoul(argv[2], nullptr, 10)) : 1337u;
    cfg.maxRotationDeg = argc > 3 ? std::atof(argv[3]) : 15.0;
    cfg.maxTranslation = argc > 4 ? std::atof(argv[4]) : 0.5;
    cfg.csvOutputPath = argc > 5 ? argv[5] : "run_suite.csv";
    const bool segments = argc > 6 ? std::atoi(argv[6]) != 0 : true;

    HostMesh A = uv_sphere(128, 80, 1.0), B = uv_sphere(128, 80, 1.0);
    struct NoMesh {
    } ma, mb;  // the reference passes CGAL meshes here; unused
    gi::ExecutionStats st;
    gi::KernelBVHController ctl(0);
    const gi::Point3 cA(0.0, 0.0, 0.0), cB(0.5, 0.0, 0.0);
    ctl.construct(ma, mb, cA, cB, A.v.data(), int(A.v.size()), A.t.data(), int(A.t.size()), 6, B.v.data(),
                  int(B.v.size()), B.t.data(), int(B.t.size()), 6, 4, st);

    gi::TestSuite suite(ctl, A.v.data(), int(A.v.size()), A.t.data(), int(A.t.size()), B.v.data(), int(B.v.size()),
                        B.t.data(), int(B.t.size()), oracle_fn(1), oracle_fn(0));
    const gi::vec3d zero{0, 0, 0}, baseTransB{0.5, 0, 0};
    const auto res = suite.runSuite(cfg, zero, zero, zero, baseTransB, &std::cout);

    int agreed = 0;
    for (const auto& r : res)
        agreed += r.gpuMainExactMatch && r.standaloneExactMatch && r.cgalParallelExactMatch &&
                  r.mainFalsePositives == 0 && r.mainFalseNegatives == 0;

    // segments of the controller path against the oracle's, on the same poses
    int seg_ok = 0;
    if (segments) {
        ctl.setWantSegments(true);
        int step = 0;
        for (const auto& r : res) {
            float t[5];
            ctl.setTransformBoth(r.rotA, r.transA, r.rotB, r.transB, t[0], t[1], t[2], t[3], t[4]);
            gi::pair2i* p = nullptr;
            size_t n = 0;
            // the reference's predicate modes 0-4 (FP32 cascade) and the plain FP64 mode in turn
            const int mode = (step % 2) ? gi::detail::kPredicateModePlainFP64 : (step / 2) % 5;
            ++step;
            ctl.runIntersectionPipeline(1, 0, 0, p, n, st, mode);
            std::free(p);
            std::vector<double> pA(3 * A.v.size()), pB(3 * B.v.size());
            gi_pose_apply(&ctl.poseA(), reinterpret_cast<const double*>(A.v.data()), A.v.size(), pA.data());
            gi_pose_apply(&ctl.poseB(), reinterpret_cast<const double*>(B.v.data()), B.v.size(), pB.data());
            OracleOut o;
            if (!oracle_run(pA.data(), uint32_t(A.v.size()), reinterpret_cast<const uint32_t*>(A.t.data()),
                            uint32_t(A.t.size()), pB.data(), uint32_t(B.v.size()),
                            reinterpret_cast<const uint32_t*>(B.t.data()), uint32_t(B.t.size()), 1, 0, o))
                return 2;
            std::vector<SegKey> g, w;
            for (const auto& s : ctl.lastSegments()) g.push_back(seg_key(s.p0, s.p1, s.faceA, s.faceB));
            for (uint64_t k = 0; k < o.nsegs; ++k) {
                const int32_t pi = o.seg_pair[k];
                w.push_back(seg_key(o.segs + 6 * k, o.segs + 6 * k + 3, o.pairs[2 * pi], o.pairs[2 * pi + 1]));
            }
            std::sort(g.begin(), g.end());
            std::sort(w.begin(), w.end());
            seg_ok += g == w;
        }
        std::printf("segments identical on %d / %zu steps\n", seg_ok, res.size());
    }
    std::printf("%d / %zu steps matched\n", agreed, res.size());
    const bool ok = agreed == int(res.size()) && (!segments || seg_ok == int(res.size()));
    return ok ? 0 : 1;
}
