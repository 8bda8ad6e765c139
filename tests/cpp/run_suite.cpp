// run_suite.cpp -- pose-sweep verification harness in C++ over gi_controller.hpp.
//
// Mirrors the reference's TestSuite::runSuite (src/CPU/TestSuite.cpp:455-596):
// a seeded std::mt19937 perturbs B's Euler rotation and translation around a
// base pose for numSteps steps; every step runs the persistent controller
// (KernelBVHController path) and the one-shot pipeline
// (runGridForestIntersectionPipeline path) and compares both with the ground
// truth, here the exact CPU oracle (the reference uses CGAL).  The comparison
// is on the pair sets (false positives / false negatives, as
// src/CPU/TestSuite.cpp:285-296 counts them), not only on the counts.  One CSV
// row per step.  Exit status 0 iff every step matched exactly.
//
// Usage: run_suite [steps] [seed] [maxRotDeg] [maxTrans] [csv] [segments(0|1)]
#include <algorithm>
#include <chrono>
#include <cmath>
#include <cstdio>
#include <cstdlib>
#include <random>
#include <set>
#include <string>
#include <utility>
#include <vector>

#include "gi/gi_controller.hpp"

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

using PairSet = std::set<std::pair<int, int>>;

PairSet to_set(const gi::pair2i* p, size_t n)
{
    PairSet s;
    for (size_t i = 0; i < n; ++i) s.insert({p[i].x, p[i].y});
    return s;
}

void diff(const PairSet& got, const PairSet& truth, size_t& fp, size_t& fn)
{
    fp = fn = 0;
    for (auto& p : got) fp += truth.count(p) == 0;
    for (auto& p : truth) fn += got.count(p) == 0;
}

double now_ms()
{
    return std::chrono::duration<double, std::milli>(std::chrono::steady_clock::now().time_since_epoch()).count();
}

}  // namespace

int main(int argc, char** argv)
{
    const int steps = argc > 1 ? std::atoi(argv[1]) : 10;
    const unsigned seed = argc > 2 ? unsigned(std::strtoul(argv[2], nullptr, 10)) : 42u;
    const double maxRot = argc > 3 ? std::atof(argv[3]) : 30.0;
    const double maxTrans = argc > 4 ? std::atof(argv[4]) : 0.25;
    const std::string csv = argc > 5 ? argv[5] : "run_suite.csv";
    const bool segments = argc > 6 ? std::atoi(argv[6]) != 0 : true;

    HostMesh A = uv_sphere(128, 80, 1.0), B = uv_sphere(128, 80, 1.0);
    struct NoMesh {} ma, mb;  // the reference passes CGAL meshes here; unused
    gi::ExecutionStats st;
    gi::KernelBVHController ctl(0);
    ctl.setWantSegments(segments);
    ctl.construct(ma, mb, gi::Point3(0, 0, 0), gi::Point3(0, 0, 0), A.v.data(), int(A.v.size()), A.t.data(),
                  int(A.t.size()), 6, B.v.data(), int(B.v.size()), B.t.data(), int(B.t.size()), 6, 4, st);

    const gi::vec3d baseRotA{0, 0, 0}, baseTransA{0, 0, 0}, baseRotB{0, 0, 0}, baseTransB{0.5, 0, 0};
    std::mt19937 rng(seed);
    std::uniform_real_distribution<double> rotDist(-maxRot, maxRot), transDist(-maxTrans, maxTrans);

    FILE* f = std::fopen(csv.c_str(), "w");
    if (f)
        std::fprintf(f, "step,rotBx,rotBy,rotBz,transBx,transBy,transBz,truth,controller,standalone,fp,fn,"
                        "fp_standalone,fn_standalone,segments,controller_ms,standalone_ms,oracle_ms\n");
    int agreed = 0;
    for (int i = 0; i < steps; ++i) {
        gi::vec3d rotB{baseRotB.x + rotDist(rng), baseRotB.y + rotDist(rng), baseRotB.z + rotDist(rng)};
        gi::vec3d transB{baseTransB.x + transDist(rng), baseTransB.y + transDist(rng), baseTransB.z + transDist(rng)};
        float t0, t1, t2, t3, t4;
        ctl.setTransformBoth(baseRotA, baseTransA, rotB, transB, t0, t1, t2, t3, t4);

        double c0 = now_ms();
        gi::pair2i* pairs = nullptr;
        size_t n = 0;
        ctl.runIntersectionPipeline(1, 0, 0, pairs, n, st, 0);
        const double ctl_ms = now_ms() - c0;
        PairSet got = to_set(pairs, n);
        std::free(pairs);

        c0 = now_ms();
        gi::pair2i* p2 = nullptr;
        size_t n2 = 0;
        gi::ExecutionStats st2;
        gi::runGridForestIntersectionPipeline(ma, mb, A.v.data(), int(A.v.size()), A.t.data(), int(A.t.size()), 64,
                                              B.v.data(), int(B.v.size()), B.t.data(), int(B.t.size()), 64, 1, 0, 0,
                                              4, st2, p2, n2, gi::Point3(0, 0, 0), gi::Point3(0, 0, 0), baseRotA,
                                              baseTransA, rotB, transB);
        const double sa_ms = now_ms() - c0;
        PairSet got2 = to_set(p2, n2);
        std::free(p2);

        // ground truth: the exact oracle under the same Euler poses
        const double ra[3] = {baseRotA.x, baseRotA.y, baseRotA.z}, ta[3] = {baseTransA.x, baseTransA.y, baseTransA.z};
        const double rb[3] = {rotB.x, rotB.y, rotB.z}, tb[3] = {transB.x, transB.y, transB.z};
        const double zero[3] = {0, 0, 0};
        oc_pose pa, pb;
        oc_pose_from_euler_deg(ra, zero, ta, &pa);
        oc_pose_from_euler_deg(rb, zero, tb, &pb);
        int32_t* op = nullptr;
        uint64_t on = 0;
        double* os = nullptr;
        int32_t* osp = nullptr;
        uint64_t ons = 0;
        oc_stats ost;
        c0 = now_ms();
        int rc = oc_intersect_meshes(reinterpret_cast<const double*>(A.v.data()), uint32_t(A.v.size()),
                                     reinterpret_cast<const uint32_t*>(A.t.data()), uint32_t(A.t.size()), &pa,
                                     reinterpret_cast<const double*>(B.v.data()), uint32_t(B.v.size()),
                                     reinterpret_cast<const uint32_t*>(B.t.data()), uint32_t(B.t.size()), &pb,
                                     segments ? 1 : 0, 0, 0, &op, &on, &os, &osp, &ons, &ost);
        const double or_ms = now_ms() - c0;
        if (rc != 0) {
            std::fprintf(stderr, "oracle failed at step %d\n", i);
            return 2;
        }
        PairSet truth;
        for (uint64_t k = 0; k < on; ++k) truth.insert({op[2 * k], op[2 * k + 1]});

        // segments: same count and the same endpoints (as unordered endpoint pairs, per pair)
        bool seg_ok = true;
        if (segments) {
            const auto& gs = ctl.lastSegments();
            if (gs.size() != ons) seg_ok = false;
            auto key = [](const double* a, const double* b, int fa, int fb) {
                std::vector<double> k{double(fa), double(fb)};
                const bool sw = std::lexicographical_compare(b, b + 3, a, a + 3);
                const double* lo = sw ? b : a;
                const double* hi = sw ? a : b;
                k.insert(k.end(), lo, lo + 3);
                k.insert(k.end(), hi, hi + 3);
                return k;
            };
            std::vector<std::vector<double>> g, o;
            for (auto& s : gs) g.push_back(key(s.p0, s.p1, s.faceA, s.faceB));
            for (uint64_t k = 0; k < ons; ++k) {
                const int32_t pi = osp[k];
                o.push_back(key(os + 6 * k, os + 6 * k + 3, op[2 * pi], op[2 * pi + 1]));
            }
            std::sort(g.begin(), g.end());
            std::sort(o.begin(), o.end());
            seg_ok = seg_ok && g == o;
        }
        oc_free(op);
        oc_free(os);
        oc_free(osp);

        size_t fp, fn, fp2, fn2;
        diff(got, truth, fp, fn);
        diff(got2, truth, fp2, fn2);
        const bool ok = fp == 0 && fn == 0 && fp2 == 0 && fn2 == 0 && seg_ok;
        agreed += ok;
        std::printf("test %3d: truth=%zu controller=%zu standalone=%zu fp=%zu fn=%zu segs=%s %s  ctl=%.2fms "
                    "oneshot=%.2fms oracle=%.1fms\n",
                    i, truth.size(), got.size(), got2.size(), fp + fp2, fn + fn2, seg_ok ? "ok" : "MISMATCH",
                    ok ? "[ALL COINCIDED]" : "[DISTINCTIONS FOUND]", ctl_ms, sa_ms, or_ms);
        if (f)
            std::fprintf(f, "%d,%.17g,%.17g,%.17g,%.17g,%.17g,%.17g,%zu,%zu,%zu,%zu,%zu,%zu,%zu,%d,%.4f,%.4f,%.4f\n", i,
                         rotB.x, rotB.y, rotB.z, transB.x, transB.y, transB.z, truth.size(), got.size(), got2.size(),
                         fp, fn, fp2, fn2, seg_ok ? 1 : 0, ctl_ms, sa_ms, or_ms);
    }
    if (f) std::fclose(f);
    std::printf("steps with full consensus: %d / %d\n", agreed, steps);
    return agreed == steps ? 0 : 1;
}
