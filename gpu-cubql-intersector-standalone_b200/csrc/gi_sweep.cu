// gi_sweep.cu -- the pose sequence of a seeded pose sweep (host code).
//
// The reference's verification sweep (TestSuite::runSuite,
// src/CPU/TestSuite.cpp:455-505) keeps mesh A at its base pose and perturbs B
// per step by rotations uniform in [-max_rot, max_rot] degrees and translations
// uniform in [-max_trans, max_trans], drawn from std::mt19937(seed) through
// std::uniform_real_distribution<double>.  Each of B's two vectors is built by
// one make_double3(base.x + draw, base.y + draw, base.z + draw) call whose
// argument order C++ leaves unspecified; GCC evaluates such arguments right to
// left, so a GCC build of the reference draws z, then y, then x.  The draws
// here are sequenced explicitly in that order, with the same engine and
// distribution, so that a seed gives the reference's poses when both are built
// against libstdc++.
#include <random>

#include "gi/gi.h"

extern "C" gi_status gi_sweep_poses(uint32_t seed, uint32_t nsteps, double max_rot_deg, double max_trans,
                                    const double base_rot_b[3], const double base_trans_b[3], double* rot_b_out,
                                    double* trans_b_out)
{
    if ((nsteps && (!rot_b_out || !trans_b_out)) || !(max_rot_deg >= 0.0) || !(max_trans >= 0.0))
        return GI_ERR_INVALID_ARG;
    const double zero[3] = {0.0, 0.0, 0.0};
    const double* br = base_rot_b ? base_rot_b : zero;
    const double* bt = base_trans_b ? base_trans_b : zero;
    std::mt19937 rng(seed);
    std::uniform_real_distribution<double> rot(-max_rot_deg, max_rot_deg);
    std::uniform_real_distribution<double> trans(-max_trans, max_trans);
    for (uint32_t s = 0; s < nsteps; s++) {
        double* r = rot_b_out + 3 * (size_t)s;
        double* t = trans_b_out + 3 * (size_t)s;
        for (int c = 2; c >= 0; c--) r[c] = br[c] + rot(rng);
        for (int c = 2; c >= 0; c--) t[c] = bt[c] + trans(rng);
    }
    return GI_OK;
}
