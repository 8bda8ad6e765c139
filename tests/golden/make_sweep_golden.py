"""Generates tests/golden/sweep_poses.json: B's per-step Euler angles and
translations of the reference's seeded sweep (src/CPU/TestSuite.cpp:478-505)
as a GCC build of it computes them.  The reference draws each vector inside
one make_double3(base.x + draw, base.y + draw, base.z + draw) call, whose
argument order C++ leaves to the compiler; the statement is restated below in
that form and compiled with g++ and CUDA's vector_types.h, so the file records
what GCC does with it (std::mt19937 + std::uniform_real_distribution<double>
from libstdc++).

Run from the repository root:  python tests/golden/make_sweep_golden.py
"""
import json
import os
import subprocess
import tempfile

HERE = os.path.dirname(os.path.abspath(__file__))
CASES = [  # seed, steps, max rotation (deg), max translation, base rotation of B, base translation of B
    (1337, 6, 15.0, 0.5, (0.0, 0.0, 0.0), (0.0, 0.0, 0.0)),
    (42, 4, 30.0, 0.25, (0.0, 0.0, 0.0), (0.5, 0.0, 0.0)),
    (7, 3, 5.0, 0.05, (10.0, -20.0, 30.0), (0.1, 0.2, -0.3)),
]

PROGRAM = r"""
#include <cstdio>
#include <cstdlib>
#include <random>
#include <vector_types.h>
#include <vector_functions.h>
int main(int argc, char** argv) {
  const unsigned seed = unsigned(std::strtoul(argv[1], nullptr, 10));
  const int steps = std::atoi(argv[2]);
  const double maxRot = std::atof(argv[3]), maxTrans = std::atof(argv[4]);
  const double3 baseRotB = make_double3(std::atof(argv[5]), std::atof(argv[6]), std::atof(argv[7]));
  const double3 baseTransB = make_double3(std::atof(argv[8]), std::atof(argv[9]), std::atof(argv[10]));
  std::mt19937 rng(seed);
  std::uniform_real_distribution<double> rotDist(-maxRot, maxRot);
  std::uniform_real_distribution<double> transDist(-maxTrans, maxTrans);
  for (int i = 0; i < steps; ++i) {
    double3 rotB = make_double3(baseRotB.x + rotDist(rng), baseRotB.y + rotDist(rng), baseRotB.z + rotDist(rng));
    double3 transB = make_double3(baseTransB.x + transDist(rng), baseTransB.y + transDist(rng),
                                  baseTransB.z + transDist(rng));
    std::printf("%a %a %a %a %a %a\n", rotB.x, rotB.y, rotB.z, transB.x, transB.y, transB.z);
  }
}
"""


def main():
    out = []
    with tempfile.TemporaryDirectory() as td:
        src, exe = os.path.join(td, "sweep.cpp"), os.path.join(td, "sweep")
        open(src, "w").write(PROGRAM)
        subprocess.run(["g++", "-O2", "-I/usr/local/cuda/include", src, "-o", exe], check=True)
        for seed, steps, mr, mt, br, bt in CASES:
            args = [str(seed), str(steps), repr(mr), repr(mt)] + [repr(x) for x in br + bt]
            lines = subprocess.run([exe] + args, check=True, capture_output=True, text=True).stdout.split("\n")
            rows = [l.split() for l in lines if l.strip()]
            out.append(dict(seed=seed, steps=steps, max_rot_deg=mr, max_trans=mt, base_rot_b=br, base_trans_b=bt,
                            rot_b=[r[:3] for r in rows], trans_b=[r[3:] for r in rows]))
    with open(os.path.join(HERE, "sweep_poses.json"), "w") as f:
        json.dump(out, f, indent=1)
        f.write("\n")


if __name__ == "__main__":
    main()
