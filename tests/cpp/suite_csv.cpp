// suite_csv.cpp -- host-only checks of gi::TestSuite's CSV writers and file
// naming (include/gi/gi_suite.hpp); runs without a device.
//   suite_csv <dir>  writes <dir>/sweep.csv and its two breakdown files from two
//   hand-made results and prints the derived names of a few paths.
#include <cstdio>
#include <string>
#include <vector>

#include "gi/gi_suite.hpp"

int main(int argc, char** argv)
{
    if (argc < 2) return 2;
    const std::string dir = argv[1];
    std::vector<gi::VerificationResult> rs(2);
    rs[0].stepIndex = 0;
    rs[0].groundTruthCount = 768;
    rs[0].candidatePairs = 12345;
    rs[0].totalPossiblePairs = 20224ull * 20224ull;
    rs[0].candidateYield = 12345.0 / double(rs[0].totalPossiblePairs);
    rs[0].surfaceOverlapRatio = 0.0123456789012345;
    rs[0].gpuMainTimeMs = 0.33333333333333;
    rs[0].standaloneTimeMs = 12.5;
    rs[0].cgalClassicTimeMs = 1000.0 / 3.0;
    rs[0].gpuMainExactMatch = rs[0].standaloneExactMatch = true;
    rs[0].mainStats.detail.ms_total = 0.25;
    rs[0].mainStats.detail.ms_traverse = 0.125;
    rs[0].mainStats.detail.ms_exact = 0.0625;
    rs[0].mainStats.detail.ms_sort = 0.03125;
    rs[0].mainStats.detail.candidates = 12345;
    rs[0].mainStats.detail.pairs = 768;
    rs[0].mainStats.confirmedGreenPairs = 12300;
    rs[0].mainStats.confirmedYellowPairs = 45;
    rs[1].stepIndex = 1;
    const std::string base = dir + "/sweep.csv";
    if (!gi::TestSuite::exportToCSV(base, rs)) return 3;
    if (!gi::TestSuite::exportStandardComputeCSV(gi::TestSuite::deriveFilename(base, "_standard_breakdown"), rs))
        return 3;
    if (!gi::TestSuite::exportStandaloneComputeCSV(gi::TestSuite::deriveFilename(base, "_standalone_breakdown"), rs))
        return 3;
    // the reference's predicate modes (0-4) and the added plain-FP64 mode map to precision forms
    for (int mode = -1; mode <= 6; ++mode) {
        try {
            std::printf("mode %d -> %d\n", mode, int(gi::detail::precision_for_predicate_mode(mode)));
        } catch (const gi::Error& e) {
            std::printf("mode %d -> error %d\n", mode, int(e.status));
        }
    }
    for (const char* p : {"benchmark_results.csv", "out.d/run", "run", "a/b.c/d.csv", ".hidden", "dir/.hidden"})
        std::printf("%s -> %s\n", p, gi::TestSuite::deriveFilename(p, "_x").c_str());
    return 0;
}
