// Test infrastructure: a small program around the reference's own IntersectionHistory
// (src/CPU/IntersectionHistory.h, header-only), compiled from the reference
// sources by history_ref.mk into oracle/_ref/history_ref.  It reads runs as
// record files and writes the reference's CSVs, against which the library's
// gi_records_write_csv / gi_pairs_diff output is compared byte for byte.
//
// Record file: uint64 n, then n records of int32 faceA, faceB, vA0..vA2,
// vB0..vB2 and 18 doubles (a_v0, a_v1, a_v2, b_v0, b_v1, b_v2; x, y, z).
//
//   history_ref export run.bin out.csv
//   history_ref diff run1.bin run2.bin <filter> out.csv
//
// The time of the export call itself is printed to stderr as "export_ms=<ms>".
#include <chrono>
#include <cstdint>
#include <cstdio>
#include <sstream>
#include <string>

#include "CPU/IntersectionHistory.h"

static bool read_run(const char* path, std::vector<IntersectingTriangleRecord>& out)
{
    FILE* f = std::fopen(path, "rb");
    if (!f) return false;
    uint64_t n = 0;
    bool ok = std::fread(&n, 8, 1, f) == 1;
    for (uint64_t i = 0; ok && i < n; i++) {
        int32_t iv[8];
        double dv[18];
        ok = std::fread(iv, 4, 8, f) == 8 && std::fread(dv, 8, 18, f) == 18;
        if (!ok) break;
        IntersectingTriangleRecord r;
        r.faceA = iv[0];
        r.faceB = iv[1];
        r.vA0_idx = iv[2], r.vA1_idx = iv[3], r.vA2_idx = iv[4];
        r.vB0_idx = iv[5], r.vB1_idx = iv[6], r.vB2_idx = iv[7];
        double3* pts[6] = {&r.a_v0, &r.a_v1, &r.a_v2, &r.b_v0, &r.b_v1, &r.b_v2};
        for (int k = 0; k < 6; k++) { pts[k]->x = dv[3 * k]; pts[k]->y = dv[3 * k + 1]; pts[k]->z = dv[3 * k + 2]; }
        out.push_back(r);
    }
    std::fclose(f);
    return ok;
}

int main(int argc, char** argv)
{
    if (argc < 2) return 2;
    const std::string cmd = argv[1];
    IntersectionHistory h;
    if (cmd == "export" && argc == 4) {
        std::vector<IntersectingTriangleRecord> r;
        if (!read_run(argv[2], r)) return 3;
        h.recordRun("run", 0.0, r);
        const auto t0 = std::chrono::steady_clock::now();
        const bool ok = h.exportRunToCsv(0, argv[3]);
        const auto t1 = std::chrono::steady_clock::now();
        std::fprintf(stderr, "export_ms=%.3f\n", std::chrono::duration<double, std::milli>(t1 - t0).count());
        return ok ? 0 : 4;
    }
    if (cmd == "diff" && argc == 6) {
        std::vector<IntersectingTriangleRecord> r1, r2;
        if (!read_run(argv[2], r1) || !read_run(argv[3], r2)) return 3;
        h.recordRun("run1", 0.0, r1);
        h.recordRun("run2", 0.0, r2);
        const auto t0 = std::chrono::steady_clock::now();
        const bool ok = h.exportDiff(0, 1, argv[4], argv[5]);
        const auto t1 = std::chrono::steady_clock::now();
        std::fprintf(stderr, "export_ms=%.3f\n", std::chrono::duration<double, std::milli>(t1 - t0).count());
        return ok ? 0 : 4;
    }
    return 2;
}
