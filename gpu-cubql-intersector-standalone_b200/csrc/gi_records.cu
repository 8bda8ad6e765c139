// gi_records.cu -- run records: CSV export of intersecting pairs with their
// vertex indices and posed coordinates, and the set diff of two runs (host
// code; needs no device).
//
// The reference keeps these as IntersectingTriangleRecord rows inside
// IntersectionHistory (src/CPU/IntersectionHistory.h:12-30 the record,
// :114-160 exportRunToCsv, :162-232 exportDiff) and writes them through an
// ostream at setprecision(17), i.e. every double as printf("%.17g").  Here a
// run is kept as its pair list plus the posed vertex and triangle arrays; the
// rows are formatted on demand with std::to_chars (general format, precision
// 17, which is specified to match %.17g) on several threads, in blocks that are
// written to the file in pair order.  The diff merges the two pair lists as
// sorted (faceA, faceB) keys with int ordering, the order of the reference's
// std::set of records.
#include <algorithm>
#include <charconv>
#include <cstdio>
#include <cstring>
#include <string>
#include <thread>
#include <vector>

#include "gi/gi.h"

namespace {

constexpr const char* kHeader =
    "FaceA,FaceB,VA0_Idx,VA1_Idx,VA2_Idx,VB0_Idx,VB1_Idx,VB2_Idx,"
    "A_V0_X,A_V0_Y,A_V0_Z,A_V1_X,A_V1_Y,A_V1_Z,A_V2_X,A_V2_Y,A_V2_Z,"
    "B_V0_X,B_V0_Y,B_V0_Z,B_V1_X,B_V1_Y,B_V1_Z,B_V2_X,B_V2_Y,B_V2_Z\n";

// widest row: category + 8 ints (11 chars) + 18 doubles (%.17g is at most 24
// chars: sign, 17 digits, point, e-308) + 26 separators
constexpr size_t kRowMax = 8 * 12 + 18 * 25 + 8;

inline char* put_int(char* p, int64_t v)
{
    return std::to_chars(p, p + 24, v).ptr;
}

inline char* put_g17(char* p, double v)
{
    return std::to_chars(p, p + 32, v, std::chars_format::general, 17).ptr;
}

bool mesh_ok(const gi_record_mesh* m)
{
    return m && (m->nt == 0 || m->tris) && (m->nv == 0 || m->verts_xyz);
}

// one row; pairs, faces and vertex indices were validated before
char* put_row(char* p, const char* cat, size_t cat_len, const gi_record_mesh& A, const gi_record_mesh& B, int32_t fa,
              int32_t fb)
{
    if (cat_len) {
        std::memcpy(p, cat, cat_len);
        p += cat_len;
        *p++ = ',';
    }
    const uint32_t* ta = A.tris + 3 * (size_t)fa;
    const uint32_t* tb = B.tris + 3 * (size_t)fb;
    p = put_int(p, fa);
    *p++ = ',';
    p = put_int(p, fb);
    for (int k = 0; k < 3; k++) {
        *p++ = ',';
        p = put_int(p, ta[k]);
    }
    for (int k = 0; k < 3; k++) {
        *p++ = ',';
        p = put_int(p, tb[k]);
    }
    for (int k = 0; k < 3; k++)
        for (int c = 0; c < 3; c++) {
            *p++ = ',';
            p = put_g17(p, A.verts_xyz[3 * (size_t)ta[k] + c]);
        }
    for (int k = 0; k < 3; k++)
        for (int c = 0; c < 3; c++) {
            *p++ = ',';
            p = put_g17(p, B.verts_xyz[3 * (size_t)tb[k] + c]);
        }
    *p++ = '\n';
    return p;
}

inline uint64_t pair_key(const int32_t* p)
{
    // int order of (faceA, faceB) as unsigned order of the biased halves
    return ((uint64_t)((uint32_t)p[0] ^ 0x80000000u) << 32) | (uint32_t)((uint32_t)p[1] ^ 0x80000000u);
}

inline void key_pair(uint64_t k, int32_t* p)
{
    p[0] = (int32_t)((uint32_t)(k >> 32) ^ 0x80000000u);
    p[1] = (int32_t)((uint32_t)k ^ 0x80000000u);
}

void sorted_keys(const int32_t* pairs, uint64_t n, std::vector<uint64_t>& k)
{
    k.resize(n);
    bool sorted = true;
    for (uint64_t i = 0; i < n; i++) {
        k[i] = pair_key(pairs + 2 * i);
        if (i && k[i] < k[i - 1]) sorted = false;
    }
    if (!sorted) std::sort(k.begin(), k.end());
    k.erase(std::unique(k.begin(), k.end()), k.end());
}

}  // namespace

extern "C" gi_status gi_records_write_csv(const char* path, int32_t append, int32_t header, const char* category,
                                          const gi_record_mesh* A, const gi_record_mesh* B, const int32_t* pairs_ab,
                                          uint64_t n, uint32_t nthreads)
{
    if (!path || !mesh_ok(A) || !mesh_ok(B) || (n && !pairs_ab)) return GI_ERR_INVALID_ARG;
    // validate every pair and the vertex indices it reaches before writing anything
    for (uint64_t i = 0; i < n; i++) {
        const int32_t fa = pairs_ab[2 * i], fb = pairs_ab[2 * i + 1];
        if (fa < 0 || fb < 0 || (uint32_t)fa >= A->nt || (uint32_t)fb >= B->nt) return GI_ERR_INVALID_ARG;
        const uint32_t* ta = A->tris + 3 * (size_t)fa;
        const uint32_t* tb = B->tris + 3 * (size_t)fb;
        for (int k = 0; k < 3; k++)
            if (ta[k] >= A->nv || tb[k] >= B->nv) return GI_ERR_INVALID_ARG;
    }
    const size_t cat_len = category ? std::strlen(category) : 0;
    if (cat_len > 256) return GI_ERR_INVALID_ARG;
    FILE* f = std::fopen(path, append ? "ab" : "wb");
    if (!f) {
        std::fprintf(stderr, "gi_records_write_csv: cannot open %s\n", path);
        return GI_ERR_INVALID_ARG;
    }
    bool ok = true;
    if (header) {
        if (cat_len) ok = std::fputs("DiffCategory,", f) >= 0;
        ok = ok && std::fputs(kHeader, f) >= 0;
    }
    if (nthreads == 0) nthreads = std::max(1u, std::thread::hardware_concurrency());
    const uint64_t block = 8192;  // rows per thread per round
    const unsigned nt = (unsigned)std::max<uint64_t>(1, std::min<uint64_t>(nthreads, (n + block - 1) / block));
    std::vector<std::string> buf(nt);
    std::vector<size_t> used(nt, 0);
    for (auto& b : buf) b.resize(block * (kRowMax + cat_len));
    for (uint64_t base = 0; ok && base < n; base += block * nt) {
        auto work = [&](unsigned t) {
            const uint64_t a = base + t * block, e = std::min(n, a + block);
            char* p = buf[t].data();
            char* q = p;
            for (uint64_t i = a; i < e; i++) q = put_row(q, category, cat_len, *A, *B, pairs_ab[2 * i], pairs_ab[2 * i + 1]);
            used[t] = (size_t)(q - p);
        };
        std::vector<std::thread> th;
        for (unsigned t = 1; t < nt; t++) th.emplace_back(work, t);
        work(0);
        for (auto& x : th) x.join();
        for (unsigned t = 0; t < nt && ok; t++)
            if (used[t]) ok = std::fwrite(buf[t].data(), 1, used[t], f) == used[t];
    }
    ok = (std::fclose(f) == 0) && ok;
    if (!ok) {
        std::fprintf(stderr, "gi_records_write_csv: write to %s failed\n", path);
        return GI_ERR_INVALID_ARG;
    }
    return GI_OK;
}

extern "C" gi_status gi_pairs_diff(const int32_t* pairs1, uint64_t n1, const int32_t* pairs2, uint64_t n2,
                                   int32_t* only1, uint64_t* n_only1, int32_t* only2, uint64_t* n_only2,
                                   int32_t* both, uint64_t* n_both)
{
    if ((n1 && !pairs1) || (n2 && !pairs2) || !n_only1 || !n_only2 || !n_both) return GI_ERR_INVALID_ARG;
    if ((n1 && (!only1 || !both)) || (n2 && !only2)) return GI_ERR_INVALID_ARG;
    std::vector<uint64_t> k1, k2;
    sorted_keys(pairs1, n1, k1);
    sorted_keys(pairs2, n2, k2);
    uint64_t i = 0, j = 0, o1 = 0, o2 = 0, b = 0;
    while (i < k1.size() && j < k2.size()) {
        if (k1[i] < k2[j]) key_pair(k1[i++], only1 + 2 * o1++);
        else if (k2[j] < k1[i]) key_pair(k2[j++], only2 + 2 * o2++);
        else {
            key_pair(k1[i++], both + 2 * b++);
            j++;
        }
    }
    while (i < k1.size()) key_pair(k1[i++], only1 + 2 * o1++);
    while (j < k2.size()) key_pair(k2[j++], only2 + 2 * o2++);
    *n_only1 = o1;
    *n_only2 = o2;
    *n_both = b;
    return GI_OK;
}
