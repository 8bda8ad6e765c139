// gi_ingest.cu -- mesh ingestion upstream of the intersection path: OFF files
// parsed on the host threads, scene normalisation on the device.
//
// The reference loads OFF files as a polygon soup (CGAL::IO::read_OFF in
// src/CPU/RobustOffLoader.h:140-150, or its mmap fast path
// src/CPU/ParallelCgalOffLoader.h:35-186), fan-triangulates polygons, drops
// rows with a repeated vertex index and faces duplicating an earlier one
// (RobustOffLoader.h:155-186), and then normalises the scene: the box of both
// meshes is centred and, optionally, scaled so its largest side spans 2
// (apps/mainApplication.cpp:166-187, 637-680: x' = (x - c) * s in FP64).
// The same steps are done here without CGAL.  Orientation and the splitting
// of non-manifold vertices (RobustOffLoader.h:190-212) are not needed: the
// intersection of closed triangles depends on neither.
#include <fcntl.h>
#include <sys/mman.h>
#include <sys/stat.h>
#include <unistd.h>

#include <algorithm>
#include <array>
#include <charconv>
#include <cmath>
#include <cstring>
#include <thread>
#include <vector>

#include "gi_host.h"

struct gi_off_mesh {
    std::vector<double> verts;      // 3 per vertex
    std::vector<uint32_t> tris;     // 3 per triangle
    std::vector<uint32_t> face_row; // OFF face row each triangle came from
};

namespace {

struct Mapped {
    const char* p = nullptr;
    size_t n = 0;
    ~Mapped()
    {
        if (p) munmap(const_cast<char*>(p), n);
    }
};

inline bool is_space(char c) { return c == ' ' || c == '\t' || c == '\r' || c == '\n' || c == '\f' || c == '\v'; }

// Parses the next number of a line ([s, e), comments end the line); false at the end.
template <class T>
inline bool next_num(const char*& s, const char* e, T& v)
{
    while (s < e && is_space(*s)) s++;
    if (s >= e || *s == '#') return false;
    if (*s == '+') s++;
    auto r = std::from_chars(s, e, v);
    if (r.ec != std::errc()) return false;
    s = r.ptr;
    return true;
}

// Data lines of the file (not blank, not comment-only): [begin, end) offsets.
void split_lines(const char* p, size_t n, unsigned nthreads, std::vector<std::pair<size_t, size_t>>& out)
{
    nthreads = std::max(1u, std::min<unsigned>(nthreads, (unsigned)(n / (1 << 16) + 1)));
    std::vector<std::vector<std::pair<size_t, size_t>>> part(nthreads);
    std::vector<std::thread> th;
    const size_t chunk = (n + nthreads - 1) / nthreads;
    for (unsigned t = 0; t < nthreads; t++)
        th.emplace_back([&, t] {
            size_t a = std::min(n, t * chunk), b = std::min(n, a + chunk);
            // a line belongs to the chunk where it starts
            if (a > 0)
                while (a < b && p[a - 1] != '\n') a++;
            size_t s = a;
            while (s < b) {
                const char* nl = static_cast<const char*>(memchr(p + s, '\n', n - s));
                const size_t e = nl ? (size_t)(nl - p) : n;
                size_t q = s;
                while (q < e && is_space(p[q])) q++;
                if (q < e && p[q] != '#') part[t].emplace_back(s, e);
                s = e + 1;
            }
        });
    for (auto& x : th) x.join();
    size_t tot = 0;
    for (auto& v : part) tot += v.size();
    out.clear();
    out.reserve(tot);
    for (auto& v : part) out.insert(out.end(), v.begin(), v.end());
}

template <class F>
void parallel_for(size_t n, unsigned nthreads, F f)
{
    nthreads = std::max(1u, std::min<unsigned>(nthreads, (unsigned)(n / 4096 + 1)));
    std::vector<std::thread> th;
    const size_t chunk = (n + nthreads - 1) / nthreads;
    for (unsigned t = 0; t < nthreads; t++)
        th.emplace_back([&, t] {
            const size_t a = std::min(n, t * chunk), b = std::min(n, a + chunk);
            f(a, b);
        });
    for (auto& x : th) x.join();
}

gi_status load_off(const char* path, unsigned nthreads, gi_off_mesh* m, gi_off_report* rep, std::string* err)
{
    const int fd = open(path, O_RDONLY);
    if (fd < 0) {
        *err = std::string("cannot open ") + path;
        return GI_ERR_INVALID_ARG;
    }
    struct stat sb;
    if (fstat(fd, &sb) != 0 || sb.st_size <= 0) {
        close(fd);
        *err = std::string("empty or unreadable file ") + path;
        return GI_ERR_INVALID_ARG;
    }
    Mapped f;
    f.n = (size_t)sb.st_size;
    void* mp = mmap(nullptr, f.n, PROT_READ, MAP_PRIVATE, fd, 0);
    close(fd);
    if (mp == MAP_FAILED) {
        *err = std::string("cannot map ") + path;
        return GI_ERR_INVALID_ARG;
    }
    f.p = static_cast<const char*>(mp);
    if (nthreads == 0) nthreads = std::max(1u, std::thread::hardware_concurrency());
    std::vector<std::pair<size_t, size_t>> lines;
    split_lines(f.p, f.n, nthreads, lines);
    // header: a keyword ending in "OFF" (OFF, COFF, NOFF, ...), then the counts,
    // on the same line or the next data line
    size_t li = 0;
    if (lines.empty()) {
        *err = "no OFF header";
        return GI_ERR_INVALID_ARG;
    }
    const char* s = f.p + lines[0].first;
    const char* e = f.p + lines[0].second;
    while (s < e && is_space(*s)) s++;
    const char* kw = s;
    while (s < e && !is_space(*s)) s++;
    const std::string key(kw, s);
    if (key.size() < 3 || key.compare(key.size() - 3, 3, "OFF") != 0) {
        *err = "no OFF header";
        return GI_ERR_INVALID_ARG;
    }
    uint64_t cnt[3] = {0, 0, 0};
    int got = 0;
    while (got < 3) {
        uint64_t v;
        if (next_num(s, e, v)) {
            cnt[got++] = v;
            continue;
        }
        if (got >= 2) break;  // the edge count may be missing
        if (++li >= lines.size()) {
            *err = "truncated OFF header";
            return GI_ERR_INVALID_ARG;
        }
        s = f.p + lines[li].first;
        e = f.p + lines[li].second;
    }
    li++;
    const uint64_t nv = cnt[0], nf = cnt[1];
    if (nv > 0xffffffffull || nf > 0xffffffffull || lines.size() < li + nv + nf) {
        *err = "OFF counts exceed the file";
        return GI_ERR_INVALID_ARG;
    }
    rep->file_vertices = nv;
    rep->file_polygons = nf;
    // vertices (extra columns, e.g. colours, are ignored)
    m->verts.assign(3 * nv, 0.0);
    std::vector<char> bad(3, 0);  // per phase: vertices, face sizes, face indices
    parallel_for(nv, nthreads, [&](size_t a, size_t b) {
        for (size_t k = a; k < b; k++) {
            const char* q = f.p + lines[li + k].first;
            const char* qe = f.p + lines[li + k].second;
            for (int c = 0; c < 3; c++)
                if (!next_num(q, qe, m->verts[3 * k + c])) bad[0] = 1;
        }
    });
    if (bad[0]) {
        *err = "malformed vertex line";
        return GI_ERR_INVALID_ARG;
    }
    // faces: count the fan triangles of every row, then fill in row order
    const size_t lf = li + nv;
    std::vector<uint32_t> ntri(nf + 1, 0);
    parallel_for(nf, nthreads, [&](size_t a, size_t b) {
        for (size_t k = a; k < b; k++) {
            const char* q = f.p + lines[lf + k].first;
            const char* qe = f.p + lines[lf + k].second;
            uint64_t deg = 0;
            if (!next_num(q, qe, deg) || deg > (1u << 20)) bad[1] = 1;
            ntri[k] = deg >= 3 ? (uint32_t)(deg - 2) : 0u;
        }
    });
    if (bad[1]) {
        *err = "malformed face line";
        return GI_ERR_INVALID_ARG;
    }
    std::vector<uint64_t> off(nf + 1, 0);
    for (size_t k = 0; k < nf; k++) off[k + 1] = off[k] + ntri[k];
    const uint64_t nfan = off[nf];
    std::vector<uint32_t> t(3 * nfan);
    std::vector<uint32_t> row(nfan);
    std::vector<uint8_t> degen(nfan, 0);
    parallel_for(nf, nthreads, [&](size_t a, size_t b) {
        std::vector<uint32_t> idx;
        for (size_t k = a; k < b; k++) {
            const char* q = f.p + lines[lf + k].first;
            const char* qe = f.p + lines[lf + k].second;
            uint64_t deg = 0;
            next_num(q, qe, deg);
            idx.resize(deg);
            for (uint64_t c = 0; c < deg; c++) {
                uint64_t v = 0;
                if (!next_num(q, qe, v) || v >= nv) bad[2] = 1;
                idx[c] = (uint32_t)std::min<uint64_t>(v, nv ? nv - 1 : 0);
            }
            for (uint64_t c = 1; c + 1 < deg; c++) {  // fan: (p0, pk, pk+1)
                const uint64_t o = off[k] + c - 1;
                t[3 * o] = idx[0];
                t[3 * o + 1] = idx[c];
                t[3 * o + 2] = idx[c + 1];
                row[o] = (uint32_t)k;
                degen[o] = idx[0] == idx[c] || idx[c] == idx[c + 1] || idx[0] == idx[c + 1];
            }
        }
    });
    if (bad[2]) {
        *err = "face index out of range or malformed";
        return GI_ERR_INVALID_ARG;
    }
    uint64_t extra = 0, short_cnt = 0;
    for (size_t k = 0; k < nf; k++) {
        if (ntri[k] > 1) extra += ntri[k] - 1;
        if (ntri[k] == 0) short_cnt++;
    }
    // drop triangles with a repeated index, then later copies of a vertex set
    std::vector<std::array<uint32_t, 4>> keys;
    keys.reserve(nfan);
    uint64_t ndeg = short_cnt;
    for (uint64_t o = 0; o < nfan; o++) {
        if (degen[o]) {
            ndeg++;
            continue;
        }
        std::array<uint32_t, 4> kx{t[3 * o], t[3 * o + 1], t[3 * o + 2], (uint32_t)o};
        std::sort(kx.begin(), kx.begin() + 3);
        keys.push_back(kx);
    }
    std::sort(keys.begin(), keys.end());
    std::vector<uint8_t> keep(nfan, 0);
    uint64_t ndup = 0;
    for (size_t i = 0; i < keys.size(); i++) {
        if (i > 0 && keys[i][0] == keys[i - 1][0] && keys[i][1] == keys[i - 1][1] && keys[i][2] == keys[i - 1][2]) {
            ndup++;
            continue;
        }
        keep[keys[i][3]] = 1;
    }
    m->tris.clear();
    m->face_row.clear();
    m->tris.reserve(3 * (nfan - ndup - ndeg + short_cnt));
    for (uint64_t o = 0; o < nfan; o++)
        if (keep[o]) {
            m->tris.insert(m->tris.end(), &t[3 * o], &t[3 * o] + 3);
            m->face_row.push_back(row[o]);
        }
    rep->extra_fan_triangles = extra;
    rep->dropped_degenerate = ndeg;
    rep->dropped_duplicate = ndup;
    if (m->tris.size() / 3 > 0x7fffffffull) {
        *err = "too many triangles";
        return GI_ERR_INVALID_ARG;
    }
    return GI_OK;
}

// ---- scene normalisation on the device ------------------------------------
constexpr int kNormThreads = 256;
constexpr int kNormBlocks = 512;

// Per-block min/max of x, y, z over nv points (partials: 6 per block).
__global__ void __launch_bounds__(kNormThreads) k_box(const double* __restrict__ v, uint32_t nv,
                                                      double* __restrict__ part)
{
    __shared__ double s[6][kNormThreads];
    double lo[3] = {INFINITY, INFINITY, INFINITY}, hi[3] = {-INFINITY, -INFINITY, -INFINITY};
    for (size_t i = blockIdx.x * (size_t)blockDim.x + threadIdx.x; i < nv; i += (size_t)gridDim.x * blockDim.x)
        for (int c = 0; c < 3; c++) {
            const double x = v[3 * i + c];
            lo[c] = fmin(lo[c], x);
            hi[c] = fmax(hi[c], x);
        }
    for (int c = 0; c < 3; c++) {
        s[c][threadIdx.x] = lo[c];
        s[3 + c][threadIdx.x] = hi[c];
    }
    __syncthreads();
    for (int w = kNormThreads / 2; w > 0; w >>= 1) {
        if ((int)threadIdx.x < w)
            for (int c = 0; c < 3; c++) {
                s[c][threadIdx.x] = fmin(s[c][threadIdx.x], s[c][threadIdx.x + w]);
                s[3 + c][threadIdx.x] = fmax(s[3 + c][threadIdx.x], s[3 + c][threadIdx.x + w]);
            }
        __syncthreads();
    }
    if (threadIdx.x < 6) part[6 * blockIdx.x + threadIdx.x] = s[threadIdx.x][0];
}

// x' = (x - c) * s, rounded per operation (no fused multiply-add), as the
// reference's normalizeMeshCoordinatesParallel.
__global__ void __launch_bounds__(kNormThreads) k_normalize(double* __restrict__ v, uint32_t nv, double cx,
                                                            double cy, double cz, double scale)
{
    for (size_t i = blockIdx.x * (size_t)blockDim.x + threadIdx.x; i < nv; i += (size_t)gridDim.x * blockDim.x) {
        v[3 * i] = __dmul_rn(__dsub_rn(v[3 * i], cx), scale);
        v[3 * i + 1] = __dmul_rn(__dsub_rn(v[3 * i + 1], cy), scale);
        v[3 * i + 2] = __dmul_rn(__dsub_rn(v[3 * i + 2], cz), scale);
    }
}

// Box of nv device points into lo/hi (host), through per-block partials.
gi_status device_box(gi_ctx* c, const double* d_v, uint32_t nv, double* part, double lo[3], double hi[3])
{
    for (int k = 0; k < 3; k++) {
        lo[k] = INFINITY;
        hi[k] = -INFINITY;
    }
    if (nv == 0) return GI_OK;
    k_box<<<kNormBlocks, kNormThreads, 0, c->st>>>(d_v, nv, part);
    gi::note_launches(1);
    std::vector<double> h(6 * kNormBlocks);
    CK(c, cudaMemcpyAsync(h.data(), part, sizeof(double) * h.size(), cudaMemcpyDeviceToHost, c->st), "box");
    CK(c, cudaStreamSynchronize(c->st), "box");
    for (int b = 0; b < kNormBlocks; b++)
        for (int k = 0; k < 3; k++) {
            lo[k] = std::min(lo[k], h[6 * b + k]);
            hi[k] = std::max(hi[k], h[6 * b + 3 + k]);
        }
    return GI_OK;
}

}  // namespace

extern "C" gi_status gi_off_load(const char* path, uint32_t nthreads, gi_off_mesh** out, gi_off_report* rep)
{
    if (!path || !out) return GI_ERR_INVALID_ARG;
    *out = nullptr;
    gi_off_report r{};
    gi_off_mesh* m = new (std::nothrow) gi_off_mesh();
    if (!m) return GI_ERR_OOM;
    std::string err;
    gi_status s = load_off(path, nthreads, m, &r, &err);
    if (s != GI_OK) {
        delete m;
        fprintf(stderr, "gi_off_load: %s\n", err.c_str());
        return s;
    }
    if (rep) *rep = r;
    *out = m;
    return GI_OK;
}

extern "C" gi_status gi_off_arrays(const gi_off_mesh* m, const double** verts_xyz, uint32_t* nv,
                                   const uint32_t** tris, uint32_t* nt, const uint32_t** face_row)
{
    if (!m) return GI_ERR_INVALID_ARG;
    if (verts_xyz) *verts_xyz = m->verts.data();
    if (nv) *nv = (uint32_t)(m->verts.size() / 3);
    if (tris) *tris = m->tris.data();
    if (nt) *nt = (uint32_t)(m->tris.size() / 3);
    if (face_row) *face_row = m->face_row.data();
    return GI_OK;
}

extern "C" gi_status gi_off_free(gi_off_mesh* m)
{
    if (!m) return GI_ERR_INVALID_ARG;
    delete m;
    return GI_OK;
}

extern "C" gi_status gi_scene_load(gi_ctx* c, const char* path_a, const char* path_b, int32_t scale_to_unit,
                                   gi_mesh** A, gi_mesh** B, gi_scene* scene, gi_off_report* rep_a,
                                   gi_off_report* rep_b)
{
    if (!c || !path_a || !path_b || !A || !B) return GI_ERR_INVALID_ARG;
    *A = *B = nullptr;
    gi_off_mesh *ma = nullptr, *mb = nullptr;
    gi_status s = gi_off_load(path_a, 0, &ma, rep_a);
    if (s != GI_OK) return set_err(c, s, "loading mesh A");
    s = gi_off_load(path_b, 0, &mb, rep_b);
    if (s != GI_OK) {
        gi_off_free(ma);
        return set_err(c, s, "loading mesh B");
    }
    const uint32_t nva = (uint32_t)(ma->verts.size() / 3), nvb = (uint32_t)(mb->verts.size() / 3);
    double *dva = nullptr, *dvb = nullptr, *part = nullptr;
    gi_scene sc{};
    {
        std::lock_guard<std::mutex> lk(c->mu);
        cudaSetDevice(c->device);
        auto fail = [&](gi_status st, const char* what, cudaError_t e) {
            if (dva) cudaFreeAsync(dva, c->st);
            if (dvb) cudaFreeAsync(dvb, c->st);
            if (part) cudaFreeAsync(part, c->st);
            gi_off_free(ma);
            gi_off_free(mb);
            return set_err(c, st, what, e);
        };
        cudaError_t e = gi::pool_alloc(&dva, sizeof(double) * (ma->verts.size() + 1), c->pool, c->st);
        if (e == cudaSuccess) e = gi::pool_alloc(&dvb, sizeof(double) * (mb->verts.size() + 1), c->pool, c->st);
        if (e == cudaSuccess) e = gi::pool_alloc(&part, sizeof(double) * 6 * kNormBlocks, c->pool, c->st);
        if (e != cudaSuccess) return fail(GI_ERR_OOM, "scene buffers", e);
        if (nva) e = cudaMemcpyAsync(dva, ma->verts.data(), sizeof(double) * ma->verts.size(), cudaMemcpyHostToDevice, c->st);
        if (e == cudaSuccess && nvb)
            e = cudaMemcpyAsync(dvb, mb->verts.data(), sizeof(double) * mb->verts.size(), cudaMemcpyHostToDevice, c->st);
        if (e != cudaSuccess) return fail(GI_ERR_CUDA, "scene upload", e);
        // scene box, centre and scale (apps/mainApplication.cpp:644-660)
        double la[3], ha[3], lb[3], hb[3];
        if ((s = device_box(c, dva, nva, part, la, ha)) != GI_OK || (s = device_box(c, dvb, nvb, part, lb, hb)) != GI_OK)
            return fail(s, "scene box", cudaSuccess);
        double span = 0.0;
        for (int k = 0; k < 3; k++) {
            const double lo = std::min(la[k], lb[k]), hi = std::max(ha[k], hb[k]);
            sc.center[k] = 0.5 * (lo + hi);
            span = std::max(span, hi - lo);
        }
        sc.max_span = span;
        sc.scale = (scale_to_unit && span > 0.0) ? 2.0 / span : 1.0;
        for (auto [dv, n] : {std::make_pair(dva, nva), std::make_pair(dvb, nvb)})
            if (n) {
                k_normalize<<<kNormBlocks, kNormThreads, 0, c->st>>>(dv, n, sc.center[0], sc.center[1], sc.center[2],
                                                                     sc.scale);
                gi::note_launches(1);
            }
        if ((e = cudaGetLastError()) != cudaSuccess) return fail(GI_ERR_CUDA, "normalise", e);
        // box centres of the normalised meshes: the rotation centres of the poses
        if ((s = device_box(c, dva, nva, part, la, ha)) != GI_OK || (s = device_box(c, dvb, nvb, part, lb, hb)) != GI_OK)
            return fail(s, "mesh boxes", cudaSuccess);
        for (int k = 0; k < 3; k++) {
            sc.center_a[k] = nva ? 0.5 * (la[k] + ha[k]) : 0.0;
            sc.center_b[k] = nvb ? 0.5 * (lb[k] + hb[k]) : 0.0;
        }
    }
    // the meshes are built from the normalised device arrays; triangles from the host
    uint32_t *dta = nullptr, *dtb = nullptr;
    cudaError_t e = cudaSuccess;
    {
        std::lock_guard<std::mutex> lk(c->mu);
        e = gi::pool_alloc(&dta, sizeof(uint32_t) * (ma->tris.size() + 1), c->pool, c->st);
        if (e == cudaSuccess) e = gi::pool_alloc(&dtb, sizeof(uint32_t) * (mb->tris.size() + 1), c->pool, c->st);
        if (e == cudaSuccess && !ma->tris.empty())
            e = cudaMemcpyAsync(dta, ma->tris.data(), sizeof(uint32_t) * ma->tris.size(), cudaMemcpyHostToDevice, c->st);
        if (e == cudaSuccess && !mb->tris.empty())
            e = cudaMemcpyAsync(dtb, mb->tris.data(), sizeof(uint32_t) * mb->tris.size(), cudaMemcpyHostToDevice, c->st);
    }
    if (e == cudaSuccess) {
        s = gi_mesh_upload_device(c, dva, nva, dta, (uint32_t)(ma->tris.size() / 3), A);
        if (s == GI_OK) s = gi_mesh_upload_device(c, dvb, nvb, dtb, (uint32_t)(mb->tris.size() / 3), B);
        if (s != GI_OK && *A) {
            gi_mesh_release(c, *A);
            *A = nullptr;
        }
    } else {
        s = set_err(c, GI_ERR_OOM, "scene triangles", e);
    }
    {
        std::lock_guard<std::mutex> lk(c->mu);
        for (void* p : {(void*)dva, (void*)dvb, (void*)part, (void*)dta, (void*)dtb})
            if (p) cudaFreeAsync(p, c->st);
    }
    gi_off_free(ma);
    gi_off_free(mb);
    if (s == GI_OK && scene) *scene = sc;
    return s;
}

extern "C" gi_status gi_mesh_download(const gi_mesh* m, double* verts_xyz_out)
{
    if (!m || (!verts_xyz_out && m->b.nv)) return GI_ERR_INVALID_ARG;
    gi_ctx* c = m->ctx;
    std::lock_guard<std::mutex> lk(c->mu);
    cudaSetDevice(c->device);
    if (m->b.nv) {
        CK(c, cudaMemcpyAsync(verts_xyz_out, m->b.verts, sizeof(double) * 3 * (size_t)m->b.nv, cudaMemcpyDeviceToHost,
                              c->st),
           "download vertices");
        CK(c, cudaStreamSynchronize(c->st), "download vertices");
    }
    return GI_OK;
}
