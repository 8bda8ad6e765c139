// gi_curves.cu -- intersection curves: the segments of a result chained into
// polylines (host code over a gi_result).
//
// The reference stops at a segment soup (src/CPU/MeshIntersectionCurves.cpp:
// 27-91 returns one IntersectionSegment per crossing, a zero-length one per
// touching point and the three edges of every coplanar overlap triangle).
// Here the segments are joined into curves.  Every endpoint is an exact
// intersection point rounded correctly to FP64, so the point where a shared
// mesh edge crosses the other mesh comes out bit-identical from both triangles
// that share the edge; endpoints are therefore matched by exact equality.
//
//  - vertices: distinct endpoints (-0.0 and +0.0 are the same point);
//  - edges: segments with distinct endpoints, each vertex pair once;
//    zero-length segments (touching points) become isolated vertices;
//  - coplanar regions: a pair with a coplanar triangle overlap contributes the
//    overlap triangle's three edges; with drop_coplanar_interior, an edge that
//    only such outlines contribute, two or more times, is interior to the
//    region and is dropped, so a region is represented by its boundary;
//  - curves: maximal chains through vertices of degree 2; a chain that comes
//    back to its start is closed; vertices of degree 0 (isolated points) are
//    one-vertex curves, and branch vertices (degree >= 3) end chains.
#include <algorithm>
#include <atomic>
#include <cstring>
#include <thread>
#include <vector>

#include "gi_host.h"

struct gi_curves {
    std::vector<double> verts;         // 3 per vertex
    std::vector<uint64_t> offsets;     // curve c: vertex ids idx[offsets[c] .. offsets[c+1])
    std::vector<uint32_t> idx;
    std::vector<uint8_t> closed;       // 1: the curve closes (its last vertex joins its first)
    std::vector<uint64_t> job_curves;  // batch: job j owns curves [job_curves[j], job_curves[j + 1])
};

namespace {

struct PtKey {
    uint64_t b[3];
    bool operator==(const PtKey& o) const { return b[0] == o.b[0] && b[1] == o.b[1] && b[2] == o.b[2]; }
};

// splitmix64 finaliser: every input bit reaches the low bits the tables index with
inline uint64_t mix64(uint64_t x)
{
    x ^= x >> 30;
    x *= 0xbf58476d1ce4e5b9ull;
    x ^= x >> 27;
    x *= 0x94d049bb133111ebull;
    x ^= x >> 31;
    return x;
}
inline uint64_t hash_pt(const PtKey& k)
{
    return mix64(k.b[0] ^ mix64(k.b[1] ^ mix64(k.b[2])));
}

// Open-addressing hash table (linear probing, power-of-two capacity of at
// least twice the number of keys it will hold): one flat allocation instead of
// a node per entry, kept between calls (reset clears only the flags).
template <class K, class V>
struct FlatMap {
    std::vector<K> keys;
    std::vector<V> vals;
    std::vector<uint8_t> used;
    size_t mask = 0;
    void reset(size_t max_keys)
    {
        size_t cap = 16;
        while (cap < 2 * max_keys + 1) cap <<= 1;
        if (keys.size() < cap) {
            keys.resize(cap);
            vals.resize(cap);
        }
        used.assign(cap, 0);
        mask = cap - 1;
    }
    // the value of k, inserted as v when absent; second: inserted
    template <class Hash>
    std::pair<V*, bool> emplace(const K& k, const V& v, Hash hash)
    {
        size_t h = (size_t)hash(k) & mask;
        while (used[h]) {
            if (keys[h] == k) return {&vals[h], false};
            h = (h + 1) & mask;
        }
        used[h] = 1;
        keys[h] = k;
        vals[h] = v;
        return {&vals[h], true};
    }
};

inline PtKey key_of(const double* p)
{
    PtKey k;
    for (int c = 0; c < 3; c++) {
        const double v = p[c] == 0.0 ? 0.0 : p[c];  // one key for -0.0 and +0.0
        std::memcpy(&k.b[c], &v, 8);
    }
    return k;
}

struct EdgeInfo {
    uint32_t coplanar = 0, other = 0;
};

// Working tables of one thread, kept between calls: a call on a result of
// similar size allocates nothing but its own output (fresh allocations and
// their first-touch page faults cost more than the hashing itself).
struct CurveScratch {
    std::vector<uint32_t> per_pair;
    std::vector<uint64_t> vslot;
    std::vector<PtKey> vkeys;
    FlatMap<uint64_t, EdgeInfo> edges;
    std::vector<uint64_t> edge_keys;
    std::vector<std::pair<uint32_t, uint32_t>> el;
    std::vector<uint32_t> deg, nbr, nedge;
    std::vector<uint64_t> start, fill;
    std::vector<uint8_t> used;
};

CurveScratch& scratch()
{
    thread_local CurveScratch sc;
    return sc;
}

}  // namespace

// The curves of one result (or one job of a batch): segments seg6[0 .. nsegs),
// segment s of pair seg_pair[s] - pair_base in [0, npairs).
template <class PairIndex>
static void build_curves(const double* seg6, const PairIndex* seg_pair, int64_t pair_base, uint64_t nsegs,
                         uint64_t npairs, int32_t drop_coplanar_interior, gi_curves* cv)
{
    struct View {
        const double* segs;
        const PairIndex* sp;
        int64_t base;
        uint64_t nsegs, npairs;
        int64_t seg_pair_at(uint64_t s) const { return (int64_t)sp[s] - base; }
    } rr{seg6, seg_pair, pair_base, nsegs, npairs}, *r = &rr;
    const uint64_t ns = r->nsegs;
    CurveScratch& sc = scratch();
    // segments per pair: three mark a coplanar overlap triangle
    std::vector<uint32_t>& per_pair = sc.per_pair;
    per_pair.assign(r->npairs, 0);
    for (uint64_t s = 0; s < ns; s++) {
        const int64_t q = r->seg_pair_at(s);
        if (q >= 0 && (uint64_t)q < r->npairs) per_pair[q]++;
    }
    // vertex table: 8-byte slots (hash tag, vertex id + 1) over keys stored once in vertex order
    size_t vcap = 16;
    while (vcap < 4 * ns + 1) vcap <<= 1;
    std::vector<uint64_t>& vslot = sc.vslot;
    vslot.assign(vcap, 0);
    std::vector<PtKey>& vkeys = sc.vkeys;
    vkeys.clear();
    vkeys.reserve(2 * ns);
    cv->verts.reserve(6 * ns);
    auto vertex = [&](const double* p) {
        const PtKey k = key_of(p);
        const uint64_t h = hash_pt(k);
        const uint32_t tag = (uint32_t)(h >> 32);
        size_t i = (size_t)h & (vcap - 1);
        for (;;) {
            const uint64_t e = vslot[i];
            if (e == 0) break;
            const uint32_t id = (uint32_t)e - 1u;
            if ((uint32_t)(e >> 32) == tag && vkeys[id] == k) return id;
            i = (i + 1) & (vcap - 1);
        }
        const uint32_t id = (uint32_t)vkeys.size();
        vslot[i] = ((uint64_t)tag << 32) | (uint64_t)(id + 1u);
        vkeys.push_back(k);
        cv->verts.insert(cv->verts.end(), p, p + 3);
        return id;
    };
    FlatMap<uint64_t, EdgeInfo>& edges = sc.edges;
    edges.reset(ns);
    std::vector<uint64_t>& edge_keys = sc.edge_keys;  // distinct edges in first-seen order
    edge_keys.clear();
    edge_keys.reserve(ns);
    for (uint64_t s = 0; s < ns; s++) {
        const double* a = r->segs + 6 * s;
        const uint32_t u = vertex(a), v = vertex(a + 3);
        if (u == v) continue;  // touching point: an isolated vertex unless an edge reaches it
        const uint64_t k = u < v ? ((uint64_t)u << 32) | v : ((uint64_t)v << 32) | u;
        const int64_t q = r->seg_pair_at(s);
        const bool cop = q >= 0 && (uint64_t)q < r->npairs && per_pair[q] == 3;
        auto it = edges.emplace(k, EdgeInfo{}, mix64);
        if (it.second) edge_keys.push_back(k);
        EdgeInfo& e = *it.first;
        if (cop) e.coplanar++;
        else e.other++;
    }
    const uint32_t nv = (uint32_t)(cv->verts.size() / 3);
    std::vector<std::pair<uint32_t, uint32_t>>& el = sc.el;
    el.clear();
    el.reserve(edge_keys.size());
    for (uint64_t k : edge_keys) {
        const EdgeInfo& e = *edges.emplace(k, EdgeInfo{}, mix64).first;
        if (drop_coplanar_interior && e.other == 0 && e.coplanar >= 2) continue;
        el.emplace_back((uint32_t)(k >> 32), (uint32_t)(k & 0xffffffffu));
    }
    // edges in first-seen order: the curve order follows the segment order (deterministic)
    // adjacency (CSR)
    std::vector<uint32_t>& deg = sc.deg;
    deg.assign(nv + 1, 0);
    for (auto& e : el) {
        deg[e.first]++;
        deg[e.second]++;
    }
    std::vector<uint64_t>& start = sc.start;
    start.assign(nv + 1, 0);
    for (uint32_t v = 0; v < nv; v++) start[v + 1] = start[v] + deg[v];
    std::vector<uint32_t>& nbr = sc.nbr;
    std::vector<uint32_t>& nedge = sc.nedge;
    nbr.resize(2 * el.size());
    nedge.resize(2 * el.size());
    std::vector<uint64_t>& fill = sc.fill;
    fill.assign(start.begin(), start.end() - 1);
    for (uint32_t i = 0; i < (uint32_t)el.size(); i++) {
        const uint32_t a = el[i].first, b = el[i].second;
        nbr[fill[a]] = b;
        nedge[fill[a]++] = i;
        nbr[fill[b]] = a;
        nedge[fill[b]++] = i;
    }
    std::vector<uint8_t>& used = sc.used;
    used.assign(el.size(), 0);
    cv->offsets.push_back(0);
    auto walk = [&](uint32_t v0, uint64_t slot) {
        // follow unused edges from v0 through vertices of degree 2
        cv->idx.push_back(v0);
        uint64_t sl = slot;
        for (;;) {
            const uint32_t e = nedge[sl];
            used[e] = 1;
            const uint32_t w = nbr[sl];
            if (w == v0 && deg[v0] == 2) {
                cv->closed.push_back(1);
                break;
            }
            cv->idx.push_back(w);
            if (deg[w] != 2) {
                cv->closed.push_back(0);
                break;
            }
            uint64_t nx = start[w];
            if (used[nedge[nx]]) nx++;
            if (nx >= start[w + 1] || used[nedge[nx]]) {
                cv->closed.push_back(0);
                break;
            }
            sl = nx;
        }
        cv->offsets.push_back(cv->idx.size());
    };
    // open chains start at vertices of degree != 2
    for (uint32_t v = 0; v < nv; v++) {
        if (deg[v] == 2) continue;
        if (deg[v] == 0) {
            cv->idx.push_back(v);
            cv->closed.push_back(0);
            cv->offsets.push_back(cv->idx.size());
            continue;
        }
        for (uint64_t s = start[v]; s < start[v + 1]; s++)
            if (!used[nedge[s]]) walk(v, s);
    }
    // what remains is closed loops of degree-2 vertices
    for (uint32_t v = 0; v < nv; v++)
        for (uint64_t s = start[v]; s < start[v + 1]; s++)
            if (!used[nedge[s]]) walk(v, s);
}

extern "C" gi_status gi_curves_build(const double* seg6, const int32_t* seg_pair, uint64_t nsegs, uint64_t npairs,
                                     int32_t drop_coplanar_interior, gi_curves** out)
{
    if (!out || (nsegs && (!seg6 || !seg_pair))) return GI_ERR_INVALID_ARG;
    *out = nullptr;
    gi_curves* cv = new (std::nothrow) gi_curves();
    if (!cv) return GI_ERR_OOM;
    try {
        build_curves(seg6, seg_pair, 0, nsegs, npairs, drop_coplanar_interior, cv);
    } catch (const std::bad_alloc&) {
        delete cv;
        return GI_ERR_OOM;
    }
    *out = cv;
    return GI_OK;
}

extern "C" gi_status gi_curves_build_jobs(const double* seg6, const int64_t* seg_pair, uint64_t nsegs,
                                          const int64_t* pair_offsets, uint32_t njobs, int32_t drop_coplanar_interior,
                                          gi_curves** out)
{
    if (!out || !pair_offsets || (nsegs && (!seg6 || !seg_pair))) return GI_ERR_INVALID_ARG;
    *out = nullptr;
    for (uint32_t j = 0; j < njobs; j++)
        if (pair_offsets[j + 1] < pair_offsets[j]) return GI_ERR_INVALID_ARG;
    for (uint64_t s = 1; s < nsegs; s++)
        if (seg_pair[s] < seg_pair[s - 1]) return GI_ERR_INVALID_ARG;  // segments ordered by pair
    // each job's segment range (the segments are ordered by pair, the pairs by job)
    std::vector<uint64_t> sfirst(njobs + 1, 0);
    uint64_t s = 0;
    for (uint32_t j = 0; j < njobs; j++) {
        while (s < nsegs && seg_pair[s] < pair_offsets[j]) s++;
        sfirst[j] = s;
    }
    sfirst[njobs] = nsegs;
    gi_curves* cv = new (std::nothrow) gi_curves();
    if (!cv) return GI_ERR_OOM;
    std::vector<gi_curves> part(njobs);
    std::atomic<uint32_t> next{0};
    std::atomic<bool> oom{false};
    auto work = [&]() {
        for (;;) {
            const uint32_t j = next.fetch_add(1);
            if (j >= njobs) return;
            try {
                build_curves(seg6 + 6 * sfirst[j], seg_pair + sfirst[j], pair_offsets[j], sfirst[j + 1] - sfirst[j],
                             (uint64_t)(pair_offsets[j + 1] - pair_offsets[j]), drop_coplanar_interior, &part[j]);
            } catch (const std::bad_alloc&) {
                oom = true;
                return;
            }
        }
    };
    // the jobs are independent: host threads take them one at a time
    const unsigned nt = std::max(1u, std::min<unsigned>(std::thread::hardware_concurrency(), std::max(1u, njobs / 4u)));
    auto run = [&](auto&& body) {
        std::vector<std::thread> pool;
        for (unsigned t = 1; t < nt; t++) pool.emplace_back(body);
        body();
        for (auto& t : pool) t.join();
    };
    run(work);
    if (oom) {
        delete cv;
        return GI_ERR_OOM;
    }
    // concatenated in job order, vertex ids and curve offsets rebased: prefix
    // counts first, then each thread copies its jobs into place
    std::vector<uint64_t> vb(njobs + 1, 0), ib(njobs + 1, 0), cb(njobs + 1, 0);
    for (uint32_t j = 0; j < njobs; j++) {
        vb[j + 1] = vb[j] + part[j].verts.size() / 3;
        ib[j + 1] = ib[j] + part[j].idx.size();
        cb[j + 1] = cb[j] + part[j].closed.size();
    }
    try {
        cv->verts.resize(3 * vb[njobs]);
        cv->idx.resize(ib[njobs]);
        cv->closed.resize(cb[njobs]);
        cv->offsets.resize(cb[njobs] + 1);
        cv->job_curves.assign(cb.begin(), cb.end());
    } catch (const std::bad_alloc&) {
        delete cv;
        return GI_ERR_OOM;
    }
    cv->offsets[0] = 0;
    next = 0;
    run([&]() {
        for (;;) {
            const uint32_t j = next.fetch_add(1);
            if (j >= njobs) return;
            const gi_curves& p = part[j];
            std::copy(p.verts.begin(), p.verts.end(), cv->verts.begin() + 3 * vb[j]);
            const uint32_t v0 = (uint32_t)vb[j];
            for (size_t k = 0; k < p.idx.size(); k++) cv->idx[ib[j] + k] = v0 + p.idx[k];
            for (size_t c = 0; c < p.closed.size(); c++) {
                cv->closed[cb[j] + c] = p.closed[c];
                cv->offsets[cb[j] + c + 1] = ib[j] + p.offsets[c + 1];
            }
            gi_curves().verts.swap(const_cast<gi_curves&>(p).verts);  // release the part as it is copied
        }
    });
    *out = cv;
    return GI_OK;
}

extern "C" gi_status gi_curves_job_offsets(const gi_curves* c, const uint64_t** job_curves, uint64_t* njobs)
{
    if (!c || !job_curves || !njobs) return GI_ERR_INVALID_ARG;
    *job_curves = c->job_curves.data();
    *njobs = c->job_curves.empty() ? 0 : c->job_curves.size() - 1;
    return GI_OK;
}

extern "C" gi_status gi_result_curves(const gi_result* r, int32_t drop_coplanar_interior, gi_curves** out)
{
    if (!r || !out) return GI_ERR_INVALID_ARG;
    return gi_curves_build(r->segs, r->seg_pair, r->nsegs, r->npairs, drop_coplanar_interior, out);
}

extern "C" gi_status gi_curves_vertices(const gi_curves* c, const double** xyz, uint64_t* n)
{
    if (!c || !xyz || !n) return GI_ERR_INVALID_ARG;
    *xyz = c->verts.data();
    *n = c->verts.size() / 3;
    return GI_OK;
}

extern "C" gi_status gi_curves_polylines(const gi_curves* c, const uint64_t** offsets, const uint32_t** verts,
                                         const uint8_t** closed, uint64_t* ncurves)
{
    if (!c || !offsets || !verts || !closed || !ncurves) return GI_ERR_INVALID_ARG;
    *offsets = c->offsets.data();
    *verts = c->idx.data();
    *closed = c->closed.data();
    *ncurves = c->closed.size();
    return GI_OK;
}

extern "C" gi_status gi_curves_free(gi_curves* c)
{
    if (!c) return GI_ERR_INVALID_ARG;
    delete c;
    return GI_OK;
}
