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
#include <cstring>
#include <vector>

#include "gi_host.h"

struct gi_curves {
    std::vector<double> verts;         // 3 per vertex
    std::vector<uint64_t> offsets;     // curve c: vertex ids idx[offsets[c] .. offsets[c+1])
    std::vector<uint32_t> idx;
    std::vector<uint8_t> closed;       // 1: the curve closes (its last vertex joins its first)
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
// a node per entry.
template <class K, class V>
struct FlatMap {
    std::vector<K> keys;
    std::vector<V> vals;
    std::vector<uint8_t> used;
    size_t mask = 0;
    explicit FlatMap(size_t max_keys)
    {
        size_t cap = 16;
        while (cap < 2 * max_keys + 1) cap <<= 1;
        keys.resize(cap);
        vals.resize(cap);
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

}  // namespace

extern "C" gi_status gi_curves_build(const double* seg6, const int32_t* seg_pair, uint64_t nsegs, uint64_t npairs,
                                     int32_t drop_coplanar_interior, gi_curves** out)
{
    if (!out || (nsegs && (!seg6 || !seg_pair))) return GI_ERR_INVALID_ARG;
    *out = nullptr;
    gi_curves* cv = new (std::nothrow) gi_curves();
    if (!cv) return GI_ERR_OOM;
    struct {
        const double* segs;
        const int32_t* seg_pair;
        uint64_t nsegs, npairs;
    } rr{seg6, seg_pair, nsegs, npairs}, *r = &rr;
    const uint64_t ns = r->nsegs;
    // segments per pair: three mark a coplanar overlap triangle
    std::vector<uint32_t> per_pair(r->npairs, 0);
    for (uint64_t s = 0; s < ns; s++)
        if (r->seg_pair[s] >= 0 && (uint64_t)r->seg_pair[s] < r->npairs) per_pair[r->seg_pair[s]]++;
    // vertex table: 8-byte slots (hash tag, vertex id + 1) over keys stored once in vertex order
    size_t vcap = 16;
    while (vcap < 4 * ns + 1) vcap <<= 1;
    std::vector<uint64_t> vslot(vcap, 0);
    std::vector<PtKey> vkeys;
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
    struct EdgeInfo {
        uint32_t coplanar = 0, other = 0;
    };
    FlatMap<uint64_t, EdgeInfo> edges(ns);
    std::vector<uint64_t> edge_keys;  // distinct edges in first-seen order
    edge_keys.reserve(ns);
    for (uint64_t s = 0; s < ns; s++) {
        const double* a = r->segs + 6 * s;
        const uint32_t u = vertex(a), v = vertex(a + 3);
        if (u == v) continue;  // touching point: an isolated vertex unless an edge reaches it
        const uint64_t k = u < v ? ((uint64_t)u << 32) | v : ((uint64_t)v << 32) | u;
        const bool cop = r->seg_pair[s] >= 0 && (uint64_t)r->seg_pair[s] < r->npairs && per_pair[r->seg_pair[s]] == 3;
        auto it = edges.emplace(k, EdgeInfo{}, mix64);
        if (it.second) edge_keys.push_back(k);
        EdgeInfo& e = *it.first;
        if (cop) e.coplanar++;
        else e.other++;
    }
    const uint32_t nv = (uint32_t)(cv->verts.size() / 3);
    std::vector<std::pair<uint32_t, uint32_t>> el;
    el.reserve(edge_keys.size());
    for (uint64_t k : edge_keys) {
        const EdgeInfo& e = *edges.emplace(k, EdgeInfo{}, mix64).first;
        if (drop_coplanar_interior && e.other == 0 && e.coplanar >= 2) continue;
        el.emplace_back((uint32_t)(k >> 32), (uint32_t)(k & 0xffffffffu));
    }
    // edges in first-seen order: the curve order follows the segment order (deterministic)
    // adjacency (CSR)
    std::vector<uint32_t> deg(nv + 1, 0);
    for (auto& e : el) {
        deg[e.first]++;
        deg[e.second]++;
    }
    std::vector<uint64_t> start(nv + 1, 0);
    for (uint32_t v = 0; v < nv; v++) start[v + 1] = start[v] + deg[v];
    std::vector<uint32_t> nbr(2 * el.size()), nedge(2 * el.size());
    std::vector<uint64_t> fill(start.begin(), start.end() - 1);
    for (uint32_t i = 0; i < (uint32_t)el.size(); i++) {
        const uint32_t a = el[i].first, b = el[i].second;
        nbr[fill[a]] = b;
        nedge[fill[a]++] = i;
        nbr[fill[b]] = a;
        nedge[fill[b]++] = i;
    }
    std::vector<uint8_t> used(el.size(), 0);
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
    *out = cv;
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
