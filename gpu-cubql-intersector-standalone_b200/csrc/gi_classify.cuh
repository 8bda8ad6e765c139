// gi_classify.cuh -- triangle-pair predicates and constructions on the device.
//
// Semantics (reference project paths):
//   src/CPU/YellowFilter.h:80-137            CGAL::do_intersect on closed triangles
//   src/CPU/MeshIntersectionCurves.cpp:63-78 point / segment / triangle result kinds
//   src/GPU_exact_predicates/OriginShiftedFloatPredicateCore.cuh:72-141
//       the reference's FP32 filter: 6 vertex-vs-plane signs, then edge tests,
//       anything uncertain escalates.  Here the first stage is a semi-static
//       filter (value and error bound in FP32 from FP64 differences) instead of
//       interval arithmetic, and the follow-up is exact instead of CPU CGAL.
//
// Decision procedure for two proper triangles P, Q (all signs exact):
//   s2 = sides of Q's vertices w.r.t. plane(P), s1 = sides of P's w.r.t. plane(Q);
//   all of one triangle strictly on one side -> disjoint;
//   s2 all zero -> coplanar: exact 2D tests (vertex containment, proper edge
//   crossings, a separating-edge test for the dimension of the overlap);
//   otherwise I1 = P ∩ plane(Q) and I2 = Q ∩ plane(P) lie on the line
//   L = plane(P) ∩ plane(Q).  Each endpoint X of I1 is represented by an edge
//   (cn, cp) of P with side(cn) <= 0 <= side(cp) that crosses plane(Q) at X
//   (likewise Y of I2 with an edge of Q), and orient3d(cn_X, cp_X, cn_Y, cp_Y)
//   has the sign of pos(Y) - pos(X) along L up to one orientation constant per
//   pair.  Four such signs give I1 ∩ I2, i.e. the intersection.
// Degenerate (collinear) triangles are handled as the segment or point they span.
#pragma once
#include "gi_exact.cuh"
#include "gi_internal.cuh"

namespace gi {

constexpr int kUnsure = 2;
enum { KIND_NONE = 0, KIND_POINT = 1, KIND_SEGMENT = 2, KIND_TRIANGLE = 3, KIND_POLYGON = 4 };
enum { DEC_NO = 0, DEC_YES = 1, DEC_ESC = 2 };

// Vertex i of a mesh's vertex array (FP64 x, y, z), read as the two aligned
// 16-byte vectors that hold it: its 24 bytes start on a 16-byte boundary for
// even i and 8 bytes past one for odd i.  Two loads instead of three; the
// array must be 16-byte aligned and padded by 16 bytes past its last vertex
// (mesh uploads allocate it so).  The build's box kernel reads vertices this
// way; the intersection kernels keep three scalar loads (world_vertex), which
// measured faster there (0.127 against 0.129 ms per intersect of two
// 1.3M-triangle meshes).
__device__ __forceinline__ double3 load_vertex(const double* __restrict__ V, uint32_t i)
{
    const size_t o = 3 * (size_t)i;
    const double2* q = reinterpret_cast<const double2*>(V + (o & ~(size_t)1));
    const double2 a = __ldg(q), b = __ldg(q + 1);
    const bool odd = (i & 1u) != 0u;
    return make_double3(odd ? a.y : a.x, odd ? b.x : a.y, odd ? b.y : b.x);
}

// ---------------------------------------------------------------------------
// Posed vertex, bit-identical to the host order (RotationTools.h:135-143):
// x = v - C; r = (R0 x + R1 y) + R2 z; out = (r + C) + T; no fused multiply-add.
// ---------------------------------------------------------------------------
__device__ __forceinline__ double3 world_vertex(const double* __restrict__ V, uint32_t i, const DevPose& P)
{
    double x = __ldg(V + 3 * (size_t)i), y = __ldg(V + 3 * (size_t)i + 1), z = __ldg(V + 3 * (size_t)i + 2);
    if (P.identity) return make_double3(x, y, z);
    double dx = __dsub_rn(x, P.C[0]), dy = __dsub_rn(y, P.C[1]), dz = __dsub_rn(z, P.C[2]);
    double rx = __dadd_rn(__dadd_rn(__dmul_rn(P.R[0], dx), __dmul_rn(P.R[1], dy)), __dmul_rn(P.R[2], dz));
    double ry = __dadd_rn(__dadd_rn(__dmul_rn(P.R[3], dx), __dmul_rn(P.R[4], dy)), __dmul_rn(P.R[5], dz));
    double rz = __dadd_rn(__dadd_rn(__dmul_rn(P.R[6], dx), __dmul_rn(P.R[7], dy)), __dmul_rn(P.R[8], dz));
    return make_double3(__dadd_rn(__dadd_rn(rx, P.C[0]), P.T[0]), __dadd_rn(__dadd_rn(ry, P.C[1]), P.T[1]),
                        __dadd_rn(__dadd_rn(rz, P.C[2]), P.T[2]));
}

// ---------------------------------------------------------------------------
// Semi-static filters.  Inputs are FP64 differences of exact doubles, rounded
// once to T.  For V = f . (e1 x e2) the input rounding perturbs each of the 6
// triple products by at most (1+u1)^3 - 1 <= 3.0001u and the evaluation
// (5 roundings on any path) by gamma_5 <= 5.0001u, relative to
//   perm = sum_i |f_i| (|e1_j e2_k| + |e1_k e2_j|);
// the bound used is 10u * perm.  For FP32, a difference below 2^-126 converts
// with an absolute error up to 2^-150 and products may underflow; the term
// 2^-140 (1 + M)^2 (M = largest input magnitude) covers both, and M > 2^40
// (possible FP32 overflow) escalates.  FP64 needs no such term inside the
// supported coordinate domain.  Operations use explicit _rn intrinsics so the
// compiler cannot fuse them.
// ---------------------------------------------------------------------------
template <class T>
struct FP;
template <>
struct FP<float> {
    static __device__ __forceinline__ float cv(double x) { return __double2float_rn(x); }
    static __device__ __forceinline__ float mul(float a, float b) { return __fmul_rn(a, b); }
    static __device__ __forceinline__ float add(float a, float b) { return __fadd_rn(a, b); }
    static __device__ __forceinline__ float sub(float a, float b) { return __fsub_rn(a, b); }
    static __device__ __forceinline__ float ab(float a) { return fabsf(a); }
    static __device__ __forceinline__ float mx(float a, float b) { return fmaxf(a, b); }
    static constexpr float k3 = 10.0f * 0x1p-24f;
    static constexpr float k2 = 6.0f * 0x1p-24f;
    static __device__ __forceinline__ float abs3(float m) { return 0x1p-140f * (1.0f + m) * (1.0f + m); }
    static __device__ __forceinline__ float abs2(float m) { return 0x1p-144f * (1.0f + m); }
    static __device__ __forceinline__ bool too_big(float m) { return !(m <= 0x1p40f); }
};
template <>
struct FP<double> {
    static __device__ __forceinline__ double cv(double x) { return x; }
    static __device__ __forceinline__ double mul(double a, double b) { return __dmul_rn(a, b); }
    static __device__ __forceinline__ double add(double a, double b) { return __dadd_rn(a, b); }
    static __device__ __forceinline__ double sub(double a, double b) { return __dsub_rn(a, b); }
    static __device__ __forceinline__ double ab(double a) { return fabs(a); }
    static __device__ __forceinline__ double mx(double a, double b) { return fmax(a, b); }
    static constexpr double k3 = 10.0 * 0x1p-53;
    static constexpr double k2 = 6.0 * 0x1p-53;
    static __device__ __forceinline__ double abs3(double) { return 0.0; }
    static __device__ __forceinline__ double abs2(double) { return 0.0; }
    static __device__ __forceinline__ bool too_big(double) { return false; }
};

template <class T>
struct V3 {
    T x, y, z;
};
template <class T>
__device__ __forceinline__ V3<T> vdiff(const double3& a, const double3& b)
{
    return {FP<T>::cv(__dsub_rn(a.x, b.x)), FP<T>::cv(__dsub_rn(a.y, b.y)), FP<T>::cv(__dsub_rn(a.z, b.z))};
}
template <class T>
__device__ __forceinline__ T vmax(const V3<T>& a)
{
    using F = FP<T>;
    return F::mx(F::mx(F::ab(a.x), F::ab(a.y)), F::ab(a.z));
}

template <class T>
struct Plane {
    V3<T> n, pn;  // normal e1 x e2 and its per-component permanents
    T m;          // largest |e1|, |e2| component
    bool proper;  // normal certainly nonzero
};

template <class T>
__device__ __forceinline__ Plane<T> make_plane(const V3<T>& e1, const V3<T>& e2)
{
    using F = FP<T>;
    Plane<T> P;
    T a = F::mul(e1.y, e2.z), b = F::mul(e1.z, e2.y);
    P.n.x = F::sub(a, b);
    P.pn.x = F::add(F::ab(a), F::ab(b));
    a = F::mul(e1.z, e2.x);
    b = F::mul(e1.x, e2.z);
    P.n.y = F::sub(a, b);
    P.pn.y = F::add(F::ab(a), F::ab(b));
    a = F::mul(e1.x, e2.y);
    b = F::mul(e1.y, e2.x);
    P.n.z = F::sub(a, b);
    P.pn.z = F::add(F::ab(a), F::ab(b));
    P.m = F::mx(vmax(e1), vmax(e2));
    T a2 = F::abs2(P.m);
    P.proper = !F::too_big(P.m) &&
               (F::ab(P.n.x) > F::k2 * P.pn.x + a2 || F::ab(P.n.y) > F::k2 * P.pn.y + a2 ||
                F::ab(P.n.z) > F::k2 * P.pn.z + a2);
    return P;
}

// sign of f . n with the filter bound; kUnsure when uncertain
template <class T>
__device__ __forceinline__ int filt_dot(const Plane<T>& P, const V3<T>& f)
{
    using F = FP<T>;
    T v = F::add(F::add(F::mul(f.x, P.n.x), F::mul(f.y, P.n.y)), F::mul(f.z, P.n.z));
    T perm = F::add(F::add(F::mul(F::ab(f.x), P.pn.x), F::mul(F::ab(f.y), P.pn.y)), F::mul(F::ab(f.z), P.pn.z));
    T m = F::mx(P.m, vmax(f));
    if (F::too_big(m)) return kUnsure;
    T bound = F::k3 * perm + F::abs3(m);
    return v > bound ? 1 : (v < -bound ? -1 : kUnsure);
}

// orient3d(a,b,c,d) = det[a-d; b-d; c-d] = (a-d) . ((b-d) x (c-d)), filtered
template <class T>
__device__ __forceinline__ int filt_o3(const double3& a, const double3& b, const double3& c, const double3& d)
{
    Plane<T> P = make_plane<T>(vdiff<T>(b, d), vdiff<T>(c, d));
    return filt_dot<T>(P, vdiff<T>(a, d));
}

__device__ __forceinline__ int lone_index(const int s[3])
{
    if (s[0] != s[1] && s[0] != s[2]) return 0;
    if (s[1] != s[0] && s[1] != s[2]) return 1;
    return 2;
}

// Endpoint pattern of a pair that the first stage found intersecting: in
// general position the intersection is the segment between two of the four
// edge-plane crossings X0, X1 (P's edges from its lone vertex o1, in vertex
// order, through plane(Q)) and Y0, Y1 (Q's edges from o2 through plane(P));
// xin / yin mark the crossings that lie inside the other interval.  The exact
// classification gives the same points in the same order (X's, then Y's), so a
// consumer can construct them without evaluating any sign again.
//   bit 0 valid, bits 1-2 o1, bits 3-4 o2, bits 5-6 xin, bits 7-8 yin
constexpr unsigned kPatValid = 1u;
__device__ __forceinline__ unsigned make_pattern(int o1, int o2, unsigned xin, unsigned yin)
{
    return kPatValid | ((unsigned)o1 << 1) | ((unsigned)o2 << 3) | (xin << 5) | (yin << 7);
}

// First stage: decides the general-position case (every vertex strictly off the
// other triangle's plane) with filtered signs; everything else escalates.  For
// an intersecting pair, *pat receives its endpoint pattern (make_pattern).
// The vertex of three that `i` names (0, 1, 2), by selects (no indexed array).
__device__ __forceinline__ double3 sel3(int i, const double3& a, const double3& b, const double3& c)
{
    return i == 0 ? a : (i == 1 ? b : c);
}

// Index of the vertex whose sign differs from the other two (signs not all equal).
__device__ __forceinline__ int lone3(int s0, int s1, int s2)
{
    if (s0 != s1 && s0 != s2) return 0;
    if (s1 != s0 && s1 != s2) return 1;
    return 2;
}

// First stage: decides the general-position case (every vertex strictly off the
// other triangle's plane) with filtered signs; everything else escalates.  For
// an intersecting pair, *pat receives its endpoint pattern (make_pattern).
// Inlined, on values only (the vertex choices are selects), so that nothing of
// it lives in local memory.
template <class T>
__device__ __forceinline__ int classify_fast(const double3* P, const double3* Q, unsigned* pat = nullptr)
{
    const double3 P0 = P[0], P1 = P[1], P2 = P[2], Q0 = Q[0], Q1 = Q[1], Q2 = Q[2];
    const Plane<T> pp = make_plane<T>(vdiff<T>(P1, P0), vdiff<T>(P2, P0));
    if (!pp.proper) return DEC_ESC;
    // orient3d(P0,P1,P2,X) = (P0 - X) . nP
    const int s20 = filt_dot<T>(pp, vdiff<T>(P0, Q0)), s21 = filt_dot<T>(pp, vdiff<T>(P0, Q1)),
              s22 = filt_dot<T>(pp, vdiff<T>(P0, Q2));
    if ((s20 == 1 && s21 == 1 && s22 == 1) || (s20 == -1 && s21 == -1 && s22 == -1)) return DEC_NO;
    const Plane<T> pq = make_plane<T>(vdiff<T>(Q1, Q0), vdiff<T>(Q2, Q0));
    if (!pq.proper) return DEC_ESC;
    const int s10 = filt_dot<T>(pq, vdiff<T>(Q0, P0)), s11 = filt_dot<T>(pq, vdiff<T>(Q0, P1)),
              s12 = filt_dot<T>(pq, vdiff<T>(Q0, P2));
    if ((s10 == 1 && s11 == 1 && s12 == 1) || (s10 == -1 && s11 == -1 && s12 == -1)) return DEC_NO;
    if (s10 == kUnsure || s11 == kUnsure || s12 == kUnsure || s20 == kUnsure || s21 == kUnsure || s22 == kUnsure)
        return DEC_ESC;
    // both intervals consist of two edge crossings from the lone vertex; the
    // edges in vertex order of their other end, each from its negative end
    const int o1 = lone3(s10, s11, s12), o2 = lone3(s20, s21, s22);
    const bool neg1 = (o1 == 0 ? s10 : (o1 == 1 ? s11 : s12)) < 0;
    const bool neg2 = (o2 == 0 ? s20 : (o2 == 1 ? s21 : s22)) < 0;
    const double3 L1 = sel3(o1, P0, P1, P2), A1 = o1 == 0 ? P1 : P0, B1 = o1 == 2 ? P1 : P2;
    const double3 L2 = sel3(o2, Q0, Q1, Q2), A2 = o2 == 0 ? Q1 : Q0, B2 = o2 == 2 ? Q1 : Q2;
    const double3 xn0 = neg1 ? L1 : A1, xp0 = neg1 ? A1 : L1, xn1 = neg1 ? L1 : B1, xp1 = neg1 ? B1 : L1;
    const double3 yn0 = neg2 ? L2 : A2, yp0 = neg2 ? A2 : L2, yn1 = neg2 ? L2 : B2, yp1 = neg2 ? B2 : L2;
    const int c00 = filt_o3<T>(xn0, xp0, yn0, yp0);
    if (c00 == kUnsure) return DEC_ESC;
    const int c01 = filt_o3<T>(xn0, xp0, yn1, yp1);
    if (c01 == kUnsure) return DEC_ESC;
    const int c10 = filt_o3<T>(xn1, xp1, yn0, yp0);
    if (c10 == kUnsure) return DEC_ESC;
    const int c11 = filt_o3<T>(xn1, xp1, yn1, yp1);
    if (c11 == kUnsure) return DEC_ESC;
    const unsigned xin = (c00 * c01 < 0 ? 1u : 0u) | (c10 * c11 < 0 ? 2u : 0u);
    const unsigned yin = (c00 * c10 < 0 ? 1u : 0u) | (c01 * c11 < 0 ? 2u : 0u);
    if (!(xin | yin)) return DEC_NO;
    if (pat) *pat = make_pattern(o1, o2, xin, yin);
    return DEC_YES;
}

// ---------------------------------------------------------------------------
// Exact signs: FP64 filter (Shewchuk's orient3d/orient2d bound A, same
// operation order as the oracle), then integer arithmetic on a common grid.
// ---------------------------------------------------------------------------
// FP64 filter of one orient3d sign (Shewchuk's bound A): +1 / -1, or kUnsure.
__device__ __forceinline__ int o3_filter64(const double3& a, const double3& b, const double3& c, const double3& d)
{
    double adx = __dsub_rn(a.x, d.x), ady = __dsub_rn(a.y, d.y), adz = __dsub_rn(a.z, d.z);
    double bdx = __dsub_rn(b.x, d.x), bdy = __dsub_rn(b.y, d.y), bdz = __dsub_rn(b.z, d.z);
    double cdx = __dsub_rn(c.x, d.x), cdy = __dsub_rn(c.y, d.y), cdz = __dsub_rn(c.z, d.z);
    double bdxcdy = __dmul_rn(bdx, cdy), cdxbdy = __dmul_rn(cdx, bdy);
    double cdxady = __dmul_rn(cdx, ady), adxcdy = __dmul_rn(adx, cdy);
    double adxbdy = __dmul_rn(adx, bdy), bdxady = __dmul_rn(bdx, ady);
    double det = __dadd_rn(__dadd_rn(__dmul_rn(adz, __dsub_rn(bdxcdy, cdxbdy)),
                                     __dmul_rn(bdz, __dsub_rn(cdxady, adxcdy))),
                           __dmul_rn(cdz, __dsub_rn(adxbdy, bdxady)));
    double perm = __dadd_rn(
        __dadd_rn(__dmul_rn(__dadd_rn(fabs(bdxcdy), fabs(cdxbdy)), fabs(adz)),
                  __dmul_rn(__dadd_rn(fabs(cdxady), fabs(adxcdy)), fabs(bdz))),
        __dmul_rn(__dadd_rn(fabs(adxbdy), fabs(bdxady)), fabs(cdz)));
    double eb = __dmul_rn((7.0 + 56.0 * 0x1p-53) * 0x1p-53, perm);
    if (det > eb) return 1;
    if (-det > eb) return -1;
    return kUnsure;
}

// FP64 filter of one orient2d sign in the plane that drops axis `drop`
// (Shewchuk's bound A): +1 / -1, or kUnsure.
__device__ __forceinline__ int o2_filter64(const double3& a, const double3& b, const double3& c, int drop)
{
    const double* A = &a.x;
    const double* B = &b.x;
    const double* C = &c.x;
    int u = (drop + 1) % 3, v = (drop + 2) % 3;
    double l = __dmul_rn(__dsub_rn(A[u], C[u]), __dsub_rn(B[v], C[v]));
    double r = __dmul_rn(__dsub_rn(A[v], C[v]), __dsub_rn(B[u], C[u]));
    double det = __dsub_rn(l, r);
    double eb = __dmul_rn((3.0 + 16.0 * 0x1p-53) * 0x1p-53, __dadd_rn(fabs(l), fabs(r)));
    if (det > eb) return 1;
    if (-det > eb) return -1;
    return kUnsure;
}

struct ExactSigns {
    unsigned* err;
    unsigned long long nexact;

    __device__ __noinline__ int o3(const double3& a, const double3& b, const double3& c, const double3& d)
    {
        const int f = o3_filter64(a, b, c, d);
        if (f != kUnsure) return f;
        nexact++;
        return ex::o3_exact_sign(&a.x, &b.x, &c.x, &d.x, err);
    }
    __device__ __noinline__ int o2(const double3& a, const double3& b, const double3& c, int drop)
    {
        const int f = o2_filter64(a, b, c, drop);
        if (f != kUnsure) return f;
        nexact++;
        return ex::o2_exact_sign(&a.x, &b.x, &c.x, drop, err);
    }
};

// ---------------------------------------------------------------------------
// Exact classification with symbolic result points.
// pts[0..2] = triangle P, pts[3..5] = triangle Q.
// ---------------------------------------------------------------------------
enum { PK_VERTEX = 0, PK_PLANE = 1, PK_LINE2 = 2 };
struct SymPt {
    unsigned char kind, a, b, p, q, r, drop, pad;
};
struct TTRes {
    int kind;
    int n;
    SymPt pt[6];
};

__device__ __forceinline__ SymPt sp_vertex(int a)
{
    SymPt s = {PK_VERTEX, (unsigned char)a, 0, 0, 0, 0, 0, 0};
    return s;
}
__device__ __forceinline__ SymPt sp_plane(int a, int b, int p, int q, int r)
{
    SymPt s = {PK_PLANE, (unsigned char)a, (unsigned char)b, (unsigned char)p, (unsigned char)q, (unsigned char)r, 0, 0};
    return s;
}
__device__ __forceinline__ SymPt sp_line2(int a, int b, int p, int q, int drop)
{
    SymPt s = {PK_LINE2, (unsigned char)a, (unsigned char)b, (unsigned char)p, (unsigned char)q, 0,
               (unsigned char)drop, 0};
    return s;
}
__device__ __forceinline__ const double* cp(const double3* pts, int i)
{
    return &pts[i].x;
}
__device__ __forceinline__ bool pt_eq(const double3& a, const double3& b)
{
    return a.x == b.x && a.y == b.y && a.z == b.z;
}
__device__ __forceinline__ bool within_bounds(const double3& a, const double3& b, const double3& c)
{
    const double* A = &a.x;
    const double* B = &b.x;
    const double* C = &c.x;
    for (int k = 0; k < 3; k++) {
        double lo = A[k] < B[k] ? A[k] : B[k];
        double hi = A[k] < B[k] ? B[k] : A[k];
        if (C[k] < lo || C[k] > hi) return false;
    }
    return true;
}

struct Shape {
    int shape;  // 2 proper, 1 segment, 0 point
    int drop;
    int e0, e1;
};

static __device__ __noinline__ Shape tri_shape(const double3* pts, int base, ExactSigns& S)
{
    Shape s;
    s.drop = -1;
    s.e0 = s.e1 = base;
    const double* v0 = cp(pts, base);
    const double* v1 = cp(pts, base + 1);
    const double* v2 = cp(pts, base + 2);
    double n[3];
    for (int k = 0; k < 3; k++) {
        int u = (k + 1) % 3, w = (k + 2) % 3;
        n[k] = fabs((v1[u] - v0[u]) * (v2[w] - v0[w]) - (v1[w] - v0[w]) * (v2[u] - v0[u]));
    }
    int order[3] = {0, 1, 2};
    for (int i = 0; i < 3; i++)
        for (int j = i + 1; j < 3; j++)
            if (n[order[j]] > n[order[i]]) {
                int t = order[i];
                order[i] = order[j];
                order[j] = t;
            }
    for (int i = 0; i < 3; i++)
        if (S.o2(pts[base], pts[base + 1], pts[base + 2], order[i]) != 0) {
            s.shape = 2;
            s.drop = order[i];
            return s;
        }
    if (pt_eq(pts[base], pts[base + 1]) && pt_eq(pts[base + 1], pts[base + 2])) {
        s.shape = 0;
        return s;
    }
    int m = 0;
    for (int k = 0; k < 3; k++)
        if (!(v0[k] == v1[k] && v1[k] == v2[k])) {
            m = k;
            break;
        }
    int imin = 0, imax = 0;
    for (int i = 1; i < 3; i++) {
        if (cp(pts, base + i)[m] < cp(pts, base + imin)[m]) imin = i;
        if (cp(pts, base + i)[m] > cp(pts, base + imax)[m]) imax = i;
    }
    s.shape = 1;
    s.e0 = base + imin;
    s.e1 = base + imax;
    return s;
}

static __device__ __noinline__ bool pt_in_tri2d(const double3* pts, int p, int t0, int drop, ExactSigns& S)
{
    int s0 = S.o2(pts[t0], pts[t0 + 1], pts[p], drop);
    int s1 = S.o2(pts[t0 + 1], pts[t0 + 2], pts[p], drop);
    int s2 = S.o2(pts[t0 + 2], pts[t0], pts[p], drop);
    bool pos = s0 > 0 || s1 > 0 || s2 > 0, neg = s0 < 0 || s1 < 0 || s2 < 0;
    return !(pos && neg);
}
static __device__ __noinline__ bool collinear3(const double3* pts, int a, int b, int c, ExactSigns& S)
{
    return S.o2(pts[a], pts[b], pts[c], 0) == 0 && S.o2(pts[a], pts[b], pts[c], 1) == 0 &&
           S.o2(pts[a], pts[b], pts[c], 2) == 0;
}

// --- rational parameters along a segment e0->e1 (degenerate triangles only) ---
struct ParamPt {
    SymPt pt;
    int kind;  // 0: vertex w (index pt.a), 1: cut by 2D line (p,q)
};
// exact value of the parameter as num/den on the grid of pts (scale-free ratio)
static __device__ __noinline__ bool param_value(const double3* pts, const ParamPt& x, int e0, int e1, int m,
                                         const ex::Grid& g, ex::Big& num, ex::Big& den)
{
    using namespace ex;
    bool ok = true;
    if (x.kind == 0) {
        Big w, a, b;
        ok &= big_from_bits(dbits(cp(pts, x.pt.a)[m]), g.E, w);
        ok &= big_from_bits(dbits(cp(pts, e0)[m]), g.E, a);
        ok &= big_from_bits(dbits(cp(pts, e1)[m]), g.E, b);
        ok &= big_addsub(w, a, -1, num);
        ok &= big_addsub(b, a, -1, den);
        return ok;
    }
    Big P[3], Q[3], A[3], B[3], sb;
    for (int k = 0; k < 3; k++) {
        ok &= big_from_bits(dbits(cp(pts, x.pt.p)[k]), g.E, P[k]);
        ok &= big_from_bits(dbits(cp(pts, x.pt.q)[k]), g.E, Q[k]);
        ok &= big_from_bits(dbits(cp(pts, e0)[k]), g.E, A[k]);
        ok &= big_from_bits(dbits(cp(pts, e1)[k]), g.E, B[k]);
    }
    ok &= big_o2_value(P, Q, A, x.pt.drop, num);
    ok &= big_o2_value(P, Q, B, x.pt.drop, sb);
    ok &= big_addsub(num, sb, -1, den);
    return ok;
}
static __device__ __noinline__ int param_cmp(const double3* pts, const ParamPt& x, const ParamPt& y, int e0, int e1,
                                      int m, unsigned* err)
{
    using namespace ex;
    Grid g = grid_begin();
    for (int i = 0; i < 6; i++)
        for (int k = 0; k < 3; k++) grid_add(g, dbits(cp(pts, i)[k]));
    grid_finish(g);
    Big n1, d1, n2, d2, t1, t2;
    bool ok = param_value(pts, x, e0, e1, m, g, n1, d1);
    ok &= param_value(pts, y, e0, e1, m, g, n2, d2);
    ok &= big_mul(n1, d2, t1);
    ok &= big_mul(n2, d1, t2);
    ok &= big_addsub(t1, t2, -1, t1);
    if (!ok) {
        atomicOr(err, kErrExactCapacity);
        return 0;
    }
    return big_sign(t1) * big_sign(d1) * big_sign(d2);
}

__device__ __forceinline__ int seg_axis(const double3& a, const double3& b)
{
    const double* A = &a.x;
    const double* B = &b.x;
    double best = -1.0;
    int m = 0;
    for (int k = 0; k < 3; k++) {
        double d = fabs(B[k] - A[k]);
        if (B[k] != A[k] && d > best) {
            best = d;
            m = k;
        }
    }
    return m;
}

static __device__ __noinline__ void seg_tri(const double3* pts, int e0, int e1, int t0, int drop, TTRes& r, ExactSigns& S)
{
    int s0 = S.o3(pts[t0], pts[t0 + 1], pts[t0 + 2], pts[e0]);
    int s1 = S.o3(pts[t0], pts[t0 + 1], pts[t0 + 2], pts[e1]);
    r.n = 0;
    if (s0 * s1 > 0) {
        r.kind = KIND_NONE;
        return;
    }
    if (s0 != 0 || s1 != 0) {
        SymPt x = s0 == 0 ? sp_vertex(e0) : (s1 == 0 ? sp_vertex(e1) : sp_plane(e0, e1, t0, t0 + 1, t0 + 2));
        int a = S.o3(pts[e0], pts[e1], pts[t0], pts[t0 + 1]);
        int b = S.o3(pts[e0], pts[e1], pts[t0 + 1], pts[t0 + 2]);
        int c = S.o3(pts[e0], pts[e1], pts[t0 + 2], pts[t0]);
        bool pos = a > 0 || b > 0 || c > 0, neg = a < 0 || b < 0 || c < 0;
        if (pos && neg) {
            r.kind = KIND_NONE;
            return;
        }
        r.kind = KIND_POINT;
        r.pt[r.n++] = x;
        return;
    }
    ParamPt c[8];
    int nc = 0;
    int m = seg_axis(pts[e0], pts[e1]);
    if (pt_in_tri2d(pts, e0, t0, drop, S)) c[nc++] = {sp_vertex(e0), 0};
    if (pt_in_tri2d(pts, e1, t0, drop, S)) c[nc++] = {sp_vertex(e1), 0};
    for (int k = 0; k < 3; k++) {
        int w0 = t0 + k, w1 = t0 + (k + 1) % 3;
        int da = S.o2(pts[w0], pts[w1], pts[e0], drop), db = S.o2(pts[w0], pts[w1], pts[e1], drop);
        int d3 = S.o2(pts[e0], pts[e1], pts[w0], drop), d4 = S.o2(pts[e0], pts[e1], pts[w1], drop);
        if (da * db < 0 && d3 * d4 < 0) c[nc++] = {sp_line2(e0, e1, w0, w1, drop), 1};
    }
    for (int k = 0; k < 3; k++) {
        int w = t0 + k;
        if (S.o2(pts[e0], pts[e1], pts[w], drop) == 0 && within_bounds(pts[e0], pts[e1], pts[w]) &&
            !pt_eq(pts[w], pts[e0]) && !pt_eq(pts[w], pts[e1]))
            c[nc++] = {sp_vertex(w), 0};
    }
    if (nc == 0) {
        r.kind = KIND_NONE;
        return;
    }
    int imin = 0, imax = 0;
    for (int i = 1; i < nc; i++) {
        if (param_cmp(pts, c[i], c[imin], e0, e1, m, S.err) < 0) imin = i;
        if (param_cmp(pts, c[i], c[imax], e0, e1, m, S.err) > 0) imax = i;
    }
    if (param_cmp(pts, c[imin], c[imax], e0, e1, m, S.err) == 0) {
        r.kind = KIND_POINT;
        r.pt[r.n++] = c[imin].pt;
    } else {
        r.kind = KIND_SEGMENT;
        r.pt[r.n++] = c[imin].pt;
        r.pt[r.n++] = c[imax].pt;
    }
}

static __device__ __noinline__ void seg_seg(const double3* pts, int e0, int e1, int f0, int f1, TTRes& r, ExactSigns& S)
{
    r.n = 0;
    r.kind = KIND_NONE;
    if (S.o3(pts[e0], pts[e1], pts[f0], pts[f1]) != 0) return;
    bool c0 = collinear3(pts, e0, e1, f0, S), c1 = collinear3(pts, e0, e1, f1, S);
    if (c0 && c1) {
        int m = seg_axis(pts[e0], pts[e1]);
        int ea = cp(pts, e0)[m] < cp(pts, e1)[m] ? e0 : e1;
        int eb = cp(pts, e0)[m] < cp(pts, e1)[m] ? e1 : e0;
        int fa = cp(pts, f0)[m] < cp(pts, f1)[m] ? f0 : f1;
        int fb = cp(pts, f0)[m] < cp(pts, f1)[m] ? f1 : f0;
        int lo = cp(pts, ea)[m] >= cp(pts, fa)[m] ? ea : fa;
        int hi = cp(pts, eb)[m] <= cp(pts, fb)[m] ? eb : fb;
        if (cp(pts, lo)[m] > cp(pts, hi)[m]) return;
        if (cp(pts, lo)[m] == cp(pts, hi)[m]) {
            r.kind = KIND_POINT;
            r.pt[r.n++] = sp_vertex(lo);
            return;
        }
        r.kind = KIND_SEGMENT;
        r.pt[r.n++] = sp_vertex(lo);
        r.pt[r.n++] = sp_vertex(hi);
        return;
    }
    int fx = c0 ? f1 : f0;
    int drop = 0;
    for (int k = 0; k < 3; k++)
        if (S.o2(pts[e0], pts[e1], pts[fx], k) != 0) {
            drop = k;
            break;
        }
    int d1 = S.o2(pts[f0], pts[f1], pts[e0], drop), d2 = S.o2(pts[f0], pts[f1], pts[e1], drop);
    int d3 = S.o2(pts[e0], pts[e1], pts[f0], drop), d4 = S.o2(pts[e0], pts[e1], pts[f1], drop);
    if (d1 * d2 < 0 && d3 * d4 < 0) {
        r.kind = KIND_POINT;
        r.pt[r.n++] = sp_line2(e0, e1, f0, f1, drop);
        return;
    }
    int touch = -1;
    if (d1 == 0 && within_bounds(pts[f0], pts[f1], pts[e0])) touch = e0;
    else if (d2 == 0 && within_bounds(pts[f0], pts[f1], pts[e1])) touch = e1;
    else if (d3 == 0 && within_bounds(pts[e0], pts[e1], pts[f0])) touch = f0;
    else if (d4 == 0 && within_bounds(pts[e0], pts[e1], pts[f1])) touch = f1;
    if (touch >= 0) {
        r.kind = KIND_POINT;
        r.pt[r.n++] = sp_vertex(touch);
    }
}

static __device__ __noinline__ void coplanar_tt(const double3* pts, int drop, TTRes& r, ExactSigns& S)
{
    int sig1 = S.o2(pts[0], pts[1], pts[2], drop);
    int sig2 = S.o2(pts[3], pts[4], pts[5], drop);
    int E2[3][3], E1[3][3];
    for (int j = 0; j < 3; j++)
        for (int i = 0; i < 3; i++) E2[j][i] = sig2 * S.o2(pts[3 + j], pts[3 + (j + 1) % 3], pts[i], drop);
    for (int i = 0; i < 3; i++)
        for (int j = 0; j < 3; j++) E1[i][j] = sig1 * S.o2(pts[i], pts[(i + 1) % 3], pts[3 + j], drop);
    bool v1in[3], v2in[3], any = false;
    for (int i = 0; i < 3; i++) {
        v1in[i] = E2[0][i] >= 0 && E2[1][i] >= 0 && E2[2][i] >= 0;
        any |= v1in[i];
    }
    for (int j = 0; j < 3; j++) {
        v2in[j] = E1[0][j] >= 0 && E1[1][j] >= 0 && E1[2][j] >= 0;
        any |= v2in[j];
    }
    bool prop[3][3];
    int nprop = 0;
    for (int i = 0; i < 3; i++)
        for (int j = 0; j < 3; j++) {
            int d1 = E2[j][i], d2 = E2[j][(i + 1) % 3], d3 = E1[i][j], d4 = E1[i][(j + 1) % 3];
            prop[i][j] = (d1 * d2 < 0) && (d3 * d4 < 0);
            nprop += prop[i][j];
        }
    r.n = 0;
    if (!any && nprop == 0) {
        r.kind = KIND_NONE;
        return;
    }
    bool sep = false;
    for (int j = 0; j < 3 && !sep; j++)
        if (E2[j][0] <= 0 && E2[j][1] <= 0 && E2[j][2] <= 0) sep = true;
    for (int i = 0; i < 3 && !sep; i++)
        if (E1[i][0] <= 0 && E1[i][1] <= 0 && E1[i][2] <= 0) sep = true;
    int vp[6];
    int nv = 0;
    for (int i = 0; i < 3; i++)
        if (v1in[i]) vp[nv++] = i;
    for (int j = 0; j < 3; j++) {
        if (!v2in[j]) continue;
        bool dup = false;
        for (int k = 0; k < nv; k++)
            if (pt_eq(pts[vp[k]], pts[3 + j])) dup = true;
        if (!dup) vp[nv++] = 3 + j;
    }
    if (!sep) {
        for (int k = 0; k < nv; k++) r.pt[r.n++] = sp_vertex(vp[k]);
        for (int i = 0; i < 3; i++)
            for (int j = 0; j < 3; j++)
                if (prop[i][j]) r.pt[r.n++] = sp_line2(i, (i + 1) % 3, 3 + j, 3 + (j + 1) % 3, drop);
        r.kind = r.n == 3 ? KIND_TRIANGLE : KIND_POLYGON;
        return;
    }
    if (nv == 1) {
        r.kind = KIND_POINT;
        r.pt[r.n++] = sp_vertex(vp[0]);
        return;
    }
    int m = 0;
    for (int k = 0; k < 3; k++) {
        bool same = true;
        for (int q = 1; q < nv; q++)
            if (cp(pts, vp[q])[k] != cp(pts, vp[0])[k]) same = false;
        if (!same) {
            m = k;
            break;
        }
    }
    int imin = 0, imax = 0;
    for (int q = 1; q < nv; q++) {
        if (cp(pts, vp[q])[m] < cp(pts, vp[imin])[m]) imin = q;
        if (cp(pts, vp[q])[m] > cp(pts, vp[imax])[m]) imax = q;
    }
    r.kind = KIND_SEGMENT;
    r.pt[r.n++] = sp_vertex(vp[imin]);
    r.pt[r.n++] = sp_vertex(vp[imax]);
}

struct LinePt {
    SymPt pt;
    int cn, cpos;  // crossing representation: side(cn) <= 0 <= side(cpos)
};

// interval T ∩ plane(O) from the sides s of T's vertices (T, O = base indices 0 or 3)
__device__ __forceinline__ int build_interval(int T, const int s[3], int O, LinePt out[2])
{
    int z = (s[0] == 0) + (s[1] == 0) + (s[2] == 0);
    if (z == 2) {
        int o = s[0] != 0 ? 0 : (s[1] != 0 ? 1 : 2);
        int k = 0;
        for (int i = 0; i < 3; i++) {
            if (i == o) continue;
            out[k].pt = sp_vertex(T + i);
            out[k].cn = s[o] < 0 ? T + o : T + i;
            out[k].cpos = s[o] < 0 ? T + i : T + o;
            k++;
        }
        return 2;
    }
    if (z == 1) {
        int u = s[0] == 0 ? 0 : (s[1] == 0 ? 1 : 2);
        int x = (u + 1) % 3, y = (u + 2) % 3;
        out[0].pt = sp_vertex(T + u);
        out[0].cn = s[x] < 0 ? T + x : T + u;
        out[0].cpos = s[x] < 0 ? T + u : T + x;
        if (s[x] * s[y] > 0) return 1;
        out[1].pt = sp_plane(T + x, T + y, O, O + 1, O + 2);
        out[1].cn = s[x] < 0 ? T + x : T + y;
        out[1].cpos = s[x] < 0 ? T + y : T + x;
        return 2;
    }
    int o = lone_index(s);
    int k = 0;
    for (int i = 0; i < 3; i++) {
        if (i == o) continue;
        out[k].pt = sp_plane(T + o, T + i, O, O + 1, O + 2);
        out[k].cn = s[o] < 0 ? T + o : T + i;
        out[k].cpos = s[o] < 0 ? T + i : T + o;
        k++;
    }
    return 2;
}

static __device__ __noinline__ void general_tt(const double3* pts, const int s1[3], const int s2[3], TTRes& r, ExactSigns& S)
{
    LinePt I1[2], I2[2];
    int n1 = build_interval(0, s1, 3, I1);
    int n2 = build_interval(3, s2, 0, I2);
    int c[2][2] = {{0, 0}, {0, 0}};
    for (int i = 0; i < n1; i++)
        for (int j = 0; j < n2; j++) c[i][j] = S.o3(pts[I1[i].cn], pts[I1[i].cpos], pts[I2[j].cn], pts[I2[j].cpos]);
    bool xin[2] = {false, false}, yin[2] = {false, false};
    for (int i = 0; i < n1; i++) xin[i] = (n2 == 1) ? (c[i][0] == 0) : (c[i][0] * c[i][1] <= 0);
    for (int j = 0; j < n2; j++) yin[j] = (n1 == 1) ? (c[0][j] == 0) : (c[0][j] * c[1][j] <= 0);
    r.n = 0;
    for (int i = 0; i < n1; i++)
        if (xin[i]) r.pt[r.n++] = I1[i].pt;
    for (int j = 0; j < n2; j++) {
        if (!yin[j]) continue;
        bool dup = false;
        for (int i = 0; i < n1; i++)
            if (xin[i] && c[i][j] == 0) dup = true;
        if (!dup) r.pt[r.n++] = I2[j].pt;
    }
    r.kind = r.n == 0 ? KIND_NONE : (r.n == 1 ? KIND_POINT : KIND_SEGMENT);
}

static __device__ __noinline__ void classify_exact(const double3* pts, TTRes& r, ExactSigns& S)
{
    r.n = 0;
    r.kind = KIND_NONE;
    Shape sp = tri_shape(pts, 0, S), sq = tri_shape(pts, 3, S);
    if (sp.shape == 2 && sq.shape == 2) {
        int s1[3], s2[3];
        for (int j = 0; j < 3; j++) s2[j] = S.o3(pts[0], pts[1], pts[2], pts[3 + j]);
        if ((s2[0] > 0 && s2[1] > 0 && s2[2] > 0) || (s2[0] < 0 && s2[1] < 0 && s2[2] < 0)) return;
        for (int i = 0; i < 3; i++) s1[i] = S.o3(pts[3], pts[4], pts[5], pts[i]);
        if ((s1[0] > 0 && s1[1] > 0 && s1[2] > 0) || (s1[0] < 0 && s1[1] < 0 && s1[2] < 0)) return;
        if (s2[0] == 0 && s2[1] == 0 && s2[2] == 0) {
            coplanar_tt(pts, sp.drop, r, S);
            return;
        }
        general_tt(pts, s1, s2, r, S);
        return;
    }
    if (sp.shape == 2 && sq.shape == 1) { seg_tri(pts, sq.e0, sq.e1, 0, sp.drop, r, S); return; }
    if (sp.shape == 1 && sq.shape == 2) { seg_tri(pts, sp.e0, sp.e1, 3, sq.drop, r, S); return; }
    if (sp.shape == 2 && sq.shape == 0) {
        if (S.o3(pts[0], pts[1], pts[2], pts[sq.e0]) == 0 && pt_in_tri2d(pts, sq.e0, 0, sp.drop, S)) {
            r.kind = KIND_POINT;
            r.pt[r.n++] = sp_vertex(sq.e0);
        }
        return;
    }
    if (sp.shape == 0 && sq.shape == 2) {
        if (S.o3(pts[3], pts[4], pts[5], pts[sp.e0]) == 0 && pt_in_tri2d(pts, sp.e0, 3, sq.drop, S)) {
            r.kind = KIND_POINT;
            r.pt[r.n++] = sp_vertex(sp.e0);
        }
        return;
    }
    if (sp.shape == 1 && sq.shape == 1) { seg_seg(pts, sp.e0, sp.e1, sq.e0, sq.e1, r, S); return; }
    if (sp.shape == 1 && sq.shape == 0) {
        if (collinear3(pts, sp.e0, sp.e1, sq.e0, S) && within_bounds(pts[sp.e0], pts[sp.e1], pts[sq.e0])) {
            r.kind = KIND_POINT;
            r.pt[r.n++] = sp_vertex(sq.e0);
        }
        return;
    }
    if (sp.shape == 0 && sq.shape == 1) {
        if (collinear3(pts, sq.e0, sq.e1, sp.e0, S) && within_bounds(pts[sq.e0], pts[sq.e1], pts[sp.e0])) {
            r.kind = KIND_POINT;
            r.pt[r.n++] = sp_vertex(sp.e0);
        }
        return;
    }
    if (pt_eq(pts[sp.e0], pts[sq.e0])) {
        r.kind = KIND_POINT;
        r.pt[r.n++] = sp_vertex(sp.e0);
    }
}

// ---------------------------------------------------------------------------
// Double-double arithmetic (error-free transforms; the DW algorithms analysed
// by Joldes, Muller & Popescu, "Tight and rigorous error bounds for basic
// building blocks of double-word arithmetic", 2017).
// ---------------------------------------------------------------------------
struct dd {
    double hi, lo;
};
__device__ __forceinline__ dd two_sum_dd(double a, double b)
{
    double s = __dadd_rn(a, b);
    double bv = __dsub_rn(s, a);
    double av = __dsub_rn(s, bv);
    return {s, __dadd_rn(__dsub_rn(a, av), __dsub_rn(b, bv))};
}
__device__ __forceinline__ dd fast_two_sum_dd(double a, double b)
{
    double s = __dadd_rn(a, b);
    return {s, __dsub_rn(b, __dsub_rn(s, a))};
}
__device__ __forceinline__ dd two_diff_dd(double a, double b)
{
    return two_sum_dd(a, -b);
}
__device__ __forceinline__ dd dd_add(dd x, dd y)  // AccurateDWPlusDW, rel. err <= 3u^2/(1-4u)
{
    dd s = two_sum_dd(x.hi, y.hi);
    dd t = two_sum_dd(x.lo, y.lo);
    double c = __dadd_rn(s.lo, t.hi);
    dd v = fast_two_sum_dd(s.hi, c);
    double w = __dadd_rn(t.lo, v.lo);
    return fast_two_sum_dd(v.hi, w);
}
__device__ __forceinline__ dd dd_neg(dd x)
{
    return {-x.hi, -x.lo};
}
__device__ __forceinline__ dd dd_mul(dd x, dd y)  // DWTimesDW3, rel. err <= 4u^2
{
    double ch = __dmul_rn(x.hi, y.hi);
    double cl1 = fma(x.hi, y.hi, -ch);
    double tl0 = __dmul_rn(x.lo, y.lo);
    double tl1 = fma(x.hi, y.lo, tl0);
    double cl2 = fma(x.lo, y.hi, tl1);
    double cl3 = __dadd_rn(cl1, cl2);
    return fast_two_sum_dd(ch, cl3);
}
__device__ __forceinline__ dd dd_mul_d(dd x, double y)  // DWTimesFP3, rel. err <= 2u^2
{
    double ch = __dmul_rn(x.hi, y);
    double cl1 = fma(x.hi, y, -ch);
    double cl3 = fma(x.lo, y, cl1);
    return fast_two_sum_dd(ch, cl3);
}
__device__ __forceinline__ dd dd_div(dd x, dd y)  // DWDivDW2, rel. err <= 15u^2 + 56u^3
{
    double th = __ddiv_rn(x.hi, y.hi);
    dd r = dd_mul_d(y, th);
    dd pi = two_sum_dd(x.hi, -r.hi);
    double dh = __dsub_rn(pi.lo, r.lo);
    double dl = __dadd_rn(dh, x.lo);
    double d = __dadd_rn(pi.hi, dl);
    double tl = __ddiv_rn(d, y.hi);
    return fast_two_sum_dd(th, tl);
}

// orient3d(p,q,r,x) = det[p-x; q-x; r-x] in double-double; *perm receives the
// permanent.  |error| <= 21u^2 perm (4u^2 products, 3u^2 sums); callers use 64u^2.
__device__ __forceinline__ dd o3_dd_f(const double3& p, const double3& q, const double3& r, const double3& x,
                                     double* perm)
{
    dd adx = two_diff_dd(p.x, x.x), ady = two_diff_dd(p.y, x.y), adz = two_diff_dd(p.z, x.z);
    dd bdx = two_diff_dd(q.x, x.x), bdy = two_diff_dd(q.y, x.y), bdz = two_diff_dd(q.z, x.z);
    dd cdx = two_diff_dd(r.x, x.x), cdy = two_diff_dd(r.y, x.y), cdz = two_diff_dd(r.z, x.z);
    dd p1 = dd_mul(bdx, cdy), p2 = dd_mul(cdx, bdy);
    dd p3 = dd_mul(cdx, ady), p4 = dd_mul(adx, cdy);
    dd p5 = dd_mul(adx, bdy), p6 = dd_mul(bdx, ady);
    dd m1 = dd_add(p1, dd_neg(p2)), m2 = dd_add(p3, dd_neg(p4)), m3 = dd_add(p5, dd_neg(p6));
    dd det = dd_add(dd_add(dd_mul(adz, m1), dd_mul(bdz, m2)), dd_mul(cdz, m3));
    *perm = (fabs(p1.hi) + fabs(p2.hi)) * fabs(adz.hi) + (fabs(p3.hi) + fabs(p4.hi)) * fabs(bdz.hi) +
            (fabs(p5.hi) + fabs(p6.hi)) * fabs(cdz.hi);
    return det;
}
static __device__ __noinline__ dd o3_dd(const double3& p, const double3& q, const double3& r, const double3& x, double* perm)
{
    return o3_dd_f(p, q, r, x, perm);
}
// orient2d(p,q,x) on the projection dropping `drop`; |error| <= 15u^2 perm
static __device__ __noinline__ dd o2_dd(const double3& p, const double3& q, const double3& x, int drop, double* perm)
{
    const double* P = &p.x;
    const double* Q = &q.x;
    const double* X = &x.x;
    int u = (drop + 1) % 3, v = (drop + 2) % 3;
    dd l = dd_mul(two_diff_dd(P[u], X[u]), two_diff_dd(Q[v], X[v]));
    dd rr = dd_mul(two_diff_dd(P[v], X[v]), two_diff_dd(Q[u], X[u]));
    *perm = fabs(l.hi) + fabs(rr.hi);
    return dd_add(l, dd_neg(rr));
}

// ---------------------------------------------------------------------------
// Constructed point X = a + t (b - a), t = sa / (sa - sb), sa and sb of strictly
// opposite signs.  Fast path: double-double value and a rigorous error bound;
// the result is accepted when the whole error interval rounds to one double
// (Ziv's rounding test), otherwise the exact integer path decides.  Both give
// the correctly rounded coordinate.
// ---------------------------------------------------------------------------
__device__ __forceinline__ bool ziv_round(dd x, double err, double* out)
{
    double hi = x.hi;
    if (!(err < 1e300) || hi == 0.0) return false;
    double up = nextafter(hi, INFINITY) - hi;
    double dn = hi - nextafter(hi, -INFINITY);
    double e = err * (1.0 + 0x1p-20) + 0x1p-1074;
    if (x.lo + e < 0.5 * up && x.lo - e > -0.5 * dn) {
        *out = hi;
        return true;
    }
    return false;
}

static __device__ __noinline__ bool construct_exact(const double3* pts, const SymPt& s, double3& out)
{
    using namespace ex;
    int idx[5] = {s.p, s.q, s.r, s.a, s.b};
    int np = (s.kind == PK_PLANE) ? 5 : 5;
    if (s.kind == PK_LINE2) idx[2] = s.p;
    Grid g = grid_begin();
    for (int i = 0; i < np; i++)
        for (int k = 0; k < 3; k++) grid_add(g, dbits(cp(pts, idx[i])[k]));
    grid_finish(g);
    Big P[3], Q[3], R[3], A[3], B[3];
    bool ok = true;
    for (int k = 0; k < 3; k++) {
        ok &= big_from_bits(dbits(cp(pts, s.p)[k]), g.E, P[k]);
        ok &= big_from_bits(dbits(cp(pts, s.q)[k]), g.E, Q[k]);
        ok &= big_from_bits(dbits(cp(pts, idx[2])[k]), g.E, R[k]);
        ok &= big_from_bits(dbits(cp(pts, s.a)[k]), g.E, A[k]);
        ok &= big_from_bits(dbits(cp(pts, s.b)[k]), g.E, B[k]);
    }
    Big sa, sb, D, t1, t2;
    if (s.kind == PK_PLANE) {
        ok &= big_o3_value(P, Q, R, A, sa);
        ok &= big_o3_value(P, Q, R, B, sb);
    } else {
        ok &= big_o2_value(P, Q, A, s.drop, sa);
        ok &= big_o2_value(P, Q, B, s.drop, sb);
    }
    ok &= big_addsub(sa, sb, -1, D);
    if (!ok || D.n == 0) return false;
    double* o = &out.x;
    for (int k = 0; k < 3; k++) {
        ok &= big_mul(sa, B[k], t1);
        ok &= big_mul(sb, A[k], t2);
        ok &= big_addsub(t1, t2, -1, t1);
        if (!ok) return false;
        o[k] = round_quot(t1, D, g.E, &ok);
    }
    return ok;
}

// Fast path of a constructed point from its two side values sa, sb (with error
// bounds Ea, Eb): true when every coordinate passed the rounding test.
__device__ __forceinline__ bool construct_fast(const double3& a, const double3& b, dd sa, dd sb, double Ea, double Eb,
                                               double3& out)
{
    const double u2 = 0x1p-106;
    dd D = dd_add(sa, dd_neg(sb));
    double aD = fabs(D.hi);
    bool fast = aD > 8.0 * (Ea + Eb) && aD > 0x1p-900;
    double res[3];
    if (fast) {
        dd t = dd_div(sa, D);
        double err_t = 2.0 * (Ea + Eb) / aD * 1.01 + 32.0 * u2;
        const double* A = &a.x;
        const double* B = &b.x;
        for (int k = 0; k < 3 && fast; k++) {
            dd df = two_diff_dd(B[k], A[k]);
            dd pr = dd_mul(t, df);
            dd X = dd_add({A[k], 0.0}, pr);
            double ad = fabs(df.hi);
            double err = err_t * ad * 1.01 + 16.0 * u2 * (fabs(A[k]) + ad + fabs(X.hi));
            if (B[k] == A[k]) {
                res[k] = A[k];
                continue;
            }
            fast = ziv_round(X, err, &res[k]);
        }
    }
    if (fast) out = make_double3(res[0], res[1], res[2]);
    return fast;
}

// The crossing of edge (a, b) with plane(p, q, r), fast path only, on values in
// registers (inlined): false when the rounding test failed (construct_point
// then decides exactly).
__device__ __forceinline__ bool construct_plane_fast(const double3& p, const double3& q, const double3& r,
                                                     const double3& a, const double3& b, double3& out)
{
    const double u2 = 0x1p-106;
    double pa, pb;
    const dd sa = o3_dd_f(p, q, r, a, &pa);
    const dd sb = o3_dd_f(p, q, r, b, &pb);
    return construct_fast(a, b, sa, sb, 64.0 * u2 * pa, 64.0 * u2 * pb, out);
}

// returns false only on exact-arithmetic capacity failure
static __device__ __noinline__ bool construct_point(const double3* pts, const SymPt& s, double3& out, unsigned long long* nexact)
{
    if (s.kind == PK_VERTEX) {
        out = pts[s.a];
        return true;
    }
    const double3& a = pts[s.a];
    const double3& b = pts[s.b];
    double pa, pb;
    dd sa, sb;
    const double u2 = 0x1p-106;
    double Ea, Eb;
    if (s.kind == PK_PLANE) {
        sa = o3_dd(pts[s.p], pts[s.q], pts[s.r], a, &pa);
        sb = o3_dd(pts[s.p], pts[s.q], pts[s.r], b, &pb);
        Ea = 64.0 * u2 * pa;
        Eb = 64.0 * u2 * pb;
    } else {
        sa = o2_dd(pts[s.p], pts[s.q], a, s.drop, &pa);
        sb = o2_dd(pts[s.p], pts[s.q], b, s.drop, &pb);
        Ea = 32.0 * u2 * pa;
        Eb = 32.0 * u2 * pb;
    }
    if (construct_fast(a, b, sa, sb, Ea, Eb, out)) return true;
    atomicAdd(nexact, 1ull);
    return construct_exact(pts, s, out);
}

// Symbolic result of a pair from its endpoint pattern (make_pattern): the same
// points, in the same order, as classify_exact gives for it.
__device__ __forceinline__ void pattern_result(unsigned pat, TTRes& r)
{
    const int o1 = (pat >> 1) & 3, o2 = (pat >> 3) & 3;
    const unsigned xin = (pat >> 5) & 3, yin = (pat >> 7) & 3;
    r.n = 0;
    int k = 0;
    for (int i = 0; i < 3; i++) {
        if (i == o1) continue;
        if ((xin >> k) & 1u) r.pt[r.n++] = sp_plane(o1, i, 3, 4, 5);
        k++;
    }
    k = 0;
    for (int j = 0; j < 3; j++) {
        if (j == o2) continue;
        if ((yin >> k) & 1u) r.pt[r.n++] = sp_plane(3 + o2, 3 + j, 0, 1, 2);
        k++;
    }
    r.kind = r.n == 1 ? KIND_POINT : KIND_SEGMENT;
}

}  // namespace gi
