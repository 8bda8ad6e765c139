// gi_exact.cuh -- exact arithmetic on the device.
//
// Every finite double is m * 2^e with integer m.  For one predicate call the
// coordinates involved are put on a common grid 2^E (E = the lowest set-bit
// exponent among them), so coordinate differences, determinants and the
// numerators/denominators of constructed points are exact integers.
//   * int128 fast path when every scaled coordinate fits in 40 bits (integer
//     grids such as the coplanar 2^20 stress case);
//   * multi-limb integers (64-bit limbs) otherwise.
// Constructed points X = a + t (b - a), t = sa / (sa - sb), are rounded to
// nearest-even from the exact rational N / D by long division.
//
// The signs computed here are the mathematically exact orient3d / orient2d
// signs, the same quantities the reference's CGAL::do_intersect decides on
// (src/CPU/YellowFilter.h:80-137 in the reference project).
#pragma once
#include <cstdint>
#include <cuda_runtime.h>

namespace gi {
namespace ex {

constexpr int kLMax = 24;  // 1536-bit magnitudes; the supported domain (|x| in [2^-100, 2^100]) needs < 1200

struct Big {
    uint64_t w[kLMax];
    int n;    // used limbs; 0 means zero
    int neg;  // sign of a nonzero value
};

__device__ __forceinline__ void big_zero(Big& a)
{
    a.n = 0;
    a.neg = 0;
}
__device__ __forceinline__ void big_trim(Big& a)
{
    while (a.n > 0 && a.w[a.n - 1] == 0) a.n--;
    if (a.n == 0) a.neg = 0;
}
__device__ __forceinline__ int big_sign(const Big& a)
{
    return a.n == 0 ? 0 : (a.neg ? -1 : 1);
}
__device__ __forceinline__ void big_copy(const Big& a, Big& r)
{
    r.n = a.n;
    r.neg = a.neg;
    for (int i = 0; i < a.n; i++) r.w[i] = a.w[i];
}
__device__ __forceinline__ int mag_cmp(const Big& a, const Big& b)
{
    if (a.n != b.n) return a.n < b.n ? -1 : 1;
    for (int i = a.n - 1; i >= 0; --i)
        if (a.w[i] != b.w[i]) return a.w[i] < b.w[i] ? -1 : 1;
    return 0;
}
// |r| = |a| + |b| (r may alias a or b); false on capacity overflow
__device__ __forceinline__ bool mag_add(const Big& a, const Big& b, Big& r)
{
    int n = a.n > b.n ? a.n : b.n;
    uint64_t carry = 0;
    for (int i = 0; i < n; i++) {
        uint64_t x = i < a.n ? a.w[i] : 0ull;
        uint64_t y = i < b.n ? b.w[i] : 0ull;
        uint64_t s = x + y;
        uint64_t c1 = s < x;
        uint64_t s2 = s + carry;
        uint64_t c2 = s2 < s;
        r.w[i] = s2;
        carry = c1 | c2;
    }
    if (carry) {
        if (n >= kLMax) return false;
        r.w[n++] = carry;
    }
    r.n = n;
    return true;
}
// |r| = |a| - |b|, requires |a| >= |b| (r may alias a or b)
__device__ __forceinline__ void mag_sub(const Big& a, const Big& b, Big& r)
{
    uint64_t borrow = 0;
    int n = a.n;
    for (int i = 0; i < n; i++) {
        uint64_t x = a.w[i];
        uint64_t y = i < b.n ? b.w[i] : 0ull;
        uint64_t d = x - y;
        uint64_t b1 = x < y;
        uint64_t d2 = d - borrow;
        uint64_t b2 = d < borrow;
        r.w[i] = d2;
        borrow = b1 | b2;
    }
    r.n = n;
    big_trim(r);
}
// r = a + sb * b  (sb = +1 or -1); r may alias a or b
__device__ __forceinline__ bool big_addsub(const Big& a, const Big& b, int sb, Big& r)
{
    int an = a.neg;
    int bn = (b.n == 0) ? 0 : (sb > 0 ? b.neg : !b.neg);
    if (b.n == 0) {
        if (&r != &a) big_copy(a, r);
        return true;
    }
    if (a.n == 0) {
        if (&r != &b) big_copy(b, r);
        r.neg = bn;
        return true;
    }
    if (an == bn) {
        if (!mag_add(a, b, r)) return false;
        r.neg = an;
        return true;
    }
    int c = mag_cmp(a, b);
    if (c >= 0) {
        mag_sub(a, b, r);
        if (r.n) r.neg = an;
    } else {
        mag_sub(b, a, r);
        if (r.n) r.neg = bn;
    }
    return true;
}
// r = a * b (r must not alias a or b)
__device__ __forceinline__ bool big_mul(const Big& a, const Big& b, Big& r)
{
    if (a.n == 0 || b.n == 0) {
        big_zero(r);
        return true;
    }
    int n = a.n + b.n;
    if (n > kLMax) return false;
    for (int i = 0; i < n; i++) r.w[i] = 0;
    for (int i = 0; i < a.n; i++) {
        unsigned __int128 carry = 0;
        uint64_t ai = a.w[i];
        for (int j = 0; j < b.n; j++) {
            unsigned __int128 t = (unsigned __int128)ai * b.w[j] + r.w[i + j] + carry;
            r.w[i + j] = (uint64_t)t;
            carry = t >> 64;
        }
        r.w[i + b.n] = (uint64_t)carry;
    }
    r.n = n;
    r.neg = a.neg ^ b.neg;
    big_trim(r);
    return true;
}
__device__ __forceinline__ int big_bitlen(const Big& a)
{
    if (a.n == 0) return 0;
    return 64 * (a.n - 1) + (64 - __clzll((long long)a.w[a.n - 1]));
}
// r = |a| << s (magnitude only); r may alias a
__device__ __forceinline__ bool mag_shl(const Big& a, int s, Big& r)
{
    if (a.n == 0) {
        big_zero(r);
        return true;
    }
    int ls = s >> 6, bs = s & 63;
    int n = a.n + ls + 1;
    if (n > kLMax) {
        // the top limb may be unnecessary
        if (n - 1 > kLMax) return false;
    }
    uint64_t top = bs ? (a.w[a.n - 1] >> (64 - bs)) : 0ull;
    if (top && n > kLMax) return false;
    for (int i = a.n - 1; i >= 0; --i) {
        uint64_t v = a.w[i] << bs;
        if (bs && i > 0) v |= a.w[i - 1] >> (64 - bs);
        r.w[i + ls] = v;
    }
    for (int i = 0; i < ls; i++) r.w[i] = 0;
    r.n = a.n + ls;
    if (top) r.w[r.n++] = top;
    r.neg = 0;
    big_trim(r);
    return true;
}

// ---- doubles on a common grid ---------------------------------------------
struct DBits {
    uint64_t mant;  // odd (or 0)
    int elow;       // exponent of the lowest set bit
    int ehigh;      // exponent of the highest set bit + 1
    int neg;
};
__device__ __forceinline__ DBits dbits(double x)
{
    DBits r;
    uint64_t b = (uint64_t)__double_as_longlong(x);
    r.neg = (int)(b >> 63);
    int ex = (int)((b >> 52) & 0x7FF);
    uint64_t m = b & ((1ull << 52) - 1);
    int e;
    if (ex == 0) {
        e = -1074;
    } else {
        m |= (1ull << 52);
        e = ex - 1075;
    }
    if (m == 0) {
        r.mant = 0;
        r.elow = 1 << 20;
        r.ehigh = -(1 << 20);
        return r;
    }
    int tz = __ffsll((long long)m) - 1;
    m >>= tz;
    r.mant = m;
    r.elow = e + tz;
    r.ehigh = r.elow + (64 - __clzll((long long)m));
    return r;
}
__device__ __forceinline__ bool big_from_bits(const DBits& d, int E, Big& r)
{
    if (d.mant == 0) {
        big_zero(r);
        return true;
    }
    r.w[0] = d.mant;
    r.n = 1;
    r.neg = 0;
    if (!mag_shl(r, d.elow - E, r)) return false;
    r.neg = d.neg;
    return true;
}

struct Grid {
    int E;     // common exponent
    int span;  // bits of the largest scaled magnitude
};
__device__ __forceinline__ void grid_add(Grid& g, const DBits& d)
{
    if (d.mant == 0) return;
    if (d.elow < g.E) g.E = d.elow;
    if (d.ehigh > g.span) g.span = d.ehigh;  // holds ehigh max until finish
}
__device__ __forceinline__ Grid grid_begin()
{
    Grid g;
    g.E = 1 << 20;
    g.span = -(1 << 20);
    return g;
}
__device__ __forceinline__ void grid_finish(Grid& g)
{
    if (g.E == (1 << 20)) {  // all zero
        g.E = 0;
        g.span = 0;
        return;
    }
    g.span = g.span - g.E;
}

// ---- exact orient3d / orient2d signs ----------------------------------------
// int128 path: scaled coordinates < 2^40, differences < 2^41, triple products < 2^123.
__device__ __forceinline__ long long scaled_i64(const DBits& d, int E)
{
    if (d.mant == 0) return 0;
    long long v = (long long)(d.mant << (d.elow - E));
    return d.neg ? -v : v;
}

// Integer branch that decided an exact sign (reported through `path`).
constexpr int kPathInt128 = 0, kPathMultiLimb = 1, kPathCapacity = 2;

// det[a-d; b-d; c-d] exact sign. err |= kErrExactCapacity if outside capacity.
// path (optional): the branch that ran, kPathInt128 or kPathMultiLimb (kPathCapacity on failure).
static __device__ __noinline__ int o3_exact_sign(const double* a, const double* b, const double* c, const double* d,
                                                 unsigned* err, int* path = nullptr)
{
    DBits bits[12];
    const double* P[4] = {a, b, c, d};
    Grid g = grid_begin();
    for (int i = 0; i < 4; i++)
        for (int k = 0; k < 3; k++) {
            bits[3 * i + k] = dbits(P[i][k]);
            grid_add(g, bits[3 * i + k]);
        }
    grid_finish(g);
    if (g.span <= 40) {
        if (path) *path = kPathInt128;
        long long v[12];
        for (int i = 0; i < 12; i++) v[i] = scaled_i64(bits[i], g.E);
        __int128 adx = v[0] - v[9], ady = v[1] - v[10], adz = v[2] - v[11];
        __int128 bdx = v[3] - v[9], bdy = v[4] - v[10], bdz = v[5] - v[11];
        __int128 cdx = v[6] - v[9], cdy = v[7] - v[10], cdz = v[8] - v[11];
        __int128 det = adz * (bdx * cdy - cdx * bdy) + bdz * (cdx * ady - adx * cdy) + cdz * (adx * bdy - bdx * ady);
        return (det > 0) - (det < 0);
    }
    if (path) *path = kPathMultiLimb;
    Big V[12];
    for (int i = 0; i < 12; i++)
        if (!big_from_bits(bits[i], g.E, V[i])) {
            if (path) *path = kPathCapacity;
            atomicOr(err, 2u);
            return 0;
        }
    // differences in place: V[0..8] -= V[9..11]
    bool ok = true;
    for (int i = 0; i < 3; i++)
        for (int k = 0; k < 3; k++) ok &= big_addsub(V[3 * i + k], V[9 + k], -1, V[3 * i + k]);
    Big t1, t2, acc;
    big_zero(acc);
    // adz*(bdx*cdy - cdx*bdy) + bdz*(cdx*ady - adx*cdy) + cdz*(adx*bdy - bdx*ady)
    const int X = 0, Y = 1, Z = 2;
    const int A = 0, Bq = 3, Cq = 6;
    int tri[3][5] = {{A, Bq, Cq, Cq, Bq}, {Bq, Cq, A, A, Cq}, {Cq, A, Bq, Bq, A}};
    for (int t = 0; t < 3; t++) {
        int z = tri[t][0];
        // m = V[p].x * V[q].y - V[r].x * V[s].y
        ok &= big_mul(V[tri[t][1] + X], V[tri[t][2] + Y], t1);
        ok &= big_mul(V[tri[t][3] + X], V[tri[t][4] + Y], t2);
        ok &= big_addsub(t1, t2, -1, t1);
        ok &= big_mul(t1, V[z + Z], t2);
        ok &= big_addsub(acc, t2, +1, acc);
    }
    if (!ok) {
        if (path) *path = kPathCapacity;
        atomicOr(err, 2u);
        return 0;
    }
    return big_sign(acc);
}

static __device__ __noinline__ int o2_exact_sign(const double* a, const double* b, const double* c, int drop,
                                                 unsigned* err, int* path = nullptr)
{
    int u = (drop + 1) % 3, v = (drop + 2) % 3;
    double q[6] = {a[u], a[v], b[u], b[v], c[u], c[v]};
    DBits bits[6];
    Grid g = grid_begin();
    for (int i = 0; i < 6; i++) {
        bits[i] = dbits(q[i]);
        grid_add(g, bits[i]);
    }
    grid_finish(g);
    if (g.span <= 60) {
        if (path) *path = kPathInt128;
        __int128 s[6];
        for (int i = 0; i < 6; i++) {
            if (bits[i].mant == 0) {
                s[i] = 0;
                continue;
            }
            __int128 m = (__int128)bits[i].mant << (bits[i].elow - g.E);
            s[i] = bits[i].neg ? -m : m;
        }
        __int128 acu = s[0] - s[4], acv = s[1] - s[5], bcu = s[2] - s[4], bcv = s[3] - s[5];
        __int128 det = acu * bcv - acv * bcu;
        return (det > 0) - (det < 0);
    }
    if (path) *path = kPathMultiLimb;
    Big V[6];
    for (int i = 0; i < 6; i++)
        if (!big_from_bits(bits[i], g.E, V[i])) {
            if (path) *path = kPathCapacity;
            atomicOr(err, 2u);
            return 0;
        }
    bool ok = true;
    ok &= big_addsub(V[0], V[4], -1, V[0]);
    ok &= big_addsub(V[1], V[5], -1, V[1]);
    ok &= big_addsub(V[2], V[4], -1, V[2]);
    ok &= big_addsub(V[3], V[5], -1, V[3]);
    Big t1, t2;
    ok &= big_mul(V[0], V[3], t1);
    ok &= big_mul(V[1], V[2], t2);
    ok &= big_addsub(t1, t2, -1, t1);
    if (!ok) {
        if (path) *path = kPathCapacity;
        atomicOr(err, 2u);
        return 0;
    }
    return big_sign(t1);
}

// ---- exact construction ------------------------------------------------------
// Exact side values on a grid: for PLANE points sa = det[p-a; q-a; r-a] (scale 2^3E);
// for LINE2 points sa = orient2d(p, q, a) (scale 2^2E).
static __device__ __noinline__ bool big_o3_value(const Big* P, const Big* Q, const Big* R, const Big* X, Big& out)
{
    // det[P-X; Q-X; R-X]
    Big d[9];
    bool ok = true;
    for (int k = 0; k < 3; k++) {
        ok &= big_addsub(P[k], X[k], -1, d[k]);
        ok &= big_addsub(Q[k], X[k], -1, d[3 + k]);
        ok &= big_addsub(R[k], X[k], -1, d[6 + k]);
    }
    Big t1, t2;
    big_zero(out);
    const int A = 0, Bq = 3, Cq = 6;
    int tri[3][5] = {{A, Bq, Cq, Cq, Bq}, {Bq, Cq, A, A, Cq}, {Cq, A, Bq, Bq, A}};
    for (int t = 0; t < 3; t++) {
        ok &= big_mul(d[tri[t][1] + 0], d[tri[t][2] + 1], t1);
        ok &= big_mul(d[tri[t][3] + 0], d[tri[t][4] + 1], t2);
        ok &= big_addsub(t1, t2, -1, t1);
        ok &= big_mul(t1, d[tri[t][0] + 2], t2);
        ok &= big_addsub(out, t2, +1, out);
    }
    return ok;
}
static __device__ __noinline__ bool big_o2_value(const Big* P, const Big* Q, const Big* X, int drop, Big& out)
{
    int u = (drop + 1) % 3, v = (drop + 2) % 3;
    Big acu, acv, bcu, bcv, t1, t2;
    bool ok = true;
    ok &= big_addsub(P[u], X[u], -1, acu);
    ok &= big_addsub(P[v], X[v], -1, acv);
    ok &= big_addsub(Q[u], X[u], -1, bcu);
    ok &= big_addsub(Q[v], X[v], -1, bcv);
    ok &= big_mul(acu, bcv, t1);
    ok &= big_mul(acv, bcu, t2);
    ok &= big_addsub(t1, t2, -1, out);
    return ok;
}

// Round (N / D) * 2^E to the nearest double (ties to even). D != 0.
static __device__ __noinline__ double round_quot(const Big& N, const Big& D, int E, bool* ok)
{
    if (N.n == 0) return 0.0;
    int neg = N.neg ^ D.neg;
    Big n, d, t;
    big_copy(N, n);
    n.neg = 0;
    big_copy(D, d);
    d.neg = 0;
    int ln = big_bitlen(n), ld = big_bitlen(d);
    // scale so that the quotient has 56 or 57 bits: q = floor(n * 2^s / d)
    int s = 56 - (ln - ld);
    if (s > 0) {
        if (!mag_shl(n, s, n)) {
            *ok = false;
            return 0.0;
        }
    } else if (s < 0) {
        if (!mag_shl(d, -s, d)) {
            *ok = false;
            return 0.0;
        }
    }
    // long division, quotient < 2^58
    uint64_t q = 0;
    for (int bit = 57; bit >= 0; --bit) {
        if (!mag_shl(d, bit, t)) continue;  // t larger than capacity means t > n
        if (mag_cmp(n, t) >= 0) {
            mag_sub(n, t, n);
            q |= (1ull << bit);
        }
    }
    int sticky = n.n != 0;
    int qb = 64 - __clzll((long long)q);
    int k = qb - 53;  // extra bits beyond the 53-bit significand
    uint64_t mant = q >> k;
    uint64_t rem = q & ((1ull << k) - 1);
    uint64_t half = 1ull << (k - 1);
    if (rem > half || (rem == half && (sticky || (mant & 1ull)))) {
        mant++;
        if (mant == (1ull << 53)) {
            mant >>= 1;
            k++;
        }
    }
    double r = ldexp((double)mant, E - s + k);
    return neg ? -r : r;
}

}  // namespace ex
}  // namespace gi
