/*
 * gi_oracle.c -- CPU exact oracle (TEST INFRASTRUCTURE, see gi_oracle.h).
 *
 * Only tests/, __graft_entry__.smoke() and bench.py's CPU-baseline leg load
 * this library, as the checker.  Build: oracle/Makefile (-O2 -ffp-contract=off).
 *
 * Reference behaviour restated here (paths inside the reference project):
 *   src/CPU/RotationTools.h:28-53     Euler -> R = Rz*Ry*Rx            (oc_pose_from_euler_deg)
 *   src/CPU/RotationTools.h:129-145   x=v-c; r=R*x; out=(r+c)+t         (oc_transform_vertices)
 *   src/CPU/YellowFilter.h:80-137     exact do_intersect on pairs       (oc_tri_tri_intersect)
 *   src/CPU/MeshIntersectionCurves.cpp:63-78  segment / point / triangle output rule
 *   src/CPU/TestSuite.cpp:79-102      face-face ground truth over box-overlapping pairs
 *   src/CPU/TestSuite.cpp:24-32       canonical (a,b) pair sets          (sorted output)
 */
#define _GNU_SOURCE
#include "gi_oracle.h"

#include <math.h>
#include <pthread.h>
#include <stdatomic.h>
#include <stdlib.h>
#include <string.h>
#include <time.h>
#include <unistd.h>

/* ------------------------------------------------------------------------- */
/* Error-free transformations (Knuth two-sum, Dekker fast-two-sum, fma product) */
/* ------------------------------------------------------------------------- */
static inline void fast_two_sum(double a, double b, double* x, double* y)
{
    double s = a + b;
    double bv = s - a;
    *x = s;
    *y = b - bv;
}
static inline void two_sum(double a, double b, double* x, double* y)
{
    double s = a + b;
    double bv = s - a;
    double av = s - bv;
    double br = b - bv;
    double ar = a - av;
    *x = s;
    *y = ar + br;
}
static inline void two_diff(double a, double b, double* x, double* y)
{
    double s = a - b;
    double bv = a - s;
    double av = s + bv;
    double br = bv - b;
    double ar = a - av;
    *x = s;
    *y = ar + br;
}
static inline void two_prod(double a, double b, double* x, double* y)
{
    double p = a * b;
    *x = p;
    *y = fma(a, b, -p);
}

/* ------------------------------------------------------------------------- */
/* Expansions: nonoverlapping components, increasing magnitude, zero-free    */
/* (a single 0.0 component represents zero).                                  */
/* ------------------------------------------------------------------------- */
static __thread uint64_t tl_exact_calls;

/* Per-thread scratch for the construction paths (heap, freed at thread exit;
 * large __thread arrays would not fit the static TLS of a dlopen'ed library). */
#define CR_MAX 6200
#define SCRATCH_DOUBLES (8 * CR_MAX)
static pthread_key_t g_scratch_key;
static pthread_once_t g_scratch_once = PTHREAD_ONCE_INIT;
static void scratch_key_init(void) { pthread_key_create(&g_scratch_key, free); }
static double* scratch(void)
{
    pthread_once(&g_scratch_once, scratch_key_init);
    double* p = (double*)pthread_getspecific(g_scratch_key);
    if (!p) {
        p = (double*)malloc(sizeof(double) * SCRATCH_DOUBLES);
        pthread_setspecific(g_scratch_key, p);
    }
    return p;
}

/* h = e + b.  h may alias e; h needs room for elen + 1 entries. */
static int exp_grow(int elen, const double* e, double b, double* h)
{
    double q = b, qn, hh;
    int k = 0;
    for (int i = 0; i < elen; i++) {
        double ei = e[i];
        two_sum(q, ei, &qn, &hh);
        q = qn;
        if (hh != 0.0) h[k++] = hh;
    }
    if (q != 0.0 || k == 0) h[k++] = q;
    return k;
}

/* h = e + f (repeated growth; O(elen * flen), exact). h must not alias f. */
static int exp_add(int elen, const double* e, int flen, const double* f, double* h)
{
    if (h != e) memcpy(h, e, sizeof(double) * (size_t)elen);
    int hl = elen;
    for (int j = 0; j < flen; j++) {
        if (f[j] == 0.0) continue;
        hl = exp_grow(hl, h, f[j], h);
    }
    return hl;
}

/* h = e * b.  h needs 2*elen entries. */
static int exp_scale(int elen, const double* e, double b, double* h)
{
    if (b == 0.0) { h[0] = 0.0; return 1; }
    double q, hh, p1, p0, s;
    int k = 0;
    two_prod(e[0], b, &q, &hh);
    if (hh != 0.0) h[k++] = hh;
    for (int i = 1; i < elen; i++) {
        two_prod(e[i], b, &p1, &p0);
        two_sum(q, p0, &s, &hh);
        if (hh != 0.0) h[k++] = hh;
        fast_two_sum(p1, s, &q, &hh);
        if (hh != 0.0) h[k++] = hh;
    }
    if (q != 0.0 || k == 0) h[k++] = q;
    return k;
}

/* h = e * f.  h needs 2*elen*flen entries; tmp the same. */
static int exp_mul(int elen, const double* e, int flen, const double* f, double* h, double* tmp)
{
    int hl = 1;
    h[0] = 0.0;
    for (int j = 0; j < flen; j++) {
        if (f[j] == 0.0) continue;
        int tl = exp_scale(elen, e, f[j], tmp);
        hl = exp_add(hl, h, tl, tmp, h);
    }
    return hl;
}

static void exp_neg(int n, double* e)
{
    for (int i = 0; i < n; i++) e[i] = -e[i];
}
static int exp_sign(int n, const double* e)
{
    double t = e[n - 1];
    return (t > 0.0) - (t < 0.0);
}
static double exp_est(int n, const double* e)
{
    double s = 0.0;
    for (int i = 0; i < n; i++) s += e[i];
    return s;
}
static int exp_diff2(double a, double b, double* out)
{
    double x, y;
    two_diff(a, b, &x, &y);
    if (x == 0.0) { out[0] = 0.0; return 1; }
    if (y == 0.0) { out[0] = x; return 1; }
    out[0] = y;
    out[1] = x;
    return 2;
}

/* ------------------------------------------------------------------------- */
/* orient3d / orient2d: FP64 semi-static filter, then exact expansions       */
/* ------------------------------------------------------------------------- */
#define EPS64 (0x1p-53)
static const double O3_ERRB = (7.0 + 56.0 * EPS64) * EPS64; /* Shewchuk's orient3d bound A */
static const double O2_ERRB = (3.0 + 16.0 * EPS64) * EPS64; /* Shewchuk's orient2d bound A */

#define O3_MAXLEN 200
/* exact value of det[a-d; b-d; c-d] as an expansion; returns its length. */
static int o3_exact(const double* a, const double* b, const double* c, const double* d, double* out)
{
    double adx[2], ady[2], adz[2], bdx[2], bdy[2], bdz[2], cdx[2], cdy[2], cdz[2];
    int nadx = exp_diff2(a[0], d[0], adx), nady = exp_diff2(a[1], d[1], ady), nadz = exp_diff2(a[2], d[2], adz);
    int nbdx = exp_diff2(b[0], d[0], bdx), nbdy = exp_diff2(b[1], d[1], bdy), nbdz = exp_diff2(b[2], d[2], bdz);
    int ncdx = exp_diff2(c[0], d[0], cdx), ncdy = exp_diff2(c[1], d[1], cdy), ncdz = exp_diff2(c[2], d[2], cdz);
    double t1[8], t2[8], tmp[8], m[16], term[64], tmp2[64], acc1[64], acc2[128];
    int n1, n2, nm, nt, na;
    /* adz * (bdx*cdy - cdx*bdy) */
    n1 = exp_mul(nbdx, bdx, ncdy, cdy, t1, tmp);
    n2 = exp_mul(ncdx, cdx, nbdy, bdy, t2, tmp);
    exp_neg(n2, t2);
    nm = exp_add(n1, t1, n2, t2, m);
    nt = exp_mul(nm, m, nadz, adz, term, tmp2);
    memcpy(acc1, term, sizeof(double) * (size_t)nt);
    na = nt;
    /* bdz * (cdx*ady - adx*cdy) */
    n1 = exp_mul(ncdx, cdx, nady, ady, t1, tmp);
    n2 = exp_mul(nadx, adx, ncdy, cdy, t2, tmp);
    exp_neg(n2, t2);
    nm = exp_add(n1, t1, n2, t2, m);
    nt = exp_mul(nm, m, nbdz, bdz, term, tmp2);
    na = exp_add(na, acc1, nt, term, acc2);
    /* cdz * (adx*bdy - bdx*ady) */
    n1 = exp_mul(nadx, adx, nbdy, bdy, t1, tmp);
    n2 = exp_mul(nbdx, bdx, nady, ady, t2, tmp);
    exp_neg(n2, t2);
    nm = exp_add(n1, t1, n2, t2, m);
    nt = exp_mul(nm, m, ncdz, cdz, term, tmp2);
    na = exp_add(na, acc2, nt, term, out);
    return na;
}

static int orient3d_sign(const double* a, const double* b, const double* c, const double* d)
{
    double adx = a[0] - d[0], ady = a[1] - d[1], adz = a[2] - d[2];
    double bdx = b[0] - d[0], bdy = b[1] - d[1], bdz = b[2] - d[2];
    double cdx = c[0] - d[0], cdy = c[1] - d[1], cdz = c[2] - d[2];
    double bdxcdy = bdx * cdy, cdxbdy = cdx * bdy;
    double cdxady = cdx * ady, adxcdy = adx * cdy;
    double adxbdy = adx * bdy, bdxady = bdx * ady;
    double det = adz * (bdxcdy - cdxbdy) + bdz * (cdxady - adxcdy) + cdz * (adxbdy - bdxady);
    double perm = (fabs(bdxcdy) + fabs(cdxbdy)) * fabs(adz) + (fabs(cdxady) + fabs(adxcdy)) * fabs(bdz) +
                  (fabs(adxbdy) + fabs(bdxady)) * fabs(cdz);
    double eb = O3_ERRB * perm;
    if (det > eb) return 1;
    if (-det > eb) return -1;
    tl_exact_calls++;
    double e[O3_MAXLEN];
    int n = o3_exact(a, b, c, d, e);
    return exp_sign(n, e);
}

static inline void proj_axes(int drop, int* u, int* v)
{
    *u = (drop + 1) % 3;
    *v = (drop + 2) % 3;
}

/* exact (a_u-c_u)(b_v-c_v) - (a_v-c_v)(b_u-c_u) */
static int o2_exact(const double* a, const double* b, const double* c, int drop, double* out)
{
    int u, v;
    proj_axes(drop, &u, &v);
    double acu[2], acv[2], bcu[2], bcv[2];
    int n_acu = exp_diff2(a[u], c[u], acu), n_acv = exp_diff2(a[v], c[v], acv);
    int n_bcu = exp_diff2(b[u], c[u], bcu), n_bcv = exp_diff2(b[v], c[v], bcv);
    double t1[8], t2[8], tmp[8];
    int n1 = exp_mul(n_acu, acu, n_bcv, bcv, t1, tmp);
    int n2 = exp_mul(n_acv, acv, n_bcu, bcu, t2, tmp);
    exp_neg(n2, t2);
    return exp_add(n1, t1, n2, t2, out);
}

static int orient2d_sign(const double* a, const double* b, const double* c, int drop)
{
    int u, v;
    proj_axes(drop, &u, &v);
    double l = (a[u] - c[u]) * (b[v] - c[v]);
    double r = (a[v] - c[v]) * (b[u] - c[u]);
    double det = l - r;
    double eb = O2_ERRB * (fabs(l) + fabs(r));
    if (det > eb) return 1;
    if (-det > eb) return -1;
    tl_exact_calls++;
    double e[20];
    int n = o2_exact(a, b, c, drop, e);
    return exp_sign(n, e);
}

/* ------------------------------------------------------------------------- */
/* Sign log (test hook): while enabled, every orient3d / orient2d call of the  */
/* decision procedure is recorded with its inputs and exact sign, so that a    */
/* test can replay the same calls through the device's predicates.            */
/* ------------------------------------------------------------------------- */
static pthread_mutex_t g_log_mu = PTHREAD_MUTEX_INITIALIZER;
static volatile int g_log_on;
static double* g_log_pts;   /* 12 doubles per entry (orient2d: 9 used) */
static int32_t* g_log_meta; /* kind (0 orient3d, 1 orient2d), drop, sign per entry */
static uint64_t g_log_n, g_log_cap;

static void sign_log(int kind, const double* a, const double* b, const double* c, const double* d, int drop, int sgn)
{
    pthread_mutex_lock(&g_log_mu);
    if (g_log_on && g_log_n < g_log_cap) {
        double* p = g_log_pts + 12 * g_log_n;
        memset(p, 0, 12 * sizeof(double));
        memcpy(p, a, 3 * sizeof(double));
        memcpy(p + 3, b, 3 * sizeof(double));
        memcpy(p + 6, c, 3 * sizeof(double));
        if (d) memcpy(p + 9, d, 3 * sizeof(double));
        int32_t* m = g_log_meta + 3 * g_log_n;
        m[0] = kind;
        m[1] = drop;
        m[2] = sgn;
        g_log_n++;
    }
    pthread_mutex_unlock(&g_log_mu);
}

int oc_sign_log_begin(uint64_t cap)
{
    pthread_mutex_lock(&g_log_mu);
    free(g_log_pts);
    free(g_log_meta);
    g_log_pts = (double*)malloc(sizeof(double) * 12 * (cap ? cap : 1));
    g_log_meta = (int32_t*)malloc(sizeof(int32_t) * 3 * (cap ? cap : 1));
    g_log_n = 0;
    g_log_cap = (g_log_pts && g_log_meta) ? cap : 0;
    g_log_on = g_log_cap != 0;
    int ok = g_log_on ? 0 : -1;
    pthread_mutex_unlock(&g_log_mu);
    return ok;
}

uint64_t oc_sign_log_end(double** pts, int32_t** meta)
{
    pthread_mutex_lock(&g_log_mu);
    g_log_on = 0;
    uint64_t n = g_log_n;
    *pts = g_log_pts;
    *meta = g_log_meta;
    g_log_pts = NULL;
    g_log_meta = NULL;
    g_log_n = g_log_cap = 0;
    pthread_mutex_unlock(&g_log_mu);
    return n;
}

int oc_orient3d(const double* a, const double* b, const double* c, const double* d)
{
    const int s = orient3d_sign(a, b, c, d);
    if (g_log_on) sign_log(0, a, b, c, d, -1, s);
    return s;
}

int oc_orient2d(const double* a, const double* b, const double* c, int drop)
{
    const int s = orient2d_sign(a, b, c, drop);
    if (g_log_on) sign_log(1, a, b, c, NULL, drop, s);
    return s;
}

/* ------------------------------------------------------------------------- */
/* Correctly rounded N / D (round to nearest, ties to even)                   */
/* ------------------------------------------------------------------------- */
/* sign(N - (q + h) * D); uses scratch region [4, 8) * CR_MAX */
static int sign_n_minus_qd(int nn, const double* N, int nd, const double* D, double q, double h)
{
    double* buf = scratch() + 4 * CR_MAX;
    double *t1 = buf, *t2 = buf + CR_MAX, *t3 = buf + 2 * CR_MAX, *t4 = buf + 3 * CR_MAX;
    int n1 = exp_scale(nd, D, q, t1);
    int n3 = n1;
    if (h != 0.0) {
        int n2 = exp_scale(nd, D, h, t2);
        n3 = exp_add(n1, t1, n2, t2, t3);
    } else {
        memcpy(t3, t1, sizeof(double) * (size_t)n1);
    }
    exp_neg(n3, t3);
    int n4 = exp_add(n3, t3, nn, N, t4);
    return exp_sign(n4, t4);
}

static int is_even_double(double q)
{
    uint64_t u;
    memcpy(&u, &q, sizeof u);
    return (u & 1u) == 0;
}

static double round_div(int nn, const double* N, int nd, const double* D)
{
    int sd = exp_sign(nd, D);
    if (exp_sign(nn, N) == 0) return 0.0;
    double q = exp_est(nn, N) / exp_est(nd, D);
    for (int it = 0; it < 256; it++) {
        int c = sign_n_minus_qd(nn, N, nd, D, q, 0.0) * sd; /* sign(N/D - q) */
        if (c == 0) return q;
        double qn = nextafter(q, c > 0 ? INFINITY : -INFINITY);
        double h = (qn - q) * 0.5;
        int cm = sign_n_minus_qd(nn, N, nd, D, q, h) * sd; /* sign(N/D - (q+h)) */
        if (cm == 0) return is_even_double(q) ? q : qn;
        if (cm == c) { q = qn; continue; }
        return q;
    }
    return q; /* unreachable for inputs inside the supported domain */
}

/* ------------------------------------------------------------------------- */
/* Symbolic points                                                            */
/* ------------------------------------------------------------------------- */
enum { PK_VERTEX = 0, PK_PLANE = 1, PK_LINE2 = 2 };
typedef struct {
    int kind;
    const double *a, *b;    /* vertex a, or the segment a->b that is cut */
    const double *p, *q, *r; /* cutting plane (p,q,r) or 2D line (p,q) */
    int drop;
} SymPt;

static SymPt sp_vertex(const double* a)
{
    SymPt s;
    memset(&s, 0, sizeof s);
    s.kind = PK_VERTEX;
    s.a = a;
    return s;
}
static SymPt sp_plane(const double* a, const double* b, const double* p, const double* q, const double* r)
{
    SymPt s;
    memset(&s, 0, sizeof s);
    s.kind = PK_PLANE;
    s.a = a; s.b = b; s.p = p; s.q = q; s.r = r;
    return s;
}
static SymPt sp_line2(const double* a, const double* b, const double* p, const double* q, int drop)
{
    SymPt s;
    memset(&s, 0, sizeof s);
    s.kind = PK_LINE2;
    s.a = a; s.b = b; s.p = p; s.q = q; s.drop = drop;
    return s;
}

/* X = (sa*b - sb*a) / (sa - sb), sa/sb the exact side values of a and b. */
static void sp_construct(const SymPt* s, double* out)
{
    if (s->kind == PK_VERTEX) {
        out[0] = s->a[0]; out[1] = s->a[1]; out[2] = s->a[2];
        return;
    }
    double sa[O3_MAXLEN], sb[O3_MAXLEN];
    int na, nb;
    if (s->kind == PK_PLANE) {
        na = o3_exact(s->p, s->q, s->r, s->a, sa);
        nb = o3_exact(s->p, s->q, s->r, s->b, sb);
    } else {
        na = o2_exact(s->p, s->q, s->a, s->drop, sa);
        nb = o2_exact(s->p, s->q, s->b, s->drop, sb);
    }
    double* buf = scratch(); /* region [0, 4) * CR_MAX */
    double *D = buf, *N = buf + CR_MAX, *t1 = buf + 2 * CR_MAX, *t2 = buf + 3 * CR_MAX;
    double nsb[O3_MAXLEN];
    memcpy(nsb, sb, sizeof(double) * (size_t)nb);
    exp_neg(nb, nsb);
    int nD = exp_add(na, sa, nb, nsb, D);
    for (int i = 0; i < 3; i++) {
        int n1 = exp_scale(na, sa, s->b[i], t1);
        int n2 = exp_scale(nb, nsb, s->a[i], t2); /* -sb * a_i */
        int nN = exp_add(n1, t1, n2, t2, N);
        out[i] = round_div(nN, N, nD, D);
    }
}

/* ------------------------------------------------------------------------- */
/* Triangle-triangle classification                                           */
/* ------------------------------------------------------------------------- */
typedef struct {
    int kind;  /* OC_* */
    int n;     /* number of symbolic points */
    SymPt pt[6];
} TTRes;

static int pt_eq(const double* a, const double* b)
{
    return a[0] == b[0] && a[1] == b[1] && a[2] == b[2];
}

/* 3D collinearity of a, b, c (exact). */
static int collinear3(const double* a, const double* b, const double* c)
{
    return oc_orient2d(a, b, c, 0) == 0 && oc_orient2d(a, b, c, 1) == 0 && oc_orient2d(a, b, c, 2) == 0;
}

/* shape: 2 = proper triangle (drop = an axis with nonzero normal component),
 *        1 = segment (e0, e1 extreme points), 0 = point (e0). */
typedef struct {
    int shape;
    int drop;
    const double *e0, *e1;
} Shape;

static Shape tri_shape(const double* const v[3])
{
    Shape s;
    s.e0 = s.e1 = NULL;
    s.drop = -1;
    /* prefer the axis of the largest approximate normal component */
    double n[3];
    for (int k = 0; k < 3; k++) {
        int u = (k + 1) % 3, w = (k + 2) % 3;
        n[k] = fabs((v[1][u] - v[0][u]) * (v[2][w] - v[0][w]) - (v[1][w] - v[0][w]) * (v[2][u] - v[0][u]));
    }
    int order[3] = {0, 1, 2};
    for (int i = 0; i < 3; i++)
        for (int j = i + 1; j < 3; j++)
            if (n[order[j]] > n[order[i]]) { int t = order[i]; order[i] = order[j]; order[j] = t; }
    for (int i = 0; i < 3; i++) {
        if (oc_orient2d(v[0], v[1], v[2], order[i]) != 0) {
            s.shape = 2;
            s.drop = order[i];
            return s;
        }
    }
    if (pt_eq(v[0], v[1]) && pt_eq(v[1], v[2])) {
        s.shape = 0;
        s.e0 = v[0];
        return s;
    }
    int m = 0;
    for (int k = 0; k < 3; k++)
        if (!(v[0][k] == v[1][k] && v[1][k] == v[2][k])) { m = k; break; }
    int imin = 0, imax = 0;
    for (int i = 1; i < 3; i++) {
        if (v[i][m] < v[imin][m]) imin = i;
        if (v[i][m] > v[imax][m]) imax = i;
    }
    s.shape = 1;
    s.e0 = v[imin];
    s.e1 = v[imax];
    return s;
}

/* closed 2D point-in-triangle for a proper triangle (projection drop). */
static int pt_in_tri2d(const double* p, const double* const t[3], int drop)
{
    int s0 = oc_orient2d(t[0], t[1], p, drop);
    int s1 = oc_orient2d(t[1], t[2], p, drop);
    int s2 = oc_orient2d(t[2], t[0], p, drop);
    int pos = (s0 > 0) || (s1 > 0) || (s2 > 0);
    int neg = (s0 < 0) || (s1 < 0) || (s2 < 0);
    return !(pos && neg);
}

/* c within the axis-aligned bounds of segment [a,b] on every coordinate */
static int within_bounds(const double* a, const double* b, const double* c)
{
    for (int k = 0; k < 3; k++) {
        double lo = a[k] < b[k] ? a[k] : b[k];
        double hi = a[k] < b[k] ? b[k] : a[k];
        if (c[k] < lo || c[k] > hi) return 0;
    }
    return 1;
}

static void res_set(TTRes* r, int kind)
{
    r->kind = kind;
}
static void res_add(TTRes* r, SymPt p)
{
    r->pt[r->n++] = p;
}

/* --- points on a segment's line, ordered by an exact rational parameter --- */
#define PP_MAX 40 /* o2 values have <= 16 components, their differences <= 32 */
typedef struct {
    SymPt pt;
    double num[PP_MAX];
    int nnum;
    double den[PP_MAX];
    int nden;
} ParamPt;

/* sign(t1 - t2) with t = num/den */
static int param_cmp(const ParamPt* x, const ParamPt* y)
{
    double* buf = scratch(); /* 3 regions of 2 * PP_MAX * PP_MAX <= 4 * CR_MAX doubles */
    double* p1 = buf;
    double* p2 = buf + 2 * PP_MAX * PP_MAX;
    double* tmp = buf + 4 * PP_MAX * PP_MAX;
    int n1 = exp_mul(x->nnum, x->num, y->nden, y->den, p1, tmp);
    int n2 = exp_mul(y->nnum, y->num, x->nden, x->den, p2, tmp);
    exp_neg(n2, p2);
    int n3 = exp_add(n1, p1, n2, p2, tmp);
    return exp_sign(n3, tmp) * exp_sign(x->nden, x->den) * exp_sign(y->nden, y->den);
}

/* parameter of a point lying on segment e0->e1 (axis m where e0 != e1) */
static void param_vertex(ParamPt* pp, const double* w, const double* e0, const double* e1, int m)
{
    pp->pt = sp_vertex(w);
    pp->nnum = exp_diff2(w[m], e0[m], pp->num);
    pp->nden = exp_diff2(e1[m], e0[m], pp->den);
}
/* parameter of the cut of e0->e1 by 2D line (p,q): t = sa / (sa - sb) */
static void param_line2(ParamPt* pp, const double* e0, const double* e1, const double* p, const double* q,
                        int drop)
{
    double sa[PP_MAX], sb[PP_MAX];
    int na = o2_exact(p, q, e0, drop, sa);
    int nb = o2_exact(p, q, e1, drop, sb);
    pp->pt = sp_line2(e0, e1, p, q, drop);
    memcpy(pp->num, sa, sizeof(double) * (size_t)na);
    pp->nnum = na;
    exp_neg(nb, sb);
    pp->nden = exp_add(na, sa, nb, sb, pp->den);
}

static int seg_axis(const double* e0, const double* e1)
{
    double best = -1.0;
    int m = 0;
    for (int k = 0; k < 3; k++) {
        double d = fabs(e1[k] - e0[k]);
        if (e1[k] != e0[k] && d > best) { best = d; m = k; }
    }
    return m;
}

/* reduce a candidate list on a line to point / segment */
static void finish_on_line(ParamPt* c, int nc, TTRes* r)
{
    if (nc == 0) { res_set(r, OC_NONE); return; }
    int imin = 0, imax = 0;
    for (int i = 1; i < nc; i++) {
        if (param_cmp(&c[i], &c[imin]) < 0) imin = i;
        if (param_cmp(&c[i], &c[imax]) > 0) imax = i;
    }
    if (param_cmp(&c[imin], &c[imax]) == 0) {
        res_set(r, OC_POINT);
        res_add(r, c[imin].pt);
    } else {
        res_set(r, OC_SEGMENT);
        res_add(r, c[imin].pt);
        res_add(r, c[imax].pt);
    }
}

/* segment [e0,e1] vs proper triangle t (with projection drop). */
static void seg_tri(const double* e0, const double* e1, const double* const t[3], int drop, TTRes* r)
{
    int s0 = oc_orient3d(t[0], t[1], t[2], e0);
    int s1 = oc_orient3d(t[0], t[1], t[2], e1);
    if (s0 * s1 > 0) { res_set(r, OC_NONE); return; }
    if (s0 != 0 || s1 != 0) {
        SymPt x;
        if (s0 == 0) x = sp_vertex(e0);
        else if (s1 == 0) x = sp_vertex(e1);
        else x = sp_plane(e0, e1, t[0], t[1], t[2]);
        int a = oc_orient3d(e0, e1, t[0], t[1]);
        int b = oc_orient3d(e0, e1, t[1], t[2]);
        int c = oc_orient3d(e0, e1, t[2], t[0]);
        int pos = a > 0 || b > 0 || c > 0, neg = a < 0 || b < 0 || c < 0;
        if (pos && neg) { res_set(r, OC_NONE); return; }
        res_set(r, OC_POINT);
        res_add(r, x);
        return;
    }
    /* coplanar: clip the segment by the triangle */
    ParamPt* c = (ParamPt*)malloc(sizeof(ParamPt) * 8);
    int nc = 0;
    int m = seg_axis(e0, e1);
    if (pt_in_tri2d(e0, t, drop)) { param_vertex(&c[nc++], e0, e0, e1, m); }
    if (pt_in_tri2d(e1, t, drop)) { param_vertex(&c[nc++], e1, e0, e1, m); }
    for (int k = 0; k < 3; k++) {
        const double* w0 = t[k];
        const double* w1 = t[(k + 1) % 3];
        int da = oc_orient2d(w0, w1, e0, drop), db = oc_orient2d(w0, w1, e1, drop);
        int d3 = oc_orient2d(e0, e1, w0, drop), d4 = oc_orient2d(e0, e1, w1, drop);
        if (da * db < 0 && d3 * d4 < 0) param_line2(&c[nc++], e0, e1, w0, w1, drop);
    }
    for (int k = 0; k < 3; k++) {
        const double* w = t[k];
        if (oc_orient2d(e0, e1, w, drop) == 0 && within_bounds(e0, e1, w) && !pt_eq(w, e0) && !pt_eq(w, e1))
            param_vertex(&c[nc++], w, e0, e1, m);
    }
    finish_on_line(c, nc, r);
    free(c);
}

static void pt_tri(const double* p, const double* const t[3], int drop, TTRes* r)
{
    if (oc_orient3d(t[0], t[1], t[2], p) != 0 || !pt_in_tri2d(p, t, drop)) { res_set(r, OC_NONE); return; }
    res_set(r, OC_POINT);
    res_add(r, sp_vertex(p));
}

static void pt_seg(const double* p, const double* e0, const double* e1, TTRes* r)
{
    if (collinear3(e0, e1, p) && within_bounds(e0, e1, p)) {
        res_set(r, OC_POINT);
        res_add(r, sp_vertex(p));
    } else {
        res_set(r, OC_NONE);
    }
}

static void seg_seg(const double* e0, const double* e1, const double* f0, const double* f1, TTRes* r)
{
    if (oc_orient3d(e0, e1, f0, f1) != 0) { res_set(r, OC_NONE); return; }
    int c0 = collinear3(e0, e1, f0), c1 = collinear3(e0, e1, f1);
    if (c0 && c1) {
        int m = seg_axis(e0, e1);
        const double* ea = e0[m] < e1[m] ? e0 : e1;
        const double* eb = e0[m] < e1[m] ? e1 : e0;
        const double* fa = f0[m] < f1[m] ? f0 : f1;
        const double* fb = f0[m] < f1[m] ? f1 : f0;
        const double* lo = ea[m] >= fa[m] ? ea : fa;
        const double* hi = eb[m] <= fb[m] ? eb : fb;
        if (lo[m] > hi[m]) { res_set(r, OC_NONE); return; }
        if (lo[m] == hi[m]) { res_set(r, OC_POINT); res_add(r, sp_vertex(lo)); return; }
        res_set(r, OC_SEGMENT);
        res_add(r, sp_vertex(lo));
        res_add(r, sp_vertex(hi));
        return;
    }
    const double* fx = c0 ? f1 : f0;
    int drop = 0;
    for (int k = 0; k < 3; k++)
        if (oc_orient2d(e0, e1, fx, k) != 0) { drop = k; break; }
    int d1 = oc_orient2d(f0, f1, e0, drop), d2 = oc_orient2d(f0, f1, e1, drop);
    int d3 = oc_orient2d(e0, e1, f0, drop), d4 = oc_orient2d(e0, e1, f1, drop);
    if (d1 * d2 < 0 && d3 * d4 < 0) {
        res_set(r, OC_POINT);
        res_add(r, sp_line2(e0, e1, f0, f1, drop));
        return;
    }
    const double* touch = NULL;
    if (d1 == 0 && within_bounds(f0, f1, e0)) touch = e0;
    else if (d2 == 0 && within_bounds(f0, f1, e1)) touch = e1;
    else if (d3 == 0 && within_bounds(e0, e1, f0)) touch = f0;
    else if (d4 == 0 && within_bounds(e0, e1, f1)) touch = f1;
    if (touch) { res_set(r, OC_POINT); res_add(r, sp_vertex(touch)); return; }
    res_set(r, OC_NONE);
}

/* --- proper x proper, coplanar ------------------------------------------- */
static void coplanar_tt(const double* const P[3], const double* const Q[3], int drop, TTRes* r, int want)
{
    int sig1 = oc_orient2d(P[0], P[1], P[2], drop);
    int sig2 = oc_orient2d(Q[0], Q[1], Q[2], drop);
    int E2[3][3]; /* E2[j][i]: P[i] vs Q edge j */
    int E1[3][3]; /* E1[i][j]: Q[j] vs P edge i */
    for (int j = 0; j < 3; j++)
        for (int i = 0; i < 3; i++) E2[j][i] = sig2 * oc_orient2d(Q[j], Q[(j + 1) % 3], P[i], drop);
    for (int i = 0; i < 3; i++)
        for (int j = 0; j < 3; j++) E1[i][j] = sig1 * oc_orient2d(P[i], P[(i + 1) % 3], Q[j], drop);
    int v1in[3], v2in[3];
    int any = 0;
    for (int i = 0; i < 3; i++) {
        v1in[i] = E2[0][i] >= 0 && E2[1][i] >= 0 && E2[2][i] >= 0;
        any |= v1in[i];
    }
    for (int j = 0; j < 3; j++) {
        v2in[j] = E1[0][j] >= 0 && E1[1][j] >= 0 && E1[2][j] >= 0;
        any |= v2in[j];
    }
    int prop[3][3];
    int nprop = 0;
    for (int i = 0; i < 3; i++)
        for (int j = 0; j < 3; j++) {
            int d1 = E2[j][i], d2 = E2[j][(i + 1) % 3], d3 = E1[i][j], d4 = E1[i][(j + 1) % 3];
            prop[i][j] = (d1 * d2 < 0) && (d3 * d4 < 0);
            nprop += prop[i][j];
        }
    if (!any && nprop == 0) { res_set(r, OC_NONE); return; }
    if (!want) { res_set(r, OC_POINT); return; }
    /* dimension-2 test: no edge line separates the triangles */
    int sep = 0;
    for (int j = 0; j < 3 && !sep; j++)
        if (E2[j][0] <= 0 && E2[j][1] <= 0 && E2[j][2] <= 0) sep = 1;
    for (int i = 0; i < 3 && !sep; i++)
        if (E1[i][0] <= 0 && E1[i][1] <= 0 && E1[i][2] <= 0) sep = 1;
    /* distinct vertex points */
    const double* vp[6];
    int nv = 0;
    for (int i = 0; i < 3; i++)
        if (v1in[i]) vp[nv++] = P[i];
    for (int j = 0; j < 3; j++) {
        if (!v2in[j]) continue;
        int dup = 0;
        for (int k = 0; k < nv; k++)
            if (pt_eq(vp[k], Q[j])) dup = 1;
        if (!dup) vp[nv++] = Q[j];
    }
    if (!sep) {
        r->n = 0;
        for (int k = 0; k < nv; k++) res_add(r, sp_vertex(vp[k]));
        for (int i = 0; i < 3; i++)
            for (int j = 0; j < 3; j++)
                if (prop[i][j]) res_add(r, sp_line2(P[i], P[(i + 1) % 3], Q[j], Q[(j + 1) % 3], drop));
        res_set(r, r->n == 3 ? OC_TRIANGLE : OC_POLYGON);
        return;
    }
    /* lower-dimensional: all points collinear; keep the two extremes */
    if (nv == 1) { res_set(r, OC_POINT); res_add(r, sp_vertex(vp[0])); return; }
    int m = 0;
    for (int k = 0; k < 3; k++) {
        int same = 1;
        for (int q = 1; q < nv; q++)
            if (vp[q][k] != vp[0][k]) same = 0;
        if (!same) { m = k; break; }
    }
    int imin = 0, imax = 0;
    for (int q = 1; q < nv; q++) {
        if (vp[q][m] < vp[imin][m]) imin = q;
        if (vp[q][m] > vp[imax][m]) imax = q;
    }
    res_set(r, OC_SEGMENT);
    res_add(r, sp_vertex(vp[imin]));
    res_add(r, sp_vertex(vp[imax]));
}

/* --- proper x proper, not coplanar ---------------------------------------- */
typedef struct {
    SymPt pt;
    const double *cn, *cp; /* crossing representation: side(cn) <= 0 <= side(cp) */
} LinePt;

static void rep_from(const double* u, const double* x, int sx, LinePt* lp)
{
    if (sx < 0) { lp->cn = x; lp->cp = u; }
    else { lp->cn = u; lp->cp = x; }
}

/* interval T ∩ plane(other), s = sides of T's vertices w.r.t. other */
static int build_interval(const double* const T[3], const int s[3], const double* const O[3], LinePt out[2])
{
    int z = (s[0] == 0) + (s[1] == 0) + (s[2] == 0);
    if (z == 2) {
        int o = s[0] != 0 ? 0 : (s[1] != 0 ? 1 : 2);
        int k = 0;
        for (int i = 0; i < 3; i++) {
            if (i == o) continue;
            out[k].pt = sp_vertex(T[i]);
            rep_from(T[i], T[o], s[o], &out[k]);
            k++;
        }
        return 2;
    }
    if (z == 1) {
        int u = s[0] == 0 ? 0 : (s[1] == 0 ? 1 : 2);
        int x = (u + 1) % 3, y = (u + 2) % 3;
        out[0].pt = sp_vertex(T[u]);
        rep_from(T[u], T[x], s[x], &out[0]);
        if (s[x] * s[y] > 0) return 1;
        out[1].pt = sp_plane(T[x], T[y], O[0], O[1], O[2]);
        out[1].cn = s[x] < 0 ? T[x] : T[y];
        out[1].cp = s[x] < 0 ? T[y] : T[x];
        return 2;
    }
    int o;
    if (s[0] != s[1] && s[0] != s[2]) o = 0;
    else if (s[1] != s[0] && s[1] != s[2]) o = 1;
    else o = 2;
    int k = 0;
    for (int i = 0; i < 3; i++) {
        if (i == o) continue;
        out[k].pt = sp_plane(T[o], T[i], O[0], O[1], O[2]);
        out[k].cn = s[o] < 0 ? T[o] : T[i];
        out[k].cp = s[o] < 0 ? T[i] : T[o];
        k++;
    }
    return 2;
}

static void general_tt(const double* const P[3], const double* const Q[3], const int s1[3], const int s2[3],
                       TTRes* r, int want)
{
    LinePt I1[2], I2[2];
    int n1 = build_interval(P, s1, Q, I1);
    int n2 = build_interval(Q, s2, P, I2);
    int cmp[2][2];
    for (int i = 0; i < n1; i++)
        for (int j = 0; j < n2; j++) cmp[i][j] = oc_orient3d(I1[i].cn, I1[i].cp, I2[j].cn, I2[j].cp);
    int xin[2] = {0, 0}, yin[2] = {0, 0};
    for (int i = 0; i < n1; i++) xin[i] = (n2 == 1) ? (cmp[i][0] == 0) : (cmp[i][0] * cmp[i][1] <= 0);
    for (int j = 0; j < n2; j++) yin[j] = (n1 == 1) ? (cmp[0][j] == 0) : (cmp[0][j] * cmp[1][j] <= 0);
    r->n = 0;
    for (int i = 0; i < n1; i++)
        if (xin[i]) res_add(r, I1[i].pt);
    for (int j = 0; j < n2; j++) {
        if (!yin[j]) continue;
        int dup = 0;
        for (int i = 0; i < n1; i++)
            if (xin[i] && cmp[i][j] == 0) dup = 1;
        if (!dup) res_add(r, I2[j].pt);
    }
    (void)want;
    r->kind = r->n == 0 ? OC_NONE : (r->n == 1 ? OC_POINT : OC_SEGMENT);
}

static void classify(const double* const P[3], const double* const Q[3], TTRes* r, int want)
{
    r->n = 0;
    r->kind = OC_NONE;
    Shape sp = tri_shape(P), sq = tri_shape(Q);
    if (sp.shape == 2 && sq.shape == 2) {
        int s2[3], s1[3];
        for (int j = 0; j < 3; j++) s2[j] = oc_orient3d(P[0], P[1], P[2], Q[j]);
        if ((s2[0] > 0 && s2[1] > 0 && s2[2] > 0) || (s2[0] < 0 && s2[1] < 0 && s2[2] < 0)) return;
        for (int i = 0; i < 3; i++) s1[i] = oc_orient3d(Q[0], Q[1], Q[2], P[i]);
        if ((s1[0] > 0 && s1[1] > 0 && s1[2] > 0) || (s1[0] < 0 && s1[1] < 0 && s1[2] < 0)) return;
        if (s2[0] == 0 && s2[1] == 0 && s2[2] == 0) {
            coplanar_tt(P, Q, sp.drop, r, want);
            return;
        }
        general_tt(P, Q, s1, s2, r, want);
        return;
    }
    if (sp.shape == 2 && sq.shape == 1) { seg_tri(sq.e0, sq.e1, P, sp.drop, r); return; }
    if (sp.shape == 1 && sq.shape == 2) { seg_tri(sp.e0, sp.e1, Q, sq.drop, r); return; }
    if (sp.shape == 2 && sq.shape == 0) { pt_tri(sq.e0, P, sp.drop, r); return; }
    if (sp.shape == 0 && sq.shape == 2) { pt_tri(sp.e0, Q, sq.drop, r); return; }
    if (sp.shape == 1 && sq.shape == 1) { seg_seg(sp.e0, sp.e1, sq.e0, sq.e1, r); return; }
    if (sp.shape == 1 && sq.shape == 0) { pt_seg(sq.e0, sp.e0, sp.e1, r); return; }
    if (sp.shape == 0 && sq.shape == 1) { pt_seg(sp.e0, sq.e0, sq.e1, r); return; }
    if (pt_eq(sp.e0, sq.e0)) { res_set(r, OC_POINT); res_add(r, sp_vertex(sp.e0)); }
}

int oc_tri_tri_intersect(const double* t1, const double* t2)
{
    const double* P[3] = {t1, t1 + 3, t1 + 6};
    const double* Q[3] = {t2, t2 + 3, t2 + 6};
    TTRes r;
    classify(P, Q, &r, 0);
    return r.kind != OC_NONE;
}

int oc_tri_tri_construct(const double* t1, const double* t2, double* pts, int* npts)
{
    const double* P[3] = {t1, t1 + 3, t1 + 6};
    const double* Q[3] = {t2, t2 + 3, t2 + 6};
    TTRes r;
    classify(P, Q, &r, 1);
    for (int k = 0; k < r.n; k++) sp_construct(&r.pt[k], pts + 3 * k);
    *npts = r.n;
    return r.kind;
}

/* ------------------------------------------------------------------------- */
/* Pose                                                                       */
/* ------------------------------------------------------------------------- */
void oc_pose_identity(oc_pose* p)
{
    memset(p, 0, sizeof *p);
    p->R[0] = p->R[4] = p->R[8] = 1.0;
    p->identity = 1;
}

/* RotationTools.h:28-53: R = Rz * Ry * Rx from degrees. */
void oc_pose_from_euler_deg(const double rot_deg[3], const double center[3], const double trans[3], oc_pose* out)
{
    const double d2r = 3.14159265358979323846 / 180.0;
    double rx = rot_deg[0] * d2r, ry = rot_deg[1] * d2r, rz = rot_deg[2] * d2r;
    double cx = cos(rx), sx = sin(rx), cy = cos(ry), sy = sin(ry), cz = cos(rz), sz = sin(rz);
    out->R[0] = cy * cz;
    out->R[1] = sx * sy * cz - cx * sz;
    out->R[2] = cx * sy * cz + sx * sz;
    out->R[3] = cy * sz;
    out->R[4] = sx * sy * sz + cx * cz;
    out->R[5] = cx * sy * sz - sx * cz;
    out->R[6] = -sy;
    out->R[7] = sx * cy;
    out->R[8] = cx * cy;
    for (int i = 0; i < 3; i++) {
        out->C[i] = center[i];
        out->T[i] = trans[i];
    }
    out->identity = (rot_deg[0] == 0.0 && rot_deg[1] == 0.0 && rot_deg[2] == 0.0 && trans[0] == 0.0 &&
                     trans[1] == 0.0 && trans[2] == 0.0);
}

/* RotationTools.h:135-143: x = v - c; r = R x (left-to-right sums); out = (r + c) + t */
void oc_transform_vertices(const oc_pose* p, const double* vin, size_t nv, double* vout)
{
    if (p->identity) {
        memmove(vout, vin, sizeof(double) * 3 * nv);
        return;
    }
    const double* R = p->R;
    for (size_t i = 0; i < nv; i++) {
        double x = vin[3 * i] - p->C[0], y = vin[3 * i + 1] - p->C[1], z = vin[3 * i + 2] - p->C[2];
        double rx = R[0] * x + R[1] * y + R[2] * z;
        double ry = R[3] * x + R[4] * y + R[5] * z;
        double rz = R[6] * x + R[7] * y + R[8] * z;
        vout[3 * i] = rx + p->C[0] + p->T[0];
        vout[3 * i + 1] = ry + p->C[1] + p->T[1];
        vout[3 * i + 2] = rz + p->C[2] + p->T[2];
    }
}

/* ------------------------------------------------------------------------- */
/* Mesh level: CPU BVH over exact FP64 boxes of B, threads over A triangles   */
/* ------------------------------------------------------------------------- */
typedef struct {
    double lo[3], hi[3];
    int32_t left, right; /* children, or -1 for a leaf */
    uint32_t start, count;
} CNode;

typedef struct {
    CNode* nodes;
    uint32_t nnodes;
    uint32_t* idx;
    const double* box; /* 6 per triangle: lo xyz, hi xyz */
} CBvh;

static void box_of(const double* v, const uint32_t* t, uint32_t i, double* b)
{
    const double* p0 = v + 3 * (size_t)t[3 * (size_t)i];
    const double* p1 = v + 3 * (size_t)t[3 * (size_t)i + 1];
    const double* p2 = v + 3 * (size_t)t[3 * (size_t)i + 2];
    for (int k = 0; k < 3; k++) {
        double lo = p0[k], hi = p0[k];
        if (p1[k] < lo) lo = p1[k];
        if (p1[k] > hi) hi = p1[k];
        if (p2[k] < lo) lo = p2[k];
        if (p2[k] > hi) hi = p2[k];
        b[k] = lo;
        b[3 + k] = hi;
    }
}

static uint32_t bvh_build_rec(CBvh* h, uint32_t start, uint32_t count)
{
    uint32_t id = h->nnodes++;
    CNode* n = &h->nodes[id];
    for (int k = 0; k < 3; k++) { n->lo[k] = INFINITY; n->hi[k] = -INFINITY; }
    double clo[3] = {INFINITY, INFINITY, INFINITY}, chi[3] = {-INFINITY, -INFINITY, -INFINITY};
    for (uint32_t i = start; i < start + count; i++) {
        const double* b = h->box + 6 * (size_t)h->idx[i];
        for (int k = 0; k < 3; k++) {
            if (b[k] < n->lo[k]) n->lo[k] = b[k];
            if (b[3 + k] > n->hi[k]) n->hi[k] = b[3 + k];
            double c = 0.5 * (b[k] + b[3 + k]);
            if (c < clo[k]) clo[k] = c;
            if (c > chi[k]) chi[k] = c;
        }
    }
    if (count <= 4) {
        n->left = n->right = -1;
        n->start = start;
        n->count = count;
        return id;
    }
    int ax = 0;
    double ext = chi[0] - clo[0];
    for (int k = 1; k < 3; k++)
        if (chi[k] - clo[k] > ext) { ext = chi[k] - clo[k]; ax = k; }
    /* quickselect the median by centroid along ax (Hoare partition) */
    int64_t lo = start, hi = (int64_t)start + count - 1, mid = start + count / 2;
    while (lo < hi) {
        const double* pb = h->box + 6 * (size_t)h->idx[(lo + hi) / 2];
        double pivot = pb[ax] + pb[3 + ax];
        int64_t i = lo, j = hi;
        while (i <= j) {
            while (h->box[6 * (size_t)h->idx[i] + ax] + h->box[6 * (size_t)h->idx[i] + 3 + ax] < pivot) i++;
            while (h->box[6 * (size_t)h->idx[j] + ax] + h->box[6 * (size_t)h->idx[j] + 3 + ax] > pivot) j--;
            if (i <= j) {
                uint32_t t = h->idx[i];
                h->idx[i] = h->idx[j];
                h->idx[j] = t;
                i++;
                j--;
            }
        }
        if (mid <= j) hi = j;
        else if (mid >= i) lo = i;
        else break;
    }
    uint32_t nl = (uint32_t)mid - start;
    int32_t l = (int32_t)bvh_build_rec(h, start, nl);
    int32_t r = (int32_t)bvh_build_rec(h, (uint32_t)mid, count - nl);
    n = &h->nodes[id];
    n->left = l;
    n->right = r;
    n->start = start;
    n->count = count;
    return id;
}

typedef struct {
    const double *wA, *wB;
    const uint32_t *tA, *tB;
    uint32_t ntA;
    const CBvh* bvh;
    int want_segments;
    atomic_uint next;
    uint32_t chunk;
} Job;

typedef struct {
    int32_t* pairs; /* a, b */
    uint32_t* nseg; /* per pair */
    double* segs;   /* 6 per segment */
    uint64_t np, cap_p, ns, cap_s;
    uint64_t candidates;
    uint64_t exact_calls;
} Local;

static void local_push(Local* L, int32_t a, int32_t b, const double* segs, uint32_t ns)
{
    if (L->np == L->cap_p) {
        L->cap_p = L->cap_p ? L->cap_p * 2 : 1024;
        L->pairs = (int32_t*)realloc(L->pairs, sizeof(int32_t) * 2 * L->cap_p);
        L->nseg = (uint32_t*)realloc(L->nseg, sizeof(uint32_t) * L->cap_p);
    }
    L->pairs[2 * L->np] = a;
    L->pairs[2 * L->np + 1] = b;
    L->nseg[L->np] = ns;
    L->np++;
    if (ns) {
        while (L->ns + ns > L->cap_s) {
            L->cap_s = L->cap_s ? L->cap_s * 2 : 1024;
            L->segs = (double*)realloc(L->segs, sizeof(double) * 6 * L->cap_s);
        }
        memcpy(L->segs + 6 * L->ns, segs, sizeof(double) * 6 * ns);
        L->ns += ns;
    }
}

static uint32_t segments_of(int kind, const double* pts, double* segs)
{
    if (kind == OC_POINT) {
        memcpy(segs, pts, 3 * sizeof(double));
        memcpy(segs + 3, pts, 3 * sizeof(double));
        return 1;
    }
    if (kind == OC_SEGMENT) {
        memcpy(segs, pts, 6 * sizeof(double));
        return 1;
    }
    if (kind == OC_TRIANGLE) {
        for (int e = 0; e < 3; e++) {
            memcpy(segs + 6 * e, pts + 3 * e, 3 * sizeof(double));
            memcpy(segs + 6 * e + 3, pts + 3 * ((e + 1) % 3), 3 * sizeof(double));
        }
        return 3;
    }
    return 0;
}

static void process_pair(const Job* J, Local* L, uint32_t a, uint32_t b)
{
    const uint32_t* ta = J->tA + 3 * (size_t)a;
    const uint32_t* tb = J->tB + 3 * (size_t)b;
    const double* P[3] = {J->wA + 3 * (size_t)ta[0], J->wA + 3 * (size_t)ta[1], J->wA + 3 * (size_t)ta[2]};
    const double* Q[3] = {J->wB + 3 * (size_t)tb[0], J->wB + 3 * (size_t)tb[1], J->wB + 3 * (size_t)tb[2]};
    TTRes r;
    classify(P, Q, &r, J->want_segments);
    if (r.kind == OC_NONE) return;
    double pts[18], segs[18];
    uint32_t ns = 0;
    if (J->want_segments) {
        for (int k = 0; k < r.n; k++) sp_construct(&r.pt[k], pts + 3 * k);
        ns = segments_of(r.kind, pts, segs);
    }
    local_push(L, (int32_t)a, (int32_t)b, segs, ns);
}

typedef struct {
    Job* J;
    Local L;
} Worker;

static void* worker_main(void* arg)
{
    Worker* W = (Worker*)arg;
    Job* J = W->J;
    Local* L = &W->L;
    tl_exact_calls = 0;
    uint32_t stack[256];
    for (;;) {
        uint32_t s = atomic_fetch_add(&J->next, J->chunk);
        if (s >= J->ntA) break;
        uint32_t e = s + J->chunk < J->ntA ? s + J->chunk : J->ntA;
        for (uint32_t a = s; a < e; a++) {
            double ba[6];
            box_of(J->wA, J->tA, a, ba);
            int sp = 0;
            stack[sp++] = 0;
            while (sp) {
                const CNode* n = &J->bvh->nodes[stack[--sp]];
                if (n->lo[0] > ba[3] || n->hi[0] < ba[0] || n->lo[1] > ba[4] || n->hi[1] < ba[1] ||
                    n->lo[2] > ba[5] || n->hi[2] < ba[2])
                    continue;
                if (n->left < 0) {
                    for (uint32_t k = n->start; k < n->start + n->count; k++) {
                        uint32_t b = J->bvh->idx[k];
                        const double* bb = J->bvh->box + 6 * (size_t)b;
                        if (bb[0] > ba[3] || bb[3] < ba[0] || bb[1] > ba[4] || bb[4] < ba[1] || bb[2] > ba[5] ||
                            bb[5] < ba[2])
                            continue;
                        L->candidates++;
                        process_pair(J, L, a, b);
                    }
                } else {
                    stack[sp++] = (uint32_t)n->left;
                    stack[sp++] = (uint32_t)n->right;
                }
            }
        }
    }
    L->exact_calls = tl_exact_calls;
    return NULL;
}

typedef struct {
    int32_t a, b;
    uint64_t seg_off;
    uint32_t nseg;
} Rec;

static int rec_cmp(const void* x, const void* y)
{
    const Rec* p = (const Rec*)x;
    const Rec* q = (const Rec*)y;
    if (p->a != q->a) return p->a < q->a ? -1 : 1;
    if (p->b != q->b) return p->b < q->b ? -1 : 1;
    return 0;
}

int oc_hw_threads(void)
{
    long n = sysconf(_SC_NPROCESSORS_ONLN);
    return n > 0 ? (int)n : 1;
}

static double now_ms(void)
{
    struct timespec ts;
    clock_gettime(CLOCK_MONOTONIC, &ts);
    return ts.tv_sec * 1e3 + ts.tv_nsec * 1e-6;
}

int oc_intersect_meshes(const double* vA, uint32_t nvA, const uint32_t* tA, uint32_t ntA, const oc_pose* pA,
                        const double* vB, uint32_t nvB, const uint32_t* tB, uint32_t ntB, const oc_pose* pB,
                        int want_segments, int nthreads, uint32_t a_limit, int32_t** pairs, uint64_t* npairs,
                        double** segs, int32_t** seg_pair, uint64_t* nsegs, oc_stats* stats)
{
    double t0 = now_ms();
    *pairs = NULL;
    *npairs = 0;
    if (segs) *segs = NULL;
    if (seg_pair) *seg_pair = NULL;
    if (nsegs) *nsegs = 0;
    for (uint64_t i = 0; i < 3ull * ntA; i++)
        if (tA[i] >= nvA) return -1;
    for (uint64_t i = 0; i < 3ull * ntB; i++)
        if (tB[i] >= nvB) return -1;
    if (ntA == 0 || ntB == 0) {
        if (stats) memset(stats, 0, sizeof *stats);
        return 0;
    }
    double* wA = (double*)malloc(sizeof(double) * 3 * (size_t)nvA);
    double* wB = (double*)malloc(sizeof(double) * 3 * (size_t)nvB);
    oc_transform_vertices(pA, vA, nvA, wA);
    oc_transform_vertices(pB, vB, nvB, wB);
    double* boxB = (double*)malloc(sizeof(double) * 6 * (size_t)ntB);
    for (uint32_t i = 0; i < ntB; i++) box_of(wB, tB, i, boxB + 6 * (size_t)i);
    CBvh h;
    h.nodes = (CNode*)malloc(sizeof(CNode) * 2 * (size_t)ntB);
    h.nnodes = 0;
    h.idx = (uint32_t*)malloc(sizeof(uint32_t) * ntB);
    for (uint32_t i = 0; i < ntB; i++) h.idx[i] = i;
    h.box = boxB;
    bvh_build_rec(&h, 0, ntB);

    Job J;
    J.wA = wA; J.wB = wB; J.tA = tA; J.tB = tB;
    J.ntA = (a_limit > 0 && a_limit < ntA) ? a_limit : ntA;
    J.bvh = &h;
    J.want_segments = want_segments;
    atomic_init(&J.next, 0);
    J.chunk = 64;
    if (nthreads <= 0) nthreads = oc_hw_threads();
    Worker* W = (Worker*)calloc((size_t)nthreads, sizeof(Worker));
    pthread_t* th = (pthread_t*)malloc(sizeof(pthread_t) * (size_t)nthreads);
    pthread_attr_t attr;
    pthread_attr_init(&attr);
    pthread_attr_setstacksize(&attr, 16u << 20);
    for (int i = 0; i < nthreads; i++) {
        W[i].J = &J;
        pthread_create(&th[i], &attr, worker_main, &W[i]);
    }
    for (int i = 0; i < nthreads; i++) pthread_join(th[i], NULL);
    pthread_attr_destroy(&attr);

    uint64_t np = 0, ns = 0, cand = 0, ex = 0;
    for (int i = 0; i < nthreads; i++) {
        np += W[i].L.np;
        ns += W[i].L.ns;
        cand += W[i].L.candidates;
        ex += W[i].L.exact_calls;
    }
    Rec* recs = (Rec*)malloc(sizeof(Rec) * (np ? np : 1));
    double* allsegs = (double*)malloc(sizeof(double) * 6 * (ns ? ns : 1));
    uint64_t k = 0, so = 0;
    for (int i = 0; i < nthreads; i++) {
        Local* L = &W[i].L;
        uint64_t lo = 0;
        for (uint64_t j = 0; j < L->np; j++) {
            recs[k].a = L->pairs[2 * j];
            recs[k].b = L->pairs[2 * j + 1];
            recs[k].nseg = L->nseg[j];
            recs[k].seg_off = so;
            if (L->nseg[j]) memcpy(allsegs + 6 * so, L->segs + 6 * lo, sizeof(double) * 6 * L->nseg[j]);
            so += L->nseg[j];
            lo += L->nseg[j];
            k++;
        }
        free(L->pairs);
        free(L->nseg);
        free(L->segs);
    }
    qsort(recs, np, sizeof(Rec), rec_cmp);
    int32_t* P = (int32_t*)malloc(sizeof(int32_t) * 2 * (np ? np : 1));
    double* S = want_segments ? (double*)malloc(sizeof(double) * 6 * (ns ? ns : 1)) : NULL;
    int32_t* SP = want_segments ? (int32_t*)malloc(sizeof(int32_t) * (ns ? ns : 1)) : NULL;
    uint64_t sw = 0;
    for (uint64_t j = 0; j < np; j++) {
        P[2 * j] = recs[j].a;
        P[2 * j + 1] = recs[j].b;
        if (want_segments) {
            for (uint32_t q = 0; q < recs[j].nseg; q++) {
                memcpy(S + 6 * sw, allsegs + 6 * (recs[j].seg_off + q), sizeof(double) * 6);
                SP[sw] = (int32_t)j;
                sw++;
            }
        }
    }
    free(recs);
    free(allsegs);
    free(W);
    free(th);
    free(h.nodes);
    free(h.idx);
    free(boxB);
    free(wA);
    free(wB);
    *pairs = P;
    *npairs = np;
    if (want_segments) {
        if (segs) *segs = S; else free(S);
        if (seg_pair) *seg_pair = SP; else free(SP);
        if (nsegs) *nsegs = sw;
    }
    if (stats) {
        stats->candidates = cand;
        stats->pairs = np;
        stats->segments = sw;
        stats->filter_failures = ex;
        stats->ms_total = now_ms() - t0;
    }
    return 0;
}

/* Exact test of an explicit pair list on `nthreads` threads: the CPU side of
 * the reference's pair-list filter (filterYellowPairsTBB,
 * src/CPU/YellowFilter.h:80-137, CGAL do_intersect over a pair list on TBB
 * threads).  Vertices are posed once; the list is split into equal slices. */
typedef struct {
    const double *wA, *wB;
    const uint32_t *tA, *tB;
    const int32_t* pairs;
    uint8_t* out;
    uint64_t lo, hi;
} PairSlice;

static void* pair_slice_main(void* arg)
{
    PairSlice* S = (PairSlice*)arg;
    for (uint64_t i = S->lo; i < S->hi; i++) {
        const uint32_t* ta = S->tA + 3 * (size_t)S->pairs[2 * i];
        const uint32_t* tb = S->tB + 3 * (size_t)S->pairs[2 * i + 1];
        const double* T1[3] = {S->wA + 3 * (size_t)ta[0], S->wA + 3 * (size_t)ta[1], S->wA + 3 * (size_t)ta[2]};
        const double* T2[3] = {S->wB + 3 * (size_t)tb[0], S->wB + 3 * (size_t)tb[1], S->wB + 3 * (size_t)tb[2]};
        TTRes r;
        classify(T1, T2, &r, 0);
        S->out[i] = r.kind != OC_NONE;
    }
    return NULL;
}

int oc_classify_pairs(const double* vA, uint32_t nvA, const uint32_t* tA, uint32_t ntA, const oc_pose* pA,
                      const double* vB, uint32_t nvB, const uint32_t* tB, uint32_t ntB, const oc_pose* pB,
                      const int32_t* pairs, uint64_t n, uint8_t* out, int nthreads)
{
    for (uint64_t i = 0; i < n; i++)
        if (pairs[2 * i] < 0 || (uint32_t)pairs[2 * i] >= ntA || pairs[2 * i + 1] < 0 || (uint32_t)pairs[2 * i + 1] >= ntB)
            return -1;
    for (uint64_t i = 0; i < 3 * (uint64_t)ntA; i++)
        if (tA[i] >= nvA) return -1;
    for (uint64_t i = 0; i < 3 * (uint64_t)ntB; i++)
        if (tB[i] >= nvB) return -1;
    double* wA = (double*)malloc(sizeof(double) * 3 * (size_t)(nvA ? nvA : 1));
    double* wB = (double*)malloc(sizeof(double) * 3 * (size_t)(nvB ? nvB : 1));
    oc_transform_vertices(pA, vA, nvA, wA);
    oc_transform_vertices(pB, vB, nvB, wB);
    if (nthreads <= 0) nthreads = oc_hw_threads();
    PairSlice* S = (PairSlice*)calloc((size_t)nthreads, sizeof(PairSlice));
    pthread_t* th = (pthread_t*)malloc(sizeof(pthread_t) * (size_t)nthreads);
    for (int k = 0; k < nthreads; k++) {
        S[k].wA = wA;
        S[k].wB = wB;
        S[k].tA = tA;
        S[k].tB = tB;
        S[k].pairs = pairs;
        S[k].out = out;
        S[k].lo = n * (uint64_t)k / (uint64_t)nthreads;
        S[k].hi = n * (uint64_t)(k + 1) / (uint64_t)nthreads;
        pthread_create(&th[k], NULL, pair_slice_main, &S[k]);
    }
    for (int k = 0; k < nthreads; k++) pthread_join(th[k], NULL);
    free(th);
    free(S);
    free(wA);
    free(wB);
    return 0;
}

int oc_intersect_meshes_bruteforce(const double* vA, uint32_t nvA, const uint32_t* tA, uint32_t ntA,
                                   const oc_pose* pA, const double* vB, uint32_t nvB, const uint32_t* tB,
                                   uint32_t ntB, const oc_pose* pB, int32_t** pairs, uint64_t* npairs)
{
    double* wA = (double*)malloc(sizeof(double) * 3 * (size_t)(nvA ? nvA : 1));
    double* wB = (double*)malloc(sizeof(double) * 3 * (size_t)(nvB ? nvB : 1));
    oc_transform_vertices(pA, vA, nvA, wA);
    oc_transform_vertices(pB, vB, nvB, wB);
    uint64_t cap = 1024, n = 0;
    int32_t* P = (int32_t*)malloc(sizeof(int32_t) * 2 * cap);
    for (uint32_t a = 0; a < ntA; a++) {
        const uint32_t* ta = tA + 3 * (size_t)a;
        const double* T1[3] = {wA + 3 * (size_t)ta[0], wA + 3 * (size_t)ta[1], wA + 3 * (size_t)ta[2]};
        for (uint32_t b = 0; b < ntB; b++) {
            const uint32_t* tb = tB + 3 * (size_t)b;
            const double* T2[3] = {wB + 3 * (size_t)tb[0], wB + 3 * (size_t)tb[1], wB + 3 * (size_t)tb[2]};
            TTRes r;
            classify(T1, T2, &r, 0);
            if (r.kind == OC_NONE) continue;
            if (n == cap) {
                cap *= 2;
                P = (int32_t*)realloc(P, sizeof(int32_t) * 2 * cap);
            }
            P[2 * n] = (int32_t)a;
            P[2 * n + 1] = (int32_t)b;
            n++;
        }
    }
    free(wA);
    free(wB);
    *pairs = P;
    *npairs = n;
    return 0;
}

void oc_free(void* p)
{
    free(p);
}
