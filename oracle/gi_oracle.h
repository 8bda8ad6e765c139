/*
 * gi_oracle.h -- CPU exact oracle for the mesh-mesh intersection path.
 *
 * TEST INFRASTRUCTURE ONLY.  This library is the checker that the CUDA
 * library is compared against (tests/, __graft_entry__.smoke() and the CPU
 * baseline leg of bench.py).  The product path never links or calls it.
 *
 * What it restates from the reference (YuryUoL/gpu-cubql-intersector-standalone):
 *   - pose semantics: Euler degrees, R = Rz*Ry*Rx, applied about a centre plus
 *     a translation, evaluated left to right in FP64 without FMA contraction
 *     (src/CPU/RotationTools.h:28-53 makeRotationMatrixDeg,
 *      src/CPU/RotationTools.h:129-145 transformCgalMesh -- the ground-truth
 *      transform used by src/CPU/TestSuite.cpp:235-321).
 *   - the pair predicate: CGAL::do_intersect(Triangle_3, Triangle_3) on closed
 *     triangles with exact predicates (src/CPU/YellowFilter.h:80-137 and the
 *     CGAL PMP face-face ground truth, src/CPU/TestSuite.cpp:79-102).  CGAL is
 *     not available here; the predicate is restated from its mathematical
 *     definition (closed point sets) with exact orient3d / orient2d signs.
 *   - the segment output rule of CGAL::intersection(Triangle_3, Triangle_3)
 *     as consumed by src/CPU/MeshIntersectionCurves.cpp:63-78: a segment gives
 *     one segment, a point gives a degenerate segment, a coplanar triangle
 *     overlap gives its three edges, a coplanar overlap polygon with four or
 *     more corners gives nothing (the reference has no branch for it).
 *   - pair sets are compared as canonical sets of (faceA, faceB)
 *     (src/CPU/TestSuite.cpp:24-32, 285-296); outputs here are sorted by (a, b).
 *
 * Exact arithmetic: floating-point expansions built from error-free
 * transformations (two-sum, two-product via fma), following Shewchuk,
 * "Adaptive Precision Floating-Point Arithmetic and Fast Robust Geometric
 * Predicates" (1997).  Signs are exact and constructed points are correctly
 * rounded (round to nearest, ties to even) for inputs inside the supported
 * domain: finite coordinates with |x| <= 2^200 and x == 0 or |x| >= 2^-200.
 *
 * PARITY UNPINNED by reference artefacts: the reference ships no golden
 * vectors, known-answer tests or stored outputs for this path (its TestSuite
 * compares against live CGAL), and its path cannot be built here (CGAL, Boost,
 * TBB and cuBQL are absent), so no reference output pins this restatement.
 * It is checked instead against an independent exact-rational restatement
 * (tests/fraction_ref.py, Python fractions: Sutherland-Hodgman clipping and
 * exact hulls), against hand-derived known answers, and against brute force
 * over all pairs (tests/golden/, tests/test_oracle.py).
 */
#ifndef GI_ORACLE_H
#define GI_ORACLE_H

#include <stddef.h>
#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

/* Pose: world = R * (v - C) + C + T, evaluated as in transformCgalMesh. */
typedef struct {
    double R[9];
    double C[3];
    double T[3];
    int identity; /* 1: vertices are used unchanged */
} oc_pose;

/* Intersection kinds (match gi.h GI_KIND_*). */
enum { OC_NONE = 0, OC_POINT = 1, OC_SEGMENT = 2, OC_TRIANGLE = 3, OC_POLYGON = 4 };

/* Pose helpers. */
void oc_pose_identity(oc_pose* p);
void oc_pose_from_euler_deg(const double rot_deg[3], const double center[3],
                            const double trans[3], oc_pose* out);
void oc_transform_vertices(const oc_pose* p, const double* vin, size_t nv, double* vout);

/* Exact predicate signs (-1, 0, +1). orient3d(a,b,c,d) = det[a-d; b-d; c-d]. */
int oc_orient3d(const double* a, const double* b, const double* c, const double* d);
/* orient2d on the projection dropping coordinate `drop` (0=x,1=y,2=z),
 * using the cyclic pair (drop+1, drop+2). */
int oc_orient2d(const double* a, const double* b, const double* c, int drop);

/* Sign log (test hook): between begin and end, every oc_orient3d / oc_orient2d
 * call (also those made inside the intersection tests) is recorded, up to cap
 * entries: 12 doubles per entry (a, b, c, d; orient2d leaves d zero) and 3
 * int32 (kind 0 = orient3d / 1 = orient2d, drop axis or -1, exact sign).  end
 * returns the count and hands over both arrays (free with oc_free). */
int oc_sign_log_begin(uint64_t cap);
uint64_t oc_sign_log_end(double** pts, int32_t** meta);

/* Closed-triangle intersection test (9 doubles per triangle, vertex-major). */
int oc_tri_tri_intersect(const double* t1, const double* t2);

/* Exact intersection set of two closed triangles.
 * Returns the kind; `npts` receives the number of output points written to
 * pts (3 doubles each): POINT 1, SEGMENT 2, TRIANGLE 3, POLYGON k (>= 4, up to 6).
 * Points are correctly rounded doubles. */
int oc_tri_tri_construct(const double* t1, const double* t2, double* pts, int* npts);

/* Statistics of one mesh-mesh run. */
typedef struct {
    uint64_t candidates;      /* exact-box-overlapping triangle pairs tested */
    uint64_t pairs;           /* intersecting pairs */
    uint64_t segments;        /* emitted segments */
    uint64_t filter_failures; /* orient calls that needed expansion arithmetic */
    double ms_total;
} oc_stats;

/* Mesh-mesh intersection on the CPU with `nthreads` threads (0 = all cores).
 * Outputs are malloc'd and owned by the caller (free with oc_free):
 *   pairs: 2 int32 per pair, sorted by (a, b);
 *   segs:  6 doubles per segment, grouped by pair in pair order;
 *   seg_pair: pair index of each segment.
 * If want_segments == 0 the segment outputs are left NULL / 0.
 * a_limit > 0 restricts the run to A triangles [0, a_limit) (bounded samples).
 * Returns 0 on success, negative on error. */
int oc_intersect_meshes(const double* vA, uint32_t nvA, const uint32_t* tA, uint32_t ntA,
                        const oc_pose* pA,
                        const double* vB, uint32_t nvB, const uint32_t* tB, uint32_t ntB,
                        const oc_pose* pB,
                        int want_segments, int nthreads, uint32_t a_limit,
                        int32_t** pairs, uint64_t* npairs,
                        double** segs, int32_t** seg_pair, uint64_t* nsegs,
                        oc_stats* stats);

/* Exact test of each (a, b) of an explicit pair list (out[i] = 1 iff the posed
 * triangles A[a] and B[b] share a point) on `nthreads` threads (0 = all).
 * Returns -1 (nothing written) for an index out of range. */
int oc_classify_pairs(const double* vA, uint32_t nvA, const uint32_t* tA, uint32_t ntA, const oc_pose* pA,
                      const double* vB, uint32_t nvB, const uint32_t* tB, uint32_t ntB, const oc_pose* pB,
                      const int32_t* pairs, uint64_t n, uint8_t* out, int nthreads);

/* Brute-force candidate-free variant for tiny meshes (all pairs, 1 thread). */
int oc_intersect_meshes_bruteforce(const double* vA, uint32_t nvA, const uint32_t* tA, uint32_t ntA,
                                   const oc_pose* pA,
                                   const double* vB, uint32_t nvB, const uint32_t* tB, uint32_t ntB,
                                   const oc_pose* pB,
                                   int32_t** pairs, uint64_t* npairs);

void oc_free(void* p);
int oc_hw_threads(void);

#ifdef __cplusplus
}
#endif
#endif
