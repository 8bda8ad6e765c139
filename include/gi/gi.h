/*
 * gi.h -- C ABI of the B200 mesh-mesh intersector.
 *
 * Plain C: opaque handles, POD structs, pointers and sizes, status codes.
 * Every entry point returns gi_status; nothing exits the process.
 *
 * Each entry point replaces a piece of the reference's GPUIntersector
 * interface (YuryUoL/gpu-cubql-intersector-standalone, paths in that project):
 *
 *   KernelBVHController (src/GPUIntersector/KernelBVHController.h:36-95)
 *     constructor / cleanup() / ~KernelBVHController   -> gi_create, gi_destroy
 *     construct(...)            (KernelBVHController.h:46-57, .cu:444-597)
 *                               -> gi_mesh_upload (once per mesh; the library
 *                                  copies the arrays and builds the BVH)
 *     setTransformBoth(...)     (KernelBVHController.h:72-77, .cu:289-412)
 *                               -> gi_pose_from_euler_deg (+ the poses passed
 *                                  to gi_intersect; no refit is needed)
 *     runIntersectionPipeline(...) (KernelBVHController.h:60-63, .cu:603-699)
 *                               -> gi_intersect + gi_result_pairs / _stats
 *     clearGPU / reconstructGPU (KernelBVHController.h:66-69)
 *                               -> gi_mesh_release / gi_mesh_upload
 *   runGridForestIntersectionPipeline (src/GPUIntersector/StandaloneBVHPipeline.h:27-43)
 *                               -> gi_intersect_oneshot
 *   computeExactIntersectionCurves (src/CPU/MeshIntersectionCurves.h:24-29)
 *                               -> gi_intersect with want_segments = 1,
 *                                  gi_result_segments
 *   ExecutionStats / IntersectionTimeTracker (src/common/ExecutionStats.h:12-46,
 *     src/common/IntersectionTimeTracker.h:6-43)  -> gi_stats
 *
 * Semantics: a pair (a, b) is reported iff the closed triangles A[a] and B[b],
 * after applying their poses in FP64 (world = R*(v - C) + C + T, evaluated left
 * to right without fused multiply-add, as src/CPU/RotationTools.h:129-145),
 * share at least one point.  The decision is exact.  Segments follow
 * src/CPU/MeshIntersectionCurves.cpp:63-78: a crossing segment gives one
 * segment, a single touching point gives a zero-length segment, a coplanar
 * overlap that is a triangle gives its three edges, and a coplanar overlap
 * polygon with four or more corners gives none.  Segment endpoints are the
 * exact intersection points correctly rounded to FP64.
 *
 * Supported coordinate domain (exactness guarantee): finite doubles with
 * |x| <= 2^100 and x == 0 or |x| >= 2^-100, for input vertices, pose entries and posed
 * vertices alike.  gi_mesh_upload rejects inputs outside it (GI_ERR_RANGE).
 *
 * Threading: one gi_ctx owns one CUDA stream; calls on the same context are
 * serialised by the caller.  Different contexts may run concurrently.
 *
 * Device-pointer arguments (gi_mesh_upload_device, gi_classify_pairs,
 * gi_classify_pairs_noalloc): the library reads and writes them on the
 * context's own stream, which is a non-blocking stream and is NOT ordered after
 * the caller's streams (for example torch's current stream).  Before such a
 * call, the work that produces the inputs (and any earlier work on the output
 * buffer) must be complete: synchronise the producing stream, or call
 * gi_wait_stream with it.  These calls block until their own device work is
 * done, so the outputs are complete when they return and later work on any
 * stream may read or overwrite them.
 */
#ifndef GI_GI_H
#define GI_GI_H

#include <stddef.h>
#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

#define GI_ABI_VERSION 1

typedef enum {
    GI_OK = 0,
    GI_ERR_INVALID_ARG = 1, /* null pointer, bad index, bad size */
    GI_ERR_OOM = 2,         /* device or host allocation failed, or HBM budget exceeded */
    GI_ERR_CAPACITY = 3,    /* an internal buffer stayed too small after the retries */
    GI_ERR_TIMEOUT = 4,     /* a bounded device wait ran out (reported, never hung) */
    GI_ERR_CUDA = 5,        /* CUDA runtime error (see gi_last_error) */
    GI_ERR_RANGE = 6,       /* coordinates outside the supported domain */
    GI_ERR_NOT_READY = 7,   /* serving: the request is still in flight */
    GI_ERR_NO_DEVICE = 8    /* no CUDA device or the kernels are not loadable */
} gi_status;

typedef struct gi_ctx gi_ctx;
typedef struct gi_mesh gi_mesh;
typedef struct gi_result gi_result;
typedef struct gi_server gi_server;

/* Context options. */
/* gi_options.flags */
#define GI_FLAG_TINY_BUFFERS 1u /* start every intersect buffer at 64 entries: exercises the
                                   capacity-overflow / retry path (host-side fault injection) */
/* The traversal shape is autotuned per workload class on the context's own
 * calls.  GI_FLAG_FIXED_SHAPE | GI_FLAG_SHAPE(k), k in 0..7, fixes it instead
 * (every shape gives the same results): bit 2 selects the level-synchronous
 * traversal (grid barriers between the levels) over the work-queue one; bit 1
 * the quad form (one node pair per quad of lanes; level-synchronous: on levels
 * of at most 8 node pairs per warp); bit 0 one block per SM instead of all
 * resident blocks (work queue) or the split form, in which a third of the
 * blocks only filter candidates as the levels publish them (level-synchronous). */
#define GI_FLAG_FIXED_SHAPE 0x100u
#define GI_FLAG_SHAPE(k) ((((uint32_t)(k)) & 7u) << 9)

typedef struct {
    int32_t device;             /* CUDA device ordinal */
    uint32_t flags;             /* GI_FLAG_* */
    uint64_t hbm_budget_bytes;  /* 0 = no budget; else mesh + scratch bytes allowed */
} gi_options;

/* Rigid (or general affine) pose: world = R * (v - center) + center + trans. */
typedef struct {
    double R[9]; /* row-major */
    double center[3];
    double trans[3];
    int32_t identity; /* 1: vertices are used unchanged (R, center, trans ignored) */
    int32_t reserved;
} gi_pose;

/* Precision modes. */
#define GI_PREC_FP32_CASCADE 0 /* FP32 boxes + FP32 filter -> FP64 filter -> exact */
#define GI_PREC_FP64 1         /* FP64 boxes + FP64 filter -> exact (plain FP64 form) */

typedef struct {
    int32_t want_segments;  /* 1: emit intersection segments */
    int32_t precision_mode; /* GI_PREC_* */
    int32_t sort_output;    /* 1: pairs sorted by (a, b) (default 1) */
    int32_t reserved;
} gi_intersect_opts;

/* Result statistics (mirrors ExecutionStats / IntersectionTimeTracker). */
typedef struct {
    uint64_t tris_a, tris_b;
    uint64_t nodes_a, nodes_b;        /* wide BVH nodes */
    uint64_t node_pairs;              /* BVH node pairs expanded by the traversal */
    uint64_t candidates;              /* box-overlapping triangle pairs tested */
    uint64_t filter_decided;          /* pairs decided by the first filter stage */
    uint64_t escalated;               /* pairs sent to the FP64 / exact stage */
    uint64_t exact_signs;             /* orientation signs resolved exactly */
    uint64_t exact_points;            /* constructed points that needed exact division */
    uint64_t pairs;                   /* intersecting pairs */
    uint64_t segments;                /* emitted segments */
    uint32_t levels;                  /* traversal levels */
    uint32_t retries;                 /* capacity retries */
    uint32_t launches;                /* kernels launched by this call */
    uint32_t traverse_shape;          /* traversal shape used (GI_FLAG_SHAPE numbering) */
    double ms_traverse;               /* device time: traversal + first filter */
    double ms_exact;                  /* device time: FP64 / exact stage */
    double ms_segments;               /* device time: segment construction */
    double ms_sort;                   /* device time: output ordering (the part after segment construction
                                         ends; ranking overlaps the segments).  With the one-launch
                                         finish (finish_phases = 4), ms_exact, ms_segments and ms_sort
                                         are its phases' own spans (its timestamps) and ms_traverse the
                                         rest of the call, the hand-off between the launches included */
    double ms_total;                  /* device time of the whole call */
    /* level-synchronous traversal only (else level_times = 0): level_end_ms[l]
     * is the time from the traversal's start to the end of level l (level 0:
     * the seeding from the cut pairs; level l > 0 expands the node pairs made
     * by level l - 1 and filters its leaf pairs), for the first level_times levels */
    uint32_t level_times;
    uint32_t reserved2;
    double level_end_ms[32];
    /* one-launch finish after the traversal (sorted output of a small result;
     * else finish_phases = 0): finish_ms[k] is the time from the launch's start
     * to the end of its exact phase (k = 0), of its key and segment phase (1:
     * the last block's arrival), of the count scan (2: the release of the
     * others), and of its last block (3) */
    uint32_t finish_phases;
    uint32_t reserved3;
    double finish_ms[4];
} gi_stats;

/* Batched job: one mesh pair with its poses. */
typedef struct {
    const gi_mesh* A;
    const gi_mesh* B;
    gi_pose pose_a;
    gi_pose pose_b;
} gi_pair_job;

/* Serving options. */
typedef struct {
    uint32_t max_inflight;  /* requests admitted per device round (0 = 256) */
    uint32_t flags;         /* reserved */
    gi_intersect_opts opts; /* options applied to every request */
} gi_server_opts;

/* ---- context ------------------------------------------------------------ */
gi_status gi_create(const gi_options* opts, gi_ctx** out);
gi_status gi_destroy(gi_ctx* ctx);
const char* gi_status_string(gi_status s);
const char* gi_last_error(const gi_ctx* ctx);
gi_status gi_device_count(int32_t* n);
/* Orders the context's streams after all work queued so far on `stream` (a
 * cudaStream_t passed as a pointer; NULL names the legacy default stream), so
 * that device inputs produced there are complete before the context's next
 * call reads them.  Queues a wait; does not block the host.  No counterpart in
 * the reference, whose calls run on the legacy default stream with device-wide
 * synchronisation (src/GPUIntersector/KernelBVHController.cu:258-261). */
gi_status gi_wait_stream(gi_ctx* ctx, void* stream);

/* ---- meshes (KernelBVHController::construct) ----------------------------- */
/* Host arrays: verts_xyz[3*nv] doubles, tris[3*nt] vertex indices. */
gi_status gi_mesh_upload(gi_ctx* ctx, const double* verts_xyz, uint32_t nv, const uint32_t* tris, uint32_t nt,
                         gi_mesh** out);
/* Same, from device pointers already resident on the context's device. */
gi_status gi_mesh_upload_device(gi_ctx* ctx, const double* d_verts_xyz, uint32_t nv, const uint32_t* d_tris,
                                uint32_t nt, gi_mesh** out);
gi_status gi_mesh_release(gi_ctx* ctx, gi_mesh* mesh);
gi_status gi_mesh_info(const gi_mesh* mesh, uint32_t* nv, uint32_t* nt, uint64_t* nodes, uint64_t* device_bytes);
/* Device time in ms of the mesh's validation and BVH build (CUDA events around
 * the build kernels on the build stream; the upload's copies are not in it):
 * ExecutionStats::buildRefitMeshAMs / buildRefitMeshBMs
 * (src/common/ExecutionStats.h:25-26). */
gi_status gi_mesh_build_ms(const gi_mesh* mesh, double* ms);

/* ---- poses (setTransformBoth, RotationTools.h:28-70) ---------------------- */
gi_status gi_pose_identity(gi_pose* out);
gi_status gi_pose_from_euler_deg(const double rot_deg[3], const double center[3], const double trans[3],
                                 gi_pose* out);
/* world coordinates of vertices under a pose, on the host (same FP64 order) */
gi_status gi_pose_apply(const gi_pose* pose, const double* verts_xyz, uint64_t nv, double* out_xyz);

/* ---- intersection (runIntersectionPipeline) ------------------------------ */
gi_status gi_intersect_opts_default(gi_intersect_opts* out);
gi_status gi_intersect(gi_ctx* ctx, const gi_mesh* A, const gi_pose* pose_a, const gi_mesh* B,
                       const gi_pose* pose_b, const gi_intersect_opts* opts, gi_result** out);
/* One-shot from host arrays: upload, build, intersect, release
 * (runGridForestIntersectionPipeline). */
gi_status gi_intersect_oneshot(gi_ctx* ctx, const double* vA, uint32_t nvA, const uint32_t* tA, uint32_t ntA,
                               const gi_pose* pose_a, const double* vB, uint32_t nvB, const uint32_t* tB,
                               uint32_t ntB, const gi_pose* pose_b, const gi_intersect_opts* opts,
                               gi_result** out);
/* Batched: all jobs in one persistent device pass; out[i] receives job i's result. */
gi_status gi_intersect_batch(gi_ctx* ctx, const gi_pair_job* jobs, uint32_t njobs, const gi_intersect_opts* opts,
                             gi_result** out);

/* Exact closed-triangle test over an explicit candidate list: d_out[i] = 1 iff
 * A[d_pairs[2i]] and B[d_pairs[2i+1]] intersect under the poses.  Replaces the
 * reference's predicate kernels over a pair list plus its CPU fallback
 * (src/GPU_exact_predicates/OriginShiftedFloatPredicate.cu:7-26,
 *  src/GPU_exact_predicates/DoublePredicate.cu:166-201, src/CPU/YellowFilter.h:80-137).
 * d_pairs (2 int32 per pair) and d_out (1 byte per pair) are device pointers on
 * the context's device; scratch for the escalated pairs comes from the
 * context's stream-ordered pool.  Bad indices give GI_ERR_INVALID_ARG. */
gi_status gi_classify_pairs(gi_ctx* ctx, const gi_mesh* A, const gi_pose* pose_a, const gi_mesh* B,
                            const gi_pose* pose_b, const int32_t* d_pairs, uint32_t npairs, int32_t precision_mode,
                            uint8_t* d_out);

/* gi_classify_pairs without any allocation at call time.  No counterpart in
 * the reference: it is an addition for callers that may not allocate device
 * memory while they run (a control loop whose memory budget is fixed at
 * start-up, or a host framework whose caching allocator owns the free HBM).
 * Same arguments, semantics and results as gi_classify_pairs; the escalation
 * scratch is one fixed 4 MiB array in the library's device memory per device.
 *  - npairs above GI_NOALLOC_MAX_PAIRS -> GI_ERR_CAPACITY, nothing queued;
 *  - the first call on a device does a one-time set-up (looks up the array's
 *    device address with that device current); make that first call before
 *    any stream capture begins;
 *  - the array is shared by all contexts on a device: calls whose device work
 *    overlaps in time race on it.  Every call blocks until its device work is
 *    done, so calls issued one after another from the host are safe. */
#define GI_NOALLOC_MAX_PAIRS 1048576u
gi_status gi_classify_pairs_noalloc(gi_ctx* ctx, const gi_mesh* A, const gi_pose* pose_a, const gi_mesh* B,
                                    const gi_pose* pose_b, const int32_t* d_pairs, uint32_t npairs,
                                    int32_t precision_mode, uint8_t* d_out);

/* ---- predicate signs (diagnostics of the exact path) ----------------------- */
/* The device's orientation predicates on caller-given points, stage by stage,
 * so that every sign the intersection path can take is checkable against an
 * exact evaluation.  Replaces, for inspection, the reference's device
 * predicates: orient3d_interval (src/GPU_exact_predicates/GPUPredicatesCommon.h:
 * 38-100), orient3d_double_interval (src/GPU_exact_predicates/DoublePredicate.cu:
 * 75-93) and orient3d_exact_V2 / the 2D SAT tests
 * (src/GPU_exact_predicates/ExactBigIntPredicate.cu:180-212, 236-272).
 *   GI_PRED_ORIENT3D: pts holds 12 doubles per query (a, b, c, d); the sign is
 *     that of det[a - d; b - d; c - d] (positive when d lies below the plane
 *     through a, b, c oriented counter-clockwise).
 *   GI_PRED_ORIENT2D: pts holds 9 doubles per query (a, b, c) and drop[i] in
 *     0..2 names the coordinate left out; with (u, v) = (drop + 1, drop + 2) mod
 *     3 the sign is that of (a_u - c_u)(b_v - c_v) - (a_v - c_v)(b_u - c_u).
 * out receives 8 bytes per query:
 *   [0] FP32 semi-static filter, line-order form   [1] FP32 filter, vertex-versus-plane form
 *   [2] FP64 semi-static filter, line-order form   [3] FP64 filter, vertex-versus-plane form
 *   [4] FP64 filter of the exact stage             [5] exact integer sign (always computed)
 *   [6] the exact stage's answer (filter, then integers)
 *   [7] integer branch of [5]: GI_BRANCH_INT128, GI_BRANCH_MULTILIMB or GI_BRANCH_CAPACITY
 * Signs are -1, 0, +1; a filter that does not decide gives GI_SIGN_UNDECIDED;
 * orient2d has no FP32 or semi-static form (GI_SIGN_NA in [0..3]).
 * Host arrays in and out; the call blocks.  Coordinates outside the supported
 * domain give GI_ERR_RANGE, at most 2^26 queries per call. */
#define GI_PRED_ORIENT3D 0
#define GI_PRED_ORIENT2D 1
#define GI_SIGN_UNDECIDED 2
#define GI_SIGN_NA 3
#define GI_BRANCH_INT128 0
#define GI_BRANCH_MULTILIMB 1
#define GI_BRANCH_CAPACITY 2
gi_status gi_predicate_signs(gi_ctx* ctx, int32_t kind, const double* pts, const int32_t* drop, uint64_t n,
                             int8_t* out);

/* ---- ingestion (upstream of the path) -------------------------------------- */
/* OFF files as the reference loads them (src/CPU/RobustOffLoader.h:120-186,
 * src/CPU/ParallelCgalOffLoader.h:35-186): polygons fan-triangulated as
 * (p0, pk, pk+1), triangles with a repeated vertex index dropped, and later
 * copies of a triangle's vertex set dropped.  Parsed on `nthreads` host threads
 * (0: all) from a memory-mapped file. */
typedef struct {
    uint64_t file_vertices, file_polygons; /* counts in the file */
    uint64_t extra_fan_triangles;          /* added by fan-triangulating polygons with > 3 corners */
    uint64_t dropped_degenerate;           /* rows with < 3 corners, fan triangles with a repeated index */
    uint64_t dropped_duplicate;            /* triangles repeating an earlier triangle's vertex set */
} gi_off_report;
typedef struct gi_off_mesh gi_off_mesh;
gi_status gi_off_load(const char* path, uint32_t nthreads, gi_off_mesh** out, gi_off_report* report);
/* host arrays of a loaded file; face_row[i]: the file's face row triangle i came from */
gi_status gi_off_arrays(const gi_off_mesh* m, const double** verts_xyz, uint32_t* nv, const uint32_t** tris,
                        uint32_t* nt, const uint32_t** face_row);
gi_status gi_off_free(gi_off_mesh* m);

/* Scene normalisation (apps/mainApplication.cpp:166-187, 637-680): the box of
 * both meshes is centred and, with scale_to_unit, scaled so that its largest
 * side spans 2: x' = (x - center) * scale in FP64, no fused multiply-add. */
typedef struct {
    double center[3];   /* centre of the scene box, subtracted from every vertex */
    double scale;       /* 2 / max_span with scale_to_unit, else 1 */
    double max_span;    /* largest side of the scene box before scaling */
    double center_a[3]; /* box centres of the normalised meshes: the rotation centres of their poses */
    double center_b[3];
} gi_scene;
/* Loads two OFF files, normalises them on the device and builds both meshes
 * (the reference's load command). */
gi_status gi_scene_load(gi_ctx* ctx, const char* path_a, const char* path_b, int32_t scale_to_unit, gi_mesh** A,
                        gi_mesh** B, gi_scene* scene, gi_off_report* report_a, gi_off_report* report_b);
/* The mesh's vertices (3 doubles each, as stored on the device) into verts_xyz_out. */
gi_status gi_mesh_download(const gi_mesh* mesh, double* verts_xyz_out);

/* ---- intersection curves (downstream of the path) ------------------------- */
/* The segments of a result chained into polylines (the reference stops at the
 * segment soup of src/CPU/MeshIntersectionCurves.cpp:27-91).  Endpoints are
 * matched by exact equality (they are exact points rounded correctly, so a
 * crossing on a shared mesh edge is bit-identical from both sides); equal
 * edges are merged; zero-length segments become one-vertex curves; chains
 * run through vertices of degree 2 and a chain back to its start is closed.
 * With drop_coplanar_interior, an edge contributed two or more times and only
 * by coplanar overlap triangles (pairs with three segments) is dropped, so a
 * coplanar region is kept as its boundary.  Host code; needs no device. */
typedef struct gi_curves gi_curves;
gi_status gi_curves_build(const double* seg6, const int32_t* seg_pair, uint64_t nsegs, uint64_t npairs,
                          int32_t drop_coplanar_interior, gi_curves** out);
gi_status gi_result_curves(const gi_result* r, int32_t drop_coplanar_interior, gi_curves** out);
gi_status gi_curves_vertices(const gi_curves* c, const double** xyz, uint64_t* n);
/* curve k: vertex ids verts[offsets[k] .. offsets[k+1]), closed[k] = 1 if it closes */
gi_status gi_curves_polylines(const gi_curves* c, const uint64_t** offsets, const uint32_t** verts,
                              const uint8_t** closed, uint64_t* ncurves);
gi_status gi_curves_free(gi_curves* c);
/* The curves of every job of a batch in one call (the flat batch arrays of
 * gi_intersect_batch results): segments seg6[0 .. nsegs) ordered by their
 * pair, seg_pair[s] a batch-wide pair index, job j owning pairs
 * [pair_offsets[j], pair_offsets[j + 1]).  Each job's curves are those
 * gi_curves_build gives for the job alone; the jobs are assembled on host
 * threads and concatenated in job order (vertex ids across the batch), and
 * gi_curves_job_offsets gives each job's range of curves. */
gi_status gi_curves_build_jobs(const double* seg6, const int64_t* seg_pair, uint64_t nsegs,
                               const int64_t* pair_offsets, uint32_t njobs, int32_t drop_coplanar_interior,
                               gi_curves** out);
/* job j: curves [job_curves[j], job_curves[j + 1]) */
gi_status gi_curves_job_offsets(const gi_curves* c, const uint64_t** job_curves, uint64_t* njobs);

/* ---- run records: CSV export and run diffs (tooling around the path) ------ */
/* The reference's IntersectionHistory (src/CPU/IntersectionHistory.h:12-232)
 * keeps per intersecting pair a record of the face ids, the six vertex indices
 * and the eighteen posed coordinates, exports a run to CSV (exportRunToCsv,
 * :114-160) and diffs two runs by (faceA, faceB) (exportDiff, :162-232).  Here
 * a run is its pair list plus the posed meshes (gi_pose_apply of the inputs).
 * Host code; needs no device. */
typedef struct {
    const double* verts_xyz; /* posed vertices, 3 doubles each */
    uint32_t nv;
    const uint32_t* tris;    /* 3 vertex indices per triangle */
    uint32_t nt;
} gi_record_mesh;
/* One row per pair in the given order: [category,]FaceA,FaceB,VA0_Idx..VB2_Idx,
 * A_V0_X..B_V2_Z with every double as %.17g (the reference's setprecision(17)).
 * header: write the header line first (with a DiffCategory column when
 * category is given).  append: append to the file.  nthreads: 0 = all.  Every
 * pair and vertex index is checked before anything is written
 * (GI_ERR_INVALID_ARG). */
gi_status gi_records_write_csv(const char* path, int32_t append, int32_t header, const char* category,
                               const gi_record_mesh* A, const gi_record_mesh* B, const int32_t* pairs_ab, uint64_t n,
                               uint32_t nthreads);
/* Set diff of two pair lists by (faceA, faceB), duplicates merged.  Outputs are
 * sorted by (faceA, faceB) in int order (the reference's std::set order) and
 * need room for n1, n2 and min(n1, n2) pairs. */
gi_status gi_pairs_diff(const int32_t* pairs1, uint64_t n1, const int32_t* pairs2, uint64_t n2, int32_t* only1,
                        uint64_t* n_only1, int32_t* only2, uint64_t* n_only2, int32_t* both, uint64_t* n_both);

/* ---- pose sweep (verification harness around the path) -------------------- */
/* The pose sequence of the reference's seeded sweep (TestSuite::runSuite,
 * src/CPU/TestSuite.cpp:455-505): per step, B's Euler angles (degrees) and
 * translation are its base plus uniform draws in [-max_rot_deg, max_rot_deg]
 * and [-max_trans, max_trans] from std::mt19937(seed), drawn z, y, x for the
 * rotation and then z, y, x for the translation (the order a GCC build of the
 * reference evaluates them in).  A stays at its base pose.  Null bases are
 * zero.  Outputs: 3 doubles per step each.  Host code; needs no device. */
gi_status gi_sweep_poses(uint32_t seed, uint32_t nsteps, double max_rot_deg, double max_trans,
                         const double base_rot_b[3], const double base_trans_b[3], double* rot_b_out,
                         double* trans_b_out);

/* ---- results -------------------------------------------------------------- */
/* pairs_ab: 2 int32 per pair (faceA, faceB); pointer valid until gi_result_free. */
gi_status gi_result_pairs(const gi_result* r, const int32_t** pairs_ab, uint64_t* n);
/* seg6: 6 doubles per segment (p0 xyz, p1 xyz); seg_pair: pair index per segment. */
gi_status gi_result_segments(const gi_result* r, const double** seg6, const int32_t** seg_pair, uint64_t* n);
gi_status gi_result_stats(const gi_result* r, gi_stats* out);
gi_status gi_result_free(gi_result* r);

/* ---- serving: pose-update loop with continuous batching ------------------ */
gi_status gi_server_start(gi_ctx* ctx, const gi_server_opts* opts, gi_server** out);
gi_status gi_server_submit(gi_server* s, const gi_mesh* A, const gi_pose* pose_a, const gi_mesh* B,
                           const gi_pose* pose_b, uint64_t* ticket);
/* GI_OK with *out set when done; GI_ERR_NOT_READY while in flight. */
gi_status gi_server_poll(gi_server* s, uint64_t ticket, gi_result** out);
/* Blocks until the ticket is done (bounded by timeout_ms; GI_ERR_TIMEOUT otherwise). */
gi_status gi_server_wait(gi_server* s, uint64_t ticket, uint32_t timeout_ms, gi_result** out);
gi_status gi_server_stop(gi_server* s);

#ifdef __cplusplus
}
#endif
#endif
