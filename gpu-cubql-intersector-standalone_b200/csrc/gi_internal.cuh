// gi_internal.cuh -- device-side data layout shared by the kernels of libgi.
//
// HBM layout of one resident mesh (built once by gi_mesh_upload):
//   verts     double[3*nv]            input vertices (mesh-local frame)
//   tris      uint32[3*nt]            input triangles (original order)
//   leafTri   uint4[nt]               per Morton-sorted leaf: v0, v1, v2, original id
//   leafBox   float[6*nt]             per sorted leaf: FP32 box rounded outward
//   nodes     WNode[nnodes]           4-wide BVH, 128 B per node (one cache line)
//   leafBox64 / nodes64               FP64 copies for the plain-FP64 form (built lazily)
// Traversal runs in the world frame: node boxes are mapped through the pose on
// the fly (conservatively), so a new pose needs no rebuild or refit.
#pragma once
#include <cstdint>
#include <cuda_runtime.h>

namespace gi {

constexpr uint32_t kLeaf = 0x80000000u;   // child ref: sorted leaf position
constexpr uint32_t kEmpty = 0xFFFFFFFFu;  // unused child slot

// 4-wide BVH node: child boxes in SoA so that lane i of a quad reads child i.
struct __align__(128) WNode {
    float lox[4], loy[4], loz[4], hix[4], hiy[4], hiz[4];
    uint32_t child[4];
    uint32_t pad[4];
};
static_assert(sizeof(WNode) == 128, "WNode is one 128-byte line");

struct __align__(256) WNode64 {
    double lox[4], loy[4], loz[4], hix[4], hiy[4], hiz[4];
    uint32_t child[4];
    uint32_t pad[12];
};
static_assert(sizeof(WNode64) == 256, "WNode64 is two 128-byte lines");

// Pose on the device.
//  exact vertex map: world = ((R*(v - C)) + C) + T in FP64, left to right, no FMA
//  box map (FP32):  world = Rf*v + bf, padded by rho*(|Rf|(|c|+h) + padm)
struct DevPose {
    double R[9], C[3], T[3];
    double b64[3];     // C + T - R*C (FP64), for FP64 node boxes
    double padm64[3];  // |C| + |T| + |R||C| (FP64), magnitude term of the pad
    float Rf[9], bf[3], padm[3];
    int identity;
    // world -> local (inverse) map for a near-orthonormal R: local = Ri*w + bi
    // with Ri = R^T; inv_ok = 0 when R is not orthonormal within 2^-30
    int inv_ok;
    double inv_eta;    // max |R^T R - I| entry: error of R^T as the inverse
    double Ri64[9], bi64[3], padmi64[3];
    float Rif[9], bif[3], padmi[3];
    int pad_[3];
};

struct MeshDev {
    const double* verts;
    const uint32_t* tris;
    const uint4* leafTri;
    const float* leafBox;
    const double* leafBox64;
    const WNode* nodes;
    const WNode64* nodes64;
    // cuts: node / leaf refs whose subtrees cover all leaves, the depth-3 cut in
    // entries [0, kCutMax) and the depth-4 cut in [kCutMax, kCutMax + kCut4Max)
    const uint32_t* cutRef;
    const float* cutBox;     // their boxes (6 floats each)
    const double* cutBox64;  // FP64 boxes of the same cuts (FP64 form)
    uint32_t root;  // wide node index, or kLeaf | leaf position when nt == 1
    uint32_t nv, nt, nnodes;
    const uint32_t* ncuts;  // device: entries of the depth-3 and the depth-4 cut (null for an empty mesh)
};

constexpr int kCutMax = 64;    // 4^3
constexpr int kCut4Max = 256;  // 4^4
constexpr int kCutCap = kCutMax + kCut4Max;

struct JobDev {
    MeshDev A, B;
    DevPose pa, pb;
};

constexpr int kLevelTimes = 32;  // levels whose end times are recorded

// Device counters of one intersect launch sequence (zeroed by the host).
struct Counters {
    // hot counters, each on its own 128-byte line (polled and updated by every warp)
    unsigned int q_tail;  // node-pair queue: slots reserved (pushed)
    unsigned int pad0[31];
    unsigned int q_head;  // queue slots handed out as tickets
    unsigned int pad1[31];
    // low half: node pairs that exist (made, not yet expanded; never below
    // zero); high half: candidate slots reserved.  One word, so that an
    // expansion reserves its candidate slots and updates the node-pair count
    // in one atomic, and a warp that reads the node-pair count at zero reads
    // the final candidate count in the same load.
    unsigned long long work_cand;
    unsigned int pad2[30];
    unsigned int pad3[32];
    unsigned int c_head;  // candidate slots handed out as tickets
    unsigned int pad4[31];
    unsigned int res;     // intersecting pairs
    unsigned int esc;     // escalated candidate indices
    unsigned int overflow;  // kOvf* bits
    unsigned int err;       // kErr* bits
    unsigned int abort_;    // set on overflow or a spent wait: every waiting warp stops
    unsigned int levels;    // deepest node-pair level + 1
    unsigned int nseg;      // total segments after ordering
    unsigned int obar;      // grid barrier of the small-count ordering kernel
    unsigned int order_redo;  // small-count ordering refused (too many results): rerun on the radix path
    unsigned int seed_head;  // seed tests claimed (chunks of 32)
    unsigned int seed_done;  // seed tests finished and published
    unsigned int pad5;
    unsigned long long node_pairs;
    unsigned long long filter_decided;
    unsigned long long exact_signs;
    unsigned long long exact_points;
    unsigned long long tested;  // candidates run through the first filter stage
    // level-synchronous traversal: per level slot (level % 3), node pairs made
    // (low half) and leaf pairs made (high half) during that level
    unsigned pad6[16];
    unsigned long long lvl[3];
    unsigned pad7[26];
    unsigned bar_count;  // grid barrier: blocks arrived
    unsigned pad8[31];
    unsigned bar_gen;    // grid barrier: barriers completed
    unsigned bstop;      // decision of the last completed barrier: 1 = the traversal is over (kept for the host)
    unsigned cand_total; // candidates made by the completed levels (written by the barriers' last arrivers)
    unsigned pad9[29];
    unsigned cand_ready; // candidates published to the candidate blocks (all written)
    unsigned cand_final; // 1: no candidate will be published after cand_ready
    unsigned pad10[30];
    unsigned long long t_start;                 // globaltimer at the launch's start (ns)
    unsigned long long level_ns[kLevelTimes];   // globaltimer when level l ended (its barrier completed)
    // post-traversal launch (k_finish): globaltimer at its start, after the exact
    // stage, when the last block ended its key phase, after the count scan's
    // release, and when its last block ended
    unsigned long long fin_ns[5];
    // level-synchronous traversal: the last completed barrier's level counts
    // (lvl of the finished level) and stop decision, read by each block in one load
    alignas(16) unsigned long long bpub[2];
    unsigned fin_done;  // blocks of k_finish that have ended
    unsigned pad11[31];
    unsigned fbar;      // k_finish: blocks arrived at the barrier after its key phase
    unsigned pad12[31];
    unsigned frel;      // k_finish: the last block's release (1), or its refusal (2)
    unsigned fin_over;  // k_finish: keys put on the overflow list (may exceed its capacity)
    unsigned pad13[30];
};

constexpr unsigned kOvfFrontier = 1u, kOvfCand = 2u, kOvfRes = 4u, kOvfEsc = 8u;
constexpr unsigned kErrTimeout = 1u, kErrExactCapacity = 2u;
// Counters::order_redo: the small-count ordering or the one-launch finish
// refused; kRedoCrowded: the finish found a key partition over its limit
constexpr unsigned kRedoCount = 1u, kRedoCrowded = 2u;

// Per-call buffers handed to the kernels.
struct Bufs {
    const JobDev* jobs;
    uint32_t njobs;
    uint4* queue;     // node pairs: job, node/leaf ref A, node/leaf ref B, level
    unsigned* qflag;  // per queue slot: tag of the call that published it
    uint32_t cap_queue;
    uint4* cand;      // job, leaf posA, leaf posB, 0
    unsigned* cflag;  // per candidate slot: publishing tag
    uint32_t cap_cand;
    uint4* res;       // job, triA, triB, 0   (original triangle ids)
    uint32_t cap_res;
    uint4* esc;       // escalated candidates: job, leaf posA, leaf posB, 0
    uint32_t cap_esc;
    Counters* cnt;
    unsigned tag;     // nonzero, different for every call on the context
    int precision;    // 0 FP32 cascade, 1 FP64
    int two_frame;    // also test child boxes in B's own frame (fewer pairs, more work per pair)
    int deep_seed;    // seed from the depth-4 cuts (single-pair calls) instead of the depth-3 cuts
    unsigned quad_below;  // level-synchronous traversal: levels of at most this many node pairs use the quad form
    unsigned cand_blocks; // level-synchronous traversal: blocks that only filter candidates
    unsigned publish;     // level-synchronous traversal: 1 = each level's candidates are published to the
                          // candidate blocks (0: they are filtered by every warp in the next level)
};

}  // namespace gi
