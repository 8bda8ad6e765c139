// gi_signs.cu -- the device's orientation predicates on caller-given points.
//
// Every decision of the intersection path comes down to orient3d / orient2d
// signs.  The reference computes them in FP32 and FP64 interval arithmetic
// (src/GPU_exact_predicates/GPUPredicatesCommon.h:38-100,
//  src/GPU_exact_predicates/DoublePredicate.cu:75-93) and in 384-bit integers
// on pre-rounded coordinates (src/GPU_exact_predicates/ExactBigIntPredicate.cu:
// 194-212 orient3d_exact_V2, :381-489 classifyPairBigIntV2).  This file runs
// the same device functions that the traversal's filter and the exact stage
// call (gi_classify.cuh, gi_exact.cuh) on a list of point sets and returns
// every stage's answer per query, so that each sign can be compared with an
// exact rational evaluation:
//   [0] FP32 semi-static filter, line-order form (filt_o3<float>)
//   [1] FP32 semi-static filter, vertex-versus-plane form (filt_dot<float>)
//   [2] FP64 semi-static filter, line-order form (filt_o3<double>)
//   [3] FP64 semi-static filter, vertex-versus-plane form (filt_dot<double>)
//   [4] FP64 filter in front of the exact stage (o3_filter64 / o2_filter64)
//   [5] exact integer sign, computed whatever the filters say
//   [6] the exact stage's sign (filter, then integers when it is unsure)
//   [7] integer branch of [5]: 0 int128, 1 multi-limb, 2 capacity exceeded
// Filters answer +1, 0 or -1 when they decide and GI_SIGN_UNDECIDED (2) when
// they do not; orient2d has no FP32 or semi-static form (GI_SIGN_NA, 3).
#include "gi_classify.cuh"
#include "gi_host.h"

namespace gi {

constexpr int kSignRecord = 8;
static_assert(GI_SIGN_UNDECIDED == kUnsure, "undecided code of the header and the filters");

__device__ __forceinline__ int8_t filt_code(int s)
{
    return (int8_t)(s == kUnsure ? GI_SIGN_UNDECIDED : s);
}

__global__ void __launch_bounds__(128) k_pred_signs(int kind, const double* __restrict__ pts,
                                                    const int32_t* __restrict__ drop, uint64_t n,
                                                    int8_t* __restrict__ out, unsigned* __restrict__ err)
{
    for (uint64_t i = blockIdx.x * (uint64_t)blockDim.x + threadIdx.x; i < n; i += (uint64_t)gridDim.x * blockDim.x) {
        int8_t* o = out + kSignRecord * i;
        int path = ex::kPathCapacity;
        if (kind == GI_PRED_ORIENT3D) {
            const double* p = pts + 12 * i;
            const double3 a = make_double3(p[0], p[1], p[2]), b = make_double3(p[3], p[4], p[5]);
            const double3 c = make_double3(p[6], p[7], p[8]), d = make_double3(p[9], p[10], p[11]);
            o[0] = filt_code(filt_o3<float>(a, b, c, d));
            // orient3d(a, b, c, d) = (a - d) . ((b - a) x (c - a)): the form of the
            // first filter stage's vertex-versus-plane signs
            o[1] = filt_code(filt_dot<float>(make_plane<float>(vdiff<float>(b, a), vdiff<float>(c, a)), vdiff<float>(a, d)));
            o[2] = filt_code(filt_o3<double>(a, b, c, d));
            o[3] = filt_code(filt_dot<double>(make_plane<double>(vdiff<double>(b, a), vdiff<double>(c, a)),
                                              vdiff<double>(a, d)));
            o[4] = filt_code(o3_filter64(a, b, c, d));
            o[5] = (int8_t)ex::o3_exact_sign(&a.x, &b.x, &c.x, &d.x, err, &path);
            ExactSigns S{err, 0ull};
            o[6] = (int8_t)S.o3(a, b, c, d);
        } else {
            const double* p = pts + 9 * i;
            const double3 a = make_double3(p[0], p[1], p[2]), b = make_double3(p[3], p[4], p[5]);
            const double3 c = make_double3(p[6], p[7], p[8]);
            const int dr = drop[i];
            o[0] = o[1] = o[2] = o[3] = (int8_t)GI_SIGN_NA;
            o[4] = filt_code(o2_filter64(a, b, c, dr));
            o[5] = (int8_t)ex::o2_exact_sign(&a.x, &b.x, &c.x, dr, err, &path);
            ExactSigns S{err, 0ull};
            o[6] = (int8_t)S.o2(a, b, c, dr);
        }
        o[7] = (int8_t)path;
    }
}

static bool coord_ok(double x)
{
    const double ax = fabs(x);
    return ax == 0.0 || (ax >= 0x1p-100 && ax <= 0x1p100);
}

}  // namespace gi

using namespace gi;

extern "C" gi_status gi_predicate_signs(gi_ctx* c, int32_t kind, const double* pts, const int32_t* drop, uint64_t n,
                                        int8_t* out)
{
    if (!c || (kind != GI_PRED_ORIENT3D && kind != GI_PRED_ORIENT2D)) return GI_ERR_INVALID_ARG;
    if (n == 0) return GI_OK;
    if (!pts || !out || (kind == GI_PRED_ORIENT2D && !drop)) return GI_ERR_INVALID_ARG;
    if (n > ((uint64_t)1 << 26)) return set_err(c, GI_ERR_CAPACITY, "at most 2^26 queries per call");
    const size_t per = kind == GI_PRED_ORIENT3D ? 12 : 9;
    for (size_t k = 0; k < per * n; k++)
        if (!coord_ok(pts[k])) return set_err(c, GI_ERR_RANGE, "coordinate outside the supported domain");
    if (kind == GI_PRED_ORIENT2D)
        for (uint64_t i = 0; i < n; i++)
            if (drop[i] < 0 || drop[i] > 2) return set_err(c, GI_ERR_INVALID_ARG, "drop axis outside 0..2");
    std::lock_guard<std::mutex> lk(c->mu);
    CK(c, cudaSetDevice(c->device), "set device");
    const size_t pb = sizeof(double) * per * n, db = kind == GI_PRED_ORIENT2D ? sizeof(int32_t) * n : 0;
    const size_t ob = (size_t)kSignRecord * n;
    char* buf = nullptr;
    const size_t off_d = (pb + 255) & ~(size_t)255, off_o = (off_d + db + 255) & ~(size_t)255;
    const size_t off_e = (off_o + ob + 255) & ~(size_t)255;
    CK(c, pool_alloc(&buf, off_e + 256, c->pool, c->st), "predicate signs buffers");
    double* d_pts = reinterpret_cast<double*>(buf);
    int32_t* d_drop = db ? reinterpret_cast<int32_t*>(buf + off_d) : nullptr;
    int8_t* d_out = reinterpret_cast<int8_t*>(buf + off_o);
    unsigned* d_err = reinterpret_cast<unsigned*>(buf + off_e);
    unsigned h_err = 0;
    cudaError_t e = cudaMemcpyAsync(d_pts, pts, pb, cudaMemcpyHostToDevice, c->st);
    if (e == cudaSuccess && db) e = cudaMemcpyAsync(d_drop, drop, db, cudaMemcpyHostToDevice, c->st);
    if (e == cudaSuccess) e = cudaMemsetAsync(d_err, 0, sizeof(unsigned), c->st);
    if (e == cudaSuccess) {
        const uint64_t want = (n + 127) / 128, cap = (uint64_t)c->cfg.sms * 16;
        k_pred_signs<<<(unsigned)(want < cap ? want : cap), 128, 0, c->st>>>(kind, d_pts, d_drop, n, d_out, d_err);
        note_launches(1);
        e = cudaGetLastError();
    }
    if (e == cudaSuccess) e = cudaMemcpyAsync(out, d_out, ob, cudaMemcpyDeviceToHost, c->st);
    if (e == cudaSuccess) e = cudaMemcpyAsync(&h_err, d_err, sizeof(unsigned), cudaMemcpyDeviceToHost, c->st);
    cudaFreeAsync(buf, c->st);
    if (e == cudaSuccess) e = cudaStreamSynchronize(c->st);
    if (e != cudaSuccess) return set_err(c, GI_ERR_CUDA, "predicate signs", e);
    if (h_err & kErrExactCapacity) return set_err(c, GI_ERR_RANGE, "exact arithmetic capacity exceeded");
    return GI_OK;
}
