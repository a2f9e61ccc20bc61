// query.cu -- batched collision queries and the Gaussian-surface kernel.
#include "query.cuh"

namespace frw {
namespace {

// One point per thread: drawBiggestSquareAtPoint + checkCollisons(point),
// batched (the reference issues them one walk hop at a time,
// Cuda/randomwalk.cu:102-103).  kTies: L.tree_points is set, so points with
// many exact ties can reach the whole-tree replay (compiled out otherwise).
template <bool kTies>
__global__ void __launch_bounds__(128) k_query(DevLayout L, const double2 *__restrict__ pts, int64_t n,
                                               double4 *__restrict__ sq, int64_t *__restrict__ hit,
                                               uint32_t *status) {
    int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
    uint32_t st = 0;
    if (i < n) {
        const double2 p = pts[i];
        double s[4];
        int h;
        st = query_point<false, false, kTies>(L, p.x, p.y, s, h);
        sq[i] = make_double4(s[0], s[1], s[2], s[3]);
        hit[i] = h == kNoHit ? -1 : (int64_t)h;
    }
    if (st) atomicOr(status, st);
}

__global__ void __launch_bounds__(128) k_box(DevLayout L, const double4 *__restrict__ boxes, int64_t n,
                                             bool has_ign, double4 ign, uint8_t *__restrict__ out,
                                             uint32_t *status) {
    int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
    uint32_t st = 0;
    if (i < n) {
        const double4 b = boxes[i];
        const double B[4] = {b.x, b.y, b.z, b.w};
        const double I[4] = {ign.x, ign.y, ign.z, ign.w};
        out[i] = box_collides(L, B, has_ign, I, st) ? 1 : 0;
    }
    if (st) atomicOr(status, st);
}

// RectHost::createGaussianSurface (CPU/rectHost.cpp:84-100).
__device__ void scale_rect(const double r[4], double fx, double fy, double o[4]) {
    const double mx = __dmul_rn(__dadd_rn(r[0], r[2]), 0.5);
    const double my = __dmul_rn(__dadd_rn(r[1], r[3]), 0.5);
    const double vx = __dmul_rn(__dsub_rn(r[0], mx), fx);
    const double vy = __dmul_rn(__dsub_rn(r[1], my), fy);
    o[0] = __dadd_rn(mx, vx);
    o[1] = __dadd_rn(my, vy);
    o[2] = __dsub_rn(mx, vx);
    o[3] = __dsub_rn(my, vy);
}

// Tree::getAdjustedGaussianFactor (CPU/quadTree.cpp:315-349): bisection of
// the per-axis scale factor against collisions that ignore the target.
__device__ double adjusted_factor(const DevLayout &L, const double r[4], double factor, bool axis_y,
                                  uint32_t &st) {
    bool dividing = true, first = true;
    double adj = factor, lb = 1.0, rb = factor, s[4];
    for (int i = 0; i < 10; i++) {  // GAUSSIAN_ACCURACY
        if (axis_y) scale_rect(r, 1.0, adj, s);
        else scale_rect(r, adj, 1.0, s);
        const bool isc = box_collides(L, s, true, r, st);
        if (first && !isc) break;
        if ((isc && !dividing) || (!isc && dividing)) dividing = !dividing;
        const double mid = __dmul_rn(__dadd_rn(lb, rb), 0.5);
        if (dividing) adj = rb = mid;
        else adj = lb = mid;
        first = false;
    }
    return adj;
}

// creatGaussianSurfFrom (scale mode) or the target grown by `param`.
__device__ void gauss_one(const DevLayout &L, const double4 t, int mode, double param, double o[4], uint32_t &st) {
    const double r[4] = {t.x, t.y, t.z, t.w};
    if (mode == FRW_GAUSS_SCALE) {
        if (param < 1.0) {  // creatGaussianSurfFrom returns the rect itself
            o[0] = r[0]; o[1] = r[1]; o[2] = r[2]; o[3] = r[3];
        } else {
            const double fx = adjusted_factor(L, r, param, false, st);
            const double fy = adjusted_factor(L, r, param, true, st);
            scale_rect(r, fx, fy, o);
        }
    } else {
        o[0] = __dsub_rn(r[0], param);
        o[1] = __dsub_rn(r[1], param);
        o[2] = __dadd_rn(r[2], param);
        o[3] = __dadd_rn(r[3], param);
    }
}

__global__ void k_gauss(DevLayout L, const double4 *__restrict__ targets, int n, int mode, double param,
                        double4 *__restrict__ out, uint32_t *status) {
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= n) return;
    double o[4];
    uint32_t st = 0;
    gauss_one(L, targets[i], mode, param, o, st);
    out[i] = make_double4(o[0], o[1], o[2], o[3]);
    if (st) atomicOr(status, st);
}

// One job per thread, each on its own layout (batched runs).
__global__ void k_gauss_jobs(const WalkJob *__restrict__ jobs, const double4 *__restrict__ targets, int n, int mode,
                             double param, double4 *__restrict__ out, uint32_t *status) {
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= n) return;
    double o[4];
    uint32_t st = 0;
    gauss_one(jobs[i].L, targets[i], mode, param, o, st);
    out[i] = make_double4(o[0], o[1], o[2], o[3]);
    if (st) atomicOr(status, st);
}

}  // namespace

frw_status launch_gauss_jobs(const WalkJob *d_jobs, const double *d_targets, int njobs, int mode, double param,
                             double *d_out, uint32_t *d_status, cudaStream_t stream) {
    if (njobs <= 0) return FRW_OK;
    k_gauss_jobs<<<(njobs + 63) / 64, 64, 0, stream>>>(d_jobs, (const double4 *)d_targets, njobs, mode, param,
                                                      (double4 *)d_out, d_status);
    FRW_CK(cudaGetLastError());
    return FRW_OK;
}

frw_status launch_query(const DevLayout &L, const double *d_pts, int64_t n, double *d_sq, int64_t *d_hit,
                        uint32_t *d_status, cudaStream_t stream) {
    if (n <= 0) return FRW_OK;
    const int T = 128;
    const unsigned g = (unsigned)((n + T - 1) / T);
    if (L.tree_points)
        k_query<true><<<g, T, 0, stream>>>(L, (const double2 *)d_pts, n, (double4 *)d_sq, d_hit, d_status);
    else
        k_query<false><<<g, T, 0, stream>>>(L, (const double2 *)d_pts, n, (double4 *)d_sq, d_hit, d_status);
    FRW_CK(cudaGetLastError());
    return FRW_OK;
}

frw_status launch_box_collides(const DevLayout &L, const double *d_boxes, int64_t n, bool has_ignore,
                               const double ignore[4], uint8_t *d_out, uint32_t *d_status,
                               cudaStream_t stream) {
    if (n <= 0) return FRW_OK;
    const int T = 128;
    double4 ig = has_ignore ? make_double4(ignore[0], ignore[1], ignore[2], ignore[3])
                            : make_double4(0, 0, 0, 0);
    k_box<<<(unsigned)((n + T - 1) / T), T, 0, stream>>>(L, (const double4 *)d_boxes, n, has_ignore, ig,
                                                         d_out, d_status);
    FRW_CK(cudaGetLastError());
    return FRW_OK;
}

frw_status launch_gauss(const DevLayout &L, const double *d_targets, int n, int mode, double param,
                        double *d_out, uint32_t *d_status, cudaStream_t stream) {
    if (n <= 0) return FRW_OK;
    k_gauss<<<(n + 63) / 64, 64, 0, stream>>>(L, (const double4 *)d_targets, n, mode, param,
                                              (double4 *)d_out, d_status);
    FRW_CK(cudaGetLastError());
    return FRW_OK;
}

}  // namespace frw
