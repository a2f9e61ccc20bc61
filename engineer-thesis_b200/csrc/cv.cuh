// cv.cuh -- declarations of the learned control variate (cv.cu).
#pragma once

#include <cuda_bf16.h>

#include "frw_internal.h"

namespace frw {
namespace cv {

// MLP 16 -> 64 -> 64 -> 1, SiLU.  FP32 master parameters, packed:
constexpr int kIn = 16, kHid = 64;
constexpr int oW1 = 0;                   // [64][16]  (out, in)
constexpr int oB1 = oW1 + kHid * kIn;    // [64]
constexpr int oW2 = oB1 + kHid;          // [64][64]  (out, in)
constexpr int oB2 = oW2 + kHid * kHid;   // [64]
constexpr int oW3 = oB2 + kHid;          // [64]
constexpr int oB3 = oW3 + kHid;          // [1]
constexpr int kParams = oB3 + 1;         // 5313
constexpr int kRowsPerBlock = 64;        // training chunk: 4 warps x 16 rows

// Device copy of the network: FP32 master + BF16 operand copies.
struct Net {
    float *p = nullptr;          // [kParams] master
    __nv_bfloat16 *w1 = nullptr; // [64][16]
    __nv_bfloat16 *w2 = nullptr; // [64][64]
    __nv_bfloat16 *w2t = nullptr;// [64][64] transposed (in, out)
};

frw_status net_alloc(Net *n, cudaStream_t st);
// Releases the parameters in the order of `st` (after work queued there).
void net_free(Net *n, cudaStream_t st);
frw_status net_upload(Net *n, const float *host_params, cudaStream_t st);
frw_status net_refresh_bf16(const Net &n, cudaStream_t st);

// features of points p (first-hop points) w.r.t. a target rect: the
// (dx, dy) from p to the nearest point of each edge of the target and of
// the nearest other conductor, divided by a0 and clamped to [-16, 16].
frw_status launch_features(const DevLayout &L, double4 target_rect, int target_id, const double4 *rec,
                           int64_t n, __nv_bfloat16 *xb, float *xf, cudaStream_t st);
// The MLP kernels: tcgen05 / TMEM tiles of 128 rows (cv_umma.cu, the
// default) or mma.sync tiles of 16 rows (cv.cu); frw_mlp_set_kernels picks.
// status: device word, kStDeviceWait set when a tcgen05 completion wait
// passed its bound.
int mlp_kernels();
frw_status set_mlp_kernels(int which);
frw_status launch_forward(const Net &n, const __nv_bfloat16 *x, int64_t rows, float *out, uint32_t *status,
                          cudaStream_t st);
// grad += d/dparams sum_r wt_r (f(x_r) - y_r)^2 * inv_wsum ; loss += same sum
frw_status launch_train_grad(const Net &n, const __nv_bfloat16 *x, const float *y, const float *wt, int64_t rows,
                             float inv_wsum, float *grad, double *loss, uint32_t *status, cudaStream_t st);
frw_status launch_forward_tc(const Net &n, const __nv_bfloat16 *x, int64_t rows, float *out, uint32_t *status,
                             int sms, cudaStream_t st);
// tcgen05 training step: each CTA writes its partial gradient to its slot of
// part ([train_blocks_tc(rows, sms)][kPartStride] floats); launch_reduce_adam_tc
// then sums the slots in CTA order and applies Adam at step t (1-based), or
// launch_reduce_sum_tc adds them to a gradient.
constexpr int kPartStride = (kParams + 3) & ~3;  // floats per CTA slot: 16-byte aligned slots
int train_blocks_tc(int64_t rows, int sms);
frw_status launch_train_grad_tc(const Net &n, const __nv_bfloat16 *x, const float *y, const float *wt, int64_t rows,
                                float inv_wsum, float *part, double *loss, uint32_t *status, int sms,
                                cudaStream_t st);
frw_status launch_reduce_adam_tc(const Net &n, const float *part, int nb, float *m, float *v, int t, float lr,
                                 cudaStream_t st);
frw_status launch_reduce_sum_tc(const float *part, int nb, float *grad, cudaStream_t st);
int device_sm_count();
frw_status launch_adam(const Net &n, float *grad, float *m, float *v, int *step, float lr, cudaStream_t st);
// exact mean E[f] over every (grid start, first-hop bin) pair, accumulated into *sum
frw_status launch_quad_mean(const DevLayout &L, double4 target_rect, int target_id, const double4 *gauss, uint32_t Q,
                            const double *pi_exact, const double *wx, const double *wy, double eps,
                            bool exact_perimeter, const Net &net, double *sum,
                            float *phi_out /*nullable: Q*200 phi values, item q*200+i*/, uint32_t *status,
                            cudaStream_t st);
frw_status launch_quad_mean_tc(const DevLayout &L, double4 trect, int tid, const double4 *gauss, const double4 *sqs,
                               const int *sides, uint32_t Q, const double *pi_exact, const double *wx,
                               const double *wy, double eps, bool exact, const Net &net, double *sum, float *phi_out,
                               uint32_t *status, int sms, cudaStream_t st);
// per walk record (end, weight factor c, q*200+i1 or -1): the sums of
// z = c (1{end==target} - phi), z^2, w = c 1{end==target}, w^2 with phi looked
// up in the quadrature's table
frw_status launch_cv_gather(const int64_t *end, const double *cw, const int32_t *qi, const float *phi, int64_t n,
                            int target, double *sums /*4*/, cudaStream_t st);
frw_status launch_targets(const int64_t *end, const double4 *rec, int64_t n, int target, float *y, float *wt,
                          double *wsum, cudaStream_t st);

}  // namespace cv
}  // namespace frw
