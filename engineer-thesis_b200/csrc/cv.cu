// cv.cu -- learned control variate for the capacitance estimator.
//
// Per walk the estimator of C_tt is w = c * 1{end = t}, with c the first-hop
// weight factor (walk.cu).  The control variate is f = c * phi(x1): phi is a
// small MLP (16 -> 64 -> 64 -> 1, SiLU) of the geometry seen from the
// first-hop point x1, trained so that phi(x1) ~ P(walk from x1 ends on t).
// The estimate  mean(w - f) + E[f]  is unbiased because E[f] is computed
// EXACTLY: with the grid start (Q equal arcs, Q a power of two) the pair
// (start point, first-hop bin) takes finitely many values with known
// probabilities (1/Q times the exact bin probability of the 32-bit uniform),
// so E[f] is a finite sum over Q x 200 first-hop points.  The same pass keeps
// phi of every one of those points in a table: a walk's first-hop point is a
// function of its (arc, bin), so the walks look their phi up instead of
// recomputing features and the MLP, and f is exactly the function whose mean
// was summed.
//
// Kernels: feature extraction (the nearest other conductor from the cell
// list, or one tree traversal), BF16 tensor-core MLP forward (mma.sync
// m16n8k16, FP32 accumulate, the first layer's accumulators re-packed in
// registers as the second layer's A operand), the fused exact-mean pass,
// fused forward+backward with weight gradients as tensor-core products over
// 64-row chunks, Adam, and FP64 reductions.
#include <cuda_bf16.h>

#include <atomic>

#include "cv.cuh"
#include "cv_feat.cuh"
#include "query.cuh"

namespace frw {
namespace cv {
namespace {

constexpr unsigned kFull = 0xFFFFFFFFu;

__global__ void k_features(DevLayout L, double4 trect, int tid, const double4 *__restrict__ rec, int64_t n,
                           __nv_bfloat16 *__restrict__ xb, float *__restrict__ xf) {
    const int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= n) return;
    const double4 r = rec[i];
    float f[16];
    if (r.z > 0.0) {
        edge_feats(r.x, r.y, trect.x, trect.y, trect.z, trect.w, r.z, f);
        float4 o;
        if (nearest_other(L, r.x, r.y, tid, o)) {
            edge_feats(r.x, r.y, o.x, o.y, o.z, o.w, r.z, f + 8);
        } else {
#pragma unroll
            for (int q = 8; q < 16; q++) f[q] = 16.f;
        }
    } else {
#pragma unroll
        for (int q = 0; q < 16; q++) f[q] = 0.f;
    }
    if (xb) {
        __nv_bfloat162 *o = reinterpret_cast<__nv_bfloat162 *>(xb + 16 * i);
#pragma unroll
        for (int q = 0; q < 8; q++) o[q] = __floats2bfloat162_rn(f[2 * q], f[2 * q + 1]);
    }
    if (xf)
#pragma unroll
        for (int q = 0; q < 16; q++) xf[16 * i + q] = f[q];
}

// ---------------------------------------------------------------- MLP core
__device__ __forceinline__ uint32_t pack2(float lo, float hi) {
    __nv_bfloat162 v = __floats2bfloat162_rn(lo, hi);
    return *reinterpret_cast<uint32_t *>(&v);
}

__device__ __forceinline__ uint32_t pack_h(__nv_bfloat16 lo, __nv_bfloat16 hi) {
    __nv_bfloat162 v;
    v.x = lo;
    v.y = hi;
    return *reinterpret_cast<uint32_t *>(&v);
}

// D += A(16x16, row) * B(16x8, col): BF16 inputs, FP32 accumulators.
__device__ __forceinline__ void mma16816(float d[4], const uint32_t a[4], uint32_t b0, uint32_t b1) {
    asm volatile(
        "mma.sync.aligned.m16n8k16.row.col.f32.bf16.bf16.f32 {%0,%1,%2,%3}, {%4,%5,%6,%7}, {%8,%9}, "
        "{%0,%1,%2,%3};\n"
        : "+f"(d[0]), "+f"(d[1]), "+f"(d[2]), "+f"(d[3])
        : "r"(a[0]), "r"(a[1]), "r"(a[2]), "r"(a[3]), "r"(b0), "r"(b1));
}

// sigmoid(z) = (1 + tanh(z/2)) / 2 with the hardware tanh (one MUFU op,
// relative error about 2^-11, below the BF16 rounding of the activations);
// training and evaluation use the same function, so the control variate
// stays exactly the function whose mean is summed.
__device__ __forceinline__ float tanh_hw(float x) {
    float y;
    asm("tanh.approx.f32 %0, %1;" : "=f"(y) : "f"(x));
    return y;
}
__device__ __forceinline__ float sigm(float z) { return 0.5f + 0.5f * tanh_hw(0.5f * z); }
__device__ __forceinline__ float silu(float z) { return z * sigm(z); }
__device__ __forceinline__ float dsilu(float z) {
    const float s = sigm(z);
    return s * (1.f + z * (1.f - s));
}

struct Smem {
    __nv_bfloat16 w1[kHid * kIn];
    __nv_bfloat16 w2[kHid * kHid];
    float b1[kHid], b2[kHid], w3[kHid];
    float b3;
};

__device__ __forceinline__ void load_net(Smem &S, const float *p, const __nv_bfloat16 *w1,
                                         const __nv_bfloat16 *w2) {
    for (int i = threadIdx.x; i < kHid * kIn; i += blockDim.x) S.w1[i] = w1[i];
    for (int i = threadIdx.x; i < kHid * kHid; i += blockDim.x) S.w2[i] = w2[i];
    for (int i = threadIdx.x; i < kHid; i += blockDim.x) {
        S.b1[i] = p[oB1 + i];
        S.b2[i] = p[oB2 + i];
        S.w3[i] = p[oW3 + i];
    }
    if (threadIdx.x == 0) S.b3 = p[oB3];
}

// Forward of one 16-row tile held by a warp.  xa: A fragment of X.
// Leaves z1, z2 (pre-activations, C layout), h1 as A fragments, and the
// outputs of rows g and g+8.
__device__ __forceinline__ void tile_forward(const Smem &S, const uint32_t xa[4], int g, int tg, float z1[8][4],
                                             float z2[8][4], uint32_t a2[4][4], float &out_g, float &out_g8) {
    const uint32_t *w1u = reinterpret_cast<const uint32_t *>(S.w1);
    const uint32_t *w2u = reinterpret_cast<const uint32_t *>(S.w2);
#pragma unroll
    for (int nt = 0; nt < 8; nt++) {
        const int j = nt * 8 + 2 * tg;
        z1[nt][0] = S.b1[j];
        z1[nt][1] = S.b1[j + 1];
        z1[nt][2] = S.b1[j];
        z1[nt][3] = S.b1[j + 1];
        const int row = nt * 8 + g;  // output feature of W1 (the n index)
        mma16816(z1[nt], xa, w1u[(row * kIn + 2 * tg) >> 1], w1u[(row * kIn + 2 * tg + 8) >> 1]);
    }
#pragma unroll
    for (int ks = 0; ks < 4; ks++) {
        a2[ks][0] = pack2(silu(z1[2 * ks][0]), silu(z1[2 * ks][1]));
        a2[ks][1] = pack2(silu(z1[2 * ks][2]), silu(z1[2 * ks][3]));
        a2[ks][2] = pack2(silu(z1[2 * ks + 1][0]), silu(z1[2 * ks + 1][1]));
        a2[ks][3] = pack2(silu(z1[2 * ks + 1][2]), silu(z1[2 * ks + 1][3]));
    }
    float pg = 0.f, pg8 = 0.f;
#pragma unroll
    for (int nt = 0; nt < 8; nt++) {
        const int j = nt * 8 + 2 * tg;
        z2[nt][0] = S.b2[j];
        z2[nt][1] = S.b2[j + 1];
        z2[nt][2] = S.b2[j];
        z2[nt][3] = S.b2[j + 1];
        const int row = nt * 8 + g;
#pragma unroll
        for (int ks = 0; ks < 4; ks++)
            mma16816(z2[nt], a2[ks], w2u[(row * kHid + 16 * ks + 2 * tg) >> 1],
                     w2u[(row * kHid + 16 * ks + 8 + 2 * tg) >> 1]);
        pg += silu(z2[nt][0]) * S.w3[j] + silu(z2[nt][1]) * S.w3[j + 1];
        pg8 += silu(z2[nt][2]) * S.w3[j] + silu(z2[nt][3]) * S.w3[j + 1];
    }
    pg += __shfl_xor_sync(kFull, pg, 1);
    pg += __shfl_xor_sync(kFull, pg, 2);
    pg8 += __shfl_xor_sync(kFull, pg8, 1);
    pg8 += __shfl_xor_sync(kFull, pg8, 2);
    out_g = pg + S.b3;
    out_g8 = pg8 + S.b3;
}

__device__ __forceinline__ void load_x_frag(const __nv_bfloat16 *x, int64_t r0, int64_t rows, int g, int tg,
                                            uint32_t xa[4]) {
    const uint32_t *xu = reinterpret_cast<const uint32_t *>(x);
    const int64_t ra = r0 + g, rb = r0 + g + 8;
    xa[0] = ra < rows ? xu[(ra * kIn + 2 * tg) >> 1] : 0u;
    xa[1] = rb < rows ? xu[(rb * kIn + 2 * tg) >> 1] : 0u;
    xa[2] = ra < rows ? xu[(ra * kIn + 2 * tg + 8) >> 1] : 0u;
    xa[3] = rb < rows ? xu[(rb * kIn + 2 * tg + 8) >> 1] : 0u;
}

__global__ void __launch_bounds__(128) k_forward(const float *__restrict__ p, const __nv_bfloat16 *__restrict__ w1,
                                                 const __nv_bfloat16 *__restrict__ w2,
                                                 const __nv_bfloat16 *__restrict__ x, int64_t rows,
                                                 float *__restrict__ out) {
    __shared__ Smem S;
    load_net(S, p, w1, w2);
    __syncthreads();
    const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5, g = lane >> 2, tg = lane & 3;
    const int64_t tiles = (rows + 15) / 16;
    for (int64_t t = (int64_t)blockIdx.x * 4 + warp; t < tiles; t += (int64_t)gridDim.x * 4) {
        uint32_t xa[4];
        load_x_frag(x, t * 16, rows, g, tg, xa);
        float z1[8][4], z2[8][4], og, og8;
        uint32_t a2[4][4];
        tile_forward(S, xa, g, tg, z1, z2, a2, og, og8);
        if (tg == 0) {
            if (t * 16 + g < rows) out[t * 16 + g] = og;
            if (t * 16 + g + 8 < rows) out[t * 16 + g + 8] = og8;
        }
    }
}

// Column sums over the 16 rows of a C-layout tile: v[nt][0..3] for the
// thread's columns; after the shuffles lanes 0..3 hold the sums.
__device__ __forceinline__ void col_sums(float v[8][2]) {
#pragma unroll
    for (int nt = 0; nt < 8; nt++)
#pragma unroll
        for (int e = 0; e < 2; e++) {
            float s = v[nt][e];
            s += __shfl_xor_sync(kFull, s, 4);
            s += __shfl_xor_sync(kFull, s, 8);
            s += __shfl_xor_sync(kFull, s, 16);
            v[nt][e] = s;
        }
}

struct TrainSmem {
    Smem net;
    __nv_bfloat16 w2t[kHid * kHid];
    __nv_bfloat16 h1[kRowsPerBlock * kHid];   // silu(z1), bf16
    __nv_bfloat16 dz2[kRowsPerBlock * kHid];
    __nv_bfloat16 dz1[kRowsPerBlock * kHid];
    __nv_bfloat16 xs[kRowsPerBlock * kIn];
    float db1[kHid], db2[kHid], dw3[kHid];
    float db3;
    double loss;
};

// Fused forward + backward over 64-row chunks (4 warps x 16 rows); weight
// gradients dW2 = dZ2^T H1 and dW1 = dZ1^T X are tensor-core products over
// the chunk's rows, split by output block across the warps and kept in
// registers across chunks; bias gradients by shuffle reductions.
__global__ void __launch_bounds__(128) k_train_grad(const float *__restrict__ p, const __nv_bfloat16 *__restrict__ w1,
                                                    const __nv_bfloat16 *__restrict__ w2,
                                                    const __nv_bfloat16 *__restrict__ w2t,
                                                    const __nv_bfloat16 *__restrict__ x,
                                                    const float *__restrict__ y, const float *__restrict__ wt,
                                                    int64_t rows, float inv_wsum, float *__restrict__ grad,
                                                    double *__restrict__ loss_out) {
    __shared__ TrainSmem S;
    load_net(S.net, p, w1, w2);
    for (int i = threadIdx.x; i < kHid * kHid; i += blockDim.x) S.w2t[i] = w2t[i];
    for (int i = threadIdx.x; i < kHid; i += blockDim.x) S.db1[i] = S.db2[i] = S.dw3[i] = 0.f;
    if (threadIdx.x == 0) {
        S.db3 = 0.f;
        S.loss = 0.0;
    }
    __syncthreads();
    const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5, g = lane >> 2, tg = lane & 3;
    const uint32_t *w2tu = reinterpret_cast<const uint32_t *>(S.w2t);
    float accW2[8][4], accW1[2][4];
#pragma unroll
    for (int nt = 0; nt < 8; nt++) accW2[nt][0] = accW2[nt][1] = accW2[nt][2] = accW2[nt][3] = 0.f;
#pragma unroll
    for (int nt = 0; nt < 2; nt++) accW1[nt][0] = accW1[nt][1] = accW1[nt][2] = accW1[nt][3] = 0.f;
    float db3 = 0.f;
    double lsum = 0.0;
    const int64_t chunks = (rows + kRowsPerBlock - 1) / kRowsPerBlock;
    for (int64_t ch = blockIdx.x; ch < chunks; ch += gridDim.x) {
        const int64_t r0 = ch * kRowsPerBlock + warp * 16;
        const int lr0 = warp * 16;  // local row base in the chunk staging
        uint32_t xa[4];
        load_x_frag(x, r0, rows, g, tg, xa);
        float z1[8][4], z2[8][4], og, og8;
        uint32_t a2[4][4];
        tile_forward(S.net, xa, g, tg, z1, z2, a2, og, og8);
        // dL/dout for rows g, g+8
        const int64_t ra = r0 + g, rb = r0 + g + 8;
        const float wa = ra < rows ? wt[ra] : 0.f, wb = rb < rows ? wt[rb] : 0.f;
        const float ea = ra < rows ? og - y[ra] : 0.f, eb = rb < rows ? og8 - y[rb] : 0.f;
        const float da = 2.f * wa * ea * inv_wsum, db = 2.f * wb * eb * inv_wsum;
        if (tg == 0) {
            lsum += (double)wa * ea * ea * inv_wsum + (double)wb * eb * eb * inv_wsum;
            db3 += da + db;
        }
        // stage X and H1 (bf16) for the weight-gradient products
        {
            const uint32_t *xu = reinterpret_cast<const uint32_t *>(S.xs);
            uint32_t *xsu = reinterpret_cast<uint32_t *>(S.xs);
            (void)xu;
            xsu[((lr0 + g) * kIn + 2 * tg) >> 1] = xa[0];
            xsu[((lr0 + g + 8) * kIn + 2 * tg) >> 1] = xa[1];
            xsu[((lr0 + g) * kIn + 2 * tg + 8) >> 1] = xa[2];
            xsu[((lr0 + g + 8) * kIn + 2 * tg + 8) >> 1] = xa[3];
            uint32_t *h1u = reinterpret_cast<uint32_t *>(S.h1);
#pragma unroll
            for (int ks = 0; ks < 4; ks++) {
                h1u[((lr0 + g) * kHid + 16 * ks + 2 * tg) >> 1] = a2[ks][0];
                h1u[((lr0 + g + 8) * kHid + 16 * ks + 2 * tg) >> 1] = a2[ks][1];
                h1u[((lr0 + g) * kHid + 16 * ks + 8 + 2 * tg) >> 1] = a2[ks][2];
                h1u[((lr0 + g + 8) * kHid + 16 * ks + 8 + 2 * tg) >> 1] = a2[ks][3];
            }
        }
        // dZ2 = dout * w3 * silu'(z2); dw3 and db2 partial sums
        float cs_w3[8][2], cs_b2[8][2];
        uint32_t ad[4][4];  // dZ2 as A fragments (for dH1 = dZ2 W2)
#pragma unroll
        for (int nt = 0; nt < 8; nt++) {
            const int j = nt * 8 + 2 * tg;
            const float d0 = da * S.net.w3[j] * dsilu(z2[nt][0]);
            const float d1 = da * S.net.w3[j + 1] * dsilu(z2[nt][1]);
            const float d2 = db * S.net.w3[j] * dsilu(z2[nt][2]);
            const float d3 = db * S.net.w3[j + 1] * dsilu(z2[nt][3]);
            cs_w3[nt][0] = da * silu(z2[nt][0]) + db * silu(z2[nt][2]);
            cs_w3[nt][1] = da * silu(z2[nt][1]) + db * silu(z2[nt][3]);
            cs_b2[nt][0] = d0 + d2;
            cs_b2[nt][1] = d1 + d3;
            z2[nt][0] = d0;  // reuse as dZ2
            z2[nt][1] = d1;
            z2[nt][2] = d2;
            z2[nt][3] = d3;
        }
#pragma unroll
        for (int ks = 0; ks < 4; ks++) {
            ad[ks][0] = pack2(z2[2 * ks][0], z2[2 * ks][1]);
            ad[ks][1] = pack2(z2[2 * ks][2], z2[2 * ks][3]);
            ad[ks][2] = pack2(z2[2 * ks + 1][0], z2[2 * ks + 1][1]);
            ad[ks][3] = pack2(z2[2 * ks + 1][2], z2[2 * ks + 1][3]);
            uint32_t *du = reinterpret_cast<uint32_t *>(S.dz2);
            du[((lr0 + g) * kHid + 16 * ks + 2 * tg) >> 1] = ad[ks][0];
            du[((lr0 + g + 8) * kHid + 16 * ks + 2 * tg) >> 1] = ad[ks][1];
            du[((lr0 + g) * kHid + 16 * ks + 8 + 2 * tg) >> 1] = ad[ks][2];
            du[((lr0 + g + 8) * kHid + 16 * ks + 8 + 2 * tg) >> 1] = ad[ks][3];
        }
        col_sums(cs_w3);
        col_sums(cs_b2);
        if (g == 0) {
#pragma unroll
            for (int nt = 0; nt < 8; nt++) {
                const int j = nt * 8 + 2 * tg;
                atomicAdd(&S.dw3[j], cs_w3[nt][0]);
                atomicAdd(&S.dw3[j + 1], cs_w3[nt][1]);
                atomicAdd(&S.db2[j], cs_b2[nt][0]);
                atomicAdd(&S.db2[j + 1], cs_b2[nt][1]);
            }
        }
        // dH1 = dZ2 W2  (B(k=j, n=i) = W2[j][i] = W2T[i][j]); dZ1 = dH1 * silu'(z1)
        float cs_b1[8][2];
#pragma unroll
        for (int nt = 0; nt < 8; nt++) {
            float dh[4] = {0.f, 0.f, 0.f, 0.f};
            const int row = nt * 8 + g;  // i (input feature of W2)
#pragma unroll
            for (int ks = 0; ks < 4; ks++)
                mma16816(dh, ad[ks], w2tu[(row * kHid + 16 * ks + 2 * tg) >> 1],
                         w2tu[(row * kHid + 16 * ks + 8 + 2 * tg) >> 1]);
            dh[0] *= dsilu(z1[nt][0]);
            dh[1] *= dsilu(z1[nt][1]);
            dh[2] *= dsilu(z1[nt][2]);
            dh[3] *= dsilu(z1[nt][3]);
            cs_b1[nt][0] = dh[0] + dh[2];
            cs_b1[nt][1] = dh[1] + dh[3];
            z1[nt][0] = dh[0];
            z1[nt][1] = dh[1];
            z1[nt][2] = dh[2];
            z1[nt][3] = dh[3];
        }
        {
            uint32_t *du = reinterpret_cast<uint32_t *>(S.dz1);
#pragma unroll
            for (int ks = 0; ks < 4; ks++) {
                du[((lr0 + g) * kHid + 16 * ks + 2 * tg) >> 1] = pack2(z1[2 * ks][0], z1[2 * ks][1]);
                du[((lr0 + g + 8) * kHid + 16 * ks + 2 * tg) >> 1] = pack2(z1[2 * ks][2], z1[2 * ks][3]);
                du[((lr0 + g) * kHid + 16 * ks + 8 + 2 * tg) >> 1] = pack2(z1[2 * ks + 1][0], z1[2 * ks + 1][1]);
                du[((lr0 + g + 8) * kHid + 16 * ks + 8 + 2 * tg) >> 1] = pack2(z1[2 * ks + 1][2], z1[2 * ks + 1][3]);
            }
        }
        col_sums(cs_b1);
        if (g == 0) {
#pragma unroll
            for (int nt = 0; nt < 8; nt++) {
                const int j = nt * 8 + 2 * tg;
                atomicAdd(&S.db1[j], cs_b1[nt][0]);
                atomicAdd(&S.db1[j + 1], cs_b1[nt][1]);
            }
        }
        __syncthreads();
        // weight gradients over the 64 staged rows; warp w owns output rows
        // j = 16w .. 16w+15.  A(m=j, k=r) = dZ[r][j] (transposed gather).
        const int jb = 16 * warp;
#pragma unroll
        for (int ks = 0; ks < 4; ks++) {
            const int rA = 16 * ks + 2 * tg;
            uint32_t a[4];
            a[0] = pack_h(S.dz2[rA * kHid + jb + g], S.dz2[(rA + 1) * kHid + jb + g]);
            a[1] = pack_h(S.dz2[rA * kHid + jb + g + 8], S.dz2[(rA + 1) * kHid + jb + g + 8]);
            a[2] = pack_h(S.dz2[(rA + 8) * kHid + jb + g], S.dz2[(rA + 9) * kHid + jb + g]);
            a[3] = pack_h(S.dz2[(rA + 8) * kHid + jb + g + 8], S.dz2[(rA + 9) * kHid + jb + g + 8]);
#pragma unroll
            for (int nt = 0; nt < 8; nt++) {
                const int i = 8 * nt + g;
                const uint32_t b0 = pack_h(S.h1[rA * kHid + i], S.h1[(rA + 1) * kHid + i]);
                const uint32_t b1 = pack_h(S.h1[(rA + 8) * kHid + i], S.h1[(rA + 9) * kHid + i]);
                mma16816(accW2[nt], a, b0, b1);
            }
            uint32_t c[4];
            c[0] = pack_h(S.dz1[rA * kHid + jb + g], S.dz1[(rA + 1) * kHid + jb + g]);
            c[1] = pack_h(S.dz1[rA * kHid + jb + g + 8], S.dz1[(rA + 1) * kHid + jb + g + 8]);
            c[2] = pack_h(S.dz1[(rA + 8) * kHid + jb + g], S.dz1[(rA + 9) * kHid + jb + g]);
            c[3] = pack_h(S.dz1[(rA + 8) * kHid + jb + g + 8], S.dz1[(rA + 9) * kHid + jb + g + 8]);
#pragma unroll
            for (int nt = 0; nt < 2; nt++) {
                const int f = 8 * nt + g;
                const uint32_t b0 = pack_h(S.xs[rA * kIn + f], S.xs[(rA + 1) * kIn + f]);
                const uint32_t b1 = pack_h(S.xs[(rA + 8) * kIn + f], S.xs[(rA + 9) * kIn + f]);
                mma16816(accW1[nt], c, b0, b1);
            }
        }
        __syncthreads();
    }
    // flush: each element of this block's gradient once
    const int jb = 16 * warp;
#pragma unroll
    for (int nt = 0; nt < 8; nt++) {
        const int i = 8 * nt + 2 * tg;
        atomicAdd(&grad[oW2 + (jb + g) * kHid + i], accW2[nt][0]);
        atomicAdd(&grad[oW2 + (jb + g) * kHid + i + 1], accW2[nt][1]);
        atomicAdd(&grad[oW2 + (jb + g + 8) * kHid + i], accW2[nt][2]);
        atomicAdd(&grad[oW2 + (jb + g + 8) * kHid + i + 1], accW2[nt][3]);
    }
#pragma unroll
    for (int nt = 0; nt < 2; nt++) {
        const int f = 8 * nt + 2 * tg;
        atomicAdd(&grad[oW1 + (jb + g) * kIn + f], accW1[nt][0]);
        atomicAdd(&grad[oW1 + (jb + g) * kIn + f + 1], accW1[nt][1]);
        atomicAdd(&grad[oW1 + (jb + g + 8) * kIn + f], accW1[nt][2]);
        atomicAdd(&grad[oW1 + (jb + g + 8) * kIn + f + 1], accW1[nt][3]);
    }
    if (tg == 0) {
        atomicAdd(&S.db3, db3);
        atomicAdd(&S.loss, lsum);
    }
    __syncthreads();
    for (int i = threadIdx.x; i < kHid; i += blockDim.x) {
        atomicAdd(&grad[oB1 + i], S.db1[i]);
        atomicAdd(&grad[oB2 + i], S.db2[i]);
        atomicAdd(&grad[oW3 + i], S.dw3[i]);
    }
    if (threadIdx.x == 0) {
        atomicAdd(&grad[oB3], S.db3);
        atomicAdd(loss_out, S.loss);
    }
}

// Adam on the FP32 master copy; refreshes the BF16 operand copies and
// clears the gradient.  The step counter lives on the device so a captured
// training loop replays correctly.
__global__ void k_adam(float *__restrict__ p, float *__restrict__ grad, float *__restrict__ m, float *__restrict__ v,
                       int *step, float lr, __nv_bfloat16 *__restrict__ w1, __nv_bfloat16 *__restrict__ w2,
                       __nv_bfloat16 *__restrict__ w2t) {
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    const int t = *step + 1;
    if (i < kParams) {
        const float b1 = 0.9f, b2 = 0.999f;
        const float gi = grad[i];
        const float mi = b1 * m[i] + (1.f - b1) * gi;
        const float vi = b2 * v[i] + (1.f - b2) * gi * gi;
        m[i] = mi;
        v[i] = vi;
        const float mh = mi / (1.f - powf(b1, (float)t)), vh = vi / (1.f - powf(b2, (float)t));
        const float pi = p[i] - lr * mh / (sqrtf(vh) + 1e-8f);
        p[i] = pi;
        grad[i] = 0.f;
        if (i < oB1) w1[i] = __float2bfloat16_rn(pi);
        else if (i >= oW2 && i < oB2) {
            const int k = i - oW2;
            w2[k] = __float2bfloat16_rn(pi);
            w2t[(k % kHid) * kHid + k / kHid] = __float2bfloat16_rn(pi);
        }
    }
}

__global__ void k_step_inc(int *step) { *step += 1; }

__global__ void k_refresh(const float *__restrict__ p, __nv_bfloat16 *__restrict__ w1, __nv_bfloat16 *__restrict__ w2,
                          __nv_bfloat16 *__restrict__ w2t) {
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i < oB1) w1[i] = __float2bfloat16_rn(p[i]);
    else if (i >= oW2 && i < oB2) {
        const int k = i - oW2;
        w2[k] = __float2bfloat16_rn(p[i]);
        w2t[(k % kHid) * kHid + k / kHid] = __float2bfloat16_rn(p[i]);
    }
}

// ---------------------------------------------------------------- reductions
__device__ __forceinline__ double warp_sum(double v) {
#pragma unroll
    for (int o = 16; o; o >>= 1) v += __shfl_xor_sync(kFull, v, o);
    return v;
}

// Training pairs from walk records: y = 1{end == target}, weight c^2.
__global__ void k_targets(const int64_t *__restrict__ end, const double4 *__restrict__ rec, int64_t n, int target,
                          float *__restrict__ y, float *__restrict__ wt, double *wsum) {
    double s = 0.0;
    for (int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; i < n; i += (int64_t)gridDim.x * blockDim.x) {
        const double c = rec[i].w;
        const float w = (float)(c * c);
        y[i] = end[i] == target ? 1.f : 0.f;
        wt[i] = w;
        s += (double)w;
    }
    s = warp_sum(s);
    if ((threadIdx.x & 31) == 0) atomicAdd(wsum, s);
}

// Start point q of the grid, its first square and first-hop outcome.
__global__ void k_quad_starts(DevLayout L, const double4 *__restrict__ gauss, uint32_t Q,
                              double4 *__restrict__ sq_out, int *__restrict__ side_out) {
    const uint32_t q = blockIdx.x * blockDim.x + threadIdx.x;
    if (q >= Q) return;
    const double4 g4 = gauss[0];
    const double G[4] = {g4.x, g4.y, g4.z, g4.w};
    const double u = __ddiv_rn(__dadd_rn((double)q, 0.5), (double)Q);
    double px, py;
    const int side = perimeter_point(G, u, px, py);
    int code = side;
    double sq[4] = {0, 0, 0, 0};
    if (!(px > L.bx0 && py > L.by0 && px < L.bx1 && py < L.by1)) {
        code = -1;  // escapes before the first hop
    } else {
        int hit;
        query_point(L, px, py, sq, hit);
        if (hit != kNoHit) code = -1;  // ends before the first hop
    }
    sq_out[q] = make_double4(sq[0], sq[1], sq[2], sq[3]);
    side_out[q] = code;
}

// Exact mean of f over every (grid start q, first-hop bin i): per item the
// first-hop point x1, its probability weight c * pi_i / Q, the features and
// phi(x1) on the tensor cores, summed in FP64.  Fused, so nothing of size
// Q x 200 is stored: each warp takes 32 items, stages their BF16 features
// in shared memory and runs them as two 16-row MMA tiles.
__global__ void __launch_bounds__(128) k_quad_mean(DevLayout L, double4 trect, int tid, const double4 *__restrict__ gauss,
                                                   const double4 *__restrict__ sqs, const int *__restrict__ sides,
                                                   uint32_t Q, const double *__restrict__ pi_exact,
                                                   const double *__restrict__ wx, const double *__restrict__ wy,
                                                   double eps, bool exact, const float *__restrict__ p,
                                                   const __nv_bfloat16 *__restrict__ w1,
                                                   const __nv_bfloat16 *__restrict__ w2, double *sum,
                                                   float *__restrict__ phi_out) {
    __shared__ Smem S;
    __shared__ uint32_t xs[4][32][kIn / 2];
    load_net(S, p, w1, w2);
    __syncthreads();
    const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5, g = lane >> 2, tg = lane & 3;
    const int64_t n = (int64_t)Q * FRW_NSAMPLE;
    const double4 g4 = gauss[0];
    const double perim = __dadd_rn(__dmul_rn(2.0, __dsub_rn(g4.z, g4.x)), __dmul_rn(2.0, __dsub_rn(g4.w, g4.y)));
    double acc = 0.0;
    for (int64_t b = ((int64_t)blockIdx.x * 4 + warp) * 32; b < n; b += (int64_t)gridDim.x * 128) {
        const int64_t t = b + lane;
        double wgt = 0.0;
        float f[kIn];
#pragma unroll
        for (int k = 0; k < kIn; k++) f[k] = 0.f;
        const int side = t < n ? sides[t / FRW_NSAMPLE] : -1;
        if (side >= 0) {
            const int i = (int)(t % FRW_NSAMPLE);
            const double4 s4 = sqs[t / FRW_NSAMPLE];
            const double sq[4] = {s4.x, s4.y, s4.z, s4.w};
            double x1, y1;
            point_from_index(sq, i, exact, x1, y1);
            const double a0 = __dsub_rn(sq[2], sq[0]);
            const double nx = side == 1 ? 1.0 : (side == 3 ? -1.0 : 0.0);
            const double ny = side == 2 ? 1.0 : (side == 0 ? -1.0 : 0.0);
            const double dot = __dadd_rn(__dmul_rn(wx[i], nx), __dmul_rn(wy[i], ny));
            const double c = __ddiv_rn(__dmul_rn(__dmul_rn(-eps, perim), dot), a0);
            wgt = c * pi_exact[i] / (double)Q;
            edge_feats(x1, y1, trect.x, trect.y, trect.z, trect.w, a0, f);
            float4 o;
            if (nearest_other(L, x1, y1, tid, o)) {
                edge_feats(x1, y1, o.x, o.y, o.z, o.w, a0, f + 8);
            } else {
#pragma unroll
                for (int q = 8; q < kIn; q++) f[q] = 16.f;
            }
        }
#pragma unroll
        for (int k = 0; k < kIn / 2; k++) xs[warp][lane][k] = pack2(f[2 * k], f[2 * k + 1]);
        __syncwarp();
        float mine = 0.f;
        const int row = lane & 15, src = 4 * (row & 7);
#pragma unroll
        for (int h = 0; h < 2; h++) {
            const int ra = 16 * h + g, rb = ra + 8;
            const uint32_t xa[4] = {xs[warp][ra][tg], xs[warp][rb][tg], xs[warp][ra][tg + 4], xs[warp][rb][tg + 4]};
            float z1[8][4], z2[8][4], og, og8;
            uint32_t a2[4][4];
            tile_forward(S, xa, g, tg, z1, z2, a2, og, og8);
            const double wa = __shfl_sync(kFull, wgt, ra), wb = __shfl_sync(kFull, wgt, rb);
            if (tg == 0) acc += wa * (double)og + wb * (double)og8;
            const float lo = __shfl_sync(kFull, og, src), hi = __shfl_sync(kFull, og8, src);
            if ((lane >> 4) == h) mine = row < 8 ? lo : hi;
        }
        if (phi_out && t < n) phi_out[t] = mine;  // the table the walks look phi up in
        __syncwarp();
    }
    acc = warp_sum(acc);
    if (lane == 0) atomicAdd(sum, acc);
}

// Per walk record of the grid start: f = c * phi[q * 200 + i1] from the
// quadrature's table (the same function value the exact mean sums), and the
// sums of z = c (1{end==t} - phi), z^2, w = c 1{end==t}, w^2.
__global__ void k_cv_gather(const int64_t *__restrict__ end, const double *__restrict__ cw,
                            const int32_t *__restrict__ qi, const float *__restrict__ phi, int64_t n, int target,
                            double *sums) {
    double s[4] = {0, 0, 0, 0};
    for (int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; i < n; i += (int64_t)gridDim.x * blockDim.x) {
        const double c = cw[i];
        const int32_t k = qi[i];
        const double yv = end[i] == target ? 1.0 : 0.0;
        const double f = k >= 0 ? (double)__ldg(phi + k) : 0.0;
        const double z = c * (yv - f);
        const double w = c * yv;
        s[0] += z;
        s[1] += z * z;
        s[2] += w;
        s[3] += w * w;
    }
#pragma unroll
    for (int k = 0; k < 4; k++) {
        const double t = warp_sum(s[k]);
        if ((threadIdx.x & 31) == 0) atomicAdd(&sums[k], t);
    }
}

}  // namespace

frw_status net_alloc(Net *n, cudaStream_t st) {
    FRW_CK(cudaMallocAsync((void **)&n->p, kParams * sizeof(float), st));
    FRW_CK(cudaMallocAsync((void **)&n->w1, kHid * kIn * 2, st));
    FRW_CK(cudaMallocAsync((void **)&n->w2, kHid * kHid * 2, st));
    FRW_CK(cudaMallocAsync((void **)&n->w2t, kHid * kHid * 2, st));
    return FRW_OK;
}

void net_free(Net *n, cudaStream_t st) {
    for (void *q : {(void *)n->p, (void *)n->w1, (void *)n->w2, (void *)n->w2t})
        if (q) cudaFreeAsync(q, st);
    *n = Net();
}

frw_status net_refresh_bf16(const Net &n, cudaStream_t st) {
    k_refresh<<<(kParams + 255) / 256, 256, 0, st>>>(n.p, n.w1, n.w2, n.w2t);
    FRW_CK(cudaGetLastError());
    return FRW_OK;
}

frw_status net_upload(Net *n, const float *host, cudaStream_t st) {
    FRW_CK(cudaMemcpyAsync(n->p, host, kParams * sizeof(float), cudaMemcpyHostToDevice, st));
    return net_refresh_bf16(*n, st);
}

frw_status launch_features(const DevLayout &L, double4 trect, int tid, const double4 *rec, int64_t n,
                           __nv_bfloat16 *xb, float *xf, cudaStream_t st) {
    if (n <= 0) return FRW_OK;
    k_features<<<(unsigned)((n + 127) / 128), 128, 0, st>>>(L, trect, tid, rec, n, xb, xf);
    FRW_CK(cudaGetLastError());
    return FRW_OK;
}

namespace {
std::atomic<int> g_mlp_kernels{FRW_MLP_TCGEN05};

int device_sms() {
    int dev = 0, sms = 0;
    cudaGetDevice(&dev);
    cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev);
    return sms > 0 ? sms : 1;
}
}  // namespace

int mlp_kernels() { return g_mlp_kernels.load(std::memory_order_relaxed); }

int device_sm_count() { return device_sms(); }

frw_status set_mlp_kernels(int which) {
    if (which != FRW_MLP_TCGEN05 && which != FRW_MLP_MMA_SYNC) {
        set_error("frw_mlp_set_kernels: FRW_MLP_TCGEN05 or FRW_MLP_MMA_SYNC");
        return FRW_E_ARG;
    }
    g_mlp_kernels.store(which, std::memory_order_relaxed);
    return FRW_OK;
}

frw_status launch_forward(const Net &n, const __nv_bfloat16 *x, int64_t rows, float *out, uint32_t *status,
                          cudaStream_t st) {
    if (rows <= 0) return FRW_OK;
    if (mlp_kernels() == FRW_MLP_TCGEN05) return launch_forward_tc(n, x, rows, out, status, device_sms(), st);
    const int64_t tiles = (rows + 15) / 16;
    const int blocks = (int)std::min<int64_t>((tiles + 3) / 4, 148 * 8);
    k_forward<<<blocks, 128, 0, st>>>(n.p, n.w1, n.w2, x, rows, out);
    FRW_CK(cudaGetLastError());
    return FRW_OK;
}

frw_status launch_train_grad(const Net &n, const __nv_bfloat16 *x, const float *y, const float *wt, int64_t rows,
                             float inv_wsum, float *grad, double *loss, uint32_t *status, cudaStream_t st) {
    if (rows <= 0) return FRW_OK;
    if (mlp_kernels() == FRW_MLP_TCGEN05) {  // partial sums per CTA, then added to grad
        const int sms = device_sms(), nb = train_blocks_tc(rows, sms);
        float *part = nullptr;
        FRW_CK(cudaMallocAsync(&part, (size_t)nb * kPartStride * sizeof(float), st));
        frw_status rc = launch_train_grad_tc(n, x, y, wt, rows, inv_wsum, part, loss, status, sms, st);
        if (!rc) rc = launch_reduce_sum_tc(part, nb, grad, st);
        cudaFreeAsync(part, st);
        return rc;
    }
    const int64_t chunks = (rows + kRowsPerBlock - 1) / kRowsPerBlock;
    const int blocks = (int)std::min<int64_t>(chunks, 148 * 2);
    k_train_grad<<<blocks, 128, 0, st>>>(n.p, n.w1, n.w2, n.w2t, x, y, wt, rows, inv_wsum, grad, loss);
    FRW_CK(cudaGetLastError());
    return FRW_OK;
}

frw_status launch_adam(const Net &n, float *grad, float *m, float *v, int *step, float lr, cudaStream_t st) {
    k_adam<<<(kParams + 255) / 256, 256, 0, st>>>(n.p, grad, m, v, step, lr, n.w1, n.w2, n.w2t);
    k_step_inc<<<1, 1, 0, st>>>(step);
    FRW_CK(cudaGetLastError());
    return FRW_OK;
}

frw_status launch_cv_gather(const int64_t *end, const double *cw, const int32_t *qi, const float *phi, int64_t n,
                            int target, double *sums, cudaStream_t st) {
    if (n <= 0) return FRW_OK;
    const int blocks = (int)std::min<int64_t>((n + 255) / 256, 148 * 8);
    k_cv_gather<<<blocks, 256, 0, st>>>(end, cw, qi, phi, n, target, sums);
    FRW_CK(cudaGetLastError());
    return FRW_OK;
}

frw_status launch_targets(const int64_t *end, const double4 *rec, int64_t n, int target, float *y, float *wt,
                          double *wsum, cudaStream_t st) {
    if (n <= 0) return FRW_OK;
    const int blocks = (int)std::min<int64_t>((n + 255) / 256, 148 * 8);
    k_targets<<<blocks, 256, 0, st>>>(end, rec, n, target, y, wt, wsum);
    FRW_CK(cudaGetLastError());
    return FRW_OK;
}


frw_status launch_quad_mean(const DevLayout &L, double4 trect, int tid, const double4 *gauss, uint32_t Q,
                            const double *pi_exact, const double *wx, const double *wy, double eps, bool exact,
                            const Net &net, double *sum, float *phi_out, uint32_t *status, cudaStream_t st) {
    double4 *sqs;
    int *sides;
    FRW_CK(cudaMallocAsync((void **)&sqs, (size_t)Q * sizeof(double4), st));
    FRW_CK(cudaMallocAsync((void **)&sides, (size_t)Q * sizeof(int), st));
    k_quad_starts<<<(Q + 127) / 128, 128, 0, st>>>(L, gauss, Q, sqs, sides);
    const int64_t n = (int64_t)Q * FRW_NSAMPLE;
    frw_status rc = FRW_OK;
    if (mlp_kernels() == FRW_MLP_TCGEN05) {
        rc = launch_quad_mean_tc(L, trect, tid, gauss, sqs, sides, Q, pi_exact, wx, wy, eps, exact, net, sum, phi_out,
                                 status, device_sms(), st);
    } else {
        const int blocks = (int)std::min<int64_t>((n + 127) / 128, 148 * 8);
        k_quad_mean<<<blocks, 128, 0, st>>>(L, trect, tid, gauss, sqs, sides, Q, pi_exact, wx, wy, eps, exact,
                                            net.p, net.w1, net.w2, sum, phi_out);
    }
    cudaError_t e = rc ? cudaSuccess : cudaGetLastError();
    cudaFreeAsync(sqs, st);
    cudaFreeAsync(sides, st);
    if (rc) return rc;
    FRW_CK(e);
    return FRW_OK;
}

}  // namespace cv
}  // namespace frw
