// cv_umma.cu -- the control variate's MLP (16 -> 64 -> 64 -> 1, SiLU) on the
// fifth-generation tensor cores: tcgen05.mma with BF16 operands in shared
// memory and FP32 accumulators in tensor memory (TMEM), issued by one thread
// of the CTA, completion signalled through an mbarrier, results read back
// with tcgen05.ld.  One CTA of 128 threads owns a 128-row tile at a time;
// thread t owns row t (TMEM lane t).
//
// Operand layout.  Every shared-memory operand is a grid of 8 x 8 BF16 core
// matrices (128 contiguous bytes each, no swizzle).  A [128 rows x 8G
// columns] buffer stores element (r, n) at
//     (n / 8) * 2048 + (r / 8) * 128 + (r % 8) * 16 + (n % 8) * 2,
// so the same bytes serve as a K-major operand with the rows as M (K-chunk
// stride 2048, M-group stride 128) and as an MN-major operand with the rows
// as K (K-group stride 128, MN-group stride 2048).  That lets the training
// step feed its activations to the forward products (rows = M) and to the
// weight-gradient products (rows = K) without a transpose:
//     Z1  = X  W1^T          [128 x 64]   (A = X K-major,  B = W1)
//     Z2  = H1 W2^T          [128 x 64]   (A = H1 K-major, B = W2)
//     dH1 = dZ2 W2           [128 x 64]   (A = dZ2 K-major, B = W2^T)
//     [dW2 | . | db2 ; . | dW1 | db1] = [dZ2 ; dZ1]^T [H1 | X | 1]   [128 x 96]
//     [dw3 ; db3] = [H2 ; 1]^T [dz3]                                [128 x 16]
// the last two accumulating in TMEM over every tile the CTA handles, so the
// weight and bias gradients (all of them) come out of the tensor cores.
// TMEM columns: Z1 0..63, Z2 / dH1 64..127, dW 128..223, dw3 224..239.
//
// No counterpart in the reference, which has no learned part (it discards
// the Green-function gradients, CPU/getAvgPathLen.cpp:83-84).
#include <cuda_bf16.h>

#include "cv.cuh"
#include "cv_feat.cuh"

namespace frw {
namespace cv {
namespace {

constexpr int kThreads = 128;
constexpr uint32_t kGrp = 2048;  // bytes of one 8-column group of a 128-row buffer
// shared memory map (bytes from the 1024-aligned base)
constexpr uint32_t kXH = 0;                    // 12 groups: h1 (0-7), x (8-9), ones (10), zeros (11)
constexpr uint32_t kDZ = kXH + 12 * kGrp;      // 16 groups: dz2 (0-7), dz1 (8-15)
constexpr uint32_t kH2 = kDZ + 16 * kGrp;      // 16 groups: h2 (0-7), ones (8), zeros (9-15)
constexpr uint32_t kB3 = kH2 + 16 * kGrp;      // 2 groups: (dz3, 1, 0 ...) (0), zeros (1)
// Where the weights, the FP32 vectors, the mbarrier and the reduction slot
// sit, and how much shared memory and TMEM a CTA takes.  Training: after the
// four operand buffers, 111 KB and 256 TMEM columns, so at most two CTAs per
// SM (three would exceed the SM's 228 KB) and their TMEM (2 x 256) fits the
// SM's 512 columns -- tcgen05.alloc never waits for another CTA.  Forward
// passes: XH (groups 0-9) and the forward weights only, 31 KB used, 46 KB
// reserved so that at most four CTAs share an SM, each with 128 columns (Z1,
// Z2).
struct TrainMap {
    static constexpr uint32_t W1 = kB3 + 2 * kGrp;  // W1 as B (K = 16 inputs, N = 64 outputs)
    static constexpr uint32_t W2 = W1 + 2048;       // W2 as B (K = 64 inputs, N = 64 outputs)
    static constexpr uint32_t W2T = W2 + 8192;      // W2^T as B (K = 64 outputs, N = 64 inputs)
    static constexpr uint32_t Par = W2T + 8192;     // b1[64] b2[64] w3[64] b3 (floats)
    static constexpr uint32_t Bar = Par + 1024;     // mbarrier (8 B), TMEM base (4 B)
    static constexpr uint32_t Red = Bar + 64;       // block reductions: loss (double)
    static constexpr uint32_t Smem = Red + 64;
    static constexpr uint32_t TmemCols = 256;
    static constexpr int PerSm = 2;
};
struct FwdMap {
    static constexpr uint32_t W1 = 10 * kGrp;
    static constexpr uint32_t W2 = W1 + 2048;
    static constexpr uint32_t W2T = W2;  // not loaded
    static constexpr uint32_t Par = W2 + 8192;
    static constexpr uint32_t Bar = Par + 1024;
    static constexpr uint32_t Red = Bar + 64;
    static constexpr uint32_t Smem = 46 * 1024;
    static constexpr uint32_t TmemCols = 128;
    static constexpr int PerSm = 4;
};
template <class M>
constexpr bool residency_ok() {  // (PerSm + 1) CTAs exceed the SM's shared memory, PerSm fit, TMEM fits
    return (M::PerSm + 1) * (M::Smem + 1024) > 228 * 1024 && M::PerSm * (M::Smem + 1024) <= 228 * 1024 &&
           M::PerSm * M::TmemCols <= 512 && M::Red + 64 <= M::Smem;
}
static_assert(residency_ok<TrainMap>() && residency_ok<FwdMap>(), "CTA residency and TMEM budget");

constexpr long long kWaitCycles = 2000000000ll;  // ~1 s at 2 GHz: bound of every mbarrier wait

__device__ __forceinline__ uint32_t su32(const void *p) { return (uint32_t)__cvta_generic_to_shared(p); }

// UMMA shared-memory descriptor, no swizzle: start, leading- and stride-
// dimension byte offsets (16-byte units), version 1 (bits 46-47).
__device__ __forceinline__ uint64_t sdesc(uint32_t saddr, uint32_t lbo, uint32_t sbo) {
    return (uint64_t)((saddr >> 4) & 0x3FFFu) | ((uint64_t)((lbo >> 4) & 0x3FFFu) << 16) |
           ((uint64_t)((sbo >> 4) & 0x3FFFu) << 32) | (1ull << 46);
}

// Instruction descriptor of kind::f16: D F32, A and B BF16, M = 128.
__host__ __device__ constexpr uint32_t idesc(int n, bool a_mn, bool b_mn) {
    return (1u << 4) | (1u << 7) | (1u << 10) | ((a_mn ? 1u : 0u) << 15) | ((b_mn ? 1u : 0u) << 16) |
           ((uint32_t)(n >> 3) << 17) | ((uint32_t)(128 >> 4) << 24);
}

__device__ __forceinline__ void mbar_init(uint32_t a) {
    asm volatile("mbarrier.init.shared::cta.b64 [%0], 1;" ::"r"(a) : "memory");
    asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
}

__device__ __forceinline__ bool mbar_try(uint32_t a, uint32_t parity) {
    uint32_t ok;
    asm volatile(
        "{\n\t.reg .pred p;\n\tmbarrier.try_wait.parity.shared::cta.b64 p, [%1], %2;\n\tselp.u32 %0, 1, 0, p;\n\t}"
        : "=r"(ok)
        : "r"(a), "r"(parity)
        : "memory");
    return ok != 0;
}

// Bounded wait for an mbarrier phase; false when the bound passed.
__device__ __forceinline__ bool mbar_wait(uint32_t a, uint32_t parity) {
    const long long t0 = clock64();
    while (!mbar_try(a, parity))
        if (clock64() - t0 > kWaitCycles) return false;
    return true;
}

__device__ __forceinline__ void fence_async_smem() { asm volatile("fence.proxy.async.shared::cta;" ::: "memory"); }
__device__ __forceinline__ void tc_before() { asm volatile("tcgen05.fence::before_thread_sync;" ::: "memory"); }
__device__ __forceinline__ void tc_after() { asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory"); }

__device__ __forceinline__ void mma_bf16(uint32_t d, uint64_t a, uint64_t b, uint32_t id, uint32_t acc) {
    asm volatile(
        "{\n\t.reg .pred p;\n\tsetp.ne.b32 p, %4, 0;\n\ttcgen05.mma.cta_group::1.kind::f16 [%0], %1, %2, %3, p;\n\t}"
        ::"r"(d), "l"(a), "l"(b), "r"(id), "r"(acc)
        : "memory");
}

__device__ __forceinline__ void mma_commit(uint32_t mbar) {
    asm volatile("tcgen05.commit.cta_group::1.mbarrier::arrive::one.shared::cluster.b64 [%0];" ::"r"(mbar)
                 : "memory");
}

// 32 consecutive FP32 columns of TMEM for this warp's 32 lanes (thread t:
// lane 32 w + t), waited for.
__device__ __forceinline__ void tmem_ld32(uint32_t ta, float (&v)[32]) {
    uint32_t r[32];
    asm volatile(
        "tcgen05.ld.sync.aligned.32x32b.x32.b32 {%0,%1,%2,%3,%4,%5,%6,%7,%8,%9,%10,%11,%12,%13,%14,%15,%16,%17,%18,"
        "%19,%20,%21,%22,%23,%24,%25,%26,%27,%28,%29,%30,%31}, [%32];"
        : "=r"(r[0]), "=r"(r[1]), "=r"(r[2]), "=r"(r[3]), "=r"(r[4]), "=r"(r[5]), "=r"(r[6]), "=r"(r[7]),
          "=r"(r[8]), "=r"(r[9]), "=r"(r[10]), "=r"(r[11]), "=r"(r[12]), "=r"(r[13]), "=r"(r[14]), "=r"(r[15]),
          "=r"(r[16]), "=r"(r[17]), "=r"(r[18]), "=r"(r[19]), "=r"(r[20]), "=r"(r[21]), "=r"(r[22]),
          "=r"(r[23]), "=r"(r[24]), "=r"(r[25]), "=r"(r[26]), "=r"(r[27]), "=r"(r[28]), "=r"(r[29]),
          "=r"(r[30]), "=r"(r[31])
        : "r"(ta)
        : "memory");
    asm volatile("tcgen05.wait::ld.sync.aligned;" ::: "memory");
#pragma unroll
    for (int i = 0; i < 32; i++) v[i] = __uint_as_float(r[i]);
}

__device__ __forceinline__ float tanh_hw(float x) {
    float y;
    asm("tanh.approx.f32 %0, %1;" : "=f"(y) : "f"(x));
    return y;
}
// the same SiLU as the mma.sync kernels (sigmoid through the hardware tanh)
__device__ __forceinline__ float sigm(float z) { return 0.5f + 0.5f * tanh_hw(0.5f * z); }

__device__ __forceinline__ uint32_t pack2(float lo, float hi) {
    __nv_bfloat162 v = __floats2bfloat162_rn(lo, hi);
    return *reinterpret_cast<uint32_t *>(&v);
}

// Row r's 8 values of group g of a 128-row buffer: one 16-byte store.
__device__ __forceinline__ void st_group(unsigned char *buf, int g, int r, const float *v8) {
    uint4 q;
    q.x = pack2(v8[0], v8[1]);
    q.y = pack2(v8[2], v8[3]);
    q.z = pack2(v8[4], v8[5]);
    q.w = pack2(v8[6], v8[7]);
    *reinterpret_cast<uint4 *>(buf + g * kGrp + (r >> 3) * 128 + (r & 7) * 16) = q;
}
__device__ __forceinline__ void st_group_raw(unsigned char *buf, int g, int r, uint4 q) {
    *reinterpret_cast<uint4 *>(buf + g * kGrp + (r >> 3) * 128 + (r & 7) * 16) = q;
}

// The weights as B operands (K-major core-matrix grids) and the FP32 vectors.
template <class M>
__device__ void load_weights(unsigned char *sm, const float *p, const __nv_bfloat16 *w1, const __nv_bfloat16 *w2,
                             const __nv_bfloat16 *w2t, bool need_w2t) {
    const uint4 *w1q = reinterpret_cast<const uint4 *>(w1);
    const uint4 *w2q = reinterpret_cast<const uint4 *>(w2);
    const uint4 *w2tq = reinterpret_cast<const uint4 *>(w2t);
    for (int c = threadIdx.x; c < 64 * 2; c += blockDim.x) {  // W1[n][k]: 64 rows x 2 chunks of 8
        const int n = c >> 1, kc = c & 1;
        *reinterpret_cast<uint4 *>(sm + M::W1 + (n >> 3) * 256 + kc * 128 + (n & 7) * 16) = w1q[c];
    }
    for (int c = threadIdx.x; c < 64 * 8; c += blockDim.x) {  // W2[n][k] and W2T[n][k]: 64 rows x 8 chunks
        const int n = c >> 3, kc = c & 7;
        const uint32_t off = (n >> 3) * 1024 + kc * 128 + (n & 7) * 16;
        *reinterpret_cast<uint4 *>(sm + M::W2 + off) = w2q[c];
        if (need_w2t) *reinterpret_cast<uint4 *>(sm + M::W2T + off) = w2tq[c];
    }
    float *par = reinterpret_cast<float *>(sm + M::Par);
    for (int i = threadIdx.x; i < kHid; i += blockDim.x) {
        par[i] = p[oB1 + i];
        par[64 + i] = p[oB2 + i];
        par[128 + i] = p[oW3 + i];
    }
    if (threadIdx.x == 0) par[192] = p[oB3];
}

// ---------------------------------------------------------------- forward
// CTA set-up shared by the kernels: weights into shared memory, TMEM
// allocated (warp 0), the mbarrier initialised; returns the TMEM base.
template <class M>
__device__ __forceinline__ uint32_t cta_setup(unsigned char *sm, const float *p, const __nv_bfloat16 *w1,
                                              const __nv_bfloat16 *w2, const __nv_bfloat16 *w2t, bool need_w2t) {
    load_weights<M>(sm, p, w1, w2, w2t, need_w2t);
    uint32_t *tslot = reinterpret_cast<uint32_t *>(sm + M::Bar + 8);
    if (threadIdx.x < 32) {
        asm volatile("tcgen05.alloc.cta_group::1.sync.aligned.shared::cta.b32 [%0], %1;" ::"r"(su32(tslot)),
                     "r"(M::TmemCols)
                     : "memory");
        asm volatile("tcgen05.relinquish_alloc_permit.cta_group::1.sync.aligned;" ::: "memory");
    }
    if (threadIdx.x == 0) {
        mbar_init(su32(sm + M::Bar));
        *reinterpret_cast<double *>(sm + M::Red) = 0.0;
    }
    fence_async_smem();
    tc_before();
    __syncthreads();
    tc_after();
    return *tslot;
}

// Releases the TMEM once every access is complete (warp 0, the allocator).
template <class M>
__device__ __forceinline__ void cta_teardown(uint32_t tm) {
    tc_before();
    __syncthreads();
    tc_after();
    if (threadIdx.x < 32)
        asm volatile("tcgen05.dealloc.cta_group::1.sync.aligned.b32 %0, %1;" ::"r"(tm), "r"(M::TmemCols) : "memory");
}

// Forward pass of one tile whose X rows every thread has stored in XH
// groups 8-9: Z1 = X W1^T, H1 = silu(Z1 + b1), Z2 = H1 W2^T, and this
// thread's output silu(Z2 + b2) . w3 + b3.  `fail` is block-uniform on
// return (true: a completion wait passed its bound; the output is void).
template <class M>
__device__ __forceinline__ float forward_tile(unsigned char *sm, uint32_t tm, uint32_t mbar, uint32_t &phase,
                                              bool &fail) {
    const int tid = threadIdx.x;
    const uint32_t tlane = tm + ((uint32_t)(32 * (tid >> 5)) << 16);
    const float *par = reinterpret_cast<const float *>(sm + M::Par);
    const uint32_t sxh = su32(sm + kXH), sw1 = su32(sm + M::W1), sw2 = su32(sm + M::W2);
    fence_async_smem();
    if ((fail = __syncthreads_or(fail))) return 0.f;
    if (tid == 0) {
        tc_after();
        mma_bf16(tm, sdesc(sxh + 8 * kGrp, kGrp, 128), sdesc(sw1, 128, 256), idesc(64, false, false), 0);
        mma_commit(mbar);
    }
    fail |= !mbar_wait(mbar, phase);
    phase ^= 1;
    tc_after();
#pragma unroll
    for (int c = 0; c < 2; c++) {
        float z[32];
        tmem_ld32(tlane + 32 * c, z);
#pragma unroll
        for (int i = 0; i < 32; i++) {
            const float a = z[i] + par[32 * c + i];
            z[i] = a * sigm(a);
        }
#pragma unroll
        for (int g = 0; g < 4; g++) st_group(sm + kXH, 4 * c + g, tid, z + 8 * g);
    }
    fence_async_smem();
    tc_before();
    if ((fail = __syncthreads_or(fail))) return 0.f;
    if (tid == 0) {
        tc_after();
#pragma unroll
        for (int s = 0; s < 4; s++)
            mma_bf16(tm + 64, sdesc(sxh + s * 2 * kGrp, kGrp, 128), sdesc(sw2 + s * 256, 128, 1024),
                     idesc(64, false, false), s > 0);
        mma_commit(mbar);
    }
    fail |= !mbar_wait(mbar, phase);
    phase ^= 1;
    tc_after();
    float o = par[192];
#pragma unroll
    for (int c = 0; c < 2; c++) {
        float z[32];
        tmem_ld32(tlane + 64 + 32 * c, z);
#pragma unroll
        for (int i = 0; i < 32; i++) {
            const float a = z[i] + par[64 + 32 * c + i];
            o += a * sigm(a) * par[128 + 32 * c + i];
        }
    }
    tc_before();  // the next tile's products overwrite the columns just read
    fail = __syncthreads_or(fail);
    return o;
}

// outputs of rows [0, rows)
__global__ void __launch_bounds__(kThreads) k_forward_tc(const float *__restrict__ p,
                                                         const __nv_bfloat16 *__restrict__ w1,
                                                         const __nv_bfloat16 *__restrict__ w2,
                                                         const __nv_bfloat16 *__restrict__ x, int64_t rows,
                                                         float *__restrict__ out, uint32_t *status) {
    extern __shared__ __align__(1024) unsigned char sm[];
    const int tid = threadIdx.x;
    const uint32_t tm = cta_setup<FwdMap>(sm, p, w1, w2, nullptr, false);
    const uint32_t mbar = su32(sm + FwdMap::Bar);
    uint32_t phase = 0;
    bool fail = false;
    const int64_t tiles = (rows + kThreads - 1) / kThreads;
    for (int64_t t = blockIdx.x; t < tiles && !fail; t += gridDim.x) {
        const int64_t row = t * kThreads + tid;
        uint4 x0 = make_uint4(0, 0, 0, 0), x1 = x0;
        if (row < rows) {
            const uint4 *xq = reinterpret_cast<const uint4 *>(x + row * kIn);
            x0 = xq[0];
            x1 = xq[1];
        }
        st_group_raw(sm + kXH, 8, tid, x0);
        st_group_raw(sm + kXH, 9, tid, x1);
        const float o = forward_tile<FwdMap>(sm, tm, mbar, phase, fail);
        if (!fail && row < rows) out[row] = o;
    }
    if (fail && tid == 0) atomicOr(status, kStDeviceWait);
    cta_teardown<FwdMap>(tm);
}

// The exact mean of the control variate (cv.cu's k_quad_mean) with the MLP on
// tcgen05 tiles: thread t of a tile takes item (start q, first-hop bin i),
// computes its first-hop point, probability weight and features, the tile's
// 128 feature rows go through forward_tile, and sum += weight * phi in FP64;
// phi of every item is kept for the walks' look-up.
__global__ void __launch_bounds__(kThreads) k_quad_mean_tc(
    DevLayout L, double4 trect, int target_id, const double4 *__restrict__ gauss, const double4 *__restrict__ sqs,
    const int *__restrict__ sides, uint32_t Q, const double *__restrict__ pi_exact, const double *__restrict__ wx,
    const double *__restrict__ wy, double eps, bool exact, const float *__restrict__ p,
    const __nv_bfloat16 *__restrict__ w1, const __nv_bfloat16 *__restrict__ w2, double *sum,
    float *__restrict__ phi_out, uint32_t *status) {
    extern __shared__ __align__(1024) unsigned char sm[];
    const int tid = threadIdx.x;
    const uint32_t tm = cta_setup<FwdMap>(sm, p, w1, w2, nullptr, false);
    const uint32_t mbar = su32(sm + FwdMap::Bar);
    uint32_t phase = 0;
    bool fail = false;
    const int64_t n = (int64_t)Q * FRW_NSAMPLE;
    const double4 g4 = gauss[0];
    const double perim = __dadd_rn(__dmul_rn(2.0, __dsub_rn(g4.z, g4.x)), __dmul_rn(2.0, __dsub_rn(g4.w, g4.y)));
    double acc = 0.0;
    const int64_t tiles = (n + kThreads - 1) / kThreads;
    for (int64_t tl = blockIdx.x; tl < tiles && !fail; tl += gridDim.x) {
        const int64_t t = tl * kThreads + tid;
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
            if (nearest_other(L, x1, y1, target_id, o)) {
                edge_feats(x1, y1, o.x, o.y, o.z, o.w, a0, f + 8);
            } else {
#pragma unroll
                for (int q = 8; q < kIn; q++) f[q] = 16.f;
            }
        }
        st_group(sm + kXH, 8, tid, f);
        st_group(sm + kXH, 9, tid, f + 8);
        const float phi = forward_tile<FwdMap>(sm, tm, mbar, phase, fail);
        if (!fail) {
            acc += wgt * (double)phi;
            if (phi_out && t < n) phi_out[t] = phi;
        }
    }
#pragma unroll
    for (int o = 16; o; o >>= 1) acc += __shfl_xor_sync(0xFFFFFFFFu, acc, o);
    if ((tid & 31) == 0 && !fail) atomicAdd(sum, acc);
    if (fail && tid == 0) atomicOr(status, kStDeviceWait);
    cta_teardown<FwdMap>(tm);
}

// ---------------------------------------------------------------- training
// grad += d/dparams sum_r wt_r (f(x_r) - y_r)^2 * inv_wsum; loss += the sum.
__global__ void __launch_bounds__(kThreads) k_train_grad_tc(const float *__restrict__ p,
                                                            const __nv_bfloat16 *__restrict__ w1,
                                                            const __nv_bfloat16 *__restrict__ w2,
                                                            const __nv_bfloat16 *__restrict__ w2t,
                                                            const __nv_bfloat16 *__restrict__ x,
                                                            const float *__restrict__ y, const float *__restrict__ wt,
                                                            int64_t rows, float inv_wsum, float *__restrict__ part,
                                                            double *__restrict__ loss_out, uint32_t *status) {
    extern __shared__ __align__(1024) unsigned char sm[];
    const int tid = threadIdx.x, warp = tid >> 5;
    {  // constant groups: XH ones (10) and zeros (11), H2 ones (8) and zeros (9-15), B3 zeros (1)
        const uint4 z = make_uint4(0, 0, 0, 0);
        const uint4 one = make_uint4(0x3F80u, 0, 0, 0);  // BF16 1.0 in the first column of the group
        st_group_raw(sm + kXH, 10, tid, one);
        st_group_raw(sm + kXH, 11, tid, z);
        st_group_raw(sm + kH2, 8, tid, one);
        for (int g = 9; g < 16; g++) st_group_raw(sm + kH2, g, tid, z);
        st_group_raw(sm + kB3, 1, tid, z);
    }
    const uint32_t tm = cta_setup<TrainMap>(sm, p, w1, w2, w2t, true);
    double *red = reinterpret_cast<double *>(sm + TrainMap::Red);
    const uint32_t mbar = su32(sm + TrainMap::Bar);
    const uint32_t tlane = tm + ((uint32_t)(32 * warp) << 16);
    const float *par = reinterpret_cast<const float *>(sm + TrainMap::Par);
    const uint32_t sxh = su32(sm + kXH), sdz = su32(sm + kDZ), sh2 = su32(sm + kH2), sb3 = su32(sm + kB3);
    const uint32_t sw1 = su32(sm + TrainMap::W1), sw2 = su32(sm + TrainMap::W2), sw2t = su32(sm + TrainMap::W2T);
    uint32_t phase = 0;
    bool fail = false;
    double lsum = 0.0;
    int ntile = 0;
    const int64_t tiles = (rows + kThreads - 1) / kThreads;
    for (int64_t t = blockIdx.x; t < tiles; t += gridDim.x, ntile++) {
        const int64_t row = t * kThreads + tid;
        const bool valid = row < rows;
        uint4 x0 = make_uint4(0, 0, 0, 0), x1 = x0;
        float yr = 0.f, wr = 0.f;
        if (valid) {
            const uint4 *xq = reinterpret_cast<const uint4 *>(x + row * kIn);
            x0 = xq[0];
            x1 = xq[1];
            yr = y[row];
            wr = wt[row];
        }
        st_group_raw(sm + kXH, 8, tid, x0);
        st_group_raw(sm + kXH, 9, tid, x1);
        fence_async_smem();
        if (__syncthreads_or(fail)) break;
        // Z1 = X W1^T
        if (tid == 0) {
            tc_after();
            mma_bf16(tm, sdesc(sxh + 8 * kGrp, kGrp, 128), sdesc(sw1, 128, 256), idesc(64, false, false), 0);
            mma_commit(mbar);
        }
        fail |= !mbar_wait(mbar, phase);
        phase ^= 1;
        tc_after();
#pragma unroll
        for (int c = 0; c < 2; c++) {  // H1 = silu(Z1 + b1)
            float z[32];
            tmem_ld32(tlane + 32 * c, z);
#pragma unroll
            for (int i = 0; i < 32; i++) {
                const float a = z[i] + par[32 * c + i];
                z[i] = a * sigm(a);
            }
#pragma unroll
            for (int g = 0; g < 4; g++) st_group(sm + kXH, 4 * c + g, tid, z + 8 * g);
        }
        fence_async_smem();
        tc_before();
        if (__syncthreads_or(fail)) break;
        // Z2 = H1 W2^T
        if (tid == 0) {
            tc_after();
#pragma unroll
            for (int s = 0; s < 4; s++)
                mma_bf16(tm + 64, sdesc(sxh + s * 2 * kGrp, kGrp, 128), sdesc(sw2 + s * 256, 128, 1024),
                         idesc(64, false, false), s > 0);
            mma_commit(mbar);
        }
        fail |= !mbar_wait(mbar, phase);
        phase ^= 1;
        tc_after();
        float o = par[192];
#pragma unroll
        for (int c = 0; c < 2; c++) {
            float z[32];
            tmem_ld32(tlane + 64 + 32 * c, z);
#pragma unroll
            for (int i = 0; i < 32; i++) {
                const float a = z[i] + par[64 + 32 * c + i];
                o += a * sigm(a) * par[128 + 32 * c + i];
            }
        }
        const float e = valid ? o - yr : 0.f;
        const float dz3 = 2.f * wr * e * inv_wsum;
        lsum += (double)wr * e * e * inv_wsum;
#pragma unroll
        for (int c = 0; c < 2; c++) {  // dZ2 = dz3 w3 silu'(Z2 + b2); H2 = silu(Z2 + b2)
            float z[32], h[32];
            tmem_ld32(tlane + 64 + 32 * c, z);
#pragma unroll
            for (int i = 0; i < 32; i++) {
                const float a = z[i] + par[64 + 32 * c + i];
                const float s = sigm(a);
                h[i] = a * s;
                z[i] = dz3 * par[128 + 32 * c + i] * (s * (1.f + a * (1.f - s)));
            }
#pragma unroll
            for (int g = 0; g < 4; g++) {
                st_group(sm + kDZ, 4 * c + g, tid, z + 8 * g);
                st_group(sm + kH2, 4 * c + g, tid, h + 8 * g);
            }
        }
        st_group_raw(sm + kB3, 0, tid, make_uint4(pack2(dz3, 1.f), 0, 0, 0));
        fence_async_smem();
        tc_before();
        if (__syncthreads_or(fail)) break;
        // dH1 = dZ2 W2 (into the Z2 columns, read above)
        if (tid == 0) {
            tc_after();
#pragma unroll
            for (int s = 0; s < 4; s++)
                mma_bf16(tm + 64, sdesc(sdz + s * 2 * kGrp, kGrp, 128), sdesc(sw2t + s * 256, 128, 1024),
                         idesc(64, false, false), s > 0);
            mma_commit(mbar);
        }
        fail |= !mbar_wait(mbar, phase);
        phase ^= 1;
        tc_after();
#pragma unroll
        for (int c = 0; c < 2; c++) {  // dZ1 = dH1 silu'(Z1 + b1)
            float dh[32], z[32];
            tmem_ld32(tlane + 64 + 32 * c, dh);
            tmem_ld32(tlane + 32 * c, z);
#pragma unroll
            for (int i = 0; i < 32; i++) {
                const float a = z[i] + par[32 * c + i];
                const float s = sigm(a);
                dh[i] *= s * (1.f + a * (1.f - s));
            }
#pragma unroll
            for (int g = 0; g < 4; g++) st_group(sm + kDZ, 8 + 4 * c + g, tid, dh + 8 * g);
        }
        fence_async_smem();
        tc_before();
        if (__syncthreads_or(fail)) break;
        // weight and bias gradients, accumulated over the CTA's tiles: K = the 128 rows
        if (tid == 0) {
            tc_after();
#pragma unroll
            for (int s = 0; s < 8; s++) {
                const uint32_t acc = (ntile > 0 || s > 0) ? 1u : 0u;
                mma_bf16(tm + 128, sdesc(sdz + s * 256, 128, kGrp), sdesc(sxh + s * 256, 128, kGrp),
                         idesc(96, true, true), acc);
                mma_bf16(tm + 224, sdesc(sh2 + s * 256, 128, kGrp), sdesc(sb3 + s * 256, 128, kGrp),
                         idesc(16, true, true), acc);
            }
            mma_commit(mbar);
        }
        fail |= !mbar_wait(mbar, phase);  // before the next tile rewrites the operands
        phase ^= 1;
        tc_after();
    }
    // flush this CTA's gradients: TMEM lane f holds row f of the products
    if (__syncthreads_or(fail)) {
        if (tid == 0) atomicOr(status, kStDeviceWait);
    } else if (ntile > 0) {
        // this CTA's gradient, in the packed parameter order, to its own slot
        // of the partial sums (plain stores; k_reduce_adam / k_reduce_sum add
        // the slots up in a fixed order)
        float *g = part + (size_t)blockIdx.x * kPartStride;
        float v[32];
        if (warp < 2) {  // f = tid: dW2[f][0..63], db2[f], dw3[f]
            const int f = tid;
            tmem_ld32(tlane + 128, v);
#pragma unroll
            for (int i = 0; i < 32; i += 4)
                *reinterpret_cast<float4 *>(g + oW2 + f * kHid + i) = make_float4(v[i], v[i + 1], v[i + 2], v[i + 3]);
            tmem_ld32(tlane + 160, v);
#pragma unroll
            for (int i = 0; i < 32; i += 4)
                *reinterpret_cast<float4 *>(g + oW2 + f * kHid + 32 + i) =
                    make_float4(v[i], v[i + 1], v[i + 2], v[i + 3]);
            tmem_ld32(tlane + 192, v);
            g[oB2 + f] = v[16];
            tmem_ld32(tlane + 224, v);
            g[oW3 + f] = v[0];
        } else {  // f = tid - 64: dW1[f][0..15], db1[f]; lane 64 also holds db3
            const int f = tid - 64;
            tmem_ld32(tlane + 192, v);
#pragma unroll
            for (int i = 0; i < 16; i++) g[oW1 + f * kIn + i] = v[i];
            g[oB1 + f] = v[16];
            tmem_ld32(tlane + 224, v);
            if (f == 0) g[oB3] = v[0];
        }
        // loss: warp sums, then one atomic per CTA
#pragma unroll
        for (int o = 16; o; o >>= 1) lsum += __shfl_xor_sync(0xFFFFFFFFu, lsum, o);
        if ((tid & 31) == 0) atomicAdd(red, lsum);
    }
    __syncthreads();
    if (tid == 0 && !fail && ntile > 0) atomicAdd(loss_out, red[0]);
    cta_teardown<TrainMap>(tm);
}

// The gradient of a training step: the CTAs' partial sums added in CTA
// order (so the step is reproducible), then Adam on the FP32 master copy and
// the BF16 operand copies refreshed -- the same update as cv.cu's k_adam, at
// step t (1-based).
__global__ void k_reduce_adam(const float *__restrict__ part, int nb, float *__restrict__ p, float *__restrict__ m,
                              float *__restrict__ v, int t, float lr, __nv_bfloat16 *__restrict__ w1,
                              __nv_bfloat16 *__restrict__ w2, __nv_bfloat16 *__restrict__ w2t) {
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= kParams) return;
    float gi = 0.f;
    for (int b = 0; b < nb; b++) gi += part[(size_t)b * kPartStride + i];
    const float b1 = 0.9f, b2 = 0.999f;
    const float mi = b1 * m[i] + (1.f - b1) * gi;
    const float vi = b2 * v[i] + (1.f - b2) * gi * gi;
    m[i] = mi;
    v[i] = vi;
    const float mh = mi / (1.f - powf(b1, (float)t)), vh = vi / (1.f - powf(b2, (float)t));
    const float pi = p[i] - lr * mh / (sqrtf(vh) + 1e-8f);
    p[i] = pi;
    if (i < oB1) w1[i] = __float2bfloat16_rn(pi);
    else if (i >= oW2 && i < oB2) {
        const int k = i - oW2;
        w2[k] = __float2bfloat16_rn(pi);
        w2t[(k % kHid) * kHid + k / kHid] = __float2bfloat16_rn(pi);
    }
}

// grad += the CTAs' partial sums, in CTA order.
__global__ void k_reduce_sum(const float *__restrict__ part, int nb, float *__restrict__ grad) {
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= kParams) return;
    float gi = 0.f;
    for (int b = 0; b < nb; b++) gi += part[(size_t)b * kPartStride + i];
    grad[i] += gi;
}

}  // namespace

int train_blocks_tc(int64_t rows, int sms) {
    const int64_t tiles = (rows + kThreads - 1) / kThreads;
    return (int)std::max<int64_t>(1, std::min<int64_t>(tiles, TrainMap::PerSm * (int64_t)sms));
}

frw_status launch_forward_tc(const Net &n, const __nv_bfloat16 *x, int64_t rows, float *out, uint32_t *status,
                             int sms, cudaStream_t st) {
    if (rows <= 0) return FRW_OK;
    FRW_CK(cudaFuncSetAttribute(k_forward_tc, cudaFuncAttributeMaxDynamicSharedMemorySize, FwdMap::Smem));
    const int64_t tiles = (rows + kThreads - 1) / kThreads;
    const int blocks = (int)std::min<int64_t>(tiles, FwdMap::PerSm * (int64_t)sms);
    k_forward_tc<<<blocks, kThreads, FwdMap::Smem, st>>>(n.p, n.w1, n.w2, x, rows, out, status);
    FRW_CK(cudaGetLastError());
    return FRW_OK;
}

frw_status launch_train_grad_tc(const Net &n, const __nv_bfloat16 *x, const float *y, const float *wt, int64_t rows,
                                float inv_wsum, float *part, double *loss, uint32_t *status, int sms,
                                cudaStream_t st) {
    if (rows <= 0) return FRW_OK;
    FRW_CK(cudaFuncSetAttribute(k_train_grad_tc, cudaFuncAttributeMaxDynamicSharedMemorySize, TrainMap::Smem));
    const int blocks = train_blocks_tc(rows, sms);
    k_train_grad_tc<<<blocks, kThreads, TrainMap::Smem, st>>>(n.p, n.w1, n.w2, n.w2t, x, y, wt, rows, inv_wsum, part,
                                                              loss, status);
    FRW_CK(cudaGetLastError());
    return FRW_OK;
}

frw_status launch_reduce_adam_tc(const Net &n, const float *part, int nb, float *m, float *v, int t, float lr,
                                 cudaStream_t st) {
    k_reduce_adam<<<(kParams + 255) / 256, 256, 0, st>>>(part, nb, n.p, m, v, t, lr, n.w1, n.w2, n.w2t);
    FRW_CK(cudaGetLastError());
    return FRW_OK;
}

frw_status launch_reduce_sum_tc(const float *part, int nb, float *grad, cudaStream_t st) {
    k_reduce_sum<<<(kParams + 255) / 256, 256, 0, st>>>(part, nb, grad);
    FRW_CK(cudaGetLastError());
    return FRW_OK;
}

frw_status launch_quad_mean_tc(const DevLayout &L, double4 trect, int tid, const double4 *gauss, const double4 *sqs,
                               const int *sides, uint32_t Q, const double *pi_exact, const double *wx,
                               const double *wy, double eps, bool exact, const Net &net, double *sum, float *phi_out,
                               uint32_t *status, int sms, cudaStream_t st) {
    FRW_CK(cudaFuncSetAttribute(k_quad_mean_tc, cudaFuncAttributeMaxDynamicSharedMemorySize, FwdMap::Smem));
    const int64_t tiles = ((int64_t)Q * FRW_NSAMPLE + kThreads - 1) / kThreads;
    const int blocks = (int)std::min<int64_t>(tiles, FwdMap::PerSm * (int64_t)sms);
    k_quad_mean_tc<<<blocks, kThreads, FwdMap::Smem, st>>>(L, trect, tid, gauss, sqs, sides, Q, pi_exact, wx, wy, eps, exact,
                                                    net.p, net.w1, net.w2, sum, phi_out, status);
    FRW_CK(cudaGetLastError());
    return FRW_OK;
}

}  // namespace cv
}  // namespace frw
