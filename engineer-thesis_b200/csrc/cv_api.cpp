// cv_api.cpp -- C ABI of the learned control variate (host side).
//
// frw_cv_train: walks from an independent seed give training pairs
// (features of the first-hop point, 1{walk ends on the target}, weight c^2);
// the MLP is fitted on the device (fused forward+backward + Adam per step);
// then the exact mean E[c*phi] is summed
// over the grid start x first-hop bins, keeping phi of every (arc, bin) in a
// table.  frw_cv_walk: walks recording (end, weight factor, arc * 200 + bin),
// phi looked up in the table, reduction -- the plain and the control-variate
// estimate of C_tt side by side from the same walks.
#include <math.h>
#include <string.h>

#include <algorithm>
#include <atomic>
#include <string>
#include <utility>
#include <vector>

#include "cv.cuh"
#include "frw_internal.h"

struct frw_cv {
    const frw_layout *layout = nullptr;
    int64_t target = 0;
    frw_opts opts{};
    frw::LayoutView view{};
    frw::cv::Net net;
    double mean_term = 0.0, train_loss = 0.0, train_ms = 0.0, quad_ms = 0.0;
    uint64_t train_walks = 0;
    uint32_t quad_points = 0;
    float *phi = nullptr;  // phi at every (grid arc, first-hop bin): Q x 200
};

namespace frw {
namespace {

std::atomic<int> g_cv_walk_mode{FRW_CV_WALK_FUSED};

struct Buf {
    std::vector<void *> p;
    cudaStream_t st;
    explicit Buf(cudaStream_t s) : st(s) {}
    template <typename T>
    cudaError_t get(T **x, size_t bytes) {
        cudaError_t e = cudaMallocAsync((void **)x, bytes ? bytes : 16, st);
        if (e == cudaSuccess) p.push_back(*x);
        return e;
    }
    ~Buf() {
        for (void *q : p) cudaFreeAsync(q, st);
    }
};

struct SetDevice {
    int prev = -1;
    explicit SetDevice(int d) {
        if (cudaGetDevice(&prev) != cudaSuccess) prev = -1;
        if (prev != d) cudaSetDevice(d);
    }
    ~SetDevice() {
        if (prev >= 0) cudaSetDevice(prev);
    }
};

bool pow2(uint32_t q) { return q && !(q & (q - 1)); }

// Exact probability of bin i under the 32-bit uniform u = x 2^-32 and the
// CDF search of the walk: #{x : intg[i] <= x 2^-32 < intg[i+1]} / 2^32.
void exact_bin_probs(double *pi) {
    double g[FRW_NSAMPLE], intg[FRW_NSAMPLE + 1];
    green_tables(g, intg, nullptr, nullptr);
    for (int i = 0; i < FRW_NSAMPLE; i++)
        pi[i] = (ceil(ldexp(intg[i + 1], 32)) - ceil(ldexp(intg[i], 32))) / 4294967296.0;
}

void init_params(uint64_t seed, float *p) {
    uint64_t s = seed ^ 0x5DEECE66Dull;
    auto unif = [&]() {
        uint64_t z = (s += 0x9E3779B97F4A7C15ull);
        z = (z ^ (z >> 30)) * 0xBF58476D1CE4E5B9ull;
        z = (z ^ (z >> 27)) * 0x94D049BB133111EBull;
        z ^= z >> 31;
        return (double)(z >> 11) * 0x1p-53 * 2.0 - 1.0;
    };
    memset(p, 0, sizeof(float) * cv::kParams);
    const double a1 = sqrt(6.0 / (cv::kIn + cv::kHid)), a2 = sqrt(6.0 / (2 * cv::kHid)),
                 a3 = sqrt(6.0 / (cv::kHid + 1));
    for (int i = 0; i < cv::kHid * cv::kIn; i++) p[cv::oW1 + i] = (float)(a1 * unif());
    for (int i = 0; i < cv::kHid * cv::kHid; i++) p[cv::oW2 + i] = (float)(a2 * unif());
    for (int i = 0; i < cv::kHid; i++) p[cv::oW3 + i] = (float)(a3 * unif());
    p[cv::oB3] = 0.5f;
}

frw_status check_cv_walk_opts(const frw_opts &o) {
    frw_status rc = check_opts(&o);
    if (rc) return rc;
    if (o.start_mode != FRW_START_UNIFORM || !pow2(o.start_grid) || o.start_grid > (1u << 23) || o.hop_cap < 2) {
        set_error("control variate: needs FRW_START_UNIFORM, start_grid a power of two <= 2^23 and hop_cap >= 2");
        return FRW_E_ARG;
    }
    return FRW_OK;
}

// frw_cv_walk with the control variate's sums kept by the walk kernel: one
// launch into dense rows; the estimates come from the target's row (plain:
// sums of c over walks ending on the target) and the kernel's sums of z.
frw_status cv_walk_fused(const frw_cv *M, uint64_t walks, uint64_t seed, frw_cv_result *res, cudaStream_t st) {
    const int64_t n = M->view.n;
    Buf B(st);
    unsigned long long *d_hits, *d_stats;
    double *d_s1, *d_s2, *d_pack;  // pack: sum z, sum z^2, sum w, sum w^2, status word
    uint32_t *d_status;
    cudaError_t e = B.get(&d_hits, (size_t)n * 8);
    if (e == cudaSuccess) e = B.get(&d_s1, (size_t)n * 8);
    if (e == cudaSuccess) e = B.get(&d_s2, (size_t)n * 8);
    if (e == cudaSuccess) e = B.get(&d_stats, 32);
    if (e == cudaSuccess) e = B.get(&d_pack, 48);
    if (e == cudaSuccess) e = B.get(&d_status, 4);
    if (e != cudaSuccess) return cuda_fail(e, "frw_cv_walk: allocation");
    for (auto z : {std::make_pair((void *)d_hits, (size_t)n * 8), std::make_pair((void *)d_s1, (size_t)n * 8),
                   std::make_pair((void *)d_s2, (size_t)n * 8), std::make_pair((void *)d_stats, (size_t)32),
                   std::make_pair((void *)d_pack, (size_t)48), std::make_pair((void *)d_status, (size_t)4)})
        if ((e = cudaMemsetAsync(z.first, 0, z.second, st)) != cudaSuccess) return cuda_fail(e, "frw_cv_walk: clear");
    Events ev(2);
    if (!ev.ok(2)) return cuda_fail(cudaErrorUnknown, "frw_cv_walk: cudaEventCreate");
    frw_opts o = M->opts;
    o.first_walk = 0;
    cudaEventRecord(ev[0], st);
    frw_status rc = walk_device_rows(M->layout, M->target, walks, seed, o, reinterpret_cast<uint64_t *>(d_hits), d_s1,
                                     d_s2, reinterpret_cast<uint64_t *>(d_stats), d_status, M->phi, d_pack, st);
    cudaEventRecord(ev[1], st);
    if (rc) return rc;
    e = cudaMemcpyAsync(d_pack + 2, d_s1 + M->target, 8, cudaMemcpyDeviceToDevice, st);
    if (e == cudaSuccess) e = cudaMemcpyAsync(d_pack + 3, d_s2 + M->target, 8, cudaMemcpyDeviceToDevice, st);
    if (e == cudaSuccess) e = cudaMemcpyAsync(d_pack + 4, d_status, 4, cudaMemcpyDeviceToDevice, st);
    if (e != cudaSuccess) return cuda_fail(e, "frw_cv_walk: gather");
    double h[5] = {0, 0, 0, 0, 0};
    if ((rc = read_back(h, d_pack, 40, st, "frw_cv_walk"))) return rc;
    uint32_t status_word;
    memcpy(&status_word, &h[4], 4);
    if (status_word) return status_word_error(status_word);
    float ms = 0;
    cudaEventElapsedTime(&ms, ev[0], ev[1]);
    const double N = (double)walks;
    const double mz = h[0] / N, vz = std::max(h[1] / N - mz * mz, 0.0) * N / (N - 1);
    const double mw = h[2] / N, vw = std::max(h[3] / N - mw * mw, 0.0) * N / (N - 1);
    res->walks = walks;
    res->plain = mw;
    res->plain_se = sqrt(vw / N);
    res->cv = mz + M->mean_term;
    res->cv_se = sqrt(vz / N);
    res->variance_ratio = vz > 0 ? vw / vz : 0.0;
    res->kernel_ms = ms;
    return FRW_OK;
}

}  // namespace
}  // namespace frw

using namespace frw;

extern "C" {

void frw_cv_opts_default(frw_cv_opts *o) {
    memset(o, 0, sizeof(*o));
    o->struct_size = sizeof(frw_cv_opts);
    o->train_walks = 1000000;
    o->train_seed = 0x7E57C0DEull;
    o->epochs = 4;
    o->batch = 32768;
    o->lr = 6e-3f;
}

frw_status frw_cv_train(const frw_layout *layout, int64_t target, const frw_opts *walk_opts,
                        const frw_cv_opts *cv_opts, frw_cv **out, void *stream) {
    if (!layout || !walk_opts || !out) {
        set_error("frw_cv_train: null argument");
        return FRW_E_ARG;
    }
    *out = nullptr;
    frw_cv_opts co;
    frw_cv_opts_default(&co);
    if (cv_opts) co = *cv_opts;
    if (co.struct_size != sizeof(frw_cv_opts) || co.train_walks < 64 || co.epochs < 1 || co.batch < 64 ||
        co.batch % 64 || !(co.lr > 0)) {
        set_error("frw_cv_train: bad frw_cv_opts");
        return FRW_E_ARG;
    }
    frw_status rc = check_cv_walk_opts(*walk_opts);
    if (rc) return rc;
    LayoutView v;
    rc = layout_view(layout, &v);
    if (rc) return rc;
    if (target < 0 || target >= v.n) {
        set_error("frw_cv_train: target out of range");
        return FRW_E_ARG;
    }
    SetDevice sd(v.device);
    WaitScope ws(walk_opts->timeout_ms);
    const double *tables;
    int sms;
    rc = device_tables(v.device, &tables, &sms);
    if (rc) return rc;
    cudaStream_t st = (cudaStream_t)stream;
    frw_cv *M = new frw_cv();
    M->layout = layout;
    M->target = target;
    M->opts = *walk_opts;
    M->view = v;
    M->train_walks = co.train_walks;
    auto fail = [&](frw_status r) {
        cv::net_free(&M->net, st);
        if (M->phi) cudaFreeAsync(M->phi, st);
        delete M;
        return r;
    };
    Events ev(3);
    if (!ev.ok(3)) return fail(cuda_fail(cudaErrorUnknown, "frw_cv_train: cudaEventCreate"));
    cudaEvent_t e0 = ev[0], e1 = ev[1], e2 = ev[2];
    const int64_t N = (int64_t)co.train_walks;
    {
        Buf B(st);
        int64_t *d_end;
        double4 *d_rec;
        __nv_bfloat16 *d_x;
        float *d_y, *d_wt, *d_grad, *d_m, *d_v, *d_part = nullptr;
        double *d_wsum, *d_loss;
        int *d_step;
        uint32_t *d_tstatus;
        const int steps_per_epoch = (int)((N + co.batch - 1) / co.batch);
        const int steps = steps_per_epoch * co.epochs;
        cudaError_t e = cudaSuccess;
        if (e == cudaSuccess) e = B.get(&d_end, N * 8);
        if (e == cudaSuccess) e = B.get(&d_rec, N * 32);
        if (e == cudaSuccess) e = B.get(&d_x, N * 32);
        if (e == cudaSuccess) e = B.get(&d_y, N * 4);
        if (e == cudaSuccess) e = B.get(&d_wt, N * 4);
        if (e == cudaSuccess) e = B.get(&d_grad, cv::kParams * 4);
        if (e == cudaSuccess) e = B.get(&d_m, cv::kParams * 4);
        if (e == cudaSuccess) e = B.get(&d_v, cv::kParams * 4);
        if (e == cudaSuccess) e = B.get(&d_wsum, 8);
        if (e == cudaSuccess) e = B.get(&d_loss, (size_t)steps * 8);
        if (e == cudaSuccess) e = B.get(&d_step, 4);
        if (e == cudaSuccess) e = B.get(&d_tstatus, 4);
        const bool tc = cv::mlp_kernels() == FRW_MLP_TCGEN05;
        const int sms_tc = tc ? cv::device_sm_count() : 0;
        const int nb_tc = tc ? cv::train_blocks_tc(co.batch, sms_tc) : 0;
        if (e == cudaSuccess && tc) e = B.get(&d_part, (size_t)nb_tc * cv::kPartStride * sizeof(float));
        if (e != cudaSuccess) return fail(cuda_fail(e, "frw_cv_train: allocation"));
        cudaEventRecord(e0, st);
        // training walks start anywhere on the surface: a stratified start
        // with more strata than training walks would cover only part of it
        frw_opts train_opts = *walk_opts;
        train_opts.start_strata = 0;
        rc = walk_records(layout, target, 0, (uint64_t)N, co.train_seed, train_opts, st, d_end, d_rec);
        if (rc) return fail(rc);
        const double *r = v.rects + 4 * target;
        const double4 trect = make_double4(r[0], r[1], r[2], r[3]);
        rc = cv::launch_features(v.dl, trect, (int)target, d_rec, N, d_x, nullptr, st);
        if (!rc) {
            cudaMemsetAsync(d_wsum, 0, 8, st);
            rc = cv::launch_targets(d_end, d_rec, N, (int)target, d_y, d_wt, d_wsum, st);
        }
        if (rc) return fail(rc);
        double wsum = 0.0;
        rc = read_back(&wsum, d_wsum, 8, st, "frw_cv_train: training set");
        if (rc) return fail(rc);
        if (!(wsum > 0)) {
            set_error("frw_cv_train: no training walk has a first hop");
            return fail(FRW_E_ARG);
        }
        std::vector<float> h(cv::kParams);
        init_params(co.train_seed, h.data());
        rc = cv::net_alloc(&M->net, st);
        if (!rc) rc = cv::net_upload(&M->net, h.data(), st);
        if (rc) return fail(rc);
        cudaMemsetAsync(d_grad, 0, cv::kParams * 4, st);
        cudaMemsetAsync(d_m, 0, cv::kParams * 4, st);
        cudaMemsetAsync(d_v, 0, cv::kParams * 4, st);
        cudaMemsetAsync(d_loss, 0, (size_t)steps * 8, st);
        cudaMemsetAsync(d_step, 0, 4, st);
        cudaMemsetAsync(d_tstatus, 0, 4, st);
        // the training loop: a few hundred launches, enqueued directly (the
        // host stays ahead of the device; instantiating a graph of them would
        // cost more host time than it saves)
        const double scale = (double)N / wsum;  // per-batch normalisation of the weighted MSE
        for (int s = 0; s < steps && !rc; s++) {
            const int64_t start = (int64_t)(s % steps_per_epoch) * co.batch;
            const int64_t rows = std::min<int64_t>(co.batch, N - start);
            const float inv = (float)(scale / (double)rows);
            if (tc) {  // partial gradients per CTA, summed in CTA order with the Adam step
                const int nb = cv::train_blocks_tc(rows, sms_tc);
                rc = cv::launch_train_grad_tc(M->net, d_x + 16 * start, d_y + start, d_wt + start, rows, inv, d_part,
                                              d_loss + s, d_tstatus, sms_tc, st);
                if (!rc) rc = cv::launch_reduce_adam_tc(M->net, d_part, nb, d_m, d_v, s + 1, co.lr, st);
            } else {
                rc = cv::launch_train_grad(M->net, d_x + 16 * start, d_y + start, d_wt + start, rows, inv, d_grad,
                                           d_loss + s, d_tstatus, st);
                if (!rc) rc = cv::launch_adam(M->net, d_grad, d_m, d_v, d_step, co.lr, st);
            }
        }
        if (rc) return fail(rc);
        cudaEventRecord(e1, st);
        std::vector<double> losses(steps);
        rc = read_back(losses.data(), d_loss, (size_t)steps * 8, st, "frw_cv_train: training");
        uint32_t ts = 0;
        if (!rc) rc = read_back(&ts, d_tstatus, 4, st, "frw_cv_train: training status");
        if (!rc) rc = status_word_error(ts);
        if (rc) return fail(rc);
        double l = 0;
        for (int s = steps - steps_per_epoch; s < steps; s++) l += losses[s];
        M->train_loss = l / steps_per_epoch;
    }
    // exact mean of the control variate over the grid start x first-hop bins
    {
        Buf B(st);
        const uint32_t Q = walk_opts->start_grid;
        const int64_t nq = (int64_t)Q * FRW_NSAMPLE;
        double4 *d_gauss, *d_tgt;
        double *d_pi, *d_mu;
        uint32_t *d_status;
        cudaError_t e = cudaSuccess;
        if (e == cudaSuccess) e = B.get(&d_gauss, 32);
        if (e == cudaSuccess) e = B.get(&d_tgt, 32);
        if (e == cudaSuccess) e = B.get(&d_pi, FRW_NSAMPLE * 8);
        if (e == cudaSuccess) e = B.get(&d_mu, 8);
        if (e == cudaSuccess) e = B.get(&d_status, 4);
        if (e != cudaSuccess) return fail(cuda_fail(e, "frw_cv_train: quadrature allocation"));
        double pi[FRW_NSAMPLE];
        exact_bin_probs(pi);
        const double *r = v.rects + 4 * target;
        cudaMemcpyAsync(d_pi, pi, sizeof(pi), cudaMemcpyHostToDevice, st);
        cudaMemcpyAsync(d_tgt, r, 32, cudaMemcpyHostToDevice, st);
        cudaMemsetAsync(d_mu, 0, 8, st);
        cudaMemsetAsync(d_status, 0, 4, st);
        rc = launch_gauss(v.dl, (const double *)d_tgt, 1, walk_opts->gauss_mode, walk_opts->gauss_param,
                          (double *)d_gauss, d_status, st);
        const double4 trect = make_double4(r[0], r[1], r[2], r[3]);
        if (!rc) {
            e = cudaMallocAsync(&M->phi, (size_t)nq * sizeof(float), st);
            if (e != cudaSuccess) return fail(cuda_fail(e, "frw_cv_train: phi table"));
        }
        if (!rc)
            rc = cv::launch_quad_mean(v.dl, trect, (int)target, d_gauss, Q, d_pi, tables + FRW_NSAMPLE + 1,
                                      tables + 2 * FRW_NSAMPLE + 1, walk_opts->permittivity,
                                      walk_opts->exact_perimeter != 0, M->net, d_mu, M->phi, d_status, st);
        if (rc) return fail(rc);
        uint32_t hs = 0;
        e = cudaEventRecord(e2, st);
        if (e != cudaSuccess) return fail(cuda_fail(e, "frw_cv_train: quadrature"));
        rc = read_back(&M->mean_term, d_mu, 8, st, "frw_cv_train: quadrature");
        if (!rc) rc = read_back(&hs, d_status, 4, st, "frw_cv_train: quadrature");
        if (rc) return fail(rc);
        if (hs) {
            set_error("frw_cv_train: a kernel reported an internal limit during the quadrature");
            return fail(FRW_E_KERNEL);
        }
        M->quad_points = (uint32_t)nq;
    }
    float a = 0, b = 0;
    cudaEventElapsedTime(&a, e0, e1);
    cudaEventElapsedTime(&b, e1, e2);
    M->train_ms = a;
    M->quad_ms = b;

    *out = M;
    return FRW_OK;
}

frw_status frw_cv_info_get(const frw_cv *M, frw_cv_info *info) {
    if (!M || !info) {
        set_error("null argument");
        return FRW_E_ARG;
    }
    info->mean_term = M->mean_term;
    info->train_loss = M->train_loss;
    info->train_ms = M->train_ms;
    info->quad_ms = M->quad_ms;
    info->train_walks = M->train_walks;
    info->quad_points = M->quad_points;
    return FRW_OK;
}

frw_status frw_cv_set_walk_mode(int mode) {
    if (mode != FRW_CV_WALK_FUSED && mode != FRW_CV_WALK_RECORDS) {
        set_error("frw_cv_set_walk_mode: FRW_CV_WALK_FUSED or FRW_CV_WALK_RECORDS");
        return FRW_E_ARG;
    }
    g_cv_walk_mode.store(mode, std::memory_order_relaxed);
    return FRW_OK;
}

int frw_cv_get_walk_mode(void) { return g_cv_walk_mode.load(std::memory_order_relaxed); }

frw_status frw_cv_walk(const frw_cv *M, uint64_t walks, uint64_t seed, frw_cv_result *res, void *stream) {
    if (!M || !res || walks < 2) {
        set_error("frw_cv_walk: bad arguments");
        return FRW_E_ARG;
    }
    SetDevice sd(M->view.device);
    WaitScope ws(M->opts.timeout_ms);
    cudaStream_t st = (cudaStream_t)stream;
    if (g_cv_walk_mode.load(std::memory_order_relaxed) == FRW_CV_WALK_FUSED) return cv_walk_fused(M, walks, seed, res, st);
    const uint64_t chunk = std::min<uint64_t>(walks, 1ull << 23);
    Buf B(st);
    int64_t *d_end;
    double *d_w;
    int32_t *d_q;
    double *d_sums;
    cudaError_t e = cudaSuccess;
    if (e == cudaSuccess) e = B.get(&d_end, chunk * 8);
    if (e == cudaSuccess) e = B.get(&d_w, chunk * 8);
    if (e == cudaSuccess) e = B.get(&d_q, chunk * 4);
    if (e == cudaSuccess) e = B.get(&d_sums, 32);
    if (e != cudaSuccess) return cuda_fail(e, "frw_cv_walk: allocation");
    cudaMemsetAsync(d_sums, 0, 32, st);
    Events ev(2);
    if (!ev.ok(2)) return cuda_fail(cudaErrorUnknown, "frw_cv_walk: cudaEventCreate");
    cudaEvent_t e0 = ev[0], e1 = ev[1];
    cudaEventRecord(e0, st);
    frw_status rc = FRW_OK;
    for (uint64_t first = 0; first < walks && !rc; first += chunk) {
        const uint64_t n = std::min<uint64_t>(chunk, walks - first);
        rc = walk_records(M->layout, M->target, first, n, seed, M->opts, st, d_end, nullptr, d_w, d_q);
        if (!rc) rc = cv::launch_cv_gather(d_end, d_w, d_q, M->phi, (int64_t)n, (int)M->target, d_sums, st);
    }
    cudaEventRecord(e1, st);
    double h[4] = {0, 0, 0, 0};
    if (!rc) rc = read_back(h, d_sums, 32, st, "frw_cv_walk");
    float ms = 0;
    if (!rc) cudaEventElapsedTime(&ms, e0, e1);
    if (rc) return rc;
    const double N = (double)walks;
    const double mz = h[0] / N, vz = std::max(h[1] / N - mz * mz, 0.0) * N / (N - 1);
    const double mw = h[2] / N, vw = std::max(h[3] / N - mw * mw, 0.0) * N / (N - 1);
    res->walks = walks;
    res->plain = mw;
    res->plain_se = sqrt(vw / N);
    res->cv = mz + M->mean_term;
    res->cv_se = sqrt(vz / N);
    res->variance_ratio = vz > 0 ? vw / vz : 0.0;
    res->kernel_ms = ms;
    return FRW_OK;
}

frw_status frw_cv_destroy(frw_cv *M) {
    if (!M) return FRW_OK;
    SetDevice sd(M->view.device);
    cudaError_t e = cudaDeviceSynchronize();  // nothing may still read the table
    cv::net_free(&M->net, nullptr);
    if (M->phi) cudaFreeAsync(M->phi, nullptr);
    delete M;
    FRW_CK(e);
    return FRW_OK;
}

frw_status frw_cv_params(const frw_cv *M, float *out) {
    if (!M || !out) {
        set_error("null argument");
        return FRW_E_ARG;
    }
    SetDevice sd(M->view.device);
    FRW_CK(cudaMemcpy(out, M->net.p, cv::kParams * sizeof(float), cudaMemcpyDeviceToHost));
    return FRW_OK;
}

// ---- direct access to the MLP and feature kernels (host arrays) ----
frw_status frw_mlp_forward(const float *params, const float *x, int64_t n, float *out, int device) {
    if (!params || !x || !out || n <= 0) {
        set_error("frw_mlp_forward: bad arguments");
        return FRW_E_ARG;
    }
    const double *tables;
    int sms;
    frw_status rc = device_tables(device, &tables, &sms);
    if (rc) return rc;
    SetDevice sd(device);
    cudaStream_t st = nullptr;
    Buf B(st);
    float *d_xf, *d_out;
    __nv_bfloat16 *d_x;
    uint32_t *d_status;
    FRW_CK(B.get(&d_xf, n * 64));
    FRW_CK(B.get(&d_x, n * 32));
    FRW_CK(B.get(&d_out, n * 4));
    FRW_CK(B.get(&d_status, 4));
    FRW_CK(cudaMemsetAsync(d_status, 0, 4, st));
    cv::Net net;
    rc = cv::net_alloc(&net, st);
    if (!rc) rc = cv::net_upload(&net, params, st);
    if (!rc) {
        FRW_CK(cudaMemcpyAsync(d_xf, x, n * 64, cudaMemcpyHostToDevice, st));
        std::vector<__nv_bfloat16> hb((size_t)n * 16);
        for (int64_t i = 0; i < n * 16; i++) hb[i] = __float2bfloat16_rn(x[i]);
        FRW_CK(cudaMemcpyAsync(d_x, hb.data(), n * 32, cudaMemcpyHostToDevice, st));
        rc = cv::launch_forward(net, d_x, n, d_out, d_status, st);
        uint32_t hs = 0;
        if (!rc) rc = read_back(&hs, d_status, 4, st, "frw_mlp_forward");
        if (!rc) rc = status_word_error(hs);
        if (!rc) rc = read_back(out, d_out, n * 4, st, "frw_mlp_forward");
    }
    cv::net_free(&net, st);
    return rc;
}

frw_status frw_mlp_grad(const float *params, const float *x, const float *y, const float *wt, int64_t n,
                        double inv_wsum, float *grad, double *loss, int device) {
    if (!params || !x || !y || !wt || !grad || n <= 0) {
        set_error("frw_mlp_grad: bad arguments");
        return FRW_E_ARG;
    }
    const double *tables;
    int sms;
    frw_status rc = device_tables(device, &tables, &sms);
    if (rc) return rc;
    SetDevice sd(device);
    cudaStream_t st = nullptr;
    Buf B(st);
    __nv_bfloat16 *d_x;
    float *d_y, *d_wt, *d_g;
    double *d_l;
    uint32_t *d_status;
    FRW_CK(B.get(&d_status, 4));
    FRW_CK(cudaMemsetAsync(d_status, 0, 4, st));
    FRW_CK(B.get(&d_x, n * 32));
    FRW_CK(B.get(&d_y, n * 4));
    FRW_CK(B.get(&d_wt, n * 4));
    FRW_CK(B.get(&d_g, cv::kParams * 4));
    FRW_CK(B.get(&d_l, 8));
    cv::Net net;
    rc = cv::net_alloc(&net, st);
    if (!rc) rc = cv::net_upload(&net, params, st);
    if (!rc) {
        std::vector<__nv_bfloat16> hb((size_t)n * 16);
        for (int64_t i = 0; i < n * 16; i++) hb[i] = __float2bfloat16_rn(x[i]);
        FRW_CK(cudaMemcpyAsync(d_x, hb.data(), n * 32, cudaMemcpyHostToDevice, st));
        FRW_CK(cudaMemcpyAsync(d_y, y, n * 4, cudaMemcpyHostToDevice, st));
        FRW_CK(cudaMemcpyAsync(d_wt, wt, n * 4, cudaMemcpyHostToDevice, st));
        FRW_CK(cudaMemsetAsync(d_g, 0, cv::kParams * 4, st));
        FRW_CK(cudaMemsetAsync(d_l, 0, 8, st));
        rc = cv::launch_train_grad(net, d_x, d_y, d_wt, n, (float)inv_wsum, d_g, d_l, d_status, st);
        uint32_t hs = 0;
        if (!rc) rc = read_back(&hs, d_status, 4, st, "frw_mlp_grad");
        if (!rc) rc = status_word_error(hs);
        if (!rc) rc = read_back(grad, d_g, cv::kParams * 4, st, "frw_mlp_grad");
        if (!rc && loss) rc = read_back(loss, d_l, 8, st, "frw_mlp_grad");
    }
    cv::net_free(&net, st);
    return rc;
}

frw_status frw_mlp_set_kernels(int which) { return cv::set_mlp_kernels(which); }

int frw_mlp_get_kernels(void) { return cv::mlp_kernels(); }

frw_status frw_cv_features(const frw_layout *layout, int64_t target, const double *rec4, int64_t n, float *out) {
    LayoutView v;
    frw_status rc = layout_view(layout, &v);
    if (rc) return rc;
    if (!rec4 || !out || n <= 0 || target < 0 || target >= v.n) {
        set_error("frw_cv_features: bad arguments");
        return FRW_E_ARG;
    }
    SetDevice sd(v.device);
    cudaStream_t st = nullptr;
    Buf B(st);
    double4 *d_rec;
    float *d_f;
    FRW_CK(B.get(&d_rec, n * 32));
    FRW_CK(B.get(&d_f, n * 64));
    FRW_CK(cudaMemcpyAsync(d_rec, rec4, n * 32, cudaMemcpyHostToDevice, st));
    const double *r = v.rects + 4 * target;
    rc = cv::launch_features(v.dl, make_double4(r[0], r[1], r[2], r[3]), (int)target, d_rec, n, nullptr, d_f, st);
    if (rc) return rc;
    return read_back(out, d_f, n * 64, st, "frw_cv_features");
}

}  // extern "C"
