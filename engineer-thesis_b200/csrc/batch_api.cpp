// batch_api.cpp -- many layouts (or targets) in one persistent walk launch.
//
// A batch is a job table (one job = layout, target conductor, walk count)
// walked by ONE launch of the multi-job walk kernel: every warp lane picks
// its next walk from a single global counter and keeps its job while the
// walk index stays inside the job's range (a binary search over the jobs'
// first walk indices otherwise), so jobs of very uneven size share the whole
// GPU without per-job tail effects.  The device work of a run
// (clears, the Gaussian surfaces of all jobs, the walk launch and the row
// compaction) is captured once into a CUDA graph; a run writes the seed into
// device memory and replays the graph.  Launch parameters (resident blocks
// per SM, refill threshold, walks claimed per atomic) come from a measured
// search over the batch itself (frw_batch_tune) or from the caller.
#include <math.h>
#include <string.h>

#include <algorithm>
#include <string>
#include <vector>

#include "frw_internal.h"

struct frw_batch {
    int device = 0;
    int njobs = 0;
    frw_opts opts{};
    std::vector<frw::LayoutView> views;
    std::vector<int64_t> targets, acc_base;
    std::vector<frw::WalkJob> hjobs;
    std::vector<uint64_t> walks, begin;
    int64_t rows = 0;
    uint64_t total = 0;
    frw_tuning tuning{};
    int sms = 0;
    const double *tables = nullptr;
    // device buffers
    frw::WalkJob *d_jobs = nullptr;
    double4 *d_targets = nullptr, *d_gauss = nullptr;
    uint64_t *d_seed = nullptr;
    unsigned long long *d_counter = nullptr, *d_stats = nullptr, *d_acc_n = nullptr, *d_cn = nullptr,
                       *d_cnt = nullptr;
    double *d_acc_s = nullptr, *d_acc_s2 = nullptr, *d_cs = nullptr, *d_cs2 = nullptr;
    int64_t *d_row = nullptr;
    uint32_t *d_status = nullptr;
    cudaStream_t cs = nullptr;
    cudaGraphExec_t exec = nullptr;
};

namespace frw {
namespace {

struct SetDev {
    int prev = -1;
    explicit SetDev(int d) {
        if (cudaGetDevice(&prev) != cudaSuccess) prev = -1;
        if (prev != d) cudaSetDevice(d);
    }
    ~SetDev() {
        if (prev >= 0) cudaSetDevice(prev);
    }
};

WalkParams params_for(const frw_batch *B, const WalkJob *jobs, const WalkJob &job0, uint64_t total,
                      const frw_tuning &t) {
    WalkParams P{};
    P.jobs = jobs;
    P.gauss = B->d_gauss;
    P.njobs = B->njobs;
    P.start_mode = B->opts.start_mode;
    P.exact_perimeter = B->opts.exact_perimeter;
    P.refill_min = t.refill_min > 0 ? t.refill_min : 1;
    P.start_grid = B->opts.start_grid;
    P.start_strata = B->opts.start_strata;
    P.hop_cap = B->opts.hop_cap;
    P.permittivity = B->opts.permittivity;
    P.seed_dev = B->d_seed;
    P.chunk = (uint32_t)t.chunk;
    P.total_walks = total;
    P.counter = B->d_counter;
    P.acc_n = B->d_acc_n;
    P.acc_s = B->d_acc_s;
    P.acc_s2 = B->d_acc_s2;
    P.job_stats = B->d_stats;
    P.status = B->d_status;
    P.intg = B->tables;
    P.wx = B->tables + FRW_NSAMPLE + 1;
    P.wy = B->tables + 2 * FRW_NSAMPLE + 1;
    P.job0 = job0;  // read by the single-job kernel when the batch has one job
    for (int j = 0; j < B->njobs; j++) P.tree_points |= B->hjobs[j].L.tree_points;
    return P;
}

int grid_for(const frw_batch *B, const frw_tuning &t, uint64_t total) {
    const int maxb = walk_max_blocks_per_sm(256, B->njobs > 1, B->opts.start_mode == FRW_START_UNIFORM);
    int bps = t.blocks_per_sm > 0 ? t.blocks_per_sm : maxb;
    bps = std::max(1, std::min(bps, maxb));
    uint64_t blocks = (uint64_t)B->sms * bps, need = (total + 255) / 256;
    return (int)std::max<uint64_t>(1, std::min(blocks, need));
}

// The device work of one run on stream st (graph-capturable: no host syncs).
frw_status enqueue_run(frw_batch *B, const WalkJob *jobs, const WalkJob &job0, uint64_t total, const frw_tuning &t,
                       cudaStream_t st, cudaEvent_t k0, cudaEvent_t k1) {
    FRW_CK(cudaMemsetAsync(B->d_counter, 0, 8, st));
    FRW_CK(cudaMemsetAsync(B->d_stats, 0, (size_t)B->njobs * 32, st));
    FRW_CK(cudaMemsetAsync(B->d_status, 0, 4, st));
    FRW_CK(cudaMemsetAsync(B->d_cnt, 0, 8, st));
    FRW_CK(cudaMemsetAsync(B->d_acc_n, 0, (size_t)B->rows * 8, st));
    FRW_CK(cudaMemsetAsync(B->d_acc_s, 0, (size_t)B->rows * 8, st));
    FRW_CK(cudaMemsetAsync(B->d_acc_s2, 0, (size_t)B->rows * 8, st));
    frw_status rc = launch_gauss_jobs(jobs, (const double *)B->d_targets, B->njobs, B->opts.gauss_mode,
                                      B->opts.gauss_param, (double *)B->d_gauss, B->d_status, st);
    if (rc) return rc;
    if (k0) FRW_CK(cudaEventRecord(k0, st));
    rc = launch_walk(params_for(B, jobs, job0, total, t), 256, grid_for(B, t, total), st);
    if (rc) return rc;
    if (k1) FRW_CK(cudaEventRecord(k1, st));
    return launch_compact(B->d_acc_n, B->d_acc_s, B->d_acc_s2, B->rows, B->d_row, B->d_cn, B->d_cs, B->d_cs2,
                          B->d_cnt, st);
}

frw_status build_graph(frw_batch *B) {
    if (B->exec) {
        cudaGraphExecDestroy(B->exec);
        B->exec = nullptr;
    }
    cudaGraph_t g = nullptr;
    FRW_CK(cudaStreamBeginCapture(B->cs, cudaStreamCaptureModeThreadLocal));
    frw_status rc = enqueue_run(B, B->d_jobs, B->hjobs[0], B->total, B->tuning, B->cs, nullptr, nullptr);
    cudaError_t e = cudaStreamEndCapture(B->cs, &g);
    if (rc) {
        if (g) cudaGraphDestroy(g);
        return rc;
    }
    FRW_CK(e);
    e = cudaGraphInstantiate(&B->exec, g, 0);
    cudaGraphDestroy(g);
    FRW_CK(e);
    return FRW_OK;
}

void free_batch(frw_batch *B) {
    if (B->exec) cudaGraphExecDestroy(B->exec);
    if (B->cs) cudaStreamDestroy(B->cs);
    void *ps[] = {B->d_jobs, B->d_targets, B->d_gauss, B->d_seed, B->d_counter, B->d_stats, B->d_acc_n, B->d_cn,
                  B->d_cnt, B->d_acc_s, B->d_acc_s2, B->d_cs, B->d_cs2, B->d_row, B->d_status};
    for (void *p : ps) cudaFree(p);
    delete B;
}

}  // namespace
}  // namespace frw

using namespace frw;

extern "C" {

frw_status frw_batch_create(const frw_layout *const *layouts, const int64_t *targets, const uint64_t *walks,
                            int32_t njobs, const frw_opts *opts, frw_batch **out) {
    if (!layouts || !targets || !walks || njobs <= 0 || !out) {
        set_error("frw_batch_create: bad arguments");
        return FRW_E_ARG;
    }
    *out = nullptr;
    frw_opts o;
    frw_opts_default(&o);
    if (opts) o = *opts;
    frw_status rc = check_opts(&o);
    if (rc) return rc;
    frw_batch *B = new frw_batch();
    B->njobs = njobs;
    B->opts = o;
    B->views.resize(njobs);
    for (int j = 0; j < njobs; j++) {
        rc = layout_view(layouts[j], &B->views[j]);
        if (rc) {
            delete B;
            return rc;
        }
        if (targets[j] < 0 || targets[j] >= B->views[j].n || B->views[j].device != B->views[0].device) {
            set_error("frw_batch_create: job " + std::to_string(j) + ": target out of range or layout on another device");
            delete B;
            return FRW_E_ARG;
        }
        B->targets.push_back(targets[j]);
        B->walks.push_back(walks[j]);
        B->begin.push_back(B->total);
        B->acc_base.push_back(B->rows);
        B->total += walks[j];
        B->rows += B->views[j].n;
    }
    B->device = B->views[0].device;
    SetDev sd(B->device);
    rc = device_tables(B->device, &B->tables, &B->sms);
    if (rc) {
        delete B;
        return rc;
    }
    std::vector<WalkJob> jobs(njobs);
    std::vector<double> tg(4 * (size_t)njobs);
    for (int j = 0; j < njobs; j++) {
        WalkJob &J = jobs[j];
        J = WalkJob{};
        J.L = B->views[j].dl;
        J.target = targets[j];
        J.walk_begin = B->begin[j];
        J.walks = walks[j];
        J.first_walk = 0;
        J.acc_base = B->acc_base[j];
        J.stream_id = o.stream_id + (uint32_t)j;
        memcpy(&tg[4 * (size_t)j], B->views[j].rects + 4 * targets[j], 32);
    }
    cudaError_t e = cudaSuccess;
    auto A = [&](auto **p, size_t bytes) {
        if (e == cudaSuccess) e = cudaMalloc((void **)p, bytes ? bytes : 16);
    };
    A(&B->d_jobs, sizeof(WalkJob) * njobs);
    A(&B->d_targets, 32 * (size_t)njobs);
    A(&B->d_gauss, 32 * (size_t)njobs);
    A(&B->d_seed, 8);
    A(&B->d_counter, 8);
    A(&B->d_stats, 32 * (size_t)njobs);
    A(&B->d_acc_n, 8 * (size_t)B->rows);
    A(&B->d_acc_s, 8 * (size_t)B->rows);
    A(&B->d_acc_s2, 8 * (size_t)B->rows);
    A(&B->d_row, 8 * (size_t)B->rows);
    A(&B->d_cn, 8 * (size_t)B->rows);
    A(&B->d_cs, 8 * (size_t)B->rows);
    A(&B->d_cs2, 8 * (size_t)B->rows);
    A(&B->d_cnt, 8);
    A(&B->d_status, 4);
    if (e == cudaSuccess) e = cudaStreamCreateWithFlags(&B->cs, cudaStreamNonBlocking);
    if (e == cudaSuccess) e = cudaMemcpy(B->d_jobs, jobs.data(), sizeof(WalkJob) * njobs, cudaMemcpyHostToDevice);
    B->hjobs = jobs;
    if (e == cudaSuccess) e = cudaMemcpy(B->d_targets, tg.data(), tg.size() * 8, cudaMemcpyHostToDevice);
    if (e != cudaSuccess) {
        rc = cuda_fail(e, "frw_batch_create");
        free_batch(B);
        return rc;
    }
    B->tuning.struct_size = sizeof(frw_tuning);
    B->tuning.blocks_per_sm = o.blocks_per_sm;
    B->tuning.refill_min = o.refill_min > 0 ? o.refill_min : 1;
    B->tuning.chunk = 128;
    rc = build_graph(B);
    if (rc) {
        free_batch(B);
        return rc;
    }
    *out = B;
    return FRW_OK;
}

frw_status frw_batch_set_tuning(frw_batch *B, const frw_tuning *t) {
    if (!B || !t || t->struct_size != sizeof(frw_tuning) || t->chunk < 32 || t->chunk > (1 << 20)) {
        set_error("frw_batch_set_tuning: bad arguments");
        return FRW_E_ARG;
    }
    SetDev sd(B->device);
    B->tuning = *t;
    return build_graph(B);
}

frw_status frw_batch_get_tuning(const frw_batch *B, frw_tuning *t) {
    if (!B || !t) {
        set_error("null argument");
        return FRW_E_ARG;
    }
    *t = B->tuning;
    return FRW_OK;
}

frw_status frw_batch_tune(frw_batch *B, uint64_t trial_walks, frw_tuning *chosen) {
    if (!B || trial_walks == 0) {
        set_error("frw_batch_tune: bad arguments");
        return FRW_E_ARG;
    }
    SetDev sd(B->device);
    // a scaled copy of the job table: same jobs, trial_walks in total
    std::vector<WalkJob> jobs(B->njobs);
    jobs = B->hjobs;
    const double f = std::min(1.0, (double)trial_walks / (double)B->total);
    uint64_t tot = 0;
    for (int j = 0; j < B->njobs; j++) {
        jobs[j].walk_begin = tot;
        jobs[j].walks = std::max<uint64_t>(1, (uint64_t)llround(f * (double)B->walks[j]));
        tot += jobs[j].walks;
    }
    WalkJob *d_tj = nullptr;
    FRW_CK(cudaMalloc(&d_tj, sizeof(WalkJob) * B->njobs));
    struct Free {
        void *p;
        ~Free() { cudaFree(p); }
    } free_tj{d_tj};
    FRW_CK(cudaMemcpy(d_tj, jobs.data(), sizeof(WalkJob) * B->njobs, cudaMemcpyHostToDevice));
    const uint64_t seed = 0x5EEDull;
    FRW_CK(cudaMemcpy(B->d_seed, &seed, 8, cudaMemcpyHostToDevice));
    Events ev(2);
    if (!ev.ok(2)) {
        set_error("frw_batch_tune: cudaEventCreate failed");
        return FRW_E_CUDA;
    }
    cudaEvent_t k0 = ev[0], k1 = ev[1];
    const int maxb =
        std::max(1, walk_max_blocks_per_sm(256, B->njobs > 1, B->opts.start_mode == FRW_START_UNIFORM));
    const int refills[] = {1, 4, 16};
    const int chunks[] = {32, 128, 512};
    frw_tuning best = B->tuning;
    best.ms = 1e30;
    frw_status rc = FRW_OK;
    for (int bps = 1; bps <= maxb && !rc; bps++)
        for (int rf : refills)
            for (int ch : chunks) {
                frw_tuning t = B->tuning;
                t.blocks_per_sm = bps;
                t.refill_min = rf;
                t.chunk = ch;
                float ms = 0.f;
                for (int rep = 0; rep < 2 && !rc; rep++) {  // first run warms caches
                    rc = enqueue_run(B, d_tj, jobs[0], tot, t, B->cs, k0, k1);
                    if (!rc) rc = wait_stream(B->cs, "frw_batch_tune: trial");
                    if (!rc) cudaEventElapsedTime(&ms, k0, k1);
                }
                if (rc) break;
                if (ms < best.ms) {
                    best = t;
                    best.ms = ms;
                }
            }
    if (rc) return rc;
    B->tuning = best;
    if (chosen) *chosen = best;
    return build_graph(B);
}

frw_status frw_batch_run(frw_batch *B, uint64_t seed, frw_result *results, void *stream) {
    if (!B) {
        set_error("frw_batch_run: null batch");
        return FRW_E_ARG;
    }
    SetDev sd(B->device);
    cudaStream_t us = (cudaStream_t)stream;
    Events evs(3);
    if (!evs.ok(3)) {
        set_error("frw_batch_run: cudaEventCreate failed");
        return FRW_E_CUDA;
    }
    cudaEvent_t ev = evs[0], t0 = evs[1], t1 = evs[2];
    // order after the caller's stream, run on the batch stream
    FRW_CK(cudaEventRecord(ev, us));
    FRW_CK(cudaStreamWaitEvent(B->cs, ev, 0));
    FRW_CK(cudaMemcpyAsync(B->d_seed, &seed, 8, cudaMemcpyHostToDevice, B->cs));
    cudaEventRecord(t0, B->cs);
    FRW_CK(cudaGraphLaunch(B->exec, B->cs));
    cudaEventRecord(t1, B->cs);
    unsigned long long cnt = 0;
    uint32_t status = 0;
    std::vector<unsigned long long> stats(4 * (size_t)B->njobs);
    std::vector<double> gauss(4 * (size_t)B->njobs);
    {
        WaitScope ws(B->opts.timeout_ms);
        frw_status rc = wait_stream(B->cs, "frw_batch_run");
        if (rc) return rc;
    }
    FRW_CK(cudaMemcpyAsync(&cnt, B->d_cnt, 8, cudaMemcpyDeviceToHost, B->cs));
    FRW_CK(cudaMemcpyAsync(&status, B->d_status, 4, cudaMemcpyDeviceToHost, B->cs));
    FRW_CK(cudaMemcpyAsync(stats.data(), B->d_stats, stats.size() * 8, cudaMemcpyDeviceToHost, B->cs));
    FRW_CK(cudaMemcpyAsync(gauss.data(), B->d_gauss, gauss.size() * 8, cudaMemcpyDeviceToHost, B->cs));
    FRW_CK(cudaStreamSynchronize(B->cs));
    std::vector<int64_t> row(cnt);
    std::vector<unsigned long long> n(cnt);
    std::vector<double> s(cnt), s2(cnt);
    if (cnt) {
        FRW_CK(cudaMemcpyAsync(row.data(), B->d_row, cnt * 8, cudaMemcpyDeviceToHost, B->cs));
        FRW_CK(cudaMemcpyAsync(n.data(), B->d_cn, cnt * 8, cudaMemcpyDeviceToHost, B->cs));
        FRW_CK(cudaMemcpyAsync(s.data(), B->d_cs, cnt * 8, cudaMemcpyDeviceToHost, B->cs));
        FRW_CK(cudaMemcpyAsync(s2.data(), B->d_cs2, cnt * 8, cudaMemcpyDeviceToHost, B->cs));
        FRW_CK(cudaStreamSynchronize(B->cs));
    }
    float ms = 0.f;
    cudaEventElapsedTime(&ms, t0, t1);
    if (status) {
        set_error("frw_batch_run: a kernel reported an internal limit");
        return FRW_E_KERNEL;
    }
    if (!results) return FRW_OK;
    std::vector<size_t> ord(cnt);
    for (size_t i = 0; i < cnt; i++) ord[i] = i;
    std::sort(ord.begin(), ord.end(), [&](size_t a, size_t b) { return row[a] < row[b]; });
    size_t k = 0;
    for (int j = 0; j < B->njobs; j++) {
        frw_result &R = results[j];
        const uint64_t W = B->walks[j];
        const double N = (double)W;
        if (stats[4 * j + 3] != W) {
            set_error("frw_batch_run: job " + std::to_string(j) + " finished " + std::to_string(stats[4 * j + 3]) +
                      " of " + std::to_string(W) + " walks");
            return FRW_E_KERNEL;
        }
        R.walks = W;
        R.escaped = stats[4 * j];
        R.aborted = stats[4 * j + 1];
        R.hops_total = stats[4 * j + 2];
        memcpy(R.gauss, &gauss[4 * (size_t)j], 32);
        R.kernel_ms = ms;
        const int64_t lo = B->acc_base[j], hi = lo + B->views[j].n;
        int64_t e = 0;
        uint64_t on_target = 0;
        while (k < cnt && row[ord[k]] < hi) {
            const size_t i = ord[k++];
            const int64_t cond = row[i] - lo;
            if (cond == B->targets[j]) on_target = n[i];
            if (e < R.capacity) {
                const double mean = s[i] / N;
                const double var = W > 1 ? std::max(s2[i] / N - mean * mean, 0.0) * N / (N - 1.0) : 0.0;
                if (R.conductor) R.conductor[e] = cond;
                if (R.hits) R.hits[e] = n[i];
                if (R.cap) R.cap[e] = mean;
                if (R.cap_se) R.cap_se[e] = sqrt(var / N);
                if (R.sum_w) R.sum_w[e] = s[i];
                if (R.sum_w2) R.sum_w2[e] = s2[i];
            }
            e++;
        }
        R.n_entries = e;
        R.fraction_other = W ? (double)(W - on_target) / N : 0.0;
    }
    return FRW_OK;
}

frw_status frw_batch_destroy(frw_batch *B) {
    if (!B) return FRW_OK;
    SetDev sd(B->device);
    free_batch(B);
    return FRW_OK;
}

}  // extern "C"
