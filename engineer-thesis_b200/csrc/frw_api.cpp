// frw_api.cpp -- the extern "C" boundary (include/frw.h) over the CUDA kernels.
//
// Host responsibilities only: argument checking, the reference's layout
// reader and bounds rule, device buffers and streams, and turning the
// device accumulators into the estimator's rows.  Every compute step runs on
// the device; there is no CPU path to fall back to.
#include <math.h>
#include <stdio.h>

#include <cmath>
#include <cstddef>
#include <string.h>
#include <time.h>

#include <algorithm>
#include <atomic>
#include <chrono>
#include <map>
#include <memory>
#include <mutex>
#include <new>
#include <thread>
#include <string>
#include <vector>

#include "frw_internal.h"
#include "layout_io.h"

namespace frw {
// Host copies of layout rects are kept for reuse when their layout is
// destroyed (a few buffers, 1 GiB at most), so that a layout created again at
// the same or a smaller size is written into memory already mapped instead of
// faulting in fresh pages.
class HostRectPool {
    std::mutex mu_;
    std::vector<std::pair<size_t, double *>> free_;  // (capacity in doubles, buffer)
    size_t held_ = 0;                                // doubles held in free_
    static constexpr size_t kMaxHeld = (1ull << 30) / sizeof(double);
    static constexpr size_t kMaxBuffers = 4;

  public:
    double *get(size_t n, size_t *cap) {
        {
            std::lock_guard<std::mutex> g(mu_);
            size_t best = free_.size();
            for (size_t i = 0; i < free_.size(); i++)
                if (free_[i].first >= n && (best == free_.size() || free_[i].first < free_[best].first)) best = i;
            if (best < free_.size() && free_[best].first <= 2 * n + 4096) {  // not a much larger buffer
                double *p = free_[best].second;
                *cap = free_[best].first;
                held_ -= *cap;
                free_.erase(free_.begin() + (std::ptrdiff_t)best);
                return p;
            }
        }
        *cap = n;
        return new (std::nothrow) double[n];
    }
    void put(double *p, size_t cap) {
        std::lock_guard<std::mutex> g(mu_);
        if (cap > kMaxHeld) {
            delete[] p;
            return;
        }
        free_.emplace_back(cap, p);
        held_ += cap;
        while (held_ > kMaxHeld || free_.size() > kMaxBuffers) {  // drop the oldest
            held_ -= free_.front().first;
            delete[] free_.front().second;
            free_.erase(free_.begin());
        }
    }
};
// never destroyed: layouts released during process exit may still return
// their buffers
HostRectPool &host_rects() {
    static HostRectPool *pool = new HostRectPool();
    return *pool;
}

struct HostRects {
    double *p = nullptr;
    size_t cap = 0;
    HostRects() = default;
    HostRects(const HostRects &) = delete;
    HostRects &operator=(const HostRects &) = delete;
    ~HostRects() {
        if (p) host_rects().put(p, cap);
    }
    bool acquire(size_t n) {
        p = host_rects().get(n, &cap);
        return p != nullptr;
    }
    double *get() const { return p; }
};
}  // namespace frw

struct frw_layout {
    int device = 0;
    int64_t n = 0;
    frw::HostRects rects;  // [4 n] layer order, as given
    double bounds[4] = {0, 0, 0, 0};
    frw::TreeBuffers T;
    frw::CellBuffers cells;
    frw::DevLayout dl{};
    float build_ms = 0.f;
    int leaf_max = frw::kDefaultLeafMax;
};

namespace frw {
namespace {

thread_local std::string g_err;

struct DeviceCtx {
    bool ready = false;
    int sms = 0;
    int cc_major = 0, cc_minor = 0;
    double *tables = nullptr;  // intg[201] | wx[200] | wy[200]
    int walk_bps[2] = {0, 0};  // resident walk blocks per SM by uniform start (occupancy query, cached)
};
std::mutex g_mu;
std::map<int, DeviceCtx> g_ctx;

// Keeps the caller's current device.
struct DeviceGuard {
    int prev = -1;
    explicit DeviceGuard(int dev) {
        if (cudaGetDevice(&prev) != cudaSuccess) prev = -1;
        if (prev != dev) cudaSetDevice(dev);
    }
    ~DeviceGuard() {
        int cur = -1;
        if (prev >= 0 && cudaGetDevice(&cur) == cudaSuccess && cur != prev) cudaSetDevice(prev);
    }
};

frw_status device_ctx(int dev, DeviceCtx **out) {
    std::lock_guard<std::mutex> lk(g_mu);
    DeviceCtx &c = g_ctx[dev];
    if (!c.ready) {
        int ndev = 0;
        cudaError_t e = cudaGetDeviceCount(&ndev);
        if (e != cudaSuccess || ndev <= dev || dev < 0) {
            set_error("no CUDA device " + std::to_string(dev) +
                      (e != cudaSuccess ? std::string(": ") + cudaGetErrorString(e) : std::string()));
            return FRW_E_DEVICE;
        }
        cudaDeviceProp p;
        FRW_CK(cudaGetDeviceProperties(&p, dev));
        if (p.major != 10) {
            set_error("device " + std::to_string(dev) + " is sm_" + std::to_string(p.major) +
                      std::to_string(p.minor) + "; this library is built for sm_100a only");
            return FRW_E_DEVICE;
        }
        c.sms = p.multiProcessorCount;
        c.cc_major = p.major;
        c.cc_minor = p.minor;
        DeviceGuard g(dev);
        double h[FRW_NSAMPLE + 1 + 2 * FRW_NSAMPLE];
        green_tables(nullptr, h, h + FRW_NSAMPLE + 1, h + 2 * FRW_NSAMPLE + 1);
        FRW_CK(cudaMalloc(&c.tables, sizeof(h)));
        FRW_CK(cudaMemcpy(c.tables, h, sizeof(h), cudaMemcpyHostToDevice));
        // keep stream-ordered allocations pooled between calls
        cudaMemPool_t pool;
        if (cudaDeviceGetDefaultMemPool(&pool, dev) == cudaSuccess) {
            uint64_t thr = UINT64_MAX;
            cudaMemPoolSetAttribute(pool, cudaMemPoolAttrReleaseThreshold, &thr);
        }
        c.ready = true;
    }
    *out = &c;
    return FRW_OK;
}

std::atomic<int64_t> g_wait_default_us{0};  // process-wide wait limit, microseconds (0: none)
thread_local double t_wait_ms = -1.0;         // limit of the call in progress (< 0: the default)

// Polls `ev` until it completes or the limit in force passes.
frw_status poll_event(cudaEvent_t ev, const char *what) {
    const double lim = wait_limit_ms();
    if (lim <= 0) {
        cudaError_t e = cudaEventSynchronize(ev);
        return e == cudaSuccess ? FRW_OK : cuda_fail(e, what);
    }
    const auto t0 = std::chrono::steady_clock::now();
    for (;;) {
        cudaError_t e = cudaEventQuery(ev);
        if (e == cudaSuccess) return FRW_OK;
        if (e != cudaErrorNotReady) return cuda_fail(e, what);
        const double ms = std::chrono::duration<double, std::milli>(std::chrono::steady_clock::now() - t0).count();
        if (ms > lim) {
            set_error(std::string(what) + ": the host wait limit of " + std::to_string(lim) +
                      " ms passed before the device finished (its work keeps running; buffers it uses are "
                      "released in stream order)");
            return FRW_E_TIMEOUT;
        }
        // short device steps (a layout build waits on several of tens of us)
        // are polled without sleeping, whose wake-up can take far longer than
        // the step on a loaded host; long waits sleep between polls
        if (ms < 2.0) std::this_thread::yield();
        else std::this_thread::sleep_for(std::chrono::microseconds(ms < 50.0 ? 20 : 200));
    }
}

// The message of a nonzero kernel status word.
frw_status status_error(uint32_t h) {
    if (h) {
        std::string m = "kernel reported:";
        if (h & kStCandOverflow) m += " near-tie candidate list overflow;";
        if (h & kStStackOverflow) m += " traversal stack overflow;";
        if (h & kStReplayCap) m += " bisection replay iteration bound exceeded;";
        if (h & kStBadInput) m += " invalid input;";
        if (h & kStDeviceWait) m += " a device-side wait passed its bound;";
        set_error(m);
        return FRW_E_KERNEL;
    }
    return FRW_OK;
}

// Reads the kernel status word (after the stream has drained).
frw_status check_status(const uint32_t *d_status, cudaStream_t st) {
    uint32_t h = 0;
    frw_status rc = read_back(&h, d_status, 4, st, "status read-back");
    if (rc) return rc;
    return status_error(h);
}

bool fp32_exact(double v) { return (double)(float)v == v && fabs(v) < 16777216.0; }

frw_status validate_opts(const frw_opts *o) {
    if (!o) return FRW_OK;
    if (o->struct_size != sizeof(frw_opts)) {
        set_error("frw_opts.struct_size mismatch (call frw_opts_default)");
        return FRW_E_ARG;
    }
    if (o->gauss_mode != FRW_GAUSS_SCALE && o->gauss_mode != FRW_GAUSS_OFFSET) {
        set_error("frw_opts.gauss_mode");
        return FRW_E_ARG;
    }
    if (o->start_mode != FRW_START_GREEN && o->start_mode != FRW_START_UNIFORM) {
        set_error("frw_opts.start_mode");
        return FRW_E_ARG;
    }
    if (!(o->gauss_param >= 0) || o->hop_cap < 1) {
        set_error("frw_opts.gauss_param / hop_cap");
        return FRW_E_ARG;
    }
    if (!(o->timeout_ms >= 0)) {
        set_error("frw_opts.timeout_ms must be >= 0");
        return FRW_E_ARG;
    }
    if (o->start_grid && o->start_mode != FRW_START_UNIFORM) {
        set_error("frw_opts.start_grid needs FRW_START_UNIFORM");
        return FRW_E_ARG;
    }
    return FRW_OK;
}

// Device scratch owned by one call, released on the stream at scope exit.
struct Scratch {
    cudaStream_t st;
    std::vector<void *> ptrs;
    explicit Scratch(cudaStream_t s) : st(s) {}
    template <typename T>
    cudaError_t get(T **p, size_t bytes) {
        cudaError_t e = cudaMallocAsync((void **)p, bytes ? bytes : 16, st);
        if (e == cudaSuccess) ptrs.push_back(*p);
        return e;
    }
    ~Scratch() {
        for (void *p : ptrs) cudaFreeAsync(p, st);
    }
};

struct WalkRun {
    // outputs
    uint64_t escaped = 0, aborted = 0, hops = 0, done = 0;
    double gauss[4] = {0, 0, 0, 0};
    float kernel_ms = 0.f;
    std::vector<int64_t> row;
    std::vector<unsigned long long> n;
    std::vector<double> s, s2;
};

// One job on one layout; records optional; host results optional.
frw_status run_walks(const frw_layout *lay, int64_t target, uint64_t first_walk, uint64_t walks,
                     uint64_t seed, const frw_opts &o, cudaStream_t st, int64_t *rec_end, int32_t *rec_hops,
                     int32_t *rec_bin, double *rec_w, WalkRun *out, double4 *rec_cv = nullptr,
                     int32_t *rec_q = nullptr) {
    DeviceCtx *ctx;
    frw_status rc = device_ctx(lay->device, &ctx);
    if (rc) return rc;
    if (target < 0 || target >= lay->n) {
        set_error("target conductor index out of range");
        return FRW_E_ARG;
    }
    // one scratch block: a header cleared with the per-conductor rows in one
    // memset, read back in one copy; compacted rows after it
    struct Hdr {
        double4 gauss;
        unsigned long long stats[4], counter, cnt;
        uint32_t status, pad;
        double4 tgt;
    };
    static_assert(sizeof(Hdr) % 16 == 0, "header keeps 16-byte alignment");
    const int64_t rows = lay->n;  // the kernel flushes every conductor it reaches
    const size_t R = (size_t)std::max<int64_t>(rows, 1);
    Scratch S(st);
    char *blk;
    FRW_CK(S.get(&blk, sizeof(Hdr) + R * 8 * (out ? 7 : 3)));
    Hdr *h = reinterpret_cast<Hdr *>(blk);
    unsigned long long *d_acc_n = reinterpret_cast<unsigned long long *>(blk + sizeof(Hdr));
    double *d_acc_s = reinterpret_cast<double *>(d_acc_n + R);
    double *d_acc_s2 = d_acc_s + R;
    double4 *d_tgt = &h->tgt, *d_gauss = &h->gauss;
    uint32_t *d_status = &h->status;
    unsigned long long *d_counter = &h->counter, *d_stats = h->stats;
    const double *r = lay->rects.get() + 4 * target;
    const double tg[4] = {r[0], r[1], r[2], r[3]};
    FRW_CK(cudaMemsetAsync(blk, 0, offsetof(Hdr, tgt), st));
    if (rows) FRW_CK(cudaMemsetAsync(d_acc_n, 0, R * 24, st));
    FRW_CK(cudaMemcpyAsync(d_tgt, tg, sizeof(tg), cudaMemcpyHostToDevice, st));
    rc = launch_gauss(lay->dl, (const double *)d_tgt, 1, o.gauss_mode, o.gauss_param, (double *)d_gauss,
                      d_status, st);
    if (rc) return rc;

    WalkParams P{};
    P.job0.L = lay->dl;
    P.job0.target = target;
    P.job0.walk_begin = 0;
    P.job0.walks = walks;
    P.job0.first_walk = first_walk;
    P.job0.acc_base = 0;
    P.job0.stream_id = o.stream_id;
    P.jobs = nullptr;
    P.gauss = d_gauss;
    P.njobs = 1;
    P.start_mode = o.start_mode;
    P.exact_perimeter = o.exact_perimeter;
    P.refill_min = o.refill_min > 0 ? o.refill_min : 1;
    P.start_grid = o.start_grid;
    P.start_strata = o.start_strata;
    P.hop_cap = o.hop_cap;
    P.permittivity = o.permittivity;
    P.seed = seed;
    P.total_walks = walks;
    P.counter = d_counter;
    P.acc_n = d_acc_n;
    P.acc_s = d_acc_s;
    P.acc_s2 = d_acc_s2;
    P.job_stats = d_stats;
    P.status = d_status;
    P.rec_end = rec_end;
    P.rec_hops = rec_hops;
    P.rec_bin = rec_bin;
    P.rec_w = rec_w;
    P.rec_cv = rec_cv;
    P.rec_q = rec_q;
    P.intg = ctx->tables;
    P.wx = ctx->tables + FRW_NSAMPLE + 1;
    P.wy = ctx->tables + 2 * FRW_NSAMPLE + 1;
    const int threads = 256;
    const int uni = o.start_mode == FRW_START_UNIFORM;
    if (!ctx->walk_bps[uni]) ctx->walk_bps[uni] = walk_max_blocks_per_sm(threads, false, uni);
    int bps = o.blocks_per_sm > 0 ? o.blocks_per_sm : ctx->walk_bps[uni];
    if (bps < 1) bps = 1;
    int blocks = ctx->sms * bps;
    const uint64_t need = (walks + threads - 1) / threads;
    if ((uint64_t)blocks > need) blocks = (int)std::max<uint64_t>(need, 1);

    Events ev(out ? 2 : 0);
    cudaEvent_t e0 = ev[0], e1 = ev[1];
    if (out) {
        if (!ev.ok(2)) return cuda_fail(cudaErrorUnknown, "cudaEventCreate");
        FRW_CK(cudaEventRecord(e0, st));
    }
    if (walks > 0) {
        rc = launch_walk(P, threads, blocks, st);
        if (rc) return rc;
    }
    if (!out) {
        // stream-ordered call: report kernel limits only when the caller syncs;
        // the status word is checked here synchronously to keep errors loud.
        return check_status(d_status, st);
    }
    FRW_CK(cudaEventRecord(e1, st));
    // compact nonzero rows (after the accumulators in the same block)
    int64_t *d_row = reinterpret_cast<int64_t *>(d_acc_s2 + R);
    unsigned long long *d_cn = reinterpret_cast<unsigned long long *>(d_row + R);
    double *d_cs = reinterpret_cast<double *>(d_cn + R);
    double *d_cs2 = d_cs + R;
    rc = launch_compact(d_acc_n, d_acc_s, d_acc_s2, rows, d_row, d_cn, d_cs, d_cs2, &h->cnt, st);
    if (rc) return rc;
    Hdr hh;
    rc = read_back(&hh, h, offsetof(Hdr, tgt), st, "walk results");
    if (rc) return rc;
    rc = status_error(hh.status);
    if (rc) return rc;
    const unsigned long long h_cnt = hh.cnt;
    memcpy(out->gauss, &hh.gauss, sizeof(out->gauss));
    out->row.resize(h_cnt);
    out->n.resize(h_cnt);
    out->s.resize(h_cnt);
    out->s2.resize(h_cnt);
    if (h_cnt) {
        FRW_CK(cudaMemcpyAsync(out->row.data(), d_row, h_cnt * 8, cudaMemcpyDeviceToHost, st));
        FRW_CK(cudaMemcpyAsync(out->n.data(), d_cn, h_cnt * 8, cudaMemcpyDeviceToHost, st));
        FRW_CK(cudaMemcpyAsync(out->s.data(), d_cs, h_cnt * 8, cudaMemcpyDeviceToHost, st));
        FRW_CK(cudaMemcpyAsync(out->s2.data(), d_cs2, h_cnt * 8, cudaMemcpyDeviceToHost, st));
        FRW_CK(cudaStreamSynchronize(st));
    }
    out->escaped = hh.stats[0];
    out->aborted = hh.stats[1];
    out->hops = hh.stats[2];
    out->done = hh.stats[3];
    cudaEventElapsedTime(&out->kernel_ms, e0, e1);
    if (out->done != walks) {
        set_error("walk kernel finished " + std::to_string(out->done) + " of " + std::to_string(walks) +
                  " walks");
        return FRW_E_KERNEL;
    }
    return FRW_OK;
}

}  // namespace

void set_error(const std::string &msg) { g_err = msg; }

frw_status status_word_error(uint32_t status) { return status_error(status); }

double wait_limit_ms() {
    return t_wait_ms >= 0 ? t_wait_ms : (double)g_wait_default_us.load(std::memory_order_relaxed) * 1e-3;
}

WaitScope::WaitScope(double ms) : prev(t_wait_ms) {
    if (ms > 0) t_wait_ms = ms;
}
WaitScope::~WaitScope() { t_wait_ms = prev; }

frw_status wait_event(cudaEvent_t ev, const char *what) { return poll_event(ev, what); }

frw_status wait_stream(cudaStream_t st, const char *what) {
    if (wait_limit_ms() <= 0) {
        cudaError_t e = cudaStreamSynchronize(st);
        return e == cudaSuccess ? FRW_OK : cuda_fail(e, what);
    }
    cudaEvent_t ev;
    cudaError_t e = cudaEventCreateWithFlags(&ev, cudaEventDisableTiming);
    if (e != cudaSuccess) return cuda_fail(e, what);
    e = cudaEventRecord(ev, st);
    frw_status rc = e == cudaSuccess ? poll_event(ev, what) : cuda_fail(e, what);
    cudaEventDestroy(ev);
    return rc;
}

frw_status read_back(void *host, const void *dev, size_t bytes, cudaStream_t st, const char *what, bool staged) {
    // small reads (sizes, counts, status words) go through a pinned buffer of
    // the calling thread: one copy behind the stream's work and one bounded
    // wait; a copy whose wait gave up may still land, so its buffer is left
    // to it
    constexpr size_t kStage = 4096;
    struct Stage {  // released when the thread ends
        void *p = nullptr;
        ~Stage() {
            if (p) cudaFreeHost(p);
        }
    };
    static thread_local Stage stage;
    if (staged && bytes <= kStage) {
        if (!stage.p && cudaMallocHost(&stage.p, kStage) != cudaSuccess) {
            stage.p = nullptr;
            cudaGetLastError();
        }
        if (stage.p) {
            cudaError_t e = cudaMemcpyAsync(stage.p, dev, bytes, cudaMemcpyDeviceToHost, st);
            if (e != cudaSuccess) return cuda_fail(e, what);
            frw_status rc = wait_stream(st, what);
            if (rc) {
                stage.p = nullptr;  // the copy may still land there: the buffer is left to it
                return rc;
            }
            memcpy(host, stage.p, bytes);
            return FRW_OK;
        }
    }
    frw_status rc = wait_stream(st, what);
    if (rc) return rc;
    cudaError_t e = cudaMemcpyAsync(host, dev, bytes, cudaMemcpyDeviceToHost, st);
    if (e == cudaSuccess) e = cudaStreamSynchronize(st);  // only this copy is left on the stream
    return e == cudaSuccess ? FRW_OK : cuda_fail(e, what);
}

// The FP64 host copy of a layout's rects (layer order), converted by host
// threads that run while the device checks the rects and builds the layout;
// join() before the copy is read or freed.
struct HostCopy {
    std::vector<std::thread> th;
    void start(const float *in, int64_t n, double *out) {
        const int64_t kChunk = 1 << 17;
        const int nt = (int)std::min<int64_t>((n + kChunk - 1) / kChunk,
                                              std::max<unsigned>(1, std::min(8u, std::thread::hardware_concurrency())));
        for (int t = 0; t < nt; t++)
            th.emplace_back([=] {
                const int64_t a = 4 * (n * t / nt), b = 4 * (n * (t + 1) / nt);
                for (int64_t i = a; i < b; i++) out[i] = in[i];
            });
    }
    void join() {
        for (auto &x : th) x.join();
        th.clear();
    }
    ~HostCopy() { join(); }
};

frw_status layout_view(const frw_layout *L, LayoutView *out) {
    if (!L) {
        set_error("null layout");
        return FRW_E_ARG;
    }
    out->dl = L->dl;
    out->device = L->device;
    out->n = L->n;
    out->rects = L->rects.get();
    return FRW_OK;
}

frw_status device_tables(int device, const double **tables, int *sms) {
    DeviceCtx *c;
    frw_status rc = device_ctx(device, &c);
    if (rc) return rc;
    *tables = c->tables;
    *sms = c->sms;
    return FRW_OK;
}

frw_status check_opts(const frw_opts *o) { return validate_opts(o); }

frw_status walk_records(const frw_layout *L, int64_t target, uint64_t first_walk, uint64_t walks, uint64_t seed,
                        const frw_opts &o, cudaStream_t st, int64_t *rec_end, double4 *rec_cv, double *rec_w,
                        int32_t *rec_q) {
    return run_walks(L, target, first_walk, walks, seed, o, st, rec_end, nullptr, nullptr, rec_w, nullptr, rec_cv,
                     rec_q);
}

frw_status cuda_fail(cudaError_t e, const char *what) {
    g_err = std::string(what) + ": " + cudaGetErrorName(e) + " (" + cudaGetErrorString(e) + ")";
    if (e == cudaErrorMemoryAllocation) return FRW_E_OOM;
    if (e == cudaErrorNoDevice || e == cudaErrorInsufficientDriver || e == cudaErrorInvalidDevice)
        return FRW_E_DEVICE;
    return FRW_E_CUDA;
}

}  // namespace frw

using namespace frw;

extern "C" {

const char *frw_version(void) { return "frw-b200 0.1 (sm_100a)"; }

const char *frw_last_error(void) { return g_err.c_str(); }

frw_status frw_device_check(int device) {
    DeviceCtx *c;
    return device_ctx(device, &c);
}

frw_status frw_set_wait_limit(double ms) {
    if (!(ms >= 0) || ms > 1e12) {
        set_error("frw_set_wait_limit: ms must be in [0, 1e12]");
        return FRW_E_ARG;
    }
    g_wait_default_us.store((int64_t)(ms * 1e3), std::memory_order_relaxed);
    return FRW_OK;
}

double frw_get_wait_limit(void) { return (double)g_wait_default_us.load(std::memory_order_relaxed) * 1e-3; }

frw_status frw_green_table(double *g, double *intg) {
    green_tables(g, intg, nullptr, nullptr);
    return FRW_OK;
}

void frw_opts_default(frw_opts *o) {
    memset(o, 0, sizeof(*o));
    o->struct_size = sizeof(frw_opts);
    o->gauss_mode = FRW_GAUSS_SCALE;
    o->gauss_param = 1.5;
    o->start_mode = FRW_START_GREEN;
    o->exact_perimeter = 0;
    o->hop_cap = 100000;
    o->permittivity = 8.854187817620e-12;
    o->stream_id = 0;
    o->threads_per_block = 256;
    o->blocks_per_sm = 0;
    o->refill_min = 1;
}

frw_status frw_layout_create(const float *rects, int64_t n, const double *bounds, int device, void *stream,
                             frw_layout **out) {
    if (!out || !rects || n <= 0) {
        set_error("frw_layout_create: null pointer or empty layout");
        return FRW_E_ARG;
    }
    *out = nullptr;
    if (n >= (1ll << 26)) {
        set_error("frw_layout_create: at most 2^26-1 rects per layout");
        return FRW_E_ARG;
    }
    if (bounds && (!(bounds[0] <= bounds[2] && bounds[1] <= bounds[3]) || !std::isfinite(bounds[0]) ||
                   !std::isfinite(bounds[1]) || !std::isfinite(bounds[2]) || !std::isfinite(bounds[3]))) {
        set_error("bounds invalid");
        return FRW_E_ARG;
    }
    DeviceCtx *ctx;
    frw_status rc = device_ctx(device, &ctx);
    if (rc) return rc;
    frw_layout *L = new frw_layout();
    L->device = device;
    L->n = n;
    if (!L->rects.acquire((size_t)n * 4)) {
        delete L;
        set_error("frw_layout_create: host memory for the rect copy");
        return FRW_E_OOM;
    }
    const double *b = L->bounds;
    DeviceGuard g(device);
    cudaStream_t st = (cudaStream_t)stream;
    float4 *d_in = nullptr;
    HostCopy copy;
    auto fail = [&](frw_status r) {
        copy.join();
        if (d_in) cudaFreeAsync(d_in, st);
        free_tree(&L->T, st);
        free_cells(&L->cells, st);
        delete L;
        return r;
    };
    cudaError_t e = cudaMallocAsync(&d_in, (size_t)n * 16, st);
    if (e != cudaSuccess) return fail(cuda_fail(e, "cudaMallocAsync rects"));
    e = cudaMemcpyAsync(d_in, rects, (size_t)n * 16, cudaMemcpyHostToDevice, st);
    if (e != cudaSuccess) return fail(cuda_fail(e, "upload rects"));
    copy.start(rects, n, L->rects.get());
    {
        // the rects are checked on the device; errors name the first offending rect
        int64_t bad = -1;
        int why = 0;
        double ext[4];
        rc = check_rects(d_in, n, bounds, ctx->sms, st, &bad, &why, ext);
        if (rc) return fail(rc);
        if (bad >= 0) {
            const std::string r = "rect " + std::to_string(bad);
            set_error(why == 1 ? r + ": coordinate not finite or |c| >= 2^24"
                               : why == 2 ? r + ": inverted (need x0 <= x1 and y0 <= y1)" : r + " lies outside the bounds");
            return fail(FRW_E_ARG);
        }
        if (bounds) memcpy(L->bounds, bounds, 4 * sizeof(double));
        else bounds_from_extent(ext[0], ext[1], ext[2], ext[3], L->bounds);
    }
    rc = build_tree(d_in, (int32_t)n, L->bounds, L->leaf_max, st, &L->T, &L->build_ms);
    if (rc) return fail(rc);
    cudaFreeAsync(d_in, st);
    d_in = nullptr;
    DevLayout &dl = L->dl;
    dl.rects = L->T.rects;
    dl.ids = L->T.ids;
    dl.nbox = L->T.nbox;
    dl.nref = L->T.nref;
    dl.bx0 = b[0];
    dl.by0 = b[1];
    dl.bx1 = b[2];
    dl.by1 = b[3];
    {
        // drawBiggestSquareAtPoint: dist = (H > W ? H : W) * 0.05
        const double bw = b[2] - b[0], bh = b[3] - b[1];
        double dist = (bh > bw) ? bh : bw;
        dist *= 0.05;
        dl.dist0 = dist;
        // the replay's bisection halves dist while it is above MIN_DIST
        // ((double)0.095f; halving a positive normal double is exact)
        int halvings = 0;
        for (double d = dist; d > (double)0.095f && halvings < 64; d *= 0.5) halvings++;
        dl.halvings = halvings;
        // tie window: every box of a replay has coordinates below
        // M = 4 * max(|bounds|, W, H) + 16 after <= 256 roundings of at most
        // M * 2^-53 each, i.e. within M * 2^-45; delta = M * 2^-40 leaves 32x.
        double M = std::max(std::max(fabs(b[0]), fabs(b[1])), std::max(fabs(b[2]), fabs(b[3])));
        // FP32 pre-filter: a point inside the bounds rounds to float within
        // ulp(Mb)/2 and a float difference of two such values within ulp(Mb),
        // so FP32 gaps are within 1.5 ulp(Mb) of the exact ones and the
        // rounded limit within another ulp; 4 ulp(Mb) is a safe margin.
        const double Mb = std::max(M, 1.0);
        int ex = 0;
        frexp(Mb, &ex);  // Mb in [2^(ex-1), 2^ex)
        dl.slack = (float)ldexp(4.0, ex - 1 - 23);
        M = 4.0 * std::max(M, std::max(bw, bh)) + 16.0;
        dl.delta = ldexp(M, -40);
    }
    dl.n = (int32_t)n;
    dl.nodes = L->T.nodes;
    rc = build_cells(dl, kDefaultCellsPerRect, kDefaultCellMax, st, &L->cells);
    if (rc) return fail(rc);
    attach_cells(dl, L->cells);
    copy.join();
    *out = L;
    return FRW_OK;
}

frw_status frw_parse_layout(const char *path, int layer, double *rects_out, int64_t capacity, int64_t *n_out,
                            double *bounds_out, int32_t *layers_out) {
    if (!path || !n_out) {
        set_error("frw_parse_layout: null argument");
        return FRW_E_ARG;
    }
    *n_out = 0;
    std::vector<double> r;
    int nl = 0;
    frw_status rc = parse_layout_file(path, layer, &r, &nl);
    if (layers_out) *layers_out = nl;
    if (rc) return rc;
    const int64_t n = (int64_t)r.size() / 4;
    *n_out = n;
    if (bounds_out) {
        if (n) reference_bounds(r.data(), n, bounds_out);
        else memset(bounds_out, 0, 4 * sizeof(double));
    }
    if (rects_out) {
        if (capacity < n) {
            set_error("frw_parse_layout: layer " + std::to_string(layer) + " has " + std::to_string(n) +
                      " rects, capacity " + std::to_string(capacity));
            return FRW_E_ARG;
        }
        if (n) memcpy(rects_out, r.data(), r.size() * sizeof(double));
    }
    return FRW_OK;
}

frw_status frw_layout_from_file(const char *path, int layer, int device, frw_layout **out) {
    if (!path || !out) {
        set_error("frw_layout_from_file: null argument");
        return FRW_E_ARG;
    }
    std::vector<double> r;
    frw_status rc = parse_layout_file(path, layer, &r, nullptr);
    if (rc) return rc;
    const int64_t n = (int64_t)r.size() / 4;
    if (n == 0) {
        set_error(std::string(path) + ": layer " + std::to_string(layer) + " has no rects");
        return FRW_E_ARG;
    }
    std::vector<float> f(r.size());
    for (size_t i = 0; i < r.size(); i++) {
        if (!fp32_exact(r[i])) {
            set_error(std::string(path) + ": coordinate " + std::to_string(r[i]) +
                      " is not exactly representable in FP32 (|c| < 2^24 required)");
            return FRW_E_ARG;
        }
        f[i] = (float)r[i];
    }
    double b[4];
    reference_bounds(r.data(), n, b);
    return frw_layout_create(f.data(), n, b, device, nullptr, out);
}

frw_status frw_layout_destroy(frw_layout *L) {
    if (!L) return FRW_OK;
    DeviceGuard g(L->device);
    // like cudaFree: nothing on the device may still read the layout
    cudaError_t e = cudaDeviceSynchronize();
    free_tree(&L->T, nullptr);
    free_cells(&L->cells, nullptr);
    delete L;
    FRW_CK(e);
    return FRW_OK;
}

frw_status frw_layout_info_get(const frw_layout *L, frw_layout_info *info) {
    if (!L || !info) {
        set_error("null argument");
        return FRW_E_ARG;
    }
    info->n_rects = L->n;
    info->n_nodes = L->T.nodes;
    info->depth = L->T.depth;
    info->leaf_max = L->leaf_max;
    memcpy(info->bounds, L->bounds, sizeof(info->bounds));
    info->device_bytes = L->T.bytes;
    info->device = L->device;
    info->build_ms = L->build_ms;
    return FRW_OK;
}

frw_status frw_layout_set_cells(frw_layout *L, double cells_per_rect, int max_per_cell, void *stream) {
    if (!L) {
        set_error("null layout");
        return FRW_E_ARG;
    }
    if (cells_per_rect < 0 || !std::isfinite(cells_per_rect)) {
        set_error("frw_layout_set_cells: cells_per_rect must be finite and >= 0");
        return FRW_E_ARG;
    }
    DeviceGuard g(L->device);
    cudaStream_t st = (cudaStream_t)stream;
    FRW_CK(cudaStreamSynchronize(st));
    CellBuffers c;
    if (cells_per_rect > 0) {
        DevLayout tree_only = L->dl;
        tree_only.cells = nullptr;
        frw_status rc = build_cells(tree_only, cells_per_rect, max_per_cell > 0 ? max_per_cell : kDefaultCellMax,
                                    st, &c);
        if (rc) return rc;
    }
    FRW_CK(cudaDeviceSynchronize());  // no launch may still read the old lists
    free_cells(&L->cells, nullptr);
    L->cells = c;
    L->dl.cells = nullptr;
    L->dl.tree_points = 1;
    if (c.cells) attach_cells(L->dl, c);
    return FRW_OK;
}

frw_status frw_layout_cells_info(const frw_layout *L, frw_cells_info *info) {
    if (!L || !info) {
        set_error("null argument");
        return FRW_E_ARG;
    }
    const CellBuffers &c = L->cells;
    info->cells = c.ncells;
    info->nx = c.nx;
    info->ny = c.ny;
    info->cell_side = c.side;
    info->entries = c.entries;
    info->overflow_cells = c.overflow;
    info->device_bytes = c.bytes;
    info->build_ms = c.build_ms;
    return FRW_OK;
}

frw_status frw_layout_rects(const frw_layout *L, double *out) {
    if (!L || !out) {
        set_error("null argument");
        return FRW_E_ARG;
    }
    memcpy(out, L->rects.get(), (size_t)L->n * 4 * sizeof(double));
    return FRW_OK;
}

frw_status frw_query_batch(const frw_layout *L, const double *pts, int64_t n, double *sq, int64_t *hit, int mem,
                           void *stream) {
    if (!L || (n > 0 && (!pts || !sq || !hit)) || n < 0) {
        set_error("frw_query_batch: bad arguments");
        return FRW_E_ARG;
    }
    if (n == 0) return FRW_OK;
    if (mem == FRW_MEM_DEVICE && (((uintptr_t)pts & 15) || ((uintptr_t)sq & 31) || ((uintptr_t)hit & 7))) {
        set_error("frw_query_batch: device buffers must be aligned (points 16 B, squares 32 B, hits 8 B)");
        return FRW_E_ARG;
    }
    DeviceGuard g(L->device);
    cudaStream_t st = (cudaStream_t)stream;
    Scratch S(st);
    uint32_t *d_status;
    FRW_CK(S.get(&d_status, 4));
    FRW_CK(cudaMemsetAsync(d_status, 0, 4, st));
    const double *dp = pts;
    double *ds = sq;
    int64_t *dh = hit;
    if (mem == FRW_MEM_HOST) {
        double *a, *b;
        int64_t *c;
        FRW_CK(S.get(&a, n * 16));
        FRW_CK(S.get(&b, n * 32));
        FRW_CK(S.get(&c, n * 8));
        FRW_CK(cudaMemcpyAsync(a, pts, n * 16, cudaMemcpyHostToDevice, st));
        dp = a;
        ds = b;
        dh = c;
    }
    frw_status rc = launch_query(L->dl, dp, n, ds, dh, d_status, st);
    if (rc) return rc;
    rc = check_status(d_status, st);  // bounded wait for the queries, then their status
    if (rc) return rc;
    if (mem == FRW_MEM_HOST) {
        FRW_CK(cudaMemcpyAsync(sq, ds, n * 32, cudaMemcpyDeviceToHost, st));
        FRW_CK(cudaMemcpyAsync(hit, dh, n * 8, cudaMemcpyDeviceToHost, st));
        FRW_CK(cudaStreamSynchronize(st));
    }
    return FRW_OK;
}

frw_status frw_box_collides_batch(const frw_layout *L, const double *boxes, int64_t n, const double *ignore,
                                  uint8_t *out, int mem, void *stream) {
    if (!L || (n > 0 && (!boxes || !out)) || n < 0) {
        set_error("frw_box_collides_batch: bad arguments");
        return FRW_E_ARG;
    }
    if (n == 0) return FRW_OK;
    if (mem == FRW_MEM_DEVICE && ((uintptr_t)boxes & 31)) {
        set_error("frw_box_collides_batch: device boxes must be 32-byte aligned");
        return FRW_E_ARG;
    }
    DeviceGuard g(L->device);
    cudaStream_t st = (cudaStream_t)stream;
    Scratch S(st);
    uint32_t *d_status;
    FRW_CK(S.get(&d_status, 4));
    FRW_CK(cudaMemsetAsync(d_status, 0, 4, st));
    const double *db = boxes;
    uint8_t *dout = out;
    if (mem == FRW_MEM_HOST) {
        double *a;
        uint8_t *c;
        FRW_CK(S.get(&a, n * 32));
        FRW_CK(S.get(&c, n));
        FRW_CK(cudaMemcpyAsync(a, boxes, n * 32, cudaMemcpyHostToDevice, st));
        db = a;
        dout = c;
    }
    frw_status rc = launch_box_collides(L->dl, db, n, ignore != nullptr, ignore, dout, d_status, st);
    if (rc) return rc;
    rc = check_status(d_status, st);
    if (rc) return rc;
    if (mem == FRW_MEM_HOST) {
        FRW_CK(cudaMemcpyAsync(out, dout, n, cudaMemcpyDeviceToHost, st));
        FRW_CK(cudaStreamSynchronize(st));
    }
    return FRW_OK;
}

frw_status frw_gauss_surface(const frw_layout *L, int64_t target, const frw_opts *opts, double out[4],
                             void *stream) {
    frw_opts o;
    frw_opts_default(&o);
    if (opts) o = *opts;
    frw_status rc = validate_opts(&o);
    if (rc) return rc;
    WaitScope ws(o.timeout_ms);
    if (!L || !out || target < 0 || target >= L->n) {
        set_error("frw_gauss_surface: bad arguments");
        return FRW_E_ARG;
    }
    DeviceGuard g(L->device);
    cudaStream_t st = (cudaStream_t)stream;
    Scratch S(st);
    double *d_t, *d_o;
    uint32_t *d_status;
    FRW_CK(S.get(&d_t, 32));
    FRW_CK(S.get(&d_o, 32));
    FRW_CK(S.get(&d_status, 4));
    FRW_CK(cudaMemsetAsync(d_status, 0, 4, st));
    FRW_CK(cudaMemcpyAsync(d_t, L->rects.get() + 4 * target, 32, cudaMemcpyHostToDevice, st));
    rc = launch_gauss(L->dl, d_t, 1, o.gauss_mode, o.gauss_param, d_o, d_status, st);
    if (rc) return rc;
    rc = check_status(d_status, st);
    if (rc) return rc;
    return read_back(out, d_o, 32, st, "frw_gauss_surface");
}

frw_status frw_walk(const frw_layout *L, int64_t target, uint64_t walks, uint64_t seed, const frw_opts *opts,
                    frw_result *res, void *stream) {
    frw_opts o;
    frw_opts_default(&o);
    if (opts) o = *opts;
    frw_status rc = validate_opts(&o);
    if (rc) return rc;
    WaitScope ws(o.timeout_ms);
    if (!L || !res) {
        set_error("frw_walk: null argument");
        return FRW_E_ARG;
    }
    DeviceGuard g(L->device);
    WalkRun R;
    rc = run_walks(L, target, o.first_walk, walks, seed, o, (cudaStream_t)stream, nullptr, nullptr, nullptr, nullptr,
                   &R);
    if (rc) return rc;
    res->walks = walks;
    res->escaped = R.escaped;
    res->aborted = R.aborted;
    res->hops_total = R.hops;
    memcpy(res->gauss, R.gauss, sizeof(res->gauss));
    res->kernel_ms = R.kernel_ms;
    std::vector<size_t> ord(R.row.size());
    for (size_t i = 0; i < ord.size(); i++) ord[i] = i;
    std::sort(ord.begin(), ord.end(), [&](size_t a, size_t b) { return R.row[a] < R.row[b]; });
    uint64_t on_target = 0;
    res->n_entries = (int64_t)ord.size();
    const double N = (double)walks;
    for (size_t k = 0; k < ord.size(); k++) {
        const size_t i = ord[k];
        if (R.row[i] == target) on_target = R.n[i];
        if ((int64_t)k >= res->capacity) continue;
        const double mean = R.s[i] / N;
        const double var = walks > 1 ? std::max(R.s2[i] / N - mean * mean, 0.0) * N / (N - 1.0) : 0.0;
        if (res->conductor) res->conductor[k] = R.row[i];
        if (res->hits) res->hits[k] = R.n[i];
        if (res->cap) res->cap[k] = mean;
        if (res->cap_se) res->cap_se[k] = sqrt(var / N);
        if (res->sum_w) res->sum_w[k] = R.s[i];
        if (res->sum_w2) res->sum_w2[k] = R.s2[i];
    }
    res->fraction_other = walks ? (double)(walks - on_target) / N : 0.0;
    return FRW_OK;
}

frw_status frw_walk_device(const frw_layout *L, int64_t target, uint64_t walks, uint64_t seed, const frw_opts *opts,
                           uint64_t *hits, double *sum_w, double *sum_w2, uint64_t *stats, uint32_t *status,
                           void *stream) {
    frw_opts o;
    frw_opts_default(&o);
    if (opts) o = *opts;
    frw_status rc = validate_opts(&o);
    if (rc) return rc;
    if (!L || !hits || !sum_w || !sum_w2 || !stats || !status) {
        set_error("frw_walk_device: null argument");
        return FRW_E_ARG;
    }
    return walk_device_rows(L, target, walks, seed, o, hits, sum_w, sum_w2, stats, status, nullptr, nullptr,
                            (cudaStream_t)stream);
}

}  // extern "C"

// The walks of frw_walk_device into device rows, optionally with the control
// variate's sums; no host wait.
frw_status frw::walk_device_rows(const frw_layout *L, int64_t target, uint64_t walks, uint64_t seed,
                                 const frw_opts &o, uint64_t *hits, double *sum_w, double *sum_w2, uint64_t *stats,
                                 uint32_t *status, const float *cv_phi, double *cv_sums, cudaStream_t st) {
    frw_status rc = FRW_OK;
    if (target < 0 || target >= L->n) {
        set_error("target conductor index out of range");
        return FRW_E_ARG;
    }
    DeviceGuard g(L->device);
    DeviceCtx *ctx;
    rc = device_ctx(L->device, &ctx);
    if (rc) return rc;
    Scratch S(st);
    char *blk;
    FRW_CK(S.get(&blk, 64 + 32));  // counter, then the target rect (32 B) and its Gaussian surface
    unsigned long long *d_counter = reinterpret_cast<unsigned long long *>(blk);
    double4 *d_tgt = reinterpret_cast<double4 *>(blk + 32);
    double4 *d_gauss = reinterpret_cast<double4 *>(blk + 64);
    const double *r = L->rects.get() + 4 * target;
    const double tg[4] = {r[0], r[1], r[2], r[3]};
    FRW_CK(cudaMemsetAsync(d_counter, 0, 8, st));
    FRW_CK(cudaMemcpyAsync(d_tgt, tg, sizeof(tg), cudaMemcpyHostToDevice, st));
    rc = launch_gauss(L->dl, (const double *)d_tgt, 1, o.gauss_mode, o.gauss_param, (double *)d_gauss, status, st);
    if (rc || walks == 0) return rc;
    WalkParams P{};
    P.job0.L = L->dl;
    P.job0.target = target;
    P.job0.walks = walks;
    P.job0.first_walk = o.first_walk;
    P.job0.stream_id = o.stream_id;
    P.gauss = d_gauss;
    P.njobs = 1;
    P.start_mode = o.start_mode;
    P.exact_perimeter = o.exact_perimeter;
    P.refill_min = o.refill_min > 0 ? o.refill_min : 1;
    P.start_grid = o.start_grid;
    P.start_strata = o.start_strata;
    P.hop_cap = o.hop_cap;
    P.permittivity = o.permittivity;
    P.seed = seed;
    P.total_walks = walks;
    P.counter = d_counter;
    P.acc_n = reinterpret_cast<unsigned long long *>(hits);
    P.acc_s = sum_w;
    P.acc_s2 = sum_w2;
    P.job_stats = reinterpret_cast<unsigned long long *>(stats);
    P.status = status;
    P.intg = ctx->tables;
    P.wx = ctx->tables + FRW_NSAMPLE + 1;
    P.wy = ctx->tables + 2 * FRW_NSAMPLE + 1;
    P.cv_phi = cv_phi;
    P.cv_sums = cv_sums;
    const int uni = o.start_mode == FRW_START_UNIFORM;
    if (!ctx->walk_bps[uni]) ctx->walk_bps[uni] = walk_max_blocks_per_sm(256, false, uni);
    int bps = o.blocks_per_sm > 0 ? o.blocks_per_sm : std::max(ctx->walk_bps[uni], 1);
    int blocks = ctx->sms * bps;
    const uint64_t need = (walks + 255) / 256;
    if ((uint64_t)blocks > need) blocks = (int)std::max<uint64_t>(need, 1);
    return launch_walk(P, 256, blocks, st);
}

extern "C" {

frw_status frw_rows_compact(const frw_layout *L, const uint64_t *hits, const double *sum_w, const double *sum_w2,
                            int64_t capacity, int64_t *idx, uint64_t *out_hits, double *out_sum_w, double *out_sum_w2,
                            uint64_t *count, void *stream) {
    if (!L || !hits || !sum_w || !sum_w2 || !count || capacity < 0 ||
        (capacity > 0 && (!idx || !out_hits || !out_sum_w || !out_sum_w2))) {
        set_error("frw_rows_compact: null argument or negative capacity");
        return FRW_E_ARG;
    }
    DeviceGuard g(L->device);
    cudaStream_t st = (cudaStream_t)stream;
    FRW_CK(cudaMemsetAsync(count, 0, 8, st));
    return launch_compact(reinterpret_cast<const unsigned long long *>(hits), sum_w, sum_w2, L->n, idx,
                          reinterpret_cast<unsigned long long *>(out_hits), out_sum_w, out_sum_w2,
                          reinterpret_cast<unsigned long long *>(count), st, capacity);
}

frw_status frw_walk_trace(const frw_layout *L, int64_t target, uint64_t first_walk, uint64_t walks, uint64_t seed,
                          const frw_opts *opts, int64_t *end, int32_t *hops, int32_t *bin1, double *weight,
                          int mem, void *stream) {
    frw_opts o;
    frw_opts_default(&o);
    if (opts) o = *opts;
    frw_status rc = validate_opts(&o);
    if (rc) return rc;
    WaitScope ws(o.timeout_ms);
    if (!L) {
        set_error("frw_walk_trace: null layout");
        return FRW_E_ARG;
    }
    DeviceGuard g(L->device);
    cudaStream_t st = (cudaStream_t)stream;
    Scratch S(st);
    int64_t *de;
    int32_t *dh, *db;
    double *dw;
    // the kernel writes all four records; absent ones go to scratch
    const bool host = mem == FRW_MEM_HOST;
    if (host || !end) FRW_CK(S.get(&de, walks * 8)); else de = end;
    if (host || !hops) FRW_CK(S.get(&dh, walks * 4)); else dh = hops;
    if (host || !bin1) FRW_CK(S.get(&db, walks * 4)); else db = bin1;
    if (host || !weight) FRW_CK(S.get(&dw, walks * 8)); else dw = weight;
    rc = run_walks(L, target, first_walk, walks, seed, o, st, de, dh, db, dw, nullptr);
    if (rc) return rc;
    if (host) {
        if (end) FRW_CK(cudaMemcpyAsync(end, de, walks * 8, cudaMemcpyDeviceToHost, st));
        if (hops) FRW_CK(cudaMemcpyAsync(hops, dh, walks * 4, cudaMemcpyDeviceToHost, st));
        if (bin1) FRW_CK(cudaMemcpyAsync(bin1, db, walks * 4, cudaMemcpyDeviceToHost, st));
        if (weight) FRW_CK(cudaMemcpyAsync(weight, dw, walks * 8, cudaMemcpyDeviceToHost, st));
        FRW_CK(cudaStreamSynchronize(st));
    }
    return FRW_OK;
}

frw_status frw_avg_path_len(const char *path, int64_t iter_num, int64_t rect_id, int layer, uint64_t seed,
                            int device, const char *hist_path, double *fraction) {
    if (iter_num <= 0 || !fraction) {
        set_error("frw_avg_path_len: iter_num must be positive");
        return FRW_E_ARG;
    }
    frw_layout *L = nullptr;
    frw_status rc = frw_layout_from_file(path, layer, device, &L);
    if (rc) return rc;
    if (rect_id < 0 || rect_id >= L->n) {
        frw_layout_destroy(L);
        set_error("rect id out of range");
        return FRW_E_ARG;
    }
    frw_opts o;
    frw_opts_default(&o);  // reference start and Gaussian surface
    std::vector<int64_t> cond(L->n);
    std::vector<uint64_t> hits(L->n);
    frw_result r{};
    r.capacity = L->n;
    r.conductor = cond.data();
    r.hits = hits.data();
    rc = frw_walk(L, rect_id, (uint64_t)iter_num, seed, &o, &r, nullptr);
    if (rc == FRW_OK) {
        *fraction = r.fraction_other;
        if (hist_path) {
            // the reference's "<ts>wyniki.txt" layout (Cuda/getAvgPathLenCUDA.cu:23-48):
            // one line per rect reached, then the escaped share
            FILE *f = fopen(hist_path, "w");
            if (!f) {
                set_error(std::string("cannot write ") + hist_path);
                rc = FRW_E_IO;
            } else {
                fprintf(f, "[GPU]\n");
                if (r.escaped)
                    fprintf(f, "Ile scie\xc5\xbc" "ek wysz\xc5\x82o poza granice warstwy: %g%%\n",
                            (float)r.escaped / (float)iter_num * 100);
                for (int64_t k = 0; k < std::min(r.n_entries, r.capacity); k++) {
                    const double *q = L->rects.get() + 4 * cond[k];
                    fprintf(f, "%g %g %g %g: %g%%\n", q[0], q[1], q[2], q[3],
                            ((float)hits[k] / (float)iter_num) * 100);
                }
                fclose(f);
            }
        }
    }
    frw_layout_destroy(L);
    return rc;
}

frw_status frw_generate_layout(uint64_t seed, int64_t n, double domain, int32_t wmin, int32_t wmax, double gap,
                               float *out) {
    if (!out) {
        set_error("null output");
        return FRW_E_ARG;
    }
    return generate_layout(seed, n, domain, wmin, wmax, gap, out);
}

frw_status frw_write_layout(const char *path, const float *rects, int64_t n, const char *name) {
    if (!path || !rects || n <= 0) {
        set_error("frw_write_layout: bad arguments");
        return FRW_E_ARG;
    }
    return write_layout(path, rects, n, name);
}

}  // extern "C"
