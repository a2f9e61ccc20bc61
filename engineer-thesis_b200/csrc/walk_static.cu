// walk_static.cu -- frw_walk_trace_static: the per-walk trace with its device
// scratch in a fixed, file-scope array instead of allocations.
//
// Who needs it: callers that may not allocate device memory during the
// call -- host applications that hand every byte of the GPU to their own
// pool allocator, real-time loops that forbid allocator latency or
// synchronisation, and plugins whose host process owns the CUDA context.
// They pass the layout, the walk range and four device output arrays; the
// call allocates neither device nor host memory on its success path.
//
// The scratch of the walk kernel (walk counter, per-job totals, status word,
// target and Gaussian rects, and the per-conductor rows the kernel flushes
// into) lives in g_walk_scratch below, sized for layouts of at most
// kStaticMaxRects conductors (128 B + 24 B per conductor = 1.5 MiB).  Every
// GPU that loads the library holds this array until the process exits.
#include <mutex>

#include "frw_internal.h"

namespace frw {
namespace {

constexpr int64_t kStaticMaxRects = 1 << 16;
constexpr size_t kHead = 128;  // counter 8 | job stats 32 | status 4 | pad | target 32 @64 | gauss 32 @96
constexpr size_t kStaticBytes = kHead + 24 * (size_t)kStaticMaxRects;

static __device__ __align__(256) unsigned char g_walk_scratch[kStaticBytes];

constexpr int kMaxDevices = 64;
std::mutex g_mu;
unsigned char *g_addr[kMaxDevices];  // device address of g_walk_scratch, per device

// Resolves the array's device address once per device (the host-side name
// g_walk_scratch is only a stand-in and must never be passed to a kernel).
frw_status scratch_address(int dev, unsigned char **out) {
    if (dev < 0 || dev >= kMaxDevices) {
        set_error("frw_walk_trace_static: device index out of range");
        return FRW_E_ARG;
    }
    std::lock_guard<std::mutex> lk(g_mu);
    if (!g_addr[dev]) {
        void *p = nullptr;
        cudaError_t e = cudaGetSymbolAddress(&p, g_walk_scratch);
        if (e != cudaSuccess) return cuda_fail(e, "cudaGetSymbolAddress(g_walk_scratch)");
        g_addr[dev] = (unsigned char *)p;
    }
    *out = g_addr[dev];
    return FRW_OK;
}

}  // namespace
}  // namespace frw

using namespace frw;

extern "C" frw_status frw_walk_trace_static(const frw_layout *layout, int64_t target, uint64_t first_walk,
                                            uint64_t walks, uint64_t seed, const frw_opts *opts, int64_t *end,
                                            int32_t *hops, int32_t *bin1, double *weight, void *stream) {
    frw_opts o;
    frw_opts_default(&o);
    if (opts) o = *opts;
    frw_status rc = check_opts(&o);
    if (rc) return rc;
    LayoutView v;
    rc = layout_view(layout, &v);
    if (rc) return rc;
    if (v.n > kStaticMaxRects) {
        set_error("frw_walk_trace_static: the layout has more than 65,536 rects (the static scratch limit); "
                  "use frw_walk_trace");
        return FRW_E_ARG;
    }
    if (target < 0 || target >= v.n || !end || !hops || !bin1 || !weight) {
        set_error("frw_walk_trace_static: target out of range or a null output array");
        return FRW_E_ARG;
    }
    if (walks == 0) return FRW_OK;
    int prev = -1;
    if (cudaGetDevice(&prev) != cudaSuccess) prev = -1;
    if (prev != v.device) {
        cudaError_t e = cudaSetDevice(v.device);
        if (e != cudaSuccess) return cuda_fail(e, "cudaSetDevice");
    }
    cudaStream_t st = (cudaStream_t)stream;
    unsigned char *base = nullptr;
    const double *tables = nullptr;
    int sms = 0;
    rc = scratch_address(v.device, &base);
    if (!rc) rc = device_tables(v.device, &tables, &sms);
    unsigned long long *counter = (unsigned long long *)base;
    unsigned long long *stats = (unsigned long long *)(base + 8);
    uint32_t *status = (uint32_t *)(base + 40);
    double *tgt = (double *)(base + 64);
    double4 *gauss = (double4 *)(base + 96);
    unsigned long long *acc_n = (unsigned long long *)(base + kHead);
    double *acc_s = (double *)(base + kHead + 8 * (size_t)v.n);
    double *acc_s2 = (double *)(base + kHead + 16 * (size_t)v.n);
    cudaError_t e = cudaSuccess;
    // the array keeps the previous call's contents: clear what must start at 0
    if (!rc) e = cudaMemsetAsync(base, 0, kHead + 24 * (size_t)v.n, st);
    if (!rc && e == cudaSuccess)
        e = cudaMemcpyAsync(tgt, v.rects + 4 * target, 32, cudaMemcpyHostToDevice, st);
    if (!rc && e != cudaSuccess) rc = cuda_fail(e, "frw_walk_trace_static: scratch set-up");
    if (!rc) rc = launch_gauss(v.dl, tgt, 1, o.gauss_mode, o.gauss_param, (double *)gauss, status, st);
    if (!rc) {
        WalkParams P{};
        P.job0.L = v.dl;
        P.job0.target = target;
        P.job0.walks = walks;
        P.job0.first_walk = first_walk;
        P.job0.stream_id = o.stream_id;
        P.gauss = gauss;
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
        P.counter = counter;
        P.acc_n = acc_n;
        P.acc_s = acc_s;
        P.acc_s2 = acc_s2;
        P.job_stats = stats;
        P.status = status;
        P.rec_end = end;
        P.rec_hops = hops;
        P.rec_bin = bin1;
        P.rec_w = weight;
        P.intg = tables;
        P.wx = tables + FRW_NSAMPLE + 1;
        P.wy = tables + 2 * FRW_NSAMPLE + 1;
        int bps = o.blocks_per_sm > 0 ? o.blocks_per_sm
                                      : walk_max_blocks_per_sm(256, false, o.start_mode == FRW_START_UNIFORM);
        if (bps < 1) bps = 1;
        uint64_t blocks = (uint64_t)sms * bps, need = (walks + 255) / 256;
        if (blocks > need) blocks = need;
        rc = launch_walk(P, 256, (int)blocks, st);
    }
    if (!rc) {
        // status word and completed-walk count (host stack, no allocation),
        // read once the stream has drained within the call's wait limit
        WaitScope ws(o.timeout_ms);
        uint32_t h_status = 0;
        unsigned long long h_stats[4] = {0, 0, 0, 0};
        rc = read_back(&h_status, status, 4, st, "frw_walk_trace_static", false);
        if (!rc) rc = read_back(h_stats, stats, 32, st, "frw_walk_trace_static", false);
        if (!rc && h_status) {
            set_error("frw_walk_trace_static: kernel reported an internal limit");
            rc = FRW_E_KERNEL;
        } else if (!rc && h_stats[3] != walks) {
            set_error("frw_walk_trace_static: walk kernel did not finish every walk");
            rc = FRW_E_KERNEL;
        }
    }
    if (prev >= 0 && prev != v.device) cudaSetDevice(prev);
    return rc;
}
