// frw_internal.h -- shared declarations of the FRW library (host + device).
#pragma once

#include <cuda_runtime.h>
#include <stdint.h>

#include <string>

#include "../../include/frw.h"

namespace frw {

// ---- quadtree layout in HBM --------------------------------------------------
// Rects are stored Morton-sorted as float4 (x0,y0,x1,y1): 16-byte vector
// loads, exact because every accepted coordinate is FP32-representable.
// Each internal node holds the boxes of its four children (4 x float4 = 64 B,
// 64-byte aligned) in `nbox` and their references (int4) in `nref`:
//   ref >= 0         internal node index
//   ref == -1        empty quadrant
//   ref <= -2        leaf: -2 - ((first_rect << 5) | count), count <= 31
constexpr int kLeafBits = 5;
constexpr int kLeafCountMax = (1 << kLeafBits) - 1;
constexpr int kRefEmpty = -1;
constexpr int kDefaultLeafMax = 8;

#if defined(__CUDACC__)
#define FRW_HD __host__ __device__ inline
#else
#define FRW_HD inline
#endif
FRW_HD int leaf_ref(int first, int count) { return -2 - ((first << kLeafBits) | count); }
FRW_HD int leaf_first(int ref) { return (-2 - ref) >> kLeafBits; }
FRW_HD int leaf_count(int ref) { return (-2 - ref) & kLeafCountMax; }

struct DevLayout {
    const float4 *rects;  // [n] Morton order
    const int32_t *ids;   // [n] Morton position -> layer index
    const float4 *nbox;   // [4 * nodes]
    const int4 *nref;     // [nodes]
    double bx0, by0, bx1, by1;  // layer bounds (reference getLayerSize)
    double dist0;               // 0.05 * max(W, H): drawBiggestSquareAtPoint's first step
    double delta;               // tie window of the clearance replay (see query.cuh)
    float slack;                // FP32 pre-filter margin: 4 ulp_f32(max |bound|)
    int32_t n, nodes;
    int32_t halvings;  // bisection steps of the replay with dist above MIN_DIST: dist0 halved that often
    // cell lists (optional, cells == nullptr: tree only): a gnx x gny grid of
    // side 1/ginv from (gx0, gy0); cell (start, count) into crects / cids,
    // count < 0 when the cell overflowed and its points use the tree
    const int2 *cells;
    const float4 *crects;
    const int32_t *cids;
    const float *crad;  // per cell: every rect within this L-inf distance of any point of the cell is listed
    double gx0, gy0, ginv;
    int32_t gnx, gny;
    // 1 when the tree answers some points (no cell lists, or overflowed
    // cells): only then can a point have more near ties than the tree's
    // candidate list holds
    int32_t tree_points = 1;
};

// ---- device status word (atomicOr'ed by kernels, read back by the host) ----
enum : uint32_t {
    kStCandOverflow = 1u,   // more near-tied rects than the candidate list holds
    kStStackOverflow = 2u,  // traversal stack overflow
    kStReplayCap = 4u,      // bisection replay exceeded its iteration bound
    kStBadInput = 8u,       // a kernel met an input outside its contract
    kStDeviceWait = 16u,    // a device-side wait (mbarrier) passed its bound
};

// ---- walk jobs ----------------------------------------------------------------
struct WalkJob {
    DevLayout L;
    int64_t target;       // layer index
    uint64_t walk_begin;  // first global walk index of this job
    uint64_t walks;       // walks of this job
    uint64_t first_walk;  // Philox walk index of the job's first walk
    int64_t acc_base;     // accumulator offset (per-conductor rows)
    uint32_t stream_id;
    int32_t pad;
};

struct WalkParams {
    WalkJob job0;          // the job of a single-job launch (read from parameter space)
    const WalkJob *jobs;   // [njobs] for a multi-job launch
    const double4 *gauss;  // [njobs] Gaussian surfaces (written on the device by launch_gauss)
    int32_t njobs;
    int32_t start_mode;
    int32_t exact_perimeter;
    int32_t refill_min;
    uint32_t start_grid;   // 0: continuous uniform start; Q: midpoints of Q equal arcs
    uint32_t start_strata; // 0: off; S: walk w draws its start in stratum w mod S
    int64_t hop_cap;
    double permittivity;
    uint64_t seed;
    const uint64_t *seed_dev;  // when set, the seed is read here (captured graphs replay with new seeds)
    uint32_t chunk;            // walks a warp claims per global atomic (0: 128)
    uint64_t total_walks;
    unsigned long long *counter;  // global walk counter (refill)
    // per-conductor accumulators (dense rows, acc_base + layer index)
    unsigned long long *acc_n;
    double *acc_s;
    double *acc_s2;
    // per-job scalars [njobs][4]: escaped, aborted, hops, done
    unsigned long long *job_stats;
    uint32_t *status;
    // optional per-walk records (indexed by global walk index)
    int64_t *rec_end;
    int32_t *rec_hops;
    int32_t *rec_bin;
    double *rec_w;
    int32_t *rec_q;   // optional: first-hop cell q * 200 + bin of the grid start (-1: no first hop)
    double4 *rec_cv;  // optional: (first-hop point x, y, first square side a0, weight factor c)
    // optional control variate (single job, uniform grid start, no records):
    // phi per (grid arc q, first-hop bin) at q * 200 + bin, and the sums of
    // z = c (y - phi) and z^2 over all walks (y = 1 on the target), added here
    const float *cv_phi;
    double *cv_sums;
    // tables
    const double *intg;  // [201]
    const double *wx;    // [200]
    const double *wy;    // [200]
    // 1 when some job's layout has tree_points set: the walk kernel then
    // carries the whole-tree replay for points with many exact ties
    int32_t tree_points;
};

// ---- host helpers ----------------------------------------------------------
void set_error(const std::string &msg);
frw_status cuda_fail(cudaError_t e, const char *what);

// FRW_E_KERNEL with a message naming the bits of a nonzero kernel status word.
frw_status status_word_error(uint32_t status);

// Bounded host waits.  The limit in force on the calling thread (ms; <= 0:
// none) is the process-wide default (frw_set_wait_limit) unless a WaitScope
// set another for the call.  A wait that outlives it returns FRW_E_TIMEOUT
// and leaves the stream's work running: every buffer that work uses is
// released in stream order (cudaFreeAsync on the same stream), so nothing is
// freed under it, and no copy into host memory has been enqueued yet (reads
// of device results always come after a completed wait).
double wait_limit_ms();
struct WaitScope {
    double prev;
    explicit WaitScope(double ms);  // ms <= 0 keeps the limit in force
    ~WaitScope();
};
// Waits until everything enqueued on `st` so far has finished.
frw_status wait_stream(cudaStream_t st, const char *what);
// Waits for a recorded event.
frw_status wait_event(cudaEvent_t e, const char *what);
// A small device result after everything enqueued on `st` so far, with a
// bounded wait.  staged: through a pinned buffer of the calling thread (made
// on its first use), one copy queued behind the work and one wait; else a
// wait, then a synchronous copy (no allocation).
frw_status read_back(void *host, const void *dev, size_t bytes, cudaStream_t st, const char *what,
                     bool staged = true);

// CUDA events destroyed at scope exit, error paths included.
struct Events {
    cudaEvent_t e[4] = {nullptr, nullptr, nullptr, nullptr};
    explicit Events(int n, unsigned flags = cudaEventDefault) {
        for (int i = 0; i < n && i < 4; i++)
            if (cudaEventCreateWithFlags(&e[i], flags) != cudaSuccess) e[i] = nullptr;
    }
    bool ok(int n) const {
        for (int i = 0; i < n; i++)
            if (!e[i]) return false;
        return true;
    }
    cudaEvent_t operator[](int i) const { return e[i]; }
    ~Events() {
        for (cudaEvent_t x : e)
            if (x) cudaEventDestroy(x);
    }
    Events(const Events &) = delete;
    Events &operator=(const Events &) = delete;
};

#define FRW_CK(call)                                          \
    do {                                                      \
        cudaError_t e__ = (call);                             \
        if (e__ != cudaSuccess) return cuda_fail(e__, #call); \
    } while (0)

// tree_build.cu
struct TreeBuffers {
    float4 *rects = nullptr;
    int32_t *ids = nullptr;
    float4 *nbox = nullptr;
    int4 *nref = nullptr;
    int32_t nodes = 0, depth = 0;
    int64_t bytes = 0;
};
// Device check of a layout's rects (finite, |c| < 2^24, x0 <= x1 and
// y0 <= y1, inside `given` when not null) and the extent of the rects:
// bad = index of the first offending rect (-1: none) and why its reason
// (1 coordinate, 2 inverted, 3 outside the given bounds); ext = min x0,
// min y0, max x1, max y1.  Waits for the stream (bounded).
struct RectCheck {
    unsigned long long bad;
    unsigned key[4];
};
frw_status check_rects(const float4 *d_rects, int64_t n, const double *given, int sms, cudaStream_t stream,
                       int64_t *bad, int *why, double ext[4]);
frw_status build_tree(const float4 *d_rects_in, int32_t n, const double bounds[4], int leaf_max,
                      cudaStream_t stream, TreeBuffers *out, float *build_ms);
// Layout buffers come from the device's stream-ordered pool; the free calls
// release them in the order of `stream` (callers make sure nothing still
// reads them on another stream).
void free_tree(TreeBuffers *t, cudaStream_t stream);

// Cell lists over a built tree (DevLayout L with cells == nullptr): every
// rect whose L-inf distance to a cell can be within 2 delta of the clearance
// of a point of the cell, per cell, at most max_per_cell of them.
struct CellBuffers {
    int2 *cells = nullptr;
    float4 *crects = nullptr;
    int32_t *cids = nullptr;
    float *crad = nullptr;
    int64_t ncells = 0, entries = 0, overflow = 0, bytes = 0;
    double gx0 = 0, gy0 = 0, side = 0, ginv = 0;
    int32_t nx = 0, ny = 0;
    float build_ms = 0.f;
};
constexpr double kDefaultCellsPerRect = 16.0;
constexpr int kDefaultCellMax = 32;
constexpr int64_t kMaxCells = 1ll << 26;
frw_status build_cells(const DevLayout &L, double cells_per_rect, int max_per_cell, cudaStream_t stream,
                       CellBuffers *out);
void free_cells(CellBuffers *c, cudaStream_t stream);
// Exclusive scan of n int64 values into out (in and out must not alias);
// sums holds scan_i64_tiles(n) tile totals, *grand receives the total.
int64_t scan_i64_tiles(int64_t n);
void launch_scan_i64(const int64_t *in, int64_t n, int64_t *out, int64_t *sums, int64_t *grand, cudaStream_t stream);
void attach_cells(DevLayout &L, const CellBuffers &c);

// query.cu
frw_status launch_query(const DevLayout &L, const double *d_pts, int64_t n, double *d_sq,
                        int64_t *d_hit, uint32_t *d_status, cudaStream_t stream);
frw_status launch_box_collides(const DevLayout &L, const double *d_boxes, int64_t n, bool has_ignore,
                               const double ignore[4], uint8_t *d_out, uint32_t *d_status,
                               cudaStream_t stream);
frw_status launch_gauss(const DevLayout &L, const double *d_targets /*[n][4]*/, int n, int mode,
                        double param, double *d_out, uint32_t *d_status, cudaStream_t stream);
// one Gaussian surface per job, each on its job's layout
frw_status launch_gauss_jobs(const WalkJob *d_jobs, const double *d_targets, int njobs, int mode, double param,
                             double *d_out, uint32_t *d_status, cudaStream_t stream);

// walk.cu
frw_status launch_walk(const WalkParams &P, int threads, int blocks, cudaStream_t stream);
// Resident k_walk blocks per SM for one job or many, uniform start or not.
int walk_max_blocks_per_sm(int threads, bool multi, bool uniform);
// Compacts the nonzero accumulator rows (at most cap of them written; cap < 0:
// rows): their count, written or not, goes to *d_count.
frw_status launch_compact(const unsigned long long *acc_n, const double *acc_s, const double *acc_s2,
                          int64_t rows, int64_t *out_row, unsigned long long *out_n, double *out_s,
                          double *out_s2, unsigned long long *d_count, cudaStream_t stream, int64_t cap = -1);

// host_green.cpp
void green_tables(double *g, double *intg, double *wx, double *wy);

// frw_api.cpp: read-only views for other host files (no allocation once the
// device has been initialised by a layout)
struct LayoutView {
    DevLayout dl;
    int device;
    int64_t n;
    const double *rects;  // host copy, layer order
};
frw_status layout_view(const frw_layout *layout, LayoutView *out);
frw_status device_tables(int device, const double **tables, int *sms);
frw_status check_opts(const frw_opts *opts);
// walks with per-walk end and (first-hop point, a0, weight factor) records (device arrays)
frw_status walk_records(const frw_layout *layout, int64_t target, uint64_t first_walk, uint64_t walks,
                        uint64_t seed, const frw_opts &o, cudaStream_t st, int64_t *rec_end, double4 *rec_cv,
                        double *rec_w = nullptr, int32_t *rec_q = nullptr);
// The walks of frw_walk_device into device rows (hits, sum_w, sum_w2 per
// conductor; stats; status), optionally with the control variate's sums
// (cv_phi / cv_sums of WalkParams); no host wait.
frw_status walk_device_rows(const frw_layout *layout, int64_t target, uint64_t walks, uint64_t seed,
                            const frw_opts &o, uint64_t *hits, double *sum_w, double *sum_w2, uint64_t *stats,
                            uint32_t *status, const float *cv_phi, double *cv_sums, cudaStream_t st);

}  // namespace frw
