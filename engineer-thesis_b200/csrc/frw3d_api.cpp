// frw3d_api.cpp -- the extern "C" boundary of the 3-D walk path
// (include/frw3d.h): argument checks, layouts (boxes, bounds, the device
// cell grid), the cube tables on each device and the estimator's rows.
// Every compute step runs on the device; there is no CPU path.
#include <math.h>
#include <string.h>

#include <algorithm>
#include <cmath>
#include <map>
#include <memory>
#include <mutex>
#include <string>
#include <utility>
#include <vector>

#include "frw3d_internal.h"
#include "layout_io.h"

struct frw3_layout {
    int device = 0;
    int64_t n = 0;
    std::vector<float> boxes;  // input order, 6 per box
    double bounds[6] = {0, 0, 0, 0, 0, 0};
    double min_edge = 0;
    float *d_boxes = nullptr;
    frw::Grid3Buffers grid;
    frw::Dev3Layout dl{};
};

namespace frw {
namespace {

struct Dev3Guard {
    int prev = -1;
    explicit Dev3Guard(int dev) {
        if (cudaGetDevice(&prev) != cudaSuccess) prev = -1;
        if (prev != dev) cudaSetDevice(dev);
    }
    ~Dev3Guard() {
        int cur = -1;
        if (prev >= 0 && cudaGetDevice(&cur) == cudaSuccess && cur != prev) cudaSetDevice(prev);
    }
};

// Device copies of the cube tables, one per (device, n), kept for the
// process lifetime.
std::mutex g_tab_mu;
std::map<std::pair<int, int>, Cube3Tables> g_tabs;

frw_status device_cube_tables(int dev, int n, const Cube3Tables **out) {
    std::lock_guard<std::mutex> lk(g_tab_mu);
    auto key = std::make_pair(dev, n);
    auto it = g_tabs.find(key);
    if (it != g_tabs.end()) {
        *out = &it->second;
        return FRW_OK;
    }
    const int nb = 6 * n * n;
    std::vector<uint32_t> thr(nb);
    std::vector<uint16_t> guide(1 << kGuide3Bits);
    std::vector<double> w(3 * (size_t)nb), offs(n);
    if (!cube_walk_tables(n, thr.data(), guide.data(), w.data(), offs.data())) {
        set_error("cube table of resolution " + std::to_string(n) + " has an empty bin before its end");
        return FRW_E_ARG;
    }
    Cube3Tables T;
    T.n = n;
    T.nb = nb;
    Dev3Guard g(dev);
    FRW_CK(cudaMalloc(&T.thr, thr.size() * 4));
    FRW_CK(cudaMalloc(&T.guide, guide.size() * 2));
    FRW_CK(cudaMalloc(&T.w, w.size() * 8));
    FRW_CK(cudaMalloc(&T.offs, offs.size() * 8));
    FRW_CK(cudaMemcpy(T.thr, thr.data(), thr.size() * 4, cudaMemcpyHostToDevice));
    FRW_CK(cudaMemcpy(T.guide, guide.data(), guide.size() * 2, cudaMemcpyHostToDevice));
    FRW_CK(cudaMemcpy(T.w, w.data(), w.size() * 8, cudaMemcpyHostToDevice));
    FRW_CK(cudaMemcpy(T.offs, offs.data(), offs.size() * 8, cudaMemcpyHostToDevice));
    auto res = g_tabs.emplace(key, T);
    *out = &res.first->second;
    return FRW_OK;
}

bool fp32_exact3(double v) { return std::isfinite(v) && (double)(float)v == v && fabs(v) < 16777216.0; }

// Interiors pairwise disjoint (touching faces allowed): boxes are binned
// into a hash grid of cells about one box across (count -> prefix -> fill),
// and the boxes sharing a cell are compared pairwise.
frw_status check_disjoint(const float *b, int64_t n) {
    double emax = 0, lo[3] = {INFINITY, INFINITY, INFINITY}, hi[3] = {-INFINITY, -INFINITY, -INFINITY};
    for (int64_t i = 0; i < n; i++)
        for (int c = 0; c < 3; c++) {
            emax = std::max(emax, (double)b[6 * i + 3 + c] - b[6 * i + c]);
            lo[c] = std::min(lo[c], (double)b[6 * i + c]);
            hi[c] = std::max(hi[c], (double)b[6 * i + 3 + c]);
        }
    double vol = 1.0;
    for (int c = 0; c < 3; c++) vol *= std::max(hi[c] - lo[c], 1e-30);
    double cs = std::max(emax, std::cbrt(vol / (double)n));
    int64_t nc[3], total;
    for (;;) {
        total = 1;
        for (int c = 0; c < 3; c++) {
            nc[c] = std::max<int64_t>(1, (int64_t)floor((hi[c] - lo[c]) / cs) + 1);
            total *= nc[c];
        }
        if (total <= 8 * n + 64) break;
        cs *= 1.25;
    }
    auto range = [&](const float *p, int64_t c0[3], int64_t c1[3]) {
        for (int c = 0; c < 3; c++) {
            c0[c] = std::min(nc[c] - 1, (int64_t)floor((p[c] - lo[c]) / cs));
            c1[c] = std::min(nc[c] - 1, (int64_t)floor((p[3 + c] - lo[c]) / cs));
        }
    };
    std::vector<int64_t> start((size_t)total + 1, 0);
    std::vector<int32_t> items;
    for (int pass = 0; pass < 2; pass++) {
        for (int64_t i = 0; i < n; i++) {
            int64_t c0[3], c1[3];
            range(b + 6 * i, c0, c1);
            for (int64_t z = c0[2]; z <= c1[2]; z++)
                for (int64_t y = c0[1]; y <= c1[1]; y++)
                    for (int64_t x = c0[0]; x <= c1[0]; x++) {
                        const int64_t cell = (z * nc[1] + y) * nc[0] + x;
                        if (pass == 0) start[(size_t)cell + 1]++;
                        else items[(size_t)start[(size_t)cell]++] = (int32_t)i;
                    }
        }
        if (pass == 0) {
            for (int64_t c = 0; c < total; c++) start[(size_t)c + 1] += start[(size_t)c];
            items.resize((size_t)start[(size_t)total]);
        } else {
            for (int64_t c = total; c > 0; c--) start[(size_t)c] = start[(size_t)c - 1];
            start[0] = 0;
        }
    }
    for (int64_t cell = 0; cell < total; cell++)
        for (int64_t u = start[(size_t)cell]; u < start[(size_t)cell + 1]; u++)
            for (int64_t v = u + 1; v < start[(size_t)cell + 1]; v++) {
                const int32_t i = items[(size_t)u], j = items[(size_t)v];
                const float *p = b + 6 * (int64_t)i, *q = b + 6 * (int64_t)j;
                bool ov = true;
                for (int c = 0; c < 3 && ov; c++) ov = p[c] < q[3 + c] && q[c] < p[3 + c];
                if (ov) {
                    set_error("boxes " + std::to_string(std::min(i, j)) + " and " + std::to_string(std::max(i, j)) +
                              " overlap");
                    return FRW_E_ARG;
                }
            }
    return FRW_OK;
}

frw_status check_opts3(const frw3_opts *o) {
    if (!o || o->struct_size != sizeof(frw3_opts)) {
        set_error("frw3_opts.struct_size mismatch (call frw3_opts_default)");
        return FRW_E_ARG;
    }
    if (!(o->gauss_offset > 0) || !std::isfinite(o->gauss_offset) || !(o->shell >= 0 || o->shell <= 0) ||
        o->hop_cap < 1 || !std::isfinite(o->permittivity) || o->nsample < 1 || o->nsample > FRW3_NSAMPLE_MAX ||
        o->blocks_per_sm < 0 || o->refill_min < 0 || o->refill_min > 32) {
        set_error("frw3_opts: need gauss_offset > 0, hop_cap >= 1, nsample in [1, 100], refill_min in [0, 32]");
        return FRW_E_ARG;
    }
    return FRW_OK;
}

// Scratch of one walk call, returned to the stream-ordered pool at scope exit.
struct Scratch3 {
    void *p = nullptr;
    cudaStream_t st;
    explicit Scratch3(cudaStream_t s) : st(s) {}
    ~Scratch3() {
        if (p) cudaFreeAsync(p, st);
    }
};

// The layout's device status word (set only if a lookup ever found no list
// on the whole chain of grid levels, which the build rules out).
frw_status check_grid_status(const frw3_layout *L, cudaStream_t st) {
    uint32_t h = 0;
    frw_status rc = read_back(&h, L->grid.status, 4, st, "3-D grid status");
    if (rc) return rc;
    if (h) {
        set_error("3-D grid: a lookup found no candidate list on any level");
        return FRW_E_KERNEL;
    }
    return FRW_OK;
}

frw_status prepare_walk(const frw3_layout *L, int64_t target, uint64_t first, uint64_t walks, uint64_t seed,
                        const frw3_opts *o, Walk3Params *P, double *shell_used) {
    frw_status rc = check_opts3(o);
    if (rc) return rc;
    if (target < 0 || target >= L->n) {
        set_error("target box out of range");
        return FRW_E_ARG;
    }
    if (first + walks < first) {
        set_error("walk index range overflows");
        return FRW_E_ARG;
    }
    const Cube3Tables *T = nullptr;
    rc = device_cube_tables(L->device, o->nsample, &T);
    if (rc) return rc;
    memset(P, 0, sizeof(*P));
    P->L = L->dl;
    P->thr = T->thr;
    P->guide = T->guide;
    P->w = T->w;
    P->offs = T->offs;
    P->n = T->n;
    P->nb = T->nb;
    if (T->n > 1) {
        P->magic_n = (uint32_t)((((uint64_t)1 << 32) + (uint64_t)T->n - 1) / (uint64_t)T->n);
        P->magic_nn = (uint32_t)((((uint64_t)1 << 32) + (uint64_t)(T->n * T->n) - 1) / (uint64_t)(T->n * T->n));
    }
    P->refill_min = o->refill_min < 1 ? 1 : (o->refill_min > 32 ? 32 : o->refill_min);
    P->start_strata = o->start_strata;
    const float *tb = L->boxes.data() + 6 * target;
    for (int c = 0; c < 3; c++) {
        P->G[c] = (double)tb[c] - o->gauss_offset;
        P->G[3 + c] = (double)tb[3 + c] + o->gauss_offset;
    }
    const double gw = P->G[3] - P->G[0], gh = P->G[4] - P->G[1], gd = P->G[5] - P->G[2];
    P->S = 2.0 * (gw * gh) + 2.0 * (gw * gd) + 2.0 * (gh * gd);
    P->target = target;
    P->shell = o->shell > 0 ? o->shell : 1e-3 * L->min_edge;
    P->hop_cap = o->hop_cap;
    P->perm = o->permittivity;
    P->seed = seed;
    P->stream = o->stream_id;
    P->first = first;
    P->walks = walks;
    *shell_used = P->shell;
    return FRW_OK;
}

int walk_blocks(int dev, int bps_opt) {
    const double *t2;
    int sms = 148;
    if (device_tables(dev, &t2, &sms) != FRW_OK) sms = 148;
    static std::mutex mu;
    static std::map<int, int> bps_cache;
    int bps;
    {
        std::lock_guard<std::mutex> lk(mu);
        auto it = bps_cache.find(dev);
        if (it == bps_cache.end()) it = bps_cache.emplace(dev, walk3_max_blocks_per_sm()).first;
        bps = it->second;
    }
    if (bps_opt > 0) bps = std::min(bps, bps_opt);
    return sms * bps;
}

}  // namespace
}  // namespace frw

using namespace frw;

extern "C" {

frw_status frw3_cube_green_table(int n, double *g, double *dgdx, double *dgdy, double *dgdz, double *intg) {
    if (!cube_green_table(n, g, dgdx, dgdy, dgdz, intg)) {
        set_error("frw3_cube_green_table: n must be in [1, 100]");
        return FRW_E_ARG;
    }
    return FRW_OK;
}

frw_status frw3_green_cube(double a, double eta, double dzeta, double *g) {
    if (!g || !(a > 0) || !(eta >= 0 && eta < 6 * a) || !(dzeta >= 0 && dzeta < 6 * a) ||
        floor(eta / a) != floor(dzeta / a)) {
        set_error("frw3_green_cube: need a > 0 and eta, dzeta in [k a, (k+1) a) of one face");
        return FRW_E_ARG;
    }
    *g = cube_green_point(a, eta, dzeta);
    return FRW_OK;
}

frw_status frw3_deriv_green_cube(double a, double eta, double dzeta, double dg[3]) {
    if (!dg || !(a > 0) || !(eta >= 0 && eta < 6 * a) || !(dzeta >= 0 && dzeta < 6 * a) ||
        floor(eta / a) != floor(dzeta / a)) {
        set_error("frw3_deriv_green_cube: need a > 0 and eta, dzeta in [k a, (k+1) a) of one face");
        return FRW_E_ARG;
    }
    cube_deriv_point(dg, a, eta, dzeta);
    return FRW_OK;
}

frw_status frw3_layout_create(const float *boxes, int64_t n, const double *bounds, double cells_per_box, int device,
                              frw3_layout **out) {
    if (!out || !boxes || n <= 0) {
        set_error("frw3_layout_create: null pointer or empty layout");
        return FRW_E_ARG;
    }
    *out = nullptr;
    if (n >= (1ll << 26)) {
        set_error("frw3_layout_create: at most 2^26-1 boxes per layout");
        return FRW_E_ARG;
    }
    const double *t2;
    int sms;
    frw_status rc = device_tables(device, &t2, &sms);
    if (rc) return rc;
    double lo[3] = {INFINITY, INFINITY, INFINITY}, hi[3] = {-INFINITY, -INFINITY, -INFINITY}, emin = INFINITY;
    for (int64_t i = 0; i < n; i++) {
        const float *q = boxes + 6 * i;
        for (int c = 0; c < 3; c++) {
            if (!fp32_exact3(q[c]) || !fp32_exact3(q[3 + c])) {
                set_error("box " + std::to_string(i) + ": coordinate not finite or |c| >= 2^24");
                return FRW_E_ARG;
            }
            if (!(q[c] < q[3 + c])) {
                set_error("box " + std::to_string(i) + ": empty or inverted (need x0 < x1, y0 < y1, z0 < z1)");
                return FRW_E_ARG;
            }
            lo[c] = std::min(lo[c], (double)q[c]);
            hi[c] = std::max(hi[c], (double)q[3 + c]);
            emin = std::min(emin, (double)q[3 + c] - (double)q[c]);
        }
    }
    rc = check_disjoint(boxes, n);
    if (rc) return rc;
    auto L = std::make_unique<frw3_layout>();
    L->device = device;
    L->n = n;
    L->boxes.assign(boxes, boxes + 6 * n);
    L->min_edge = emin;
    if (bounds) {
        for (int c = 0; c < 3; c++) {
            if (!(bounds[c] < bounds[3 + c]) || !std::isfinite(bounds[c]) || !std::isfinite(bounds[3 + c]) ||
                bounds[c] > lo[c] || bounds[3 + c] < hi[c]) {
                set_error("frw3_layout_create: bounds must be finite and contain every box");
                return FRW_E_ARG;
            }
            L->bounds[c] = bounds[c];
            L->bounds[3 + c] = bounds[3 + c];
        }
    } else {
        const int add = (int)((hi[0] - lo[0]) * 0.01);
        for (int c = 0; c < 3; c++) {
            L->bounds[c] = lo[c] - add;
            L->bounds[3 + c] = hi[c] + add;
        }
    }
    Dev3Guard g(device);
    cudaStream_t st = nullptr;
    const size_t bytes = (size_t)n * 6 * sizeof(float);
    FRW_CK(cudaMallocAsync(&L->d_boxes, bytes, st));
    cudaError_t e = cudaMemcpyAsync(L->d_boxes, boxes, bytes, cudaMemcpyHostToDevice, st);
    if (e != cudaSuccess) {
        cudaFreeAsync(L->d_boxes, st);
        return cuda_fail(e, "upload boxes");
    }
    rc = build_grid3(L->d_boxes, n, L->bounds, cells_per_box > 0 ? cells_per_box : 8.0, st, &L->grid);
    if (rc) {
        cudaFreeAsync(L->d_boxes, st);  // stream-ordered: after any build work still queued
        return rc;
    }
    attach_grid3(L->dl, L->grid, L->bounds);
    *out = L.release();
    return FRW_OK;
}

frw_status frw3_layout_from_file(const char *path, const double *z0, const double *z1, int nz, const double *bounds,
                                 double cells_per_box, int device, frw3_layout **out) {
    if (!path || !z0 || !z1 || nz < 1 || !out) {
        set_error("frw3_layout_from_file: null argument or nz < 1");
        return FRW_E_ARG;
    }
    std::vector<float> boxes;
    int nlayers = 0;
    for (int k = 0; k < nz; k++) {
        std::vector<double> r;
        frw_status rc = parse_layout_file(path, k, &r, &nlayers);
        if (rc) return rc;
        if (k == 0 && nlayers != nz) {
            set_error("frw3_layout_from_file: the file has " + std::to_string(nlayers) + " layers, " +
                      std::to_string(nz) + " z ranges given");
            return FRW_E_ARG;
        }
        if (!(z0[k] < z1[k]) || !fp32_exact3(z0[k]) || !fp32_exact3(z1[k])) {
            set_error("frw3_layout_from_file: z range " + std::to_string(k) + " empty or not FP32-exact");
            return FRW_E_ARG;
        }
        for (size_t i = 0; i + 3 < r.size(); i += 4) {
            const double b[6] = {r[i], r[i + 1], z0[k], r[i + 2], r[i + 3], z1[k]};
            for (double v : b) boxes.push_back((float)v);
        }
    }
    if (boxes.empty()) {
        set_error("frw3_layout_from_file: no rects");
        return FRW_E_IO;
    }
    return frw3_layout_create(boxes.data(), (int64_t)(boxes.size() / 6), bounds, cells_per_box, device, out);
}

frw_status frw3_layout_destroy(frw3_layout *L) {
    if (!L) return FRW_OK;
    Dev3Guard g(L->device);
    // like cudaFree: nothing on the device may still read the layout
    cudaError_t e = cudaDeviceSynchronize();
    free_grid3(&L->grid, nullptr);
    if (L->d_boxes) cudaFreeAsync(L->d_boxes, nullptr);
    delete L;
    FRW_CK(e);
    return FRW_OK;
}

frw_status frw3_layout_info_get(const frw3_layout *L, frw3_layout_info *info) {
    if (!L || !info) {
        set_error("null argument");
        return FRW_E_ARG;
    }
    memset(info, 0, sizeof(*info));
    info->n = L->n;
    info->device = L->device;
    info->grid[0] = L->grid.nx;
    info->grid[1] = L->grid.ny;
    info->grid[2] = L->grid.nz;
    memcpy(info->bounds, L->bounds, sizeof(info->bounds));
    info->cell_side = L->grid.side;
    info->min_edge = L->min_edge;
    info->list_entries = L->grid.entries;
    info->max_list = L->grid.max_list;
    info->mean_list = L->grid.ncells ? (double)L->grid.entries / (double)L->grid.ncells : 0.0;
    info->build_ms = L->grid.build_ms;
    info->levels = 1 + L->grid.nup;
    info->deferred_cells = L->grid.deferred;
    info->upper_entries = L->grid.up_entries;
    return FRW_OK;
}

frw_status frw3_layout_boxes(const frw3_layout *L, float *out) {
    if (!L || !out) {
        set_error("null argument");
        return FRW_E_ARG;
    }
    memcpy(out, L->boxes.data(), L->boxes.size() * sizeof(float));
    return FRW_OK;
}

frw_status frw3_query_batch(const frw3_layout *L, const double *pts, int64_t n, double *clear, int64_t *nearest,
                            int mem, void *stream) {
    if (!L || n < 0 || (n > 0 && !pts) || (mem != FRW_MEM_HOST && mem != FRW_MEM_DEVICE)) {
        set_error("frw3_query_batch: bad arguments");
        return FRW_E_ARG;
    }
    if (n == 0) return FRW_OK;
    Dev3Guard g(L->device);
    cudaStream_t st = (cudaStream_t)stream;
    if (mem == FRW_MEM_DEVICE) {
        frw_status rc = launch_query3(L->dl, pts, n, clear, nearest, st);
        if (rc) return rc;
        return check_grid_status(L, st);
    }
    Scratch3 s(st);
    const size_t pb = (size_t)n * 24, cb = clear ? (size_t)n * 8 : 0, nbt = nearest ? (size_t)n * 8 : 0;
    FRW_CK(cudaMallocAsync(&s.p, pb + cb + nbt, st));
    char *base = (char *)s.p;
    double *dp = (double *)base, *dc = clear ? (double *)(base + pb) : nullptr;
    int64_t *dn = nearest ? (int64_t *)(base + pb + cb) : nullptr;
    FRW_CK(cudaMemcpyAsync(dp, pts, pb, cudaMemcpyHostToDevice, st));
    frw_status rc = launch_query3(L->dl, dp, n, dc, dn, st);
    if (rc) return rc;
    rc = check_grid_status(L, st);  // bounded wait for the queries, then the grid status
    if (rc) return rc;
    if (clear) FRW_CK(cudaMemcpyAsync(clear, dc, cb, cudaMemcpyDeviceToHost, st));
    if (nearest) FRW_CK(cudaMemcpyAsync(nearest, dn, nbt, cudaMemcpyDeviceToHost, st));
    FRW_CK(cudaStreamSynchronize(st));
    return FRW_OK;
}

void frw3_opts_default(frw3_opts *o) {
    memset(o, 0, sizeof(*o));
    o->struct_size = sizeof(frw3_opts);
    o->gauss_offset = 1.0;
    o->shell = 0.0;
    o->hop_cap = 100000;
    o->permittivity = 8.854187817620e-12;
    o->stream_id = 0;
    o->nsample = FRW3_NSAMPLE_DEFAULT;
    o->first_walk = 0;
    o->blocks_per_sm = 0;
    o->refill_min = 4;
    o->start_strata = 0;
}

frw_status frw3_walk(const frw3_layout *L, int64_t target, uint64_t walks, uint64_t seed, const frw3_opts *o,
                     frw3_result *res, void *stream) {
    if (!L || !res) {
        set_error("null argument");
        return FRW_E_ARG;
    }
    Walk3Params P;
    double shell;
    frw_status rc = prepare_walk(L, target, o ? o->first_walk : 0, walks, seed, o, &P, &shell);
    if (rc) return rc;
    Dev3Guard g(L->device);
    cudaStream_t st = (cudaStream_t)stream;
    const int64_t n = L->n;
    // scratch: counter | stats[4] | hits[n] | sum_w[n] | sum_w2[n]
    const size_t bytes = (size_t)(5 + 3 * n) * 8;
    Scratch3 s(st);
    FRW_CK(cudaMallocAsync(&s.p, bytes, st));
    FRW_CK(cudaMemsetAsync(s.p, 0, bytes, st));
    unsigned long long *u = (unsigned long long *)s.p;
    P.counter = u;
    P.stats = u + 1;
    P.hits = u + 5;
    P.sum_w = (double *)(u + 5 + n);
    P.sum_w2 = (double *)(u + 5 + 2 * n);
    Events ev(2);
    if (!ev.ok(2)) return cuda_fail(cudaErrorUnknown, "event create");
    FRW_CK(cudaEventRecord(ev[0], st));
    if (walks > 0) {
        rc = launch_walk3(P, walk_blocks(L->device, o->blocks_per_sm), st);
        if (rc) return rc;
    }
    FRW_CK(cudaEventRecord(ev[1], st));
    std::vector<unsigned long long> h(5 + 3 * (size_t)n);
    rc = read_back(h.data(), s.p, bytes, st, "frw3_walk");
    if (rc) return rc;
    float ms = 0;
    cudaEventElapsedTime(&ms, ev[0], ev[1]);
    const unsigned long long *stats = h.data() + 1, *hits = h.data() + 5;
    const double *sw = (const double *)(h.data() + 5 + n), *sw2 = (const double *)(h.data() + 5 + 2 * n);
    if (stats[3] != walks) {
        set_error("3-D walk kernel finished " + std::to_string(stats[3]) + " of " + std::to_string(walks) + " walks");
        return FRW_E_KERNEL;
    }
    rc = check_grid_status(L, st);
    if (rc) return rc;
    res->walks = walks;
    res->escaped = stats[0];
    res->aborted = stats[1];
    res->hops_total = stats[2];
    memcpy(res->gauss, P.G, sizeof(res->gauss));
    res->shell = shell;
    res->kernel_ms = ms;
    res->fraction_other = walks ? (double)(walks - hits[target]) / (double)walks : 0.0;
    int64_t k = 0;
    for (int64_t i = 0; i < n; i++) {
        if (!hits[i]) continue;
        if (k < res->capacity) {
            const double N = (double)walks, m = sw[i] / N;
            const double var = std::max(sw2[i] / N - m * m, 0.0);
            if (res->conductor) res->conductor[k] = i;
            if (res->hits) res->hits[k] = hits[i];
            if (res->cap) res->cap[k] = m;
            if (res->cap_se) res->cap_se[k] = walks > 1 ? sqrt(var / (N - 1)) : 0.0;
            if (res->sum_w) res->sum_w[k] = sw[i];
            if (res->sum_w2) res->sum_w2[k] = sw2[i];
        }
        k++;
    }
    res->n_entries = k;
    return FRW_OK;
}

frw_status frw3_walk_device(const frw3_layout *L, int64_t target, uint64_t walks, uint64_t seed, const frw3_opts *opts,
                            uint64_t *hits, double *sum_w, double *sum_w2, uint64_t *stats, uint32_t *status,
                            void *stream) {
    if (!L || !hits || !sum_w || !sum_w2 || !stats || !status) {
        set_error("frw3_walk_device: null argument");
        return FRW_E_ARG;
    }
    frw3_opts o;
    frw3_opts_default(&o);
    if (opts) o = *opts;
    Walk3Params P;
    double shell;
    frw_status rc = prepare_walk(L, target, o.first_walk, walks, seed, &o, &P, &shell);
    if (rc) return rc;
    if (walks == 0) return FRW_OK;
    Dev3Guard g(L->device);
    cudaStream_t st = (cudaStream_t)stream;
    Scratch3 s(st);
    FRW_CK(cudaMallocAsync(&s.p, 8, st));
    FRW_CK(cudaMemsetAsync(s.p, 0, 8, st));
    P.counter = (unsigned long long *)s.p;
    P.hits = (unsigned long long *)hits;
    P.sum_w = sum_w;
    P.sum_w2 = sum_w2;
    P.stats = (unsigned long long *)stats;
    P.L.status = status;  // lookup failures go to the caller's word
    return launch_walk3(P, walk_blocks(L->device, o.blocks_per_sm), st);
}

frw_status frw3_walk_batch(const frw3_layout *L, const int64_t *targets, int32_t ntargets, uint64_t walks_per_target,
                           uint64_t seed, const frw3_opts *opts, frw3_result *results, void *stream) {
    if (!L || !targets || !results || ntargets < 1) {
        set_error("frw3_walk_batch: null argument or no targets");
        return FRW_E_ARG;
    }
    const int64_t n = L->n;
    if ((int64_t)ntargets * n > (int64_t(1) << 27)) {
        set_error("frw3_walk_batch: targets x boxes must stay below 2^27 (rows of every target are kept)");
        return FRW_E_ARG;
    }
    if (walks_per_target && (uint64_t)ntargets > UINT64_MAX / walks_per_target) {
        set_error("frw3_walk_batch: walk count overflows");
        return FRW_E_ARG;
    }
    frw3_opts o;
    frw3_opts_default(&o);
    if (opts) o = *opts;
    Walk3Params P;
    double shell;
    // validates the options and the first target; builds the shared parameters
    frw_status rc = prepare_walk(L, targets[0], o.first_walk, walks_per_target, seed, &o, &P, &shell);
    if (rc) return rc;
    std::vector<Job3> jobs((size_t)ntargets);
    for (int32_t t = 0; t < ntargets; t++) {
        const int64_t k = targets[t];
        if (k < 0 || k >= n) {
            set_error("frw3_walk_batch: target " + std::to_string(t) + " out of range");
            return FRW_E_ARG;
        }
        const float *tb = L->boxes.data() + 6 * k;
        for (int c = 0; c < 3; c++) {
            jobs[t].G[c] = (double)tb[c] - o.gauss_offset;
            jobs[t].G[3 + c] = (double)tb[3 + c] + o.gauss_offset;
        }
        const double gw = jobs[t].G[3] - jobs[t].G[0], gh = jobs[t].G[4] - jobs[t].G[1],
                     gd = jobs[t].G[5] - jobs[t].G[2];
        jobs[t].S = 2.0 * (gw * gh) + 2.0 * (gw * gd) + 2.0 * (gh * gd);
        jobs[t].target = k;
    }
    Dev3Guard g(L->device);
    cudaStream_t st = (cudaStream_t)stream;
    const uint64_t total = (uint64_t)ntargets * walks_per_target;
    // scratch: counter | stats[4 T] | hits[T n] | sum_w[T n] | sum_w2[T n] | jobs
    const size_t nrow = (size_t)ntargets * (size_t)n;
    const size_t words = 1 + 4 * (size_t)ntargets + 3 * nrow;
    const size_t bytes = words * 8 + jobs.size() * sizeof(Job3);
    Scratch3 s(st);
    FRW_CK(cudaMallocAsync(&s.p, bytes, st));
    FRW_CK(cudaMemsetAsync(s.p, 0, words * 8, st));
    unsigned long long *u = (unsigned long long *)s.p;
    Job3 *d_jobs = (Job3 *)(u + words);
    FRW_CK(cudaMemcpyAsync(d_jobs, jobs.data(), jobs.size() * sizeof(Job3), cudaMemcpyHostToDevice, st));
    P.counter = u;
    P.stats = u + 1;
    P.hits = u + 1 + 4 * ntargets;
    P.sum_w = (double *)(P.hits + nrow);
    P.sum_w2 = P.sum_w + nrow;
    P.jobs = d_jobs;
    P.walks_per_job = walks_per_target;
    P.nboxes = n;
    P.walks = total;
    Events ev(2);
    if (!ev.ok(2)) return cuda_fail(cudaErrorUnknown, "event create");
    FRW_CK(cudaEventRecord(ev[0], st));
    if (total > 0) {
        rc = launch_walk3_batch(P, walk_blocks(L->device, o.blocks_per_sm), st);
        if (rc) return rc;
    }
    FRW_CK(cudaEventRecord(ev[1], st));
    std::vector<unsigned long long> h(words);
    rc = read_back(h.data(), s.p, words * 8, st, "frw3_walk_batch");
    if (rc) return rc;
    rc = check_grid_status(L, st);
    if (rc) return rc;
    float ms = 0;
    cudaEventElapsedTime(&ms, ev[0], ev[1]);
    const unsigned long long *hits_all = h.data() + 1 + 4 * ntargets;
    const double *sw_all = (const double *)(hits_all + nrow), *sw2_all = sw_all + nrow;
    for (int32_t t = 0; t < ntargets; t++) {
        const unsigned long long *stt = h.data() + 1 + 4 * t;
        if (stt[3] != walks_per_target) {
            set_error("3-D batch: target " + std::to_string(t) + " finished " + std::to_string(stt[3]) + " of " +
                      std::to_string(walks_per_target) + " walks");
            return FRW_E_KERNEL;
        }
        frw3_result *res = results + t;
        const unsigned long long *hits = hits_all + (size_t)t * n;
        const double *sw = sw_all + (size_t)t * n, *sw2 = sw2_all + (size_t)t * n;
        const int64_t tk = targets[t];
        res->walks = walks_per_target;
        res->escaped = stt[0];
        res->aborted = stt[1];
        res->hops_total = stt[2];
        memcpy(res->gauss, jobs[t].G, sizeof(res->gauss));
        res->shell = shell;
        res->kernel_ms = ms;
        res->fraction_other =
            walks_per_target ? (double)(walks_per_target - hits[tk]) / (double)walks_per_target : 0.0;
        int64_t k = 0;
        for (int64_t i = 0; i < n; i++) {
            if (!hits[i]) continue;
            if (k < res->capacity) {
                const double N = (double)walks_per_target, m = sw[i] / N;
                const double var = std::max(sw2[i] / N - m * m, 0.0);
                if (res->conductor) res->conductor[k] = i;
                if (res->hits) res->hits[k] = hits[i];
                if (res->cap) res->cap[k] = m;
                if (res->cap_se) res->cap_se[k] = walks_per_target > 1 ? sqrt(var / (N - 1)) : 0.0;
                if (res->sum_w) res->sum_w[k] = sw[i];
                if (res->sum_w2) res->sum_w2[k] = sw2[i];
            }
            k++;
        }
        res->n_entries = k;
    }
    return FRW_OK;
}

frw_status frw3_walk_trace(const frw3_layout *L, int64_t target, uint64_t first_walk, uint64_t walks, uint64_t seed,
                           const frw3_opts *o, int64_t *end, int32_t *hops, int32_t *bin1, double *weight, int mem,
                           void *stream) {
    if (!L || (mem != FRW_MEM_HOST && mem != FRW_MEM_DEVICE)) {
        set_error("frw3_walk_trace: bad arguments");
        return FRW_E_ARG;
    }
    Walk3Params P;
    double shell;
    frw_status rc = prepare_walk(L, target, first_walk, walks, seed, o, &P, &shell);
    if (rc) return rc;
    if (walks == 0) return FRW_OK;
    Dev3Guard g(L->device);
    cudaStream_t st = (cudaStream_t)stream;
    const size_t W = (size_t)walks;
    const size_t rec = mem == FRW_MEM_HOST ? W * ((end ? 8 : 0) + (hops ? 4 : 0) + (bin1 ? 4 : 0) + (weight ? 8 : 0)) : 0;
    Scratch3 s(st);
    FRW_CK(cudaMallocAsync(&s.p, 40 + rec, st));
    FRW_CK(cudaMemsetAsync(s.p, 0, 40, st));
    char *base = (char *)s.p;
    P.counter = (unsigned long long *)base;
    P.stats = (unsigned long long *)(base + 8);
    if (mem == FRW_MEM_DEVICE) {
        P.rec_end = end;
        P.rec_hops = hops;
        P.rec_bin = bin1;
        P.rec_w = weight;
    } else {
        char *r = base + 40;
        if (end) { P.rec_end = (int64_t *)r; r += W * 8; }
        if (weight) { P.rec_w = (double *)r; r += W * 8; }
        if (hops) { P.rec_hops = (int32_t *)r; r += W * 4; }
        if (bin1) { P.rec_bin = (int32_t *)r; r += W * 4; }
    }
    if (!P.rec_end && !P.rec_hops && !P.rec_bin && !P.rec_w) {
        set_error("frw3_walk_trace: no output array");
        return FRW_E_ARG;
    }
    rc = launch_walk3(P, walk_blocks(L->device, o->blocks_per_sm), st);
    if (rc) return rc;
    rc = wait_stream(st, "frw3_walk_trace");
    if (rc) return rc;
    if (mem == FRW_MEM_HOST) {
        if (end) FRW_CK(cudaMemcpyAsync(end, P.rec_end, W * 8, cudaMemcpyDeviceToHost, st));
        if (weight) FRW_CK(cudaMemcpyAsync(weight, P.rec_w, W * 8, cudaMemcpyDeviceToHost, st));
        if (hops) FRW_CK(cudaMemcpyAsync(hops, P.rec_hops, W * 4, cudaMemcpyDeviceToHost, st));
        if (bin1) FRW_CK(cudaMemcpyAsync(bin1, P.rec_bin, W * 4, cudaMemcpyDeviceToHost, st));
    }
    unsigned long long done = 0;
    FRW_CK(cudaMemcpyAsync(&done, P.stats + 3, 8, cudaMemcpyDeviceToHost, st));
    FRW_CK(cudaStreamSynchronize(st));
    if (done != walks) {
        set_error("3-D walk kernel finished " + std::to_string(done) + " of " + std::to_string(walks) + " walks");
        return FRW_E_KERNEL;
    }
    return check_grid_status(L, st);
}

frw_status frw3_generate_layout(uint64_t seed, int64_t n, double domain, double zdomain, int32_t wmin, int32_t wmax,
                                int32_t zmin, int32_t zmax, int32_t gap, float *out) {
    if (!out) {
        set_error("null output");
        return FRW_E_ARG;
    }
    return generate_layout3(seed, n, domain, zdomain, wmin, wmax, zmin, zmax, (double)gap, out);
}

}  // extern "C"
