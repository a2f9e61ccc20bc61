// cell_build.cu -- cell lists: a uniform grid over the layer bounds whose
// cells list the rects a clearance query from inside the cell can need.
//
// For a point p of cell C with centre c and side s,
//     d*(p) <= d*(c) + |p - c|_inf <= d*(c) + s/2 =: U_C
// (d* is 1-Lipschitz in the L-inf norm, bounds distance included), and a
// rect R with gap(R, p) <= d*(p) + 2 delta has L-inf distance to C at most
// U_C + 2 delta.  So the rects touching C grown by
//     r_C = max(U_C, 0) + 2 delta + margin
// are every rect the query at p can find nearest, tied within 2 delta, or
// containing p (max with 0).  The margin (M * 2^-30, M the layout's
// coordinate scale) covers the rounding of the cell index of p and of the
// cell's coordinates, both of order M * 2^-50.  Built from the tree: one
// clearance query at each cell centre and one box enumeration per cell (the
// count pass), a scan, then the fill pass, which copies the rects the count
// pass staged (the first kStage of each cell) and enumerates again only the
// longer cells, from the radius the count pass kept.  Large grids first
// build coarse cells (4 x 4 cells each) that way and then answer each cell's
// clearance and enumeration from its coarse cell's list instead of the tree.
// Cells with more than max_per_cell rects keep count -1 and their points use
// the tree.
#include <cuda_runtime.h>

#include <algorithm>
#include <cmath>
#include <initializer_list>

#include "query.cuh"

namespace frw {
namespace {

constexpr int kScanThreads = 1024;
constexpr int kScanItems = 8;
constexpr int kScanTile = kScanThreads * kScanItems;
// rect indices staged per cell by the count pass (a cell of the configs'
// density lists about 2 rects)
constexpr int kStage = 4;

// Visits the tree's rects touching the closed box B, in tree order, until
// visit() returns false.  Returns false when the traversal stack overflowed
// (the visit is then incomplete).
template <typename F>
__device__ __forceinline__ bool touching(const DevLayout &L, const double B[4], F &&visit) {
    int stk[kStackMax];
    int sp = 1;
    stk[0] = 0;
    while (sp > 0) {
        const int nd = stk[--sp];
        const int4 rf = __ldg(L.nref + nd);
        const int ref[4] = {rf.x, rf.y, rf.z, rf.w};
        for (int c = 0; c < 4; c++) {
            if (ref[c] == kRefEmpty) continue;
            const float4 b = __ldg(L.nbox + 4 * nd + c);
            if (!((double)b.z >= B[0] && B[2] >= (double)b.x && (double)b.w >= B[1] && B[3] >= (double)b.y))
                continue;
            if (ref[c] >= 0) {
                if (sp == kStackMax) return false;
                stk[sp++] = ref[c];
                continue;
            }
            const int f = leaf_first(ref[c]), m = leaf_count(ref[c]);
            for (int k = f; k < f + m; k++) {
                const float4 r = __ldg(L.rects + k);
                if ((double)r.z >= B[0] && B[2] >= (double)r.x && (double)r.w >= B[1] && B[3] >= (double)r.y)
                    if (!visit(k, r)) return true;
            }
        }
    }
    return true;
}

struct Grid {
    double gx0, gy0, side, margin;
    int nx, ny;
};

// The count pass visits the cells in tiles of 8 x 4, one tile per warp, so
// that a warp's tree traversals start from neighbouring points and take
// similar paths: thread t gets cell (tile_x * 8 + t % 8, tile_y * 4 + t % 32
// / 8) of tile t / 32, or -1 past the grid's edge.
constexpr int kTileW = 8, kTileH = 4;
__device__ __forceinline__ int64_t tiled_cell(const Grid &G, int64_t t) {
    const int64_t tile = t >> 5;
    const int lane = (int)(t & 31);
    const int64_t tiles_x = (G.nx + kTileW - 1) / kTileW;
    const int64_t ix = (tile % tiles_x) * kTileW + (lane % kTileW), iy = (tile / tiles_x) * kTileH + lane / kTileW;
    return ix < G.nx && iy < G.ny ? iy * G.nx + ix : -1;
}
int64_t tiled_threads(int64_t nx, int64_t ny) {
    return ((nx + kTileW - 1) / kTileW) * ((ny + kTileH - 1) / kTileH) * 32;
}

// The box of cell c grown by r.
__device__ __forceinline__ void grown_box(const Grid &G, int64_t c, double r, double B[4]) {
    const int ix = (int)(c % G.nx), iy = (int)(c / G.nx);
    const double x0 = G.gx0 + ix * G.side, y0 = G.gy0 + iy * G.side;
    B[0] = x0 - r;
    B[1] = y0 - r;
    B[2] = (x0 + G.side) + r;
    B[3] = (y0 + G.side) + r;
}

// The radius r_C of cell c (plus `extra`) from the clearance at the cell
// centre: the tree's, or, when L carries coarse cell lists, the coarse
// list's (the same value: the list holds every rect the query can need).
__device__ __forceinline__ double cell_radius(const DevLayout &L, const Grid &G, int64_t c, double extra) {
    const int ix = (int)(c % G.nx), iy = (int)(c / G.nx);
    const double x0 = G.gx0 + ix * G.side, y0 = G.gy0 + iy * G.side;
    Cands C;
    int hit;
    double best;
    clearance(L, x0 + 0.5 * G.side, y0 + 0.5 * G.side, C, hit, best);
    return fmax(best, 0.0) + 0.5 * G.side + 2.0 * L.delta + G.margin + extra;
}

// Where cell c's rects come from: the entries of the coarse cell (of
// factor x factor cells) that covers it, when L carries coarse lists and that
// coarse cell did not overflow; else (count -1) the tree.
__device__ __forceinline__ int2 coarse_range(const DevLayout &L, const Grid &G, int factor, int64_t c) {
    if (!L.cells) return make_int2(0, -1);
    const int ix = (int)(c % G.nx), iy = (int)(c / G.nx);
    return __ldg(L.cells + (int64_t)(iy / factor) * L.gnx + ix / factor);
}

// Visits the rects touching B, from the coarse entries ce (positions into
// L.crects) or from the tree (Morton positions) when ce.y < 0.  A fine
// cell's grown box lies inside its coarse cell's grown box (the coarse radius
// carries an extra margin over the Lipschitz bound r_fine <= r_coarse), so
// the coarse list holds every rect touching it.
template <typename F>
__device__ __forceinline__ bool touching_from(const DevLayout &L, int2 ce, const double B[4], F &&visit) {
    if (ce.y < 0) return touching(L, B, visit);
    for (int k = ce.x; k < ce.x + ce.y; k++) {
        const float4 r = __ldg(L.crects + k);
        if ((double)r.z >= B[0] && B[2] >= (double)r.x && (double)r.w >= B[1] && B[3] >= (double)r.y)
            if (!visit(k, r)) return true;
    }
    return true;
}

// Per cell: its list length, or -1 (in cells[c].y) when it exceeds cap or
// the enumeration was incomplete; cnt[c] = entries to reserve; rad[c] its
// radius and stage[kStage c ..] the source positions of its first kStage
// rects, for the fill pass.
__global__ void k_cell_count(DevLayout L, Grid G, int factor, double extra, int cap, int64_t *__restrict__ cnt,
                             int2 *__restrict__ cells, float *__restrict__ crad, double *__restrict__ rad,
                             int32_t *__restrict__ stage, unsigned long long *overflow, int64_t nthreads) {
    const int64_t t = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (t >= nthreads) return;
    const int64_t c = tiled_cell(G, t);
    if (c < 0) return;
    const double r = cell_radius(L, G, c, extra);
    double B[4];
    grown_box(G, c, r, B);
    rad[c] = r;
    // a point of the cell lies within margin/2 of it whatever the rounding of
    // its cell index, so every rect within r - margin of the point is listed
    crad[c] = __double2float_rd(r - G.margin);
    int n = 0;
    int32_t *sg = stage + kStage * c;
    const bool complete = touching_from(L, coarse_range(L, G, factor, c), B, [&](int k, float4) {
        if (n < kStage) sg[n] = k;
        return ++n <= cap;
    });
    const bool ok = complete && n <= cap;
    cnt[c] = ok ? n : 0;
    cells[c] = make_int2(0, ok ? n : -1);
    if (!ok) atomicAdd(overflow, 1ull);
}

// Writes the lists of the cells that did not overflow: the staged rects, or
// for longer lists the enumeration of the same grown box from the same source
// again (its order is deterministic, so it meets the same rects as the
// count).
__global__ void k_cell_fill(DevLayout L, Grid G, int factor, const int64_t *__restrict__ start,
                            const double *__restrict__ rad, const int32_t *__restrict__ stage,
                            int2 *__restrict__ cells, float4 *__restrict__ crects, int32_t *__restrict__ cids,
                            int64_t ncells) {
    const int64_t c = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (c >= ncells) return;
    const int m = cells[c].y;
    if (m < 0) return;
    const int64_t s = start[c];
    const int2 ce = coarse_range(L, G, factor, c);
    const float4 *src = ce.y < 0 ? L.rects : L.crects;
    const int32_t *sid = ce.y < 0 ? L.ids : L.cids;
    if (m <= kStage) {
        for (int i = 0; i < m; i++) {
            const int k = stage[kStage * c + i];
            crects[s + i] = __ldg(src + k);
            cids[s + i] = __ldg(sid + k);
        }
    } else {
        double B[4];
        grown_box(G, c, rad[c], B);
        int n = 0;
        touching_from(L, ce, B, [&](int k, float4 r) {
            if (n >= m) return false;
            crects[s + n] = r;
            cids[s + n] = __ldg(sid + k);
            return ++n < m;
        });
    }
    cells[c] = make_int2((int)s, m);
}

// Exclusive scan of int64 values: tile sums, a one-block scan of the tile
// sums, then each tile rescanned with its offset.
__device__ __forceinline__ int64_t block_excl_scan(int64_t v, int64_t *warp_tot, int64_t &total) {
    const int lane = threadIdx.x & 31, w = threadIdx.x >> 5;
    int64_t x = v;
#pragma unroll
    for (int o = 1; o < 32; o <<= 1) {
        const int64_t y = __shfl_up_sync(0xFFFFFFFFu, x, o);
        if (lane >= o) x += y;
    }
    if (lane == 31) warp_tot[w] = x;
    __syncthreads();
    if (w == 0) {
        int64_t t = lane < kScanThreads / 32 ? warp_tot[lane] : 0;
#pragma unroll
        for (int o = 1; o < 32; o <<= 1) {
            const int64_t y = __shfl_up_sync(0xFFFFFFFFu, t, o);
            if (lane >= o) t += y;
        }
        warp_tot[lane] = t;  // inclusive over warps
    }
    __syncthreads();
    total = warp_tot[kScanThreads / 32 - 1];
    const int64_t before = w ? warp_tot[w - 1] : 0;
    __syncthreads();
    return before + x - v;
}

__global__ void __launch_bounds__(kScanThreads) k_tile_sums(const int64_t *__restrict__ in, int64_t n,
                                                          int64_t *__restrict__ sums) {
    __shared__ int64_t wt[32];
    const int64_t base = (int64_t)blockIdx.x * kScanTile + (int64_t)threadIdx.x * kScanItems;
    int64_t s = 0;
    for (int k = 0; k < kScanItems; k++)
        if (base + k < n) s += in[base + k];
    int64_t total;
    block_excl_scan(s, wt, total);
    if (threadIdx.x == 0) sums[blockIdx.x] = total;
}

__global__ void __launch_bounds__(kScanThreads) k_scan_sums(int64_t *sums, int64_t n, int64_t *grand) {
    __shared__ int64_t wt[32];
    int64_t carry = 0;
    for (int64_t b = 0; b < n; b += kScanThreads) {
        const int64_t i = b + threadIdx.x;
        const int64_t v = i < n ? sums[i] : 0;
        int64_t total;
        const int64_t e = block_excl_scan(v, wt, total);
        if (i < n) sums[i] = carry + e;
        carry += total;
    }
    if (threadIdx.x == 0) *grand = carry;
}

__global__ void __launch_bounds__(kScanThreads) k_tile_scan(const int64_t *__restrict__ in, int64_t n,
                                                          const int64_t *__restrict__ offs,
                                                          int64_t *__restrict__ out) {
    __shared__ int64_t wt[32];
    const int64_t base = (int64_t)blockIdx.x * kScanTile + (int64_t)threadIdx.x * kScanItems;
    int64_t v[kScanItems], s = 0;
    for (int k = 0; k < kScanItems; k++) {
        v[k] = base + k < n ? in[base + k] : 0;
        s += v[k];
    }
    int64_t total;
    int64_t run = offs[blockIdx.x] + block_excl_scan(s, wt, total);
    for (int k = 0; k < kScanItems; k++) {
        if (base + k < n) out[base + k] = run;
        run += v[k];
    }
}

}  // namespace

void free_cells(CellBuffers *c, cudaStream_t st) {
    for (void *p : {(void *)c->cells, (void *)c->crects, (void *)c->cids, (void *)c->crad})
        if (p) cudaFreeAsync(p, st);
    *c = CellBuffers();
}

void attach_cells(DevLayout &L, const CellBuffers &c) {
    L.cells = c.cells;
    L.crects = c.crects;
    L.cids = c.cids;
    L.crad = c.crad;
    L.gx0 = c.gx0;
    L.gy0 = c.gy0;
    L.ginv = c.ginv;
    L.gnx = c.nx;
    L.gny = c.ny;
    L.tree_points = c.cells == nullptr || c.overflow > 0;
}

namespace {

// Coarse cells, of kCoarse x kCoarse cells each, serve the fine build on
// grids of at least kTwoLevelMin cells: their lists (from the tree, up to
// kCoarseCap rects) answer the fine cells' clearance and enumeration, so the
// tree is traversed once per coarse cell instead of once per cell.
constexpr int kCoarse = 4;
constexpr int64_t kTwoLevelMin = 1 << 16;
constexpr int kCoarseCap = 64;

// Count -> scan -> fill of the cells of grid G over L (with coarse lists of
// factor `factor` attached, or the tree alone); the cell buffers in C.
frw_status build_grid(const DevLayout &L, const Grid &G, int factor, double extra, int cap, cudaStream_t st,
                      CellBuffers &C) {
    const int64_t ncells = (int64_t)G.nx * G.ny;
    C.ncells = ncells;
    C.nx = G.nx;
    C.ny = G.ny;
    C.gx0 = G.gx0;
    C.gy0 = G.gy0;
    C.side = G.side;
    C.ginv = 1.0 / G.side;
    int64_t *cnt = nullptr, *start = nullptr, *sums = nullptr, *grand = nullptr;
    double *rad = nullptr;
    int32_t *stage = nullptr;
    unsigned long long *ovf = nullptr;
    const int64_t tiles = (ncells + kScanTile - 1) / kScanTile;
    frw_status rc = FRW_OK;
    auto ck = [&](cudaError_t e, const char *what) {
        if (e != cudaSuccess && rc == FRW_OK) rc = cuda_fail(e, what);
        return rc == FRW_OK;
    };
    do {
        if (!ck(cudaMallocAsync(&C.cells, (size_t)ncells * sizeof(int2), st), "malloc cells")) break;
        if (!ck(cudaMallocAsync(&C.crad, (size_t)ncells * sizeof(float), st), "malloc cell radii")) break;
        if (!ck(cudaMallocAsync(&cnt, (size_t)ncells * 8, st), "malloc cell counts")) break;
        if (!ck(cudaMallocAsync(&start, (size_t)ncells * 8, st), "malloc cell starts")) break;
        if (!ck(cudaMallocAsync(&rad, (size_t)ncells * 8, st), "malloc cell radii (build)")) break;
        if (!ck(cudaMallocAsync(&stage, (size_t)ncells * kStage * 4, st), "malloc staged rects")) break;
        if (!ck(cudaMallocAsync(&sums, (size_t)tiles * 8, st), "malloc tile sums")) break;
        // the list total and the overflow count side by side: one read-back
        if (!ck(cudaMallocAsync(&grand, 16, st), "malloc total")) break;
        ovf = reinterpret_cast<unsigned long long *>(grand + 1);
        if (!ck(cudaMemsetAsync(ovf, 0, 8, st), "memset")) break;
        const unsigned blocks = (unsigned)((ncells + 127) / 128);
        const int64_t nt = tiled_threads(G.nx, G.ny);
        k_cell_count<<<(unsigned)((nt + 127) / 128), 128, 0, st>>>(L, G, factor, extra, cap, cnt, C.cells, C.crad,
                                                                  rad, stage, ovf, nt);
        k_tile_sums<<<(unsigned)tiles, kScanThreads, 0, st>>>(cnt, ncells, sums);
        k_scan_sums<<<1, kScanThreads, 0, st>>>(sums, tiles, grand);
        k_tile_scan<<<(unsigned)tiles, kScanThreads, 0, st>>>(cnt, ncells, sums, start);
        if (!ck(cudaGetLastError(), "cell count")) break;
        unsigned long long h[2] = {0, 0};  // list total, overflowed cells
        if ((rc = read_back(h, grand, 16, st, "build_cells: list total"))) break;
        const int64_t total = (int64_t)h[0];
        if (total > INT32_MAX) {
            set_error("build_cells: more than 2^31 list entries; use fewer cells per rect");
            rc = FRW_E_ARG;
            break;
        }
        C.entries = total;
        C.overflow = (int64_t)h[1];
        if (!ck(cudaMallocAsync(&C.crects, (size_t)std::max<int64_t>(total, 1) * 16, st), "malloc cell rects")) break;
        if (!ck(cudaMallocAsync(&C.cids, (size_t)std::max<int64_t>(total, 1) * 4, st), "malloc cell ids")) break;
        if (total > 0)
            k_cell_fill<<<blocks, 128, 0, st>>>(L, G, factor, start, rad, stage, C.cells, C.crects, C.cids, ncells);
        if (!ck(cudaGetLastError(), "cell fill")) break;
    } while (0);
    for (void *p : {(void *)cnt, (void *)start, (void *)sums, (void *)grand, (void *)rad, (void *)stage})
        if (p) cudaFreeAsync(p, st);
    C.bytes = ncells * (int64_t)(sizeof(int2) + sizeof(float)) + C.entries * 20;
    return rc;
}

}  // namespace

frw_status build_cells(const DevLayout &Lin, double cells_per_rect, int cap, cudaStream_t st, CellBuffers *out) {
    *out = CellBuffers();
    if (!(cells_per_rect > 0) || cap < 1 || cap > (1 << 16)) {
        set_error("build_cells: cells_per_rect must be > 0 and max_per_cell in [1, 65536]");
        return FRW_E_ARG;
    }
    DevLayout L = Lin;
    L.cells = nullptr;  // the build queries the tree (and coarse lists of its own)
    const double W = L.bx1 - L.bx0, H = L.by1 - L.by0;
    const double target = std::min((double)kMaxCells, std::max(1.0, cells_per_rect * (double)L.n));
    double side = std::sqrt(std::max(W * H, 1e-300) / target);
    if (!(side > 0) || !std::isfinite(side)) side = std::max(std::max(W, H), 1.0);
    side = std::max(side, std::max(W, H) / 65536.0);  // at most 2^16 cells per axis
    if (!(side > 0)) side = 1.0;
    int64_t nx = 0, ny = 0;
    for (;;) {
        nx = std::max<int64_t>(1, (int64_t)std::ceil(W / side));
        ny = std::max<int64_t>(1, (int64_t)std::ceil(H / side));
        if (nx * ny <= kMaxCells && nx <= 65536 && ny <= 65536) break;
        side *= 1.25;
    }
    const int64_t ncells = nx * ny;
    const double M = 4.0 * std::max(std::max(std::max(std::fabs(L.bx0), std::fabs(L.by0)),
                                             std::max(std::fabs(L.bx1), std::fabs(L.by1))),
                                    std::max(W, H)) +
                     16.0;
    const double margin = std::ldexp(M, -30);
    const Grid G{L.bx0, L.by0, side, margin, (int)nx, (int)ny};

    cudaEvent_t e0, e1;
    FRW_CK(cudaEventCreate(&e0));
    FRW_CK(cudaEventCreate(&e1));
    CellBuffers C, K;  // the cells; coarse cells serving their build
    frw_status rc = FRW_OK;
    do {
        if (cudaEventRecord(e0, st) != cudaSuccess) {
            rc = cuda_fail(cudaGetLastError(), "event");
            break;
        }
        if (ncells >= kTwoLevelMin) {
            // coarse radius one margin above the Lipschitz bound r_cell <= r_coarse
            const Grid Gk{L.bx0, L.by0, side * kCoarse, margin, (int)((nx + kCoarse - 1) / kCoarse),
                          (int)((ny + kCoarse - 1) / kCoarse)};
            if ((rc = build_grid(L, Gk, 1, margin, kCoarseCap, st, K))) break;
            DevLayout Lk = L;
            attach_cells(Lk, K);
            rc = build_grid(Lk, G, kCoarse, 0.0, cap, st, C);
        } else {
            rc = build_grid(L, G, 1, 0.0, cap, st, C);
        }
        if (rc) break;
        if (cudaEventRecord(e1, st) != cudaSuccess) {
            rc = cuda_fail(cudaGetLastError(), "event");
            break;
        }
        if ((rc = wait_event(e1, "build_cells"))) break;
        cudaEventElapsedTime(&C.build_ms, e0, e1);
    } while (0);
    free_cells(&K, st);
    cudaEventDestroy(e0);
    cudaEventDestroy(e1);
    if (rc != FRW_OK) {
        free_cells(&C, st);
        return rc;
    }
    *out = C;
    return FRW_OK;
}

int64_t scan_i64_tiles(int64_t n) { return (n + kScanTile - 1) / kScanTile; }

void launch_scan_i64(const int64_t *in, int64_t n, int64_t *out, int64_t *sums, int64_t *grand, cudaStream_t st) {
    const int64_t tiles = scan_i64_tiles(n);
    k_tile_sums<<<(unsigned)tiles, kScanThreads, 0, st>>>(in, n, sums);
    k_scan_sums<<<1, kScanThreads, 0, st>>>(sums, tiles, grand);
    k_tile_scan<<<(unsigned)tiles, kScanThreads, 0, st>>>(in, n, sums, out);
}

}  // namespace frw
