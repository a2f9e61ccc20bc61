// frw3d_internal.h -- declarations of the 3-D walk path (host + device).
#pragma once

#include <cuda_runtime.h>
#include <stdint.h>

#include "../../include/frw3d.h"
#include "frw_internal.h"

namespace frw {

// ---- cell grid in HBM ----------------------------------------------------------
// Cubic cells of side s over the bounds.  Cell c lists every box whose
// L-infinity distance from the cell centre is at most D_c + 2 h + margin
// (D_c = distance from the centre to its nearest box, h = s/2): the nearest
// box of any point of the cell is among them.  Entries are copies of the
// boxes, two float4 each: (x0, y0, z0, id bits) and (x1, y1, z1, d_c) with
// d_c <= the box's distance from the cell centre, sorted by d_c: a query
// reads one 8-byte cell record and 32 bytes per candidate, and stops once
// d_c - (h + margin) exceeds its best distance.
//
// A cell whose search would reach more than kRingCap3 rings of cells (it lies
// far from every box) has no list of its own: its record holds kDefer3 and
// its points are looked up in the next level, a grid of cells twice as
// large with the same origin (cell i of level l lies in cell i >> 1 of level
// l + 1).  Coarser levels build lists only for the cells that deferred
// points reach; the top level (at most 2 kRingCap3 + 1 cells per axis) has
// no cap.  So the build visits at most (2 kRingCap3 + 1)^3 bins per cell
// however sparse the layout is.
constexpr int kRingCap3 = 4;
constexpr uint32_t kDefer3 = 0xFFFFFFFFu;
constexpr int kMaxLevels3 = 16;
constexpr uint32_t kSt3LevelChain = 1u;  // a lookup reached the top level without a list (never expected)

struct Level3 {
    const uint2 *cells;
    const float4 *lists;
    double ginv, hq;
    int nx, ny, nz, pad;
};

struct Dev3Layout {
    const uint2 *cells;    // [ncells] (first entry, entry count) or (0, kDefer3)
    const float4 *lists;   // [2 * entries]
    double g0x, g0y, g0z;  // grid origin (every level)
    double ginv;           // 1 / cell side
    double hq;             // half a cell side + rounding margin
    int nx, ny, nz;
    int nup;               // coarser levels
    const Level3 *up;      // [nup] device array
    uint32_t *status;      // kSt3* bits (device word of the layout)
    double b[6];           // bounds (x0,y0,z0,x1,y1,z1), open
};

struct Grid3Buffers {
    // level 0
    uint2 *cells = nullptr;
    float4 *lists = nullptr;
    int64_t ncells = 0, entries = 0;
    int nx = 0, ny = 0, nz = 0;
    double g0[3] = {0, 0, 0};
    double side = 0;
    double margin = 0;
    // coarser levels (device buffers owned here) and their descriptors
    int nup = 0;
    uint2 *up_cells[kMaxLevels3] = {};
    float4 *up_lists[kMaxLevels3] = {};
    Level3 *up = nullptr;          // device copy of the descriptors
    int64_t up_entries = 0;        // list entries of all coarser levels
    int64_t deferred = 0;          // level-0 cells that defer
    uint32_t *status = nullptr;
    int32_t max_list = 0;
    float build_ms = 0;
};

// Device copy of the cube table for one resolution n: CDF thresholds as
// 32-bit integers (bin b is chosen for a Philox word x iff thr[b] <= x <
// thr[b+1], thr[b] = ceil(intg[b] * 2^32) -- the same bin as comparing
// x * 2^-32 with intg in FP64), a guide over the top 14 bits of x, the
// first-hop weight vectors and the landing offsets (2 i + 1 - n) / n.
constexpr int kGuide3Bits = 14;
struct Cube3Tables {
    int n = 0, nb = 0;
    uint32_t *thr = nullptr;    // [nb]
    uint16_t *guide = nullptr;  // [1 << kGuide3Bits]
    double *w = nullptr;        // [3 nb]
    double *offs = nullptr;     // [n]
};

// One target of a batched run: its Gaussian box, area and box index.
struct Job3 {
    double G[6];
    double S;
    int64_t target;
};

struct Walk3Params {
    Dev3Layout L;
    const uint32_t *thr;
    const uint16_t *guide;
    const double *w;
    const double *offs;
    int n, nb;
    uint32_t magic_n, magic_nn;  // ceil(2^32 / n), ceil(2^32 / n^2) (n > 1)
    int refill_min;              // refill idle lanes once this many are idle (1..32)
    uint32_t start_strata;       // 0 = off; S: walk w starts in stratum w mod S
    double G[6];  // Gaussian box
    double S;     // its area
    int64_t target;
    double shell;
    int64_t hop_cap;
    double perm;
    uint64_t seed;
    uint32_t stream;
    uint64_t first, walks;
    unsigned long long *counter;  // walks claimed (cleared by the caller)
    // rows (capacitance mode): per box, plus stats[4] = escaped, aborted, hops, walks
    unsigned long long *hits;
    double *sum_w, *sum_w2;
    unsigned long long *stats;
    // batched runs (k_walk3<true>): walk j is walk j % walks_per_job of job
    // j / walks_per_job; rows and stats of job t start at t * nboxes, 4 t
    const Job3 *jobs;
    uint64_t walks_per_job;
    int64_t nboxes;
    // records (trace mode), indexed by walk - first
    int64_t *rec_end;
    int32_t *rec_hops, *rec_bin;
    double *rec_w;
};

// host_cube_green.cpp
// Cube table of resolution n (6 n^2 bins), bit-identical to the reference's
// precompute_unit_cube_green; computed once per n and cached.  Any output
// may be NULL.  Returns false for n outside [1, FRW3_NSAMPLE_MAX].
bool cube_green_table(int n, double *g, double *dgdx, double *dgdy, double *dgdz, double *intg);
double cube_green_point(double a, double eta, double dzeta);
void cube_deriv_point(double *dg, double a, double eta, double dzeta);
// Host images of the device tables (thresholds, guide, weights, offsets).
bool cube_walk_tables(int n, uint32_t *thr, uint16_t *guide, double *w, double *offs);

// walk3d.cu
frw_status build_grid3(const float *d_boxes, int64_t n, const double bounds[6], double cells_per_box,
                       cudaStream_t stream, Grid3Buffers *out);
void free_grid3(Grid3Buffers *g, cudaStream_t stream);
void attach_grid3(Dev3Layout &L, const Grid3Buffers &g, const double bounds[6]);
frw_status launch_query3(const Dev3Layout &L, const double *d_pts, int64_t n, double *d_clear,
                         int64_t *d_nearest, cudaStream_t stream);
frw_status launch_walk3(const Walk3Params &P, int blocks, cudaStream_t stream);
frw_status launch_walk3_batch(const Walk3Params &P, int blocks, cudaStream_t stream);
int walk3_max_blocks_per_sm();
int walk3_threads();

}  // namespace frw
