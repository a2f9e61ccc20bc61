/*
 * frw3d.h -- C ABI of the 3-D floating-random-walk path (box conductors,
 * cube transition domains) of the B200 FRW library (libfrw.so).
 *
 * Status codes, frw_last_error(), frw_device_check() and the stream and
 * memory conventions are those of frw.h.
 *
 * Correspondence with the reference (piogrzej/engineer-thesis, randomWalk/):
 *   frw3_cube_green_table   <- precompute_unit_cube_green
 *       (green/green.h:79-80, green/green.cpp:392-431), bit-identical
 *   frw3_green_cube         <- green_cube (green/green.h:71, green/green.cpp:232-267)
 *   frw3_deriv_green_cube   <- deriv_green_cube (green/green.h:75, green/green.cpp:311-388)
 *   frw3_layout_from_file   <- the multi-layer reader (CPU/Parser.cpp:15-50,
 *       layers closed by "<<" lines) with every layer extruded to a z range
 * The reference ships the cube Green's function but never calls it: it has
 * no 3-D walk, query or layout.  The walk here is the 2-D walk of
 * CPU/mainFunctions.cpp:48-90 lifted to three dimensions:
 *   - the transition domain at p is the largest cube centred on p that
 *     touches no box: half-side d = L-infinity distance from p to the nearest
 *     box (ties: lowest index), found through a cell grid on the device;
 *   - the walk ends on that box when d <= shell, leaves through the bounds
 *     (open box, potential 0) or ends as aborted after hop_cap queries;
 *   - otherwise it lands on the cube's surface at the centre of one of the
 *     6 n^2 table cells, drawn from the cube table's CDF with one 32-bit
 *     Philox4x32-10 word;
 *   - walks start uniformly on the Gaussian box (target grown by an offset)
 *     and carry the capacitance weight c = eps * S * (w_b . n0) / a0
 *     (S = Gaussian area, n0 its outward normal at the start, a0 = side of the
 *     first cube, w_b = -grad G(b) * (1/n^2) / P(b) from the table's
 *     derivative columns).
 */
#ifndef FRW3D_H
#define FRW3D_H

#include <stddef.h>
#include <stdint.h>

#include "frw.h"

#ifdef __cplusplus
extern "C" {
#endif

typedef struct frw3_layout frw3_layout;

#define FRW3_NSAMPLE_DEFAULT 50 /* cube table cells per face edge (6 * 50^2 bins) */
#define FRW3_NSAMPLE_MAX 100

/* ---- cube Green's function (host, FP64) ---- */
/* precompute_unit_cube_green(g, dgdx, dgdy, dgdz, intg, n): 6 n^2 entries per
 * array (face k, row i, column j at k n^2 + i n + j), intg has 6 n^2 + 1.
 * Any pointer may be NULL.  n in [1, FRW3_NSAMPLE_MAX]. */
frw_status frw3_cube_green_table(int n, double *g, double *dgdx, double *dgdy, double *dgdz, double *intg);
/* green_cube(a, eta, dzeta) and deriv_green_cube(dg, a, eta, dzeta):
 * eta, dzeta in [0, 6a) on the same face; dg = -grad G. */
frw_status frw3_green_cube(double a, double eta, double dzeta, double *g);
frw_status frw3_deriv_green_cube(double a, double eta, double dzeta, double dg[3]);

/* ---- layouts ---- */
/* boxes: host array of n*6 floats (x0,y0,z0,x1,y1,z1), x0 < x1, y0 < y1,
 * z0 < z1, interiors pairwise disjoint (checked; touching faces allowed).
 * The device grid has cells_per_box x n cells; cells far from every box
 * (empty regions, wide bounds) defer to coarser grids, so the build visits a
 * bounded number of bins per cell however sparse the layout is.
 * bounds: 6 doubles (x0,y0,z0,x1,y1,z1) or NULL for the bounding box grown
 * by int(0.01 * x extent) on every side (the 2-D reader's rule,
 * CPU/Parser.cpp:51-87).  cells_per_box: cell-grid density (<= 0: 8). */
frw_status frw3_layout_create(const float *boxes, int64_t n, const double *bounds, double cells_per_box,
                              int device, frw3_layout **out);
/* Reads every layer of a reference layout file and extrudes layer k to
 * [z0[k], z1[k]]; nz must equal the file's layer count (after the skipped
 * first one).  bounds as above. */
frw_status frw3_layout_from_file(const char *path, const double *z0, const double *z1, int nz,
                                 const double *bounds, double cells_per_box, int device, frw3_layout **out);
frw_status frw3_layout_destroy(frw3_layout *layout);

typedef struct frw3_layout_info {
    int64_t n;              /* boxes */
    int device;
    int32_t grid[3];        /* cells per axis */
    double bounds[6];
    double cell_side;
    double min_edge;        /* smallest box edge (default shell = 1e-3 x this) */
    int64_t list_entries;   /* total length of the per-cell candidate lists */
    int32_t max_list;       /* longest list */
    double mean_list;       /* mean list length over cells */
    float build_ms;         /* device time of the grid build */
    int32_t levels;         /* grid levels: 1 + the coarser levels that far cells defer to */
    int64_t deferred_cells; /* finest-level cells far from every box (looked up one level up) */
    int64_t upper_entries;  /* list entries of the coarser levels */
} frw3_layout_info;
frw_status frw3_layout_info_get(const frw3_layout *layout, frw3_layout_info *info);
/* The layout's boxes (n*6 floats, input order). */
frw_status frw3_layout_boxes(const frw3_layout *layout, float *out);

/* ---- queries ---- */
/* For each point (x,y,z): clearance d (L-infinity distance to the nearest
 * box, 0 inside one) and that box's index (ties: lowest).  mem: FRW_MEM_*
 * for all four pointers. */
frw_status frw3_query_batch(const frw3_layout *layout, const double *pts_xyz, int64_t n, double *clear,
                            int64_t *nearest, int mem, void *stream);

/* ---- walks ---- */
typedef struct frw3_opts {
    uint32_t struct_size;  /* sizeof(frw3_opts) */
    double gauss_offset;   /* Gaussian box = target grown by this on every side (> shell) */
    double shell;          /* absorption distance; <= 0: 1e-3 x the smallest box edge */
    int64_t hop_cap;
    double permittivity;   /* F/m */
    uint32_t stream_id;    /* Philox counter word 3 */
    int32_t nsample;       /* cube table cells per face edge */
    uint64_t first_walk;   /* Philox index of the first walk (runs over disjoint ranges add up) */
    int32_t blocks_per_sm; /* 0: library choice */
    int32_t refill_min;    /* a warp starts new walks once this many lanes are idle (default 4; 0 or 1: at
                              once; <= 32).  Results do not depend on it. */
    uint32_t start_strata; /* 0 = off; S > 0: walk w starts in stratum w mod S of the Gaussian surface (its
                              first uniform u0 becomes (w mod S + u0) / S, which orders the surface by
                              face and position), as frw_opts.start_strata does in 2-D.  Unbiased when the
                              walk range covers every stratum equally; the reported standard error stays the
                              i.i.d. one, an upper bound. */
} frw3_opts;
void frw3_opts_default(frw3_opts *opts);

typedef struct frw3_result {
    uint64_t walks, escaped, aborted, hops_total;
    double gauss[6];
    double shell;            /* the shell used */
    double fraction_other;   /* walks not ending on the target, escapes included */
    double kernel_ms;
    int64_t capacity;        /* length of the caller-owned rows below */
    int64_t n_entries;       /* boxes reached (may exceed capacity: rows truncated) */
    int64_t *conductor;      /* box index, ascending */
    uint64_t *hits;
    double *cap;             /* C_target,k in F (capacitance weights / walks) */
    double *cap_se;
    double *sum_w;           /* optional */
    double *sum_w2;          /* optional */
} frw3_result;

/* `walks` walks from the Gaussian box of box `target`; walk i draws only
 * from (seed, stream_id, first_walk + i), so results do not depend on the
 * launch configuration. */
frw_status frw3_walk(const frw3_layout *layout, int64_t target, uint64_t walks, uint64_t seed,
                     const frw3_opts *opts, frw3_result *result, void *stream);
/* The same walks accumulated into caller-owned DEVICE arrays on the layout's
 * device, stream-ordered, without host synchronisation (the 3-D twin of
 * frw_walk_device): for every box k (arrays of n entries) hits[k] += walks
 * ending on k, sum_w[k] += their weights, sum_w2[k] += the squared weights;
 * stats[0..3] += escaped, aborted, clearance queries, walks done;
 * *status |= grid lookup failure bits (never expected; nonzero: treat as
 * FRW_E_KERNEL).  The caller clears the arrays once; runs over disjoint walk
 * ranges add up, and so do the arrays of several devices (one all-reduce).
 * A walk counter comes from the device's stream-ordered memory pool. */
frw_status frw3_walk_device(const frw3_layout *layout, int64_t target, uint64_t walks, uint64_t seed,
                            const frw3_opts *opts, uint64_t *hits, double *sum_w, double *sum_w2, uint64_t *stats,
                            uint32_t *status, void *stream);
/* Several targets of one layout in one persistent launch (rows of a
 * capacitance matrix): walks_per_target walks from each of targets[0..T-1],
 * results[t] filled as frw3_walk fills its result (caller-owned rows, the
 * launch's kernel_ms in every entry).  Walk i of target t draws the same
 * random numbers as walk i of frw3_walk(target t) with the same seed and
 * options, so each row equals that call's (the reference's getAvgPathLen
 * runs one target per call, CPU/getAvgPathLen.cpp:35-114).  T x n must stay
 * below 2^27: every target's full row is accumulated on the device. */
frw_status frw3_walk_batch(const frw3_layout *layout, const int64_t *targets, int32_t ntargets,
                           uint64_t walks_per_target, uint64_t seed, const frw3_opts *opts, frw3_result *results,
                           void *stream);
/* Per-walk records (arrays of `walks` entries, any may be NULL): end box
 * (-1 escaped, -2 aborted), clearance queries, first-hop bin (-1 none) and
 * the capacitance weight c. */
frw_status frw3_walk_trace(const frw3_layout *layout, int64_t target, uint64_t first_walk, uint64_t walks,
                           uint64_t seed, const frw3_opts *opts, int64_t *end, int32_t *hops, int32_t *bin1,
                           double *weight, int mem, void *stream);

/* Seeded synthetic layout: n boxes with integer corners uniform in
 * [0,domain)^2 x [0,zdomain), edges uniform integers in [wmin, wmax]
 * (z edges in [zmin, zmax]), L-infinity gap >= gap; splitmix64 from seed. */
frw_status frw3_generate_layout(uint64_t seed, int64_t n, double domain, double zdomain, int32_t wmin,
                                int32_t wmax, int32_t zmin, int32_t zmax, int32_t gap, float *out);

#ifdef __cplusplus
}
#endif

#endif /* FRW3D_H */
