/*
 * frwcpu3d.h -- CPU oracle for the 3-D floating-random-walk path.
 *
 * TEST INFRASTRUCTURE ONLY.  Nothing in the product (engineer-thesis_b200/)
 * includes, links or calls this code; only tests/, the smoke check and the
 * CPU-baseline leg of bench.py load liboracle.so, and only as the checker.
 *
 * The reference (piogrzej/engineer-thesis, randomWalk/) ships the unit-cube
 * surface Green's function -- green_cube, deriv_green_cube and
 * precompute_unit_cube_green (green/green.h:64-80, green/green.cpp:232-431)
 * -- but never calls it: it has no 3-D walk.  This file holds
 *   - the cube table, restated from the mathematics (Poisson kernel of a
 *     cube seen from its centre) and pinned bit-for-bit against the
 *     reference's own precompute_unit_cube_green compiled from its sources
 *     (oracle/_ref);
 *   - the 3-D walk the library runs on the GPU, written here as the
 *     definition its kernels are checked against (brute-force nearest box,
 *     or a cell grid whose answers equal the brute force).  There is no
 *     reference walk to pin it against: parity for the walk is GPU == this
 *     file, bit for bit, plus the physical identities the tests check.
 *
 * Boxes are 6 doubles (x0, y0, z0, x1, y1, z1), x0 < x1, y0 < y1, z0 < z1.
 */
#ifndef FRWCPU3D_H
#define FRWCPU3D_H

#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

#define OC3_END_ESCAPED (-1)
#define OC3_END_ABORTED (-2)

/* precompute_unit_cube_green(g, dgdx, dgdy, dgdz, intg, n): 6 n^2 samples
 * (face k, row i, column j at index k n^2 + i n + j) of the surface Green's
 * function of the unit cube seen from its centre, its negated gradient with
 * respect to the centre, and the normalised cumulative intg[6 n^2 + 1]. */
void oc3_cube_green_table(int n, double *g, double *dgdx, double *dgdy, double *dgdz, double *intg);
/* Green's function of a cube of side a at surface parameter (eta, dzeta) in
 * [0, 6a)^2 (green_cube, green/green.cpp:232-267) and its negated gradient
 * (deriv_green_cube, green/green.cpp:311-388). */
double oc3_green_cube(double a, double eta, double dzeta);
void oc3_deriv_green_cube(double *dg, double a, double eta, double dzeta);

/* First-hop weight vectors w[3 b + c] = dg_c(b) * (1 / n^2) / (intg[b+1] - intg[b]). */
void oc3_weight_table(int n, const double *intg, const double *dgdx, const double *dgdy,
                      const double *dgdz, double *w);

/* Bounding box of the boxes grown by int(0.01 * x extent) on every side (the
 * 2-D reader's rule, CPU/Parser.cpp:51-87, applied to three axes). */
void oc3_layout_bounds(const double *boxes, int64_t n, double out[6]);
/* 1e-3 x the smallest box edge: the default absorption shell. */
double oc3_default_shell(const double *boxes, int64_t n);

/* L-infinity distance from p to the nearest box and its index (ties: lowest
 * index), by brute force. */
void oc3_nearest(const double *boxes, int64_t n, const double p[3], double *d, int64_t *id);

/* A uniform cell grid over the bounds with the boxes binned by overlap; its
 * nearest-box answers equal oc3_nearest's.  with_lists: also build per-cell
 * candidate lists (fast queries; the build costs seconds at 10^6 boxes),
 * else every query runs a ring search over the bins. */
typedef struct oc3_grid oc3_grid;
oc3_grid *oc3_grid_create(const double *boxes, int64_t n, const double bounds[6], double boxes_per_cell,
                          int with_lists);
void oc3_grid_destroy(oc3_grid *g);
void oc3_grid_nearest(const oc3_grid *g, const double p[3], double *d, int64_t *id);

/* nearest for m points (grid may be NULL: brute force). */
void oc3_query_batch(const double *boxes, int64_t n, const oc3_grid *grid, const double *pts, int64_t m,
                     double *d, int64_t *id);

typedef struct oc3_cfg {
    int64_t target;
    double offset;       /* Gaussian surface = target grown by offset on every side */
    double shell;        /* a walk ends on the nearest box once within this distance */
    int64_t hop_cap;     /* walks with this many clearance queries end as aborted */
    double permittivity;
    uint64_t seed;
    uint32_t stream;
    int nsample;         /* cube table resolution n (6 n^2 bins) */
    uint32_t start_strata; /* 0 = off; S > 0: walk w starts in stratum w mod S of the surface */
} oc3_cfg;

/* Walks first .. first+count-1 (grid may be NULL: brute force).  Per walk:
 * end box (or OC3_END_*), clearance queries, first-hop bin (-1 without one)
 * and the capacitance weight c = eps * S * (w_bin . n0) / a0. */
int oc3_walk_run(const double *boxes, int64_t n, const double bounds[6], const oc3_grid *grid,
                 const oc3_cfg *cfg, uint64_t first, uint64_t count, int64_t *end, int32_t *hops,
                 int32_t *bin1, double *weight);

#ifdef __cplusplus
}
#endif

#endif /* FRWCPU3D_H */
