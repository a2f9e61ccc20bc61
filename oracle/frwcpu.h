/*
 * frwcpu.h -- CPU oracle for the floating-random-walk (FRW) hot path.
 *
 * TEST INFRASTRUCTURE ONLY.  Nothing in the product (engineer-thesis_b200/)
 * includes, links or calls this code; only tests/, the smoke check and the
 * CPU-baseline leg of bench.py load liboracle.so, and only as the checker.
 *
 * This is an FP64 restatement, in plain C, of the reference's CPU path
 * (piogrzej/engineer-thesis, randomWalk/):
 *   - layout reader            CPU/Parser.cpp:15-125
 *   - rectangle geometry       CPU/rectHost.cpp:43-161
 *   - quadtree + queries       CPU/quadTree.cpp:38-364
 *   - walk loop                CPU/mainFunctions.cpp:40-90
 *   - estimator                CPU/getAvgPathLen.cpp:91-113
 *   - unit-square Green table  green/green.cpp:125-152 (restated from the
 *                              mathematics: Poisson kernel of a square)
 * Two query semantics are provided:
 *   complete  -- the predicate the reference intends (and its GPU DFS
 *                implements, Cuda/d_quadTree.cu:136-193): a box collides when
 *                it leaves the layer bounds or overlaps ANY rectangle;
 *   defect    -- the reference CPU tree exactly as shipped, including the
 *                sibling-stack defect of Tree::checkCollisions
 *                (CPU/quadTree.cpp:148-198, addNodesToStack receives its
 *                stack pointer by value) and first-child point descent
 *                (CPU/quadTree.cpp:240-262).
 * Parity pins: the defect mode is checked bit-for-bit against the reference
 * compiled from its own sources (oracle/_ref), and the Green table against
 * the reference's precompute_unit_square_green output.
 *
 * Rectangles are 4 doubles (x0, y0, x1, y1) = (topLeft.x, topLeft.y,
 * bottomRight.x, bottomRight.y) with y growing downwards as in the
 * reference's layout files.
 */
#ifndef FRWCPU_H
#define FRWCPU_H

#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

#define OC_NSAMPLE 200          /* defines.h:28 NSAMPLE */
#define OC_MAX_LEVELS 11        /* defines.h:20 MAX_LEVELS */
#define OC_MAX_OBJECTS 4        /* defines.h:23 MAX_OBJECTS */
#define OC_GAUSS_ACCURACY 10    /* defines.h:22 GAUSSIAN_ACCURACY */
#define OC_INIT_FACTOR 0.05     /* defines.h:21 BIGGEST_SQUARE_INIT_FACTOR */
#define OC_BOUNDS_MUL 0.01      /* defines.h:17 BOUNDS_MUL_FACTOR */
#define OC_PERMITTIVITY 8.854187817620e-12

/* ---- status codes (mirror include/frw.h) ---- */
#define OC_OK 0
#define OC_E_ARG -1
#define OC_E_IO -2
#define OC_E_OOM -4

/* ---- layout reader ---- */
/* Parse a reference layout file; returns the rects of layer `layer` in file
 * order (malloc'd, free with oc_free) and the number of layers found. */
int oc_parse_layout(const char *path, int layer, double **rects_out,
                    int64_t *n_out, int *nlayers_out);
void oc_free(void *p);
/* Parser::getLayerSize (CPU/Parser.cpp:51-87). */
void oc_layer_bounds(const double *rects, int64_t n, double out[4]);

/* ---- Green's function tables ---- */
/* g[nsample] and the normalised cumulative intg[nsample+1] of the unit-square
 * Poisson kernel seen from the centre (reference truncation: odd n <= 19). */
void oc_green_table(int nsample, double *g, double *intg);
/* Per-bin first-hop gradient weights W_i = (Delta eta / pi_i) * grad K at the
 * landing point of bin i (unit square, screen axes, clockwise from the
 * top-left corner, bin i lands on segment i-1).  Corner bins get 0. */
void oc_weight_table(int nsample, const double *intg, double *wx, double *wy);
/* Linear CDF scan of mainFunctions.cpp:40-46, clamped to [0, nsample-1]. */
int oc_bin_index(const double *intg, int nsample, double r);

/* ---- Philox4x32-10 (Salmon et al., SC'11) ---- */
void oc_philox4x32_10(const uint32_t ctr[4], const uint32_t key[2], uint32_t out[4]);
/* 53-bit uniform in [0,1) from two 32-bit words. */
double oc_u01(uint32_t a, uint32_t b);

/* ---- geometry ---- */
/* RectHost::getPointFromNindex (CPU/rectHost.cpp:107-161).  exact_perimeter=0
 * truncates the perimeter to int as the CPU reference does
 * (rectHost.cpp:102-105); 1 keeps it double as the GPU reference does
 * (Cuda/d_Rect.cu:29-32). */
void oc_point_from_index(const double sq[4], int index, int nsample,
                         int exact_perimeter, double out[2]);
/* RectHost::createGaussianSurface (CPU/rectHost.cpp:84-100). */
void oc_scale_rect(const double r[4], double fx, double fy, double out[4]);

/* ---- complete index (uniform grid; exact brute-force predicate) ---- */
typedef struct oc_grid oc_grid;
oc_grid *oc_grid_create(const double *rects, int64_t n, const double bounds[4]);
void oc_grid_destroy(oc_grid *g);
/* Tree::checkCollisions(box, ignore) with complete semantics.  ignore may be
 * NULL; rects equal to *ignore coordinate-wise are skipped. */
int oc_grid_box_collides(const oc_grid *g, const double box[4], const double *ignore);
/* Lowest layer index of a rect containing p (closed), or -1. */
int64_t oc_grid_point_hit(const oc_grid *g, double px, double py);
/* Tree::drawBiggestSquareAtPoint (CPU/quadTree.cpp:264-312), complete. */
void oc_grid_biggest_square(const oc_grid *g, double px, double py, double out[4]);
void oc_grid_query_batch(const oc_grid *g, const double *pts, int64_t n,
                         double *sq_out, int64_t *hit_out);
/* Tree::creatGaussianSurfFrom (CPU/quadTree.cpp:315-364), complete. */
void oc_grid_gauss_scale(const oc_grid *g, const double r[4], double factor, double out[4]);

/* ---- reference CPU quadtree, restated with its insertion-order structure ---- */
typedef struct oc_rtree oc_rtree;
oc_rtree *oc_rtree_create(const double *rects, int64_t n, const double bounds[4]);
void oc_rtree_destroy(oc_rtree *t);
/* defect=1: sibling-stack defect as shipped; defect=0: complete DFS. */
int oc_rtree_box_collides(const oc_rtree *t, const double box[4], const double *ignore, int defect);
/* First-child descent of CPU/quadTree.cpp:240-262; returns the layer index
 * of the rect found or -1. */
int64_t oc_rtree_point_hit(const oc_rtree *t, double px, double py);
void oc_rtree_biggest_square(const oc_rtree *t, double px, double py, int defect, double out[4]);
void oc_rtree_gauss_scale(const oc_rtree *t, const double r[4], double factor, int defect, double out[4]);
void oc_rtree_stats(const oc_rtree *t, int64_t *nodes, int64_t *stored_objects, int *max_level);

/* ---- walks ---- */
#define OC_GAUSS_SCALE 0
#define OC_GAUSS_OFFSET 1
#define OC_START_GREEN 0
#define OC_START_UNIFORM 1
#define OC_END_ESCAPED (-1)
#define OC_END_ABORTED (-2)

typedef struct oc_walk_cfg {
    int64_t target;        /* layer index of the target conductor */
    int gauss_mode;        /* OC_GAUSS_SCALE | OC_GAUSS_OFFSET */
    double gauss_param;    /* scale factor or offset */
    int start_mode;        /* OC_START_GREEN | OC_START_UNIFORM */
    int exact_perimeter;   /* see oc_point_from_index */
    int64_t hop_cap;       /* walks longer than this end as aborted */
    double permittivity;
    uint64_t seed;
    uint32_t stream;       /* Philox counter word 3 */
    uint32_t start_grid;   /* uniform start: 0 continuous, Q = midpoints of Q equal arcs */
    uint32_t start_strata; /* 0 off; S: walk w starts in stratum w mod S, u = (w mod S + u) / S */
} oc_walk_cfg;

/* Gaussian surface of cfg->target (complete semantics). */
void oc_walk_gauss_surface(const oc_grid *g, const double *rects, const oc_walk_cfg *cfg,
                           double out[4]);
/* Run walks [first, first+count) of the Philox stream; per-walk records:
 * end conductor (layer index / OC_END_*), hop count, first-hop bin and the
 * weight factor c (0 without a first hop or in green-start mode; the walk
 * adds c to its end conductor only).  cv_out (nullable): 4 doubles per walk,
 * first-hop point x, y, first square side a0, c. */
int oc_walk_run(const oc_grid *g, const double *rects, const oc_walk_cfg *cfg,
                uint64_t first, uint64_t count, int64_t *end_out, int32_t *hops_out,
                int32_t *bin_out, double *weight_out, double *cv_out);
/* One reference-style walk driven by an explicit stream of uniforms r in
 * [0,1) (green-start mode, CPU perimeter), on either the grid (complete) or
 * the restated reference tree (defect=1/0).  Returns the end rect index or
 * OC_END_ESCAPED; *used = uniforms consumed, *hops = query count. */
int64_t oc_walk_stream(const oc_grid *g, const oc_rtree *t, int defect,
                       const double gauss[4], const double *intg, const double *r,
                       int64_t nr, int64_t *used, int32_t *hops);

/* ---- synthetic layouts ---- */
/* The benchmark layouts, restated from the product's generator contract
 * (include/frw.h, frw_generate_layout) so that CPU-side legs can make the
 * same rects without loading the product library: a splitmix64 stream from
 * `seed`; per attempt w = U[wmin, wmax], h = U[wmin, wmax], x0 = U[0, D - w],
 * y0 = U[0, D - h] (U[a, b] = a + next() mod (b - a + 1), D = floor(domain));
 * accepted when the L-infinity gap to every accepted rect is >= gap.  Writes
 * n*4 doubles (integers); returns OC_E_ARG when 64*n + 1000 attempts do not
 * place n rects.  The reference's own generator (utils/TestGenerator.cpp:
 * 49-105, sizes 1-24, no gap) is not used by any benchmark config. */
int oc_generate_layout(uint64_t seed, int64_t n, double domain, int wmin, int wmax, double gap,
                       double *out);

/* ---- control-variate features ---- */
/* For each point rec4[i] = (x, y, a0, unused): (dx, dy) from the point to the
 * nearest point of each edge (top, right, bottom, left) of rect `target`,
 * then of the nearest other rect (smallest L-inf gap, then smallest index),
 * each divided by a0 and clamped to [-16, 16]; 16 floats per point, all 0
 * when a0 <= 0, the second eight 16 when there is no other rect. */
void oc_cv_features(const double *rects, int64_t n, int64_t target, const double *rec4, int64_t m,
                    float *out);

#ifdef __cplusplus
}
#endif
#endif
