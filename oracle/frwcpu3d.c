/*
 * frwcpu3d.c -- CPU oracle for the 3-D floating-random-walk path.
 * TEST INFRASTRUCTURE ONLY (see frwcpu3d.h).  Compiled with
 * -ffp-contract=off: every expression rounds exactly as written, which the
 * GPU kernels reproduce with _rn intrinsics.
 */
#include "frwcpu3d.h"
#include "frwcpu.h"

#include <math.h>
#include <stdlib.h>
#include <string.h>

#define PI_D 3.14159265358979323846

/* ------------------------------------------------------------------------ */
/* Green's function of the unit cube seen from its centre                   */
/* ------------------------------------------------------------------------ */
/*
 * Laplace's equation in [0,a]^3 with data f on the face z = 0 and zero on the
 * other faces is solved by
 *   u(x,y,z) = sum_{m,n>=1} b_mn sin(m pi x/a) sin(n pi y/a) sinh(g_mn (a-z)/a) / sinh(g_mn),
 *   b_mn = (4/a^2) int f(x,y) sin(m pi x/a) sin(n pi y/a) dx dy,   g_mn = pi sqrt(m^2+n^2),
 * so from the centre the landing density on that face is
 *   K(x,y) = (4/a^2) sum_{m,n odd} s_m s_n sin(m pi x/a) sin(n pi y/a) / (2 cosh(g_mn/2)),
 * s_k = sin(k pi/2) = (-1)^((k-1)/2), and 1/(2 cosh(g/2)) = q (1-q^2)/(1-q^4)
 * with q = e^{-g/2}.  The six faces are parametrised by (eta, dzeta) in
 * [k a, (k+1) a)^2 (green/green.h:66-70); for odd m and n the shift by k a
 * multiplies both sines by (-1)^k, so one formula covers all faces.  Terms
 * up to m, n = 19 (NTERMS 20, green/green.cpp:21) are summed m-major with the
 * factors multiplied in the order of green/green.cpp:232-267, which makes the
 * table bit-identical to the reference's (checked against oracle/_ref).
 */
static double sg(unsigned k) { return ((k >> 1) & 1u) ? -1.0 : 1.0; } /* s_k for odd k, cos(k pi/2) for even k */

double oc3_green_cube(double a, double eta, double dzeta) {
    const double pi = PI_D;
    double es = pi * eta / a, zs = pi * dzeta / a;
    double acc = 0.0;
    for (uint64_t m = 1; m <= 20; m += 2) {
        double sin_m = sg((unsigned)m) * sin((double)m * es);
        for (uint64_t n = 1; n <= 20; n += 2) {
            double e = -0.5 * sqrt((double)(m * m + n * n)) * pi;
            double q = exp(e);
            double c = q * (1.0 - q * q) / (1.0 - exp(4.0 * e));
            acc += sg((unsigned)n) * c * sin((double)n * zs) * sin_m;
        }
    }
    return acc * (4 / (a * a));
}

/*
 * Gradient of K with respect to the source point, at the centre, in the
 * face's own parameters (es along its first axis, zs along its second, both
 * scaled by pi/a); the caller multiplies by -4 pi / a^3:
 *   normal   A = sum_{m,n odd}         s_m s_n r_mn c'_mn sin(m es) sin(n zs)
 *   1st axis B = sum_{m even, n odd}   m t_m s_n c_mn     sin(m es) sin(n zs)
 *   2nd axis C = sum_{m odd, n even}   n s_m t_n c_mn     sin(m es) sin(n zs)
 * r_mn = sqrt(m^2+n^2), c_mn = 1/(2 cosh(g/2)), c'_mn = q (1+q^2)/(1-q^4) =
 * 1/(2 sinh(g/2)), t_k = cos(k pi/2); m, n run to 20 (green/green.cpp:270-306).
 */
static void face_grad(double es, double zs, double *A, double *B, double *C) {
    const double pi = PI_D;
    double a = 0.0, b = 0.0, c = 0.0;
    for (unsigned m = 1; m <= 20; m++) {
        double sin_m = sin(m * es);
        for (unsigned n = 1; n <= 20; n++) {
            double r = sqrt((double)(m * m + n * n));
            double e = -0.5 * sqrt((double)(m * m + n * n)) * pi;
            double q = exp(e);
            double den = 1.0 - exp(4.0 * e);
            double sin_n = sin(n * zs);
            double s = sg(m) * sg(n);
            if (n & 1) {
                if (m & 1) a += s * (r * (q * (1.0 + q * q) / den) * sin_n * sin_m);
                else b += s * (m * (q * (1.0 - q * q) / den) * sin_n * sin_m);
            } else if (m & 1) {
                c += s * (n * (q * (1.0 - q * q) / den) * sin_n * sin_m);
            }
        }
    }
    *A = a;
    *B = b;
    *C = c;
}

/*
 * -grad K on the face that (eta, dzeta) lies on (green/green.cpp:311-388).
 * Faces: 0 (u,v,0)  1 (1,u,v)  2 (1-v,1,u)  3 (1-u,1-v,1)  4 (0,1-u,1-v)
 * 5 (v,0,1-u) in units of a, u = eta - k a, v = dzeta - k a.  Faces 2 and 5
 * take their first axis from v.  The face's normal sum and its two tangential
 * sums land on the cube axes with the signs of that parametrisation.
 */
void oc3_deriv_green_cube(double *dg, double a, double eta, double dzeta) {
    const double pi = PI_D;
    int k = eta < a ? 0 : eta < 2 * a ? 1 : eta < 3 * a ? 2 : eta < 4 * a ? 3 : eta < 5 * a ? 4 : 5;
    double es = pi * (eta - k * a) / a, zs = pi * (dzeta - k * a) / a;
    double A, B, C, x, y, z;
    if (k == 2 || k == 5) face_grad(zs, es, &A, &B, &C);
    else face_grad(es, zs, &A, &B, &C);
    switch (k) {
    case 0: x = B; y = C; z = -A; break;
    case 1: x = A; y = B; z = C; break;
    case 2: x = -B; y = A; z = C; break;
    case 3: x = -B; y = -C; z = A; break;
    case 4: x = -A; y = -B; z = -C; break;
    default: x = B; y = -A; z = -C; break;
    }
    double scale = -4.0 * pi / (a * a * a);
    dg[0] = x * scale;
    dg[1] = y * scale;
    dg[2] = z * scale;
}

/* Samples at the centres (eta, dzeta) = ((i+1/2)/n, (k n + j + 1/2)/n) of an
 * n x n grid on every face; the running sum of g times the cell area,
 * normalised to 1 at the end (green/green.cpp:392-431). */
void oc3_cube_green_table(int n, double *g, double *dgdx, double *dgdy, double *dgdz, double *intg) {
    size_t N = (size_t)n;
    double delta = 1.0 / n;
    double prev_int = 0.0, prev_g = 0.0;
    for (size_t k = 0; k < 6; k++)
        for (size_t i = k * N; i < (k + 1) * N; i++)
            for (size_t j = 0; j < N; j++) {
                double eta = (i + 0.5) * delta;
                double dzeta = (k * N + j + 0.5) * delta;
                size_t idx = i * N + j;
                double d[3];
                double gv = oc3_green_cube(1.0, eta, dzeta);
                oc3_deriv_green_cube(d, 1.0, eta, dzeta);
                if (g) g[idx] = gv;
                if (dgdx) dgdx[idx] = d[0];
                if (dgdy) dgdy[idx] = d[1];
                if (dgdz) dgdz[idx] = d[2];
                double cum = prev_int + prev_g * delta * delta;
                if (intg) intg[idx] = cum;
                prev_int = cum;
                prev_g = gv;
            }
    if (intg) {
        size_t last = 6 * N * N;
        intg[last] = prev_int + prev_g * delta * delta;
        double alpha = 1.0 / intg[last];
        for (size_t i = 0; i <= last; i++) intg[i] *= alpha;
    }
}

void oc3_weight_table(int n, const double *intg, const double *dgdx, const double *dgdy,
                      const double *dgdz, double *w) {
    size_t B = 6 * (size_t)n * (size_t)n;
    double area = 1.0 / ((double)n * (double)n);
    for (size_t b = 0; b < B; b++) {
        double pi_b = intg[b + 1] - intg[b];
        double f = pi_b > 0 ? area / pi_b : 0.0;
        w[3 * b] = dgdx[b] * f;
        w[3 * b + 1] = dgdy[b] * f;
        w[3 * b + 2] = dgdz[b] * f;
    }
}

/* ------------------------------------------------------------------------ */
/* Layout geometry                                                          */
/* ------------------------------------------------------------------------ */
void oc3_layout_bounds(const double *b, int64_t n, double out[6]) {
    double lo[3] = {b[0], b[1], b[2]}, hi[3] = {b[3], b[4], b[5]};
    for (int64_t i = 1; i < n; i++)
        for (int c = 0; c < 3; c++) {
            if (b[6 * i + c] < lo[c]) lo[c] = b[6 * i + c];
            if (b[6 * i + 3 + c] > hi[c]) hi[c] = b[6 * i + 3 + c];
        }
    int add = (int)((hi[0] - lo[0]) * OC_BOUNDS_MUL);
    for (int c = 0; c < 3; c++) {
        out[c] = lo[c] - add;
        out[3 + c] = hi[c] + add;
    }
}

double oc3_default_shell(const double *b, int64_t n) {
    double e = INFINITY;
    for (int64_t i = 0; i < n; i++)
        for (int c = 0; c < 3; c++) {
            double w = b[6 * i + 3 + c] - b[6 * i + c];
            if (w < e) e = w;
        }
    return 1e-3 * e;
}

/* L-infinity distance from p to box b: the largest per-axis gap (0 inside). */
static inline double box_dist(const double *b, const double *p) {
    double d = 0.0;
    for (int c = 0; c < 3; c++) {
        double lo = b[c] - p[c], hi = p[c] - b[3 + c];
        if (lo > d) d = lo;
        if (hi > d) d = hi;
    }
    return d;
}

void oc3_nearest(const double *boxes, int64_t n, const double p[3], double *d, int64_t *id) {
    double best = INFINITY;
    int64_t bi = -1;
    for (int64_t i = 0; i < n; i++) {
        double v = box_dist(boxes + 6 * i, p);
        if (v < best) {
            best = v;
            bi = i;
        }
    }
    *d = best;
    *id = bi;
}

/* Cell grid: cubic cells over the bounds, each binning the boxes that
 * overlap it.  A ring search over the bins (rings of cells around the
 * query's cell until a ring's inner distance exceeds the best distance)
 * answers any point exactly.  For speed each cell also keeps a candidate
 * list: every box within D_c + 2h + margin of its centre (D_c = the centre's
 * nearest-box distance, h = half a cell side), sorted by that distance; the
 * nearest box of any point of the cell is on it, and a scan can stop at the
 * first entry whose centre distance minus (h + margin) exceeds the best. */
struct oc3_grid {
    const double *boxes;
    int64_t n;
    double o[3], side, inv, h, margin;
    int64_t nc[3];
    int64_t *start, *items;
    int64_t *lstart, *lbox; /* candidate lists: cell c holds lbox[lstart[c] .. lstart[c+1]) */
    double *lkey;           /* each entry's distance from its cell centre */
};

static int build_lists(oc3_grid *g);

static int64_t cell_clamp(double v, double o, double inv, int64_t nc) {
    double t = floor((v - o) * inv);
    if (t < 0) return 0;
    if (t >= (double)nc) return nc - 1;
    return (int64_t)t;
}

oc3_grid *oc3_grid_create(const double *boxes, int64_t n, const double bounds[6], double boxes_per_cell,
                          int with_lists) {
    oc3_grid *g = (oc3_grid *)calloc(1, sizeof(oc3_grid));
    if (!g) return NULL;
    g->boxes = boxes;
    g->n = n;
    double ext[3], vol = 1.0;
    for (int c = 0; c < 3; c++) {
        g->o[c] = bounds[c];
        ext[c] = bounds[3 + c] - bounds[c];
        vol *= ext[c];
    }
    double cells = (double)n / (boxes_per_cell > 0 ? boxes_per_cell : 1.0);
    if (cells < 1) cells = 1;
    g->side = cbrt(vol / cells);
    int64_t total = 1;
    for (int c = 0; c < 3; c++) {
        g->nc[c] = (int64_t)ceil(ext[c] / g->side);
        if (g->nc[c] < 1) g->nc[c] = 1;
        if (g->nc[c] > 4096) g->nc[c] = 4096;
        total *= g->nc[c];
    }
    /* cells at least as large as the bounds need per axis */
    double s = g->side;
    for (int c = 0; c < 3; c++)
        if (ext[c] / (double)g->nc[c] > s) s = ext[c] / (double)g->nc[c];
    g->side = s;
    g->inv = 1.0 / s;
    g->start = (int64_t *)calloc((size_t)total + 1, sizeof(int64_t));
    if (!g->start) { free(g); return NULL; }
    int64_t lo[3], hi[3];
    for (int pass = 0; pass < 2; pass++) {
        for (int64_t i = 0; i < n; i++) {
            const double *b = boxes + 6 * i;
            for (int c = 0; c < 3; c++) {
                lo[c] = cell_clamp(b[c], g->o[c], g->inv, g->nc[c]);
                hi[c] = cell_clamp(b[3 + c], g->o[c], g->inv, g->nc[c]);
            }
            for (int64_t z = lo[2]; z <= hi[2]; z++)
                for (int64_t y = lo[1]; y <= hi[1]; y++)
                    for (int64_t x = lo[0]; x <= hi[0]; x++) {
                        int64_t cid = (z * g->nc[1] + y) * g->nc[0] + x;
                        if (pass == 0) g->start[cid + 1]++;
                        else g->items[g->start[cid]++] = i;
                    }
        }
        if (pass == 0) {
            for (int64_t c = 0; c < total; c++) g->start[c + 1] += g->start[c];
            g->items = (int64_t *)malloc(sizeof(int64_t) * (size_t)(g->start[total] ? g->start[total] : 1));
            if (!g->items) { free(g->start); free(g); return NULL; }
        } else {
            for (int64_t c = total; c > 0; c--) g->start[c] = g->start[c - 1];
            g->start[0] = 0;
        }
    }
    double M = 16.0;
    for (int c = 0; c < 3; c++) {
        double a = fabs(bounds[c]) > fabs(bounds[3 + c]) ? fabs(bounds[c]) : fabs(bounds[3 + c]);
        if (4.0 * a > M) M = 4.0 * a;
        if (4.0 * ext[c] > M) M = 4.0 * ext[c];
    }
    g->h = 0.5 * g->side;
    g->margin = ldexp(M, -30); /* far above the rounding of a cell index or a distance */
    if (with_lists && !build_lists(g)) { /* without lists every query takes the ring search */
        free(g->lstart);
        free(g->lbox);
        free(g->lkey);
        g->lstart = g->lbox = NULL;
        g->lkey = NULL;
    }
    return g;
}

void oc3_grid_destroy(oc3_grid *g) {
    if (!g) return;
    free(g->start);
    free(g->items);
    free(g->lstart);
    free(g->lbox);
    free(g->lkey);
    free(g);
}

static void ring_nearest(const oc3_grid *g, const double p[3], double *d, int64_t *id) {
    int64_t c0[3];
    for (int c = 0; c < 3; c++) c0[c] = cell_clamp(p[c], g->o[c], g->inv, g->nc[c]);
    double best = INFINITY;
    int64_t bi = -1;
    int64_t rmax = g->nc[0];
    if (g->nc[1] > rmax) rmax = g->nc[1];
    if (g->nc[2] > rmax) rmax = g->nc[2];
    double slack = 1e-9 * g->side;
    for (int64_t r = 0; r <= rmax; r++) {
        if (r > 0) {
            /* every box not seen yet lies in cells of ring >= r: at least the
             * distance from p to the outside of the ring-(r-1) cube away. */
            double lim = INFINITY;
            int open = 0;
            for (int c = 0; c < 3; c++) {
                int64_t a = c0[c] - (r - 1), b = c0[c] + r;
                if (a > 0) { double v = p[c] - (g->o[c] + (double)a * g->side); if (v < lim) lim = v; open = 1; }
                if (b < g->nc[c]) { double v = (g->o[c] + (double)b * g->side) - p[c]; if (v < lim) lim = v; open = 1; }
            }
            if (!open) break;                /* the whole grid has been scanned */
            if (best < lim - slack) break;   /* strict: an equal distance may still win on index */
        }
        for (int64_t z = c0[2] - r; z <= c0[2] + r; z++) {
            if (z < 0 || z >= g->nc[2]) continue;
            for (int64_t y = c0[1] - r; y <= c0[1] + r; y++) {
                if (y < 0 || y >= g->nc[1]) continue;
                int64_t ring_yz = llabs(z - c0[2]) > llabs(y - c0[1]) ? llabs(z - c0[2]) : llabs(y - c0[1]);
                for (int64_t x = c0[0] - r; x <= c0[0] + r; x++) {
                    if (x < 0 || x >= g->nc[0]) continue;
                    int64_t ring = llabs(x - c0[0]) > ring_yz ? llabs(x - c0[0]) : ring_yz;
                    if (ring != r) continue;
                    int64_t cid = (z * g->nc[1] + y) * g->nc[0] + x;
                    for (int64_t k = g->start[cid]; k < g->start[cid + 1]; k++) {
                        int64_t i = g->items[k];
                        double v = box_dist(g->boxes + 6 * i, p);
                        if (v < best || (v == best && i < bi)) {
                            best = v;
                            bi = i;
                        }
                    }
                }
            }
        }
    }
    *d = best;
    *id = bi;
}

typedef struct { double key; int64_t box; } cand3;
static int cand3_cmp(const void *a, const void *b) {
    const cand3 *x = (const cand3 *)a, *y = (const cand3 *)b;
    if (x->key != y->key) return x->key < y->key ? -1 : 1;
    return x->box < y->box ? -1 : (x->box > y->box);
}

/* The per-cell candidate lists (count, then fill), deduplicated with a
 * per-box stamp of the last cell that took the box. */
static int build_lists(oc3_grid *g) {
    int64_t total = g->nc[0] * g->nc[1] * g->nc[2];
    int64_t *stamp = (int64_t *)malloc(sizeof(int64_t) * (size_t)(g->n ? g->n : 1));
    cand3 *buf = (cand3 *)malloc(sizeof(cand3) * (size_t)(g->n ? g->n : 1));
    g->lstart = (int64_t *)calloc((size_t)total + 1, sizeof(int64_t));
    if (!stamp || !buf || !g->lstart) { free(stamp); free(buf); return 0; }
    for (int pass = 0; pass < 2; pass++) {
        for (int64_t i = 0; i < g->n; i++) stamp[i] = -1;
        for (int64_t cid = 0; cid < total; cid++) {
            int64_t cc[3] = {cid % g->nc[0], (cid / g->nc[0]) % g->nc[1], cid / (g->nc[0] * g->nc[1])};
            double pc[3], D;
            int64_t nid;
            for (int c = 0; c < 3; c++) pc[c] = g->o[c] + ((double)cc[c] + 0.5) * g->side;
            ring_nearest(g, pc, &D, &nid);
            double R = D + 2.0 * g->h + g->margin;
            int64_t rr = (int64_t)ceil(R / g->side) + 1, m = 0;
            int64_t lo[3], hi[3];
            for (int c = 0; c < 3; c++) {
                lo[c] = cc[c] - rr < 0 ? 0 : cc[c] - rr;
                hi[c] = cc[c] + rr >= g->nc[c] ? g->nc[c] - 1 : cc[c] + rr;
            }
            for (int64_t z = lo[2]; z <= hi[2]; z++)
                for (int64_t y = lo[1]; y <= hi[1]; y++)
                    for (int64_t x = lo[0]; x <= hi[0]; x++) {
                        int64_t q = (z * g->nc[1] + y) * g->nc[0] + x;
                        for (int64_t k = g->start[q]; k < g->start[q + 1]; k++) {
                            int64_t i = g->items[k];
                            if (stamp[i] == cid) continue;
                            stamp[i] = cid;
                            double v = box_dist(g->boxes + 6 * i, pc);
                            if (v > R) continue;
                            buf[m].key = v;
                            buf[m].box = i;
                            m++;
                        }
                    }
            if (pass == 0) {
                g->lstart[cid + 1] = m;
            } else {
                qsort(buf, (size_t)m, sizeof(cand3), cand3_cmp);
                for (int64_t k = 0; k < m; k++) {
                    g->lbox[g->lstart[cid] + k] = buf[k].box;
                    g->lkey[g->lstart[cid] + k] = buf[k].key;
                }
            }
        }
        if (pass == 0) {
            for (int64_t c = 0; c < total; c++) g->lstart[c + 1] += g->lstart[c];
            size_t ne = (size_t)(g->lstart[total] ? g->lstart[total] : 1);
            g->lbox = (int64_t *)malloc(sizeof(int64_t) * ne);
            g->lkey = (double *)malloc(sizeof(double) * ne);
            if (!g->lbox || !g->lkey) { free(stamp); free(buf); return 0; }
        }
    }
    free(stamp);
    free(buf);
    return 1;
}

void oc3_grid_nearest(const oc3_grid *g, const double p[3], double *d, int64_t *id) {
    int64_t c0[3];
    for (int c = 0; c < 3; c++) {
        double t = floor((p[c] - g->o[c]) * g->inv);
        if (!(t >= 0.0) || t >= (double)g->nc[c] || !g->lstart) { /* outside the grid: the ring search */
            ring_nearest(g, p, d, id);
            return;
        }
        c0[c] = (int64_t)t;
    }
    int64_t cid = (c0[2] * g->nc[1] + c0[1]) * g->nc[0] + c0[0];
    double best = INFINITY, lim = g->h + g->margin;
    int64_t bi = -1;
    for (int64_t k = g->lstart[cid]; k < g->lstart[cid + 1]; k++) {
        if (g->lkey[k] - lim > best) break; /* it and every later entry are farther */
        int64_t i = g->lbox[k];
        double v = box_dist(g->boxes + 6 * i, p);
        if (v < best || (v == best && i < bi)) {
            best = v;
            bi = i;
        }
    }
    *d = best;
    *id = bi;
}

void oc3_query_batch(const double *boxes, int64_t n, const oc3_grid *grid, const double *pts, int64_t m,
                     double *d, int64_t *id) {
    for (int64_t i = 0; i < m; i++) {
        if (grid) oc3_grid_nearest(grid, pts + 3 * i, d + i, id + i);
        else oc3_nearest(boxes, n, pts + 3 * i, d + i, id + i);
    }
}

/* ------------------------------------------------------------------------ */
/* Walk                                                                     */
/* ------------------------------------------------------------------------ */
/* Uniform number t of walk w: word t % 4 of the Philox4x32-10 block
 * (t / 4, walk, stream) under key seed.  t = 0, 1 place the start point;
 * landing L (1-based) uses t = L + 1. */
static uint32_t draw32(uint64_t seed, uint32_t stream, uint64_t walk, uint32_t t) {
    uint32_t ctr[4] = {t >> 2, (uint32_t)walk, (uint32_t)(walk >> 32), stream};
    uint32_t key[2] = {(uint32_t)seed, (uint32_t)(seed >> 32)};
    uint32_t o[4];
    oc_philox4x32_10(ctr, key, o);
    return o[t & 3];
}

/* Last bin b with intg[b] <= u. */
static int bin3(const double *intg, int nb, double u) {
    int lo = 0, hi = nb; /* intg[lo] <= u < intg[hi] (intg[nb] = 1 > u) */
    while (hi - lo > 1) {
        int mid = (lo + hi) >> 1;
        if (intg[mid] <= u) lo = mid;
        else hi = mid;
    }
    return lo;
}

/* Start point on the Gaussian box G: faces z0, z1, y0, y1, x0, x1 chosen in
 * proportion to area by u0 (the remainder places the first coordinate), u1
 * places the second; n0 = outward axis (0 x, 1 y, 2 z) and its sign. */
static void gauss_point(const double G[6], double S, double u0, double u1, double p[3], int *axis,
                        double *sgn) {
    double w = G[3] - G[0], h = G[4] - G[1], d = G[5] - G[2];
    double area[3] = {w * h, w * d, h * d};
    double s = u0 * S;
    int f = 0;
    for (; f < 5; f++) {
        double a = area[f >> 1];
        if (s < a) break;
        s = s - a;
    }
    double t = s / area[f >> 1];
    if (t > 1.0) t = 1.0;
    int hi = f & 1;
    switch (f >> 1) {
    case 0: /* z faces: x from t, y from u1 */
        p[0] = G[0] + t * w; p[1] = G[1] + u1 * h; p[2] = hi ? G[5] : G[2]; *axis = 2; break;
    case 1: /* y faces: x from t, z from u1 */
        p[0] = G[0] + t * w; p[1] = hi ? G[4] : G[1]; p[2] = G[2] + u1 * d; *axis = 1; break;
    default: /* x faces: y from t, z from u1 */
        p[0] = hi ? G[3] : G[0]; p[1] = G[1] + t * h; p[2] = G[2] + u1 * d; *axis = 0; break;
    }
    *sgn = hi ? 1.0 : -1.0;
}

/* Landing on the cube of half-side h centred on p at the centre of bin b:
 * face k, row i, column j; o_i = (2 i + 1 - n) / n is the offset of the
 * row's centre from the face centre in half-sides. */
static void land(int n, int b, double h, double p[3]) {
    int nn = n * n, k = b / nn, i = (b % nn) / n, j = b % n;
    double oi = (double)(2 * i + 1 - n) / (double)n, oj = (double)(2 * j + 1 - n) / (double)n;
    double x = p[0], y = p[1], z = p[2];
    switch (k) {
    case 0: p[0] = x + h * oi; p[1] = y + h * oj; p[2] = z - h; break;
    case 1: p[0] = x + h; p[1] = y + h * oi; p[2] = z + h * oj; break;
    case 2: p[0] = x - h * oj; p[1] = y + h; p[2] = z + h * oi; break;
    case 3: p[0] = x - h * oi; p[1] = y - h * oj; p[2] = z + h; break;
    case 4: p[0] = x - h; p[1] = y - h * oi; p[2] = z - h * oj; break;
    default: p[0] = x + h * oj; p[1] = y - h; p[2] = z - h * oi; break;
    }
}

int oc3_walk_run(const double *boxes, int64_t n, const double bounds[6], const oc3_grid *grid,
                 const oc3_cfg *cfg, uint64_t first, uint64_t count, int64_t *end_out,
                 int32_t *hops_out, int32_t *bin_out, double *weight_out) {
    if (cfg->target < 0 || cfg->target >= n || cfg->nsample < 1) return OC_E_ARG;
    int N = cfg->nsample, nb = 6 * N * N;
    /* the table of the last resolution used is kept (a 50 x 50 table takes
     * about a third of a second to evaluate); the oracle is single-threaded */
    static int cached_n = 0;
    static double *g = NULL, *intg = NULL, *w = NULL;
    if (cached_n != N) {
        free(g);
        free(intg);
        free(w);
        cached_n = 0;
        g = (double *)malloc(sizeof(double) * (size_t)nb * 4);
        intg = (double *)malloc(sizeof(double) * (size_t)(nb + 1));
        w = (double *)malloc(sizeof(double) * (size_t)nb * 3);
        if (!g || !intg || !w) {
            free(g); free(intg); free(w);
            g = intg = w = NULL;
            return OC_E_OOM;
        }
        oc3_cube_green_table(N, g, g + nb, g + 2 * nb, g + 3 * nb, intg);
        oc3_weight_table(N, intg, g + nb, g + 2 * nb, g + 3 * nb, w);
        cached_n = N;
    }
    const double *T = boxes + 6 * cfg->target;
    double G[6];
    for (int c = 0; c < 3; c++) {
        G[c] = T[c] - cfg->offset;
        G[3 + c] = T[3 + c] + cfg->offset;
    }
    double gw = G[3] - G[0], gh = G[4] - G[1], gd = G[5] - G[2];
    double S = 2.0 * (gw * gh) + 2.0 * (gw * gd) + 2.0 * (gh * gd);
    for (uint64_t k = 0; k < count; k++) {
        uint64_t wk = first + k;
        double u0 = draw32(cfg->seed, cfg->stream, wk, 0) * (1.0 / 4294967296.0);
        if (cfg->start_strata)
            u0 = ((double)(uint32_t)(wk % cfg->start_strata) + u0) / (double)cfg->start_strata;
        double u1 = draw32(cfg->seed, cfg->stream, wk, 1) * (1.0 / 4294967296.0);
        double p[3], sgn;
        int axis;
        gauss_point(G, S, u0, u1, p, &axis, &sgn);
        int64_t end;
        int32_t hops = 0, b1 = -1;
        double a0 = 0.0;
        for (;;) {
            if (!(p[0] > bounds[0] && p[1] > bounds[1] && p[2] > bounds[2] && p[0] < bounds[3] &&
                  p[1] < bounds[4] && p[2] < bounds[5])) {
                end = OC3_END_ESCAPED;
                break;
            }
            double d;
            int64_t id;
            if (grid) oc3_grid_nearest(grid, p, &d, &id);
            else oc3_nearest(boxes, n, p, &d, &id);
            hops++;
            if (d <= cfg->shell) { end = id; break; }
            if (hops >= cfg->hop_cap) { end = OC3_END_ABORTED; break; }
            uint32_t x = draw32(cfg->seed, cfg->stream, wk, (uint32_t)hops + 1);
            int b = bin3(intg, nb, x * (1.0 / 4294967296.0));
            land(N, b, d, p);
            if (hops == 1) { b1 = b; a0 = 2.0 * d; }
        }
        double c = 0.0;
        if (b1 >= 0) c = cfg->permittivity * S * (sgn * w[3 * b1 + axis]) / a0;
        end_out[k] = end;
        hops_out[k] = hops;
        bin_out[k] = b1;
        weight_out[k] = c;
    }
    return OC_OK;
}
