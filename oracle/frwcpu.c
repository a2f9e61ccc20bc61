/*
 * frwcpu.c -- CPU oracle for the FRW hot path.  TEST INFRASTRUCTURE ONLY:
 * the checker that tests/, the smoke check and bench.py's cpu_baseline leg
 * compare the CUDA product against.  Never linked into the product.
 *
 * Built with -ffp-contract=off so every FP64 expression rounds exactly as
 * written; the reference's expressions are evaluated in the reference's
 * operand order wherever the result feeds a comparison (bit-exact parity).
 * Each function cites the reference lines it restates.
 */
#include "frwcpu.h"

#include <math.h>
#include <stdio.h>
#include <stdlib.h>
#include <string.h>

void oc_free(void *p) { free(p); }

/* ------------------------------------------------------------------------ */
/* Layout reader: CPU/Parser.cpp:15-50 (parse), :89-125 (loadRectFromLine)  */
/* ------------------------------------------------------------------------ */

/* The reference reads with std::istream::getline(line, 50): a line of 50 or
 * more characters (before the newline) sets failbit and ends the read loop.
 * A layer is closed by every line containing "<<" except the first one; rects
 * after the last delimiter are never stored.  A line containing "rect" is
 * parsed as a header token followed by 4 numbers (lines with another count
 * are undefined behaviour in the reference and rejected here). */
#define OC_MAX_LINE 50

typedef struct {
    double *v;
    int64_t n, cap;
} dvec;

static int dvec_push4(dvec *d, const double r[4]) {
    if (d->n + 1 > d->cap) {
        int64_t nc = d->cap ? d->cap * 2 : 1024;
        double *nv = (double *)realloc(d->v, (size_t)nc * 4 * sizeof(double));
        if (!nv) return OC_E_OOM;
        d->v = nv;
        d->cap = nc;
    }
    memcpy(d->v + 4 * d->n, r, 4 * sizeof(double));
    d->n++;
    return OC_OK;
}

static int parse_rect_line(const char *line, double r[4]) {
    const char *s = line;
    while (*s == ' ' || *s == '\t' || *s == '\r') s++;
    while (*s && *s != ' ' && *s != '\t' && *s != '\r') s++; /* header token */
    int k = 0;
    for (;;) {
        while (*s == ' ' || *s == '\t' || *s == '\r') s++;
        if (!*s) break;
        char *end = NULL;
        double v = strtod(s, &end);
        if (end == s) break; /* istream >> double fails here */
        if (k == 4) return OC_E_IO;
        r[k++] = v;
        s = end;
    }
    return k == 4 ? OC_OK : OC_E_IO;
}

int oc_parse_layout(const char *path, int layer, double **rects_out, int64_t *n_out,
                    int *nlayers_out) {
    *rects_out = NULL;
    *n_out = 0;
    if (nlayers_out) *nlayers_out = 0;
    FILE *f = fopen(path, "rb");
    if (!f) return OC_E_IO;
    dvec cur = {0}, keep = {0};
    int nlayers = 0, first = 1, st = OC_OK;
    char line[OC_MAX_LINE + 2];
    int len = 0, c, eof = 0;
    while (!eof) {
        /* getline(line, 50) */
        len = 0;
        int got_any = 0, fail = 0;
        for (;;) {
            c = fgetc(f);
            if (c == EOF) { eof = 1; break; }
            got_any = 1;
            if (c == '\n') break;
            if (len == OC_MAX_LINE - 1) { fail = 1; break; }
            line[len++] = (char)c;
        }
        line[len] = 0;
        if (fail || (!got_any && eof)) break;
        if (strstr(line, "<<")) {
            if (first) { first = 0; continue; }
            if (nlayers == layer) {
                keep = cur;
                cur.v = NULL; cur.n = cur.cap = 0;
            }
            cur.n = 0;
            nlayers++;
            continue;
        }
        if (strstr(line, "rect")) {
            double r[4];
            st = parse_rect_line(line, r);
            if (st != OC_OK) break;
            st = dvec_push4(&cur, r);
            if (st != OC_OK) break;
        }
    }
    fclose(f);
    free(cur.v);
    if (nlayers_out) *nlayers_out = nlayers;
    if (st != OC_OK) { free(keep.v); return st; }
    if (layer < 0 || layer >= nlayers) { free(keep.v); return OC_E_ARG; }
    *rects_out = keep.v;
    *n_out = keep.n;
    return OC_OK;
}

/* Parser::getLayerSize, CPU/Parser.cpp:51-87: bounding box grown by
 * int(0.01 * width) on BOTH axes (add_space_h is computed but unused). */
void oc_layer_bounds(const double *r, int64_t n, double out[4]) {
    double lx = r[0], ty = r[1], rx = r[2], by = r[3];
    for (int64_t i = 1; i < n; i++) {
        const double *q = r + 4 * i;
        if (q[0] < lx) lx = q[0];
        if (q[1] < ty) ty = q[1];
        if (q[2] > rx) rx = q[2];
        if (q[3] > by) by = q[3];
    }
    int add_w = (int)((rx - lx) * OC_BOUNDS_MUL);
    out[0] = lx - add_w;
    out[1] = ty - add_w;
    out[2] = rx + add_w;
    out[3] = by + add_w;
}

/* ------------------------------------------------------------------------ */
/* Green's function of the unit square seen from its centre                 */
/* ------------------------------------------------------------------------ */
/*
 * Laplace's equation on [0,1]^2 with data f on the side y=0 and zero on the
 * other three sides is solved by
 *     u(x,y) = sum_n b_n sin(n pi x) sinh(n pi (1-y)) / sinh(n pi),
 *     b_n    = 2 int f(xi) sin(n pi xi) dxi,
 * so the Poisson kernel from the centre to the boundary point xi is
 *     K(xi) = 2 sum_{n odd} (-1)^((n-1)/2) c_n sin(n pi xi),
 *     c_n   = sinh(n pi/2)/sinh(n pi) = q (1 - q^2) / (1 - e^{-2 pi n}),
 *             q = e^{-n pi / 2}.
 * The perimeter parameter eta in [0,4) runs over the four sides; on side k,
 * sin(n pi eta) = (-1)^k sin(n pi (eta-k)) for odd n, hence the alternating
 * side sign.  Truncation at n <= 19 (ten odd terms) and the sample points
 * eta_i = (i+1/2)*4/N are those of green/green.cpp:27-54,125-152; the
 * table must match the reference to the last bit because the walk compares
 * uniforms against it, so the terms are accumulated in the same order.
 */
static double unit_square_kernel(double eta) {
    const double pi = 3.14159265358979323846;
    double phase = pi * eta / 1.0;
    double acc = 0.0, sgn = 1.0;
    for (uint64_t n = 1; n <= 20; n += 2) {
        double q = exp(-0.5 * n * pi);
        double den = 1.0 - exp(-2.0 * pi * n);
        acc += sgn * (q * (1.0 - q * q) / den) * sin(n * phase);
        sgn *= -1;
    }
    int side = (eta <= 1.0) ? 0 : (eta <= 2.0) ? 1 : (eta <= 3.0) ? 2 : 3;
    return acc * ((side & 1) ? -2.0 / 1.0 : 2.0 / 1.0);
}

void oc_green_table(int nsample, double *g, double *intg) {
    double d_eta = 4.0 / nsample;
    for (uint64_t i = 0; i < (uint64_t)nsample; i++) g[i] = unit_square_kernel((i + 0.5) * d_eta);
    intg[0] = 0.0;
    for (uint64_t i = 1; i <= (uint64_t)nsample; i++) intg[i] = intg[i - 1] + g[i - 1] * d_eta;
    double alpha = 1.0 / intg[nsample];
    for (int i = 0; i <= nsample; i++) intg[i] *= alpha;
}

/*
 * Gradient of K with respect to the source point, at the centre:
 *   normal part (towards the side)  N(xi) = 2 pi sum_{n odd}  (-1)^((n-1)/2) n ch_n sin(n pi xi),
 *   tangential part (along the side) T(xi) = 2 pi sum_{n even} (-1)^(n/2)     n c_n  sin(n pi xi),
 *   ch_n = cosh(n pi/2)/sinh(n pi),  c_n = sinh(n pi/2)/sinh(n pi).
 * Sides in screen axes (y down), clockwise from the top-left corner:
 *   top: along (1,0), outward (0,-1); right: (0,1),(1,0);
 *   bottom: (-1,0),(0,1); left: (0,-1),(-1,0).
 */
static void unit_square_grad(double xi, double *nrm, double *tan) {
    const double pi = 3.14159265358979323846;
    double sn = 0.0, st = 0.0;
    for (int n = 1; n <= 80; n++) {
        double q = exp(-0.5 * n * pi);
        double den = 1.0 - exp(-2.0 * pi * n);
        double s = sin(n * pi * xi);
        if (n & 1) {
            double sg = ((n >> 1) & 1) ? -1.0 : 1.0;
            sn += sg * n * (q * (1.0 + q * q) / den) * s;
        } else {
            double sg = ((n >> 1) & 1) ? -1.0 : 1.0;
            st += sg * n * (q * (1.0 - q * q) / den) * s;
        }
    }
    *nrm = 2.0 * pi * sn;
    *tan = 2.0 * pi * st;
}

void oc_weight_table(int nsample, const double *intg, double *wx, double *wy) {
    static const double along[4][2] = {{1, 0}, {0, 1}, {-1, 0}, {0, -1}};
    static const double outw[4][2] = {{0, -1}, {1, 0}, {0, 1}, {-1, 0}};
    int nside = nsample / 4;
    for (int i = 0; i < nsample; i++) {
        int s = i / nside, j = i % nside;
        if (j == 0) { wx[i] = wy[i] = 0.0; continue; } /* corner landing */
        double xi = ((j - 1) + 0.5) / nside;
        double nr, tg;
        unit_square_grad(xi, &nr, &tg);
        double pi_i = intg[i + 1] - intg[i];
        double f = (1.0 / nside) / pi_i;
        wx[i] = (tg * along[s][0] + nr * outw[s][0]) * f;
        wy[i] = (tg * along[s][1] + nr * outw[s][1]) * f;
    }
}

/* getIndex, CPU/mainFunctions.cpp:40-46: the first i with
 * intg[i] <= r < intg[i+1]; r >= intg[N] (undefined in the reference) is
 * clamped to the last bin. */
int oc_bin_index(const double *intg, int nsample, double r) {
    for (int i = 0; i < nsample; i++)
        if (intg[i] <= r && intg[i + 1] > r) return i;
    return nsample - 1;
}

/* ------------------------------------------------------------------------ */
/* Philox4x32-10                                                            */
/* ------------------------------------------------------------------------ */
void oc_philox4x32_10(const uint32_t ctr[4], const uint32_t key[2], uint32_t out[4]) {
    uint32_t c0 = ctr[0], c1 = ctr[1], c2 = ctr[2], c3 = ctr[3];
    uint32_t k0 = key[0], k1 = key[1];
    for (int r = 0; r < 10; r++) {
        if (r) { k0 += 0x9E3779B9u; k1 += 0xBB67AE85u; }
        uint64_t p0 = (uint64_t)0xD2511F53u * c0;
        uint64_t p1 = (uint64_t)0xCD9E8D57u * c2;
        uint32_t n0 = (uint32_t)(p1 >> 32) ^ c1 ^ k0;
        uint32_t n1 = (uint32_t)p1;
        uint32_t n2 = (uint32_t)(p0 >> 32) ^ c3 ^ k1;
        uint32_t n3 = (uint32_t)p0;
        c0 = n0; c1 = n1; c2 = n2; c3 = n3;
    }
    out[0] = c0; out[1] = c1; out[2] = c2; out[3] = c3;
}

double oc_u01(uint32_t a, uint32_t b) {
    uint64_t m = ((uint64_t)(a >> 5) << 26) | (uint64_t)(b >> 6);
    return (double)m * (1.0 / 9007199254740992.0);
}

/* ------------------------------------------------------------------------ */
/* Geometry: CPU/rectHost.cpp                                               */
/* ------------------------------------------------------------------------ */
/* RectHost::rectsCollision (rectHost.cpp:43-52), closed intervals;
 * a = the stored object, b = the query box. */
static inline int collide(const double *a, const double *b) {
    return a[2] >= b[0] && b[2] >= a[0] && a[3] >= b[1] && b[3] >= a[1];
}
/* RectHost::rectContains(point), closed (rectHost.cpp:54-63). */
static inline int contains_pt(const double *a, double x, double y) {
    return x >= a[0] && y >= a[1] && x <= a[2] && y <= a[3];
}
/* Tree::isInBounds(rect), inclusive (quadTree.cpp:38-47). */
static inline int box_in(const double *b, const double *r) {
    return r[1] >= b[1] && r[0] >= b[0] && r[3] <= b[3] && r[2] <= b[2];
}
/* Tree::isInBounds(point), strict (quadTree.cpp:49-59). */
static inline int pt_in(const double *b, double x, double y) {
    return x > b[0] && y > b[1] && x < b[2] && y < b[3];
}
static inline int same_rect(const double *a, const double *b) {
    return a[0] == b[0] && a[1] == b[1] && a[2] == b[2] && a[3] == b[3];
}

/* RectHost::getPointFromNindex, rectHost.cpp:107-161.  Branch structure and
 * operand order are those of the reference (they decide which comparisons
 * tie); perimeter is truncated to int unless exact_perimeter. */
void oc_point_from_index(const double sq[4], int index, int nsample, int exact_perimeter,
                         double out[2]) {
    double per2 = 2 * (sq[2] - sq[0]) + 2 * (sq[3] - sq[1]);
    double perimeter = exact_perimeter ? per2 : (double)(int)per2;
    double v = perimeter / (double)nsample;
    double h = sq[3] - sq[1];
    double w = sq[2] - sq[0];
    double iv = index * v, jv = (index - 1) * v;
    if (iv < w) {
        out[0] = (double)(int)(jv + v / 2 + sq[0]);
        out[1] = sq[1];
    } else if (jv < w && iv > w) {
        out[0] = sq[2];
        out[1] = sq[1];
    } else if (iv < (w + h)) {
        out[0] = sq[2];
        if (jv > w) out[1] = sq[1] + jv - w + v / 2;
        else out[1] = sq[1] + iv - w + (iv - w) / 2;
    } else if (jv < (w + h) && iv > (w + h)) {
        out[0] = sq[2];
        out[1] = sq[3];
    } else if (iv < (2 * w + h)) {
        out[1] = sq[3];
        if (jv > w + h) out[0] = sq[2] - (jv - w - h + v / 2);
        else out[0] = sq[2] - (iv - w - h + (iv - w - h) / 2);
    } else if (jv < (2 * w + h) && iv > (2 * w + h)) {
        out[0] = sq[0];
        out[1] = sq[3];
    } else {
        out[0] = sq[0];
        if (jv > 2 * w + h) out[1] = sq[3] - (jv - 2 * w - h + v / 2);
        else out[1] = sq[3] - (iv - 2 * w - h + (iv - 2 * w - h) / 2);
    }
}

/* RectHost::createGaussianSurface, rectHost.cpp:84-100. */
void oc_scale_rect(const double r[4], double fx, double fy, double out[4]) {
    double mx = (r[0] + r[2]) / 2.;
    double my = (r[1] + r[3]) / 2.;
    double vx = r[0] - mx;
    double vy = r[1] - my;
    vx *= fx;
    vy *= fy;
    out[0] = mx + vx;
    out[1] = my + vy;
    out[2] = mx - vx;
    out[3] = my - vy;
}

/* ------------------------------------------------------------------------ */
/* Complete index: uniform bucket grid, exact closed-interval predicates     */
/* ------------------------------------------------------------------------ */
struct oc_grid {
    double b[4];
    const double *r;
    int64_t n;
    int nx, ny;
    double cs;
    int64_t *start;
    int64_t *items;
};

static inline int cell_of(double v, double lo, double cs, int nc) {
    double f = floor((v - lo) / cs);
    if (!(f >= 0)) return 0; /* also NaN */
    if (f >= nc - 1) return nc - 1;
    return (int)f;
}

oc_grid *oc_grid_create(const double *rects, int64_t n, const double bounds[4]) {
    oc_grid *g = (oc_grid *)calloc(1, sizeof(oc_grid));
    if (!g) return NULL;
    memcpy(g->b, bounds, sizeof(g->b));
    g->r = rects;
    g->n = n;
    double W = bounds[2] - bounds[0], H = bounds[3] - bounds[1];
    double ext = W > H ? W : H;
    if (!(ext > 0)) ext = 1;
    double cs = n > 0 ? sqrt(W * H / (double)n) : ext;
    if (!(cs > 0)) cs = ext;
    if (ext / cs > 4096) cs = ext / 4096;
    g->cs = cs;
    g->nx = (int)(W / cs) + 1;
    g->ny = (int)(H / cs) + 1;
    int64_t nc = (int64_t)g->nx * g->ny;
    int64_t *cnt = (int64_t *)calloc((size_t)nc + 1, sizeof(int64_t));
    if (!cnt) { free(g); return NULL; }
    for (int pass = 0; pass < 2; pass++) {
        for (int64_t i = 0; i < n; i++) {
            const double *q = rects + 4 * i;
            int a0 = cell_of(q[0], bounds[0], cs, g->nx), a1 = cell_of(q[2], bounds[0], cs, g->nx);
            int b0 = cell_of(q[1], bounds[1], cs, g->ny), b1 = cell_of(q[3], bounds[1], cs, g->ny);
            if (a0 > a1) { int t = a0; a0 = a1; a1 = t; }
            if (b0 > b1) { int t = b0; b0 = b1; b1 = t; }
            for (int y = b0; y <= b1; y++)
                for (int x = a0; x <= a1; x++) {
                    int64_t c = (int64_t)y * g->nx + x;
                    if (pass == 0) cnt[c + 1]++;
                    else g->items[cnt[c]++] = i;
                }
        }
        if (pass == 0) {
            for (int64_t c = 0; c < nc; c++) cnt[c + 1] += cnt[c];
            g->items = (int64_t *)malloc((size_t)(cnt[nc] + 1) * sizeof(int64_t));
            g->start = (int64_t *)malloc((size_t)(nc + 1) * sizeof(int64_t));
            if (!g->items || !g->start) { free(cnt); oc_grid_destroy(g); return NULL; }
            memcpy(g->start, cnt, (size_t)(nc + 1) * sizeof(int64_t));
        }
    }
    free(cnt);
    return g;
}

void oc_grid_destroy(oc_grid *g) {
    if (!g) return;
    free(g->start);
    free(g->items);
    free(g);
}

int oc_grid_box_collides(const oc_grid *g, const double box[4], const double *ignore) {
    if (!box_in(g->b, box)) return 1;
    int a0 = cell_of(box[0], g->b[0], g->cs, g->nx), a1 = cell_of(box[2], g->b[0], g->cs, g->nx);
    int b0 = cell_of(box[1], g->b[1], g->cs, g->ny), b1 = cell_of(box[3], g->b[1], g->cs, g->ny);
    if (a0 > a1) { int t = a0; a0 = a1; a1 = t; }
    if (b0 > b1) { int t = b0; b0 = b1; b1 = t; }
    for (int y = b0; y <= b1; y++)
        for (int x = a0; x <= a1; x++) {
            int64_t c = (int64_t)y * g->nx + x;
            for (int64_t k = g->start[c]; k < g->start[c + 1]; k++) {
                const double *q = g->r + 4 * g->items[k];
                if (ignore && same_rect(q, ignore)) continue;
                if (collide(q, box)) return 1;
            }
        }
    return 0;
}

int64_t oc_grid_point_hit(const oc_grid *g, double px, double py) {
    int x = cell_of(px, g->b[0], g->cs, g->nx), y = cell_of(py, g->b[1], g->cs, g->ny);
    int64_t c = (int64_t)y * g->nx + x, best = -1;
    for (int64_t k = g->start[c]; k < g->start[c + 1]; k++) {
        int64_t i = g->items[k];
        if (contains_pt(g->r + 4 * i, px, py) && (best < 0 || i < best)) best = i;
    }
    return best;
}

/* Tree::drawBiggestSquareAtPoint, CPU/quadTree.cpp:264-312, parameterised
 * over the box predicate. */
typedef int (*box_pred)(const void *ctx, const double box[4]);

static void biggest_square(const void *ctx, box_pred coll, const double *bounds, double px,
                           double py, double out[4]) {
    const double MIN_DIST = (double).095f;
    int isc, maxReached = 0;
    double dist;
    double o[4] = {px - 1, py - 1, px + 1, py + 1};
    double init[4] = {px - 2, py - 2, px + 2, py + 2};
    double bw = bounds[2] - bounds[0], bh = bounds[3] - bounds[1];
    dist = (bh > bw) ? bh : bw;
    dist *= OC_INIT_FACTOR;
    if (coll(ctx, o)) { memcpy(out, o, sizeof(o)); return; }
    if (coll(ctx, init)) { memcpy(out, init, sizeof(init)); return; }
    while ((isc = coll(ctx, o)) || !maxReached || dist > MIN_DIST) {
        if (isc) {
            if (dist > MIN_DIST) dist /= 2;
            maxReached = 1;
            o[0] += dist; o[1] += dist; o[2] -= dist; o[3] -= dist;
        } else {
            if (maxReached) dist /= 2;
            o[0] -= dist; o[1] -= dist; o[2] += dist; o[3] += dist;
        }
    }
    memcpy(out, o, sizeof(o));
}

static int grid_pred(const void *ctx, const double box[4]) {
    return oc_grid_box_collides((const oc_grid *)ctx, box, NULL);
}

void oc_grid_biggest_square(const oc_grid *g, double px, double py, double out[4]) {
    biggest_square(g, grid_pred, g->b, px, py, out);
}

void oc_grid_query_batch(const oc_grid *g, const double *pts, int64_t n, double *sq_out,
                         int64_t *hit_out) {
    for (int64_t i = 0; i < n; i++) {
        oc_grid_biggest_square(g, pts[2 * i], pts[2 * i + 1], sq_out + 4 * i);
        hit_out[i] = oc_grid_point_hit(g, pts[2 * i], pts[2 * i + 1]);
    }
}

/* Tree::getAdjustedGaussianFactor + creatGaussianSurfFrom,
 * CPU/quadTree.cpp:315-364 (the surface ignores rects equal to r). */
typedef int (*box_pred_ign)(const void *ctx, const double box[4], const double *ignore);

static double adjusted_factor(const void *ctx, box_pred_ign coll, const double r[4],
                              double factor, int axis_y) {
    int isc, dividing = 1, first = 1;
    double adj = factor, lb = 1., rb = factor, s[4];
    for (int i = 0; i < OC_GAUSS_ACCURACY; i++) {
        if (axis_y) oc_scale_rect(r, 1., adj, s);
        else oc_scale_rect(r, adj, 1., s);
        isc = coll(ctx, s, r); /* !isInBounds || checkCollisions: the latter tests bounds too */
        if (first && !isc) break;
        if ((isc && !dividing) || (!isc && dividing)) dividing = !dividing;
        if (dividing) adj = rb = (lb + rb) / 2.;
        else adj = lb = (lb + rb) / 2.;
        first = 0;
    }
    return adj;
}

static void gauss_scale(const void *ctx, box_pred_ign coll, const double r[4], double factor,
                        double out[4]) {
    if (factor < 1) { memcpy(out, r, 4 * sizeof(double)); return; }
    double fx = adjusted_factor(ctx, coll, r, factor, 0);
    double fy = adjusted_factor(ctx, coll, r, factor, 1);
    oc_scale_rect(r, fx, fy, out);
}

static int grid_pred_ign(const void *ctx, const double box[4], const double *ignore) {
    return oc_grid_box_collides((const oc_grid *)ctx, box, ignore);
}

void oc_grid_gauss_scale(const oc_grid *g, const double r[4], double factor, double out[4]) {
    gauss_scale(g, grid_pred_ign, r, factor, out);
}

/* ------------------------------------------------------------------------ */
/* The reference CPU quadtree, CPU/quadTree.cpp:73-262, restated            */
/* ------------------------------------------------------------------------ */
typedef struct {
    int level, split;
    double b[4];
    int child[4];
    int64_t *obj; /* layer indices, list order */
    int64_t head, n, cap;
} rnode;

struct oc_rtree {
    rnode *nd;
    int64_t nn, cap;
    const double *r;
    int oom;
};

static int rt_new(oc_rtree *t, int level, const double b[4]) {
    if (t->nn == t->cap) {
        int64_t nc = t->cap ? t->cap * 2 : 256;
        rnode *p = (rnode *)realloc(t->nd, (size_t)nc * sizeof(rnode));
        if (!p) { t->oom = 1; return -1; }
        t->nd = p;
        t->cap = nc;
    }
    rnode *x = &t->nd[t->nn];
    memset(x, 0, sizeof(*x));
    x->level = level;
    memcpy(x->b, b, sizeof(x->b));
    for (int i = 0; i < 4; i++) x->child[i] = -1;
    return (int)t->nn++;
}

static void rt_push(oc_rtree *t, int id, int64_t v) {
    rnode *x = &t->nd[id];
    if (x->head + x->n == x->cap) {
        if (x->head > 0) {
            memmove(x->obj, x->obj + x->head, (size_t)x->n * sizeof(int64_t));
            x->head = 0;
        } else {
            int64_t nc = x->cap ? x->cap * 2 : 8;
            int64_t *p = (int64_t *)realloc(x->obj, (size_t)nc * sizeof(int64_t));
            if (!p) { t->oom = 1; return; }
            x->obj = p;
            x->cap = nc;
        }
    }
    x->obj[x->head + x->n++] = v;
}

static int64_t rt_pop_front(oc_rtree *t, int id) {
    rnode *x = &t->nd[id];
    int64_t v = x->obj[x->head++];
    x->n--;
    return v;
}

/* Tree::split, quadTree.cpp:73-102: children UL, UR, LR, LL. */
static void rt_split(oc_rtree *t, int id) {
    double b[4];
    memcpy(b, t->nd[id].b, sizeof(b));
    int lvl = t->nd[id].level;
    double sw = b[0] + ((b[2] - b[0]) / 2);
    double sh = b[1] + ((b[3] - b[1]) / 2);
    double ul[4] = {b[0], b[1], sw, sh};
    double ur[4] = {sw, b[1], b[2], sh};
    double lr[4] = {sw, sh, b[2], b[3]};
    double ll[4] = {b[0], sh, sw, b[3]};
    int c0 = rt_new(t, lvl + 1, ul), c1 = rt_new(t, lvl + 1, ur);
    int c2 = rt_new(t, lvl + 1, lr), c3 = rt_new(t, lvl + 1, ll);
    rnode *x = &t->nd[id];
    x->child[0] = c0; x->child[1] = c1; x->child[2] = c2; x->child[3] = c3;
    x->split = 1;
}

/* Tree::insert, quadTree.cpp:105-146, including its redistribution loop
 * (which moves about half of the objects down and also re-appends them to
 * the parent) and the level-11 node that splits but then refuses inserts. */
static int rt_insert(oc_rtree *t, int id, int64_t ri) {
    const double *r = t->r + 4 * ri;
    if (!box_in(t->nd[id].b, r)) return 0;
    if (t->nd[id].n < OC_MAX_OBJECTS && !t->nd[id].split) {
        rt_push(t, id, ri);
        return 1;
    } else if (t->nd[id].n >= OC_MAX_OBJECTS && !t->nd[id].split) {
        rt_split(t, id);
        int64_t counter = t->nd[id].n;
        for (int64_t i = 0; i < counter; ++i) {
            int64_t tmp = rt_pop_front(t, id);
            for (int c = 0; c < 4; ++c)
                if (rt_insert(t, t->nd[id].child[c], tmp)) { counter--; break; }
            rt_push(t, id, tmp);
            counter--;
        }
    }
    if (t->nd[id].level < OC_MAX_LEVELS && t->nd[id].split) {
        for (int c = 0; c < 4; ++c)
            if (rt_insert(t, t->nd[id].child[c], ri)) return 1;
        rt_push(t, id, ri);
        return 1;
    }
    return 0;
}

oc_rtree *oc_rtree_create(const double *rects, int64_t n, const double bounds[4]) {
    oc_rtree *t = (oc_rtree *)calloc(1, sizeof(oc_rtree));
    if (!t) return NULL;
    t->r = rects;
    rt_new(t, 0, bounds);
    for (int64_t i = 0; i < n && !t->oom; i++) rt_insert(t, 0, i); /* createTree, mainFunctions.cpp:33-38 */
    if (t->oom) { oc_rtree_destroy(t); return NULL; }
    return t;
}

void oc_rtree_destroy(oc_rtree *t) {
    if (!t) return;
    for (int64_t i = 0; i < t->nn; i++) free(t->nd[i].obj);
    free(t->nd);
    free(t);
}

void oc_rtree_stats(const oc_rtree *t, int64_t *nodes, int64_t *stored, int *max_level) {
    int64_t s = 0;
    int ml = 0;
    for (int64_t i = 0; i < t->nn; i++) {
        s += t->nd[i].n;
        if (t->nd[i].level > ml) ml = t->nd[i].level;
    }
    *nodes = t->nn;
    *stored = s;
    *max_level = ml;
}

/* Tree::checkCollisions, quadTree.cpp:148-198.  With defect=1 the siblings
 * that addNodesToStack writes never become visible to the caller (its stack
 * pointer is a by-value copy), so only the first overlapping child is ever
 * followed.  defect=0 keeps them (the GPU twin's complete DFS). */
int oc_rtree_box_collides(const oc_rtree *t, const double box[4], const double *ignore,
                          int defect) {
    if (!box_in(t->nd[0].b, box)) return 1;
    int stack[4 * (OC_MAX_LEVELS + 2) * 4];
    int sp = 0, node = 0;
    while (node >= 0) {
        const rnode *x = &t->nd[node];
        for (int64_t k = 0; k < x->n; k++) {
            const double *q = t->r + 4 * x->obj[x->head + k];
            if (!(ignore && same_rect(q, ignore)) && collide(q, box)) return 1;
        }
        int cl[4] = {0, 0, 0, 0}, any = 0;
        if (x->split)
            for (int c = 0; c < 4; c++) any |= cl[c] = collide(t->nd[x->child[c]].b, box);
        if (!any) {
            node = sp > 0 ? stack[--sp] : -1;
        } else {
            int next = -1;
            for (int c = 0; c < 4; c++)
                if (cl[c]) { next = x->child[c]; break; }
            if (!defect)
                for (int c = 0; c < 4; c++)
                    if (cl[c] && x->child[c] != next) stack[sp++] = x->child[c];
            node = next;
        }
    }
    return 0;
}

/* Tree::checkCollisons(point), quadTree.cpp:240-262: at each level the own
 * objects are tested in list order, then only the FIRST child containing p is
 * followed. */
int64_t oc_rtree_point_hit(const oc_rtree *t, double px, double py) {
    int cur = 0, next = -1;
    for (;;) {
        const rnode *x = &t->nd[cur];
        if (x->split)
            for (int c = 0; c < 4; c++)
                if (contains_pt(t->nd[x->child[c]].b, px, py)) { next = x->child[c]; break; }
        for (int64_t k = 0; k < x->n; k++) {
            int64_t i = x->obj[x->head + k];
            if (contains_pt(t->r + 4 * i, px, py)) return i;
        }
        if (!x->split || next < 0) return -1;
        if (next == cur) return -1; /* the reference would spin here; p left the tree */
        cur = next;
    }
}

typedef struct {
    const oc_rtree *t;
    int defect;
} rt_ctx;

static int rt_pred(const void *ctx, const double box[4]) {
    const rt_ctx *c = (const rt_ctx *)ctx;
    return oc_rtree_box_collides(c->t, box, NULL, c->defect);
}
static int rt_pred_ign(const void *ctx, const double box[4], const double *ignore) {
    const rt_ctx *c = (const rt_ctx *)ctx;
    return oc_rtree_box_collides(c->t, box, ignore, c->defect);
}

void oc_rtree_biggest_square(const oc_rtree *t, double px, double py, int defect, double out[4]) {
    rt_ctx c = {t, defect};
    biggest_square(&c, rt_pred, t->nd[0].b, px, py, out);
}

void oc_rtree_gauss_scale(const oc_rtree *t, const double r[4], double factor, int defect,
                          double out[4]) {
    rt_ctx c = {t, defect};
    gauss_scale(&c, rt_pred_ign, r, factor, out);
}

/* ------------------------------------------------------------------------ */
/* Walks                                                                    */
/* ------------------------------------------------------------------------ */
void oc_walk_gauss_surface(const oc_grid *g, const double *rects, const oc_walk_cfg *cfg,
                           double out[4]) {
    const double *R = rects + 4 * cfg->target;
    if (cfg->gauss_mode == OC_GAUSS_SCALE) {
        oc_grid_gauss_scale(g, R, cfg->gauss_param, out);
    } else {
        double d = cfg->gauss_param;
        out[0] = R[0] - d; out[1] = R[1] - d; out[2] = R[2] + d; out[3] = R[3] + d;
    }
}

/* Uniform point on the perimeter of G, clockwise from the top-left corner,
 * with the outward normal of the side it lands on. */
static void perimeter_point(const double G[4], double u, double p[2], double n[2]) {
    double w = G[2] - G[0], h = G[3] - G[1];
    double s = u * (2 * w + 2 * h);
    if (s < w) { p[0] = G[0] + s; p[1] = G[1]; n[0] = 0; n[1] = -1; }
    else if (s < w + h) { p[0] = G[2]; p[1] = G[1] + (s - w); n[0] = 1; n[1] = 0; }
    else if (s < 2 * w + h) { p[0] = G[2] - (s - w - h); p[1] = G[3]; n[0] = 0; n[1] = 1; }
    else { p[0] = G[0]; p[1] = G[3] - (s - 2 * w - h); n[0] = -1; n[1] = 0; }
}

/* Uniform number of hop `hop` of walk `walk`: Philox4x32-10 block
 * (hop / 4, walk, stream) under key `seed`, word hop % 4, scaled by 2^-32. */
static double draw(uint64_t seed, uint32_t stream, uint64_t walk, uint32_t hop) {
    uint32_t ctr[4] = {hop >> 2, (uint32_t)walk, (uint32_t)(walk >> 32), stream};
    uint32_t key[2] = {(uint32_t)seed, (uint32_t)(seed >> 32)};
    uint32_t o[4];
    oc_philox4x32_10(ctr, key, o);
    return (double)o[hop & 3] * (1.0 / 4294967296.0);
}

/* The walk of CPU/mainFunctions.cpp:48-90 on complete queries, with the
 * uniform-start capacitance weight
 *   w = -eps * L * (W_{i1} . n(p0)) / a0
 * (L = Gaussian perimeter, a0 = side of the first transition square, i1 =
 * first-hop bin, n = outward normal of the Gaussian side at p0). */
int oc_walk_run(const oc_grid *g, const double *rects, const oc_walk_cfg *cfg, uint64_t first,
                uint64_t count, int64_t *end_out, int32_t *hops_out, int32_t *bin_out,
                double *weight_out, double *cv_out) {
    /* the tables are the same for every call: evaluated once (the oracle is
     * single-threaded) */
    static int ready = 0;
    static double gtab[OC_NSAMPLE], intg[OC_NSAMPLE + 1], wx[OC_NSAMPLE], wy[OC_NSAMPLE];
    if (!ready) {
        oc_green_table(OC_NSAMPLE, gtab, intg);
        oc_weight_table(OC_NSAMPLE, intg, wx, wy);
        ready = 1;
    }
    double G[4];
    oc_walk_gauss_surface(g, rects, cfg, G);
    double L = 2 * (G[2] - G[0]) + 2 * (G[3] - G[1]);
    for (uint64_t k = 0; k < count; k++) {
        uint64_t w = first + k;
        double u0, p[2], nrm[2] = {0, 0}, sq[4];
        uint32_t hop = 0;
        u0 = draw(cfg->seed, cfg->stream, w, hop);
        if (cfg->start_strata) u0 = ((double)(uint32_t)(w % cfg->start_strata) + u0) / (double)cfg->start_strata;
        if (cfg->start_mode == OC_START_UNIFORM) {
            if (cfg->start_grid) {
                uint32_t q = (uint32_t)(u0 * (double)cfg->start_grid);
                u0 = ((double)q + 0.5) / (double)cfg->start_grid;
            }
            perimeter_point(G, u0, p, nrm);
        } else {
            oc_point_from_index(G, oc_bin_index(intg, OC_NSAMPLE, u0), OC_NSAMPLE,
                                cfg->exact_perimeter, p);
        }
        int64_t end;
        int32_t hops = 0, bin1 = -1;
        double a0 = 0.0, p1[2] = {0.0, 0.0};
        for (;;) {
            if (!pt_in(g->b, p[0], p[1])) { end = OC_END_ESCAPED; break; }
            oc_grid_biggest_square(g, p[0], p[1], sq);
            int64_t hit = oc_grid_point_hit(g, p[0], p[1]);
            hops++;
            if (hit >= 0) { end = hit; break; }
            if (hops >= cfg->hop_cap) { end = OC_END_ABORTED; break; }
            hop++;
            u0 = draw(cfg->seed, cfg->stream, w, hop);
            int bin = oc_bin_index(intg, OC_NSAMPLE, u0);
            oc_point_from_index(sq, bin, OC_NSAMPLE, cfg->exact_perimeter, p);
            if (hop == 1) { bin1 = bin; a0 = sq[2] - sq[0]; p1[0] = p[0]; p1[1] = p[1]; }
        }
        double c = 0.0;
        if (cfg->start_mode == OC_START_UNIFORM && bin1 >= 0)
            c = -cfg->permittivity * L * (wx[bin1] * nrm[0] + wy[bin1] * nrm[1]) / a0;
        end_out[k] = end;
        hops_out[k] = hops;
        bin_out[k] = bin1;
        weight_out[k] = c;
        if (cv_out) {
            cv_out[4 * k] = p1[0];
            cv_out[4 * k + 1] = p1[1];
            cv_out[4 * k + 2] = a0;
            cv_out[4 * k + 3] = c;
        }
    }
    return OC_OK;
}

int64_t oc_walk_stream(const oc_grid *g, const oc_rtree *t, int defect, const double gauss[4],
                       const double *intg, const double *r, int64_t nr, int64_t *used,
                       int32_t *hops) {
    const double *b = t ? t->nd[0].b : g->b;
    double sq[4], p[2];
    memcpy(sq, gauss, sizeof(sq));
    int64_t k = 0, end = OC_END_ESCAPED;
    int32_t h = 0;
    for (;;) {
        if (k >= nr) { end = OC_END_ABORTED; break; }
        oc_point_from_index(sq, oc_bin_index(intg, OC_NSAMPLE, r[k++]), OC_NSAMPLE, 0, p);
        if (!pt_in(b, p[0], p[1])) { end = OC_END_ESCAPED; break; }
        int64_t hit;
        if (t) {
            oc_rtree_biggest_square(t, p[0], p[1], defect, sq);
            hit = defect ? oc_rtree_point_hit(t, p[0], p[1]) : oc_grid_point_hit(g, p[0], p[1]);
        } else {
            oc_grid_biggest_square(g, p[0], p[1], sq);
            hit = oc_grid_point_hit(g, p[0], p[1]);
        }
        h++;
        if (hit >= 0) { end = hit; break; }
    }
    *used = k;
    *hops = h;
    return end;
}

/* ------------------------------------------------------------------------ */
/* Control-variate features (brute force over all rects)                    */
/* ------------------------------------------------------------------------ */
/* d / a0 as d * (1 / a0), clamped to [-16, 16] */
static float cv_feat(double d, double inv) {
    double v = d * inv;
    v = fmin(fmax(v, -16.0), 16.0);
    return (float)v;
}

static void cv_edges(double px, double py, const double *r, double a0, float *f) {
    double cx = fmin(fmax(px, r[0]), r[2]), cy = fmin(fmax(py, r[1]), r[3]);
    double inv = 1.0 / a0;
    f[0] = cv_feat(cx - px, inv);
    f[1] = cv_feat(r[1] - py, inv);
    f[2] = cv_feat(r[2] - px, inv);
    f[3] = cv_feat(cy - py, inv);
    f[4] = f[0];
    f[5] = cv_feat(r[3] - py, inv);
    f[6] = cv_feat(r[0] - px, inv);
    f[7] = f[3];
}

void oc_cv_features(const double *rects, int64_t n, int64_t target, const double *rec4, int64_t m,
                    float *out) {
    for (int64_t i = 0; i < m; i++) {
        double px = rec4[4 * i], py = rec4[4 * i + 1], a0 = rec4[4 * i + 2];
        float *f = out + 16 * i;
        if (!(a0 > 0.0)) {
            for (int q = 0; q < 16; q++) f[q] = 0.f;
            continue;
        }
        cv_edges(px, py, rects + 4 * target, a0, f);
        int64_t bk = -1;
        double best = 1e300;
        for (int64_t k = 0; k < n; k++) {
            if (k == target) continue;
            const double *r = rects + 4 * k;
            double g = fmax(fmax(r[0] - px, px - r[2]), fmax(r[1] - py, py - r[3]));
            if (g < best) { best = g; bk = k; }
        }
        if (bk >= 0) cv_edges(px, py, rects + 4 * bk, a0, f + 8);
        else for (int q = 8; q < 16; q++) f[q] = 16.f;
    }
}

/* ---------------------------------------------------------------- layouts */
/* splitmix64 (Steele, Lea and Flood, "Fast splittable pseudorandom number
 * generators", OOPSLA 2014). */
static uint64_t sm64_next(uint64_t *s) {
    uint64_t z = (*s += 0x9E3779B97F4A7C15ull);
    z = (z ^ (z >> 30)) * 0xBF58476D1CE4E5B9ull;
    z = (z ^ (z >> 27)) * 0x94D049BB133111EBull;
    return z ^ (z >> 31);
}

static int64_t sm64_range(uint64_t *s, int64_t a, int64_t b) {
    return a + (int64_t)(sm64_next(s) % (uint64_t)(b - a + 1));
}

/* Rejection against accepted rects bucketed by the cell of their lower
 * corner; cells are wider than wmax + gap, so every rect within `gap` of a
 * candidate has its lower corner in the candidate's cell range widened by
 * one cell on each side. */
int oc_generate_layout(uint64_t seed, int64_t n, double domain, int wmin, int wmax, double gap,
                       double *out) {
    if (n <= 0 || wmin < 1 || wmax < wmin || domain < wmax || gap < 0 || domain >= 16777216.0)
        return OC_E_ARG;
    const int64_t D = (int64_t)floor(domain);
    const int64_t cs = (int64_t)wmax + (int64_t)ceil(gap) + 1;
    const int64_t nc = D / cs + 1;
    if (nc > (1 << 20)) return OC_E_ARG;
    int32_t *head = (int32_t *)malloc((size_t)(nc * nc) * sizeof(int32_t));
    int32_t *next = (int32_t *)malloc((size_t)n * sizeof(int32_t));
    if (!head || !next) {
        free(head);
        free(next);
        return OC_E_OOM;
    }
    for (int64_t i = 0; i < nc * nc; i++) head[i] = -1;
    uint64_t s = seed;
    int64_t got = 0, tries = 0;
    int rc = OC_OK;
    while (got < n) {
        if (++tries > 64 * n + 1000) {
            rc = OC_E_ARG;
            break;
        }
        const int64_t w = sm64_range(&s, wmin, wmax), h = sm64_range(&s, wmin, wmax);
        const int64_t x0 = sm64_range(&s, 0, D - w), y0 = sm64_range(&s, 0, D - h);
        const int64_t x1 = x0 + w, y1 = y0 + h;
        int64_t ax = x0 / cs - 1, bx = x0 / cs + 1, ay = y0 / cs - 1, by = y0 / cs + 1;
        if (ax < 0) ax = 0;
        if (ay < 0) ay = 0;
        if (bx > nc - 1) bx = nc - 1;
        if (by > nc - 1) by = nc - 1;
        int ok = 1;
        for (int64_t cy = ay; cy <= by && ok; cy++)
            for (int64_t cx = ax; cx <= bx && ok; cx++)
                for (int32_t j = head[cy * nc + cx]; j >= 0 && ok; j = next[j]) {
                    const double *q = out + 4 * (int64_t)j;
                    const double gx = fmax(q[0] - (double)x1, (double)x0 - q[2]);
                    const double gy = fmax(q[1] - (double)y1, (double)y0 - q[3]);
                    if (fmax(gx, gy) < gap) ok = 0;
                }
        if (!ok) continue;
        double *o = out + 4 * got;
        o[0] = (double)x0;
        o[1] = (double)y0;
        o[2] = (double)x1;
        o[3] = (double)y1;
        const int64_t c = (y0 / cs) * nc + x0 / cs;
        next[got] = head[c];
        head[c] = (int32_t)got;
        got++;
    }
    free(head);
    free(next);
    return rc;
}
