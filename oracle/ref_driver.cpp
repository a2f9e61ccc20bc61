// ref_driver.cpp -- TEST INFRASTRUCTURE ONLY.
//
// A thin extern "C" driver around the UNMODIFIED reference CPU sources
// (piogrzej/engineer-thesis, randomWalk/CPU, randomWalk/green,
// randomWalk/utils), which oracle/Makefile compiles in place from the
// reference checkout into oracle/_ref/librefcpu.so.  Nothing here is copied
// from the reference: this file only calls its public functions, so that the
// tests can pin the C oracle (frwcpu.c) against the reference's own code and
// bench.py can time the reference's CPU walk as the baseline arm.
//
// The reference keeps its tree and RNG in globals and is single-threaded, so
// the driver holds one layout at a time; run several processes for
// throughput.  Nothing below triggers the reference's file loggers (they are
// only created on error paths).

#include "CPU/Parser.h"
#include "CPU/mainFunctions.h"
#include "CPU/quadTree.h"
#include "CPU/rectHost.h"
#include "green/green.h"
#include "green/randgen.h"

#include <stdint.h>
#include <string.h>
#include <array>
#include <map>
#include <vector>

// runRandomWalk (CPU/mainFunctions.cpp:12-31) references the CUDA driver;
// the CPU-only build supplies a stub that is never called.
floatingPoint getAvgPathLenCUDA(char *, int, int, bool, int) { return -1.0; }

namespace {
std::vector<RectHost> g_layer;
RectHost g_bounds;
Tree *g_tree = nullptr;
std::map<std::array<double, 4>, int64_t> g_index;  // lexicographic; first index wins
REAL64_t g_g[NSAMPLE], g_dgdx[NSAMPLE], g_dgdy[NSAMPLE], g_intg[NSAMPLE + 1];

void to4(const RectHost &r, double *o) {
    o[0] = r.topLeft.x;
    o[1] = r.topLeft.y;
    o[2] = r.bottomRight.x;
    o[3] = r.bottomRight.y;
}
RectHost from4(const double *a) { return RectHost(point(a[0], a[1]), point(a[2], a[3])); }
int64_t index_of(const RectHost &r) {
    auto it = g_index.find({r.topLeft.x, r.topLeft.y, r.bottomRight.x, r.bottomRight.y});
    return it == g_index.end() ? -1 : it->second;
}
void build_index() {
    g_index.clear();
    for (size_t i = 0; i < g_layer.size(); i++) {
        const RectHost &r = g_layer[i];
        g_index.insert({{r.topLeft.x, r.topLeft.y, r.bottomRight.x, r.bottomRight.y}, (int64_t)i});
    }
}
}  // namespace

extern "C" {

// Parser::parse + getLayerAt + getLayerSize (CPU/Parser.cpp:15-87), then
// createTree (CPU/mainFunctions.cpp:33-38).  Returns the rect count or -1.
int64_t ref_load(const char *path, int layer) {
    static char delim[] = "<<";
    Parser parser(delim);
    parser.parse(path);
    if (layer < 0 || layer >= parser.getLayerCount()) return -1;
    g_layer = parser.getLayerAt(layer);
    if (g_layer.empty()) return -1;
    g_bounds = parser.getLayerSize(layer);
    delete g_tree;  // the reference has no Tree destructor; the nodes leak
    g_tree = new Tree(0, (int)g_layer.size(), g_bounds);
    createTree(g_tree, g_layer);
    precompute_unit_square_green(g_g, g_dgdx, g_dgdy, g_intg, NSAMPLE);
    build_index();
    return (int64_t)g_layer.size();
}

// Same as ref_load but from caller-supplied rects and bounds.
int64_t ref_load_rects(const double *rects, int64_t n, const double *bounds) {
    g_layer.clear();
    for (int64_t i = 0; i < n; i++) g_layer.push_back(from4(rects + 4 * i));
    g_bounds = from4(bounds);
    delete g_tree;
    g_tree = new Tree(0, (int)g_layer.size(), g_bounds);
    createTree(g_tree, g_layer);
    precompute_unit_square_green(g_g, g_dgdx, g_dgdy, g_intg, NSAMPLE);
    build_index();
    return (int64_t)g_layer.size();
}

void ref_rects(double *out) {
    for (size_t i = 0; i < g_layer.size(); i++) to4(g_layer[i], out + 4 * i);
}
void ref_bounds(double *out) { to4(g_bounds, out); }

void ref_green(double *g, double *dgdx, double *dgdy, double *intg) {
    memcpy(g, g_g, sizeof(g_g));
    memcpy(dgdx, g_dgdx, sizeof(g_dgdx));
    memcpy(dgdy, g_dgdy, sizeof(g_dgdy));
    memcpy(intg, g_intg, sizeof(g_intg));
}

// The reference's unit-cube table, precompute_unit_cube_green
// (green/green.h:79-80, green/green.cpp:392-431; never called by the
// reference itself): 6 n^2 samples per array, intg of 6 n^2 + 1.
void ref_unit_cube_green(int n, double *g, double *dgdx, double *dgdy, double *dgdz, double *intg) {
    precompute_unit_cube_green(g, dgdx, dgdy, dgdz, intg, (UINTpt_t)n);
}

// green_cube / deriv_green_cube (green/green.cpp:232-267,311-388) at one point.
double ref_green_cube(double a, double eta, double dzeta) { return green_cube(a, eta, dzeta); }
void ref_deriv_green_cube(double *dg, double a, double eta, double dzeta) {
    deriv_green_cube(dg, a, eta, dzeta);
}

int ref_get_index(double r) { return getIndex(g_intg, r); }

void ref_point_from_index(const double *sq, int index, double *out) {
    RectHost s = from4(sq);
    point p = s.getPointFromNindex(index, NSAMPLE);
    out[0] = p.x;
    out[1] = p.y;
}

int ref_box_collides(const double *box, const double *ignore) {
    return ignore ? g_tree->checkCollisions(from4(box), from4(ignore))
                  : g_tree->checkCollisions(from4(box));
}

void ref_biggest_square(double px, double py, double *out) {
    to4(g_tree->drawBiggestSquareAtPoint(point(px, py)), out);
}

// Tree::checkCollisons(point): the layer index of the rect returned, or -1.
int64_t ref_point_hit(double px, double py, double *rect_out) {
    RectHost r;
    if (!g_tree->checkCollisons(point(px, py), r)) return -1;
    if (rect_out) to4(r, rect_out);
    return index_of(r);
}

void ref_query_batch(const double *pts, int64_t n, double *sq_out, int64_t *hit_out) {
    for (int64_t i = 0; i < n; i++) {
        ref_biggest_square(pts[2 * i], pts[2 * i + 1], sq_out + 4 * i);
        hit_out[i] = ref_point_hit(pts[2 * i], pts[2 * i + 1], nullptr);
    }
}

void ref_gauss(int64_t target, double factor, double *out) {
    to4(g_tree->creatGaussianSurfFrom(g_layer[target], factor), out);
}

// Walks of RandomWalk (CPU/mainFunctions.cpp:48-90) with the reference's
// JKISS generator seeded ONCE (JKISS_seed) instead of the per-walk
// /dev/urandom reseed, so runs are reproducible.  The body calls the same
// reference functions in the same order.  The uniforms consumed are written
// to r_out (capacity r_cap; the count is returned through *r_used) so the
// C oracle can replay the identical trajectories.  r == 1.0 would make the
// reference's getIndex read past intg[NSAMPLE]; such draws are redrawn.
int ref_walks_seeded(int64_t target, int64_t n, uint32_t s0, uint32_t s1, uint32_t s2,
                     uint32_t s3, int64_t *end_out, int32_t *hops_out, double *r_out,
                     int64_t r_cap, int64_t *r_used) {
    JKISS_seed(s0, s1 ? s1 : 1u, s2, s3 % 698769068u + 1u, 0);
    myrand = JKISS;
    MY_RAND_MAX = 4294967295ull;
    const RectHost &R = g_layer[target];
    RectHost square0 = g_tree->creatGaussianSurfFrom(R, 1.5);
    int64_t used = 0;
    for (int64_t w = 0; w < n; w++) {
        RectHost square = square0, output;
        int count = 0;
        bool hit = false, broken = false;
        do {
            floatingPoint r;
            do {
                r = myrand() / (floatingPoint)(MY_RAND_MAX);
            } while (r >= 1.0);
            if (r_out && used < r_cap) r_out[used] = r;
            used++;
            point p = square.getPointFromNindex(getIndex(g_intg, r), NSAMPLE);
            if (false == g_tree->isInBounds(p)) {
                broken = true;
                break;
            }
            square = g_tree->drawBiggestSquareAtPoint(p);
            hit = g_tree->checkCollisons(p, output);
            count++;
        } while (false == hit);
        end_out[w] = broken ? -1 : index_of(output);
        hops_out[w] = count;
    }
    if (r_used) *r_used = used;
    return 0;
}

// The reference walk exactly as shipped: RandomWalk itself, which calls
// rng_init(1) (100,000 warm-up draws after a /dev/urandom reseed) at the
// start of every walk.  Used only to time the shipped CPU path.
int ref_walks_as_shipped(int64_t target, int64_t n, int64_t *end_out, int32_t *hops_out) {
    const RectHost R = g_layer[target];
    for (int64_t w = 0; w < n; w++) {
        int count = 0;
        RectHost out = RandomWalk(R, g_tree, count, g_intg, (int)w);
        end_out[w] = (out == RectHost()) ? -1 : index_of(out);
        hops_out[w] = count;
    }
    return 0;
}

}  // extern "C"
