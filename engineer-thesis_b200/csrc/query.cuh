// query.cuh -- device-side collision queries on the flat Morton quadtree.
//
// The reference answers drawBiggestSquareAtPoint (CPU/quadTree.cpp:264-312,
// Cuda/d_quadTree.cu:86-134) with 17-26 full tree traversals per point: one
// checkCollisions(box) per step of an expand/bisect loop.  Here ONE traversal
// per point computes the L-infinity clearance
//     d* = min( distance to the layer bounds, min_R gap(R, p) ),
//     gap(R, p) = max(R.x0 - p.x, p.x - R.x1, R.y0 - p.y, p.y - R.y1),
// and the short list of rects whose gap lies within 2*delta of d*; the loop is
// then replayed on scalars with the reference's own FP64 operations.  Every
// box of the loop is p +- h up to the rounding of its four coordinates
// (each within eps of the others, eps << delta), so a rect outside the list
// can only touch such a box when the box's smallest extent already exceeds d*
// + delta, and then the nearest rect (in the list) touches it too.  Hence
//     collides(box) = outside(bounds) || any(listed rect touches box)
// exactly, and the returned square is bit-identical to the reference's.
// The point query (checkCollisons(point), CPU/quadTree.cpp:240-262) falls out
// of the same traversal: rects with gap <= 0 contain p (closed intervals).
#pragma once

#include <cuda_runtime.h>

#include "frw_internal.h"

namespace frw {

constexpr int kStackMax = 64;
constexpr int kCandMax = 8;
constexpr int kReplayCap = 256;
constexpr int kNoHit = 0x7FFFFFFF;
constexpr double kMinDist = (double).095f;  // drawBiggestSquareAtPoint MIN_DIST

// The rects the replay tests for boxes within delta of the clearance: a
// point answered by a cell list keeps its cell's whole list (first >= 0:
// the cell-list entries first .. first + n - 1), a superset of the near
// ties; a point answered by the tree keeps the near-tie list idx[0 .. n) of
// tree rects (first == -1).  Testing more rects than the ties is as exact:
// every listed rect is a real rect of the layout.  More ties than kCandMax
// (rects whose near sides line up tie exactly) set first = -2: the replay's
// boxes near the clearance are then tested against the whole tree.
struct Cands {
    int idx[kCandMax];  // tree: positions of the near-tied rects among the tree's rects
    float g[kCandMax];  // their gaps, rounded down (keeping extra entries is harmless)
    int n;
    int first;
};

// L-infinity distance from a point (in FP32) to a box, 0 inside.
__device__ __forceinline__ float lb_box_f(const float4 b, float px, float py) {
    return fmaxf(fmaxf(fmaxf(b.x - px, px - b.z), fmaxf(b.y - py, py - b.w)), 0.f);
}

// One rect of a leaf or a cell list: FP32 screen, then the exact FP64 gap;
// tightens `best`, keeps the near-tie list and the containing rect.
// kTies: a full list marks the point (C.first = -2) for the whole-tree
// replay; otherwise a full list is an error.
template <bool kTies>
__device__ __forceinline__ void scan_rect(const float4 r, int k, const int32_t *ids, double px, double py,
                                          float pxf, float pyf, double r2, float slack, float &limf,
                                          double &best, int &hit, Cands &C, uint32_t &st) {
    const float gf = fmaxf(fmaxf(r.x - pxf, pxf - r.z), fmaxf(r.y - pyf, pyf - r.w));
    if (gf > limf) return;
    const double x0 = r.x, y0 = r.y, x1 = r.z, y1 = r.w;
    const double g = fmax(fmax(x0 - px, px - x1), fmax(y0 - py, py - y1));
    if (g <= 0.0 && px >= x0 && py >= y0 && px <= x1 && py <= y1) {
        const int id = __ldg(ids + k);
        hit = id < hit ? id : hit;
    }
    if (g < best) {
        best = g;
        limf = (float)(fmax(best, 0.0) + r2) + slack;
        int j = 0;
        for (int q = 0; q < C.n; q++)
            if ((double)C.g[q] <= best + r2) {
                C.idx[j] = C.idx[q];
                C.g[j] = C.g[q];
                j++;
            }
        C.n = j;
    }
    if (g <= best + r2) {
        if (C.n < kCandMax) {
            C.idx[C.n] = k;
            C.g[C.n] = __double2float_rd(g);
            C.n++;
        } else if (kTies) {
            // more ties than the list holds (rects with aligned sides tie
            // exactly: a column of equal x0 seen from its left): the replay's
            // boxes near the clearance are then tested against the whole tree
            C.first = -2;
        } else {
            st |= kStCandOverflow;
        }
    }
}

// The tree part of clearance (no cell lists, or an overflowed cell): one
// depth-first, nearest-child-first traversal from the bounds distance in
// `best`; FP32 screens (errors below slack), the exact FP64 gap only for
// rects that can matter.
template <bool kTies>
__device__ __forceinline__ uint32_t tree_clearance(const float4 *nbox, const int4 *nref, const float4 *rects,
                                                   const int32_t *ids, double px, double py, double r2, float slack,
                                                   Cands &C, int &hit, double &best) {
    uint32_t st = 0;
    const float pxf = (float)px, pyf = (float)py;
    float limf = (float)(fmax(best, 0.0) + r2) + slack;  // screen: FP32 value > limf => exact > limit
    int stk_node[kStackMax];
    float stk_lb[kStackMax];
    int sp = 0;
    int nd = 0;  // node being visited; the nearest qualifying child is visited next directly
    for (;;) {
        const float4 *bp = nbox + 4 * nd;
        float4 b[4];
        b[0] = __ldg(bp);
        b[1] = __ldg(bp + 1);
        b[2] = __ldg(bp + 2);
        b[3] = __ldg(bp + 3);
        const int4 rf = __ldg(nref + nd);
        const int ref[4] = {rf.x, rf.y, rf.z, rf.w};
        float lb[4];
#pragma unroll
        for (int c = 0; c < 4; c++) lb[c] = ref[c] == kRefEmpty ? 3.0e38f : lb_box_f(b[c], pxf, pyf);
        // leaves of this node first: they tighten `best` before descending
#pragma unroll
        for (int c = 0; c < 4; c++) {
            if (ref[c] >= kRefEmpty || lb[c] > limf) continue;
            const int f = leaf_first(ref[c]), m = leaf_count(ref[c]);
            for (int k = f; k < f + m; k++)
                scan_rect<kTies>(__ldg(rects + k), k, ids, px, py, pxf, pyf, r2, slack, limf, best, hit, C, st);
        }
        // internal children within reach: visit the nearest next, stack the rest
        int next = -1;
        float nlb = 0.f;
#pragma unroll
        for (int c = 0; c < 4; c++) {
            if (ref[c] < 0 || lb[c] > limf) continue;
            int push = ref[c];
            float plb = lb[c];
            if (next < 0 || lb[c] < nlb) {
                push = next;
                plb = nlb;
                next = ref[c];
                nlb = lb[c];
            }
            if (push >= 0) {
                if (sp < kStackMax) {
                    stk_node[sp] = push;
                    stk_lb[sp] = plb;
                    sp++;
                } else {
                    st |= kStStackOverflow;
                }
            }
        }
        if (next >= 0) {
            nd = next;
            continue;
        }
        // nothing below: resume the most recent stacked subtree still in reach
        while (sp > 0 && stk_lb[sp - 1] > limf) --sp;
        if (sp == 0) break;
        nd = stk_node[--sp];
    }
    return st;
}

// The same, out of line (a call: smaller code where the tree is rare).
template <bool kTies>
static __device__ __noinline__ uint32_t tree_clearance_call(const float4 *nbox, const int4 *nref,
                                                            const float4 *rects, const int32_t *ids, double px,
                                                            double py, double r2, float slack, Cands &C, int &hit,
                                                            double &best) {
    return tree_clearance<kTies>(nbox, nref, rects, ids, px, py, r2, slack, C, hit, best);
}

// The clearance of p and its near-tie list.  With cell lists the list of
// p's cell holds every rect that can come within 2*delta of the clearance of
// any point of the cell (the cell's radius is bounded by the clearance of
// its centre plus half a side, with a margin far above the rounding of the
// cell index), so scanning it gives the same d*, the same containing rect and
// a superset of the same ties as the whole tree; a list holds about two
// rects, so every one gets the exact FP64 gap without an FP32 screen, and
// the list itself stands for the ties.  Otherwise (no cell lists, or an
// overflowed cell): one depth-first, nearest-child-first traversal.  Node
// boxes and rect gaps are screened in FP32 (errors below L.slack); only
// rects that can matter -- inside the current tie window or containing p --
// get the exact FP64 gap.  Returns status bits.
// kInside: the caller has checked that p lies inside the bounds.
// kOutOfLineTree: the tree traversal is a call (smaller code at the caller).
// kTies: see scan_rect.
template <bool kInside = false, bool kOutOfLineTree = false, bool kTies = true>
__device__ __forceinline__ uint32_t clearance(const DevLayout &L, double px, double py, Cands &C,
                                              int &hit, double &best, double bd = -1.0) {
    uint32_t st = 0;
    const double r2 = 2.0 * L.delta;
    // bd: the bounds distance, when the caller has it (kInside)
    best = kInside ? bd : fmin(fmin(px - L.bx0, L.bx1 - px), fmin(py - L.by0, L.by1 - py));
    hit = kNoHit;
    C.n = 0;
    C.first = -1;
    // outside the closed bounds no rect can contain p and p+-1 already
    // leaves the bounds: nothing to look up
    if (!kInside && !(px >= L.bx0 && py >= L.by0 && px <= L.bx1 && py <= L.by1)) return 0;
    if (L.cells) {
        int ix = (int)__dmul_rn(__dsub_rn(px, L.gx0), L.ginv);
        int iy = (int)__dmul_rn(__dsub_rn(py, L.gy0), L.ginv);
        ix = ix < 0 ? 0 : (ix >= L.gnx ? L.gnx - 1 : ix);
        iy = iy < 0 ? 0 : (iy >= L.gny ? L.gny - 1 : iy);
        const int2 ce = __ldg(L.cells + (int64_t)iy * L.gnx + ix);
        if (ce.y >= 0) {
            C.first = ce.x;
            C.n = ce.y;
#pragma unroll 2
            for (int k = ce.x; k < ce.x + ce.y; k++) {
                const float4 r = __ldg(L.crects + k);
                const double x0 = r.x, y0 = r.y, x1 = r.z, y1 = r.w;
                const double g = fmax(fmax(x0 - px, px - x1), fmax(y0 - py, py - y1));
                if (g <= 0.0) {  // each difference is <= 0 exactly when p is on that side
                    const int id = __ldg(L.cids + k);
                    hit = id < hit ? id : hit;
                }
                best = fmin(best, g);
            }
            return st;
        }
    }
    if (kOutOfLineTree)
        return tree_clearance_call<kTies>(L.nbox, L.nref, L.rects, L.ids, px, py, r2, L.slack, C, hit, best);
    return tree_clearance<kTies>(L.nbox, L.nref, L.rects, L.ids, px, py, r2, L.slack, C, hit, best);
}

__device__ __forceinline__ bool tree_box(const float4 *nbox, const int4 *nref, const float4 *rects,
                                         const double B[4], bool has_ign, const double ign[4], uint32_t &st);

// Tree::checkCollisions(box) restricted to the near-tie list (exact for the
// boxes of the replay, see the file comment).  Only boxes within delta of the
// clearance get here (rarely), so the listed rects are read back on demand
// rather than held in registers through the whole replay.
__device__ __forceinline__ bool collides_listed(const DevLayout &L, const Cands &C, const double o[4]) {
    if (!(o[1] >= L.by0 && o[0] >= L.bx0 && o[3] <= L.by1 && o[2] <= L.bx1)) return true;
    for (int q = 0; q < C.n; q++) {
        const float4 r = __ldg(C.first >= 0 ? L.crects + C.first + q : L.rects + C.idx[q]);
        if ((double)r.z >= o[0] && o[2] >= (double)r.x && (double)r.w >= o[1] && o[3] >= (double)r.y)
            return true;
    }
    return false;
}

// Decision of one box of the replay.  Its four extents (distances from p to
// its sides) lie within eps << delta of each other, so comparing one extent
// with the clearance d* settles every box farther than delta from d*: all
// extents above d* means the nearest obstacle (bounds side or listed rect) is
// touched; all below means nothing can be.  Only boxes within delta of d*
// take the exact predicate.  The extent is compared as a coordinate: the x1
// side against p.x + (d* +- delta), both rounded once per query -- a shift of
// the window by an ulp of p.x, far inside the 32x margin of delta over eps.
struct Window {
    double hi, lo;  // x1 beyond hi: collides; below lo: free
};

__device__ __forceinline__ Window replay_window(const DevLayout &L, double px, double dstar) {
    return Window{__dadd_rn(px, __dadd_rn(dstar, L.delta)), __dadd_rn(px, __dsub_rn(dstar, L.delta))};
}

// kTree: the near-tie list overflowed (C.first == -2) and the exact
// predicate is the whole tree's checkCollisions(box).
template <bool kTree>
__device__ __forceinline__ bool collides_box(const DevLayout &L, const Cands &C, const double o[4],
                                             const Window &W, uint32_t &st) {
    bool c = o[2] > W.hi;
    if (!c && !(o[2] < W.lo)) {  // rare: within delta of the clearance
        if (kTree)
            c = !(o[1] >= L.by0 && o[0] >= L.bx0 && o[3] <= L.by1 && o[2] <= L.bx1) ||
                tree_box(L.nbox, L.nref, L.rects, o, false, nullptr, st);
        else
            c = collides_listed(L, C, o);
    }
    return c;
}

// dist / 2 for the replay's step sizes (normal, positive, above MIN_DIST/2):
// one less in the exponent field is exactly the correctly rounded half, so
// the integer pipe does it.  A positive double's bit pattern orders like its
// value, so the MIN_DIST test is an integer compare too.
__device__ __forceinline__ double half_of(double d) {
    return __longlong_as_double(__double_as_longlong(d) - 0x0010000000000000ll);
}
__device__ __forceinline__ bool above_min(double d) {
    return __double_as_longlong(d) > __double_as_longlong(kMinDist);
}
// d when shrinking (the box collides), -d when growing: the sign bit set by
// an integer operation on the high word.
__device__ __forceinline__ double signed_step(double d, bool shrink) {
    const int hi = __double2hiint(d) ^ (shrink ? 0 : (int)0x80000000);
    return __hiloint2double(hi, __double2loint(d));
}

// drawBiggestSquareAtPoint replayed on scalars: same operations, same order,
// explicit round-to-nearest intrinsics (no contraction); the halvings as
// above.
template <bool kTree = false>
__device__ __forceinline__ uint32_t replay_square(const DevLayout &L, const Cands &C, double px,
                                                  double py, double dstar, double sq[4]) {
    const Window W = replay_window(L, px, dstar);
    uint32_t st = 0;
    double o[4] = {__dsub_rn(px, 1.0), __dsub_rn(py, 1.0), __dadd_rn(px, 1.0), __dadd_rn(py, 1.0)};
    if (collides_box<kTree>(L, C, o, W, st)) {
        sq[0] = o[0]; sq[1] = o[1]; sq[2] = o[2]; sq[3] = o[3];
        return st;
    }
    const double in2[4] = {__dsub_rn(px, 2.0), __dsub_rn(py, 2.0), __dadd_rn(px, 2.0),
                           __dadd_rn(py, 2.0)};
    if (collides_box<kTree>(L, C, in2, W, st)) {
        sq[0] = in2[0]; sq[1] = in2[1]; sq[2] = in2[2]; sq[3] = in2[3];
        return st;
    }
    double dist = L.dist0;
    // the loop's first box is p +- 1 again, already found free: its step (grow
    // by dist, no halving before the first collision) is taken directly
    o[0] = __dsub_rn(o[0], dist);
    o[1] = __dsub_rn(o[1], dist);
    o[2] = __dadd_rn(o[2], dist);
    o[3] = __dadd_rn(o[3], dist);
    int it = 1;
    // Growth (the reference's maxReached still false): grow by dist, without
    // halving, until a box collides.
    bool isc = collides_box<kTree>(L, C, o, W, st);
    while (!isc) {
        o[0] = __dsub_rn(o[0], dist);
        o[1] = __dsub_rn(o[1], dist);
        o[2] = __dadd_rn(o[2], dist);
        o[3] = __dadd_rn(o[3], dist);
        if (++it > kReplayCap) {
            st |= kStReplayCap;
            sq[0] = o[0]; sq[1] = o[1]; sq[2] = o[2]; sq[3] = o[3];
            return st;
        }
        isc = collides_box<kTree>(L, C, o, W, st);
    }
    // Bisection (maxReached): the loop runs while the box collides or dist is
    // above MIN_DIST; a colliding box shrinks by dist, halved first while above
    // MIN_DIST, a free one grows by half of dist.  While dist is above MIN_DIST
    // every step halves it whatever the collision, so those steps are the
    // first L.halvings of the loop, a count fixed by the layout (dist starts at
    // dist0 every query); each is one signed step -- x + (-d) rounds exactly as
    // x - d -- so a warp whose lanes disagree on the collision issues the four
    // updates once.  After them the loop shrinks by dist while the box
    // collides.
    if (it + L.halvings > kReplayCap) {  // the iteration bound falls inside the halvings
        st |= kStReplayCap;
        sq[0] = o[0]; sq[1] = o[1]; sq[2] = o[2]; sq[3] = o[3];
        return st;
    }
#pragma unroll 4
    for (int k = 0; k < L.halvings; k++) {
        dist = half_of(dist);
        const double sd = signed_step(dist, isc);
        o[0] = __dadd_rn(o[0], sd);
        o[1] = __dadd_rn(o[1], sd);
        o[2] = __dsub_rn(o[2], sd);
        o[3] = __dsub_rn(o[3], sd);
        isc = collides_box<kTree>(L, C, o, W, st);
    }
    while (isc) {
        o[0] = __dadd_rn(o[0], dist);
        o[1] = __dadd_rn(o[1], dist);
        o[2] = __dsub_rn(o[2], dist);
        o[3] = __dsub_rn(o[3], dist);
        if (++it > kReplayCap - L.halvings) {
            st |= kStReplayCap;
            break;
        }
        isc = collides_box<kTree>(L, C, o, W, st);
    }
    sq[0] = o[0]; sq[1] = o[1]; sq[2] = o[2]; sq[3] = o[3];
    return st;
}

// The replay against the whole tree, out of line: one call site per query,
// taken only by points with more near ties than the list holds.
struct ReplayOut {
    double sq[4];
    uint32_t st;
};
static __device__ __noinline__ ReplayOut replay_tree_call(const DevLayout L, double px, double py,
                                                          double dstar) {
    Cands C;
    C.n = 0;
    C.first = -2;
    ReplayOut r;
    r.st = replay_square<true>(L, C, px, py, dstar, r.sq);
    return r;
}

// drawBiggestSquareAtPoint + checkCollisons(point) for one point.  kTies:
// points with more near ties than the list holds take the whole-tree replay
// (else they report kStCandOverflow).
template <bool kInside = false, bool kOutOfLineTree = false, bool kTies = true>
__device__ __forceinline__ uint32_t query_point(const DevLayout &L, double px, double py, double sq[4],
                                                int &hit, double bd = -1.0) {
    Cands C;
    double best;
    uint32_t st = clearance<kInside, kOutOfLineTree, kTies>(L, px, py, C, hit, best, bd);
    if (kTies && C.first == -2) {
        const ReplayOut r = replay_tree_call(L, px, py, best);
        sq[0] = r.sq[0]; sq[1] = r.sq[1]; sq[2] = r.sq[2]; sq[3] = r.sq[3];
        st |= r.st;
    } else {
        st |= replay_square(L, C, px, py, best, sq);
    }
    return st;
}

// Tree::checkCollisions(box, ignore) for an arbitrary box (complete DFS).
__device__ __forceinline__ bool tree_box(const float4 *nbox, const int4 *nref, const float4 *rects,
                                         const double B[4], bool has_ign, const double ign[4], uint32_t &st) {
    int stk[kStackMax];
    int sp = 1;
    stk[0] = 0;
    while (sp > 0) {
        const int nd = stk[--sp];
        const int4 rf = __ldg(nref + nd);
        const int ref[4] = {rf.x, rf.y, rf.z, rf.w};
        for (int c = 0; c < 4; c++) {
            if (ref[c] == kRefEmpty) continue;
            const float4 b = __ldg(nbox + 4 * nd + c);
            if (!((double)b.z >= B[0] && B[2] >= (double)b.x && (double)b.w >= B[1] && B[3] >= (double)b.y))
                continue;
            if (ref[c] >= 0) {
                if (sp < kStackMax) stk[sp++] = ref[c];
                else st |= kStStackOverflow;
                continue;
            }
            const int f = leaf_first(ref[c]), m = leaf_count(ref[c]);
            for (int k = f; k < f + m; k++) {
                const float4 r = __ldg(rects + k);
                const double x0 = r.x, y0 = r.y, x1 = r.z, y1 = r.w;
                if (has_ign && x0 == ign[0] && y0 == ign[1] && x1 == ign[2] && y1 == ign[3]) continue;
                if (x1 >= B[0] && B[2] >= x0 && y1 >= B[1] && B[3] >= y0) return true;
            }
        }
    }
    return false;
}
__device__ __forceinline__ bool box_collides(const DevLayout &L, const double B[4], bool has_ign,
                                             const double ign[4], uint32_t &st) {
    if (!(B[1] >= L.by0 && B[0] >= L.bx0 && B[3] <= L.by1 && B[2] <= L.bx1)) return true;
    return tree_box(L.nbox, L.nref, L.rects, B, has_ign, ign, st);
}

// x / 200 for an integer-valued x in [0, 2^31), correctly rounded without the
// division sequence: q0 = x * RN(1/200), then one fused correction with the
// exact residual x - q0 * 200 (Markstein's quotient refinement).  Checked
// against IEEE division for every integer in the range.
static_assert(FRW_NSAMPLE == 200, "div200 is for the 200-bin perimeter");
__device__ __forceinline__ double div200(double x) {
    constexpr double r = 1.0 / 200.0;
    const double q0 = __dmul_rn(x, r);
    const double res = __fma_rn(-q0, 200.0, x);
    return __fma_rn(res, r, q0);
}

// RectHost::getPointFromNindex (CPU/rectHost.cpp:107-161; GPU twin
// Cuda/d_Rect.cu:34-101): branch structure and operand order kept because
// they decide ties; the perimeter is truncated to int unless `exact`.
__device__ __forceinline__ void point_from_index(const double s[4], int index, bool exact, double &ox,
                                                 double &oy) {
    const double per2 = __dadd_rn(__dmul_rn(2.0, __dsub_rn(s[2], s[0])), __dmul_rn(2.0, __dsub_rn(s[3], s[1])));
    const double perim = exact ? per2 : (double)__double2int_rz(per2);
    const double v = exact ? __ddiv_rn(perim, (double)FRW_NSAMPLE) : div200(perim);
    const double h = __dsub_rn(s[3], s[1]);
    const double w = __dsub_rn(s[2], s[0]);
    const double iv = __dmul_rn((double)index, v), jv = __dmul_rn((double)(index - 1), v);
    const double hv = __dmul_rn(v, 0.5);
    const double wh = __dadd_rn(w, h), w2h = __dadd_rn(__dmul_rn(2.0, w), h);
    if (iv < w) {
        ox = (double)__double2int_rz(__dadd_rn(__dadd_rn(jv, hv), s[0]));
        oy = s[1];
    } else if (jv < w && iv > w) {
        ox = s[2];
        oy = s[1];
    } else if (iv < wh) {
        ox = s[2];
        if (jv > w) oy = __dadd_rn(__dsub_rn(__dadd_rn(s[1], jv), w), hv);
        else {
            const double t = __dsub_rn(iv, w);
            oy = __dadd_rn(__dsub_rn(__dadd_rn(s[1], iv), w), __dmul_rn(t, 0.5));
        }
    } else if (jv < wh && iv > wh) {
        ox = s[2];
        oy = s[3];
    } else if (iv < w2h) {
        oy = s[3];
        if (jv > wh) ox = __dsub_rn(s[2], __dadd_rn(__dsub_rn(__dsub_rn(jv, w), h), hv));
        else {
            const double t = __dsub_rn(__dsub_rn(iv, w), h);
            ox = __dsub_rn(s[2], __dadd_rn(t, __dmul_rn(t, 0.5)));
        }
    } else if (jv < w2h && iv > w2h) {
        ox = s[0];
        oy = s[3];
    } else {
        ox = s[0];
        const double w2 = __dmul_rn(2.0, w);
        if (jv > w2h) oy = __dsub_rn(s[3], __dadd_rn(__dsub_rn(__dsub_rn(jv, w2), h), hv));
        else {
            const double t = __dsub_rn(__dsub_rn(iv, w2), h);
            oy = __dsub_rn(s[3], __dadd_rn(t, __dmul_rn(t, 0.5)));
        }
    }
}

// Uniform point on the Gaussian perimeter, clockwise from the top-left
// corner; side code 0 top, 1 right, 2 bottom, 3 left (outward normals
// (0,-1), (1,0), (0,1), (-1,0) in the layout's y-down axes).
__device__ __forceinline__ int perimeter_point(const double G[4], double u, double &x, double &y) {
    const double w = __dsub_rn(G[2], G[0]), h = __dsub_rn(G[3], G[1]);
    const double s = __dmul_rn(u, __dadd_rn(__dmul_rn(2.0, w), __dmul_rn(2.0, h)));
    if (s < w) {
        x = __dadd_rn(G[0], s);
        y = G[1];
        return 0;
    }
    if (s < __dadd_rn(w, h)) {
        x = G[2];
        y = __dadd_rn(G[1], __dsub_rn(s, w));
        return 1;
    }
    if (s < __dadd_rn(__dmul_rn(2.0, w), h)) {
        x = __dsub_rn(G[2], __dsub_rn(__dsub_rn(s, w), h));
        y = G[3];
        return 2;
    }
    x = G[0];
    y = __dsub_rn(G[3], __dsub_rn(__dsub_rn(s, __dmul_rn(2.0, w)), h));
    return 3;
}

}  // namespace frw
