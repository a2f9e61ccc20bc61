// cv_feat.cuh -- the control variate's input features of a first-hop point
// (shared by the feature, exact-mean and training kernels).
#pragma once

#include "query.cuh"

namespace frw {
namespace cv {

// ---------------------------------------------------------------- features
// d / a0 as d * (1 / a0) (one division per point), clamped to [-16, 16]
static __device__ __forceinline__ float feat(double d, double inv) {
    double v = __dmul_rn(d, inv);
    v = fmin(fmax(v, -16.0), 16.0);
    return (float)v;
}

// (dx, dy) from p to the nearest point of each edge of rect r: top, right,
// bottom, left (layout axes, y down).
static __device__ __forceinline__ void edge_feats(double px, double py, double x0, double y0, double x1, double y1,
                                           double a0, float *f) {
    const double cx = fmin(fmax(px, x0), x1), cy = fmin(fmax(py, y0), y1);
    const double dcx = __dsub_rn(cx, px), dcy = __dsub_rn(cy, py);
    const double inv = __ddiv_rn(1.0, a0);
    f[0] = feat(dcx, inv);
    f[1] = feat(__dsub_rn(y0, py), inv);
    f[2] = feat(__dsub_rn(x1, px), inv);
    f[3] = feat(dcy, inv);
    f[4] = f[0];
    f[5] = feat(__dsub_rn(y1, py), inv);
    f[6] = feat(__dsub_rn(x0, px), inv);
    f[7] = f[3];
}

// Nearest rect other than layer index `exclude` (smallest L-inf gap, then
// smallest layer index) from the tree; Morton position or -1.
static __device__ int nearest_other_tree(const DevLayout &L, double px, double py, int exclude) {
    const float pxf = (float)px, pyf = (float)py, slack = L.slack;
    double best = 1e300;
    int best_id = 0x7FFFFFFF, best_k = -1;
    float limf = 3.0e38f;
    int stk[kStackMax];
    int sp = 0, nd = 0;
    for (;;) {
        const float4 *bp = L.nbox + 4 * nd;
        const int4 rf = __ldg(L.nref + nd);
        const int ref[4] = {rf.x, rf.y, rf.z, rf.w};
        float lb[4];
#pragma unroll
        for (int c = 0; c < 4; c++) lb[c] = ref[c] == kRefEmpty ? 3.0e38f : lb_box_f(__ldg(bp + c), pxf, pyf);
#pragma unroll
        for (int c = 0; c < 4; c++) {
            if (ref[c] >= kRefEmpty || lb[c] > limf) continue;
            const int f0 = leaf_first(ref[c]), m = leaf_count(ref[c]);
            for (int k = f0; k < f0 + m; k++) {
                const float4 r = __ldg(L.rects + k);
                const float gf = fmaxf(fmaxf(r.x - pxf, pxf - r.z), fmaxf(r.y - pyf, pyf - r.w));
                if (gf > limf) continue;
                const int id = __ldg(L.ids + k);
                if (id == exclude) continue;
                const double g = fmax(fmax((double)r.x - px, px - (double)r.z), fmax((double)r.y - py, py - (double)r.w));
                if (g < best || (g == best && id < best_id)) {
                    best = g;
                    best_id = id;
                    best_k = k;
                    limf = (float)best + slack;
                }
            }
        }
        int next = -1;
        float nlb = 0.f;
#pragma unroll
        for (int c = 0; c < 4; c++) {
            if (ref[c] < 0 || lb[c] > limf) continue;
            int push = ref[c];
            if (next < 0 || lb[c] < nlb) {
                push = next;
                next = ref[c];
                nlb = lb[c];
            }
            if (push >= 0 && sp < kStackMax) stk[sp++] = push;
        }
        if (next >= 0) {
            nd = next;
            continue;
        }
        if (sp == 0) break;
        nd = stk[--sp];
    }
    return best_k;
}

// The same from p's cell list when it settles the answer: every rect within
// crad of p is listed, so a listed nearest other within crad is the nearest
// (ties included); otherwise the tree.  Writes the rect, false when none.
static __device__ __forceinline__ bool nearest_other(const DevLayout &L, double px, double py, int exclude, float4 &o) {
    if (L.cells && px >= L.bx0 && py >= L.by0 && px <= L.bx1 && py <= L.by1) {
        int ix = (int)__dmul_rn(__dsub_rn(px, L.gx0), L.ginv);
        int iy = (int)__dmul_rn(__dsub_rn(py, L.gy0), L.ginv);
        ix = ix < 0 ? 0 : (ix >= L.gnx ? L.gnx - 1 : ix);
        iy = iy < 0 ? 0 : (iy >= L.gny ? L.gny - 1 : iy);
        const int64_t cell = (int64_t)iy * L.gnx + ix;
        const int2 ce = __ldg(L.cells + cell);
        if (ce.y >= 0) {
            double best = 1e300;
            int best_id = 0x7FFFFFFF;
            float4 bo = make_float4(0.f, 0.f, 0.f, 0.f);
            for (int k = ce.x; k < ce.x + ce.y; k++) {
                const int id = __ldg(L.cids + k);
                if (id == exclude) continue;
                const float4 r = __ldg(L.crects + k);
                const double g =
                    fmax(fmax((double)r.x - px, px - (double)r.z), fmax((double)r.y - py, py - (double)r.w));
                if (g < best || (g == best && id < best_id)) {
                    best = g;
                    best_id = id;
                    bo = r;
                }
            }
            if (best <= (double)__ldg(L.crad + cell)) {
                o = bo;
                return true;
            }
        }
    }
    const int k = nearest_other_tree(L, px, py, exclude);
    if (k < 0) return false;
    o = __ldg(L.rects + k);
    return true;
}

}  // namespace cv
}  // namespace frw
