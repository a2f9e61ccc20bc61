// walk3d.cu -- 3-D floating random walk on box conductors: cell-grid build,
// clearance queries and the persistent walk kernel.
//
// The reference has no 3-D walk (its cube Green's function, green/green.cpp:
// 232-431, is never called); this is its 2-D walk (CPU/mainFunctions.cpp:
// 48-90) lifted to cubes, written for B200 the way the 2-D kernels are:
//   * the clearance query reads one cell record and a short list of box
//     copies (32 bytes each), sorted by distance from the cell centre so
//     the scan stops at the first entry that cannot be nearer -- no tree
//     descent and no stack;
//   * the cell lists are built on the device: boxes binned by overlap
//     (count -> scan -> fill), then for every cell a ring search for the
//     nearest box to its centre and a count -> scan -> fill of the boxes
//     within that distance plus a cell diagonal;
//   * the walk kernel is persistent (SM count x resident blocks); a warp
//     claims walks in chunks from one global counter and refills each idle
//     lane before every hop, so lanes stay busy while walks of very different
//     lengths finish;
//   * random numbers are Philox4x32-10 words keyed by (seed) with counter
//     (t / 4, walk, stream): the trajectory of a walk depends only on its
//     index, so the CPU oracle replays every walk bit for bit;
//   * the landing bin comes from a 2^14-entry guide in shared memory and the
//     32-bit CDF thresholds (L1-resident) -- one or two compares;
//   * FP64 geometry with explicitly rounded operations (no contraction):
//     exactly the oracle's arithmetic.
#include <math.h>

#include <algorithm>
#include <vector>

#include "frw3d_internal.h"

namespace frw {
namespace {

constexpr int kW3Threads = 256;
constexpr int kW3MinBlocks = 4;
constexpr unsigned kFull = 0xFFFFFFFFu;
constexpr uint64_t kW3Chunk = 128;  // walks a warp claims at a time
constexpr int64_t kMaxCells3 = int64_t(1) << 26;
constexpr int kMaxAxisCells3 = 1 << 14;

// ---- grid ------------------------------------------------------------------
struct Grid3 {
    double o[3];   // origin
    double side, inv, h, margin;
    int n[3];
    int cap;       // largest search radius in rings (the top level: no cap)
};

__device__ __forceinline__ int cell_axis(double v, double o, double inv, int n) {
    const double t = floor(__dmul_rn(__dsub_rn(v, o), inv));
    if (!(t >= 0.0)) return 0;
    if (t >= (double)n) return n - 1;
    return (int)t;
}

// L-infinity distance from p to the box (x0,y0,z0,x1,y1,z1): the largest
// per-axis gap, 0 inside.
__device__ __forceinline__ double box_dist(double px, double py, double pz, float4 lo, float4 hi) {
    double d = 0.0;
    d = fmax(d, __dsub_rn((double)lo.x, px));
    d = fmax(d, __dsub_rn(px, (double)hi.x));
    d = fmax(d, __dsub_rn((double)lo.y, py));
    d = fmax(d, __dsub_rn(py, (double)hi.y));
    d = fmax(d, __dsub_rn((double)lo.z, pz));
    d = fmax(d, __dsub_rn(pz, (double)hi.z));
    return d;
}

__device__ __forceinline__ void load_box(const float *__restrict__ boxes, int64_t i, float4 &lo, float4 &hi) {
    const float *b = boxes + 6 * i;
    lo = make_float4(__ldg(b), __ldg(b + 1), __ldg(b + 2), __int_as_float((int)i));
    hi = make_float4(__ldg(b + 3), __ldg(b + 4), __ldg(b + 5), 0.0f);
}

__global__ void k3_bin_count(const float *__restrict__ boxes, int64_t n, Grid3 G,
                             unsigned long long *__restrict__ cnt) {
    const int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= n) return;
    const float *b = boxes + 6 * i;
    int lo[3], hi[3];
    for (int c = 0; c < 3; c++) {
        lo[c] = cell_axis((double)b[c], G.o[c], G.inv, G.n[c]);
        hi[c] = cell_axis((double)b[3 + c], G.o[c], G.inv, G.n[c]);
    }
    for (int z = lo[2]; z <= hi[2]; z++)
        for (int y = lo[1]; y <= hi[1]; y++)
            for (int x = lo[0]; x <= hi[0]; x++)
                atomicAdd(cnt + ((int64_t)z * G.n[1] + y) * G.n[0] + x, 1ull);
}

__global__ void k3_bin_fill(const float *__restrict__ boxes, int64_t n, Grid3 G,
                            unsigned long long *__restrict__ cursor, int32_t *__restrict__ items) {
    const int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= n) return;
    const float *b = boxes + 6 * i;
    int lo[3], hi[3];
    for (int c = 0; c < 3; c++) {
        lo[c] = cell_axis((double)b[c], G.o[c], G.inv, G.n[c]);
        hi[c] = cell_axis((double)b[3 + c], G.o[c], G.inv, G.n[c]);
    }
    for (int z = lo[2]; z <= hi[2]; z++)
        for (int y = lo[1]; y <= hi[1]; y++)
            for (int x = lo[0]; x <= hi[0]; x++)
                items[atomicAdd(cursor + ((int64_t)z * G.n[1] + y) * G.n[0] + x, 1ull)] = (int32_t)i;
}

// Visits the cells of Chebyshev ring r around (cx, cy, cz) inside the grid:
// the full x range on the ring's z and y faces, else its two x ends.
template <class F>
__device__ __forceinline__ void for_ring(const Grid3 &G, int cx, int cy, int cz, int r, F &&f) {
    const int z0 = max(cz - r, 0), z1 = min(cz + r, G.n[2] - 1);
    const int y0 = max(cy - r, 0), y1 = min(cy + r, G.n[1] - 1);
    const int x0 = max(cx - r, 0), x1 = min(cx + r, G.n[0] - 1);
    for (int z = z0; z <= z1; z++)
        for (int y = y0; y <= y1; y++) {
            const int64_t row = ((int64_t)z * G.n[1] + y) * G.n[0];
            if (z == cz - r || z == cz + r || y == cy - r || y == cy + r) {
                for (int x = x0; x <= x1; x++) f(row + x);
            } else {
                if (cx - r >= 0) f(row + cx - r);
                if (r > 0 && cx + r < G.n[0]) f(row + cx + r);
            }
        }
}

// List entries (pairs of float4) ordered by (d_c in hi.w, box index in lo.w).
__device__ __forceinline__ bool entry_less(const float4 *e, int64_t a, int64_t b) {
    const float ka = e[2 * a + 1].w, kb = e[2 * b + 1].w;
    return ka < kb || (ka == kb && __float_as_int(e[2 * a].w) < __float_as_int(e[2 * b].w));
}
__device__ __forceinline__ void entry_swap(float4 *e, int64_t a, int64_t b) {
    const float4 lo = e[2 * a], hi = e[2 * a + 1];
    e[2 * a] = e[2 * b];
    e[2 * a + 1] = e[2 * b + 1];
    e[2 * b] = lo;
    e[2 * b + 1] = hi;
}
__device__ __forceinline__ void sift_down(float4 *e, int64_t root, int64_t end) {
    for (int64_t c = 2 * root + 1; c < end; c = 2 * root + 1) {
        if (c + 1 < end && entry_less(e, c, c + 1)) c++;
        if (!entry_less(e, root, c)) return;
        entry_swap(e, root, c);
        root = c;
    }
}
// One thread's list, in place: insertion for short lists (the usual case),
// heapsort for the long ones of coarse cells facing a dense cluster.
__device__ void sort_entries(float4 *e, int64_t m) {
    if (m <= 32) {
        for (int64_t a = 1; a < m; a++)
            for (int64_t b = a; b > 0 && entry_less(e, b, b - 1); b--) entry_swap(e, b, b - 1);
        return;
    }
    for (int64_t r = m / 2 - 1; r >= 0; r--) sift_down(e, r, m);
    for (int64_t end = m - 1; end > 0; end--) {
        entry_swap(e, 0, end);
        sift_down(e, 0, end);
    }
}

// Per cell: the nearest-box distance D of its centre (ring search over the
// bins: boxes in ring r are at least (2r - 1) h away), then every box within
// R = D + 2h + margin, each counted once (in the first cell, in index order,
// where its cell range meets the search cube) -- counted (kFill = false) or
// written (kFill = true).  A cell whose search needs more than G.cap rings
// defers (flag 1) and marks its parent cell of the next level as needed;
// cells outside `need` (when given) are unused (flag 2).
template <bool kFill>
__global__ void k3_cell_lists(const float *__restrict__ boxes, Grid3 G, const int64_t *__restrict__ bstart,
                              const int32_t *__restrict__ items, int64_t ncells, const uint8_t *__restrict__ need,
                              uint8_t *__restrict__ flag, uint8_t *__restrict__ need_up, int upnx, int upny,
                              unsigned long long *__restrict__ ndefer, int64_t *__restrict__ cnt,
                              const int64_t *__restrict__ lstart, float4 *__restrict__ lists) {
    const int64_t c = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (c >= ncells) return;
    if (kFill) {
        if (flag[c]) return;
    } else if (need && !need[c]) {
        cnt[c] = 0;
        flag[c] = 2;
        return;
    }
    const int cx = (int)(c % G.n[0]), cy = (int)((c / G.n[0]) % G.n[1]), cz = (int)(c / ((int64_t)G.n[0] * G.n[1]));
    const double px = __dadd_rn(G.o[0], __dmul_rn((double)cx + 0.5, G.side));
    const double py = __dadd_rn(G.o[1], __dmul_rn((double)cy + 0.5, G.side));
    const double pz = __dadd_rn(G.o[2], __dmul_rn((double)cz + 0.5, G.side));
    const int rlim = max(G.n[0], max(G.n[1], G.n[2]));
    double best = INFINITY;
    bool defer = false;
    for (int r = 0; r <= rlim; r++) {
        if (r > 0 && __dmul_rn((double)(2 * r - 1), G.h) > __dadd_rn(best, G.margin)) break;
        if (r > G.cap) {
            defer = true;
            break;
        }
        for_ring(G, cx, cy, cz, r, [&](int64_t q) {
            for (int64_t k = bstart[q]; k < bstart[q + 1]; k++) {
                float4 lo, hi;
                load_box(boxes, items[k], lo, hi);
                best = fmin(best, box_dist(px, py, pz, lo, hi));
            }
        });
    }
    const double R = __dadd_rn(__dadd_rn(best, __dmul_rn(2.0, G.h)), G.margin);
    int rmax = 0;
    if (!defer) {
        while (rmax < rlim && __dmul_rn((double)(2 * rmax + 1), G.h) <= R) rmax++;
        defer = rmax > G.cap;
    }
    if (defer) {  // only the counting pass gets here: the fill skips flagged cells
        if (!kFill) {
            cnt[c] = 0;
            flag[c] = 1;
            atomicAdd(ndefer, 1ull);
            if (need_up) need_up[((int64_t)(cz >> 1) * upny + (cy >> 1)) * upnx + (cx >> 1)] = 1;
        }
        return;
    }
    const int s0[3] = {max(cx - rmax, 0), max(cy - rmax, 0), max(cz - rmax, 0)};
    const int s1[3] = {min(cx + rmax, G.n[0] - 1), min(cy + rmax, G.n[1] - 1), min(cz + rmax, G.n[2] - 1)};
    int64_t m = 0, out = kFill ? lstart[c] : 0;
    for (int z = s0[2]; z <= s1[2]; z++)
        for (int y = s0[1]; y <= s1[1]; y++)
            for (int x = s0[0]; x <= s1[0]; x++) {
                const int64_t q = ((int64_t)z * G.n[1] + y) * G.n[0] + x;
                for (int64_t k = bstart[q]; k < bstart[q + 1]; k++) {
                    const int32_t i = items[k];
                    float4 lo, hi;
                    load_box(boxes, i, lo, hi);
                    // the box's first cell inside the search cube
                    const int fx = max(cell_axis((double)lo.x, G.o[0], G.inv, G.n[0]), s0[0]);
                    const int fy = max(cell_axis((double)lo.y, G.o[1], G.inv, G.n[1]), s0[1]);
                    const int fz = max(cell_axis((double)lo.z, G.o[2], G.inv, G.n[2]), s0[2]);
                    if (fx != x || fy != y || fz != z) continue;
                    if (box_dist(px, py, pz, lo, hi) > R) continue;
                    if (kFill) {
                        hi.w = __double2float_rd(box_dist(px, py, pz, lo, hi));
                        lists[2 * (out + m)] = lo;
                        lists[2 * (out + m) + 1] = hi;
                    }
                    m++;
                }
            }
    // order by (distance from the centre, index): a query stops at the first
    // entry that cannot win
    if (kFill) sort_entries(lists + 2 * out, m);
    if (!kFill) {
        cnt[c] = m;
        flag[c] = 0;
    }
}

__global__ void k3_cells_pack(const int64_t *__restrict__ lstart, const int64_t *__restrict__ cnt,
                              const uint8_t *__restrict__ flag, int64_t ncells, uint2 *__restrict__ cells,
                              unsigned long long *__restrict__ maxlen) {
    const int64_t c = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (c >= ncells) return;
    if (flag[c]) {
        cells[c] = make_uint2(0u, kDefer3);
        return;
    }
    cells[c] = make_uint2((uint32_t)lstart[c], (uint32_t)cnt[c]);
    atomicMax(maxlen, (unsigned long long)cnt[c]);
}

// ---- query -----------------------------------------------------------------
__device__ __forceinline__ void nearest3(const Dev3Layout &L, double px, double py, double pz, double &best,
                                         int &bid) {
    const int ix = cell_axis(px, L.g0x, L.ginv, L.nx);
    const int iy = cell_axis(py, L.g0y, L.ginv, L.ny);
    const int iz = cell_axis(pz, L.g0z, L.ginv, L.nz);
    uint2 cr = __ldg(L.cells + ((int64_t)iz * L.ny + iy) * L.nx + ix);
    const float4 *e = L.lists;
    double hq = L.hq;
    if (cr.y == kDefer3) {  // far from every box: the coarser levels
        for (int l = 0; l < L.nup && cr.y == kDefer3; l++) {
            const Level3 *V = L.up + l;
            const double gi = __ldg(&V->ginv);
            const int nx = __ldg(&V->nx), ny = __ldg(&V->ny), nz = __ldg(&V->nz);
            const int jx = cell_axis(px, L.g0x, gi, nx), jy = cell_axis(py, L.g0y, gi, ny),
                      jz = cell_axis(pz, L.g0z, gi, nz);
            const uint2 *cells = (const uint2 *)__ldg((const unsigned long long *)&V->cells);
            cr = __ldg(cells + ((int64_t)jz * ny + jy) * nx + jx);
            e = (const float4 *)__ldg((const unsigned long long *)&V->lists);
            hq = __ldg(&V->hq);
        }
        if (cr.y == kDefer3) {  // cannot happen by construction; reported, never looped on
            atomicOr(L.status, kSt3LevelChain);
            cr.y = 0;
        }
    }
    best = INFINITY;
    bid = 0x7FFFFFFF;
    e += 2 * (size_t)cr.x;
    for (uint32_t k = 0; k < cr.y; k++) {
        const float4 lo = __ldg(e + 2 * k), hi = __ldg(e + 2 * k + 1);
        // hi.w <= the entry's distance from the cell centre and the point is
        // within hq of that centre: this entry and every later one are
        // farther than the best so far
        if (__dsub_rn((double)hi.w, hq) > best) break;
        const double d = box_dist(px, py, pz, lo, hi);
        const int id = __float_as_int(lo.w);
        if (d < best || (d == best && id < bid)) {
            best = d;
            bid = id;
        }
    }
}

__global__ void k3_query(const Dev3Layout L, const double *__restrict__ pts, int64_t n, double *__restrict__ clear,
                         int64_t *__restrict__ nearest) {
    const int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= n) return;
    double d;
    int id;
    nearest3(L, pts[3 * i], pts[3 * i + 1], pts[3 * i + 2], d, id);
    if (clear) clear[i] = d;
    if (nearest) nearest[i] = id;
}

// ---- walk ------------------------------------------------------------------
__device__ __forceinline__ uint4 philox4x32_10(uint4 c, uint2 k) {
#pragma unroll
    for (int r = 0; r < 10; r++) {
        if (r) {
            k.x += 0x9E3779B9u;
            k.y += 0xBB67AE85u;
        }
        const uint32_t hi0 = __umulhi(0xD2511F53u, c.x), lo0 = 0xD2511F53u * c.x;
        const uint32_t hi1 = __umulhi(0xCD9E8D57u, c.z), lo1 = 0xCD9E8D57u * c.z;
        c = make_uint4(hi1 ^ c.y ^ k.x, lo1, hi0 ^ c.w ^ k.y, lo0);
    }
    return c;
}

__device__ __forceinline__ uint4 block3(const Walk3Params &P, uint64_t walk, uint32_t blk) {
    return philox4x32_10(make_uint4(blk, (uint32_t)walk, (uint32_t)(walk >> 32), P.stream),
                         make_uint2((uint32_t)P.seed, (uint32_t)(P.seed >> 32)));
}

__device__ __forceinline__ uint32_t word_of(const uint4 &b, uint32_t t) {
    const uint32_t k = t & 3;
    return k == 0 ? b.x : (k == 1 ? b.y : (k == 2 ? b.z : b.w));
}

struct Walker {
    double px, py, pz;
    double a0, sgn;
    uint4 rnd;
    uint64_t idx;  // walk index relative to P.first
    uint32_t rblk;
    int hops, b1, axis;
    int job;       // batched runs: the walk's job
};

// Start point on the Gaussian box: faces z0, z1, y0, y1, x0, x1 by area from
// u0 (its remainder places the first coordinate), u1 the second.
template <bool kMulti>
__device__ __forceinline__ void start_walk(const Walk3Params &P, Walker &W, uint64_t j) {
    const double *G = P.G;
    double S = P.S;
    if (kMulti) {  // walk j of the batch is walk j % walks_per_job of job j / walks_per_job
        const uint64_t q = j / P.walks_per_job;
        W.job = (int)q;
        j -= q * P.walks_per_job;
        G = P.jobs[q].G;
        S = __ldg(&P.jobs[q].S);
    }
    W.idx = j;
    W.rnd = block3(P, P.first + j, 0);
    W.rblk = 0;
    double u0 = (double)W.rnd.x * 0x1p-32;
    const double u1 = (double)W.rnd.y * 0x1p-32;
    if (P.start_strata)  // stratum (walk mod S) of the surface, by the first uniform
        u0 = __ddiv_rn(__dadd_rn((double)(uint32_t)((P.first + j) % P.start_strata), u0), (double)P.start_strata);
    const double w = __dsub_rn(G[3], G[0]), h = __dsub_rn(G[4], G[1]), d = __dsub_rn(G[5], G[2]);
    const double axy = __dmul_rn(w, h), axz = __dmul_rn(w, d), ayz = __dmul_rn(h, d);
    double s = __dmul_rn(u0, S);
    int f = 0;
    double a = axy;
    for (; f < 5; f++) {
        a = f < 2 ? axy : (f < 4 ? axz : ayz);
        if (s < a) break;
        s = __dsub_rn(s, a);
    }
    if (f == 5) a = ayz;
    double t = __ddiv_rn(s, a);
    if (t > 1.0) t = 1.0;
    const int hi = f & 1;
    if ((f >> 1) == 0) {
        W.px = __dadd_rn(G[0], __dmul_rn(t, w));
        W.py = __dadd_rn(G[1], __dmul_rn(u1, h));
        W.pz = hi ? G[5] : G[2];
        W.axis = 2;
    } else if ((f >> 1) == 1) {
        W.px = __dadd_rn(G[0], __dmul_rn(t, w));
        W.py = hi ? G[4] : G[1];
        W.pz = __dadd_rn(G[2], __dmul_rn(u1, d));
        W.axis = 1;
    } else {
        W.px = hi ? G[3] : G[0];
        W.py = __dadd_rn(G[1], __dmul_rn(t, h));
        W.pz = __dadd_rn(G[2], __dmul_rn(u1, d));
        W.axis = 0;
    }
    W.sgn = hi ? 1.0 : -1.0;
    W.hops = 0;
    W.b1 = -1;
    W.a0 = 0.0;
}

// Landing on the cube of half-side h at the centre of bin b (face k, row i,
// column j): offsets o_i = (2 i + 1 - n) / n half-sides from the face centre.
__device__ __forceinline__ void land(const Walk3Params &P, const double *s_offs, Walker &W, int b, double h) {
    // b / n^2 and r / n as multiply-highs by ceil(2^32 / d): exact for every
    // b < 6 n^2, n <= 100 (checked exhaustively); n = 1 has no division
    int k = b, r = 0, i = 0, j = 0;
    if (P.n > 1) {
        k = (int)__umulhi((unsigned)b, P.magic_nn);
        r = b - k * P.n * P.n;
        i = (int)__umulhi((unsigned)r, P.magic_n);
        j = r - i * P.n;
    }
    const double hi_ = __dmul_rn(h, s_offs[i]), hj = __dmul_rn(h, s_offs[j]);
    const double x = W.px, y = W.py, z = W.pz;
    switch (k) {
    case 0: W.px = __dadd_rn(x, hi_); W.py = __dadd_rn(y, hj); W.pz = __dsub_rn(z, h); break;
    case 1: W.px = __dadd_rn(x, h); W.py = __dadd_rn(y, hi_); W.pz = __dadd_rn(z, hj); break;
    case 2: W.px = __dsub_rn(x, hj); W.py = __dadd_rn(y, h); W.pz = __dadd_rn(z, hi_); break;
    case 3: W.px = __dsub_rn(x, hi_); W.py = __dsub_rn(y, hj); W.pz = __dadd_rn(z, h); break;
    case 4: W.px = __dsub_rn(x, h); W.py = __dsub_rn(y, hi_); W.pz = __dsub_rn(z, hj); break;
    default: W.px = __dadd_rn(x, hj); W.py = __dsub_rn(y, h); W.pz = __dsub_rn(z, hi_); break;
    }
}

// kMulti: a batch of targets of one layout (jobs); every lane keeps its
// sums for one job at a time and flushes them when it starts a walk of
// another job (jobs are contiguous walk ranges, so that is rare).
template <bool kMulti>
__device__ __forceinline__ void flush_job(const Walk3Params &P, int job, unsigned long long &tn, double &ts,
                                          double &ts2, unsigned long long &n_esc, unsigned long long &n_ab,
                                          unsigned long long &n_hops, unsigned long long &n_done) {
    if (!kMulti || job < 0) return;
    const int64_t t = __ldg(&P.jobs[job].target), row = (int64_t)job * P.nboxes + t;
    if (tn) {
        atomicAdd(P.hits + row, tn);
        atomicAdd(P.sum_w + row, ts);
        atomicAdd(P.sum_w2 + row, ts2);
    }
    unsigned long long *st = P.stats + 4 * (int64_t)job;
    if (n_esc) atomicAdd(st + 0, n_esc);
    if (n_ab) atomicAdd(st + 1, n_ab);
    if (n_done) {
        atomicAdd(st + 2, n_hops);
        atomicAdd(st + 3, n_done);
    }
    tn = n_esc = n_ab = n_hops = n_done = 0;
    ts = ts2 = 0.0;
}

template <bool kMulti>
__global__ void __launch_bounds__(kW3Threads, kW3MinBlocks) k_walk3(const Walk3Params P) {
    __shared__ uint16_t s_guide[1 << kGuide3Bits];
    __shared__ double s_offs[FRW3_NSAMPLE_MAX];
    for (int k = threadIdx.x; k < (1 << kGuide3Bits); k += blockDim.x) s_guide[k] = P.guide[k];
    for (int k = threadIdx.x; k < P.n; k += blockDim.x) s_offs[k] = P.offs[k];
    __syncthreads();

    const int lane = threadIdx.x & 31;
    const unsigned lt = (1u << lane) - 1u;
    const bool trace = P.rec_end || P.rec_hops || P.rec_bin || P.rec_w;
    Walker W;
    bool active = false;
    unsigned long long tn = 0, n_esc = 0, n_ab = 0, n_hops = 0, n_done = 0;
    double ts = 0.0, ts2 = 0.0;
    uint64_t next = 0, cend = 0;
    bool exhausted = false;
    int acc_job = -1;  // batched runs: the job the lane's sums belong to

    for (;;) {
        // refill idle lanes from the warp's chunk, claiming chunks as needed
        unsigned idle = __ballot_sync(kFull, !active);
        // refill only once refill_min lanes are idle (or none is walking):
        // fewer divergent starts, at the price of lanes idling meanwhile
        if (__popc(idle) < (unsigned)P.refill_min && idle != kFull) idle = 0;
        while (idle && !exhausted) {
            if (next >= cend) {
                unsigned long long base = 0;
                if (lane == 0) base = atomicAdd(P.counter, (unsigned long long)kW3Chunk);
                base = __shfl_sync(kFull, base, 0);
                if (base >= P.walks) {
                    exhausted = true;
                    break;
                }
                next = (uint64_t)base;
                cend = next + kW3Chunk < P.walks ? next + kW3Chunk : P.walks;
            }
            const uint64_t avail = cend - next;
            const unsigned rank = __popc(idle & lt);
            if (!active && rank < avail) {
                start_walk<kMulti>(P, W, next + rank);
                if (kMulti && W.job != acc_job) {
                    flush_job<kMulti>(P, acc_job, tn, ts, ts2, n_esc, n_ab, n_hops, n_done);
                    acc_job = W.job;
                }
                active = true;
            }
            next += (uint64_t)__popc(idle) < avail ? (uint64_t)__popc(idle) : avail;
            idle = __ballot_sync(kFull, !active);
        }
        if (__ballot_sync(kFull, active) == 0) break;
        if (!active) continue;

        // up to two hops per round of refills and walk ends
        int64_t end = -3;  // still walking
        for (int pass = 0; pass < 2; pass++) {
            double d = 0.0;
            if (!(W.px > P.L.b[0] && W.py > P.L.b[1] && W.pz > P.L.b[2] && W.px < P.L.b[3] && W.py < P.L.b[4] &&
                  W.pz < P.L.b[5])) {
                end = -1;
            } else {
                int id;
                nearest3(P.L, W.px, W.py, W.pz, d, id);
                W.hops++;
                if (d <= P.shell) end = id;
                else if (W.hops >= P.hop_cap) end = -2;
            }
            if (end != -3) break;
            const uint32_t t = (uint32_t)W.hops + 1;
            if ((t >> 2) != W.rblk) {
                W.rblk = t >> 2;
                W.rnd = block3(P, P.first + W.idx, W.rblk);
            }
            const uint32_t x = word_of(W.rnd, t);
            int b = s_guide[x >> (32 - kGuide3Bits)];
            while (b + 1 < P.nb && __ldg(P.thr + b + 1) <= x) b++;
            land(P, s_offs, W, b, d);
            if (W.hops == 1) {
                W.b1 = b;
                W.a0 = __dmul_rn(2.0, d);
            }
        }
        if (end == -3) continue;
        // the walk ended
        double c = 0.0;
        const double S = kMulti ? __ldg(&P.jobs[W.job].S) : P.S;
        const int64_t target = kMulti ? __ldg(&P.jobs[W.job].target) : P.target;
        if (W.b1 >= 0) {
            const double wv = __ldg(P.w + 3 * W.b1 + W.axis);
            c = __ddiv_rn(__dmul_rn(__dmul_rn(P.perm, S), __dmul_rn(W.sgn, wv)), W.a0);
        }
        if (kMulti) {
            if (end == target) {
                tn++;
                ts = __dadd_rn(ts, c);
                ts2 = __dadd_rn(ts2, __dmul_rn(c, c));
            } else if (end >= 0) {
                const int64_t row = (int64_t)W.job * P.nboxes + end;
                atomicAdd(P.hits + row, 1ull);
                atomicAdd(P.sum_w + row, c);
                atomicAdd(P.sum_w2 + row, __dmul_rn(c, c));
            }
        } else if (trace) {
            if (P.rec_end) P.rec_end[W.idx] = end;
            if (P.rec_hops) P.rec_hops[W.idx] = W.hops;
            if (P.rec_bin) P.rec_bin[W.idx] = W.b1;
            if (P.rec_w) P.rec_w[W.idx] = c;
        } else if (end == P.target) {
            tn++;
            ts = __dadd_rn(ts, c);
            ts2 = __dadd_rn(ts2, __dmul_rn(c, c));
        } else if (end >= 0) {
            atomicAdd(P.hits + end, 1ull);
            atomicAdd(P.sum_w + end, c);
            atomicAdd(P.sum_w2 + end, __dmul_rn(c, c));
        }
        if (end == -1) n_esc++;
        else if (end == -2) n_ab++;
        n_hops += (unsigned long long)W.hops;
        n_done++;
        active = false;
    }

    if (kMulti) {  // every lane flushes its last job's sums
        flush_job<kMulti>(P, acc_job, tn, ts, ts2, n_esc, n_ab, n_hops, n_done);
        return;
    }
    // warp totals -> global rows
#pragma unroll
    for (int o = 16; o; o >>= 1) {
        tn += __shfl_xor_sync(kFull, tn, o);
        ts += __shfl_xor_sync(kFull, ts, o);
        ts2 += __shfl_xor_sync(kFull, ts2, o);
        n_esc += __shfl_xor_sync(kFull, n_esc, o);
        n_ab += __shfl_xor_sync(kFull, n_ab, o);
        n_hops += __shfl_xor_sync(kFull, n_hops, o);
        n_done += __shfl_xor_sync(kFull, n_done, o);
    }
    if (lane == 0) {
        if (!trace && tn) {
            atomicAdd(P.hits + P.target, tn);
            atomicAdd(P.sum_w + P.target, ts);
            atomicAdd(P.sum_w2 + P.target, ts2);
        }
        if (P.stats) {
            atomicAdd(P.stats + 0, n_esc);
            atomicAdd(P.stats + 1, n_ab);
            atomicAdd(P.stats + 2, n_hops);
            atomicAdd(P.stats + 3, n_done);
        }
    }
}

}  // namespace

void free_grid3(Grid3Buffers *g, cudaStream_t st) {
    if (g->cells) cudaFreeAsync(g->cells, st);
    if (g->lists) cudaFreeAsync(g->lists, st);
    for (int l = 0; l < kMaxLevels3; l++) {
        if (g->up_cells[l]) cudaFreeAsync(g->up_cells[l], st);
        if (g->up_lists[l]) cudaFreeAsync(g->up_lists[l], st);
    }
    if (g->up) cudaFreeAsync(g->up, st);
    if (g->status) cudaFreeAsync(g->status, st);
    *g = Grid3Buffers();
}

void attach_grid3(Dev3Layout &L, const Grid3Buffers &g, const double bounds[6]) {
    L.cells = g.cells;
    L.lists = g.lists;
    L.g0x = g.g0[0];
    L.g0y = g.g0[1];
    L.g0z = g.g0[2];
    L.ginv = 1.0 / g.side;
    L.hq = 0.5 * g.side + 2.0 * g.margin;
    L.nx = g.nx;
    L.ny = g.ny;
    L.nz = g.nz;
    L.nup = g.nup;
    L.up = g.up;
    L.status = g.status;
    for (int c = 0; c < 6; c++) L.b[c] = bounds[c];
}

namespace {

// One level: bins, the count pass (lists, deferrals, the parents' needs),
// the scan, the fill pass and the cell records.  need == nullptr: every cell.
struct LevelOut {
    uint2 *cells = nullptr;
    float4 *lists = nullptr;
    int64_t entries = 0, deferred = 0;
    unsigned long long max_list = 0;
};

frw_status build_level(const float *d_boxes, int64_t n, const Grid3 &G, const uint8_t *need, uint8_t *need_up,
                       int upnx, int upny, cudaStream_t st, LevelOut *out) {
    const int64_t ncells = (int64_t)G.n[0] * G.n[1] * G.n[2];
    int64_t *bcnt = nullptr, *bstart = nullptr, *lcnt = nullptr, *lstart = nullptr, *sums = nullptr,
            *grand = nullptr;
    int32_t *items = nullptr;
    uint8_t *flag = nullptr;
    unsigned long long *dev_stats = nullptr;  // [0] deferred cells, [1] longest list
    const int64_t tiles = scan_i64_tiles(ncells + 1);
    frw_status rc = FRW_OK;
    auto ck = [&](cudaError_t e, const char *what) {
        if (e != cudaSuccess && rc == FRW_OK) rc = cuda_fail(e, what);
        return rc == FRW_OK;
    };
    do {
        const size_t cb = (size_t)(ncells + 1) * 8;
        if (!ck(cudaMallocAsync(&bcnt, cb, st), "malloc bin counts")) break;
        if (!ck(cudaMallocAsync(&bstart, cb, st), "malloc bin starts")) break;
        if (!ck(cudaMallocAsync(&lcnt, cb, st), "malloc list counts")) break;
        if (!ck(cudaMallocAsync(&lstart, cb, st), "malloc list starts")) break;
        if (!ck(cudaMallocAsync(&sums, (size_t)tiles * 8, st), "malloc tile sums")) break;
        if (!ck(cudaMallocAsync(&grand, 16, st), "malloc totals")) break;
        if (!ck(cudaMallocAsync(&flag, (size_t)ncells, st), "malloc flags")) break;
        if (!ck(cudaMallocAsync(&dev_stats, 16, st), "malloc stats")) break;
        if (!ck(cudaMallocAsync(&out->cells, (size_t)ncells * sizeof(uint2), st), "malloc cells")) break;
        if (!ck(cudaMemsetAsync(bcnt, 0, cb, st), "memset")) break;
        if (!ck(cudaMemsetAsync(lcnt, 0, cb, st), "memset")) break;
        if (!ck(cudaMemsetAsync(dev_stats, 0, 16, st), "memset")) break;
        const unsigned nb = (unsigned)((n + 255) / 256);
        k3_bin_count<<<nb, 256, 0, st>>>(d_boxes, n, G, (unsigned long long *)bcnt);
        launch_scan_i64(bcnt, ncells + 1, bstart, sums, grand, st);
        if (!ck(cudaGetLastError(), "bin count")) break;
        int64_t nitems = 0;
        if ((rc = read_back(&nitems, grand, 8, st, "build_grid3: bin total"))) break;
        if (nitems > INT32_MAX) {
            set_error("build_grid3: more than 2^31 bin entries; use fewer cells per box");
            rc = FRW_E_ARG;
            break;
        }
        if (!ck(cudaMallocAsync(&items, (size_t)std::max<int64_t>(nitems, 1) * 4, st), "malloc bins")) break;
        // the fill uses bcnt as its cursor: start it at the bin starts
        if (!ck(cudaMemcpyAsync(bcnt, bstart, cb, cudaMemcpyDeviceToDevice, st), "cursor")) break;
        k3_bin_fill<<<nb, 256, 0, st>>>(d_boxes, n, G, (unsigned long long *)bcnt, items);
        const unsigned cbk = (unsigned)((ncells + 127) / 128);
        k3_cell_lists<false><<<cbk, 128, 0, st>>>(d_boxes, G, bstart, items, ncells, need, flag, need_up, upnx, upny,
                                                  dev_stats, lcnt, nullptr, nullptr);
        launch_scan_i64(lcnt, ncells + 1, lstart, sums, grand + 1, st);
        if (!ck(cudaGetLastError(), "cell count")) break;
        int64_t total = 0;
        unsigned long long ndef = 0;
        if ((rc = read_back(&total, grand + 1, 8, st, "build_grid3: list total"))) break;
        if ((rc = read_back(&ndef, dev_stats, 8, st, "build_grid3: deferred cells"))) break;
        if (total > (int64_t)INT32_MAX) {
            set_error("build_grid3: more than 2^31 list entries; use fewer cells per box");
            rc = FRW_E_ARG;
            break;
        }
        out->entries = total;
        out->deferred = (int64_t)ndef;
        if (!ck(cudaMallocAsync(&out->lists, (size_t)std::max<int64_t>(total, 1) * 32, st), "malloc lists")) break;
        k3_cell_lists<true><<<cbk, 128, 0, st>>>(d_boxes, G, bstart, items, ncells, need, flag, nullptr, upnx, upny,
                                                 nullptr, nullptr, lstart, out->lists);
        k3_cells_pack<<<cbk, 128, 0, st>>>(lstart, lcnt, flag, ncells, out->cells, dev_stats + 1);
        if (!ck(cudaGetLastError(), "cell fill")) break;
        if ((rc = read_back(&out->max_list, dev_stats + 1, 8, st, "build_grid3: longest list"))) break;
    } while (0);
    for (void *p : {(void *)bcnt, (void *)bstart, (void *)lcnt, (void *)lstart, (void *)sums, (void *)grand,
                    (void *)items, (void *)flag, (void *)dev_stats})
        if (p) cudaFreeAsync(p, st);
    if (rc != FRW_OK) {
        if (out->cells) cudaFreeAsync(out->cells, st);
        if (out->lists) cudaFreeAsync(out->lists, st);
        *out = LevelOut();
    }
    return rc;
}

}  // namespace

frw_status build_grid3(const float *d_boxes, int64_t n, const double bounds[6], double cells_per_box,
                       cudaStream_t st, Grid3Buffers *out) {
    *out = Grid3Buffers();
    if (!(cells_per_box > 0) || n < 1 || n > INT32_MAX) {
        set_error("build_grid3: cells_per_box must be > 0 and 1 <= n < 2^31");
        return FRW_E_ARG;
    }
    double ext[3], vol = 1.0, M = 16.0;
    for (int c = 0; c < 3; c++) {
        ext[c] = bounds[3 + c] - bounds[c];
        vol *= ext[c];
        M = std::max(M, 4.0 * std::max(std::max(std::fabs(bounds[c]), std::fabs(bounds[3 + c])), ext[c]));
    }
    const double target = std::min((double)kMaxCells3, std::max(1.0, cells_per_box * (double)n));
    double side = std::cbrt(vol / target);
    if (!(side > 0) || !std::isfinite(side)) side = std::max(ext[0], std::max(ext[1], ext[2]));
    for (int c = 0; c < 3; c++) side = std::max(side, ext[c] / kMaxAxisCells3);
    int64_t nc[3];
    for (;;) {
        int64_t tot = 1;
        for (int c = 0; c < 3; c++) {
            nc[c] = std::max<int64_t>(1, (int64_t)std::ceil(ext[c] / side));
            tot *= nc[c];
        }
        if (tot <= kMaxCells3 && nc[0] <= kMaxAxisCells3 && nc[1] <= kMaxAxisCells3 && nc[2] <= kMaxAxisCells3)
            break;
        side *= 1.25;
    }
    Grid3 G;
    for (int c = 0; c < 3; c++) {
        G.o[c] = bounds[c];
        G.n[c] = (int)nc[c];
    }
    G.side = side;
    G.inv = 1.0 / side;
    G.h = 0.5 * side;
    G.margin = std::ldexp(M, -30);

    Events ev(2);
    if (!ev.ok(2)) return cuda_fail(cudaErrorUnknown, "event create");
    Grid3Buffers B;
    B.ncells = nc[0] * nc[1] * nc[2];
    B.nx = G.n[0];
    B.ny = G.n[1];
    B.nz = G.n[2];
    for (int c = 0; c < 3; c++) B.g0[c] = G.o[c];
    B.side = side;
    B.margin = G.margin;
    frw_status rc = FRW_OK;
    uint8_t *need = nullptr, *need_up = nullptr;
    std::vector<Level3> up;
    unsigned long long max_list = 0;
    auto ck = [&](cudaError_t e, const char *what) {
        if (e != cudaSuccess && rc == FRW_OK) rc = cuda_fail(e, what);
        return rc == FRW_OK;
    };
    do {
        if (!ck(cudaEventRecord(ev[0], st), "event")) break;
        if (!ck(cudaMallocAsync(&B.status, 4, st), "malloc status")) break;
        if (!ck(cudaMemsetAsync(B.status, 0, 4, st), "memset")) break;
        for (int l = 0; l < kMaxLevels3; l++) {
            const bool top = std::max(G.n[0], std::max(G.n[1], G.n[2])) <= 2 * kRingCap3 + 1 || l == kMaxLevels3 - 1;
            G.cap = top ? (1 << 28) : kRingCap3;
            const int upnx = (G.n[0] + 1) / 2, upny = (G.n[1] + 1) / 2, upnz = (G.n[2] + 1) / 2;
            const int64_t upcells = (int64_t)upnx * upny * upnz;
            if (!top) {
                if (!ck(cudaMallocAsync(&need_up, (size_t)upcells, st), "malloc needs")) break;
                if (!ck(cudaMemsetAsync(need_up, 0, (size_t)upcells, st), "memset")) break;
            }
            LevelOut lo;
            rc = build_level(d_boxes, n, G, need, top ? nullptr : need_up, upnx, upny, st, &lo);
            if (rc != FRW_OK) break;
            max_list = std::max(max_list, lo.max_list);
            if (l == 0) {
                B.cells = lo.cells;
                B.lists = lo.lists;
                B.entries = lo.entries;
                B.deferred = lo.deferred;
            } else {
                B.up_cells[l - 1] = lo.cells;
                B.up_lists[l - 1] = lo.lists;
                B.up_entries += lo.entries;
                Level3 V;
                V.cells = lo.cells;
                V.lists = lo.lists;
                V.ginv = G.inv;
                V.hq = G.h + 2.0 * G.margin;
                V.nx = G.n[0];
                V.ny = G.n[1];
                V.nz = G.n[2];
                V.pad = 0;
                up.push_back(V);
                B.nup = l;
            }
            if (need) cudaFreeAsync(need, st);
            need = need_up;
            need_up = nullptr;
            if (top || lo.deferred == 0) break;
            // the next level: cells twice as large, same origin
            G.n[0] = upnx;
            G.n[1] = upny;
            G.n[2] = upnz;
            G.side = std::ldexp(G.side, 1);
            G.inv = std::ldexp(G.inv, -1);
            G.h = std::ldexp(G.h, 1);
        }
        if (rc != FRW_OK) break;
        if (!up.empty()) {
            if (!ck(cudaMallocAsync(&B.up, up.size() * sizeof(Level3), st), "malloc levels")) break;
            if (!ck(cudaMemcpyAsync(B.up, up.data(), up.size() * sizeof(Level3), cudaMemcpyHostToDevice, st),
                    "levels"))
                break;
        }
        if (!ck(cudaEventRecord(ev[1], st), "event")) break;
        if ((rc = wait_event(ev[1], "build_grid3"))) break;
        B.max_list = (int32_t)max_list;
        cudaEventElapsedTime(&B.build_ms, ev[0], ev[1]);
    } while (0);
    if (need) cudaFreeAsync(need, st);
    if (need_up) cudaFreeAsync(need_up, st);
    if (rc != FRW_OK) {
        free_grid3(&B, st);
        return rc;
    }
    *out = B;
    return FRW_OK;
}

frw_status launch_query3(const Dev3Layout &L, const double *d_pts, int64_t n, double *d_clear, int64_t *d_nearest,
                         cudaStream_t st) {
    if (n <= 0) return FRW_OK;
    k3_query<<<(unsigned)((n + 255) / 256), 256, 0, st>>>(L, d_pts, n, d_clear, d_nearest);
    const cudaError_t e = cudaGetLastError();
    return e == cudaSuccess ? FRW_OK : cuda_fail(e, "k3_query");
}

frw_status launch_walk3(const Walk3Params &P, int blocks, cudaStream_t st) {
    k_walk3<false><<<blocks, kW3Threads, 0, st>>>(P);
    const cudaError_t e = cudaGetLastError();
    return e == cudaSuccess ? FRW_OK : cuda_fail(e, "k_walk3");
}

frw_status launch_walk3_batch(const Walk3Params &P, int blocks, cudaStream_t st) {
    k_walk3<true><<<blocks, kW3Threads, 0, st>>>(P);
    const cudaError_t e = cudaGetLastError();
    return e == cudaSuccess ? FRW_OK : cuda_fail(e, "k_walk3 batch");
}

int walk3_max_blocks_per_sm() {
    int b = 0;
    if (cudaOccupancyMaxActiveBlocksPerMultiprocessor(&b, k_walk3<false>, kW3Threads, 0) != cudaSuccess) return 1;
    return std::max(b, 1);
}

int walk3_threads() { return kW3Threads; }

}  // namespace frw
