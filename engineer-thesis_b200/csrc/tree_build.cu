// tree_build.cu -- bottom-up Morton quadtree build on the device.
//
// Replaces the reference's dynamic-parallelism build (createQuadTreeKernel,
// Cuda/createquadtree.cu:97-371: one block per node, recursive device
// launches, a 5.59 M-node array allocated up front) with:
//   1. Morton keys of the rect centres (16 bits per axis over the bounds);
//   2. a stable LSD radix sort (4 x 8-bit passes) whose scatter ranks items
//      with warp match/ballot + popc instead of shared-memory atomics;
//   3. a level-synchronous split of Morton ranges: each frontier range is cut
//      at its next base-4 digit by binary search on the sorted keys (no data
//      movement); child node ids come from a count -> scan -> emit pass, so
//      the build is deterministic; single-quadrant ranges are re-split one
//      level down without emitting a node (path compression); ranges whose
//      keys are all equal are split by index;
//   4. a bottom-up refit of the child boxes, batch by batch in reverse
//      allocation order (children are always allocated after their parent).
// Output is the flat node array of frw_internal.h: 64-byte child-box records
// plus 16-byte child references, nodes of one level contiguous.
// The tree shape does not affect query results: queries are exact whatever
// the structure (the boxes are exact FP32 unions of FP32-exact rects).
#include <cuda_runtime.h>

#include <algorithm>
#include <cstddef>
#include <cstring>
#include <initializer_list>
#include <vector>

#include "frw_internal.h"

namespace frw {
namespace {

constexpr int kRsThreads = 256;
constexpr int kRsWarps = kRsThreads / 32;
constexpr int kRsItems = 8;  // per thread
constexpr int kRsTile = kRsThreads * kRsItems;
constexpr int kRsChunk = kRsTile / kRsWarps;  // contiguous items per warp

__device__ __forceinline__ uint32_t spread_bits(uint32_t v) {
    v &= 0xFFFFu;
    v = (v | (v << 8)) & 0x00FF00FFu;
    v = (v | (v << 4)) & 0x0F0F0F0Fu;
    v = (v | (v << 2)) & 0x33333333u;
    v = (v | (v << 1)) & 0x55555555u;
    return v;
}

__global__ void k_morton(const float4 *__restrict__ rects, int n, double bx0, double by0, double sx,
                         double sy, uint32_t *__restrict__ keys, int32_t *__restrict__ vals) {
    int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= n) return;
    float4 r = rects[i];
    double cx = ((double)r.x + (double)r.z) * 0.5, cy = ((double)r.y + (double)r.w) * 0.5;
    double fx = (cx - bx0) * sx, fy = (cy - by0) * sy;  // sx = 65536 / W
    uint32_t qx = fx <= 0.0 ? 0u : (fx >= 65535.0 ? 65535u : (uint32_t)fx);
    uint32_t qy = fy <= 0.0 ? 0u : (fy >= 65535.0 ? 65535u : (uint32_t)fy);
    keys[i] = spread_bits(qx) | (spread_bits(qy) << 1);
    vals[i] = i;
}

__global__ void __launch_bounds__(kRsThreads) k_rs_hist(const uint32_t *__restrict__ keys, int n,
                                                        int shift, uint32_t *__restrict__ hist,
                                                        int nblk) {
    __shared__ uint32_t h[256];
    h[threadIdx.x] = 0;
    __syncthreads();
    int base = blockIdx.x * kRsTile;
    for (int k = 0; k < kRsItems; k++) {
        int i = base + k * kRsThreads + threadIdx.x;
        if (i < n) atomicAdd(&h[(keys[i] >> shift) & 255u], 1u);
    }
    __syncthreads();
    hist[threadIdx.x * nblk + blockIdx.x] = h[threadIdx.x];
}

// Exclusive scan of up to a few million u32/u64 values with one block.
template <typename T>
__global__ void __launch_bounds__(1024) k_scan_excl(T *data, int64_t n, T *total) {
    __shared__ T part[1024];
    int t = threadIdx.x;
    int64_t per = (n + 1023) / 1024;
    int64_t a = t * per, b = a + per < n ? a + per : n;
    T s = 0;
    for (int64_t i = a; i < b; i++) s += data[i];
    part[t] = s;
    __syncthreads();
    for (int off = 1; off < 1024; off <<= 1) {
        T v = t >= off ? part[t - off] : 0;
        __syncthreads();
        part[t] += v;
        __syncthreads();
    }
    T run = t ? part[t - 1] : 0;
    for (int64_t i = a; i < b; i++) {
        T v = data[i];
        data[i] = run;
        run += v;
    }
    if (t == 1023 && total) *total = part[1023];
}

// Stable scatter: warp w of a tile owns kRsChunk consecutive items and walks
// them 32 at a time; __match_any_sync groups equal digits, popc of the lower
// peers gives the rank inside the chunk.
__global__ void __launch_bounds__(kRsThreads) k_rs_scatter(const uint32_t *__restrict__ kin,
                                                           const int32_t *__restrict__ vin,
                                                           uint32_t *__restrict__ kout,
                                                           int32_t *__restrict__ vout, int n,
                                                           int shift, const uint32_t *__restrict__ hist,
                                                           int nblk) {
    __shared__ uint32_t cnt[kRsWarps][256];
    const int lane = threadIdx.x & 31, w = threadIdx.x >> 5;
    for (int d = threadIdx.x; d < kRsWarps * 256; d += kRsThreads) (&cnt[0][0])[d] = 0;
    __syncthreads();
    const int base = blockIdx.x * kRsTile + w * kRsChunk;
    const uint32_t lt = (1u << lane) - 1u;
    for (int c = 0; c < kRsChunk; c += 32) {
        int i = base + c + lane;
        uint32_t d = i < n ? (kin[i] >> shift) & 255u : 256u;
        uint32_t peers = __match_any_sync(0xFFFFFFFFu, d);
        if (d < 256u && (peers & lt) == 0) cnt[w][d] += __popc(peers);
        __syncwarp();
    }
    __syncthreads();
    {
        int d = threadIdx.x;  // 256 threads == 256 digits
        uint32_t off = hist[d * nblk + blockIdx.x];
        for (int ww = 0; ww < kRsWarps; ww++) {
            uint32_t t = cnt[ww][d];
            cnt[ww][d] = off;
            off += t;
        }
    }
    __syncthreads();
    for (int c = 0; c < kRsChunk; c += 32) {
        int i = base + c + lane;
        uint32_t key = i < n ? kin[i] : 0u;
        uint32_t d = i < n ? (key >> shift) & 255u : 256u;
        uint32_t peers = __match_any_sync(0xFFFFFFFFu, d);
        uint32_t pos = 0;
        if (d < 256u) pos = cnt[w][d] + __popc(peers & lt);
        __syncwarp();
        if (d < 256u) {
            kout[pos] = key;
            vout[pos] = vin[i];
            if ((peers & lt) == 0) cnt[w][d] += __popc(peers);
        }
        __syncwarp();
    }
}

__global__ void k_gather(const float4 *__restrict__ in, const int32_t *__restrict__ perm, int n,
                         float4 *__restrict__ out) {
    int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i < n) out[i] = in[perm[i]];
}

struct Frontier {
    int32_t *node, *level, *start, *end;
};

__device__ __forceinline__ int lower_digit(const uint32_t *keys, int s, int e, int shift, uint32_t d) {
    // first index in [s, e) whose digit at `shift` is >= d (digits are sorted there)
    int lo = s, hi = e;
    while (lo < hi) {
        int mid = (lo + hi) >> 1;
        if (((keys[mid] >> shift) & 3u) < d) lo = mid + 1;
        else hi = mid;
    }
    return lo;
}

__device__ __forceinline__ void child_bounds(const uint32_t *keys, int level, int s, int e, int b[5]) {
    b[0] = s;
    b[4] = e;
    if (level < 16) {
        int shift = 30 - 2 * level;
        for (int d = 1; d < 4; d++) b[d] = lower_digit(keys, s, e, shift, (uint32_t)d);
    } else {  // identical keys: split by index
        for (int d = 1; d < 4; d++) b[d] = s + (int)((int64_t)(e - s) * d / 4);
    }
}

// Per frontier entry: (new nodes << 32) | (next-frontier entries).
__device__ __forceinline__ unsigned long long split_count_one(const uint32_t *keys, const Frontier &fr, int i,
                                                              int leaf_max) {
    int b[5];
    int level = fr.level[i];
    child_bounds(keys, level, fr.start[i], fr.end[i], b);
    int nonempty = 0, big = 0;
    for (int c = 0; c < 4; c++) {
        int m = b[c + 1] - b[c];
        nonempty += m > 0;
        big += m > leaf_max;
    }
    if (nonempty == 1 && level < 16 && big == 1) return 1ull;  // compress: re-split one level down
    return ((unsigned long long)big << 32) | (unsigned long long)big;
}

__global__ void k_split_count(const uint32_t *__restrict__ keys, Frontier fr, int nfr, int leaf_max,
                              unsigned long long *__restrict__ cnt) {
    int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= nfr) return;
    cnt[i] = split_count_one(keys, fr, i, leaf_max);
}

// Per frontier entry with its scanned offsets: the node's child references
// and the next frontier's entries.
__device__ __forceinline__ void split_emit_one(const uint32_t *keys, const Frontier &fr, int i, int leaf_max,
                                               unsigned long long o, int node_base, int4 *nref,
                                               const Frontier &nx) {
    int b[5];
    int level = fr.level[i], node = fr.node[i];
    child_bounds(keys, level, fr.start[i], fr.end[i], b);
    int nonempty = 0, big = 0;
    for (int c = 0; c < 4; c++) {
        int m = b[c + 1] - b[c];
        nonempty += m > 0;
        big += m > leaf_max;
    }
    int onode = (int)(o >> 32), onext = (int)(o & 0xFFFFFFFFull);
    if (nonempty == 1 && level < 16 && big == 1) {
        nx.node[onext] = node;
        nx.level[onext] = level + 1;
        nx.start[onext] = fr.start[i];
        nx.end[onext] = fr.end[i];
        return;
    }
    int ref[4];
    int j = 0;
    for (int c = 0; c < 4; c++) {
        int m = b[c + 1] - b[c];
        if (m == 0) ref[c] = kRefEmpty;
        else if (m <= leaf_max) ref[c] = leaf_ref(b[c], m);
        else {
            int id = node_base + onode + j;
            ref[c] = id;
            nx.node[onext + j] = id;
            nx.level[onext + j] = level + 1;
            nx.start[onext + j] = b[c];
            nx.end[onext + j] = b[c + 1];
            j++;
        }
    }
    nref[node] = make_int4(ref[0], ref[1], ref[2], ref[3]);
}

__global__ void k_split_emit(const uint32_t *__restrict__ keys, Frontier fr, int nfr, int leaf_max,
                             const unsigned long long *__restrict__ off, int node_base,
                             int4 *__restrict__ nref, Frontier nx) {
    int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= nfr) return;
    split_emit_one(keys, fr, i, leaf_max, off[i], node_base, nref, nx);
}

__device__ __forceinline__ float4 box_union(float4 a, float4 b) {
    return make_float4(fminf(a.x, b.x), fminf(a.y, b.y), fmaxf(a.z, b.z), fmaxf(a.w, b.w));
}

// Child box c of `node`: the union of its child's boxes or of its leaf's rects.
__device__ __forceinline__ void refit_one(const float4 *rects, const int4 *nref, float4 *nbox, int node, int c) {
    int4 r4 = nref[node];
    int ref = c == 0 ? r4.x : c == 1 ? r4.y : c == 2 ? r4.z : r4.w;
    const float inf = __int_as_float(0x7f800000);
    float4 box = make_float4(inf, inf, -inf, -inf);
    if (ref >= 0) {
        for (int k = 0; k < 4; k++) box = box_union(box, nbox[4 * ref + k]);
    } else if (ref != kRefEmpty) {
        int f = leaf_first(ref), m = leaf_count(ref);
        for (int k = 0; k < m; k++) box = box_union(box, rects[f + k]);
    }
    nbox[4 * node + c] = box;
}

__global__ void k_refit(const float4 *__restrict__ rects, const int4 *__restrict__ nref,
                        float4 *__restrict__ nbox, int a, int b) {
    int t = blockIdx.x * blockDim.x + threadIdx.x;
    int node = a + (t >> 2), c = t & 3;
    if (node >= b) return;
    refit_one(rects, nref, nbox, node, c);
}

// Exclusive scan over one block of 1024 threads; every thread gets the total.
__device__ __forceinline__ unsigned long long block_scan_u64(unsigned long long v, unsigned long long *wt,
                                                             unsigned long long &total) {
    const int lane = threadIdx.x & 31, w = threadIdx.x >> 5;
    unsigned long long x = v;
#pragma unroll
    for (int o = 1; o < 32; o <<= 1) {
        const unsigned long long y = __shfl_up_sync(0xFFFFFFFFu, x, o);
        if (lane >= o) x += y;
    }
    if (lane == 31) wt[w] = x;
    __syncthreads();
    if (w == 0) {
        unsigned long long t = wt[lane];
#pragma unroll
        for (int o = 1; o < 32; o <<= 1) {
            const unsigned long long y = __shfl_up_sync(0xFFFFFFFFu, t, o);
            if (lane >= o) t += y;
        }
        wt[lane] = t;
    }
    __syncthreads();
    total = wt[31];
    const unsigned long long before = w ? wt[w - 1] : 0ull;
    __syncthreads();
    return before + x - v;
}

constexpr int kSmallBuild = 1 << 16;  // layouts up to this many rects split and refit in one block
constexpr int kMaxLevels = 64;

// The whole level-synchronous split and the bottom-up refit of a small
// layout in one block of 1024 threads: the same count -> scan -> emit steps
// as the multi-kernel path (so the same node numbering), with the frontier
// sizes kept on the device instead of read back per level.  out[0] nodes,
// out[1] depth, out[2] 1 when the level bound was hit.
__global__ void __launch_bounds__(1024) k_build_small(const uint32_t *__restrict__ keys, int n, Frontier fa,
                                                      Frontier fb, int leaf_max, unsigned long long *cnt,
                                                      int4 *nref, const float4 *__restrict__ rects,
                                                      float4 *nbox, int *out) {
    __shared__ unsigned long long wt[32];
    __shared__ int s_nfr, s_nodes, s_depth, s_nb, s_over;
    __shared__ int s_batch[kMaxLevels + 4];
    const int t = threadIdx.x;
    if (t == 0) {
        s_nodes = 1;
        s_depth = 0;
        s_over = 0;
        s_batch[0] = 0;
        s_batch[1] = 1;
        s_nb = 2;
        if (n <= leaf_max) {  // a layout of <= leaf_max rects still gets one internal root node
            nref[0] = make_int4(leaf_ref(0, n), kRefEmpty, kRefEmpty, kRefEmpty);
            s_nfr = 0;
        } else {
            fa.node[0] = 0;
            fa.level[0] = 0;
            fa.start[0] = 0;
            fa.end[0] = n;
            s_nfr = 1;
        }
    }
    __syncthreads();
    for (int iter = 0;; iter++) {
        const int nfr = s_nfr;
        if (nfr == 0) break;
        if (iter > kMaxLevels) {
            if (t == 0) s_over = 1;
            break;
        }
        for (int i = t; i < nfr; i += 1024) cnt[i] = split_count_one(keys, fa, i, leaf_max);
        __syncthreads();
        unsigned long long carry = 0;
        for (int b0 = 0; b0 < nfr; b0 += 1024) {
            const int i = b0 + t;
            const unsigned long long v = i < nfr ? cnt[i] : 0ull;
            unsigned long long total;
            const unsigned long long e = block_scan_u64(v, wt, total);
            if (i < nfr) cnt[i] = carry + e;
            carry += total;
        }
        __syncthreads();
        const int node_base = s_nodes;
        for (int i = t; i < nfr; i += 1024) split_emit_one(keys, fa, i, leaf_max, cnt[i], node_base, nref, fb);
        __syncthreads();
        if (t == 0) {
            const int new_nodes = (int)(carry >> 32);
            if (new_nodes > 0) {
                s_nodes += new_nodes;
                s_batch[s_nb++] = s_nodes;
                s_depth++;
            }
            s_nfr = (int)(carry & 0xFFFFFFFFull);
        }
        const Frontier tmp = fa;
        fa = fb;
        fb = tmp;
        __syncthreads();
    }
    for (int k = s_nb - 1; k > 0; k--) {
        const int a = s_batch[k - 1], b = s_batch[k];
        for (int q = t; q < 4 * (b - a); q += 1024) refit_one(rects, nref, nbox, a + (q >> 2), q & 3);
        __syncthreads();
    }
    if (t == 0) {
        out[0] = s_nodes;
        out[1] = s_depth;
        out[2] = s_over;
    }
}

// Order-preserving unsigned key of a float (+0 for -0): unsigned order of
// the keys is the order of the values.
__device__ __forceinline__ unsigned f_key(float f) {
    const unsigned u = __float_as_uint(f + 0.0f);
    return (u & 0x80000000u) ? ~u : (u | 0x80000000u);
}

// Checks every rect (finite, |c| < 2^24, not inverted, inside the given
// bounds when there are any) and reduces the extent of the valid ones:
// out->bad = min over bad rects of (index << 2 | reason), out->key = keys of
// min x0, min y0 (atomicMin) and max x1, max y1 (atomicMax).
__global__ void __launch_bounds__(256) k_check_rects(const float4 *__restrict__ rects, int64_t n, int has_given,
                                                     double g0, double g1, double g2, double g3,
                                                     RectCheck *__restrict__ out) {
    unsigned k0 = 0xFFFFFFFFu, k1 = 0xFFFFFFFFu, k2 = 0u, k3 = 0u;
    unsigned long long bad = ~0ull;
    for (int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; i < n; i += (int64_t)gridDim.x * blockDim.x) {
        const float4 q = __ldg(rects + i);
        const float c[4] = {q.x, q.y, q.z, q.w};
        bool ok = true;
#pragma unroll
        for (int k = 0; k < 4; k++) ok = ok && isfinite(c[k]) && fabsf(c[k]) < 16777216.0f;
        int why = !ok ? 1 : (!(q.x <= q.z && q.y <= q.w) ? 2 : 0);
        if (!why && has_given &&
            !((double)q.y >= g1 && (double)q.x >= g0 && (double)q.w <= g3 && (double)q.z <= g2))
            why = 3;
        if (why) {
            bad = min(bad, ((unsigned long long)i << 2) | (unsigned)why);
            continue;
        }
        k0 = min(k0, f_key(q.x));
        k1 = min(k1, f_key(q.y));
        k2 = max(k2, f_key(q.z));
        k3 = max(k3, f_key(q.w));
    }
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) {
        k0 = min(k0, __shfl_xor_sync(0xFFFFFFFFu, k0, o));
        k1 = min(k1, __shfl_xor_sync(0xFFFFFFFFu, k1, o));
        k2 = max(k2, __shfl_xor_sync(0xFFFFFFFFu, k2, o));
        k3 = max(k3, __shfl_xor_sync(0xFFFFFFFFu, k3, o));
        bad = min(bad, __shfl_xor_sync(0xFFFFFFFFu, bad, o));
    }
    __shared__ unsigned sk[4][8];
    __shared__ unsigned long long sb[8];
    const int w = threadIdx.x >> 5, lane = threadIdx.x & 31;
    if (lane == 0) {
        sk[0][w] = k0;
        sk[1][w] = k1;
        sk[2][w] = k2;
        sk[3][w] = k3;
        sb[w] = bad;
    }
    __syncthreads();
    if (threadIdx.x == 0) {
        const int nw = blockDim.x >> 5;
        for (int j = 1; j < nw; j++) {
            k0 = min(k0, sk[0][j]);
            k1 = min(k1, sk[1][j]);
            k2 = max(k2, sk[2][j]);
            k3 = max(k3, sk[3][j]);
            bad = min(bad, sb[j]);
        }
        atomicMin(&out->key[0], k0);
        atomicMin(&out->key[1], k1);
        atomicMax(&out->key[2], k2);
        atomicMax(&out->key[3], k3);
        if (bad != ~0ull) atomicMin(&out->bad, bad);
    }
}

float key_value(unsigned k) {
    const unsigned u = (k & 0x80000000u) ? (k & 0x7FFFFFFFu) : ~k;
    float f;
    memcpy(&f, &u, 4);
    return f;
}

}  // namespace

frw_status check_rects(const float4 *d_rects, int64_t n, const double *given, int sms, cudaStream_t st,
                       int64_t *bad, int *why, double ext[4]) {
    RectCheck *d = nullptr;
    FRW_CK(cudaMallocAsync(&d, sizeof(RectCheck), st));
    frw_status rc = FRW_OK;
    do {
        cudaError_t e = cudaMemsetAsync(d, 0xFF, offsetof(RectCheck, key) + 2 * sizeof(unsigned), st);
        if (e == cudaSuccess) e = cudaMemsetAsync(&d->key[2], 0, 2 * sizeof(unsigned), st);
        if (e != cudaSuccess) {
            rc = cuda_fail(e, "check_rects: memset");
            break;
        }
        const int64_t want = (n + 255) / 256;
        const unsigned blocks = (unsigned)std::max<int64_t>(1, std::min<int64_t>(want, (int64_t)std::max(sms, 1) * 8));
        k_check_rects<<<blocks, 256, 0, st>>>(d_rects, n, given != nullptr, given ? given[0] : 0.0,
                                               given ? given[1] : 0.0, given ? given[2] : 0.0,
                                               given ? given[3] : 0.0, d);
        if ((e = cudaGetLastError()) != cudaSuccess) {
            rc = cuda_fail(e, "check_rects: launch");
            break;
        }
        RectCheck h;
        if ((rc = read_back(&h, d, sizeof(h), st, "check_rects"))) break;
        *bad = h.bad == ~0ull ? -1 : (int64_t)(h.bad >> 2);
        *why = h.bad == ~0ull ? 0 : (int)(h.bad & 3);
        for (int k = 0; k < 4; k++) ext[k] = (double)key_value(h.key[k]);
    } while (0);
    cudaFreeAsync(d, st);
    return rc;
}

void free_tree(TreeBuffers *t, cudaStream_t st) {
    for (void *p : {(void *)t->rects, (void *)t->ids, (void *)t->nbox, (void *)t->nref})
        if (p) cudaFreeAsync(p, st);
    *t = TreeBuffers();
}

frw_status build_tree(const float4 *d_rects_in, int32_t n, const double bounds[4], int leaf_max,
                      cudaStream_t st, TreeBuffers *out, float *build_ms) {
    *out = TreeBuffers();
    if (n <= 0 || leaf_max < 1 || leaf_max > kLeafCountMax) {
        set_error("build_tree: bad size");
        return FRW_E_ARG;
    }
    if ((int64_t)n > (1ll << 26) - 1) {
        set_error("build_tree: more than 2^26-1 rects");
        return FRW_E_ARG;
    }
    cudaEvent_t e0, e1;
    FRW_CK(cudaEventCreate(&e0));
    FRW_CK(cudaEventCreate(&e1));

    const int nblk = (n + kRsTile - 1) / kRsTile;
    const int cap_nodes = n > 1 ? n : 1;
    uint32_t *k0 = nullptr, *k1 = nullptr, *hist = nullptr;
    int32_t *v0 = nullptr, *v1 = nullptr;
    unsigned long long *cnt = nullptr, *tot = nullptr;
    int32_t *frb = nullptr;
    TreeBuffers T;
    frw_status rc = FRW_OK;
    auto ck = [&](cudaError_t e, const char *what) {
        if (e != cudaSuccess && rc == FRW_OK) rc = cuda_fail(e, what);
        return rc == FRW_OK;
    };
    do {
        if (!ck(cudaEventRecord(e0, st), "event")) break;
        if (!ck(cudaMallocAsync(&T.rects, (size_t)n * 16, st), "malloc rects")) break;
        if (!ck(cudaMallocAsync(&T.ids, (size_t)n * 4, st), "malloc ids")) break;
        if (!ck(cudaMallocAsync(&T.nbox, (size_t)cap_nodes * 64, st), "malloc nbox")) break;
        if (!ck(cudaMallocAsync(&T.nref, (size_t)cap_nodes * 16, st), "malloc nref")) break;
        // temporaries from the stream-ordered pool (no device-wide sync)
        if (!ck(cudaMallocAsync(&k0, (size_t)n * 4, st), "malloc keys")) break;
        if (!ck(cudaMallocAsync(&k1, (size_t)n * 4, st), "malloc keys")) break;
        if (!ck(cudaMallocAsync(&v0, (size_t)n * 4, st), "malloc vals")) break;
        if (!ck(cudaMallocAsync(&v1, (size_t)n * 4, st), "malloc vals")) break;
        if (!ck(cudaMallocAsync(&hist, (size_t)256 * nblk * 4, st), "malloc hist")) break;
        if (!ck(cudaMallocAsync(&cnt, (size_t)cap_nodes * 8, st), "malloc cnt")) break;
        if (!ck(cudaMallocAsync(&tot, 16, st), "malloc tot")) break;  // scan total, or the small build's result
        if (!ck(cudaMallocAsync(&frb, (size_t)cap_nodes * 8 * 4, st), "malloc frontier")) break;

        double W = bounds[2] - bounds[0], H = bounds[3] - bounds[1];
        double sx = W > 0 ? 65536.0 / W : 0.0, sy = H > 0 ? 65536.0 / H : 0.0;
        k_morton<<<(n + 255) / 256, 256, 0, st>>>(d_rects_in, n, bounds[0], bounds[1], sx, sy, k0, v0);
        if (!ck(cudaGetLastError(), "k_morton")) break;
        for (int shift = 0; shift < 32; shift += 8) {
            k_rs_hist<<<nblk, kRsThreads, 0, st>>>(k0, n, shift, hist, nblk);
            k_scan_excl<uint32_t><<<1, 1024, 0, st>>>(hist, (int64_t)256 * nblk, nullptr);
            k_rs_scatter<<<nblk, kRsThreads, 0, st>>>(k0, v0, k1, v1, n, shift, hist, nblk);
            if (!ck(cudaGetLastError(), "radix sort")) break;
            std::swap(k0, k1);
            std::swap(v0, v1);
        }
        if (rc) break;
        k_gather<<<(n + 255) / 256, 256, 0, st>>>(d_rects_in, v0, n, T.rects);
        if (!ck(cudaMemcpyAsync(T.ids, v0, (size_t)n * 4, cudaMemcpyDeviceToDevice, st), "ids")) break;

        // level-synchronous split
        Frontier fa{frb, frb + cap_nodes, frb + 2 * cap_nodes, frb + 3 * cap_nodes};
        Frontier fb{frb + 4 * cap_nodes, frb + 5 * cap_nodes, frb + 6 * cap_nodes, frb + 7 * cap_nodes};
        if (n <= kSmallBuild) {  // one block: no host round trip per level
            k_build_small<<<1, 1024, 0, st>>>(k0, n, fa, fb, leaf_max, cnt, T.nref, T.rects, T.nbox,
                                              reinterpret_cast<int *>(tot));
            if (!ck(cudaGetLastError(), "split")) break;
            int h[4] = {0, 0, 0, 0};
            if (!ck(cudaEventRecord(e1, st), "event")) break;
            if ((rc = read_back(h, tot, 16, st, "build_tree: split result"))) break;
            if (h[2]) {
                set_error("build_tree: too many levels");
                rc = FRW_E_KERNEL;
                break;
            }
            T.nodes = h[0];
            T.depth = h[1];
            T.bytes = (int64_t)n * 20 + (int64_t)T.nodes * 80;
            float ms = 0;
            cudaEventElapsedTime(&ms, e0, e1);
            if (build_ms) *build_ms = ms;
            break;
        }
        int32_t root[4] = {0, 0, 0, n};
        if (!ck(cudaMemcpyAsync(fa.node, &root[0], 4, cudaMemcpyHostToDevice, st), "root")) break;
        if (!ck(cudaMemcpyAsync(fa.level, &root[1], 4, cudaMemcpyHostToDevice, st), "root")) break;
        if (!ck(cudaMemcpyAsync(fa.start, &root[2], 4, cudaMemcpyHostToDevice, st), "root")) break;
        if (!ck(cudaMemcpyAsync(fa.end, &root[3], 4, cudaMemcpyHostToDevice, st), "root")) break;
        int nodes = 1, nfr = 1, depth = 0;
        std::vector<int> batch = {0, 1};
        for (int iter = 0; nfr > 0; iter++) {
            if (iter > kMaxLevels) {
                set_error("build_tree: too many levels");
                rc = FRW_E_KERNEL;
                break;
            }
            k_split_count<<<(nfr + 255) / 256, 256, 0, st>>>(k0, fa, nfr, leaf_max, cnt);
            k_scan_excl<unsigned long long><<<1, 1024, 0, st>>>(cnt, nfr, tot);
            unsigned long long h_tot = 0;
            if ((rc = read_back(&h_tot, tot, 8, st, "build_tree: scan total"))) break;
            int new_nodes = (int)(h_tot >> 32), next = (int)(h_tot & 0xFFFFFFFFull);
            k_split_emit<<<(nfr + 255) / 256, 256, 0, st>>>(k0, fa, nfr, leaf_max, cnt, nodes, T.nref, fb);
            if (!ck(cudaGetLastError(), "split")) break;
            if (new_nodes > 0) {
                nodes += new_nodes;
                batch.push_back(nodes);
                depth++;
            }
            std::swap(fa, fb);
            nfr = next;
        }
        if (rc) break;
        for (int k = (int)batch.size() - 1; k > 0; k--) {
            int a = batch[k - 1], b = batch[k];
            int thr = 4 * (b - a);
            k_refit<<<(thr + 255) / 256, 256, 0, st>>>(T.rects, T.nref, T.nbox, a, b);
        }
        if (!ck(cudaGetLastError(), "refit")) break;
        T.nodes = nodes;
        T.depth = depth;
        T.bytes = (int64_t)n * 20 + (int64_t)nodes * 80;
        if (!ck(cudaEventRecord(e1, st), "event")) break;
        if ((rc = wait_event(e1, "build_tree"))) break;
        float ms = 0;
        cudaEventElapsedTime(&ms, e0, e1);
        if (build_ms) *build_ms = ms;
    } while (0);
    for (void *p : {(void *)k0, (void *)k1, (void *)v0, (void *)v1, (void *)hist, (void *)cnt, (void *)tot,
                    (void *)frb})
        if (p) cudaFreeAsync(p, st);
    cudaEventDestroy(e0);
    cudaEventDestroy(e1);
    if (rc != FRW_OK) {
        free_tree(&T, st);
        return rc;
    }
    *out = T;
    return FRW_OK;
}

}  // namespace frw
