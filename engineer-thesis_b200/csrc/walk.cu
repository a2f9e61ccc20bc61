// walk.cu -- persistent floating-random-walk kernel.
//
// Reference: one CUDA thread per walk, one launch per batch
// (randomWalkCuda, Cuda/randomwalk.cu:64-121) with curand XORWOW, a device-heap
// traversal stack per thread, a linear CDF scan in global memory and the hit
// rect written per walk for a host-side std::map histogram
// (Cuda/getAvgPathLenCUDA.cu:23-48).  Here:
//   * the grid is persistent (SM count x resident blocks); each warp lane
//     carries one walk and, when it ends, is refilled from a global walk
//     counter (one atomic per warp refill), so warps stay full while walks of
//     very different lengths finish;
//   * random numbers are counter-based Philox4x32-10 keyed by (seed) with
//     counter (hop/4, walk, stream), one 32-bit word per hop: a walk's
//     trajectory depends only on its index, never on scheduling, so every
//     walk can be replayed by the CPU oracle bit-for-bit;
//   * the Green CDF (201 doubles, and as integer thresholds on the Philox
//     word), a 256-entry guide to it and the first-hop weight tables sit in
//     shared memory; a bin is the guide's entry plus a step or two (the
//     reference's linear scan, CPU/mainFunctions.cpp:40-46, returns the same
//     index because the CDF is nondecreasing);
//   * each hop is one clearance lookup + scalar replay (query.cuh);
//   * walks ending on their job's target are summed in lane registers; other
//     ends are accumulated per (job, conductor) in a per-warp shared-memory
//     table, with Kahan-compensated FP64 sums (single writer per update) for
//     weighted walks and counts alone (shared atomics) otherwise, flushed to
//     the global rows when full and at exit, where the lane sums join it;
//   * the kernel is compiled per launch configuration: one job or many,
//     per-walk records or none, weighted (uniform) start or not, control-
//     variate sums or not.
#include "query.cuh"

namespace frw {
namespace {

constexpr int kWalkThreads = 256;
constexpr int kHopsPerRound = 2;  // hops between refill / walk-end rounds (1: 5.8% slower, 3: 5.6%)
// Resident blocks per SM: 5 blocks of 256 (40 warps) at 48 registers per
// thread, for weighted (uniform start) and unweighted walks alike (weighted
// walks spill a little more there but gain from the extra warps since the
// loop runs two hops per round; 4 blocks at 64 registers: 1.6% slower) --
// except weighted walks of many jobs, whose per-job loads need the registers
// (4 blocks at 64 registers: 6% faster than 5 at 48).
constexpr int kWalkMinBlocksMultiW = 4;
constexpr int kWalkMinBlocks = 5;
constexpr int kWarpsPerBlock = kWalkThreads / 32;
constexpr int kTabSlots = 32;  // per warp
constexpr unsigned long long kEmptyKey = ~0ull;
constexpr unsigned kFull = 0xFFFFFFFFu;
constexpr uint64_t kChunkDefault = 128;  // walks a warp claims from the global counter at a time

struct Slot {
    unsigned long long key, n;
    double s, cs, s2, cs2;
};

__device__ __forceinline__ uint4 philox10(uint4 c, uint2 k) {
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

// Philox block (hop / 4, walk, stream) under key `seed`: the four uniforms of
// hops 4k..4k+3 of one walk.
__device__ __forceinline__ uint4 draw_block(uint64_t seed, uint32_t stream, uint64_t walk, uint32_t hop) {
    return philox10(make_uint4(hop >> 2, (uint32_t)walk, (uint32_t)(walk >> 32), stream),
                    make_uint2((uint32_t)seed, (uint32_t)(seed >> 32)));
}

// The last bin lo in [0, 200) with intg[lo] <= u (intg nondecreasing,
// intg[0] = 0), by binary search.
__device__ __forceinline__ int bin_search(const double *s_intg, double u) {
    int lo = 0, hi = FRW_NSAMPLE;  // intg[lo] <= u
#pragma unroll
    for (int k = 0; k < 8; k++) {
        if (hi - lo > 1) {
            const int mid = (lo + hi) >> 1;
            if (s_intg[mid] <= u) lo = mid;
            else hi = mid;
        }
    }
    return lo;
}

// The same bin from a guide table: guide[k] = bin_search(k / 256), so the
// bin of u in [k/256, (k+1)/256) is guide[k] or one of the next few.
constexpr int kGuide = 256;
__device__ __forceinline__ int bin_of(const double *s_intg, const uint8_t *guide, double u) {
    int lo = guide[(int)__dmul_rn(u, (double)kGuide)];
    while (lo < FRW_NSAMPLE - 1 && s_intg[lo + 1] <= u) lo++;
    return lo;
}

// The same bin for u = word / 2^32, in integers: the guide entry of
// floor(u * 256) = word >> 24, then word > thr[lo + 1] exactly when
// intg[lo + 1] <= u.
__device__ __forceinline__ int bin_of_word(const uint32_t *thr, const uint8_t *guide, uint32_t word) {
    int lo = guide[word >> 24];
    while (lo < FRW_NSAMPLE - 1 && word > thr[lo + 1]) lo++;
    return lo;
}

__device__ __forceinline__ void kahan_add(double &s, double &c, double v) {
    const double y = __dsub_rn(v, c);
    const double t = __dadd_rn(s, y);
    c = __dsub_rn(__dsub_rn(t, s), y);
    s = t;
}

__device__ __forceinline__ int slot_hash(unsigned long long key) {
    return (int)((key * 0x9E3779B97F4A7C15ull) >> 59);  // 5 bits
}

// Insert one (job, conductor) aggregate; called by several lanes of a warp at
// once with DISTINCT keys (so distinct slots): empty slots are claimed with a
// shared-memory CAS, the rest of the update has a single writer.  False when
// the warp table is full.
// kW: weighted walks (uniform start); without weights every weight is 0 and
// only the counts are kept.
template <bool kW>
__device__ __forceinline__ bool tab_insert(Slot *tab, unsigned long long key, unsigned long long n, double s,
                                           double s2) {
    const int h = slot_hash(key);
    for (int probe = 0; probe < kTabSlots; probe++) {
        Slot &sl = tab[(h + probe) & (kTabSlots - 1)];
        unsigned long long k = *(volatile unsigned long long *)&sl.key;
        if (k == kEmptyKey) {
            k = atomicCAS(&sl.key, kEmptyKey, key);
            if (k == kEmptyKey) {
                sl.n = 0;
                if (kW) sl.s = sl.cs = sl.s2 = sl.cs2 = 0.0;
                k = key;
            }
        }
        if (k == key) {
            sl.n += n;
            if (kW) {
                kahan_add(sl.s, sl.cs, s);
                kahan_add(sl.s2, sl.cs2, s2);
            }
            return true;
        }
    }
    return false;
}

template <bool kMulti>
__device__ __forceinline__ const WalkJob &job_of(const WalkParams &P, int j) {
    return kMulti ? P.jobs[j] : P.job0;
}

// Counts only (no weights): one walk end of `key` added to its slot with a
// shared-memory atomic (slots are claimed by CAS and hold n = 0 while
// empty), so lanes with equal keys need no grouping.  False when the table
// is full.
__device__ __forceinline__ bool tab_count(Slot *tab, unsigned long long key, unsigned long long n) {
    const int h = slot_hash(key);
    for (int probe = 0; probe < kTabSlots; probe++) {
        Slot &sl = tab[(h + probe) & (kTabSlots - 1)];
        unsigned long long k = *(volatile unsigned long long *)&sl.key;
        if (k == kEmptyKey) {
            k = atomicCAS(&sl.key, kEmptyKey, key);
            if (k == kEmptyKey) k = key;
        }
        if (k == key) {
            atomicAdd(&sl.n, n);
            return true;
        }
    }
    return false;
}

// Whole warp: push every used slot to the global rows, then clear.
template <bool kMulti, bool kW>
__device__ void tab_flush(const WalkParams &P, Slot *tab, int lane) {
    for (int q = lane; q < kTabSlots; q += 32) {
        Slot &sl = tab[q];
        if (sl.key == kEmptyKey) continue;
        const int job = (int)(sl.key >> 32);
        const int code = (int)(uint32_t)(sl.key & 0xFFFFFFFFull) - 2;
        unsigned long long *js = P.job_stats + 4 * job;
        if (code >= 0) {
            const int64_t row = job_of<kMulti>(P, job).acc_base + code;
            atomicAdd(P.acc_n + row, sl.n);
            if (kW) {
                atomicAdd(P.acc_s + row, __dsub_rn(sl.s, sl.cs));
                atomicAdd(P.acc_s2 + row, __dsub_rn(sl.s2, sl.cs2));
            }
        } else {
            atomicAdd(js + (code == -1 ? 0 : 1), sl.n);
        }
        atomicAdd(js + 3, sl.n);
        sl.n = 0;
        sl.key = kEmptyKey;
    }
    __syncwarp();
}

// One insertion round (whole warp, convergent): lanes with `ins` add
// (cnt, s1, s2) under `key`.  Equal keys are grouped with a match; each
// group's lowest lane gathers the group's sums (in lane order) and adds them
// to the table, all groups in parallel; a full table is flushed and the rest
// retried.
template <bool kMulti, bool kW>
__device__ __forceinline__ void tab_round(const WalkParams &P, Slot *tab, int lane, unsigned lt, bool ins,
                                          unsigned long long key, unsigned long long cnt, double s1, double s2) {
    const unsigned em = __ballot_sync(kFull, ins);
    if (!em) return;
    if (!kW) {
        bool pending = ins;
        for (;;) {
            const bool failed = pending && !tab_count(tab, key, cnt);
            pending = failed;
            __syncwarp();
            if (!__any_sync(kFull, failed)) break;
            tab_flush<kMulti, kW>(P, tab, lane);  // table full: empty it, retry the rest
        }
        return;
    }
    bool lead = false;
    if (ins) lead = (__match_any_sync(em, key) & lt) == 0;
    const unsigned leaders = __ballot_sync(kFull, lead);
    for (unsigned rest = em & ~leaders; rest; rest &= rest - 1) {
        const int l = __ffs(rest) - 1;
        const unsigned long long kl = __shfl_sync(kFull, key, l), cl = __shfl_sync(kFull, cnt, l);
        double a = 0.0, b = 0.0;
        if (kW) {
            a = __shfl_sync(kFull, s1, l);
            b = __shfl_sync(kFull, s2, l);
        }
        if (lead && kl == key) {
            if (kW) {
                s1 = __dadd_rn(s1, a);
                s2 = __dadd_rn(s2, b);
            }
            cnt += cl;
        }
    }
    bool pending = lead;
    for (;;) {
        const bool failed = pending && !tab_insert<kW>(tab, key, cnt, s1, s2);
        pending = failed;
        __syncwarp();
        if (!__any_sync(kFull, failed)) break;
        tab_flush<kMulti, kW>(P, tab, lane);  // table full: empty it, retry the rest
    }
}

// kRec: per-walk records requested (some P.rec_* set); without them the
// record stores and their tests are compiled out.  kUniform: uniform start
// on the Gaussian perimeter, whose walks carry the first-hop weight; with
// the Green-CDF start every weight is 0, so the weight, its inputs and the
// weight sums are compiled out.  kCV: the control variate's sums (P.cv_phi,
// P.cv_sums) are kept beside the rows.  kTies: the tree answers some points
// (P.tree_points), and those with more exact near ties than its candidate
// list holds take the whole-tree replay; without it that code is compiled
// out of the kernel.
template <bool kMulti, bool kRec, bool kUniform, bool kCV = false, bool kTies = false>
__global__ void __launch_bounds__(kWalkThreads, kMulti && kUniform ? kWalkMinBlocksMultiW : kWalkMinBlocks)
    k_walk(const WalkParams P) {
    __shared__ double s_intg[FRW_NSAMPLE + 1];
    __shared__ double s_wx[FRW_NSAMPLE], s_wy[FRW_NSAMPLE];
    __shared__ Slot s_tab[kWarpsPerBlock][kTabSlots];
    __shared__ uint8_t s_guide[kGuide];
    __shared__ uint32_t s_thr[FRW_NSAMPLE + 1];  // ceil(intg[k] * 2^32) - 1: u >= intg[k] iff word > s_thr[k]
    __shared__ unsigned long long s_chunk[kWarpsPerBlock][2];  // per warp: unclaimed part of its walk chunk
    __shared__ unsigned long long s_lhops[kWalkThreads];       // per lane: hops of its walks (current job)
    __shared__ double s_cvz[kCV ? 2 : 1][kCV ? kWalkThreads : 1];  // per lane: sums of z and z^2

    const int lane = threadIdx.x & 31, wib = threadIdx.x >> 5;
    for (int i = threadIdx.x; i <= FRW_NSAMPLE; i += blockDim.x) {
        s_intg[i] = P.intg[i];
        // intg[k] * 2^32 is exact; its ceiling is in [1, 2^32] for k >= 1
        s_thr[i] = (uint32_t)((unsigned long long)ceil(P.intg[i] * 0x1p32) - 1ull);
    }
    for (int i = threadIdx.x; i < FRW_NSAMPLE; i += blockDim.x) {
        s_wx[i] = P.wx[i];
        s_wy[i] = P.wy[i];
    }
    Slot *tab = s_tab[wib];
    for (int q = lane; q < kTabSlots; q += 32) {
        tab[q].key = kEmptyKey;
        tab[q].n = 0;
    }
    if (lane == 0) s_chunk[wib][0] = s_chunk[wib][1] = 0;
    s_lhops[threadIdx.x] = 0;
    if (kCV) s_cvz[0][threadIdx.x] = s_cvz[1][threadIdx.x] = 0.0;
    __syncthreads();
    for (int k = threadIdx.x; k < kGuide; k += blockDim.x)
        s_guide[k] = (uint8_t)bin_search(s_intg, (double)k * (1.0 / kGuide));
    __syncthreads();

    const uint32_t lt = (1u << lane) - 1u;
    const int refill_min = P.refill_min < 1 ? 1 : (P.refill_min > 32 ? 32 : P.refill_min);
    constexpr bool uniform_start = kUniform;
    const bool exact = P.exact_perimeter != 0;
    const uint64_t seed = P.seed_dev ? *P.seed_dev : P.seed;
    const uint64_t kChunk = P.chunk ? (uint64_t)P.chunk : kChunkDefault;

    bool active = false, exhausted = false;
    int job = 0;
    uint64_t pw = 0;
    // the lane's Philox block, words (hops & ~3) .. +3: in shared memory,
    // which frees four registers (fewer spills), one load per hop
    __shared__ uint32_t s_rnd[4][kWalkThreads];
    // queries so far of the lane's walk, also the Philox word of its next
    // point (word 0 places the start, word h the point after query h)
    int32_t hops = 0, bin1 = -1;
    int32_t cvq = -1;  // control variate: the walk's (grid arc, first-hop bin) cell, -1 before its first hop
    int side = 0;
    double a0 = 0, perim = 0;
    // The rect the lane's next point is mapped on: the Gaussian surface of a
    // walk about to start, else the last square of its walk.
    double sq[4] = {0, 0, 0, 0};
    uint32_t st = 0;
    // Walks of this lane that end on its job's target (most walks: 92% on the
    // 10k-rect layout) are counted and summed in registers and reach the
    // table in one insertion when the lane changes job and at exit; the hops
    // of all its walks likewise go to the job's totals then.
    uint32_t pn = 0;
    double ps = 0.0, ps2 = 0.0;
    int pjob = 0;
    auto walk_index = [&]() {  // record index of the lane's walk
        const WalkJob &J = job_of<kMulti>(P, job);
        return J.walk_begin + (pw - J.first_walk);
    };
    auto target_key = [&](int j) {
        return ((unsigned long long)j << 32) | (uint32_t)(job_of<kMulti>(P, j).target + 2);
    };

    for (;;) {
        // ---- refill idle lanes from the warp's chunk of the walk counter ----
        const unsigned idle = __ballot_sync(kFull, !active);
        if (!exhausted && __popc(idle) >= refill_min) {
            uint64_t chunk_next = s_chunk[wib][0], chunk_end = s_chunk[wib][1];
            const uint64_t need = (uint64_t)__popc(idle), avail = chunk_end - chunk_next;
            const uint64_t r = (uint64_t)__popc(idle & lt);
            uint64_t mine;
            if (avail >= need) {
                mine = chunk_next + r;
                chunk_next += need;
            } else {  // top up: one atomic per kChunk walks per warp
                const int leader = __ffs(idle) - 1;
                unsigned long long nb = 0;
                if (lane == leader) nb = atomicAdd(P.counter, (unsigned long long)kChunk);
                nb = __shfl_sync(kFull, nb, leader);
                mine = r < avail ? chunk_next + r : nb + (r - avail);
                chunk_next = nb + (need - avail);
                chunk_end = nb + kChunk;
            }
            if (chunk_end >= P.total_walks && chunk_next >= P.total_walks) exhausted = true;
            __syncwarp();
            if (lane == 0) {
                s_chunk[wib][0] = chunk_next;
                s_chunk[wib][1] = chunk_end;
            }
            __syncwarp();
            if (!active) {
                const uint64_t gw = mine;
                if (gw < P.total_walks) {
                    if (kMulti) {  // the job whose walk range holds gw
                        const bool same = gw >= P.jobs[job].walk_begin &&
                                          (job + 1 == P.njobs || gw < P.jobs[job + 1].walk_begin);
                        if (!same) {  // walk indices only grow: search above the current job
                            int lo = gw >= P.jobs[job].walk_begin ? job : 0, hi = P.njobs;
                            while (hi - lo > 1) {
                                const int mid = (lo + hi) >> 1;
                                if (P.jobs[mid].walk_begin <= gw) lo = mid;
                                else hi = mid;
                            }
                            job = lo;
                        }
                    }
                    const WalkJob &J = job_of<kMulti>(P, job);
                    const double4 g4 = P.gauss[job];
                    sq[0] = g4.x;
                    sq[1] = g4.y;
                    sq[2] = g4.z;
                    sq[3] = g4.w;
                    pw = J.first_walk + (gw - J.walk_begin);
                    hops = 0;
                    bin1 = -1;
                    if (kCV) cvq = -1;
                    a0 = 0.0;
                    active = true;
                }
            }
            if (kMulti && __any_sync(kFull, job != pjob)) {  // leave the old job's sums behind
                const bool moved = job != pjob;
                tab_round<kMulti, kUniform>(P, tab, lane, lt, moved && pn > 0, target_key(pjob), pn, ps, ps2);
                if (moved) {
                    const unsigned long long lh = s_lhops[threadIdx.x];
                    if (lh) atomicAdd(P.job_stats + 4 * pjob + 2, lh);
                    s_lhops[threadIdx.x] = 0;
                    pn = 0;
                    ps = ps2 = 0.0;
                    pjob = job;
                }
            }
        }
        if (!__any_sync(kFull, active)) {
            if (exhausted) break;
            continue;
        }

        // ---- two hops of every active walk per round of refills and walk
        // ends (the round's bookkeeping is paid once per two hops; a walk
        // that ends in the first waits for the second) ----
        // The point: its start point on the Gaussian surface (word 0), or the
        // next hop's point on its last square (word `hops`); starts and hops
        // share the Philox draw, the bin search and the perimeter mapping, so
        // a warp runs each once per hop ----
        int code = 0x7FFFFFFF;  // != ended
        for (int pass = 0; pass < kHopsPerRound; pass++) {
            const bool go = active && code == 0x7FFFFFFF;
            if (!__any_sync(kFull, go)) break;
            double px = 0, py = 0;
            if (go) {
                const uint32_t hop = (uint32_t)hops;
                const bool starting = hops == 0;
                if ((hop & 3) == 0) {
                    const uint4 b = draw_block(seed, job_of<kMulti>(P, job).stream_id, pw, hop);
                    s_rnd[0][threadIdx.x] = b.x;
                    s_rnd[1][threadIdx.x] = b.y;
                    s_rnd[2][threadIdx.x] = b.z;
                    s_rnd[3][threadIdx.x] = b.w;
                }
                const uint32_t word = s_rnd[hop & 3][threadIdx.x];
                double u = (double)word * 0x1p-32;
                if (starting) {
                    if (kUniform)
                        perim = __dadd_rn(__dmul_rn(2.0, __dsub_rn(sq[2], sq[0])), __dmul_rn(2.0, __dsub_rn(sq[3], sq[1])));
                    if (P.start_strata) {  // stratum pw mod S of the start distribution
                        const double s = (double)(uint32_t)(pw % P.start_strata);
                        u = __ddiv_rn(__dadd_rn(s, u), (double)P.start_strata);
                    }
                    if (P.start_grid) {  // midpoint of arc floor(u*Q) of Q equal arcs
                        const uint32_t q = (uint32_t)__dmul_rn(u, (double)P.start_grid);
                        u = __ddiv_rn(__dadd_rn((double)q, 0.5), (double)P.start_grid);
                        if ((kRec && P.rec_q) || kCV) bin1 = -2 - (int)q;  // the arc rides in bin1 until the first hop
                    }
                }
                if (starting && uniform_start) {
                    side = perimeter_point(sq, u, px, py);
                } else {
                    // the bin of the word itself (u = word / 2^32) unless a
                    // stratified or grid start moved u
                    const int bin = starting && (P.start_strata || P.start_grid) ? bin_of(s_intg, s_guide, u)
                                                                                : bin_of_word(s_thr, s_guide, word);
                    point_from_index(sq, bin, exact, px, py);
                    if (hop == 1) {
                        if (kRec && P.rec_q) P.rec_q[walk_index()] = (-2 - bin1) * FRW_NSAMPLE + bin;
                        if (kCV) cvq = (-2 - bin1) * FRW_NSAMPLE + bin;
                        bin1 = bin;
                        if (kUniform || kRec) a0 = __dsub_rn(sq[2], sq[0]);
                        if (kRec && P.rec_cv)
                            *reinterpret_cast<double2 *>(&P.rec_cv[walk_index()]) = make_double2(px, py);
                    }
                }
            }

            // ---- one query of every active walk ----
            if (go) {
                const WalkJob &J = job_of<kMulti>(P, job);
                const DevLayout &L = J.L;
                // distance to the bounds: p is strictly inside exactly when it is
                // > 0 (each difference is > 0 exactly when p is on that side)
                const double bd = fmin(fmin(px - L.bx0, L.bx1 - px), fmin(py - L.by0, L.by1 - py));
                if (!(bd > 0.0)) {
                    code = -1;  // escaped: left the layer bounds
                } else {
                    int hit;
                    // the rare tree traversal (overflowed cells) is a call in the
                    // 48-register kernel, whose code it would otherwise crowd
                    st |= query_point<true, !kUniform, kTies>(L, px, py, sq, hit, bd);
                    hops++;
                    if (hit != kNoHit) code = hit;
                    else if (hops >= P.hop_cap) code = -2;
                }
            }
        }
        const bool ended = active && code != 0x7FFFFFFF;

        // ---- walk ends: weight, optional records, lane sums or per-warp table ----
        double wgt = 0.0;
        bool ins = false;
        unsigned long long key = 0;
        if (ended) {
            double c = 0.0;  // weight factor: counts for the end conductor only
            if (uniform_start && bin1 >= 0) {
                const double nx = side == 1 ? 1.0 : (side == 3 ? -1.0 : 0.0);
                const double ny = side == 2 ? 1.0 : (side == 0 ? -1.0 : 0.0);
                const double dot = __dadd_rn(__dmul_rn(s_wx[bin1], nx), __dmul_rn(s_wy[bin1], ny));
                c = __ddiv_rn(__dmul_rn(__dmul_rn(-P.permittivity, perim), dot), a0);
            }
            if (code >= 0) wgt = c;
            if (kRec) {
                const uint64_t gw = walk_index();
                if (P.rec_end) P.rec_end[gw] = code;
                if (P.rec_hops) P.rec_hops[gw] = hops;
                if (P.rec_bin) P.rec_bin[gw] = bin1 < 0 ? -1 : bin1;
                if (P.rec_w) P.rec_w[gw] = c;
                if (P.rec_q && bin1 < 0) P.rec_q[gw] = -1;
                if (P.rec_cv) {  // first-hop point written at hop 1 (zero when there was none)
                    if (bin1 < 0) *reinterpret_cast<double2 *>(&P.rec_cv[gw]) = make_double2(0.0, 0.0);
                    reinterpret_cast<double2 *>(&P.rec_cv[gw])[1] = make_double2(a0, c);
                }
            }
            active = false;
            s_lhops[threadIdx.x] += (unsigned long long)hops;
            if (kCV) {  // z = c (y - phi(q, first bin)), as the records-based gather computes it
                const double yv = (int64_t)code == job_of<kMulti>(P, job).target ? 1.0 : 0.0;
                const double f = cvq >= 0 ? (double)__ldg(P.cv_phi + cvq) : 0.0;
                const double z = __dmul_rn(c, __dsub_rn(yv, f));
                s_cvz[0][threadIdx.x] = __dadd_rn(s_cvz[0][threadIdx.x], z);
                s_cvz[1][threadIdx.x] = __dadd_rn(s_cvz[1][threadIdx.x], __dmul_rn(z, z));
            }
            if ((int64_t)code == job_of<kMulti>(P, job).target) {
                pn++;
                if (kUniform) {
                    ps = __dadd_rn(ps, wgt);
                    ps2 = __dadd_rn(ps2, __dmul_rn(wgt, wgt));
                }
            } else {
                ins = true;
                key = ((unsigned long long)job << 32) | (uint32_t)(code + 2);
            }
        }
        tab_round<kMulti, kUniform>(P, tab, lane, lt, ins, key, 1ull, wgt, __dmul_rn(wgt, wgt));
    }
    __syncwarp();
    tab_round<kMulti, kUniform>(P, tab, lane, lt, pn > 0, target_key(pjob), pn, ps, ps2);
    if (s_lhops[threadIdx.x]) atomicAdd(P.job_stats + 4 * pjob + 2, s_lhops[threadIdx.x]);
    tab_flush<kMulti, kUniform>(P, tab, lane);
    if (kCV) {
        double z1 = s_cvz[0][threadIdx.x], z2 = s_cvz[1][threadIdx.x];
#pragma unroll
        for (int o = 16; o > 0; o >>= 1) {
            z1 = __dadd_rn(z1, __shfl_xor_sync(kFull, z1, o));
            z2 = __dadd_rn(z2, __shfl_xor_sync(kFull, z2, o));
        }
        if (lane == 0) {
            atomicAdd(P.cv_sums, z1);
            atomicAdd(P.cv_sums + 1, z2);
        }
    }
    if (st) atomicOr(P.status, st);
}

// Rows with a nonzero count, in no particular order; entries past `cap` are
// counted but not written (the caller compares *count with cap).
__global__ void k_compact(const unsigned long long *__restrict__ acc_n, const double *__restrict__ acc_s,
                          const double *__restrict__ acc_s2, int64_t rows, int64_t *__restrict__ out_row,
                          unsigned long long *__restrict__ out_n, double *__restrict__ out_s,
                          double *__restrict__ out_s2, unsigned long long *count, unsigned long long cap) {
    const int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
    const bool keep = i < rows && acc_n[i] > 0;
    const unsigned m = __ballot_sync(kFull, keep);
    if (!m) return;
    const int lane = threadIdx.x & 31, leader = __ffs(m) - 1;
    unsigned long long base = 0;
    if (lane == leader) base = atomicAdd(count, (unsigned long long)__popc(m));
    base = __shfl_sync(kFull, base, leader);
    const unsigned long long o = base + __popc(m & ((1u << lane) - 1u));
    if (keep && o < cap) {
        out_row[o] = i;
        out_n[o] = acc_n[i];
        out_s[o] = acc_s[i];
        out_s2[o] = acc_s2[i];
    }
}

}  // namespace

int walk_max_blocks_per_sm(int threads, bool multi, bool uniform) {
    int b = 0;
    if (multi) {
        if (uniform) cudaOccupancyMaxActiveBlocksPerMultiprocessor(&b, k_walk<true, false, true>, threads, 0);
        else cudaOccupancyMaxActiveBlocksPerMultiprocessor(&b, k_walk<true, false, false>, threads, 0);
    } else {
        if (uniform) cudaOccupancyMaxActiveBlocksPerMultiprocessor(&b, k_walk<false, false, true>, threads, 0);
        else cudaOccupancyMaxActiveBlocksPerMultiprocessor(&b, k_walk<false, false, false>, threads, 0);
    }
    return b;
}

namespace {
template <bool kTies>
void launch_variant(const WalkParams &P, bool multi, bool rec, bool uni, bool cv, dim3 g, dim3 b,
                    cudaStream_t stream) {
    if (cv) k_walk<false, false, true, true, kTies><<<g, b, 0, stream>>>(P);
    else if (multi && rec && uni) k_walk<true, true, true, false, kTies><<<g, b, 0, stream>>>(P);
    else if (multi && rec) k_walk<true, true, false, false, kTies><<<g, b, 0, stream>>>(P);
    else if (multi && uni) k_walk<true, false, true, false, kTies><<<g, b, 0, stream>>>(P);
    else if (multi) k_walk<true, false, false, false, kTies><<<g, b, 0, stream>>>(P);
    else if (rec && uni) k_walk<false, true, true, false, kTies><<<g, b, 0, stream>>>(P);
    else if (rec) k_walk<false, true, false, false, kTies><<<g, b, 0, stream>>>(P);
    else if (uni) k_walk<false, false, true, false, kTies><<<g, b, 0, stream>>>(P);
    else k_walk<false, false, false, false, kTies><<<g, b, 0, stream>>>(P);
}
}  // namespace

frw_status launch_walk(const WalkParams &P, int threads, int blocks, cudaStream_t stream) {
    if (threads != kWalkThreads) {
        set_error("launch_walk: threads per block must be 256");
        return FRW_E_ARG;
    }
    const bool rec = P.rec_end || P.rec_hops || P.rec_bin || P.rec_w || P.rec_q || P.rec_cv;
    const bool uni = P.start_mode == FRW_START_UNIFORM;
    const bool cv = P.cv_phi || P.cv_sums;
    if (cv && (!P.cv_phi || !P.cv_sums || P.njobs != 1 || rec || !uni || P.start_grid == 0)) {
        set_error("launch_walk: the control variate needs one job, no records and the uniform grid start");
        return FRW_E_ARG;
    }
    const dim3 g(blocks), b(threads);
    if (P.tree_points || P.job0.L.tree_points)
        launch_variant<true>(P, P.njobs > 1, rec, uni, cv, g, b, stream);
    else
        launch_variant<false>(P, P.njobs > 1, rec, uni, cv, g, b, stream);
    FRW_CK(cudaGetLastError());
    return FRW_OK;
}

frw_status launch_compact(const unsigned long long *acc_n, const double *acc_s, const double *acc_s2,
                          int64_t rows, int64_t *out_row, unsigned long long *out_n, double *out_s,
                          double *out_s2, unsigned long long *d_count, cudaStream_t stream, int64_t cap) {
    if (rows <= 0) return FRW_OK;
    k_compact<<<(unsigned)((rows + 255) / 256), 256, 0, stream>>>(acc_n, acc_s, acc_s2, rows, out_row, out_n,
                                                                  out_s, out_s2, d_count,
                                                                  (unsigned long long)(cap < 0 ? rows : cap));
    FRW_CK(cudaGetLastError());
    return FRW_OK;
}

}  // namespace frw
