/*
 * frw.h -- C ABI of the B200 floating-random-walk (FRW) capacitance extractor.
 *
 * Plain C types only (no CUDA or torch types): streams are passed as void*
 * (a cudaStream_t, NULL = the legacy default stream).  Every call returns an
 * frw_status; on failure frw_last_error() returns a thread-local message.
 * Nothing in the library calls exit(), cudaDeviceReset() or falls back to the
 * CPU: without an sm_100 device every compute entry point fails with
 * FRW_E_DEVICE.
 *
 * Correspondence with the reference (piogrzej/engineer-thesis, randomWalk/):
 *   frw_layout_from_file / frw_layout_create   <- createQuadTree
 *       (Cuda/mainkernels.h:10, Cuda/createquadtree.cu:16-87) and the layout
 *       reader d_Parser/Parser (Cuda/d_parser.cpp:16-130, CPU/Parser.cpp:15-125)
 *   frw_parse_layout                           <- Parser::parse + getLayerAt +
 *       getLayerSize (CPU/Parser.cpp:15-87), host only
 *   frw_layout_destroy                         <- freeQuadTreeManager
 *       (Cuda/mainkernels.h:13, Cuda/freequadtreemanager.cu:3-11)
 *   frw_query_batch                            <- d_QuadTree::drawBiggestSquareAtPoint
 *       + d_QuadTree::checkCollisons(point) (Cuda/d_quadTree.cu:86-134,28-69;
 *       CPU twins CPU/quadTree.cpp:264-312,240-262), batched
 *   frw_box_collides_batch                     <- Tree::checkCollisions(rect, ignore)
 *       (CPU/quadTree.cpp:148-198, Cuda/d_quadTree.cu:136-193), batched
 *   frw_gauss_surface                          <- Tree::creatGaussianSurfFrom
 *       (CPU/quadTree.cpp:315-364, Cuda/d_quadTree.cu:216-265)
 *   frw_walk_trace                             <- randomWalkCudaWrapper
 *       (Cuda/mainkernels.h:9, Cuda/randomwalk.cu:123-134): per-walk outputs
 *   frw_walk                                   <- the estimator of
 *       getAvgPathLenCUDA / getAvgPathLen (Cuda/getAvgPathLenCUDA.cu:50-80,
 *       CPU/getAvgPathLen.cpp:35-114): per-conductor hits and capacitance row
 *   frw_avg_path_len                           <- getAvgPathLenCUDA
 *       (Cuda/mainkernels.h:14): the reference's one-call entry point
 *   frw_green_table                            <- precompute_unit_square_green
 *       (green/green.h:50, green/green.cpp:125-152)
 *   frw_device_check                           <- initCuda (Cuda/initCuda.cu:9-33)
 */
#ifndef FRW_H
#define FRW_H

#include <stddef.h>
#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

typedef int frw_status;
#define FRW_OK 0
#define FRW_E_ARG (-1)      /* invalid argument or layout */
#define FRW_E_IO (-2)       /* unreadable or malformed layout file */
#define FRW_E_CUDA (-3)     /* a CUDA runtime call failed */
#define FRW_E_OOM (-4)      /* device or host allocation failed */
#define FRW_E_HOPCAP (-5)   /* reserved: walks hit the hop cap (reported as counts, not failure) */
#define FRW_E_TIMEOUT (-6)  /* a bounded host wait expired (frw_set_wait_limit, frw_opts.timeout_ms) */
#define FRW_E_DEVICE (-7)   /* no usable sm_100 device */
#define FRW_E_KERNEL (-8)   /* a kernel reported an internal limit (see frw_last_error) */

typedef struct frw_layout frw_layout;

#define FRW_NSAMPLE 200 /* perimeter bins of the Green's-function table (defines.h:28) */

/* ---- diagnostics ---- */
const char *frw_version(void);
const char *frw_last_error(void);
/* Checks that `device` exists and is compute capability 10.x (replaces the
 * reference's SM >= 3.5 dynamic-parallelism check, Cuda/initCuda.cu:14-31). */
frw_status frw_device_check(int device);

/* Bound on every host wait of the library, in ms (0, the default: none);
 * a call's frw_opts.timeout_ms, when set, replaces it for that call.  When a
 * wait passes the bound the call returns FRW_E_TIMEOUT: its device work keeps
 * running, ordered before later work on the same stream; the buffers that
 * work uses are released only after it (stream-ordered frees), and no result
 * has been copied into caller memory.  The destroy calls (frw_layout_destroy,
 * frw_cv_destroy, frw_batch_destroy, frw3_layout_destroy) wait for the device
 * without a bound, like cudaFree.  The reference has no such bound: its
 * wrappers end in cudaDeviceSynchronize (Cuda/getAvgPathLenCUDA.cu:50-80). */
frw_status frw_set_wait_limit(double ms);
double frw_get_wait_limit(void);

/* ---- Green's function table ---- */
/* g[FRW_NSAMPLE] and the normalised cumulative intg[FRW_NSAMPLE+1] of the
 * unit-square surface Green's function seen from the centre; bit-identical to
 * the reference's precompute_unit_square_green.  Either pointer may be NULL. */
frw_status frw_green_table(double *g, double *intg);

/* ---- layouts ---- */
/* Reads layer `layer` of a reference layout file (lines "rect x0 y0 x1 y1";
 * layers closed by "<<" lines, the first one skipped; CPU/Parser.cpp:15-50),
 * computes the reference bounds (bbox grown by int(0.01*width) on both axes,
 * CPU/Parser.cpp:51-87) and builds the device quadtree on `device`. */
frw_status frw_layout_from_file(const char *path, int layer, int device, frw_layout **out);
/* The reader alone, on the host (no device is touched): Parser::parse +
 * getLayerAt + getLayerSize (CPU/Parser.cpp:15-87) for layer `layer` of
 * `path`.  *n_out receives the layer's rect count; when rects_out is not NULL
 * and capacity >= *n_out, the rects (file order, n*4 doubles) are written
 * there, else FRW_E_ARG reports the count needed.  bounds_out (nullable)
 * receives the reference bounds, layers_out (nullable) the number of closed
 * layers.  As in the reference, a line of 50 or more characters ends the
 * reading (std::istream::getline into a 50-byte buffer fails there) and the
 * lines after it are ignored.  A rect line without exactly four numbers
 * (undefined in the reference) is FRW_E_IO with its line number; a layer
 * that the file does not close is FRW_E_ARG. */
frw_status frw_parse_layout(const char *path, int layer, double *rects_out, int64_t capacity, int64_t *n_out,
                            double *bounds_out, int32_t *layers_out);
/* rects_xyxy: host array of n*4 floats (x0,y0,x1,y1), y downwards; every
 * coordinate must be an integer-or-float value exactly representable in
 * FP32 with |c| < 2^24.  bounds: NULL for the reference rule, else 4
 * doubles that must contain every rect.  The build runs on `stream` and the
 * call returns when the layout is ready. */
frw_status frw_layout_create(const float *rects_xyxy, int64_t n, const double *bounds, int device,
                             void *stream, frw_layout **out);
frw_status frw_layout_destroy(frw_layout *layout);

typedef struct frw_layout_info {
    int64_t n_rects;
    int64_t n_nodes;       /* internal quadtree nodes */
    int32_t depth;         /* levels below the root */
    int32_t leaf_max;      /* rects per leaf */
    double bounds[4];      /* x0, y0, x1, y1 */
    int64_t device_bytes;  /* rects + ids + nodes */
    int32_t device;
    double build_ms;       /* device time of the last tree build */
} frw_layout_info;
frw_status frw_layout_info_get(const frw_layout *layout, frw_layout_info *info);
/* Cell lists (no counterpart in the reference, which answers every query
 * from its quadtree, CPU/quadTree.cpp:148-312): a uniform grid over the
 * layer bounds whose cells each list every rect that a clearance query from
 * inside the cell can find nearest, tied or containing the point.  Queries
 * scan their cell's list instead of descending the tree; cells whose list
 * would exceed max_per_cell fall back to the tree.  Results are identical
 * with and without them.  frw_layout_create builds them with 16 cells per rect
 * and at most 32 rects per cell; frw_layout_set_cells rebuilds them
 * (cells_per_rect = 0 removes them).  It synchronises the device and must
 * not run while another call uses the layout, nor while a batch or a control
 * variate built on it exists. */
typedef struct frw_cells_info {
    int64_t cells;           /* nx * ny, 0 when the layout has none */
    int32_t nx, ny;
    double cell_side;
    int64_t entries;         /* list entries in all cells */
    int64_t overflow_cells;  /* cells answered by the tree */
    int64_t device_bytes;
    double build_ms;
} frw_cells_info;
frw_status frw_layout_set_cells(frw_layout *layout, double cells_per_rect, int max_per_cell, void *stream);
frw_status frw_layout_cells_info(const frw_layout *layout, frw_cells_info *info);
/* Copies the layout's rects (layer order, as doubles) to a host array n*4. */
frw_status frw_layout_rects(const frw_layout *layout, double *out_xyxy);

/* ---- memory location flag for batch calls ---- */
#define FRW_MEM_HOST 0   /* pointers are host memory (copied through the stream) */
#define FRW_MEM_DEVICE 1 /* pointers are device memory on the layout's device */

/* ---- collision queries ---- */
/* For each point: the reference's maximal empty square at the point
 * (drawBiggestSquareAtPoint: p+-1, p+-2, then expand/bisect from
 * 0.05*max(W,H) down to 0.095) and the conductor containing it (closed; the
 * lowest layer index when several do; -1 when none).  Complete semantics:
 * a box collides when it leaves the layer bounds or touches ANY rect.
 * Results are bit-identical to the FP64 CPU reference algorithm. */
frw_status frw_query_batch(const frw_layout *layout, const double *pts_xy, int64_t n,
                           double *sq_xyxy_out, int64_t *hit_out, int mem, void *stream);
/* Tree::checkCollisions(box, ignore) per box: 1 when the box leaves the
 * layer bounds or touches a rect other than one equal to *ignore
 * (coordinate-wise; ignore may be NULL, host memory). */
frw_status frw_box_collides_batch(const frw_layout *layout, const double *boxes_xyxy, int64_t n,
                                  const double *ignore, uint8_t *out, int mem, void *stream);

/* ---- walks ---- */
#define FRW_GAUSS_SCALE 0   /* reference creatGaussianSurfFrom(target, param) (default 1.5) */
#define FRW_GAUSS_OFFSET 1  /* target grown by param on every side */
#define FRW_START_GREEN 0   /* reference start: Green CDF mapped on the Gaussian rectangle */
#define FRW_START_UNIFORM 1 /* uniform on the Gaussian perimeter; enables capacitance weights */

typedef struct frw_opts {
    uint32_t struct_size;    /* sizeof(frw_opts) */
    int32_t gauss_mode;      /* FRW_GAUSS_* */
    double gauss_param;      /* 1.5 (scale) or the offset */
    int32_t start_mode;      /* FRW_START_* */
    int32_t exact_perimeter; /* 0: perimeter truncated to int as the CPU reference
                                (rectHost.cpp:102-105); 1: as the GPU reference (d_Rect.cu:29-32) */
    int64_t hop_cap;         /* walks longer than this end as "aborted" */
    double permittivity;     /* F/m, default 8.854187817620e-12 (green/phys.h:18) */
    uint32_t stream_id;      /* Philox counter word 3: independent streams under one seed */
    /* launch tuning (0 = library choice / autotuned) */
    int32_t threads_per_block;
    int32_t blocks_per_sm;
    int32_t refill_min;      /* refill a warp only when at least this many lanes are idle */
    uint32_t start_grid;     /* uniform start only: 0 = continuous; Q > 0 = the Q midpoints of Q equal
                                arcs of the Gaussian perimeter (the start distribution a control
                                variate's exact mean is summed over) */
    uint64_t first_walk;     /* frw_walk: Philox index of its first walk.  Runs over disjoint walk
                                ranges are independent and their rows (hits, sum_w, sum_w2) add up
                                exactly to one run over the union: a run can be checkpointed as
                                (seed, stream_id, next first_walk, rows) and resumed. */
    uint32_t start_strata;   /* 0 = off; S > 0: walk w starts in stratum w mod S of the start
                                distribution, u = (w mod S + U) / S (U the walk's first uniform),
                                for either start mode.  Unbiased when the walk range covers every
                                stratum equally (walks and first_walk multiples of S); the reported
                                standard error stays the i.i.d. one, an upper bound. */
    double timeout_ms;       /* bound on this call's host waits, in ms (0: the process-wide limit of
                                frw_set_wait_limit, by default none); see frw_set_wait_limit */
} frw_opts;
void frw_opts_default(frw_opts *opts);

typedef struct frw_result {
    /* scalar outputs */
    uint64_t walks;
    uint64_t escaped;          /* left the layer bounds (potential 0) */
    uint64_t aborted;          /* reached hop_cap */
    uint64_t hops_total;       /* collision queries issued */
    double gauss[4];           /* Gaussian surface used */
    double fraction_other;     /* walks NOT ending on the target, escapes included:
                                  the value getAvgPathLen(CUDA) returns */
    double kernel_ms;          /* device time of the walk kernel */
    /* per-conductor rows, sorted by conductor index (caller-owned, host) */
    int64_t capacity;          /* length of the arrays below */
    int64_t n_entries;         /* conductors reached (may exceed capacity: rows truncated) */
    int64_t *conductor;        /* layer index */
    uint64_t *hits;            /* walks ending on it */
    double *cap;               /* capacitance C_t,k in F/m (uniform start; 0 otherwise) */
    double *cap_se;            /* its standard error */
    double *sum_w;             /* optional: sum of the weights (rows add exactly across ranks) */
    double *sum_w2;            /* optional: sum of the squared weights */
} frw_result;

/* Runs `walks` walks from the Gaussian surface of conductor `target`
 * (layer index) with Philox stream (seed, opts->stream_id).  Walk i's random
 * numbers depend only on (seed, stream_id, i, hop), so results do not depend
 * on launch configuration. */
frw_status frw_walk(const frw_layout *layout, int64_t target, uint64_t walks, uint64_t seed,
                    const frw_opts *opts, frw_result *result, void *stream);

/* The same walks accumulated into caller-owned DEVICE arrays, stream-ordered,
 * without host synchronisation (the reference's randomWalkCudaWrapper,
 * Cuda/mainkernels.h:9, leaves its outputs on the device the same way):
 * for every conductor k (layer index, arrays of layout->n entries)
 * hits[k] += walks ending on k, sum_w[k] += their weights, sum_w2[k] += the
 * squared weights; stats[0..3] += escaped, aborted, hops, walks done;
 * *status |= kernel limit bits (nonzero: see frw_walk's FRW_E_KERNEL).  The
 * caller clears the arrays once; runs over disjoint walk ranges add up, and
 * so do the arrays of several devices (one all-reduce).  Scratch comes from
 * the device's stream-ordered memory pool. */
frw_status frw_walk_device(const frw_layout *layout, int64_t target, uint64_t walks, uint64_t seed,
                           const frw_opts *opts, uint64_t *hits, double *sum_w, double *sum_w2,
                           uint64_t *stats, uint32_t *status, void *stream);

/* Sparse form of frw_walk_device's rows, for the multi-GPU exchange (no
 * reference counterpart: the reference runs on one GPU).  For every conductor
 * k of the layout with hits[k] > 0 one entry (k, hits[k], sum_w[k],
 * sum_w2[k]) goes to the DEVICE arrays idx, out_hits, out_sum_w, out_sum_w2,
 * in no particular order, at most `capacity` of them; *count (device) is set
 * to the number of such conductors, written or not -- above `capacity` the
 * caller has to retry with more room.  Stream-ordered, no host sync.  A
 * step's walks reach a few hundred conductors of a 10^6-rect layout, so
 * ranks exchange these entries instead of 3 * n dense numbers. */
frw_status frw_rows_compact(const frw_layout *layout, const uint64_t *hits, const double *sum_w,
                            const double *sum_w2, int64_t capacity, int64_t *idx, uint64_t *out_hits,
                            double *out_sum_w, double *out_sum_w2, uint64_t *count, void *stream);

/* Same walks with per-walk records (device or host arrays of `walks`
 * entries; any may be NULL): end conductor (layer index, -1 escaped,
 * -2 aborted), hop count, first-hop bin and the walk's capacitance weight
 * factor c = -eps*L*(W_bin . n)/a0 (0 without a first hop or in green-start
 * mode); the walk adds c to the conductor in `end` and nothing when it
 * escaped or was aborted.  The
 * reference's randomWalkCudaWrapper output pair (0/1 "other" flag and hit
 * rect) is derived from `end`. */
frw_status frw_walk_trace(const frw_layout *layout, int64_t target, uint64_t first_walk,
                          uint64_t walks, uint64_t seed, const frw_opts *opts, int64_t *end,
                          int32_t *hops, int32_t *bin1, double *weight, int mem, void *stream);

/* frw_walk_trace for callers that cannot allocate device memory during the
 * call (an application that owns all GPU memory through its own pool, a
 * real-time loop that forbids allocator latency, a plugin inside a host
 * process that manages the CUDA context).  It has no counterpart in the
 * reference.  end/hops/bin1/weight are DEVICE arrays of `walks` entries on
 * the layout's device, all required.  The walk kernel's scratch lives in a
 * fixed file-scope device array sized for layouts of at most 65,536 rects
 * (1.5 MiB, held by every GPU that loads the library until exit); larger
 * layouts are rejected with FRW_E_ARG.  The first call on a device resolves
 * the array's address (cudaGetSymbolAddress) -- make that first call before
 * any stream capture.  The address is kept for the life of the process: a
 * host application that resets the device (cudaDeviceReset) must not call
 * this entry point on that device afterwards.  All calls share the array and
 * the call clears it first, so calls that overlap on the GPU (other streams
 * or threads) race: serialise them.  Returns after the stream has drained
 * (the kernel status word is checked; opts->timeout_ms bounds that wait).
 * Results equal frw_walk_trace's. */
frw_status frw_walk_trace_static(const frw_layout *layout, int64_t target, uint64_t first_walk,
                                 uint64_t walks, uint64_t seed, const frw_opts *opts, int64_t *end,
                                 int32_t *hops, int32_t *bin1, double *weight, void *stream);

/* Gaussian surface of `target` under opts (scale mode runs the reference's
 * bisection on the device). */
frw_status frw_gauss_surface(const frw_layout *layout, int64_t target, const frw_opts *opts,
                             double out_xyxy[4], void *stream);

/* The reference's one-call entry point getAvgPathLenCUDA(path, ITER_NUM,
 * RECT_ID, measure, layer): parse, build, run iter_num walks from rect_id
 * (reference start and Gaussian surface) and return the fraction of walks
 * that did not end on rect_id.  The per-rect histogram is written to
 * hist_path in the reference's "<ts>wyniki.txt" format when not NULL. */
frw_status frw_avg_path_len(const char *path, int64_t iter_num, int64_t rect_id, int layer,
                            uint64_t seed, int device, const char *hist_path, double *fraction);

/* ---- batched walks: many layouts / targets in one persistent launch ----
 * Job j walks walks[j] times from targets[j] of layouts[j] (all layouts on
 * one device) with Philox stream opts->stream_id + j; its results equal a
 * frw_walk of that job alone with stream_id = opts->stream_id + j.  The
 * device work of a run is one captured CUDA graph (clears, Gaussian
 * surfaces, ONE multi-job walk launch, row compaction); frw_batch_run
 * replays it with a new seed.  No reference counterpart (the reference runs
 * one target of one layout per process). */
typedef struct frw_batch frw_batch;
typedef struct frw_tuning {
    uint32_t struct_size;   /* sizeof(frw_tuning) */
    int32_t blocks_per_sm;  /* resident walk blocks per SM (0: occupancy limit) */
    int32_t refill_min;     /* refill a warp when at least this many lanes are idle */
    int32_t chunk;          /* walks a warp claims per global atomic (32 .. 2^20) */
    double ms;              /* walk-kernel time of the tuning trial that chose it */
} frw_tuning;
frw_status frw_batch_create(const frw_layout *const *layouts, const int64_t *targets, const uint64_t *walks,
                            int32_t njobs, const frw_opts *opts, frw_batch **out);
/* Measured search over blocks_per_sm x refill_min x chunk on a proportional
 * sample of trial_walks walks of the batch; keeps and returns the fastest. */
frw_status frw_batch_tune(frw_batch *batch, uint64_t trial_walks, frw_tuning *chosen);
frw_status frw_batch_set_tuning(frw_batch *batch, const frw_tuning *tuning);
frw_status frw_batch_get_tuning(const frw_batch *batch, frw_tuning *tuning);
/* results: njobs caller-owned frw_result (capacity and arrays per job). */
frw_status frw_batch_run(frw_batch *batch, uint64_t seed, frw_result *results, void *stream);
frw_status frw_batch_destroy(frw_batch *batch);

/* ---- learned control variate (no reference counterpart) ----
 * For C_tt the walk estimate is w = c * 1{end = t} (c: first-hop weight
 * factor).  The control variate is f = c * phi(x1), phi an MLP (16 -> 64 ->
 * 64 -> 1, SiLU; BF16 tensor-core kernels with FP32 accumulation) of 16
 * edge features of the first-hop point x1: (dx, dy) to the nearest point of
 * each edge of the target and of the nearest other conductor, divided by the
 * first square's side, clamped to +-16.  It is trained on the device on
 * walks of an independent seed (weighted least squares, weight c^2, Adam),
 * and E[f] is summed exactly over the start grid (opts.start_grid = Q, a
 * power of two) x the 200 first-hop bins, so  mean(w - f) + E[f]  is an
 * unbiased estimate of C_tt; frw_cv_walk reports it next to the plain
 * estimate from the same walks.  On the grid start the first-hop point is a
 * function of (arc, bin), so the exact-mean pass keeps phi of all Q x 200
 * points in a table (4 bytes each) and frw_cv_walk looks each walk's phi up
 * there: its walks cost about what plain walks cost. */
typedef struct frw_cv frw_cv;
typedef struct frw_cv_opts {
    uint32_t struct_size;  /* sizeof(frw_cv_opts) */
    uint64_t train_walks;  /* walks generating training pairs (default 1e6) */
    uint64_t train_seed;   /* independent of the estimation seed */
    int32_t epochs;        /* passes over the training pairs (default 4) */
    int32_t batch;         /* rows per Adam step, a multiple of 64 (default 32768) */
    float lr;              /* Adam step size (default 6e-3) */
} frw_cv_opts;
void frw_cv_opts_default(frw_cv_opts *opts);
typedef struct frw_cv_info {
    double mean_term;      /* E[f], exact over start grid x first-hop bins */
    double train_loss;     /* weighted MSE over the last epoch */
    double train_ms;       /* training walks + features + fit (device time) */
    double quad_ms;        /* exact-mean sum (device time) */
    uint64_t train_walks;
    uint32_t quad_points;  /* Q * 200 */
} frw_cv_info;
typedef struct frw_cv_result {
    uint64_t walks;
    double plain, plain_se;  /* C_tt from the plain estimator */
    double cv, cv_se;        /* C_tt with the control variate */
    double variance_ratio;   /* plain variance / control-variate variance */
    double kernel_ms;        /* device time of walks + phi look-up + sums */
} frw_cv_result;
/* walk_opts must use FRW_START_UNIFORM with start_grid a power of two <= 2^23. */
frw_status frw_cv_train(const frw_layout *layout, int64_t target, const frw_opts *walk_opts,
                        const frw_cv_opts *cv_opts, frw_cv **out, void *stream);
frw_status frw_cv_info_get(const frw_cv *cv, frw_cv_info *info);
frw_status frw_cv_walk(const frw_cv *cv, uint64_t walks, uint64_t seed, frw_cv_result *result,
                       void *stream);
/* How frw_cv_walk runs its walks (process-wide): FRW_CV_WALK_FUSED, the
 * default -- one walk launch that looks phi up at every walk's end and keeps
 * the sums of z = c (y - phi) beside the rows -- or FRW_CV_WALK_RECORDS,
 * per-walk records in chunks of 2^23 walks summed by a second kernel.  Both
 * give the same estimates up to the order of the FP64 sums. */
#define FRW_CV_WALK_FUSED 0
#define FRW_CV_WALK_RECORDS 1
frw_status frw_cv_set_walk_mode(int mode);
int frw_cv_get_walk_mode(void);
frw_status frw_cv_destroy(frw_cv *cv);
#define FRW_CV_PARAMS 5313 /* W1[64][16] b1[64] W2[64][64] b2[64] w3[64] b3 */
frw_status frw_cv_params(const frw_cv *cv, float *out);
/* Which tensor-core kernels run the MLP (process-wide): FRW_MLP_TCGEN05, the
 * default -- 128-row tiles on the fifth-generation tensor cores (tcgen05.mma,
 * accumulators in tensor memory), every weight and bias gradient a tensor-core
 * product accumulated over the tiles -- or FRW_MLP_MMA_SYNC, 16-row warp
 * tiles of mma.sync.  Both compute the same function (BF16 operands, FP32
 * accumulation) up to the order of the FP32 sums. */
#define FRW_MLP_TCGEN05 0
#define FRW_MLP_MMA_SYNC 1
frw_status frw_mlp_set_kernels(int which);
int frw_mlp_get_kernels(void);
/* The MLP and feature kernels on host arrays (FP32 in, BF16 operands on the
 * device): forward outputs, and the gradient of
 * sum_r wt_r (f(x_r) - y_r)^2 * inv_wsum with the summed loss. */
frw_status frw_mlp_forward(const float *params, const float *x, int64_t n, float *out, int device);
frw_status frw_mlp_grad(const float *params, const float *x, const float *y, const float *wt, int64_t n,
                        double inv_wsum, float *grad, double *loss, int device);
/* features of points rec4 = n x (x, y, a0, unused) relative to `target` */
frw_status frw_cv_features(const frw_layout *layout, int64_t target, const double *rec4, int64_t n,
                           float *out);

/* ---- synthetic layouts ---- */
/* Seeded generator of the benchmark layouts: n rects with integer corners in
 * [0, domain]^2, width and height uniform integers in [wmin, wmax], rejected
 * unless their L-infinity gap to every earlier rect is >= gap (splitmix64
 * stream from `seed`).  Writes n*4 floats; returns FRW_E_ARG when the domain
 * cannot hold n rects within 64*n attempts. */
frw_status frw_generate_layout(uint64_t seed, int64_t n, double domain, int32_t wmin,
                               int32_t wmax, double gap, float *out_xyxy);
/* Writes rects as a reference layout file (one layer). */
frw_status frw_write_layout(const char *path, const float *rects_xyxy, int64_t n,
                            const char *layer_name);

#ifdef __cplusplus
}
#endif
#endif /* FRW_H */
