/*
 * potts_b200.h — C ABI of the B200 (sm_100a) multiphase Potts segmentation solver.
 *
 * This library replaces the GPU path of the reference's potts-model tool:
 * the Chambolle–Cremers–Pock primal-dual iteration of
 * potts-model/potts-min-partition.{h,cpp} together with the minimal device
 * runtime it runs on (cuda-context/cuda-context.cpp, include/cuda-context.h,
 * include/cuda-details/*.h) and the cylindrical-core layout
 * (include/layout_cylinder.h).
 *
 * Conventions
 *  - Volumes use the reference's cylinder layout: index (n, row, col), n is
 *    the contiguous axis with stride `nstride` (a multiple of 32 floats), each
 *    column col stores rows [start_row[col], start_row[col] + rows_in_col)
 *    consecutively from offset base[col].  offset(n, row, col) =
 *    base[col] + (row - start_row[col]) * nstride + n
 *    (include/layout_cylinder.h:81-84).
 *  - Every function returns an int status (POTTS_OK = 0) and never throws;
 *    potts_last_error() gives a message for the calling thread.
 *  - All work is ordered on the context's stream.  A context is not
 *    thread-safe; use one context per host thread.
 *  - Plain pointers and sizes only; no C++ or framework types cross the ABI.
 */
#ifndef POTTS_B200_H
#define POTTS_B200_H

#include <stddef.h>
#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

/* include/cuda-context.h:7 — labels supported per solve: 2 .. POTTS_MAX_PHASES */
#define POTTS_MAX_PHASES 6

enum potts_status {
    POTTS_OK = 0,
    POTTS_EINVAL = 1,   /* bad argument (K, sizes, mapping, NaN parameters) */
    POTTS_ENOMEM = 2,   /* not enough device memory (potts-min-partition.cpp:571-577) */
    POTTS_ECUDA = 3,    /* a CUDA runtime call failed */
    POTTS_ETIMEOUT = 4, /* a bounded device-side wait gave up */
    POTTS_ENODEV = 5    /* no CUDA device / driver */
};

/* Host view of layout_cylinder::mapping (include/layout_cylinder.h:30-112).
 * The tables are read during the call and not retained. */
typedef struct potts_mapping {
    uint32_t n_images;         /* extent 0: number of slices along the cylinder axis */
    uint32_t rows;             /* extent 1 */
    uint32_t cols;             /* extent 2 */
    uint32_t nstride;          /* stride of the n axis (multiple of 32) */
    uint32_t col_begin;        /* first column holding rows */
    uint32_t col_end;          /* one past the last column holding rows */
    const uint32_t *start_row; /* [cols]   first stored row of each column */
    const uint32_t *base;      /* [cols+1] offset of each column; base[cols] = span */
} potts_mapping;

typedef struct potts_context potts_context; /* CudaContext (include/cuda-details/cuda-context-impl.h:35-65) */
typedef struct potts_field potts_field;     /* DeviceField<float> (include/cuda-details/device-field-impl.h:12-54) */

enum potts_variant {
    POTTS_VARIANT_FUSED = 0, /* one fused stencil launch per iteration (default) */
    POTTS_VARIANT_PLAIN = 1  /* the reference's split: a dual launch and a primal launch per iteration */
};

/* Storage of the solver state (Xi, V, Vbar).  Arithmetic is FP32 in every
 * format; the 16-bit formats round each stored value to nearest (ties to
 * even), also the Vbar the fused form keeps on chip, so that the fused and the
 * split forms give the same bits.  The reference stores FP32 only
 * (potts-min-partition.cpp:586-600); the 16-bit formats halve the bytes per
 * iteration.  Each format has its own list of compiled tile shapes. */
enum potts_storage {
    POTTS_STORE_F32 = 0,  /* FP32, as the reference */
    POTTS_STORE_BF16 = 1, /* bfloat16 (8-bit mantissa) */
    POTTS_STORE_F16 = 2,  /* IEEE binary16 (11-bit mantissa); Xi and V lie in [-1, 1] */
    POTTS_STORE_F64 = 3   /* FP64 state and FP64 arithmetic, always in the split kernel structure (the
                             variant option is ignored): the reference iteration in double precision,
                             the same bits as the FP64 CPU oracle; the yardstick of the other formats
                             on volumes too large for the CPU.  potts_solve_device rounds its V / Xi
                             outputs to FP32; potts_solve_device_f64 returns them in FP64. */
};

/* Arithmetic of the FP32 and 16-bit forms.  EXACT computes the reference's
 * IEEE single-precision operations in the reference's order (multiply-adds
 * fused where its clang build contracts them): every kernel form gives the
 * same bits as the FP32 CPU oracle.  FAST computes the same iteration with
 * fewer operations (the K-th label's terms derived from the others, no masks
 * on terms that are zero by construction, a sort-free simplex threshold,
 * reciprocal square roots in Dykstra's loop); it is held to the FP64 oracle
 * (relative L2 of V within 1e-5 and the same labels off ties on the
 * 128^3 case), and its split and fused forms give the same bits as each
 * other.  The FP64 state ignores this option. */
enum potts_arith {
    POTTS_ARITH_EXACT = 0,
    POTTS_ARITH_FAST = 1
};

typedef struct potts_options {
    int variant;      /* enum potts_variant */
    int storage;      /* enum potts_storage */
    int gap_every;    /* FP64 energies after every gap_every-th iteration; 0 = off */
    int slab_w;       /* 0: plan slabs from free memory like the reference; > 0: force this slab width */
    int track_dq;     /* 1: record max_x |V^{k+1} - V^k|^2 of every iteration on the device */
    int sync_monitor; /* 1: reference behaviour, read the monitor back and sync after every iteration */
    int tile_rows;    /* fused form: rows per tile (0 = default for K and arith) */
    int tile_slices;  /* fused form: slices (n) per tile (0 = default for K) */
    int segment_cols; /* fused form: columns one tile marches over (0 = 64, at most 64) */
    int tile_vpt;     /* fused form: consecutive slices per thread, 2 or 4 (0 = default for K) */
    int prefetch;     /* fused form: planes the load ring prefetches into L2 ahead of its loads
                         (0 = default: none, < 0 = none, at most 16) */
    int autotune;     /* batches: 1 = time every compiled tile shape and segment length, each as one
                         launch per iteration and as the persistent launch, on the batch and keep the
                         fastest (used when no tile option is set); 0 = default tile and launch form */
    int arith;        /* enum potts_arith (default EXACT) */
    int stall_plane;  /* testing the bounded waits: > 0 makes the fused kernel's first work item skip
                         the loads of that plane of its column march, so every wait for it gives up
                         after its limit (about 2 s) and the solve returns POTTS_ETIMEOUT with the
                         context still usable; 0 = off (default) */
    int persistent;   /* fused form: 1 = the iterations between two energy evaluations (all of them
                         without gap_every) run as one persistent cooperative launch that keeps every
                         block resident and passes a grid-wide barrier between iterations; batches
                         then capture a single iteration launch; 0 = one launch per iteration
                         (default 0; sync_monitor implies 0) */
} potts_options;

typedef struct potts_stats {
    int n_slabs;          /* out: slabs run */
    int slab_w;           /* out: slab width (n-slices) */
    int iters;            /* out: iterations per slab */
    float dq_last;        /* out: sqrt(max |dV|^2) of the last iteration (needs track_dq) */
    double solve_ms;      /* out: device time from init to argmax, all slabs */
    double loop_ms;       /* out: device time of the iteration launches (fused or split), all slabs */
    int loop_launches;    /* out: kernel launches inside loop_ms */
    int total_launches;   /* out: kernel launches of the whole solve */
    uint64_t state_bytes; /* out: device bytes held by the solver state */
    float *dq_trace;      /* in, optional: [iters] max |dV|^2 per iteration of the last slab (host) */
    double *energy_trace; /* in, optional: [3 * (iters / gap_every)] (lagrangian, dual, gap) (host) */
    int loop_iters;       /* out: iterations run inside loop_ms (the fused form's persistent launches run
                             many iterations each) */
} potts_stats;

/* Defaults: fused, FP32, no gap, planner-chosen slabs, track_dq = 1, no per-iteration sync. */
void potts_default_options(potts_options *opts);
const char *potts_status_string(int status);
const char *potts_last_error(void);

/* make_context() (cuda-context/cuda-context.cpp:18-20): device `device`, a new stream. */
int potts_context_create(int device, potts_context **out);
/* Same, but all work goes to the caller's cudaStream_t `stream` (not owned; NULL = the default stream). */
int potts_context_create_on_stream(int device, void *stream, potts_context **out);
void potts_context_destroy(potts_context *ctx);
int potts_context_synchronize(potts_context *ctx);
/* Kernel launches of the library on this context since the last solve began (a solve restarts the
 * count; the other calls add theirs); 0 for NULL.  No counterpart in the reference. */
long long potts_context_launches(const potts_context *ctx);
/* device_memory() (cuda-context/cuda-context.cpp:22-42): free bytes + bytes cached by this context. */
int potts_device_memory(potts_context *ctx, size_t *available, size_t *total);

/* DeviceField(mapping, stream, mr) (device-field-impl.h:24-33): uninitialised voxels. */
int potts_field_create(potts_context *ctx, const potts_mapping *map, potts_field **out);
/* upload() (cuda-context/cuda-context.cpp:49-57): copies `span` = base[cols] floats. */
int potts_field_upload(potts_context *ctx, const potts_mapping *map, const float *host, potts_field **out);
/* download() (cuda-context/cuda-context.cpp:59-77): synchronous; span must match. */
int potts_field_download(potts_context *ctx, const potts_field *field, float *host, uint64_t span);
float *potts_field_data(potts_field *field);
uint64_t potts_field_span(const potts_field *field);
void potts_field_destroy(potts_field *field);

/*
 * potts_min_partition<K> (potts-model/potts-min-partition.h:8-16,
 * potts-model/potts-min-partition.cpp:540-679).
 *   g        device field u in [0,1] (borrowed, not modified)
 *   cpu_map  host mapping of g (borrowed)
 *   ci       K labels in the normalised units of u (host array)
 *   lambda   data weight; tau1 primal step; tau2 dual step
 *   iters    iterations per slab (also the slab halo)
 *   result   out: new field with the mapping of g holding ci[argmax_i V_i]
 * opts / stats may be NULL.  Returns POTTS_ENOMEM where the reference prints
 * "Not enough memory" and returns an empty pointer.
 */
int potts_min_partition(potts_context *ctx, const potts_field *g, const potts_mapping *cpu_map, int K,
                        const float *ci, float lambda, float tau1, float tau2, int iters,
                        const potts_options *opts, potts_field **result, potts_stats *stats);

/*
 * Device-pointer form of the same solve.  d_u and every output are device
 * pointers laid out with `map` (span = base[cols] voxels per plane); each
 * output may be NULL:
 *   d_res     span floats: ci[argmax]                        (update_kernel)
 *   d_labels  span bytes:  argmax index
 *   d_V       (K-1) planes of span floats: relaxed V_0..V_{K-2} (V_{K-1} = 1 - sum)
 *   d_Xi      3(K-1) planes of span floats: dual field, plane 3*i + axis
 *             (axis 0 = n, 1 = row, 2 = col)
 * Voxels outside the mask and padding (n >= n_images) are not written.
 */
int potts_solve_device(potts_context *ctx, const potts_mapping *map, const float *d_u, int K, const float *ci,
                       float lambda, float tau1, float tau2, int iters, const potts_options *opts, float *d_res,
                       uint8_t *d_labels, float *d_V, float *d_Xi, potts_stats *stats);

/*
 * The same solve with the FP64 state (POTTS_STORE_F64 whatever opts->storage
 * says): V and Xi come back as FP64 planes (d_V: K-1 planes, d_Xi: 3(K-1)
 * planes of span doubles; each may be NULL).  The split kernels of
 * potts-model/potts-min-partition.cpp:96-488 in double precision.
 */
int potts_solve_device_f64(potts_context *ctx, const potts_mapping *map, const float *d_u, int K, const float *ci,
                           float lambda, float tau1, float tau2, int iters, const potts_options *opts, float *d_res,
                           uint8_t *d_labels, double *d_V, double *d_Xi, potts_stats *stats);

/*
 * Host-buffer form (what potts-model.cpp does around the call: upload, solve,
 * download).  h_u is span floats on the host (pinned memory is faster); the
 * outputs h_res (span floats) and h_labels (span bytes) may be NULL.  Blocks
 * until the results are on the host.
 */
int potts_solve_host(potts_context *ctx, const potts_mapping *map, const float *h_u, int K, const float *ci,
                     float lambda, float tau1, float tau2, int iters, const potts_options *opts, float *h_res,
                     uint8_t *h_labels, potts_stats *stats);

/*
 * FP64 energies (lagrangian, dual, gap) of a state (V, Xi), with the same
 * per-voxel terms as potts_stats.energy_trace, computed without allocating
 * device memory.  No counterpart in the reference.  For callers that cannot
 * call cudaMalloc (a host framework that owns the device memory pool, a
 * process whose device memory is reserved up front, a loop that cannot afford
 * an allocation's synchronisation).  Working memory is fixed, file-scope
 * device memory of the library (POTTS_STATIC_MAX_COLS column entries and one
 * partial sum per block, about 275 KB per GPU, held until the process exits).
 * d_u, d_V (K-1 planes) and d_Xi (3(K-1) planes) are device arrays laid out
 * with `map` (span = base[cols] per plane); h_out receives 3 doubles; the
 * work runs on `stream` (a cudaStream_t, NULL = default stream) on the
 * current device, and the call returns after the result is on the host.
 * Every call looks up the working memory's device address on the current
 * device (cudaGetSymbolAddress, which allocates nothing); the first lookup in
 * a process may load the library's device code, so make the first call before
 * any stream capture.  Every call uses the same working memory, so calls that
 * overlap on the GPU race; a call's working memory is fully rewritten before
 * it is read.  The mapping gets the same checks as in every solver entry
 * point, on the host, before anything runs on the GPU.  Returns POTTS_EINVAL
 * for more than POTTS_STATIC_MAX_COLS columns or an invalid mapping.
 */
#define POTTS_STATIC_MAX_COLS 16384
int potts_energies_static(const potts_mapping *map, const float *d_u, int K, const float *ci, float lambda,
                          const float *d_V, const float *d_Xi, void *stream, double *h_out);

/* ---------------------------------------------------------------------------
 * Batched solves.  No counterpart in the reference, whose caller solves one
 * volume per process run (potts-model/potts-model.cpp:139-179); the batch runs
 * a lambda / label sweep over many independent volumes of uneven size at once.
 *
 * potts_batch_create plans n volumes (each its own cylinder mapping, device u,
 * K labels and lambda; K, tau1, tau2, iters and the storage format are common)
 * and captures the whole schedule as three CUDA graphs on the context's
 * stream: set-up (per volume the u staging, init and first dual step),
 * iterations (iters - 1 launches, each ONE launch of the fused kernel over the
 * work items of every volume) and finish (per volume the last primal step and
 * the argmax).  Every potts_batch_run replays them back to back (events
 * between them time the iterations): it reads each volume's u and writes its
 * outputs again (u may change between runs; the pointers may not).  The fused
 * form only (opts->variant is ignored), no slabs (the state of all volumes must
 * fit in device memory, else POTTS_ENOMEM), gap_every is ignored.  Tile shape:
 * the options', or with opts->autotune = 1 the fastest compiled shape and
 * segment length measured on the batch (results do not depend on it).
 * ------------------------------------------------------------------------- */
typedef struct potts_batch potts_batch;

typedef struct potts_batch_volume {
    potts_mapping map; /* copied by potts_batch_create */
    const float *d_u;  /* device, map's span; read by every run */
    const float *ci;   /* [K] host labels, copied */
    float lambda;
    float *d_res;      /* optional device outputs in map's layout: ci[argmax] */
    uint8_t *d_labels; /* optional: argmax index */
    float *d_V;        /* optional: K-1 planes of map's span */
} potts_batch_volume;

typedef struct potts_batch_info {
    int n_volumes;
    int n_work;         /* work items of one iteration launch (all volumes) */
    int tile_rows, tile_slices, tile_vpt, segment_cols; /* the tile shape in use */
    uint64_t voxels;    /* in-mask voxels of all volumes */
    uint64_t state_bytes;
    int graph_launches; /* kernel launches in the captured graph */
    double autotune_ms; /* device time spent autotuning (0 without) */
    int persistent;     /* 1: the iterations run as one persistent launch, 0: one launch each */
} potts_batch_info;

int potts_batch_create(potts_context *ctx, int n_volumes, const potts_batch_volume *volumes, int K, float tau1,
                       float tau2, int iters, const potts_options *opts, potts_batch **out);
/* Replays the graph on the context's stream.  With stats: waits, then reports
 * solve_ms (the graph), loop_ms (its iteration launches), iters, the number of
 * volumes in n_slabs, dq_last / dq_trace as the maximum over the volumes. */
int potts_batch_run(potts_batch *batch, potts_stats *stats);
int potts_batch_get_info(const potts_batch *batch, potts_batch_info *info);
/* Per-volume trace of max |dV|^2 of the last run (needs track_dq): host [n_volumes * iters]. */
int potts_batch_read_dq(potts_batch *batch, float *host);
void potts_batch_destroy(potts_batch *batch);

/* ---------------------------------------------------------------------------
 * Differentiable solve.  No counterpart in the reference.
 *
 * potts_forward_ckpt runs `iters` iterations of the split form (FP32 state,
 * one slab; the same bits as potts_solve_device) on one volume, keeps the state
 * every ckpt_every iterations and after the last, and returns the segmentation
 * loss   L = -(1/|mask|) sum_x log(V_t(x) + eps)   (t = d_truth's label index
 * at x, V_K = 1 - sum V_i).  potts_backward recomputes each segment of
 * ckpt_every iterations from its checkpoint and runs the reverse-mode kernels
 * through it: dL/du into d_grad_u (device, map's span, zero outside the mask),
 * dL/dc_i and dL/dlambda (host, accumulated in FP64).  The nearest-label
 * initial state is piecewise constant in u and c and contributes nothing.
 * d_u and d_truth are read again by potts_backward: they must stay valid and
 * unchanged until then.  d_V (optional) receives V^iters (K-1 planes of span).
 * ------------------------------------------------------------------------- */
typedef struct potts_tape potts_tape;

int potts_forward_ckpt(potts_context *ctx, const potts_mapping *map, const float *d_u, const uint8_t *d_truth, int K,
                       const float *ci, float lambda, float tau1, float tau2, int iters, int ckpt_every, float eps,
                       float *d_V, double *loss, potts_tape **out);
int potts_backward(potts_tape *tape, float *d_grad_u, double *grad_ci, double *grad_lambda);
void potts_tape_destroy(potts_tape *tape);

/* ---------------------------------------------------------------------------
 * Column sharding of one volume: the iteration loop of potts_min_partition
 * (potts-model/potts-min-partition.cpp:625-660) over several GPUs, one shard
 * per GPU (a rank of an NCCL communicator), or over several shards that one
 * process holds on one context (their halos move by device copies).
 *
 * The active columns are split into contiguous ranges (potts_shard_partition:
 * about equal in-mask voxels).  Shard r owns the columns [cuts[r], cuts[r+1])
 * and holds the global columns [first, last) = one column before and two
 * after (where the volume has them).  Its u is the global u's span range
 * [base[first], base[last]) (potts_shard_bounds gives both).  Each iteration
 * is one fused launch per shard and an exchange of the Xi planes of one column
 * with each neighbour; at the end the convergence trace is reduced by max and
 * the FP64 energies by sum over all shards.  The owned voxels get the bits of
 * potts_solve_device with the same options (fused form; FP32, bfloat16 or
 * binary16 state).  Every rank must call potts_shard_solve with the same
 * iters and options.
 * ------------------------------------------------------------------------- */
typedef struct potts_shard potts_shard;

/* cuts[0 .. world]: cuts[0] = col_begin < cuts[1] < ... < cuts[world] = col_end. */
int potts_shard_partition(const potts_mapping *map, int world, uint32_t *cuts);
/* cols (optional, 4 values): first, last, own_begin, own_end (global columns);
   span (optional, 2 values): base[first], base[last] (the shard's span range in the global arrays). */
int potts_shard_bounds(const potts_mapping *map, const uint32_t *cuts, int world, int rank, uint32_t *cols,
                       uint64_t *span);
/* d_u: the shard's u (the global u + span[0]); not copied, must stay valid.  opts: as for
   potts_solve_device (fused form only; tile, arith, storage, gap_every, prefetch are used). */
int potts_shard_create(potts_context *ctx, const potts_mapping *map, const uint32_t *cuts, int world, int rank,
                       const float *d_u, int K, const float *ci, float lambda, float tau1, float tau2,
                       const potts_options *opts, potts_shard **out);
/* Shards of neighbouring ranks held by this process (one context). */
int potts_shard_link(potts_shard *left, potts_shard *right);
/* NCCL: the library loads libnccl.so.2 (the one already in the process, else the system's).
   id: 128 bytes, made on one rank and passed to every rank by the caller. */
int potts_nccl_unique_id(void *id);
int potts_nccl_comm_create(const void *id, int world, int rank, int device, void **comm);
int potts_nccl_comm_destroy(void *comm);
/* The shard exchanges with ranks rank - 1 and rank + 1 of comm (size world, this shard's rank). */
int potts_shard_set_nccl(potts_shard *shard, void *comm);
/* Solves: shards = every shard of this process (all ranks in order and linked, or one NCCL shard);
   d_res / d_labels / d_V (arrays of n pointers, or NULL; entries may be NULL): ci[argmax], the
   argmax and V (K-1 planes of the shard's span) for the owned voxels, in the shard's span layout.
   stats: dq_trace and energy_trace of the whole volume; timing of this process.  Blocks until done. */
int potts_shard_solve(potts_shard *const *shards, int n, int iters, float *const *d_res, uint8_t *const *d_labels,
                      float *const *d_V, potts_stats *stats);
void potts_shard_destroy(potts_shard *shard);

/* TV-L2 (ROF) denoising of a field in place: chambolle() of
 * totalvarmin/chambolle.cpp:220-276 (Chambolle's projection algorithm, xi and
 * v zero at the start, `iters` iterations of the div and grad steps, then
 * g <- g - lambda div xi).  The reference's caller (totalvarmin.cpp:140) uses
 * tau = 0.99 / 6 and 150 iterations.  variant: POTTS_VARIANT_FUSED (one launch
 * per iteration over 8 x 128 tiles marching along the columns, xi and v staged
 * in shared memory, xi ping-pong), POTTS_VARIANT_PLAIN (the reference's div and
 * grad launches) or 2 (one launch per iteration, v rebuilt per voxel from
 * global memory); all give the same bits.  stats
 * (optional): solve_ms, loop_ms, launches, dq_trace / dq_last of the
 * per-iteration max |dxi|^2. */
int potts_tv_denoise(potts_context *ctx, const potts_mapping *map, float *d_g, float lambda, float tau, int iters,
                     int variant, potts_stats *stats);

/* ---- Label-finding inputs: the GPU steps before the Potts solve --------------
 * Fields are device arrays laid out like `map` (the mapping's span of floats);
 * only in-mask voxels are read or written.  Results that the reference returns
 * as host values or vectors are written to host memory, and the call returns
 * after the stream has finished them. */

/* min_max() (include/min_max.h:7, min_max/min_max.cpp:18-81): min and max over
 * the in-mask voxels; FLT_MAX / -FLT_MAX for an empty mapping. */
int potts_min_max(potts_context *ctx, const potts_mapping *map, const float *d_field, float *out_min, float *out_max);
/* The same over the strictly positive values only: grad_min_max_kernel
 * (uv-hist/uv-hist-kernel.cpp:29-68), the v range of uv_hist. */
int potts_min_max_positive(potts_context *ctx, const potts_mapping *map, const float *d_field, float *out_min,
                           float *out_max);
/* grad_magn() (include/grad_magn.h:5-6, grad-magn/grad_magn.cpp:17-79): d_v =
 * 0.5 |central-difference gradient of d_u| at every in-mask voxel, -1 where a
 * neighbour along n, row or column is outside the mask.  Runs on the
 * context's stream; d_u and d_v must differ.  Fields of 16-byte lines (slice
 * count and stride multiples of 4, 16-byte aligned pointers) take the
 * column-march kernel, and the call then waits for it: POTTS_ETIMEOUT if one
 * of its bounded waits for a tile load gave up.  Other fields return with the
 * kernel enqueued. */
int potts_grad_magn(potts_context *ctx, const potts_mapping *map, const float *d_u, float *d_v);
/* calc_hist(ctx, in, range_start, range_end, nbins, delta) (include/calc_hist.h:12-13,
 * calc_hist/calc_hist.cpp:23-80,93-138): counts of nbins (1..65535) bins over
 * [range_start, range_end]; bin = round(nbins t - 0.5) clamped, t the position
 * in the range.  jitter > 0 adds a uniform value in [-jitter/2, jitter/2) to
 * every voxel and counts only voxels with range_start - jitter/2 <= x and
 * x + jitter/2 <= range_end, as the reference does; the reference draws the
 * jitter from a randomly seeded stream, here it is a function of (seed, voxel),
 * so a seed reproduces a histogram.  out_counts: nbins counts (host);
 * out_density (optional, host): counts / (in-mask voxels x bin width), the
 * reference's return value. */
int potts_calc_hist(potts_context *ctx, const potts_mapping *map, const float *d_field, float range_start,
                    float range_end, uint32_t nbins, float jitter, uint64_t seed, uint32_t *out_counts,
                    double *out_density);
/* calc_hist(ctx, in, nbins, delta) (include/calc_hist.h:9-10, calc_hist.cpp:82-91): the
 * same over [min, max] of the field, which are returned. */
int potts_calc_hist_auto(potts_context *ctx, const potts_mapping *map, const float *d_field, uint32_t nbins,
                         float jitter, uint64_t seed, uint32_t *out_counts, double *out_density, float *out_min,
                         float *out_max);
/* Layout of the 2-D histogram (uv-hist/uv-hist-kernel.cpp:112-118): row stride
 * (nbins rounded up to 32) and span ((nbins - 1) * stride + nbins counts). */
uint32_t potts_uv_hist_stride(uint32_t nbins);
uint64_t potts_uv_hist_span(uint32_t nbins);
/* uv_hist(ctx, u, v, u_start, u_end, v_start, v_end, nbins) (uv-hist/uv-hist.h:33-41,
 * uv-hist-kernel.cpp:100-197): counts of the pairs (u, v) in nbins x nbins bins,
 * row ybin (v) x column xbin (u), at ybin * stride + xbin of out_hist (host,
 * potts_uv_hist_span(nbins) counts). */
int potts_uv_hist(potts_context *ctx, const potts_mapping *map, const float *d_u, const float *d_v, float u_start,
                  float u_end, float v_start, float v_end, uint32_t nbins, uint32_t *out_hist);
/* uv_hist(ctx, u, v, nbins) (uv-hist/uv-hist.h:26-31, uv-hist-kernel.cpp:70-98): the
 * same over u in [min u, max u] and v in [min, max] of its strictly positive
 * values; out_ranges = {u_start, u_end, v_start, v_end}. */
int potts_uv_hist_auto(potts_context *ctx, const potts_mapping *map, const float *d_u, const float *d_v,
                       uint32_t nbins, uint32_t *out_hist, float *out_ranges);

/* ---- Field archive (.bin files) and the steps either side of the solve ------
 * The reference's tools exchange volumes as Field<T> archives: io::BinOArchive
 * of Field<T>::save (include/field.h:92-119, include/layout_cylinder.h:233-257,
 * include/io/writeprimitives.h, include/io/outbitstream.h).  One MSB-first bit
 * stream without an archive header: the mapping in Exp-Golomb codes (extents,
 * nstride, col_begin, col_end, the start_row and base tables as first value and
 * signed differences), for FP32 fields the bit patterns of lo and hi, then the
 * in-mask voxels column by column, row by row, n = 0 .. n_images-1, 32 bits
 * (FP32) or 16 bits (uint16) each.  The header is coded on the host; the voxel
 * payload is packed and unpacked on the GPU. */
enum potts_element {
    POTTS_ELEM_F32 = 0, /* Field<float>: 32-bit voxels, lo/hi in the header */
    POTTS_ELEM_U16 = 1  /* Field<uint16_t>: 16-bit voxels */
};

typedef struct potts_archive_info {
    uint32_t n_images, rows, cols, nstride, col_begin, col_end; /* the archive's mapping */
    uint64_t span;        /* elements of the device field it loads into (base[cols]) */
    float lo, hi;         /* Field<float>::lo()/hi() (include/field.h:79-80); 0 for uint16 */
    uint64_t header_bits; /* bits before the first voxel */
    uint64_t voxels;      /* in-mask voxels in the payload */
    uint64_t total_bytes; /* bytes of the whole archive */
} potts_archive_info;

typedef struct potts_io_stats {
    double kernel_ms; /* out: device time of the call's kernel (CUDA events around it) */
    int launches;     /* out: kernels launched */
} potts_io_stats;

/* mapping_storage::load (include/layout_cylinder.h:259-312) and the lo/hi of
 * Field<float>::load (include/field.h:121-131): parses the header of an archive
 * of element type `elem`.  start_row (cols entries) and base (cols + 1) are
 * optional; call once without them to learn cols.  POTTS_EINVAL when the bytes
 * end inside the header or the mapping is not one this library accepts. */
int potts_archive_read_header(const uint8_t *bytes, uint64_t n_bytes, int elem, potts_archive_info *info,
                              uint32_t *start_row, uint32_t *base);
/* Size in bytes of the archive of a field with this mapping (host only). */
int potts_archive_size(const potts_mapping *map, int elem, uint64_t *total_bytes, uint64_t *header_bits);
/* Field<T>::load (include/field.h:121-147) into device memory: the voxels of
 * the archive at `bytes` (host) are written to d_field (float or uint16_t
 * elements laid out by the archive's mapping, at least info.span elements =
 * `capacity`); padding slices are not written.  Returns after the copy. */
int potts_archive_load(potts_context *ctx, const uint8_t *bytes, uint64_t n_bytes, int elem, void *d_field,
                       uint64_t capacity, potts_archive_info *info, potts_io_stats *stats);
/* Field<T>::save (include/field.h:92-119) of a device field laid out by `map`
 * into host memory `out` (capacity bytes); lo/hi are stored for FP32 fields.
 * out = NULL only reports the size in *out_bytes. */
int potts_archive_save(potts_context *ctx, const potts_mapping *map, int elem, const void *d_field, float lo,
                       float hi, uint8_t *out, uint64_t capacity, uint64_t *out_bytes, potts_io_stats *stats);
/* convert_to_fp(ctx, in, lo, hi) (transpose/convert_to_fp.h:8-10,
 * transpose/convert_to_fp.cpp:11-79): d_out = 0 where v <= lo, 1 where v >= hi,
 * else (v - lo) / (hi - lo) in FP32, for a float or uint16 field.  Enqueued on
 * the context's stream; padding slices are not written. */
int potts_convert_to_fp(potts_context *ctx, const potts_mapping *map, int elem, const void *d_in, float lo, float hi,
                        float *d_out);
/* find_intensity_range(ctx, field, tail_thr) (transpose/find_intensity_range.h,
 * transpose/find_intensity_range.cpp:64-110): the 65536-bin histogram of a
 * uint16 field, lo = the last bin whose cumulative count is at most
 * tail_thr x total, hi = the first bin whose cumulative count reaches
 * (1 - tail_thr) x total, both narrowed to uint16 as the reference does.
 * out_hist (optional, host): the 65536 counts. */
int potts_find_intensity_range(potts_context *ctx, const potts_mapping *map, const uint16_t *d_field,
                               double tail_thr, uint16_t *out_lo, uint16_t *out_hi, uint64_t *out_hist);
/* Extent of the raw label box of potts-model.cpp:186-202: slices x rows x
 * cols, rows from the smallest first row to the largest end row of the columns
 * that hold rows, cols = col_end - col_begin; row_begin is the box's first row. */
int potts_raw_labels_dims(const potts_mapping *map, uint32_t *slices, uint32_t *rows, uint32_t *cols,
                          uint32_t *row_begin);
/* The raw label box (potts-model.cpp:203-217) in device memory: byte
 * ((c * rows + r) * slices + n) = min(255, max(0, round(255 v))) of voxel
 * (n, row_begin + r, col_begin + c) inside the mask, 255 outside.  Enqueued on
 * the context's stream. */
int potts_raw_labels(potts_context *ctx, const potts_mapping *map, const float *d_field, uint8_t *d_box);
/* The --rawout VTK ImageData file of potts-model.cpp:184-243 (XML header, the
 * box size as 4 little-endian bytes, the raw label box, XML footer) in host
 * memory; out = NULL only reports the size.  Byte-identical to the reference's
 * file for the same field. */
int potts_vtk_labels(potts_context *ctx, const potts_mapping *map, const float *d_field, uint8_t *out,
                     uint64_t capacity, uint64_t *out_bytes, potts_io_stats *stats);
/* write_png(img, col, lambda) (potts-model.cpp:34-49): the lines of column
 * `col` as an 8-bit grey PNG (rows down, slices across), grey =
 * saturate(round-half-even(255 |v|^(1/2.2))), as cv::pow + convertTo compute
 * it, here in FP64; written with stored deflate blocks.  out = NULL only
 * reports the size. */
int potts_png_slice(potts_context *ctx, const potts_mapping *map, const float *d_field, uint32_t col, uint8_t *out,
                    uint64_t capacity, uint64_t *out_bytes);

/* Mask constructor of layout_cylinder::mapping_storage (include/layout_cylinder.h:152-195):
 * fills start_row[cols] and base[cols+1], returns the span (base[cols]). */
uint64_t potts_cylinder_mapping(uint32_t rows, uint32_t cols, double xc, double yc, double r, uint32_t nstride,
                                uint32_t *start_row, uint32_t *base, uint32_t *col_begin, uint32_t *col_end);
/* Field<float>::get_stride (include/field.h:37-40): n rounded up to 32. */
uint32_t potts_get_stride(uint32_t n);

#ifdef __cplusplus
}
#endif

#endif /* POTTS_B200_H */
