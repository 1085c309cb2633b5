/*
 * knng.h -- C ABI of the B200 k-NN graph builder (libknng.so).
 *
 * The library builds an approximate k-nearest-neighbour graph (squared L2) with
 * the method of the reference's SolutionKmeans: repeated recursive 2-means
 * splitting of the point set into buckets, an all-pairs pass inside every
 * bucket into a bounded per-point neighbour set, and an optional
 * neighbour-of-neighbour refinement pass.  Every stage runs as sm_100a CUDA
 * kernels; the host code only sequences them.
 *
 * The reference has no plugin or FFI layer: its boundary is C++ linkage to
 * header-only static members called by main() (src/main.cpp:59).  Each entry
 * point below names the reference function it replaces.
 *
 * Conventions
 *   - Every call returns a knng_status; nothing throws across the ABI.
 *   - Points are row-major float32, n rows of d values, row stride ld_bytes
 *     (ld_bytes >= 4*d).  Host pointers unless the name says _device.
 *   - Output rows are sorted by (distance, id) ascending; rows with fewer than
 *     k neighbours are padded with id 1 (distance +inf), as padResult does.
 *   - A context is not re-entrant: one host thread at a time.  Use several
 *     contexts for concurrency.
 *   - Arithmetic: squared distances and hyperplane side tests use the
 *     reference's FP32 evaluation order (8 FMA lanes over dims l, l+8, ...,
 *     lanes summed left to right, tail dims added one by one), so given the
 *     same hyperplanes and buckets the results are bit-identical to the
 *     reference's.
 */
#ifndef KNNG_H
#define KNNG_H

#include <stddef.h>
#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

typedef struct knng_context knng_context;

typedef enum knng_status {
    KNNG_OK = 0,
    KNNG_ERR_INVALID_ARGUMENT = 1, /* null pointer, size out of range, bad stride */
    KNNG_ERR_CUDA = 2,             /* a CUDA runtime call failed; see knng_last_error */
    KNNG_ERR_OUT_OF_MEMORY = 3,    /* device allocation failed */
    KNNG_ERR_BUDGET = 4,           /* the request exceeds the context's HBM budget */
    KNNG_ERR_STATE = 5,            /* call out of order, e.g. no points loaded */
    KNNG_ERR_UNSUPPORTED = 6,      /* d or k outside the compiled set */
    KNNG_ERR_NO_DEVICE = 7,        /* no CUDA device, or the device is not sm_100 */
    KNNG_ERR_PENDING = 8           /* a served job has not ended yet */
} knng_status;

enum {
    KNNG_PRECISION_FP32 = 0,       /* exact FP32 distances everywhere (bit-exact form) */
    KNNG_PRECISION_BF16_RERANK = 1 /* bucket distances estimated in BF16 on the tensor cores (FP32
                                      accumulation, FP32 norms), each point's 128 best candidates
                                      re-ranked with exact FP32 distances; buckets <= 512 points */
};

/* Build parameters.  knng_default_params() fills the reference's values. */
typedef struct knng_params {
    uint32_t k;               /* neighbours per point, 1..128 (reference k = 100, src/Constants.hpp:24) */
    uint32_t max_leaf;        /* a node is a bucket iff its size < max_leaf (maxGroupSize,
                                 src/SolutionKmeans.hpp:152); reference alternates 200/400 */
    uint32_t max_leaf_odd;    /* if nonzero, odd repetitions use this max_leaf (the 200/400
                                 alternation of src/SolutionKmeans.hpp:582-587); 0 = max_leaf */
    uint32_t lloyd_iters;     /* 2-means iterations per split (knnIterations, :591) */
    uint32_t reps;            /* repetitions of split + bucket pass (the loop at :579-602) */
    uint32_t refine;          /* neighbour-of-neighbour passes after the repetitions (topUpSingle,
                                 :604; the reference runs 1) */
    uint32_t small_threshold; /* nodes below this size run Lloyd over all their points (:156, 3000) */
    uint32_t precision;       /* KNNG_PRECISION_* */
    uint64_t seed;            /* keys the device's counter-based RNG */
} knng_params;

/* Per-call statistics.  Times come from CUDA events on the context's stream. */
typedef struct knng_stats {
    double ms_total;          /* whole call, device time */
    double ms_split;          /* tree construction (seeding, Lloyd, side test, partition) */
    double ms_leaf;           /* bucket all-pairs + neighbour-set updates */
    double ms_leaf_kernel;    /* sum of bucket-kernel durations alone */
    double ms_refine;         /* neighbour-of-neighbour pass */
    double ms_finalize;       /* sort + pad */
    uint64_t reps_done;
    uint64_t split_levels;    /* tree levels over all repetitions */
    uint64_t split_nodes;     /* nodes split over all repetitions */
    uint64_t restarts;        /* split attempts repeated (empty cluster / side) */
    uint64_t fallback_splits; /* nodes split at the index midpoint after repeated failure */
    uint64_t buckets;         /* buckets processed over all repetitions */
    uint64_t bucket_pairs;    /* sum over buckets of b*(b-1)/2 */
    uint64_t bucket_pair_evals; /* distances the bucket kernel evaluated (ordered pairs) */
    uint64_t leaf_launches;   /* bucket-kernel launches */
    uint64_t kernel_launches; /* all kernels launched by the call */
    uint64_t refine_changed;  /* points whose set changed in the refinement pass */
    double ms_refine_join;    /* refinement: tensor-core join, direct pass (every point) */
    double ms_refine_apply;   /* refinement: survivor lists + sorted replay */
    double ms_refine_fallback;/* refinement: per-point pass for points with a lost record */
    uint64_t refine_pairs;    /* (point, candidate) pairs the join evaluated */
    uint64_t refine_filter_pass; /* pairs the tensor-core bound could not reject */
    uint64_t refine_member_skip; /* of those, candidates already in the point's list */
    uint64_t refine_exact;    /* exact FP32 distances computed by the join */
    uint64_t refine_emits;    /* survivor records written (before de-duplication) */
    uint64_t refine_overflow; /* survivor records past their point's slots (pooled) */
    double ms_refine_prep;    /* refinement: snapshot, reverse lists, scans */
    uint64_t refine_join_launches; /* join-kernel launches */
    uint64_t refine_lost;     /* points redone by the per-point pass (pool region full) */
    uint64_t refine_passes_done; /* neighbour-of-neighbour passes run, whichever kernel ran them */
    double recall_estimate;   /* knng_build_adaptive: recall on its sample at the end */
    uint64_t estimate_queries;/* knng_build_adaptive: sampled points */
} knng_stats;

/* Fills the reference's parameters: k=100, max_leaf=200, max_leaf_odd=400,
 * lloyd_iters=1, reps=8, refine=1, small_threshold=3000, FP32, seed=12345. */
void knng_default_params(knng_params* params);

const char* knng_status_string(knng_status status);

/* Creates a context on CUDA device `device`.  hbm_budget_bytes caps the
 * device memory the context may hold (0 = 90% of the device's memory, or
 * what is free when the context is created less 1 GiB, whichever is less). */
knng_status knng_create(int device, uint64_t hbm_budget_bytes, knng_context** out);
knng_status knng_destroy(knng_context* ctx);

/* Last error message of this context ("" if none). */
const char* knng_last_error(const knng_context* ctx);

/* ---------------------------------------------------------------- one call
 * Replaces SolutionKmeans::constructResult(points, numPoints, result)
 * (src/SolutionKmeans.hpp:558-616) with fixed repetition count instead of a
 * wall-clock budget.  out_ids: n*k uint32 (required); out_dists: n*k float
 * (optional, may be NULL); stats optional. */
knng_status knng_build(knng_context* ctx, const float* points, uint32_t n, uint32_t d, uint64_t ld_bytes,
                       const knng_params* params, uint32_t* out_ids, float* out_dists, knng_stats* stats);

/* Adaptive schedule, for a recall target instead of fixed counts or a time
 * budget (the reference repeats until a wall-clock bound, then tops up:
 * SolutionKmeans::constructResult, src/SolutionKmeans.hpp:579-604).  The
 * exact k nearest of `sample` evenly spaced points are found on the device
 * once (FP32 distances in the reference's order); after the first
 * min(2, params->reps) repetitions, neighbour-of-neighbour passes and further
 * repetitions are added -- a pass after each repetition, a second pass while
 * the target is missed, then another repetition -- until the recall
 * estimated on the sample reaches target_recall or params->reps repetitions
 * (0: up to 64) and params->refine passes have run.  stats->reps_done,
 * refine_passes_done and recall_estimate report what ran and reached. */
knng_status knng_build_adaptive(knng_context* ctx, const float* points, uint32_t n, uint32_t d, uint64_t ld_bytes,
                                const knng_params* params, double target_recall, uint32_t sample, uint32_t* out_ids,
                                float* out_dists, knng_stats* stats);

/* The same with device-resident input and output (pointers into the
 * context's device memory space); synchronous. */
knng_status knng_build_device(knng_context* ctx, const float* d_points, uint32_t n, uint32_t d, uint64_t ld_bytes,
                              const knng_params* params, uint32_t* d_out_ids, float* d_out_dists,
                              knng_stats* stats);

/* ---------------------------------------------------------------- stepwise
 * The stages one at a time, so that each can be fed the reference's
 * intermediate state and compared with it. */

/* Loads n points (copied into the context; on_device != 0: `points` is a
 * device pointer).  Resets indices to 0..n-1 and clears the neighbour sets. */
knng_status knng_load_points(knng_context* ctx, const float* points, uint32_t n, uint32_t d, uint64_t ld_bytes,
                             int on_device);

/* Clears every neighbour set and sets its capacity to k (1..128). */
knng_status knng_reset_sets(knng_context* ctx, uint32_t k);

/* indices = 0..n-1 (the std::iota at src/SolutionKmeans.hpp:589). */
knng_status knng_begin_rep(knng_context* ctx);

/* Stable partition of indices[starts[i], ends[i]) for `count` disjoint nodes,
 * by side = dot(coefs[i], point) >= offsets[i] with side-true points first
 * (the final-groups step, src/SolutionKmeans.hpp:188-205 and :262-304).
 * coefs: count*d floats.  out_mids[i] = starts[i] + number of side-true points. */
knng_status knng_split_nodes(knng_context* ctx, uint32_t count, const uint32_t* starts, const uint32_t* ends,
                             const float* coefs, const float* offsets, uint32_t* out_mids);

/* Farthest pair among the points at positions[offsets[i] .. offsets[i+1])
 * of indices (kmeansStartVecs, src/SolutionKmeans.hpp:68-138): out_first /
 * out_second are offsets into that list; out_ok[i] = 0 when no pair has a
 * distance above FLT_MIN. */
knng_status knng_farthest_pair(knng_context* ctx, uint32_t count, const uint64_t* offsets,
                               const uint32_t* positions, uint32_t* out_first, uint32_t* out_second,
                               int32_t* out_ok);

/* `iters` 2-means iterations per node from the given starting centres, over
 * the positions in lloyd_offsets/lloyd_positions, or over the whole node
 * [starts[i], ends[i]) when that node's list is empty (the Lloyd loops at
 * src/SolutionKmeans.hpp:161-186 and :218-260), then the final hyperplane.
 * out_ok[i] = 0 when an iteration left a cluster empty. */
knng_status knng_lloyd(knng_context* ctx, uint32_t count, const uint32_t* starts, const uint32_t* ends,
                       const uint64_t* lloyd_offsets, const uint32_t* lloyd_positions, const float* c1_start,
                       const float* c2_start, uint32_t iters, float* out_coefs, float* out_offsets,
                       int32_t* out_ok);

/* All-pairs pass over buckets [starts[i], ends[i]) of the current indices
 * (addCandidatesLessThan, src/KnnSets.hpp:131-160). */
knng_status knng_process_leaves(knng_context* ctx, uint32_t count, const uint32_t* starts, const uint32_t* ends);

/* One full device-seeded repetition: indices = iota, level-synchronous
 * recursive split, then every bucket (splitKmeansBinaryProcess,
 * src/SolutionKmeans.hpp:142-311).  rep_index keys the RNG. */
knng_status knng_run_rep(knng_context* ctx, uint32_t max_leaf, uint32_t lloyd_iters, uint32_t small_threshold,
                         uint64_t seed, uint32_t rep_index, knng_stats* stats);

/* Random-rotation KD splitter, the reference's alternative solution
 * (SolutionRandomKD, src/SolutionRandomKD.hpp:258-375, disabled at
 * src/main.cpp:58), behind the same side test, partition and bucket pass:
 * one repetition -- indices = iota, new_dims (1..32) rotated dimensions from
 * the rotation of knng_kd_rotation(new_dims, d, seed + rep_index), nodes of at
 * least max_leaf points split at the mean of a rotated dimension drawn with
 * probability proportional to its variance (the draw from a counter RNG
 * keyed by the node), points below the mean first, then every bucket.  The
 * node's own points give the statistics (the reference reads the first
 * `size` entries of the whole permutation instead). */
knng_status knng_run_rep_kd(knng_context* ctx, uint32_t max_leaf, uint32_t new_dims, uint64_t seed,
                            uint32_t rep_index, knng_stats* stats);

/* A whole build with the KD splitter, replacing
 * SolutionRandomKD::constructResult (src/SolutionRandomKD.hpp:377-430: five
 * iterations of rotateRandom + split with buckets below 400 points, then
 * finalize + padResult): loads the points (as knng_build), empty sets of
 * params->k, params->reps knng_run_rep_kd repetitions (rep_index 0, 1, ...;
 * buckets below max_leaf, or max_leaf_odd on odd repetitions when nonzero),
 * params->refine neighbour-of-neighbour passes (the reference's KD form has
 * none), then the sorted, padded lists as knng_build writes them.
 * params->precision must be KNNG_PRECISION_FP32; lloyd_iters and
 * small_threshold are not used.  new_dims: 1..32 (the reference: 30). */
knng_status knng_build_kd(knng_context* ctx, const float* points, uint32_t n, uint32_t d, uint64_t ld_bytes,
                          const knng_params* params, uint32_t new_dims, uint32_t* out_ids, float* out_dists,
                          knng_stats* stats);

/* The rotation of the KD splitter, made on the host as rotateRandom makes it
 * (src/SolutionRandomKD.hpp:258-264): new_dims vectors of d normal draws on a
 * std::mt19937 seeded with `seed` (the reference's generator starts at
 * 12345), each divided by its norm, then the reference's Gram-Schmidt
 * (src/LinearAlgebra.hpp:211-222).  out: new_dims x d floats.  No device. */
knng_status knng_kd_rotation(uint32_t new_dims, uint32_t d, uint64_t seed, float* out);

/* Bucket-pass autotuner (no counterpart in the reference; the reference has a
 * single CPU loop, src/KnnSets.hpp:131-160).  Times the FP32 bucket-pass
 * variants on one repetition of the context's own points and current sets
 * (max_leaf, lloyd_iters, small_threshold, seed as knng_run_rep, rep_index 0),
 * restoring the sets before each trial and after the last: 0 = every pair's
 * distance, 2 persistent CTAs per SM (the default); 1 = the same, 1 CTA per
 * SM; 2 = distances only for pairs a tensor-core filter cannot rule out, 2
 * CTAs per SM; 3 = the same, 1 CTA per SM.  All four give the same sets.  The
 * fastest is kept for the context's later repetitions.  out_ms[4] (optional):
 * each variant's bucket-pass ms; *out_choice (optional): the variant kept. */
knng_status knng_tune_buckets(knng_context* ctx, uint32_t max_leaf, uint32_t lloyd_iters, uint32_t small_threshold,
                              uint64_t seed, double* out_ms, uint32_t* out_choice);

/* Leaf ranges of the last knng_run_rep, in position order. */
knng_status knng_get_leaves(knng_context* ctx, uint32_t capacity, uint32_t* starts, uint32_t* ends,
                            uint32_t* out_count);

/* Neighbour-of-neighbour pass (topUpSingle, src/SolutionKmeans.hpp:480-555),
 * candidates offered in ascending id order.  out_changed and stats (its
 * refinement fields are added to) may be NULL. */
knng_status knng_refine(knng_context* ctx, uint64_t* out_changed, knng_stats* stats);

knng_status knng_get_indices(knng_context* ctx, uint32_t* out);
knng_status knng_set_indices(knng_context* ctx, const uint32_t* in);

/* Raw neighbour-set state in slot order (the fields of KnnSetScannableSimd,
 * src/KnnSets.hpp:26-31): dist/ids n*k, size n, maxslot n (0xFFFFFFFF while
 * not full), bound n (FLT_MAX while not full).  Any pointer may be NULL. */
knng_status knng_get_sets(knng_context* ctx, float* dist, uint32_t* ids, uint32_t* sizes, uint32_t* maxslot,
                          float* bounds);
knng_status knng_set_sets(knng_context* ctx, const float* dist, const uint32_t* ids, const uint32_t* sizes,
                          const uint32_t* maxslot, const float* bounds);

/* Snapshot / resume of the neighbour sets (no counterpart in the reference):
 * knng_save_sets writes the sets of the loaded points (distances, ids, sizes,
 * max slots, bounds, with n and k) to a file; knng_load_sets reads such a
 * file into a context holding the same points (same n), so that a build
 * continues from it with further repetitions (knng_run_rep with the next
 * rep_index), refinement passes and knng_finalize. */
knng_status knng_save_sets(knng_context* ctx, const char* path);
knng_status knng_load_sets(knng_context* ctx, const char* path);

/* Sorted, padded output (finalize + padResult, src/KnnSets.hpp:113-126,
 * :334-344): out_ids n*k, out_dists n*k (may be NULL). Host pointers. */
knng_status knng_finalize(knng_context* ctx, uint32_t* out_ids, float* out_dists);

/* -------------------------------------------------------------- diagnostics
 * No counterpart in the reference.  Runs one 128 x 128 tensor-core tile
 * (tcgen05.mma kind::f16, the tile the refinement pass filters with) on
 * a (m x d) and b (n x d), m, n <= 128, writing out[i*n + j] = a_i . b_j
 * with both operands rounded to FP16 and FP32 accumulation. */
knng_status knng_debug_tile_gram(knng_context* ctx, const float* a, uint32_t m, const float* b, uint32_t n,
                                 uint32_t d, float* out);

/* The same with BF16 operands (tcgen05.mma kind::f16, FP32 accumulation): the
 * tile the precision form estimates bucket distances with.  No counterpart in
 * the reference. */
knng_status knng_debug_tile_gram_bf16(knng_context* ctx, const float* a, uint32_t m, const float* b, uint32_t n,
                                      uint32_t d, float* out);

/* Poll limit of the waits the tree-construction and refinement kernels make
 * on their own bulk copies and tensor-core operations, on the context's device
 * (default 2^26 polls).  After a wait runs out the kernel records the failure,
 * drains its copies in flight with the default limit and returns; the call
 * reports KNNG_ERR_CUDA and the context stays usable.  A test sets a limit of
 * 0 to make every such wait run out.  No counterpart in the reference. */
knng_status knng_debug_set_wait_limit(knng_context* ctx, uint32_t polls);

/* ------------------------------------------------------ allocation-free pass
 * No counterpart in the reference.  For callers that cannot allocate device
 * memory during the call (code running inside another framework's memory pool
 * or under a hard memory cap, or holding only device pointers handed over by a
 * host application): the neighbour-of-neighbour pass of knng_refine, one warp
 * per point, on buffers the caller owns, allocating nothing.
 *
 *   d_points   n x d float32, rows packed (stride 4*d bytes), 16-byte aligned
 *   d_snapshot n x k uint32, written (each set's ids, sorted)
 *   d_dist, d_ids (n x k), d_size, d_maxslot, d_bound (n): the sets, in the
 *              layout of knng_get_sets; updated in place
 *   d_changed  one uint32, written: points whose set changed
 *   stream     cudaStream_t to run on (NULL: the default stream)
 * All pointers are device pointers on the current device.  The call is
 * asynchronous on `stream`.
 *
 * Its scratch is a fixed 32 MiB device array (2^22 survivor records) that
 * every GPU loading the library keeps until the process exits.  Each warp of
 * the launch owns one region of pow2(k*k) records, so the launch width follows
 * k: 256 warps at k = 100, 1,024 at k <= 64, 2,368 (16 per SM) at k <= 32.
 * k must be 1..128; larger k is rejected with KNNG_ERR_UNSUPPORTED before
 * anything runs.  Throughput: at k = 100 the pass runs about a tenth as many
 * warps as knng_refine's per-point pass and has no tensor-core join, so on
 * millions of points it takes many times longer than knng_refine; it is meant
 * for callers that cannot allocate, not as the fast path.
 * The first call in a CUDA context looks up the array's device address in
 * that context (cudaGetSymbolAddress; later calls reuse it): make that first
 * call before capturing the call into a CUDA graph.  Every call in one
 * context shares the array and it keeps the last call's records: calls that
 * overlap on the GPU in the same context (on different streams) race, so
 * serialise them.  Nothing a call needs carries over from an earlier one. */
knng_status knng_refine_pointwise_noalloc(const float* d_points, uint32_t n, uint32_t d, uint32_t k,
                                          uint32_t* d_snapshot, float* d_dist, uint32_t* d_ids, uint32_t* d_size,
                                          uint32_t* d_maxslot, float* d_bound, uint32_t* d_changed, void* stream);

/* SolutionKmeans::constructResult's wall-clock schedule
 * (src/SolutionKmeans.hpp:579-604): knng_build with time budgets instead of
 * fixed counts.  Repetitions (alternating max_leaf / max_leaf_odd) run while
 * less than build_ms has passed since the call began -- at least one, at most
 * params->reps when it is non-zero; then whole refinement passes start while
 * less than build_ms + refine_ms has passed, at most params->refine (the
 * reference cuts its single pass short instead).  stats->reps_done tells how
 * many repetitions ran.  Host pointers. */
knng_status knng_build_timed(knng_context* ctx, const float* points, uint32_t n, uint32_t d, uint64_t ld_bytes,
                             const knng_params* params, uint64_t build_ms, uint64_t refine_ms, uint32_t* out_ids,
                             float* out_dists, knng_stats* stats);

/* Batched form: many independent point sets in one build.  No counterpart in
 * the reference (one constructResult per process); each set is built as
 * knng_build would build it alone, with the same parameters and result, but
 * all sets share every launch: one set of launches per tree level across all
 * sets' nodes, one bucket launch per repetition across all sets' buckets, one
 * join per refinement pass.
 *   points       n rows (all sets concatenated), row stride ld_bytes
 *   set_offsets  n_sets + 1 ascending offsets, [0] = 0, [n_sets] = n; set s is
 *                rows [set_offsets[s], set_offsets[s+1]), at least one row
 *   on_device    nonzero: points, out_ids and out_dists are device pointers
 *   out_ids      n x k ids relative to each row's set (padding id 1 as in
 *                knng_build) */
knng_status knng_build_batch(knng_context* ctx, const float* points, uint32_t n, uint32_t d, uint64_t ld_bytes,
                             const uint32_t* set_offsets, uint32_t n_sets, int on_device, const knng_params* params,
                             uint32_t* out_ids, float* out_dists, knng_stats* stats);

/* ------------------------------------------------------------------------
 * Serving form.  No counterpart in the reference, which builds one graph per
 * process (constructResult, src/SolutionKmeans.hpp:558, called once from
 * src/main.cpp:59).  A server owns one device and an HBM budget and accepts
 * build jobs of different sizes as they arrive.  Jobs are admitted in arrival
 * order while the admitted jobs' reservations (knng_job_reservation) fit the
 * budget and fewer than max_running run; each admitted job builds on its own
 * context and stream, so concurrent jobs overlap on the device, and its
 * points and neighbour sets stay resident until its result is copied out.
 * A job runs exactly the build of knng_build with the same parameters: its
 * result is the same alone and among other jobs.
 * ------------------------------------------------------------------------ */
typedef struct knng_server knng_server;

enum { KNNG_JOB_QUEUED = 0, KNNG_JOB_RUNNING = 1, KNNG_JOB_DONE = 2, KNNG_JOB_FAILED = 3 };

typedef struct knng_job_info {
    uint32_t state;           /* KNNG_JOB_* */
    int32_t status;           /* knng_status of the build once ended */
    uint32_t n, d, k;
    uint32_t reserved0;
    uint64_t reserved_bytes;  /* HBM reserved for the job while it runs */
    double ms_queued;         /* submission to admission (so far, if still queued) */
    double ms_run;            /* admission to end (so far, if running) */
    double ms_latency;        /* submission to end (so far, if not ended) */
    knng_stats stats;         /* the build's statistics once done */
} knng_job_info;

/* HBM a job of n points, d dims, k neighbours reserves: points, order, sets,
 * refinement lists and survivor storage, plus fixed scratch. */
uint64_t knng_job_reservation(uint32_t n, uint32_t d, uint32_t k);

/* A server on `device` with an HBM budget (0: 80% of the device's memory) and
 * up to max_running concurrent jobs. */
knng_status knng_server_create(int device, uint64_t hbm_budget_bytes, uint32_t max_running, knng_server** out);

/* Queues a job.  `points` (host, row stride ld_bytes), `out_ids` (n*k) and
 * `out_dists` (n*k, nullable) must stay valid until the job has ended.
 * KNNG_ERR_BUDGET if the job's reservation exceeds the whole budget. */
knng_status knng_server_submit(knng_server* server, const float* points, uint32_t n, uint32_t d, uint64_t ld_bytes,
                               const knng_params* params, uint32_t* out_ids, float* out_dists, uint64_t* out_job);

/* Current state and timings of a job. */
knng_status knng_server_poll(knng_server* server, uint64_t job, knng_job_info* info);

/* Waits up to timeout_ms (< 0: without limit) for a job to end; KNNG_OK once
 * it has ended (info.state and info.status tell how), KNNG_ERR_PENDING if not
 * yet. */
knng_status knng_server_wait(knng_server* server, uint64_t job, int64_t timeout_ms, knng_job_info* info);

/* The error message of a failed job ("" otherwise). */
const char* knng_server_job_error(knng_server* server, uint64_t job);

/* Forgets an ended job's record (KNNG_ERR_PENDING if it has not ended). */
knng_status knng_server_release(knng_server* server, uint64_t job);

/* Refuses new jobs, cancels queued ones, waits for running ones, frees the
 * server. */
knng_status knng_server_destroy(knng_server* server);

#ifdef __cplusplus
}
#endif

#endif /* KNNG_H */
