// Host-side state of one knng_context: device buffers, the stream, error
// reporting, and the launchers every .cu file provides.
#pragma once

#include <cuda_runtime.h>

#include <cstdint>
#include <cstring>
#include <string>
#include <vector>

#include "../../include/knng.h"

namespace knng {

// Thrown inside the library only; every C entry point converts it to a status.
struct Error {
    knng_status status;
    std::string message;
};

[[noreturn]] void fail(knng_status s, const std::string& msg);
void check_cuda(cudaError_t e, const char* what);
#define KNNG_CUDA(call) ::knng::check_cuda((call), #call)

// A typed device allocation owned by the context; counts toward the budget.
struct DeviceBuffer {
    void* ptr = nullptr;
    size_t bytes = 0;
};

struct Timer {
    cudaEvent_t start = nullptr, stop = nullptr;
};

struct DevRep;  // buffers and graphs of the device-side repetition (split.cu)

struct Context {
    int device = 0;
    uint64_t budget = 0;
    uint64_t held = 0;
    cudaStream_t stream = nullptr;
    std::string last_error;

    // Points: n rows of ld floats (ld = d rounded up to 4), 16-byte aligned.
    uint32_t n = 0, d = 0, ld = 0;
    float* points = nullptr;
    bool points_borrowed = false;  // true when `points` is the caller's device buffer

    // Permutation of point ids; a second buffer for the partition scatter.
    uint32_t* indices = nullptr;
    uint32_t* indices_tmp = nullptr;

    // Independent point sets (batched builds): set s owns ids
    // [set_offsets[s], set_offsets[s+1]); one set {0, n} otherwise.  Each set
    // is its own tree root and its empty slots read as its first id.
    std::vector<uint32_t> set_offsets;
    uint32_t* d_set_offsets = nullptr;  // device copy when there is more than one set

    // Neighbour sets, slot order, capacity k per point.
    uint32_t k = 0;
    float* set_dist = nullptr;
    uint32_t* set_id = nullptr;
    uint32_t* set_size = nullptr;
    uint32_t* set_maxslot = nullptr;
    float* set_bound = nullptr;

    // Leaves of the last device-seeded repetition.
    std::vector<uint32_t> last_leaf_start, last_leaf_end;

    // Named scratch allocations, grown on demand and reused across calls.
    std::vector<std::pair<std::string, DeviceBuffer>> scratch;

    uint64_t launches = 0;

    // How a repetition's tree is built: 0 = one CUDA graph per repetition
    // (device-side levels under a WHILE node, the default), 1 = the same
    // device-side levels launched one by one, 2 = levels sequenced by the
    // host (environment KNNG_REP_LOOP=graph|device|host at creation).
    int rep_loop = 0;
    DevRep* devrep = nullptr;
    // Set while a graph is being captured: no attribute or allocation calls.
    bool capturing = false;
    int sms = 148;

    // Pinned host staging for small transfers: an upload is copied here and
    // sent asynchronously, a download lands here first; the space is reused
    // after the next synchronisation of the stream.
    unsigned char* staging = nullptr;
    size_t staging_cap = 0, staging_used = 0;

    // Neighbour-of-neighbour pass: 0 = local join on the tensor cores,
    // 1 = one warp per point (environment KNNG_REFINE=pointwise at creation).
    int refine_mode = 0;
    // Survivor storage of the join (environment at creation overrides the
    // sizes taken from the free budget): KNNG_REFINE_SLOTS = slots per point,
    // KNNG_REFINE_POOL = pool records per CTA region; -1 = from the budget.
    int refine_slots = -1;
    // The join takes points in the leaf order of the last repetition; true
    // (environment KNNG_JOIN_ORDER=id at creation): in id order.
    bool join_order_ids = false;
    // FP32 bucket pass: every pair's distance (k_leaf); true (environment
    // KNNG_LEAF=tc at creation): distances only where the tensor-core filter
    // cannot rule a pair out (k_leaf_tc).  Both give the same sets; the
    // filtered pass is slower at 10M points (the set updates dominate).
    bool leaf_tc = false;
    // Persistent CTAs per SM of the FP32 bucket pass over the device leaf
    // list (2 or 1); knng_tune_buckets may change this and leaf_tc.
    uint32_t leaf_ctas = 2;
    // A join pass skips the pairs the previous join pass offered (both edges
    // already in its lists; offering them again changes nothing): the lists
    // of the last pass are kept while snap_prev_valid.  Any change to the sets
    // other than offers clears it.  false (environment KNNG_REFINE_SKIP=0 at
    // creation): every pass offers every pair.
    bool refine_skip_old = true;
    bool snap_prev_valid = false;
    int64_t refine_pool = -1;
    // Breakdown of the last refinement pass.
    struct RefineRecord {
        double ms_join = 0, ms_apply = 0, ms_fallback = 0, ms_prep = 0;
        uint64_t pairs = 0, filter_pass = 0, member_skip = 0, exact = 0, emits = 0, overflow = 0, join_launches = 0;
        uint64_t lost = 0;
    } last_refine;
};

// Allocation helpers (budget-checked).
void* dev_alloc(Context& c, size_t bytes);
void dev_free(Context& c, void* p, size_t bytes);
void* scratch(Context& c, const char* name, size_t bytes);
// Bytes currently held by the named scratch allocation (0 if none).
size_t scratch_bytes(const Context& c, const char* name);
void release_all(Context& c);

// Transfers up to this size go through the pinned staging space.
constexpr size_t kStagedMax = 1u << 20;
// `bytes` of pinned staging space (synchronises the stream and starts over
// when the space is used up; grows it when one transfer needs more).
void* staging_take(Context& c, size_t bytes);
void staging_free(Context& c);

// Uploads `count` elements into named scratch and returns the device pointer.
template <class T>
T* upload(Context& c, const char* name, const T* host, size_t count) {
    T* d = static_cast<T*>(scratch(c, name, count * sizeof(T) + 16));
    const size_t bytes = count * sizeof(T);
    if (bytes == 0) return d;
    if (bytes <= kStagedMax) {
        void* p = staging_take(c, bytes);
        std::memcpy(p, host, bytes);
        KNNG_CUDA(cudaMemcpyAsync(d, p, bytes, cudaMemcpyHostToDevice, c.stream));
    } else {
        KNNG_CUDA(cudaMemcpyAsync(d, host, bytes, cudaMemcpyHostToDevice, c.stream));
    }
    return d;
}

template <class T>
void download(Context& c, T* host, const T* dev, size_t count) {
    const size_t bytes = count * sizeof(T);
    if (bytes > 0 && bytes <= kStagedMax) {
        void* p = staging_take(c, bytes);
        KNNG_CUDA(cudaMemcpyAsync(p, dev, bytes, cudaMemcpyDeviceToHost, c.stream));
        KNNG_CUDA(cudaStreamSynchronize(c.stream));
        std::memcpy(host, p, bytes);
    } else {
        if (bytes) KNNG_CUDA(cudaMemcpyAsync(host, dev, bytes, cudaMemcpyDeviceToHost, c.stream));
        KNNG_CUDA(cudaStreamSynchronize(c.stream));
    }
    c.staging_used = 0;  // every earlier copy through the staging space has completed
}

bool dim_supported(uint32_t d);

// Lets `kern` take as much dynamic shared memory as the device allows a block
// (the opt-in maximum less the kernel's static shared memory).  The attribute
// is process-wide per kernel, so contexts running concurrently must all set
// the same value -- this maximum, not the size of one launch (each launch
// passes its own size).
template <class Kernel>
void allow_max_smem(Context& c, Kernel kern) {
    if (c.capturing) return;  // set before the capture began
    int optin = 0;
    KNNG_CUDA(cudaDeviceGetAttribute(&optin, cudaDevAttrMaxSharedMemoryPerBlockOptin, c.device));
    cudaFuncAttributes fa{};
    KNNG_CUDA(cudaFuncGetAttributes(&fa, kern));
    KNNG_CUDA(cudaFuncSetAttribute(kern, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                   optin - static_cast<int>(fa.sharedSizeBytes)));
}

// ----------------------------------------------------------- launchers
// split.cu
void launch_iota(Context& c);
// Counter-RNG draws for `count` nodes: node i draws (draw_off[i+1]-draw_off[i])
// positions; the first seed-list-length of them go to d_seeds (CSR seed_off),
// the first Lloyd-list-length to d_lloyd (CSR lloyd_off).
void launch_draw_positions(Context& c, uint32_t count, const uint32_t* d_starts, const uint32_t* d_ends,
                           const uint32_t* d_bases, const uint32_t* d_attempts, const uint64_t* d_draw_off,
                           const uint64_t* d_seed_off,
                           const uint64_t* d_lloyd_off, uint64_t seed, uint32_t rep, uint32_t* d_seeds,
                           uint32_t* d_lloyd);
// Dense copy of the hyperplanes of the picked nodes.
void launch_gather_planes(Context& c, const float* d_coefs, const float* d_offsets, const uint32_t* d_pick,
                          uint32_t count, float* d_out_coefs, float* d_out_offsets);
// Farthest pair per node over a CSR position list; writes the two rows to
// d_c1 / d_c2 (count*ld floats) and d_ok = 0 where no pair exceeds FLT_MIN.
void launch_farthest_pair(Context& c, uint32_t count, const uint64_t* d_offsets, const uint32_t* d_positions,
                          uint32_t max_list, uint32_t* d_first, uint32_t* d_second, int32_t* d_ok, float* d_c1,
                          float* d_c2);
// `iters` Lloyd iterations per node over its CSR list (or its whole range when
// the list is empty), then the final hyperplane into d_coefs / d_offsets.
void launch_lloyd(Context& c, uint32_t count, const uint32_t* h_starts, const uint32_t* h_ends,
                  const uint64_t* h_lloyd_offsets, const uint32_t* d_lloyd_positions, float* d_c1, float* d_c2,
                  uint32_t iters, float* d_coefs, float* d_offsets, int32_t* d_ok);
// Side test + stable partition of `count` disjoint nodes; d_true[i] receives
// the number of side-true points of node i.
void launch_partition(Context& c, uint32_t count, const uint32_t* h_starts, const uint32_t* h_ends,
                      const uint32_t* d_starts, const float* d_coefs, const float* d_offsets, uint32_t* d_true);
// Device-side repetition (split.cu): the tree built by device-side levels,
// as one CUDA graph (graph = true) or launched level by level, then the
// bucket pass over the device's leaf list.
// Random-rotation KD splitter (kd.cu): the rotation vectors of a repetition
// (new_dims x d floats), and one repetition -- indices = iota, the KD tree,
// the bucket pass over its leaves.
std::vector<float> kd_rotation(uint32_t new_dims, uint32_t d, uint64_t seed);
struct KdRepResult {
    std::vector<uint32_t> leaf_start, leaf_end;
    double ms_split = 0, ms_leaf = 0;
    uint64_t levels = 0, nodes = 0, restarts = 0, fallbacks = 0;
};
void run_rep_kd(Context& c, uint32_t max_leaf, uint32_t new_dims, uint64_t seed, uint32_t rep, KdRepResult& out);
struct DevRepResult {
    std::vector<uint32_t> leaf_start, leaf_end;  // in no particular order
    double ms_split = 0, ms_leaf = 0;
    uint64_t levels = 0, nodes = 0, restarts = 0, fallbacks = 0, pairs = 0;
};
void run_rep_device(Context& c, uint32_t max_leaf, uint32_t lloyd_iters, uint32_t small_threshold, uint64_t seed,
                    uint32_t rep, uint32_t precision, bool graph, DevRepResult& out);
void devrep_release(Context& c);
// Sizing rules of the sampling plan (getSampleFromPercent, kmeansStartVecs).
uint32_t sample_count(uint32_t n);
uint32_t start_count(uint32_t n);
// leaf.cu
void launch_leaves(Context& c, uint32_t count, const uint32_t* d_starts, const uint32_t* d_ends,
                   uint32_t max_bucket, uint64_t* evals);
// Persistent bucket pass over a device list of *d_count buckets taken from
// the work counter *d_work (zeroed beforehand); *d_error is set when a
// tensor-core wait gives up.
void launch_leaves_list(Context& c, const uint32_t* d_starts, const uint32_t* d_ends, const uint32_t* d_count,
                        uint32_t* d_work, uint32_t max_bucket, uint32_t* d_error);
void launch_leaves_bf16_list(Context& c, const uint32_t* d_starts, const uint32_t* d_ends, const uint32_t* d_count,
                             uint32_t* d_work, uint32_t* d_error);
// Exact k nearest points (FP32 distances in the reference's order) of the
// nq points d_queries, ids into d_truth (nq x k, kNone past the end).
void sample_knn(Context& c, const uint32_t* d_queries, uint32_t nq, uint32_t* d_truth);
// Mean fraction of each sampled point's true k nearest held by its set.
double sample_recall(Context& c, const uint32_t* d_queries, uint32_t nq, const uint32_t* d_truth);
// Kernel attributes of the two list launchers, set before a graph capture.
void prepare_leaves_list(Context& c);
void prepare_leaves_bf16_list(Context& c);
// leaf_bf16.cu: the precision form (BF16 tensor-core estimates, the 128 best
// candidates per point re-ranked in FP32), buckets of at most 512 points.
void launch_leaves_bf16(Context& c, uint32_t count, const uint32_t* d_starts, const uint32_t* d_ends,
                        uint32_t max_bucket);
// One 128 x 128 BF16 tile a(m x d) . b(n x d)^T into d_out (m x n), m, n <= 128.
void run_tile_gram_bf16(Context& c, uint32_t d, const float* d_a, uint32_t m, const float* d_b, uint32_t n,
                        float* d_out);
// Poll limits of the kernels' bounded waits (split.cu, refine.cu).
void set_split_wait_limit(uint32_t polls);
void set_refine_wait_limit(uint32_t polls);
// refine.cu
uint64_t run_refine(Context& c);
// One tensor-core tile a(m x d) . b(n x d)^T into d_out (m x n), m, n <= 128.
void run_tile_gram(Context& c, uint32_t d, const float* d_a, uint32_t m, const float* d_b, uint32_t n, float* d_out);
// finalize.cu
void launch_finalize(Context& c, uint32_t* d_ids, float* d_dists);
void launch_reset_sets(Context& c);
// Batched builds: output ids relative to each point's set (padding stays 1).
void launch_rebase_ids(Context& c, uint32_t* d_ids);

}  // namespace knng
