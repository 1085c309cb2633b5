// C ABI of libknng.so (include/knng.h) and the host-side sequencing of the
// kernels: context and buffer management, the level-synchronous tree build of
// one repetition, and the one-call build.
//
// The reference recurses depth first over the tree, one node at a time
// (SolutionKmeans::splitKmeansBinaryProcess, src/SolutionKmeans.hpp:142-311).
// Here every node of a tree level is split by the same kernel launches, and
// the buckets of the whole repetition go to one bucket-kernel launch.  The
// host keeps the node list of the current level (a few thousand ranges) and
// reads back two small arrays per level: which nodes seeded / converged, and
// how many points went to each side.
#include <cuda_runtime.h>

#include <algorithm>
#include <chrono>
#include <cfloat>
#include <cmath>
#include <cstdio>
#include <cstdlib>
#include <cstring>
#include <new>
#include <numeric>
#include <string>
#include <vector>

#include "common.cuh"
#include "context.hpp"

namespace knng {

// Nodes whose split keeps failing (identical points) are split at the index
// midpoint after this many attempts; the reference would loop forever.
constexpr uint32_t kMaxAttempts = 64;

void fail(knng_status s, const std::string& msg) { throw Error{s, msg}; }

void check_cuda(cudaError_t e, const char* what) {
    if (e == cudaSuccess) return;
    // A non-sticky error stays as the thread's last error until read; clear
    // it so the next call on this context does not report it again.
    cudaGetLastError();
    if (e == cudaErrorMemoryAllocation) fail(KNNG_ERR_OUT_OF_MEMORY, std::string(what) + ": " + cudaGetErrorString(e));
    fail(KNNG_ERR_CUDA, std::string(what) + ": " + cudaGetErrorString(e));
}

bool dim_supported(uint32_t d) { return d == 64 || d == 100 || d == 128; }

// Device memory is stream-ordered on the context's stream (all of the
// context's work runs there), so allocating or freeing does not synchronise
// the device under other contexts' work.
void* dev_alloc(Context& c, size_t bytes) {
    if (bytes == 0) bytes = 16;
    if (c.held + bytes > c.budget) fail(KNNG_ERR_BUDGET, "device memory budget exceeded");
    void* p = nullptr;
    check_cuda(cudaMallocAsync(&p, bytes, c.stream), "cudaMallocAsync");
    c.held += bytes;
    return p;
}

void dev_free(Context& c, void* p, size_t bytes) {
    if (!p) return;
    cudaFreeAsync(p, c.stream);
    c.held -= std::min<uint64_t>(c.held, bytes == 0 ? 16 : bytes);
}

void* scratch(Context& c, const char* name, size_t bytes) {
    for (auto& e : c.scratch) {
        if (e.first == name) {
            if (e.second.bytes >= bytes) return e.second.ptr;
            KNNG_CUDA(cudaStreamSynchronize(c.stream));
            size_t grown = std::max(bytes, e.second.bytes * 3 / 2);
            if (c.held - e.second.bytes + grown > c.budget) grown = bytes;
            dev_free(c, e.second.ptr, e.second.bytes);
            e.second.ptr = nullptr;
            e.second.bytes = 0;
            e.second.ptr = dev_alloc(c, grown);
            e.second.bytes = grown;
            return e.second.ptr;
        }
    }
    DeviceBuffer b;
    b.ptr = dev_alloc(c, bytes);
    b.bytes = bytes == 0 ? 16 : bytes;
    c.scratch.emplace_back(name, b);
    return b.ptr;
}

// --------------------------------------------------------------- sizing rules

// getSampleFromPercent's sample size: (uint32)(n * (float)((ln n / ln 30)^7 / n))
// (src/SolutionKmeans.hpp:50-58).
uint32_t sample_count(uint32_t n) {
    const float frac = static_cast<float>(std::pow(std::log(static_cast<double>(n)) / std::log(30.0), 7) / n);
    return static_cast<uint32_t>(static_cast<float>(n) * frac);
}

// kmeansStartVecs' seed count: (uint32)(log10 n)^2.5 (src/SolutionKmeans.hpp:70, :105).
uint32_t start_count(uint32_t n) { return static_cast<uint32_t>(std::pow(std::log10(static_cast<double>(n)), 2.5)); }

void* staging_take(Context& c, size_t bytes) {
    bytes = (bytes + 15) / 16 * 16;
    if (bytes > c.staging_cap) {
        KNNG_CUDA(cudaStreamSynchronize(c.stream));
        staging_free(c);
        const size_t cap = std::max<size_t>(bytes, 4u << 20);
        void* p = nullptr;
        check_cuda(cudaMallocHost(&p, cap), "cudaMallocHost");
        c.staging = static_cast<unsigned char*>(p);
        c.staging_cap = cap;
        c.staging_used = 0;
    }
    if (c.staging_used + bytes > c.staging_cap) {
        // Every copy through the space must land before it is reused.
        KNNG_CUDA(cudaStreamSynchronize(c.stream));
        c.staging_used = 0;
    }
    void* p = c.staging + c.staging_used;
    c.staging_used += bytes;
    return p;
}

void staging_free(Context& c) {
    if (c.staging) cudaFreeHost(c.staging);
    c.staging = nullptr;
    c.staging_cap = c.staging_used = 0;
}

size_t scratch_bytes(const Context& c, const char* name) {
    for (const auto& e : c.scratch)
        if (e.first == name) return e.second.bytes;
    return 0;
}

namespace {

void free_points(Context& c) {
    c.snap_prev_valid = false;
    if (c.points && !c.points_borrowed) dev_free(c, c.points, static_cast<size_t>(c.n) * c.ld * sizeof(float));
    c.points = nullptr;
    c.points_borrowed = false;
}

void free_sets(Context& c) {
    c.snap_prev_valid = false;
    const size_t nk = static_cast<size_t>(c.n) * c.k;
    dev_free(c, c.set_dist, nk * sizeof(float));
    dev_free(c, c.set_id, nk * sizeof(uint32_t));
    dev_free(c, c.set_size, c.n * sizeof(uint32_t));
    dev_free(c, c.set_maxslot, c.n * sizeof(uint32_t));
    dev_free(c, c.set_bound, c.n * sizeof(float));
    c.set_dist = nullptr;
    c.set_id = nullptr;
    c.set_size = c.set_maxslot = nullptr;
    c.set_bound = nullptr;
}

}  // namespace

void release_all(Context& c) {
    if (c.stream) cudaStreamSynchronize(c.stream);
    devrep_release(c);
    free_points(c);
    free_sets(c);
    dev_free(c, c.indices, c.n * sizeof(uint32_t));
    dev_free(c, c.indices_tmp, c.n * sizeof(uint32_t));
    c.indices = c.indices_tmp = nullptr;
    for (auto& e : c.scratch) dev_free(c, e.second.ptr, e.second.bytes);
    c.scratch.clear();
    c.n = 0;
}

namespace {


struct EventPair {
    cudaEvent_t a = nullptr, b = nullptr;
    explicit EventPair(Context& c) {
        KNNG_CUDA(cudaEventCreate(&a));
        KNNG_CUDA(cudaEventCreate(&b));
        KNNG_CUDA(cudaEventRecord(a, c.stream));
    }
    double stop(Context& c) {
        KNNG_CUDA(cudaEventRecord(b, c.stream));
        KNNG_CUDA(cudaEventSynchronize(b));
        float ms = 0.f;
        KNNG_CUDA(cudaEventElapsedTime(&ms, a, b));
        return ms;
    }
    ~EventPair() {
        if (a) cudaEventDestroy(a);
        if (b) cudaEventDestroy(b);
    }
};

void require_points(Context& c) {
    if (!c.points || c.n == 0) fail(KNNG_ERR_STATE, "no points loaded");
}

void require_sets(Context& c) {
    require_points(c);
    if (!c.set_dist) fail(KNNG_ERR_STATE, "neighbour sets not initialised");
}

void alloc_sets(Context& c, uint32_t k) {
    if (k == 0 || k > static_cast<uint32_t>(kMaxK)) fail(KNNG_ERR_UNSUPPORTED, "k must be in 1..128");
    if (c.set_dist && c.k == k) {
        launch_reset_sets(c);
        return;
    }
    free_sets(c);
    c.k = k;
    const size_t nk = static_cast<size_t>(c.n) * k;
    c.set_dist = static_cast<float*>(dev_alloc(c, nk * sizeof(float)));
    c.set_id = static_cast<uint32_t*>(dev_alloc(c, nk * sizeof(uint32_t)));
    c.set_size = static_cast<uint32_t*>(dev_alloc(c, c.n * sizeof(uint32_t)));
    c.set_maxslot = static_cast<uint32_t*>(dev_alloc(c, c.n * sizeof(uint32_t)));
    c.set_bound = static_cast<float*>(dev_alloc(c, c.n * sizeof(float)));
    launch_reset_sets(c);
}

void load_points(Context& c, const float* pts, uint32_t n, uint32_t d, uint64_t ld_bytes, bool on_device,
                 bool allow_borrow) {
    if (!pts && n > 0) fail(KNNG_ERR_INVALID_ARGUMENT, "points is null");
    if (!dim_supported(d)) fail(KNNG_ERR_UNSUPPORTED, "dimension must be 64, 100 or 128");
    if (ld_bytes == 0) ld_bytes = static_cast<uint64_t>(d) * sizeof(float);
    if (ld_bytes < static_cast<uint64_t>(d) * sizeof(float) || ld_bytes % sizeof(float) != 0)
        fail(KNNG_ERR_INVALID_ARGUMENT, "ld_bytes must be a multiple of 4 and >= 4*d");
    // Same shape: keep the sets, order and scratch (only the points change,
    // whether they are copied in or borrowed).
    const bool same_shape = c.indices && c.n == n && c.d == d;
    if (!same_shape) {
        const uint32_t k = c.k;
        const bool had_sets = c.set_dist != nullptr;
        release_all(c);
        c.n = n;
        c.d = d;
        c.ld = d;  // supported dims are multiples of 4: rows stay 16-byte aligned
        c.indices = static_cast<uint32_t*>(dev_alloc(c, static_cast<size_t>(n) * sizeof(uint32_t)));
        c.indices_tmp = static_cast<uint32_t*>(dev_alloc(c, static_cast<size_t>(n) * sizeof(uint32_t)));
        if (had_sets) c.k = k;
    }
    const size_t row = static_cast<size_t>(d) * sizeof(float);
    const bool aligned = (reinterpret_cast<uintptr_t>(pts) % 16 == 0) && ld_bytes == row;
    if (on_device && allow_borrow && aligned) {
        if (c.points && !c.points_borrowed) free_points(c);
        c.points = const_cast<float*>(pts);
        c.points_borrowed = true;
    } else {
        if (!c.points || c.points_borrowed) {
            c.points = static_cast<float*>(dev_alloc(c, static_cast<size_t>(n) * row));
            c.points_borrowed = false;
        }
        const cudaMemcpyKind kind = on_device ? cudaMemcpyDeviceToDevice : cudaMemcpyHostToDevice;
        if (n > 0 && ld_bytes == row)  // packed rows: one contiguous copy
            KNNG_CUDA(cudaMemcpyAsync(c.points, pts, static_cast<size_t>(n) * row, kind, c.stream));
        else if (n > 0)
            KNNG_CUDA(cudaMemcpy2DAsync(c.points, row, pts, ld_bytes, row, n, kind, c.stream));
    }
    c.set_offsets = {0u, n};
    c.d_set_offsets = nullptr;
    launch_iota(c);
}

// ------------------------------------------------------- one repetition

struct Node {
    uint32_t start, end;
    uint32_t base;  // first id of the node's point set (RNG keys are relative to it)
};

struct RepStats {
    uint64_t levels = 0, nodes = 0, restarts = 0, fallbacks = 0;
    double ms_split = 0, ms_leaf = 0;
};

// Seeds, runs Lloyd and partitions every node of `active`; returns the
// midpoints.  Nodes that fail (no pair above FLT_MIN, an empty cluster, an
// empty side) are redrawn with the next attempt index, like the reference's
// goto restarts (src/SolutionKmeans.hpp:177-178, :203-205, :251-253, :291-293).
std::vector<uint32_t> split_level(Context& c, const std::vector<Node>& active, uint32_t lloyd_iters,
                                  uint32_t small_threshold, uint64_t seed, uint32_t rep, RepStats& st) {
    const uint32_t m = static_cast<uint32_t>(active.size());
    std::vector<uint32_t> mids(m, kNone);
    std::vector<uint32_t> attempt(m, 0);
    std::vector<uint32_t> pending(m);
    std::iota(pending.begin(), pending.end(), 0u);
    const uint32_t ld = c.ld;
    while (!pending.empty()) {
        std::vector<uint32_t> todo;
        for (uint32_t i : pending) {
            if (attempt[i] >= kMaxAttempts) {
                const Node& nd = active[i];
                mids[i] = nd.start + (nd.end - nd.start) / 2;
                ++st.fallbacks;
            } else {
                todo.push_back(i);
            }
        }
        pending.clear();
        if (todo.empty()) break;
        const uint32_t cnt = static_cast<uint32_t>(todo.size());
        // Draw lists: large nodes draw their whole sample and seed from its
        // first min(|sample|, S) entries; small nodes draw S seeds and run
        // Lloyd over their whole range.
        std::vector<uint32_t> hs(cnt), he(cnt), ha(cnt), hb(cnt);
        std::vector<uint64_t> draw_off(cnt + 1), seed_off(cnt + 1), lloyd_off(cnt + 1);
        uint64_t total = 0, seed_total = 0, lloyd_total = 0;
        uint32_t max_seed = 1;
        for (uint32_t t = 0; t < cnt; ++t) {
            const Node& nd = active[todo[t]];
            const uint32_t n = nd.end - nd.start;
            hs[t] = nd.start;
            he[t] = nd.end;
            hb[t] = nd.base;
            ha[t] = attempt[todo[t]];
            const bool large = n >= small_threshold;
            const uint32_t S = start_count(n);
            const uint32_t draws = large ? sample_count(n) : S;
            draw_off[t] = total;
            seed_off[t] = seed_total;
            lloyd_off[t] = lloyd_total;
            total += draws;
            seed_total += std::min(draws, S);
            max_seed = std::max(max_seed, std::min(draws, S));
            if (large) lloyd_total += draws;
        }
        draw_off[cnt] = total;
        seed_off[cnt] = seed_total;
        lloyd_off[cnt] = lloyd_total;
        uint32_t* d_s = upload(c, "lvl_start", hs.data(), cnt);
        uint32_t* d_e = upload(c, "lvl_end", he.data(), cnt);
        uint32_t* d_a = upload(c, "lvl_attempt", ha.data(), cnt);
        uint32_t* d_b = upload(c, "lvl_base", hb.data(), cnt);
        uint64_t* d_doff = upload(c, "lvl_draw_off", draw_off.data(), cnt + 1);
        uint64_t* d_sb = upload(c, "lvl_seed_off", seed_off.data(), cnt + 1);
        uint64_t* d_loff = upload(c, "lvl_lloyd_off", lloyd_off.data(), cnt + 1);
        uint32_t* seeds = static_cast<uint32_t*>(scratch(c, "lvl_seeds", (seed_total + 1) * sizeof(uint32_t)));
        uint32_t* lloyd = static_cast<uint32_t*>(scratch(c, "lvl_lloyd", (lloyd_total + 1) * sizeof(uint32_t)));
        launch_draw_positions(c, cnt, d_s, d_e, d_b, d_a, d_doff, d_sb, d_loff, seed, rep, seeds, lloyd);
        uint32_t* first = static_cast<uint32_t*>(scratch(c, "lvl_first", cnt * sizeof(uint32_t)));
        uint32_t* second = static_cast<uint32_t*>(scratch(c, "lvl_second", cnt * sizeof(uint32_t)));
        // ok[t]: node t seeded and converged; ok[cnt]: a Lloyd wait gave up.
        int32_t* ok = static_cast<int32_t*>(scratch(c, "lvl_ok", (cnt + 1) * sizeof(int32_t)));
        float* c1 = static_cast<float*>(scratch(c, "lvl_c1", static_cast<size_t>(cnt) * ld * sizeof(float)));
        float* c2 = static_cast<float*>(scratch(c, "lvl_c2", static_cast<size_t>(cnt) * ld * sizeof(float)));
        float* coefs = static_cast<float*>(scratch(c, "lvl_coefs", static_cast<size_t>(cnt) * ld * sizeof(float)));
        float* offs = static_cast<float*>(scratch(c, "lvl_offsets", cnt * sizeof(float)));
        launch_farthest_pair(c, cnt, d_sb, seeds, max_seed, first, second, ok, c1, c2);
        launch_lloyd(c, cnt, hs.data(), he.data(), lloyd_off.data(), lloyd, c1, c2, lloyd_iters, coefs, offs, ok);
        std::vector<int32_t> hok(cnt + 1);
        download(c, hok.data(), ok, cnt + 1);
        if (hok[cnt]) fail(KNNG_ERR_CUDA, "Lloyd sums: a bulk-copy wait gave up");
        // Partition the nodes that seeded and converged.
        std::vector<uint32_t> sel;
        for (uint32_t t = 0; t < cnt; ++t) {
            if (hok[t])
                sel.push_back(t);
            else {
                ++attempt[todo[t]];
                pending.push_back(todo[t]);
                ++st.restarts;
            }
        }
        if (!sel.empty()) {
            const uint32_t ns = static_cast<uint32_t>(sel.size());
            std::vector<uint32_t> ps(ns), pe(ns), pick(ns);
            for (uint32_t u = 0; u < ns; ++u) {
                ps[u] = hs[sel[u]];
                pe[u] = he[sel[u]];
                pick[u] = sel[u];
            }
            // Gather the selected hyperplanes into a dense array.
            float* pc = coefs;
            float* po = offs;
            if (ns != cnt) {
                pc = static_cast<float*>(scratch(c, "lvl_pcoefs", static_cast<size_t>(ns) * ld * sizeof(float)));
                po = static_cast<float*>(scratch(c, "lvl_poffs", ns * sizeof(float)));
                uint32_t* d_pick = upload(c, "lvl_pick", pick.data(), ns);
                launch_gather_planes(c, coefs, offs, d_pick, ns, pc, po);
            }
            uint32_t* d_ps = upload(c, "lvl_pstart", ps.data(), ns);
            uint32_t* d_true = static_cast<uint32_t*>(scratch(c, "lvl_true", ns * sizeof(uint32_t)));
            launch_partition(c, ns, ps.data(), pe.data(), d_ps, pc, po, d_true);
            std::vector<uint32_t> ht(ns);
            download(c, ht.data(), d_true, ns);
            for (uint32_t u = 0; u < ns; ++u) {
                const uint32_t i = todo[pick[u]];
                const uint32_t n = pe[u] - ps[u];
                if (ht[u] == 0 || ht[u] == n) {
                    ++attempt[i];
                    pending.push_back(i);
                    ++st.restarts;
                } else {
                    mids[i] = ps[u] + ht[u];
                }
            }
        }
        std::sort(pending.begin(), pending.end());
    }
    return mids;
}

void run_rep(Context& c, uint32_t max_leaf, uint32_t lloyd_iters, uint32_t small_threshold, uint64_t seed,
             uint32_t rep, RepStats& st, knng_stats* stats, uint32_t precision = KNNG_PRECISION_FP32) {
    require_sets(c);
    if (max_leaf < 2) fail(KNNG_ERR_INVALID_ARGUMENT, "max_leaf must be >= 2");
    if (c.rep_loop != 2) {
        // Device-side levels (one graph, or level by level), then the bucket
        // pass over the device's leaf list.
        DevRepResult res;
        run_rep_device(c, max_leaf, lloyd_iters, small_threshold, seed, rep, precision, c.rep_loop == 0, res);
        std::vector<std::pair<uint32_t, uint32_t>> lv(res.leaf_start.size());
        for (size_t i = 0; i < lv.size(); ++i) lv[i] = {res.leaf_start[i], res.leaf_end[i]};
        std::sort(lv.begin(), lv.end());
        c.last_leaf_start.resize(lv.size());
        c.last_leaf_end.resize(lv.size());
        for (size_t i = 0; i < lv.size(); ++i) {
            c.last_leaf_start[i] = lv[i].first;
            c.last_leaf_end[i] = lv[i].second;
        }
        st.levels += res.levels;
        st.nodes += res.nodes;
        st.restarts += res.restarts;
        st.fallbacks += res.fallbacks;
        st.ms_split += res.ms_split;
        st.ms_leaf += res.ms_leaf;
        if (stats) {
            stats->buckets += lv.size();
            stats->bucket_pairs += res.pairs;
            stats->leaf_launches += 1;
            stats->ms_leaf_kernel += res.ms_leaf;
        }
        return;
    }
    EventPair split_t(c);
    launch_iota(c);
    std::vector<Node> level;
    for (size_t s = 0; s + 1 < c.set_offsets.size(); ++s)
        level.push_back({c.set_offsets[s], c.set_offsets[s + 1], c.set_offsets[s]});
    std::vector<Node> leaves;
    while (!level.empty()) {
        std::vector<Node> active;
        for (const Node& nd : level) {
            if (nd.end - nd.start < max_leaf)
                leaves.push_back(nd);
            else
                active.push_back(nd);
        }
        if (active.empty()) break;
        ++st.levels;
        st.nodes += active.size();
        std::vector<uint32_t> mids = split_level(c, active, lloyd_iters, small_threshold, seed, rep, st);
        level.clear();
        for (size_t i = 0; i < active.size(); ++i) {
            level.push_back({active[i].start, mids[i], active[i].base});
            level.push_back({mids[i], active[i].end, active[i].base});
        }
    }
    st.ms_split += split_t.stop(c);
    std::sort(leaves.begin(), leaves.end(), [](const Node& a, const Node& b) { return a.start < b.start; });
    c.last_leaf_start.resize(leaves.size());
    c.last_leaf_end.resize(leaves.size());
    uint32_t max_bucket = 1;
    uint64_t pairs = 0;
    for (size_t i = 0; i < leaves.size(); ++i) {
        c.last_leaf_start[i] = leaves[i].start;
        c.last_leaf_end[i] = leaves[i].end;
        const uint64_t b = leaves[i].end - leaves[i].start;
        max_bucket = std::max<uint32_t>(max_bucket, static_cast<uint32_t>(b));
        pairs += b * (b - 1) / 2;
    }
    EventPair leaf_t(c);
    const uint32_t nl = static_cast<uint32_t>(leaves.size());
    uint32_t* d_ls = upload(c, "leaf_start", c.last_leaf_start.data(), nl);
    uint32_t* d_le = upload(c, "leaf_end", c.last_leaf_end.data(), nl);
    if (precision == KNNG_PRECISION_BF16_RERANK)
        launch_leaves_bf16(c, nl, d_ls, d_le, max_bucket);
    else
        launch_leaves(c, nl, d_ls, d_le, max_bucket, nullptr);
    const double leaf_ms = leaf_t.stop(c);
    st.ms_leaf += leaf_ms;
    if (stats) {
        stats->buckets += nl;
        stats->bucket_pairs += pairs;
        stats->leaf_launches += 1;
        stats->ms_leaf_kernel += leaf_ms;
    }
}

void add_rep_stats(knng_stats* s, const RepStats& st) {
    if (!s) return;
    s->split_levels += st.levels;
    s->split_nodes += st.nodes;
    s->restarts += st.restarts;
    s->fallback_splits += st.fallbacks;
    s->ms_split += st.ms_split;
    s->ms_leaf += st.ms_leaf;
}

void add_refine_stats(knng_stats* stats, const Context& c, uint64_t changed, double ms) {
    if (!stats) return;
    stats->refine_passes_done += 1;
    stats->ms_refine += ms;
    stats->refine_changed += changed;
    stats->ms_refine_join += c.last_refine.ms_join;
    stats->ms_refine_apply += c.last_refine.ms_apply;
    stats->ms_refine_fallback += c.last_refine.ms_fallback;
    stats->refine_pairs += c.last_refine.pairs;
    stats->refine_filter_pass += c.last_refine.filter_pass;
    stats->refine_member_skip += c.last_refine.member_skip;
    stats->refine_exact += c.last_refine.exact;
    stats->refine_emits += c.last_refine.emits;
    stats->refine_overflow += c.last_refine.overflow;
    stats->ms_refine_prep += c.last_refine.ms_prep;
    stats->refine_join_launches += c.last_refine.join_launches;
    stats->refine_lost += c.last_refine.lost;
}

void validate_params(const knng_params* p) {
    if (!p) fail(KNNG_ERR_INVALID_ARGUMENT, "params is null");
    if (p->k == 0 || p->k > static_cast<uint32_t>(kMaxK)) fail(KNNG_ERR_UNSUPPORTED, "k must be in 1..128");
    if (p->max_leaf < 2 || (p->max_leaf_odd != 0 && p->max_leaf_odd < 2))
        fail(KNNG_ERR_INVALID_ARGUMENT, "max_leaf must be >= 2");
    if (p->max_leaf > 4097 || p->max_leaf_odd > 4097) fail(KNNG_ERR_INVALID_ARGUMENT, "max_leaf must be <= 4097");
    if (p->precision != KNNG_PRECISION_FP32 && p->precision != KNNG_PRECISION_BF16_RERANK)
        fail(KNNG_ERR_UNSUPPORTED, "unknown precision");
    if (p->precision == KNNG_PRECISION_BF16_RERANK && (p->max_leaf > 1025 || p->max_leaf_odd > 1025))
        fail(KNNG_ERR_UNSUPPORTED, "the BF16 form takes buckets of at most 1024 points (max_leaf <= 1025)");
}

// All repetitions, then all refinement passes.  With build_ms > 0 (the
// reference's wall-clock loop, SolutionKmeans::constructResult,
// src/SolutionKmeans.hpp:579-604): repetitions run while less than build_ms
// has passed since the call began (at least one, at most p->reps when it is
// non-zero), then whole refinement passes start while less than
// build_ms + refine_ms has passed (at most p->refine).
void build_all(Context& c, const knng_params* p, knng_stats* stats, uint64_t build_ms = 0, uint64_t refine_ms = 0) {
    const auto t0 = std::chrono::steady_clock::now();
    auto elapsed_ms = [&] {
        KNNG_CUDA(cudaStreamSynchronize(c.stream));
        return static_cast<uint64_t>(
            std::chrono::duration_cast<std::chrono::milliseconds>(std::chrono::steady_clock::now() - t0).count());
    };
    const bool timed = build_ms > 0;
    alloc_sets(c, p->k);
    EventPair total_t(c);
    const uint64_t launches0 = c.launches;
    for (uint32_t r = 0; timed ? (r == 0 || ((p->reps == 0 || r < p->reps) && elapsed_ms() < build_ms)) : r < p->reps;
         ++r) {
        const uint32_t leaf = (p->max_leaf_odd != 0 && (r % 2 == 1)) ? p->max_leaf_odd : p->max_leaf;
        RepStats st;
        run_rep(c, leaf, p->lloyd_iters, p->small_threshold, p->seed, r, st, stats, p->precision);
        add_rep_stats(stats, st);
        if (stats) stats->reps_done += 1;
    }
    for (uint32_t pass = 0; pass < p->refine; ++pass) {
        if (timed && elapsed_ms() >= build_ms + refine_ms) break;
        EventPair rt(c);
        const uint64_t ch = run_refine(c);
        add_refine_stats(stats, c, ch, rt.stop(c));
    }
    const double ms = total_t.stop(c);
    if (stats) {
        stats->ms_total += ms;
        stats->kernel_launches += c.launches - launches0;
    }
}

// Adaptive schedule: repetitions and neighbour-of-neighbour passes until the
// recall estimated on `sample` evenly spaced points (their exact k nearest
// found on the device once) reaches `target`.  After the first
// min(2, max reps) repetitions: a pass follows every repetition, a second
// pass follows if the target is still missed, then another repetition; at
// most p->reps repetitions (0: 64) and p->refine passes.  The recall is
// estimated after every step.
void build_adaptive(Context& c, const knng_params* p, double target, uint32_t sample, knng_stats* stats) {
    alloc_sets(c, p->k);
    EventPair total_t(c);
    const uint64_t launches0 = c.launches;
    const uint32_t q = std::max<uint32_t>(1, std::min(sample, c.n));
    std::vector<uint32_t> hq(q);
    for (uint32_t i = 0; i < q; ++i) hq[i] = static_cast<uint32_t>((static_cast<uint64_t>(i) * c.n) / q);
    uint32_t* d_q = upload(c, "adaptive_queries", hq.data(), q);
    auto* d_truth = static_cast<uint32_t*>(scratch(c, "adaptive_truth", static_cast<size_t>(q) * c.k * sizeof(uint32_t)));
    sample_knn(c, d_q, q, d_truth);
    const uint32_t max_reps = p->reps ? p->reps : 64u, max_passes = p->refine;
    const uint32_t min_reps = std::min(2u, max_reps);
    uint32_t reps = 0, passes = 0, passes_since_rep = 0;
    double est = 0.0;
    auto rep_step = [&] {
        const uint32_t leaf = (p->max_leaf_odd != 0 && (reps % 2 == 1)) ? p->max_leaf_odd : p->max_leaf;
        RepStats st;
        run_rep(c, leaf, p->lloyd_iters, p->small_threshold, p->seed, reps, st, stats, p->precision);
        add_rep_stats(stats, st);
        if (stats) stats->reps_done += 1;
        ++reps;
        passes_since_rep = 0;
    };
    auto pass_step = [&] {
        EventPair rt(c);
        const uint64_t ch = run_refine(c);
        add_refine_stats(stats, c, ch, rt.stop(c));
        ++passes;
        ++passes_since_rep;
    };
    while (reps < min_reps) rep_step();
    est = sample_recall(c, d_q, q, d_truth);
    while (est < target) {
        if (passes_since_rep < 2 && passes < max_passes)
            pass_step();
        else if (reps < max_reps)
            rep_step();
        else if (passes < max_passes)
            pass_step();
        else
            break;
        est = sample_recall(c, d_q, q, d_truth);
    }
    const double ms = total_t.stop(c);
    if (stats) {
        stats->ms_total += ms;
        stats->kernel_launches += c.launches - launches0;
        stats->recall_estimate = est;
        stats->estimate_queries = q;
    }
}

template <class F>
knng_status guarded(knng_context* ctx, F&& f) {
    Context* c = reinterpret_cast<Context*>(ctx);
    if (!c) return KNNG_ERR_INVALID_ARGUMENT;
    try {
        KNNG_CUDA(cudaSetDevice(c->device));
        f(*c);
        c->last_error.clear();
        return KNNG_OK;
    } catch (const Error& e) {
        c->last_error = e.message;
        return e.status;
    } catch (const std::bad_alloc&) {
        c->last_error = "host allocation failed";
        return KNNG_ERR_OUT_OF_MEMORY;
    } catch (...) {
        c->last_error = "unexpected exception";
        return KNNG_ERR_CUDA;
    }
}

}  // namespace
}  // namespace knng

using knng::Context;

extern "C" {

void knng_default_params(knng_params* p) {
    if (!p) return;
    p->k = 100;
    p->max_leaf = 200;
    p->max_leaf_odd = 400;
    p->lloyd_iters = 1;
    p->reps = 8;
    p->refine = 1;
    p->small_threshold = 3000;
    p->precision = KNNG_PRECISION_FP32;
    p->seed = 12345;
}

const char* knng_status_string(knng_status s) {
    switch (s) {
        case KNNG_OK: return "ok";
        case KNNG_ERR_INVALID_ARGUMENT: return "invalid argument";
        case KNNG_ERR_CUDA: return "CUDA error";
        case KNNG_ERR_OUT_OF_MEMORY: return "out of device memory";
        case KNNG_ERR_BUDGET: return "device memory budget exceeded";
        case KNNG_ERR_STATE: return "call out of order";
        case KNNG_ERR_UNSUPPORTED: return "unsupported dimension or k";
        case KNNG_ERR_NO_DEVICE: return "no sm_100 CUDA device";
        case KNNG_ERR_PENDING: return "job has not ended";
    }
    return "unknown status";
}

knng_status knng_create(int device, uint64_t hbm_budget_bytes, knng_context** out) {
    if (!out) return KNNG_ERR_INVALID_ARGUMENT;
    *out = nullptr;
    int count = 0;
    if (cudaGetDeviceCount(&count) != cudaSuccess || count == 0) {
        cudaGetLastError();
        return KNNG_ERR_NO_DEVICE;
    }
    if (device < 0 || device >= count) return KNNG_ERR_INVALID_ARGUMENT;
    cudaDeviceProp prop;
    if (cudaGetDeviceProperties(&prop, device) != cudaSuccess) return KNNG_ERR_CUDA;
    if (prop.major != 10) return KNNG_ERR_NO_DEVICE;
    if (cudaSetDevice(device) != cudaSuccess) return KNNG_ERR_CUDA;
    auto* c = new (std::nothrow) Context();
    if (!c) return KNNG_ERR_OUT_OF_MEMORY;
    c->device = device;
    if (const char* r = std::getenv("KNNG_REFINE")) c->refine_mode = std::strcmp(r, "pointwise") == 0 ? 1 : 0;
    if (const char* r = std::getenv("KNNG_REFINE_SLOTS")) c->refine_slots = std::max(0, std::atoi(r));
    if (const char* r = std::getenv("KNNG_JOIN_ORDER")) c->join_order_ids = std::strcmp(r, "id") == 0;
    if (const char* r = std::getenv("KNNG_LEAF")) c->leaf_tc = std::strcmp(r, "tc") == 0;
    if (const char* r = std::getenv("KNNG_REFINE_SKIP")) c->refine_skip_old = std::strcmp(r, "0") != 0;
    if (const char* r = std::getenv("KNNG_REP_LOOP"))
        c->rep_loop = std::strcmp(r, "host") == 0 ? 2 : (std::strcmp(r, "device") == 0 ? 1 : 0);
    c->sms = prop.multiProcessorCount;
    if (const char* r = std::getenv("KNNG_REFINE_POOL")) c->refine_pool = std::max<long long>(0, std::atoll(r));
    if (hbm_budget_bytes) {
        c->budget = hbm_budget_bytes;
    } else {
        // 90% of the device, but no more than what is free now (less 1 GiB):
        // memory other users of the device hold is not this context's.
        c->budget = static_cast<uint64_t>(prop.totalGlobalMem * 0.9);
        // Memory freed to the device's stream-ordered pool (by contexts
        // destroyed earlier) counts as free: return what the pool keeps unused.
        cudaMemPool_t pool = nullptr;
        if (cudaDeviceGetDefaultMemPool(&pool, device) == cudaSuccess) cudaMemPoolTrimTo(pool, 0);
        cudaGetLastError();
        size_t free_b = 0, total_b = 0;
        if (cudaMemGetInfo(&free_b, &total_b) == cudaSuccess) {
            const uint64_t room = free_b > (1ull << 30) ? free_b - (1ull << 30) : 0;
            c->budget = std::min<uint64_t>(c->budget, room);
        } else {
            cudaGetLastError();
        }
    }
    if (cudaStreamCreateWithFlags(&c->stream, cudaStreamNonBlocking) != cudaSuccess) {
        delete c;
        return KNNG_ERR_CUDA;
    }
    *out = reinterpret_cast<knng_context*>(c);
    return KNNG_OK;
}

knng_status knng_destroy(knng_context* ctx) {
    Context* c = reinterpret_cast<Context*>(ctx);
    if (!c) return KNNG_ERR_INVALID_ARGUMENT;
    cudaSetDevice(c->device);
    knng::release_all(*c);
    knng::staging_free(*c);
    if (c->stream) cudaStreamDestroy(c->stream);
    delete c;
    return KNNG_OK;
}

const char* knng_last_error(const knng_context* ctx) {
    const Context* c = reinterpret_cast<const Context*>(ctx);
    return c ? c->last_error.c_str() : "null context";
}

knng_status knng_load_points(knng_context* ctx, const float* points, uint32_t n, uint32_t d, uint64_t ld_bytes,
                             int on_device) {
    return knng::guarded(ctx, [&](Context& c) {
        knng::load_points(c, points, n, d, ld_bytes, on_device != 0, false);
        if (c.k) knng::alloc_sets(c, c.k);
        KNNG_CUDA(cudaStreamSynchronize(c.stream));
    });
}

knng_status knng_reset_sets(knng_context* ctx, uint32_t k) {
    return knng::guarded(ctx, [&](Context& c) {
        knng::require_points(c);
        knng::alloc_sets(c, k);
        KNNG_CUDA(cudaStreamSynchronize(c.stream));
    });
}

knng_status knng_begin_rep(knng_context* ctx) {
    return knng::guarded(ctx, [&](Context& c) {
        knng::require_points(c);
        knng::launch_iota(c);
        KNNG_CUDA(cudaStreamSynchronize(c.stream));
    });
}

knng_status knng_split_nodes(knng_context* ctx, uint32_t count, const uint32_t* starts, const uint32_t* ends,
                             const float* coefs, const float* offsets, uint32_t* out_mids) {
    return knng::guarded(ctx, [&](Context& c) {
        knng::require_points(c);
        if (count == 0) return;
        if (!starts || !ends || !coefs || !offsets || !out_mids) knng::fail(KNNG_ERR_INVALID_ARGUMENT, "null array");
        std::vector<std::pair<uint32_t, uint32_t>> order;
        for (uint32_t i = 0; i < count; ++i) {
            if (starts[i] >= ends[i] || ends[i] > c.n) knng::fail(KNNG_ERR_INVALID_ARGUMENT, "node range out of bounds");
            order.emplace_back(starts[i], ends[i]);
        }
        std::sort(order.begin(), order.end());
        for (size_t i = 1; i < order.size(); ++i)
            if (order[i].first < order[i - 1].second) knng::fail(KNNG_ERR_INVALID_ARGUMENT, "node ranges overlap");
        uint32_t* d_s = knng::upload(c, "sn_start", starts, count);
        std::vector<float> padded(static_cast<size_t>(count) * c.ld, 0.0f);
        for (uint32_t i = 0; i < count; ++i)
            std::memcpy(&padded[static_cast<size_t>(i) * c.ld], coefs + static_cast<size_t>(i) * c.d, c.d * sizeof(float));
        float* d_c = knng::upload(c, "sn_coefs", padded.data(), padded.size());
        float* d_o = knng::upload(c, "sn_offsets", offsets, count);
        uint32_t* d_t = static_cast<uint32_t*>(knng::scratch(c, "sn_true", count * sizeof(uint32_t)));
        knng::launch_partition(c, count, starts, ends, d_s, d_c, d_o, d_t);
        std::vector<uint32_t> t(count);
        knng::download(c, t.data(), d_t, count);
        for (uint32_t i = 0; i < count; ++i) out_mids[i] = starts[i] + t[i];
    });
}

knng_status knng_farthest_pair(knng_context* ctx, uint32_t count, const uint64_t* offsets, const uint32_t* positions,
                               uint32_t* out_first, uint32_t* out_second, int32_t* out_ok) {
    return knng::guarded(ctx, [&](Context& c) {
        knng::require_points(c);
        if (count == 0) return;
        if (!offsets || !out_first || !out_second || !out_ok) knng::fail(KNNG_ERR_INVALID_ARGUMENT, "null array");
        const uint64_t total = offsets[count];
        uint32_t max_list = 1;
        for (uint32_t i = 0; i < count; ++i) {
            if (offsets[i + 1] < offsets[i]) knng::fail(KNNG_ERR_INVALID_ARGUMENT, "offsets must be non-decreasing");
            max_list = std::max<uint32_t>(max_list, static_cast<uint32_t>(offsets[i + 1] - offsets[i]));
        }
        for (uint64_t i = 0; i < total; ++i)
            if (positions[i] >= c.n) knng::fail(KNNG_ERR_INVALID_ARGUMENT, "position out of bounds");
        uint64_t* d_off = knng::upload(c, "fp_off", offsets, count + 1);
        uint32_t* d_pos = knng::upload(c, "fp_pos", positions, total);
        uint32_t* f = static_cast<uint32_t*>(knng::scratch(c, "fp_first", count * sizeof(uint32_t)));
        uint32_t* s = static_cast<uint32_t*>(knng::scratch(c, "fp_second", count * sizeof(uint32_t)));
        int32_t* ok = static_cast<int32_t*>(knng::scratch(c, "fp_ok", count * sizeof(int32_t)));
        float* c1 = static_cast<float*>(knng::scratch(c, "fp_c1", static_cast<size_t>(count) * c.ld * sizeof(float)));
        float* c2 = static_cast<float*>(knng::scratch(c, "fp_c2", static_cast<size_t>(count) * c.ld * sizeof(float)));
        knng::launch_farthest_pair(c, count, d_off, d_pos, max_list, f, s, ok, c1, c2);
        knng::download(c, out_first, f, count);
        knng::download(c, out_second, s, count);
        knng::download(c, out_ok, ok, count);
    });
}

knng_status knng_lloyd(knng_context* ctx, uint32_t count, const uint32_t* starts, const uint32_t* ends,
                       const uint64_t* lloyd_offsets, const uint32_t* lloyd_positions, const float* c1_start,
                       const float* c2_start, uint32_t iters, float* out_coefs, float* out_offsets, int32_t* out_ok) {
    return knng::guarded(ctx, [&](Context& c) {
        knng::require_points(c);
        if (count == 0) return;
        if (!starts || !ends || !lloyd_offsets || !c1_start || !c2_start || !out_coefs || !out_offsets || !out_ok)
            knng::fail(KNNG_ERR_INVALID_ARGUMENT, "null array");
        for (uint32_t i = 0; i < count; ++i)
            if (starts[i] >= ends[i] || ends[i] > c.n) knng::fail(KNNG_ERR_INVALID_ARGUMENT, "node range out of bounds");
        const uint64_t total = lloyd_offsets[count];
        for (uint64_t i = 0; i < total; ++i)
            if (lloyd_positions[i] >= c.n) knng::fail(KNNG_ERR_INVALID_ARGUMENT, "position out of bounds");
        const uint32_t ld = c.ld;
        std::vector<float> h1(static_cast<size_t>(count) * ld, 0.f), h2(static_cast<size_t>(count) * ld, 0.f);
        for (uint32_t i = 0; i < count; ++i) {
            std::memcpy(&h1[static_cast<size_t>(i) * ld], c1_start + static_cast<size_t>(i) * c.d, c.d * sizeof(float));
            std::memcpy(&h2[static_cast<size_t>(i) * ld], c2_start + static_cast<size_t>(i) * c.d, c.d * sizeof(float));
        }
        float* d1 = knng::upload(c, "ll_c1", h1.data(), h1.size());
        float* d2 = knng::upload(c, "ll_c2", h2.data(), h2.size());
        uint32_t* d_pos = knng::upload(c, "ll_pos", lloyd_positions, total);
        std::vector<int32_t> ones(count + 1, 1);
        int32_t* d_ok = knng::upload(c, "ll_ok", ones.data(), count + 1);
        float* d_coefs = static_cast<float*>(knng::scratch(c, "ll_coefs", static_cast<size_t>(count) * ld * sizeof(float)));
        float* d_offs = static_cast<float*>(knng::scratch(c, "ll_offs", count * sizeof(float)));
        knng::launch_lloyd(c, count, starts, ends, lloyd_offsets, d_pos, d1, d2, iters, d_coefs, d_offs, d_ok);
        std::vector<float> hc(static_cast<size_t>(count) * ld);
        knng::download(c, hc.data(), d_coefs, hc.size());
        for (uint32_t i = 0; i < count; ++i)
            std::memcpy(out_coefs + static_cast<size_t>(i) * c.d, &hc[static_cast<size_t>(i) * ld], c.d * sizeof(float));
        knng::download(c, out_offsets, d_offs, count);
        std::vector<int32_t> hok(count + 1);
        knng::download(c, hok.data(), d_ok, count + 1);
        if (hok[count]) knng::fail(KNNG_ERR_CUDA, "Lloyd sums: a bulk-copy wait gave up");
        std::memcpy(out_ok, hok.data(), count * sizeof(int32_t));
    });
}

knng_status knng_process_leaves(knng_context* ctx, uint32_t count, const uint32_t* starts, const uint32_t* ends) {
    return knng::guarded(ctx, [&](Context& c) {
        knng::require_sets(c);
        if (count == 0) return;
        if (!starts || !ends) knng::fail(KNNG_ERR_INVALID_ARGUMENT, "null array");
        uint32_t max_bucket = 1;
        std::vector<std::pair<uint32_t, uint32_t>> order;
        for (uint32_t i = 0; i < count; ++i) {
            if (starts[i] > ends[i] || ends[i] > c.n) knng::fail(KNNG_ERR_INVALID_ARGUMENT, "bucket out of bounds");
            if (ends[i] - starts[i] > 4096) knng::fail(KNNG_ERR_INVALID_ARGUMENT, "bucket larger than 4096");
            max_bucket = std::max(max_bucket, ends[i] - starts[i]);
            order.emplace_back(starts[i], ends[i]);
        }
        std::sort(order.begin(), order.end());
        for (size_t i = 1; i < order.size(); ++i)
            if (order[i].first < order[i - 1].second) knng::fail(KNNG_ERR_INVALID_ARGUMENT, "buckets overlap");
        uint32_t* d_s = knng::upload(c, "pl_start", starts, count);
        uint32_t* d_e = knng::upload(c, "pl_end", ends, count);
        knng::launch_leaves(c, count, d_s, d_e, max_bucket, nullptr);
        KNNG_CUDA(cudaStreamSynchronize(c.stream));
    });
}

knng_status knng_run_rep(knng_context* ctx, uint32_t max_leaf, uint32_t lloyd_iters, uint32_t small_threshold,
                         uint64_t seed, uint32_t rep_index, knng_stats* stats) {
    return knng::guarded(ctx, [&](Context& c) {
        if (max_leaf > 4097) knng::fail(KNNG_ERR_INVALID_ARGUMENT, "max_leaf must be <= 4097");
        knng::RepStats st;
        knng::run_rep(c, max_leaf, lloyd_iters, small_threshold, seed, rep_index, st, stats);
        knng::add_rep_stats(stats, st);
        if (stats) stats->reps_done += 1;
    });
}

knng_status knng_kd_rotation(uint32_t new_dims, uint32_t d, uint64_t seed, float* out) {
    if (!out || new_dims < 1 || new_dims > 32 || !knng::dim_supported(d)) return KNNG_ERR_INVALID_ARGUMENT;
    try {
        const std::vector<float> r = knng::kd_rotation(new_dims, d, seed);
        std::copy(r.begin(), r.end(), out);
    } catch (...) {
        return KNNG_ERR_OUT_OF_MEMORY;
    }
    return KNNG_OK;
}

namespace knng {

// One KD repetition with its bookkeeping: the context's leaf list and the
// repetition's statistics.
void kd_rep_step(Context& c, uint32_t max_leaf, uint32_t new_dims, uint64_t seed, uint32_t rep, knng_stats* stats) {
    KdRepResult res;
    run_rep_kd(c, max_leaf, new_dims, seed, rep, res);
    std::vector<std::pair<uint32_t, uint32_t>> lv(res.leaf_start.size());
    for (size_t i = 0; i < lv.size(); ++i) lv[i] = {res.leaf_start[i], res.leaf_end[i]};
    std::sort(lv.begin(), lv.end());
    c.last_leaf_start.resize(lv.size());
    c.last_leaf_end.resize(lv.size());
    for (size_t i = 0; i < lv.size(); ++i) {
        c.last_leaf_start[i] = lv[i].first;
        c.last_leaf_end[i] = lv[i].second;
    }
    RepStats st;
    st.levels = res.levels;
    st.nodes = res.nodes;
    st.restarts = res.restarts;
    st.fallbacks = res.fallbacks;
    st.ms_split = res.ms_split;
    st.ms_leaf = res.ms_leaf;
    add_rep_stats(stats, st);
    if (stats) {
        stats->reps_done += 1;
        stats->buckets += lv.size();
        stats->leaf_launches += lv.empty() ? 0 : 1;
        stats->ms_leaf_kernel += res.ms_leaf;
    }
}

}  // namespace knng

knng_status knng_run_rep_kd(knng_context* ctx, uint32_t max_leaf, uint32_t new_dims, uint64_t seed,
                            uint32_t rep_index, knng_stats* stats) {
    return knng::guarded(ctx, [&](Context& c) {
        if (max_leaf < 2 || max_leaf > 4097) knng::fail(KNNG_ERR_INVALID_ARGUMENT, "max_leaf must be in [2, 4097]");
        knng::require_sets(c);
        knng::kd_rep_step(c, max_leaf, new_dims, seed, rep_index, stats);
    });
}

knng_status knng_build_kd(knng_context* ctx, const float* points, uint32_t n, uint32_t d, uint64_t ld_bytes,
                          const knng_params* params, uint32_t new_dims, uint32_t* out_ids, float* out_dists,
                          knng_stats* stats) {
    return knng::guarded(ctx, [&](Context& c) {
        knng::validate_params(params);
        if (params->precision != KNNG_PRECISION_FP32)
            knng::fail(KNNG_ERR_INVALID_ARGUMENT, "the KD build computes in FP32");
        if (new_dims < 1 || new_dims > 32) knng::fail(KNNG_ERR_INVALID_ARGUMENT, "new_dims must be in [1, 32]");
        if (!out_ids) knng::fail(KNNG_ERR_INVALID_ARGUMENT, "null output");
        if (stats) std::memset(stats, 0, sizeof(*stats));
        knng::load_points(c, points, n, d, ld_bytes, false, false);
        knng::alloc_sets(c, params->k);
        knng::EventPair total_t(c);
        const uint64_t launches0 = c.launches;
        for (uint32_t r = 0; r < params->reps; ++r) {
            const uint32_t leaf = (params->max_leaf_odd != 0 && (r % 2 == 1)) ? params->max_leaf_odd : params->max_leaf;
            knng::kd_rep_step(c, leaf, new_dims, params->seed, r, stats);
        }
        for (uint32_t pass = 0; pass < params->refine; ++pass) {
            knng::EventPair rt(c);
            const uint64_t ch = knng::run_refine(c);
            knng::add_refine_stats(stats, c, ch, rt.stop(c));
        }
        const double ms = total_t.stop(c);
        if (stats) {
            stats->ms_total += ms;
            stats->kernel_launches += c.launches - launches0;
        }
        const size_t nk = static_cast<size_t>(c.n) * c.k;
        knng::EventPair ft(c);
        uint32_t* d_ids = static_cast<uint32_t*>(knng::scratch(c, "fin_ids", nk * sizeof(uint32_t)));
        float* d_dist = out_dists ? static_cast<float*>(knng::scratch(c, "fin_dist", nk * sizeof(float))) : nullptr;
        knng::launch_finalize(c, d_ids, d_dist);
        if (stats) stats->ms_finalize += ft.stop(c);
        knng::download(c, out_ids, d_ids, nk);
        if (out_dists) knng::download(c, out_dists, d_dist, nk);
    });
}

knng_status knng_tune_buckets(knng_context* ctx, uint32_t max_leaf, uint32_t lloyd_iters, uint32_t small_threshold,
                              uint64_t seed, double* out_ms, uint32_t* out_choice) {
    return knng::guarded(ctx, [&](Context& c) {
        if (max_leaf < 2 || max_leaf > 4097) knng::fail(KNNG_ERR_INVALID_ARGUMENT, "max_leaf must be in [2, 4097]");
        knng::require_sets(c);
        // The sets before the trials, restored before each trial and after.
        const size_t nk = static_cast<size_t>(c.n) * c.k;
        const size_t sizes[5] = {nk * 4, nk * 4, static_cast<size_t>(c.n) * 4, static_cast<size_t>(c.n) * 4,
                                 static_cast<size_t>(c.n) * 4};
        void* live[5] = {c.set_dist, c.set_id, c.set_size, c.set_maxslot, c.set_bound};
        void* saved[5] = {nullptr, nullptr, nullptr, nullptr, nullptr};
        const bool tc0 = c.leaf_tc;
        const uint32_t ctas0 = c.leaf_ctas;
        auto restore = [&]() {
            for (int i = 0; i < 5; ++i)
                KNNG_CUDA(cudaMemcpyAsync(live[i], saved[i], sizes[i], cudaMemcpyDeviceToDevice, c.stream));
        };
        double ms[4] = {0, 0, 0, 0};
        try {
            for (int i = 0; i < 5; ++i) {
                saved[i] = knng::dev_alloc(c, sizes[i]);
                KNNG_CUDA(cudaMemcpyAsync(saved[i], live[i], sizes[i], cudaMemcpyDeviceToDevice, c.stream));
            }
            // Variants: bucket kernel (every pair / tensor-core filtered) x
            // persistent CTAs per SM (2 / 1); the same repetition each time.
            for (uint32_t v = 0; v < 4; ++v) {
                restore();
                c.leaf_tc = v >= 2;
                c.leaf_ctas = v % 2 == 0 ? 2u : 1u;
                knng::RepStats st;
                knng::run_rep(c, max_leaf, lloyd_iters, small_threshold, seed, 0, st, nullptr);
                ms[v] = st.ms_leaf;
            }
            restore();
            KNNG_CUDA(cudaStreamSynchronize(c.stream));
        } catch (...) {
            c.leaf_tc = tc0;
            c.leaf_ctas = ctas0;
            for (int i = 0; i < 5; ++i) knng::dev_free(c, saved[i], sizes[i]);
            c.snap_prev_valid = false;
            throw;
        }
        for (int i = 0; i < 5; ++i) knng::dev_free(c, saved[i], sizes[i]);
        uint32_t best = 0;
        for (uint32_t v = 1; v < 4; ++v)
            if (ms[v] < ms[best]) best = v;
        c.leaf_tc = best >= 2;
        c.leaf_ctas = best % 2 == 0 ? 2u : 1u;
        c.snap_prev_valid = false;
        if (out_ms)
            for (int v = 0; v < 4; ++v) out_ms[v] = ms[v];
        if (out_choice) *out_choice = best;
    });
}

knng_status knng_get_leaves(knng_context* ctx, uint32_t capacity, uint32_t* starts, uint32_t* ends,
                            uint32_t* out_count) {
    return knng::guarded(ctx, [&](Context& c) {
        const uint32_t nl = static_cast<uint32_t>(c.last_leaf_start.size());
        if (out_count) *out_count = nl;
        if (!starts || !ends) return;
        const uint32_t m = std::min(capacity, nl);
        std::memcpy(starts, c.last_leaf_start.data(), m * sizeof(uint32_t));
        std::memcpy(ends, c.last_leaf_end.data(), m * sizeof(uint32_t));
    });
}

knng_status knng_refine(knng_context* ctx, uint64_t* out_changed, knng_stats* stats) {
    return knng::guarded(ctx, [&](Context& c) {
        knng::require_sets(c);
        knng::EventPair t(c);
        const uint64_t ch = knng::run_refine(c);
        const double ms = t.stop(c);
        if (out_changed) *out_changed = ch;
        knng::add_refine_stats(stats, c, ch, ms);
    });
}

knng_status knng_get_indices(knng_context* ctx, uint32_t* out) {
    return knng::guarded(ctx, [&](Context& c) {
        knng::require_points(c);
        if (!out) knng::fail(KNNG_ERR_INVALID_ARGUMENT, "null output");
        knng::download(c, out, c.indices, c.n);
    });
}

knng_status knng_set_indices(knng_context* ctx, const uint32_t* in) {
    return knng::guarded(ctx, [&](Context& c) {
        knng::require_points(c);
        if (!in) knng::fail(KNNG_ERR_INVALID_ARGUMENT, "null input");
        std::vector<uint8_t> seen(c.n, 0);
        for (uint32_t i = 0; i < c.n; ++i) {
            if (in[i] >= c.n || seen[in[i]]) knng::fail(KNNG_ERR_INVALID_ARGUMENT, "indices must be a permutation");
            seen[in[i]] = 1;
        }
        KNNG_CUDA(cudaMemcpyAsync(c.indices, in, c.n * sizeof(uint32_t), cudaMemcpyHostToDevice, c.stream));
        KNNG_CUDA(cudaStreamSynchronize(c.stream));
    });
}

knng_status knng_get_sets(knng_context* ctx, float* dist, uint32_t* ids, uint32_t* sizes, uint32_t* maxslot,
                          float* bounds) {
    return knng::guarded(ctx, [&](Context& c) {
        knng::require_sets(c);
        const size_t nk = static_cast<size_t>(c.n) * c.k;
        if (dist) knng::download(c, dist, c.set_dist, nk);
        if (ids) knng::download(c, ids, c.set_id, nk);
        if (sizes) knng::download(c, sizes, c.set_size, c.n);
        if (maxslot) knng::download(c, maxslot, c.set_maxslot, c.n);
        if (bounds) knng::download(c, bounds, c.set_bound, c.n);
    });
}

knng_status knng_set_sets(knng_context* ctx, const float* dist, const uint32_t* ids, const uint32_t* sizes,
                          const uint32_t* maxslot, const float* bounds) {
    return knng::guarded(ctx, [&](Context& c) {
        knng::require_sets(c);
        if (!dist || !ids || !sizes || !maxslot || !bounds) knng::fail(KNNG_ERR_INVALID_ARGUMENT, "null array");
        for (uint32_t i = 0; i < c.n; ++i) {
            if (sizes[i] > c.k) knng::fail(KNNG_ERR_INVALID_ARGUMENT, "set size above k");
            if (sizes[i] == c.k && maxslot[i] >= c.k) knng::fail(KNNG_ERR_INVALID_ARGUMENT, "full set without a max slot");
        }
        c.snap_prev_valid = false;  // the sets change other than by offers
        const size_t nk = static_cast<size_t>(c.n) * c.k;
        KNNG_CUDA(cudaMemcpyAsync(c.set_dist, dist, nk * sizeof(float), cudaMemcpyHostToDevice, c.stream));
        KNNG_CUDA(cudaMemcpyAsync(c.set_id, ids, nk * sizeof(uint32_t), cudaMemcpyHostToDevice, c.stream));
        KNNG_CUDA(cudaMemcpyAsync(c.set_size, sizes, c.n * sizeof(uint32_t), cudaMemcpyHostToDevice, c.stream));
        KNNG_CUDA(cudaMemcpyAsync(c.set_maxslot, maxslot, c.n * sizeof(uint32_t), cudaMemcpyHostToDevice, c.stream));
        KNNG_CUDA(cudaMemcpyAsync(c.set_bound, bounds, c.n * sizeof(float), cudaMemcpyHostToDevice, c.stream));
        KNNG_CUDA(cudaStreamSynchronize(c.stream));
    });
}

namespace {
// Neighbour-set state file: "KNNGSETS", version, n, k, 0 (5 x 4 bytes after
// the tag), then dist f32[n*k], id u32[n*k], size u32[n], max slot u32[n],
// bound f32[n], little-endian as written by this host.
constexpr char kSetsTag[8] = {'K', 'N', 'N', 'G', 'S', 'E', 'T', 'S'};
constexpr uint32_t kSetsVersion = 1;
}  // namespace

knng_status knng_save_sets(knng_context* ctx, const char* path) {
    return knng::guarded(ctx, [&](Context& c) {
        knng::require_sets(c);
        if (!path) knng::fail(KNNG_ERR_INVALID_ARGUMENT, "null path");
        const size_t nk = static_cast<size_t>(c.n) * c.k;
        std::vector<float> dist(nk), bound(c.n);
        std::vector<uint32_t> ids(nk), size(c.n), maxslot(c.n);
        knng::download(c, dist.data(), c.set_dist, nk);
        knng::download(c, ids.data(), c.set_id, nk);
        knng::download(c, size.data(), c.set_size, c.n);
        knng::download(c, maxslot.data(), c.set_maxslot, c.n);
        knng::download(c, bound.data(), c.set_bound, c.n);
        std::FILE* f = std::fopen(path, "wb");
        if (!f) knng::fail(KNNG_ERR_INVALID_ARGUMENT, std::string("cannot write ") + path);
        const uint32_t head[4] = {kSetsVersion, c.n, c.k, 0u};
        bool ok = std::fwrite(kSetsTag, 1, 8, f) == 8 && std::fwrite(head, 4, 4, f) == 4 &&
                  std::fwrite(dist.data(), 4, nk, f) == nk && std::fwrite(ids.data(), 4, nk, f) == nk &&
                  std::fwrite(size.data(), 4, c.n, f) == c.n && std::fwrite(maxslot.data(), 4, c.n, f) == c.n &&
                  std::fwrite(bound.data(), 4, c.n, f) == c.n;
        ok = (std::fclose(f) == 0) && ok;
        if (!ok) knng::fail(KNNG_ERR_INVALID_ARGUMENT, std::string("short write to ") + path);
    });
}

knng_status knng_load_sets(knng_context* ctx, const char* path) {
    return knng::guarded(ctx, [&](Context& c) {
        knng::require_points(c);
        if (!path) knng::fail(KNNG_ERR_INVALID_ARGUMENT, "null path");
        std::FILE* f = std::fopen(path, "rb");
        if (!f) knng::fail(KNNG_ERR_INVALID_ARGUMENT, std::string("cannot read ") + path);
        char tag[8];
        uint32_t head[4];
        bool ok = std::fread(tag, 1, 8, f) == 8 && std::memcmp(tag, kSetsTag, 8) == 0 &&
                  std::fread(head, 4, 4, f) == 4 && head[0] == kSetsVersion;
        if (!ok || head[1] != c.n || head[2] == 0 || head[2] > static_cast<uint32_t>(knng::kMaxK)) {
            std::fclose(f);
            knng::fail(KNNG_ERR_INVALID_ARGUMENT, "not a set-state file of this point count");
        }
        const uint32_t k = head[2];
        const size_t nk = static_cast<size_t>(c.n) * k;
        std::vector<float> dist(nk), bound(c.n);
        std::vector<uint32_t> ids(nk), size(c.n), maxslot(c.n);
        ok = std::fread(dist.data(), 4, nk, f) == nk && std::fread(ids.data(), 4, nk, f) == nk &&
             std::fread(size.data(), 4, c.n, f) == c.n && std::fread(maxslot.data(), 4, c.n, f) == c.n &&
             std::fread(bound.data(), 4, c.n, f) == c.n;
        std::fclose(f);
        if (!ok) knng::fail(KNNG_ERR_INVALID_ARGUMENT, "truncated set-state file");
        for (uint32_t i = 0; i < c.n; ++i) {
            if (size[i] > k) knng::fail(KNNG_ERR_INVALID_ARGUMENT, "set size above k");
            if (size[i] == k && maxslot[i] >= k) knng::fail(KNNG_ERR_INVALID_ARGUMENT, "full set without a max slot");
        }
        knng::alloc_sets(c, k);
        c.snap_prev_valid = false;  // the sets change other than by offers
        KNNG_CUDA(cudaMemcpyAsync(c.set_dist, dist.data(), nk * sizeof(float), cudaMemcpyHostToDevice, c.stream));
        KNNG_CUDA(cudaMemcpyAsync(c.set_id, ids.data(), nk * sizeof(uint32_t), cudaMemcpyHostToDevice, c.stream));
        KNNG_CUDA(cudaMemcpyAsync(c.set_size, size.data(), c.n * sizeof(uint32_t), cudaMemcpyHostToDevice, c.stream));
        KNNG_CUDA(
            cudaMemcpyAsync(c.set_maxslot, maxslot.data(), c.n * sizeof(uint32_t), cudaMemcpyHostToDevice, c.stream));
        KNNG_CUDA(cudaMemcpyAsync(c.set_bound, bound.data(), c.n * sizeof(float), cudaMemcpyHostToDevice, c.stream));
        KNNG_CUDA(cudaStreamSynchronize(c.stream));
    });
}

knng_status knng_finalize(knng_context* ctx, uint32_t* out_ids, float* out_dists) {
    return knng::guarded(ctx, [&](Context& c) {
        knng::require_sets(c);
        if (!out_ids) knng::fail(KNNG_ERR_INVALID_ARGUMENT, "null output");
        const size_t nk = static_cast<size_t>(c.n) * c.k;
        uint32_t* d_ids = static_cast<uint32_t*>(knng::scratch(c, "fin_ids", nk * sizeof(uint32_t)));
        float* d_dist = out_dists ? static_cast<float*>(knng::scratch(c, "fin_dist", nk * sizeof(float))) : nullptr;
        knng::launch_finalize(c, d_ids, d_dist);
        knng::download(c, out_ids, d_ids, nk);
        if (out_dists) knng::download(c, out_dists, d_dist, nk);
    });
}

knng_status knng_build(knng_context* ctx, const float* points, uint32_t n, uint32_t d, uint64_t ld_bytes,
                       const knng_params* params, uint32_t* out_ids, float* out_dists, knng_stats* stats) {
    return knng::guarded(ctx, [&](Context& c) {
        knng::validate_params(params);
        if (!out_ids) knng::fail(KNNG_ERR_INVALID_ARGUMENT, "null output");
        if (stats) std::memset(stats, 0, sizeof(*stats));
        knng::load_points(c, points, n, d, ld_bytes, false, false);
        knng::build_all(c, params, stats);
        const size_t nk = static_cast<size_t>(c.n) * c.k;
        knng::EventPair ft(c);
        uint32_t* d_ids = static_cast<uint32_t*>(knng::scratch(c, "fin_ids", nk * sizeof(uint32_t)));
        float* d_dist = out_dists ? static_cast<float*>(knng::scratch(c, "fin_dist", nk * sizeof(float))) : nullptr;
        knng::launch_finalize(c, d_ids, d_dist);
        if (stats) stats->ms_finalize += ft.stop(c);
        knng::download(c, out_ids, d_ids, nk);
        if (out_dists) knng::download(c, out_dists, d_dist, nk);
    });
}

knng_status knng_build_timed(knng_context* ctx, const float* points, uint32_t n, uint32_t d, uint64_t ld_bytes,
                             const knng_params* params, uint64_t build_ms, uint64_t refine_ms, uint32_t* out_ids,
                             float* out_dists, knng_stats* stats) {
    return knng::guarded(ctx, [&](Context& c) {
        knng::validate_params(params);
        if (!out_ids) knng::fail(KNNG_ERR_INVALID_ARGUMENT, "null output");
        if (build_ms == 0) knng::fail(KNNG_ERR_INVALID_ARGUMENT, "build_ms must be positive");
        if (stats) std::memset(stats, 0, sizeof(*stats));
        knng::load_points(c, points, n, d, ld_bytes, false, false);
        knng::build_all(c, params, stats, build_ms, refine_ms);
        const size_t nk = static_cast<size_t>(c.n) * c.k;
        knng::EventPair ft(c);
        uint32_t* d_ids = static_cast<uint32_t*>(knng::scratch(c, "fin_ids", nk * sizeof(uint32_t)));
        float* d_dist = out_dists ? static_cast<float*>(knng::scratch(c, "fin_dist", nk * sizeof(float))) : nullptr;
        knng::launch_finalize(c, d_ids, d_dist);
        if (stats) stats->ms_finalize += ft.stop(c);
        knng::download(c, out_ids, d_ids, nk);
        if (out_dists) knng::download(c, out_dists, d_dist, nk);
    });
}

knng_status knng_build_adaptive(knng_context* ctx, const float* points, uint32_t n, uint32_t d, uint64_t ld_bytes,
                                const knng_params* params, double target_recall, uint32_t sample, uint32_t* out_ids,
                                float* out_dists, knng_stats* stats) {
    return knng::guarded(ctx, [&](Context& c) {
        knng::validate_params(params);
        if (!out_ids) knng::fail(KNNG_ERR_INVALID_ARGUMENT, "null output");
        if (!(target_recall > 0.0 && target_recall <= 1.0)) knng::fail(KNNG_ERR_INVALID_ARGUMENT, "target recall must be in (0, 1]");
        if (sample == 0) knng::fail(KNNG_ERR_INVALID_ARGUMENT, "sample must be positive");
        if (stats) std::memset(stats, 0, sizeof(*stats));
        knng::load_points(c, points, n, d, ld_bytes, false, false);
        knng::build_adaptive(c, params, target_recall, sample, stats);
        const size_t nk = static_cast<size_t>(c.n) * c.k;
        knng::EventPair ft(c);
        uint32_t* d_ids = static_cast<uint32_t*>(knng::scratch(c, "fin_ids", nk * sizeof(uint32_t)));
        float* d_dist = out_dists ? static_cast<float*>(knng::scratch(c, "fin_dist", nk * sizeof(float))) : nullptr;
        knng::launch_finalize(c, d_ids, d_dist);
        if (stats) stats->ms_finalize += ft.stop(c);
        knng::download(c, out_ids, d_ids, nk);
        if (out_dists) knng::download(c, out_dists, d_dist, nk);
    });
}

knng_status knng_build_batch(knng_context* ctx, const float* points, uint32_t n, uint32_t d, uint64_t ld_bytes,
                             const uint32_t* set_offsets, uint32_t n_sets, int on_device, const knng_params* params,
                             uint32_t* out_ids, float* out_dists, knng_stats* stats) {
    return knng::guarded(ctx, [&](Context& c) {
        knng::validate_params(params);
        if (!out_ids || !set_offsets) knng::fail(KNNG_ERR_INVALID_ARGUMENT, "null output or offsets");
        if (n_sets == 0 || set_offsets[0] != 0 || set_offsets[n_sets] != n)
            knng::fail(KNNG_ERR_INVALID_ARGUMENT, "set offsets must run from 0 to n");
        for (uint32_t s = 0; s < n_sets; ++s)
            if (set_offsets[s + 1] <= set_offsets[s]) knng::fail(KNNG_ERR_INVALID_ARGUMENT, "empty or unordered set");
        if (stats) std::memset(stats, 0, sizeof(*stats));
        knng::load_points(c, points, n, d, ld_bytes, on_device != 0, on_device != 0);
        c.set_offsets.assign(set_offsets, set_offsets + n_sets + 1);
        if (n_sets > 1) c.d_set_offsets = knng::upload(c, "set_offsets", set_offsets, n_sets + 1);
        knng::build_all(c, params, stats);
        const size_t nk = static_cast<size_t>(c.n) * c.k;
        knng::EventPair ft(c);
        const uint64_t l0 = c.launches;
        uint32_t* d_ids = on_device ? out_ids : static_cast<uint32_t*>(knng::scratch(c, "fin_ids", nk * sizeof(uint32_t)));
        float* d_dist = on_device ? out_dists
                                  : (out_dists ? static_cast<float*>(knng::scratch(c, "fin_dist", nk * sizeof(float)))
                                               : nullptr);
        knng::launch_finalize(c, d_ids, d_dist);
        knng::launch_rebase_ids(c, d_ids);
        if (stats) {
            stats->ms_finalize += ft.stop(c);
            stats->kernel_launches += c.launches - l0;
        }
        if (on_device) {
            KNNG_CUDA(cudaStreamSynchronize(c.stream));
        } else {
            knng::download(c, out_ids, d_ids, nk);
            if (out_dists) knng::download(c, out_dists, d_dist, nk);
        }
    });
}

knng_status knng_build_device(knng_context* ctx, const float* d_points, uint32_t n, uint32_t d, uint64_t ld_bytes,
                              const knng_params* params, uint32_t* d_out_ids, float* d_out_dists, knng_stats* stats) {
    return knng::guarded(ctx, [&](Context& c) {
        knng::validate_params(params);
        if (!d_out_ids) knng::fail(KNNG_ERR_INVALID_ARGUMENT, "null output");
        if (stats) std::memset(stats, 0, sizeof(*stats));
        knng::load_points(c, d_points, n, d, ld_bytes, true, true);
        knng::build_all(c, params, stats);
        knng::EventPair ft(c);
        const uint64_t l0 = c.launches;
        knng::launch_finalize(c, d_out_ids, d_out_dists);
        if (stats) {
            stats->ms_finalize += ft.stop(c);
            stats->kernel_launches += c.launches - l0;
        }
        KNNG_CUDA(cudaStreamSynchronize(c.stream));
    });
}

knng_status knng_debug_tile_gram_bf16(knng_context* ctx, const float* a, uint32_t m, const float* b, uint32_t n,
                                      uint32_t d, float* out) {
    return knng::guarded(ctx, [&](Context& c) {
        if (!a || !b || !out) knng::fail(KNNG_ERR_INVALID_ARGUMENT, "null array");
        if (m == 0 || n == 0 || m > 128 || n > 128) knng::fail(KNNG_ERR_INVALID_ARGUMENT, "m and n must be in 1..128");
        if (!knng::dim_supported(d)) knng::fail(KNNG_ERR_UNSUPPORTED, "dimension must be 64, 100 or 128");
        float* da = knng::upload(c, "dbg_a", a, static_cast<size_t>(m) * d);
        float* db = knng::upload(c, "dbg_b", b, static_cast<size_t>(n) * d);
        float* dout = static_cast<float*>(knng::scratch(c, "dbg_out", static_cast<size_t>(m) * n * sizeof(float)));
        knng::run_tile_gram_bf16(c, d, da, m, db, n, dout);
        knng::download(c, out, dout, static_cast<size_t>(m) * n);
    });
}

knng_status knng_debug_set_wait_limit(knng_context* ctx, uint32_t polls) {
    return knng::guarded(ctx, [&](Context&) {
        knng::set_split_wait_limit(polls);
        knng::set_refine_wait_limit(polls);
    });
}

knng_status knng_debug_tile_gram(knng_context* ctx, const float* a, uint32_t m, const float* b, uint32_t n, uint32_t d,
                                 float* out) {
    return knng::guarded(ctx, [&](Context& c) {
        if (!a || !b || !out) knng::fail(KNNG_ERR_INVALID_ARGUMENT, "null array");
        if (m == 0 || n == 0 || m > 128 || n > 128) knng::fail(KNNG_ERR_INVALID_ARGUMENT, "m and n must be in 1..128");
        if (!knng::dim_supported(d)) knng::fail(KNNG_ERR_UNSUPPORTED, "dimension must be 64, 100 or 128");
        float* da = knng::upload(c, "dbg_a", a, static_cast<size_t>(m) * d);
        float* db = knng::upload(c, "dbg_b", b, static_cast<size_t>(n) * d);
        float* dout = static_cast<float*>(knng::scratch(c, "dbg_out", static_cast<size_t>(m) * n * sizeof(float)));
        knng::run_tile_gram(c, d, da, m, db, n, dout);
        knng::download(c, out, dout, static_cast<size_t>(m) * n);
    });
}

}  // extern "C"
