// CPU oracle for the k-NN graph build (TEST INFRASTRUCTURE ONLY).
//
// A serial, deterministic restatement of the reference's hot path, used by the
// tests, by __graft_entry__.smoke() and by bench.py's cpu_baseline leg as the
// checker of the CUDA library.  It is never linked into the product.
//
//   canonical_distance / canonical_dot   src/LinearAlgebra.hpp:53-77, :179-200
//   knnset_offer / knnset_argmax         src/KnnSets.hpp:39-57, :59-72, :82-111
//   leaf_all_pairs                       src/KnnSets.hpp:131-160
//   sample_fraction / sample_positions   src/SolutionKmeans.hpp:50-66
//   farthest_pair                        src/SolutionKmeans.hpp:68-101, :103-138
//   split_node (small / large path)      src/SolutionKmeans.hpp:142-311
//   refine                               src/SolutionKmeans.hpp:480-555
//   finalize + pad                       src/KnnSets.hpp:113-126, :334-344
//
// Arithmetic order.  Distances and dot products follow the reference's AVX2
// shape: eight lanes, lane l an FMA chain over dims l, l+8, ... below the
// largest multiple of 8 that is <= d, then the lanes summed left to right into
// 0.0f, then the tail dims added one product at a time (separate multiply and
// add; this file is compiled with -ffp-contract=off).  Centroid sums are
// accumulated in double in point order, as the reference does.
//
// Randomness.  rng_mode 0 draws from std::mt19937(seed) through
// std::uniform_int_distribution<uint32_t>, consumed in depth-first order -- the
// reference's own stream (src/Constants.hpp:22) under a serial scheduler.
// rng_mode 1 draws from the counter-based hash the CUDA library uses
// (keyed by seed, repetition, node range, attempt and draw index), so that a
// whole device-seeded build can be compared with this file.
//
// Deliberate differences, reachable only on degenerate input where the
// reference loops forever or reads out of bounds: a node whose split fails
// (identical sample points, or an empty side) is retried at most
// kMaxAttempts times and then split at its index midpoint; the arg-max of a
// set whose distances are all <= FLT_MIN returns the first slot in the
// reference's scan order instead of index -1.
#include <algorithm>
#include <cfloat>
#include <cmath>
#include <cstdint>
#include <cstring>
#include <limits>
#include <random>
#include <set>
#include <utility>
#include <vector>

namespace {

constexpr uint32_t kMaxAttempts = 64;
constexpr uint32_t kNone = 0xFFFFFFFFu;

// ---------------------------------------------------------------- arithmetic

float canonical_distance(const float* a, const float* b, uint32_t d) {
    const uint32_t main = d / 8 * 8;
    float lane[8] = {0, 0, 0, 0, 0, 0, 0, 0};
    for (uint32_t base = 0; base < main; base += 8) {
        for (uint32_t l = 0; l < 8; ++l) {
            float diff = a[base + l] - b[base + l];
            lane[l] = std::fmaf(diff, diff, lane[l]);
        }
    }
    float acc = 0.0f;
    for (uint32_t l = 0; l < 8; ++l) acc += lane[l];
    for (uint32_t i = main; i < d; ++i) {
        float diff = a[i] - b[i];
        float sq = diff * diff;
        acc += sq;
    }
    return acc;
}

float canonical_dot(const float* a, const float* b, uint32_t d) {
    const uint32_t main = d / 8 * 8;
    float lane[8] = {0, 0, 0, 0, 0, 0, 0, 0};
    for (uint32_t base = 0; base < main; base += 8) {
        for (uint32_t l = 0; l < 8; ++l) lane[l] = std::fmaf(b[base + l], a[base + l], lane[l]);
    }
    float acc = 0.0f;
    for (uint32_t l = 0; l < 8; ++l) acc += lane[l];
    for (uint32_t i = main; i < d; ++i) {
        float p = a[i] * b[i];
        acc += p;
    }
    return acc;
}

// ------------------------------------------------------------------ KnnSet
//
// One bounded set per point: k slots of (dist, id), the filled count, the slot
// holding the current maximum, and the bound (FLT_MAX until the set is full,
// then the maximum).  Unfilled slots hold id 0 and distance 0.

struct Sets {
    uint32_t k = 0;
    std::vector<float> dist;
    std::vector<uint32_t> id;
    std::vector<uint32_t> size;
    std::vector<uint32_t> maxslot;
    std::vector<float> bound;

    void reset(uint32_t n, uint32_t kk) {
        k = kk;
        dist.assign(static_cast<size_t>(n) * k, 0.0f);
        id.assign(static_cast<size_t>(n) * k, 0u);
        size.assign(n, 0u);
        maxslot.assign(n, kNone);
        bound.assign(n, FLT_MAX);
    }
};

// Slot of the largest distance, found the way the reference's 8-lane scan
// finds it: lane l keeps the first strict maximum among slots l, l+8, ...
// (slots past k read as 0), then lanes are compared left to right against a
// running maximum that starts at FLT_MIN.
uint32_t knnset_argmax(const float* dist, uint32_t k) {
    const uint32_t kpad = (k + 7) / 8 * 8;
    auto at = [&](uint32_t s) { return s < k ? dist[s] : 0.0f; };
    float lane_max[8];
    uint32_t lane_idx[8];
    for (uint32_t l = 0; l < 8; ++l) {
        lane_max[l] = at(l);
        lane_idx[l] = l;
    }
    for (uint32_t base = 8; base < kpad; base += 8) {
        for (uint32_t l = 0; l < 8; ++l) {
            float v = at(base + l);
            if (v > lane_max[l]) {
                lane_max[l] = v;
                lane_idx[l] = base + l;
            }
        }
    }
    float best = FLT_MIN;
    uint32_t best_idx = kNone;
    for (uint32_t l = 0; l < 8; ++l) {
        if (lane_max[l] > best) {
            best = lane_max[l];
            best_idx = lane_idx[l];
        }
    }
    if (best_idx == kNone) {
        // Every distance <= FLT_MIN: the reference would index slot -1.  Take the
        // first slot in scan order holding the maximum instead.
        float m = -1.0f;
        for (uint32_t l = 0; l < 8; ++l) {
            if (lane_idx[l] < k && lane_max[l] > m) {
                m = lane_max[l];
                best_idx = lane_idx[l];
            }
        }
    }
    return best_idx;
}

// Offer (cand, d) to point p; the caller has checked d < bound[p].
bool knnset_offer(Sets& s, uint32_t p, uint32_t cand, float d) {
    const uint32_t k = s.k;
    float* dist = &s.dist[static_cast<size_t>(p) * k];
    uint32_t* ids = &s.id[static_cast<size_t>(p) * k];
    uint32_t& size = s.size[p];
    for (uint32_t i = 0; i < size; ++i) {
        if (ids[i] == cand) return false;
    }
    if (size < k) {
        dist[size] = d;
        ids[size] = cand;
        ++size;
        if (size == k) {
            s.maxslot[p] = knnset_argmax(dist, k);
            s.bound[p] = dist[s.maxslot[p]];
        }
        return true;
    }
    const uint32_t slot = s.maxslot[p];
    dist[slot] = d;
    ids[slot] = cand;
    s.maxslot[p] = knnset_argmax(dist, k);
    s.bound[p] = dist[s.maxslot[p]];
    return true;
}

// ------------------------------------------------------------- randomness

uint64_t mix64(uint64_t z) {
    // splitmix64 finaliser (Steele, Lea, Flood 2014).
    z = (z ^ (z >> 30)) * 0xbf58476d1ce4e5b9ULL;
    z = (z ^ (z >> 27)) * 0x94d049bb133111ebULL;
    return z ^ (z >> 31);
}

// Draw t of node [start, end) at the given attempt: a position in [start, end).
uint32_t counter_position(uint64_t seed, uint32_t rep, uint32_t start, uint32_t end, uint32_t attempt, uint32_t t) {
    uint64_t h = mix64(seed + 0x9e3779b97f4a7c15ULL * (static_cast<uint64_t>(rep) + 1));
    h = mix64(h ^ ((static_cast<uint64_t>(start) << 32) | end));
    h = mix64(h ^ ((static_cast<uint64_t>(attempt) << 32) | t));
    const uint64_t n = end - start;
    return start + static_cast<uint32_t>(((h >> 32) * n) >> 32);
}

// ------------------------------------------------------------------ context

struct TraceNode {
    uint32_t start, end, depth, mid, large, attempts;
    std::vector<float> coefs;
    float offset;
    std::vector<float> c1_start, c2_start;
    std::vector<uint32_t> lloyd_positions;  // large nodes: the sample; small nodes: empty (whole range)
    std::vector<uint32_t> start_positions;  // the positions whose farthest pair seeded the node
};

struct Oracle {
    std::vector<float> pts;  // n x d, packed
    uint32_t n = 0, d = 0, k = 0;
    uint32_t rng_mode = 0;
    uint64_t seed = 12345;
    std::mt19937 mt{12345};
    uint32_t rep = 0;
    uint32_t small_threshold = 3000;
    std::vector<uint32_t> indices;
    Sets sets;
    std::vector<TraceNode> trace;
    std::vector<std::pair<uint32_t, uint32_t>> leaves;

    const float* row(uint32_t id) const { return &pts[static_cast<size_t>(id) * d]; }

    uint32_t draw(uint32_t start, uint32_t end, uint32_t attempt, uint32_t t) {
        if (rng_mode == 0) {
            std::uniform_int_distribution<uint32_t> u(start, end - 1);
            return u(mt);
        }
        return counter_position(seed, rep, start, end, attempt, t);
    }
};

// n * (ln n / ln 30)^7 / n, computed as the reference does (double math, float result).
float sample_fraction(uint32_t n) {
    return static_cast<float>(std::pow(std::log(static_cast<double>(n)) / std::log(30.0), 7) / n);
}

uint32_t sample_count(uint32_t n) { return static_cast<uint32_t>(static_cast<float>(n) * sample_fraction(n)); }

uint32_t start_count(uint32_t n) { return static_cast<uint32_t>(std::pow(std::log10(static_cast<double>(n)), 2.5)); }

// Farthest pair (strict >, first pair wins, running maximum from FLT_MIN)
// among the given positions; returns false when no pair exceeds FLT_MIN.
bool farthest_pair(const Oracle& o, const std::vector<uint32_t>& pos, uint32_t m, uint32_t& pi, uint32_t& pj) {
    float best = FLT_MIN;
    bool found = false;
    for (uint32_t i = 0; i + 1 < m; ++i) {
        for (uint32_t j = i + 1; j < m; ++j) {
            float dd = canonical_distance(o.row(o.indices[pos[i]]), o.row(o.indices[pos[j]]), o.d);
            if (dd > best) {
                best = dd;
                pi = i;
                pj = j;
                found = true;
            }
        }
    }
    return found;
}

// between = 0.5 * (c1 + c2); coefs = c1 - between; offset = dot(between, coefs)
void hyperplane(const std::vector<float>& c1, const std::vector<float>& c2, uint32_t d, std::vector<float>& coefs,
                float& offset) {
    std::vector<float> between(d);
    for (uint32_t i = 0; i < d; ++i) {
        float s = c1[i] + c2[i];
        between[i] = 0.5f * s;
    }
    coefs.resize(d);
    for (uint32_t i = 0; i < d; ++i) coefs[i] = c1[i] - between[i];
    offset = canonical_dot(between.data(), coefs.data(), d);
}

// Lloyd update over the given point ids; false when one side is empty.
bool lloyd_step(const Oracle& o, const std::vector<uint32_t>& ids, std::vector<float>& c1, std::vector<float>& c2) {
    std::vector<float> coefs;
    float offset;
    hyperplane(c1, c2, o.d, coefs, offset);
    std::vector<double> s1(o.d, 0.0), s2(o.d, 0.0);
    uint32_t n1 = 0, n2 = 0;
    for (uint32_t id : ids) {
        const float* p = o.row(id);
        if (canonical_dot(coefs.data(), p, o.d) >= offset) {
            ++n1;
            for (uint32_t j = 0; j < o.d; ++j) s1[j] += p[j];
        } else {
            ++n2;
            for (uint32_t j = 0; j < o.d; ++j) s2[j] += p[j];
        }
    }
    if (n1 == 0 || n2 == 0) return false;
    for (uint32_t j = 0; j < o.d; ++j) {
        c1[j] = static_cast<float>(s1[j] / n1);
        c2[j] = static_cast<float>(s2[j] / n2);
    }
    return true;
}

void leaf_all_pairs(Oracle& o, uint32_t start, uint32_t end) {
    for (uint32_t i = start; i + 1 < end; ++i) {
        const uint32_t a = o.indices[i];
        for (uint32_t j = i + 1; j < end; ++j) {
            const uint32_t b = o.indices[j];
            const float dd = canonical_distance(o.row(a), o.row(b), o.d);
            if (dd < o.sets.bound[a]) knnset_offer(o.sets, a, b, dd);
            if (dd < o.sets.bound[b]) knnset_offer(o.sets, b, a, dd);
        }
    }
}

void split_node(Oracle& o, uint32_t start, uint32_t end, uint32_t iters, uint32_t max_group, uint32_t depth) {
    const uint32_t n = end - start;
    if (n < max_group) {
        o.leaves.emplace_back(start, end);
        leaf_all_pairs(o, start, end);
        return;
    }
    const bool large = n >= o.small_threshold;
    TraceNode node;
    node.start = start;
    node.end = end;
    node.depth = depth;
    node.large = large ? 1 : 0;
    std::vector<float> coefs;
    float offset = 0.0f;
    uint32_t mid = start;
    bool done = false;
    uint32_t attempt = 0;
    for (; attempt < kMaxAttempts && !done; ++attempt) {
        // Seeds: the small path draws S positions from the range; the large path
        // draws its whole sample and seeds from its first min(|sample|, S) entries.
        std::vector<uint32_t> pos;
        std::vector<uint32_t> lloyd_ids;
        uint32_t m;
        if (large) {
            const uint32_t cnt = sample_count(n);
            pos.reserve(cnt);
            for (uint32_t t = 0; t < cnt; ++t) pos.push_back(o.draw(start, end, attempt, t));
            m = std::min<uint32_t>(cnt, start_count(n));
            lloyd_ids.reserve(cnt);
            for (uint32_t p : pos) lloyd_ids.push_back(o.indices[p]);
        } else {
            const uint32_t cnt = start_count(n);
            for (uint32_t t = 0; t < cnt; ++t) pos.push_back(o.draw(start, end, attempt, t));
            m = cnt;
            lloyd_ids.assign(o.indices.begin() + start, o.indices.begin() + end);
        }
        uint32_t pi = 0, pj = 0;
        if (!farthest_pair(o, pos, m, pi, pj)) continue;
        std::vector<float> c1(o.row(o.indices[pos[pi]]), o.row(o.indices[pos[pi]]) + o.d);
        std::vector<float> c2(o.row(o.indices[pos[pj]]), o.row(o.indices[pos[pj]]) + o.d);
        node.c1_start = c1;
        node.c2_start = c2;
        bool ok = true;
        for (uint32_t it = 0; it < iters && ok; ++it) ok = lloyd_step(o, lloyd_ids, c1, c2);
        if (!ok) continue;
        hyperplane(c1, c2, o.d, coefs, offset);
        // Stable partition of indices[start, end): side-1 points first.
        std::vector<uint32_t> g1, g2;
        g1.reserve(n);
        g2.reserve(n);
        for (uint32_t i = start; i < end; ++i) {
            const uint32_t id = o.indices[i];
            if (canonical_dot(coefs.data(), o.row(id), o.d) >= offset)
                g1.push_back(id);
            else
                g2.push_back(id);
        }
        if (g1.empty() || g2.empty()) continue;
        std::copy(g1.begin(), g1.end(), o.indices.begin() + start);
        std::copy(g2.begin(), g2.end(), o.indices.begin() + start + g1.size());
        mid = start + static_cast<uint32_t>(g1.size());
        node.lloyd_positions = large ? pos : std::vector<uint32_t>();
        node.start_positions.assign(pos.begin(), pos.begin() + m);
        done = true;
    }
    if (!done) {
        // Degenerate node: keep the order and split at the index midpoint.
        mid = start + n / 2;
        coefs.assign(o.d, 0.0f);
        offset = 0.0f;
        node.c1_start.assign(o.d, 0.0f);
        node.c2_start.assign(o.d, 0.0f);
    }
    node.attempts = attempt;
    node.mid = mid;
    node.coefs = coefs;
    node.offset = offset;
    o.trace.push_back(std::move(node));
    split_node(o, start, mid, iters, max_group, depth + 1);
    split_node(o, mid, end, iters, max_group, depth + 1);
}

}  // namespace

// ------------------------------------------------------------ KD splitter
//
// Restatement of the random-rotation KD solution's repetition
// (SolutionRandomKD::rotateRandom / split, src/SolutionRandomKD.hpp:258-375)
// with the conventions of the library's KD splitter: the node's own points
// give the statistics (the reference reads indices[0 .. size)), the dimension
// draw comes from the counter RNG, a node with every point on one side is
// redrawn up to 64 times and then halved at its index midpoint, and buckets
// go through leaf_all_pairs (the 2-means form's set).

// rotateRandom's vectors (src/SolutionRandomKD.hpp:258-264 with
// randUniformUnitVec, normalizeInPlace and gramSchmidt,
// src/LinearAlgebra.hpp:86-117, :211-222): per vector d normal draws on a
// mt19937 seeded with `seed` (a new normal_distribution each), divided by the
// square root of the float sum of float squares; then each vector minus its
// float projections on the earlier ones, without rescaling (the reference's
// normalize returns its argument).
std::vector<float> kd_vectors(uint32_t nd, uint32_t d, uint64_t seed) {
    std::mt19937 gen(static_cast<std::mt19937::result_type>(seed));
    std::vector<std::vector<float>> v(nd, std::vector<float>(d));
    for (uint32_t h = 0; h < nd; ++h) {
        std::normal_distribution<> g(0, 1);
        for (uint32_t i = 0; i < d; ++i) v[h][i] = static_cast<float>(g(gen));
        float ss = 0.0f;
        for (uint32_t i = 0; i < d; ++i) {
            const float sq = v[h][i] * v[h][i];
            ss += sq;
        }
        const double nrm = std::sqrt(static_cast<double>(ss));
        for (uint32_t i = 0; i < d; ++i) v[h][i] = static_cast<float>(v[h][i] / nrm);
    }
    std::vector<float> out(static_cast<size_t>(nd) * d);
    for (uint32_t i = 0; i < nd; ++i) {
        std::vector<float> ui = v[i];
        for (uint32_t j = 0; j < i; ++j) {
            const float* uj = &out[static_cast<size_t>(j) * d];
            const float s = canonical_dot(uj, v[i].data(), d);
            for (uint32_t t = 0; t < d; ++t) {
                const float prod = s * uj[t];
                ui[t] = ui[t] - prod;
            }
        }
        std::copy(ui.begin(), ui.end(), out.begin() + static_cast<size_t>(i) * d);
    }
    return out;
}

float kd_uniform(uint64_t seed, uint32_t rep, uint32_t start, uint32_t end, uint32_t attempt) {
    uint64_t h = mix64(seed + 0x9e3779b97f4a7c15ULL * (static_cast<uint64_t>(rep) + 1));
    h = mix64(h ^ ((static_cast<uint64_t>(start) << 32) | end));
    h = mix64(h ^ ((static_cast<uint64_t>(attempt) << 32) | 0x4b44u));
    return static_cast<float>(h >> 40) * 5.9604644775390625e-08f;
}

// pickIndexFull's choice (src/SolutionRandomKD.hpp:200-224).
uint32_t kd_pick(const std::vector<double>& var, float u) {
    std::vector<std::pair<double, uint32_t>> pairs;
    float total = 0;
    for (uint32_t j = 0; j < var.size(); ++j) {
        pairs.emplace_back(var[j], j);
        total += var[j];
    }
    std::sort(pairs.begin(), pairs.end(), std::greater{});
    const float sample = u * total;
    float so_far = 0;
    for (auto& [v, j] : pairs) {
        so_far += v;
        if (so_far >= sample) return j;
    }
    return pairs.back().second;
}

struct KdState {
    uint32_t nd = 0, max_leaf = 0;
    uint64_t seed = 0;
    std::vector<float> rot;  // n x nd
};

void kd_split(Oracle& o, const KdState& k, uint32_t start, uint32_t end, uint32_t attempt) {
    const uint32_t size = end - start;
    if (size < k.max_leaf) {
        o.leaves.emplace_back(start, end);
        leaf_all_pairs(o, start, end);
        return;
    }
    // getMean / getVariance (src/SolutionRandomKD.hpp:93-143) sum per TBB
    // block and combine in thread order; here the order is fixed: chunks of
    // 1,024 positions from the node's start, each summed in index order from
    // 0, then the chunk sums in chunk order.
    constexpr uint32_t kChunk = 1024;
    std::vector<double> mean(k.nd), var(k.nd);
    for (uint32_t c = 0; c < k.nd; ++c) {
        auto value = [&](uint32_t i) { return static_cast<double>(k.rot[static_cast<size_t>(o.indices[i]) * k.nd + c]); };
        double sum = 0;
        for (uint32_t b = start; b < end; b += kChunk) {
            double part = 0;
            for (uint32_t i = b; i < std::min(end, b + kChunk); ++i) part += value(i);
            sum += part;
        }
        mean[c] = sum / size;
        double s2 = 0;
        for (uint32_t b = start; b < end; b += kChunk) {
            double part = 0;
            for (uint32_t i = b; i < std::min(end, b + kChunk); ++i) {
                const double diff = value(i) - mean[c];
                part += diff * diff;
            }
            s2 += part;
        }
        var[c] = s2 / (size - 1);
    }
    const uint32_t dim = kd_pick(var, kd_uniform(k.seed, o.rep, start, end, attempt));
    std::vector<uint32_t> first, second;
    for (uint32_t i = start; i < end; ++i) {
        const uint32_t id = o.indices[i];
        (k.rot[static_cast<size_t>(id) * k.nd + dim] < mean[dim] ? first : second).push_back(id);
    }
    uint32_t mid = start + static_cast<uint32_t>(first.size());
    std::copy(first.begin(), first.end(), o.indices.begin() + start);
    std::copy(second.begin(), second.end(), o.indices.begin() + mid);
    if (mid == start || mid == end) {
        if (attempt + 1 < 64) {
            kd_split(o, k, start, end, attempt + 1);
            return;
        }
        mid = start + size / 2;
    }
    kd_split(o, k, start, mid, 0);
    kd_split(o, k, mid, end, 0);
}

extern "C" {

void* ko_create(const float* pts, uint32_t n, uint32_t d, uint32_t ld, uint32_t k, uint32_t rng_mode, uint64_t seed) {
    auto* o = new Oracle();
    o->n = n;
    o->d = d;
    o->k = k;
    o->rng_mode = rng_mode;
    o->seed = seed;
    o->mt.seed(static_cast<uint32_t>(seed));
    o->pts.resize(static_cast<size_t>(n) * d);
    for (uint32_t i = 0; i < n; ++i)
        std::memcpy(&o->pts[static_cast<size_t>(i) * d], pts + static_cast<size_t>(i) * ld, d * sizeof(float));
    o->indices.resize(n);
    std::iota(o->indices.begin(), o->indices.end(), 0u);
    o->sets.reset(n, k);
    return o;
}

void ko_destroy(void* h) { delete static_cast<Oracle*>(h); }

void ko_set_small_threshold(void* h, uint32_t t) { static_cast<Oracle*>(h)->small_threshold = t; }

// One repetition: indices = iota, recursive split in depth-first order, leaves
// processed as they are reached.  rep_index keys the counter RNG.
void ko_rep(void* h, uint32_t iters, uint32_t max_group, uint32_t rep_index) {
    auto* o = static_cast<Oracle*>(h);
    o->rep = rep_index;
    o->trace.clear();
    o->leaves.clear();
    std::iota(o->indices.begin(), o->indices.end(), 0u);
    if (o->n > 0) split_node(*o, 0, o->n, iters, max_group, 0);
}

// Neighbour-of-neighbour pass over a snapshot of every set's k slot ids
// (sorted, unfilled slots included as id 0); candidates in ascending id order.
uint64_t ko_refine(void* h) {
    auto* o = static_cast<Oracle*>(h);
    const uint32_t k = o->k;
    std::vector<uint32_t> snap(o->sets.id);
    for (uint32_t p = 0; p < o->n; ++p) std::sort(snap.begin() + static_cast<size_t>(p) * k, snap.begin() + static_cast<size_t>(p + 1) * k);
    uint64_t changed = 0;
    std::set<uint32_t> cand;
    for (uint32_t p = 0; p < o->n; ++p) {
        cand.clear();
        for (uint32_t a = 0; a < k; ++a) {
            const uint32_t q = snap[static_cast<size_t>(p) * k + a];
            for (uint32_t b = 0; b < k; ++b) cand.insert(snap[static_cast<size_t>(q) * k + b]);
        }
        cand.erase(p);
        uint32_t added = 0;
        for (uint32_t c : cand) {
            const float dd = canonical_distance(o->row(c), o->row(p), o->d);
            if (dd < o->sets.bound[p]) {
                if (knnset_offer(o->sets, p, c, dd)) ++added;
            }
        }
        if (added) ++changed;
    }
    return changed;
}

// Leaves over the current indices (stepwise form of the leaf stage).
void ko_process_leaves(void* h, uint32_t count, const uint32_t* starts, const uint32_t* ends) {
    auto* o = static_cast<Oracle*>(h);
    for (uint32_t i = 0; i < count; ++i) leaf_all_pairs(*o, starts[i], ends[i]);
}

void ko_get_indices(void* h, uint32_t* out) {
    auto* o = static_cast<Oracle*>(h);
    std::memcpy(out, o->indices.data(), o->n * sizeof(uint32_t));
}

void ko_set_indices(void* h, const uint32_t* in) {
    auto* o = static_cast<Oracle*>(h);
    std::memcpy(o->indices.data(), in, o->n * sizeof(uint32_t));
}

void ko_get_sets(void* h, float* dist, uint32_t* ids, uint32_t* sizes, uint32_t* maxslot, float* bounds) {
    auto* o = static_cast<Oracle*>(h);
    const size_t nk = static_cast<size_t>(o->n) * o->k;
    std::memcpy(dist, o->sets.dist.data(), nk * sizeof(float));
    std::memcpy(ids, o->sets.id.data(), nk * sizeof(uint32_t));
    std::memcpy(sizes, o->sets.size.data(), o->n * sizeof(uint32_t));
    std::memcpy(maxslot, o->sets.maxslot.data(), o->n * sizeof(uint32_t));
    std::memcpy(bounds, o->sets.bound.data(), o->n * sizeof(float));
}

void ko_set_sets(void* h, const float* dist, const uint32_t* ids, const uint32_t* sizes, const uint32_t* maxslot,
                 const float* bounds) {
    auto* o = static_cast<Oracle*>(h);
    const size_t nk = static_cast<size_t>(o->n) * o->k;
    std::memcpy(o->sets.dist.data(), dist, nk * sizeof(float));
    std::memcpy(o->sets.id.data(), ids, nk * sizeof(uint32_t));
    std::memcpy(o->sets.size.data(), sizes, o->n * sizeof(uint32_t));
    std::memcpy(o->sets.maxslot.data(), maxslot, o->n * sizeof(uint32_t));
    std::memcpy(o->sets.bound.data(), bounds, o->n * sizeof(float));
}

// Sort each set by (dist, id) ascending; pad rows shorter than k with id 1
// (distance +inf in out_dist).
void ko_finalize(void* h, uint32_t* out_ids, float* out_dist) {
    auto* o = static_cast<Oracle*>(h);
    const uint32_t k = o->k;
    std::vector<std::pair<float, uint32_t>> q;
    for (uint32_t p = 0; p < o->n; ++p) {
        q.clear();
        const uint32_t sz = o->sets.size[p];
        for (uint32_t i = 0; i < sz; ++i)
            q.emplace_back(o->sets.dist[static_cast<size_t>(p) * k + i], o->sets.id[static_cast<size_t>(p) * k + i]);
        std::sort(q.begin(), q.end());
        for (uint32_t i = 0; i < k; ++i) {
            out_ids[static_cast<size_t>(p) * k + i] = i < sz ? q[i].second : 1u;
            if (out_dist) out_dist[static_cast<size_t>(p) * k + i] = i < sz ? q[i].first : INFINITY;
        }
    }
}

uint32_t ko_trace_count(void* h) { return static_cast<uint32_t>(static_cast<Oracle*>(h)->trace.size()); }

// Per split node of the last repetition, in depth-first order.
void ko_trace_get(void* h, uint32_t* starts, uint32_t* ends, uint32_t* depths, uint32_t* mids, uint32_t* large,
                  uint32_t* attempts, float* coefs, float* offsets, float* c1_start, float* c2_start) {
    auto* o = static_cast<Oracle*>(h);
    const uint32_t d = o->d;
    for (size_t i = 0; i < o->trace.size(); ++i) {
        const TraceNode& t = o->trace[i];
        starts[i] = t.start;
        ends[i] = t.end;
        depths[i] = t.depth;
        mids[i] = t.mid;
        large[i] = t.large;
        attempts[i] = t.attempts;
        offsets[i] = t.offset;
        std::memcpy(coefs + i * d, t.coefs.data(), d * sizeof(float));
        std::memcpy(c1_start + i * d, t.c1_start.data(), d * sizeof(float));
        std::memcpy(c2_start + i * d, t.c2_start.data(), d * sizeof(float));
    }
}

// CSR of the Lloyd sample positions (large nodes) and of the seeding positions.
uint64_t ko_trace_lloyd_total(void* h) {
    uint64_t s = 0;
    for (auto& t : static_cast<Oracle*>(h)->trace) s += t.lloyd_positions.size();
    return s;
}

void ko_trace_lloyd(void* h, uint64_t* offsets, uint32_t* positions) {
    auto* o = static_cast<Oracle*>(h);
    uint64_t off = 0;
    for (size_t i = 0; i < o->trace.size(); ++i) {
        offsets[i] = off;
        for (uint32_t p : o->trace[i].lloyd_positions) positions[off++] = p;
    }
    offsets[o->trace.size()] = off;
}

uint64_t ko_trace_start_total(void* h) {
    uint64_t s = 0;
    for (auto& t : static_cast<Oracle*>(h)->trace) s += t.start_positions.size();
    return s;
}

void ko_trace_start(void* h, uint64_t* offsets, uint32_t* positions) {
    auto* o = static_cast<Oracle*>(h);
    uint64_t off = 0;
    for (size_t i = 0; i < o->trace.size(); ++i) {
        offsets[i] = off;
        for (uint32_t p : o->trace[i].start_positions) positions[off++] = p;
    }
    offsets[o->trace.size()] = off;
}

uint32_t ko_leaf_count(void* h) { return static_cast<uint32_t>(static_cast<Oracle*>(h)->leaves.size()); }

void ko_leaves(void* h, uint32_t* starts, uint32_t* ends) {
    auto* o = static_cast<Oracle*>(h);
    for (size_t i = 0; i < o->leaves.size(); ++i) {
        starts[i] = o->leaves[i].first;
        ends[i] = o->leaves[i].second;
    }
}

// `iters` Lloyd steps over the point ids ids[0..count) in that order from the
// centres c1 / c2 (src/SolutionKmeans.hpp:161-186), then the final hyperplane;
// returns 0 when a step left one side empty.
int ko_lloyd(void* h, const uint32_t* ids, uint64_t count, const float* c1_in, const float* c2_in, uint32_t iters,
             float* out_coefs, float* out_offset) {
    const Oracle& o = *static_cast<Oracle*>(h);
    std::vector<uint32_t> list(ids, ids + count);
    std::vector<float> c1(c1_in, c1_in + o.d), c2(c2_in, c2_in + o.d);
    for (uint32_t it = 0; it < iters; ++it)
        if (!lloyd_step(o, list, c1, c2)) return 0;
    std::vector<float> coefs;
    hyperplane(c1, c2, o.d, coefs, *out_offset);
    std::copy(coefs.begin(), coefs.end(), out_coefs);
    return 1;
}

float ko_distance(const float* a, const float* b, uint32_t d) { return canonical_distance(a, b, d); }

float ko_dot(const float* a, const float* b, uint32_t d) { return canonical_dot(a, b, d); }

uint32_t ko_sample_count(uint32_t n) { return sample_count(n); }

uint32_t ko_start_count(uint32_t n) { return start_count(n); }

uint32_t ko_counter_position(uint64_t seed, uint32_t rep, uint32_t start, uint32_t end, uint32_t attempt, uint32_t t) {
    return counter_position(seed, rep, start, end, attempt, t);
}

// Replays offers into one fresh set of capacity k, offering only when
// dist < bound as the leaf loop does.
void ko_knnset_replay(uint32_t k, const uint32_t* cand, const float* dist, uint32_t count, float* out_dist,
                      uint32_t* out_ids, uint32_t* out_size, uint32_t* out_maxslot, float* out_bound) {
    Sets s;
    s.reset(1, k);
    for (uint32_t t = 0; t < count; ++t) {
        if (dist[t] < s.bound[0]) knnset_offer(s, 0, cand[t], dist[t]);
    }
    std::memcpy(out_dist, s.dist.data(), k * sizeof(float));
    std::memcpy(out_ids, s.id.data(), k * sizeof(uint32_t));
    *out_size = s.size[0];
    *out_maxslot = s.maxslot[0];
    *out_bound = s.bound[0];
}


void ko_kd_vectors(uint32_t nd, uint32_t d, uint64_t seed, float* out) {
    const std::vector<float> v = kd_vectors(nd, d, seed);
    std::copy(v.begin(), v.end(), out);
}

// rot[p * nd + c] = dot(vectors[c], x_p) (the reference's dot).
void ko_kd_rotate(void* h, const float* vectors, uint32_t nd, float* out) {
    auto* o = static_cast<Oracle*>(h);
    for (uint32_t p = 0; p < o->n; ++p)
        for (uint32_t c = 0; c < nd; ++c)
            out[static_cast<size_t>(p) * nd + c] = canonical_dot(vectors + static_cast<size_t>(c) * o->d, o->row(p), o->d);
}

// One repetition with the KD splitter (rotation from kd_vectors(nd, d, seed + rep)).
void ko_kd_rep(void* h, uint32_t max_leaf, uint32_t nd, uint64_t seed, uint32_t rep_index) {
    auto* o = static_cast<Oracle*>(h);
    o->rep = rep_index;
    o->trace.clear();
    o->leaves.clear();
    std::iota(o->indices.begin(), o->indices.end(), 0u);
    KdState k;
    k.nd = nd;
    k.max_leaf = max_leaf;
    k.seed = seed;
    const std::vector<float> v = kd_vectors(nd, o->d, seed + rep_index);
    k.rot.resize(static_cast<size_t>(o->n) * nd);
    ko_kd_rotate(h, v.data(), nd, k.rot.data());
    if (o->n > 0) kd_split(*o, k, 0, o->n, 0);
}
}  // extern "C"
