// Host binned-SAH builder of one mesh's BLAS (object space), used by vkb_scene_create.
// Host-only: compiled into the library and, for its CPU tests, by a plain C++ compiler.
#pragma once
#include <algorithm>
#include <cmath>
#include <cstdint>
#include <future>
#include <thread>
#include <vector>
#include <vector_types.h>
#include <vector_functions.h>

#ifndef VKB_BLAS_LEAF_MAX
#define VKB_BLAS_LEAF_MAX 1
#endif

namespace vkb_host {

// Both child boxes of a binary node (the device layout of vkb::BvhNode).
struct alignas(16) SahNode { float4 a, b, c; int4 d; };

// Binned-SAH BLAS over one mesh's triangles (object space), built once at install:
// BVH2 nodes in the device layout (both child boxes per node), leaves of up to
// BLAS_LEAF_MAX triangles referenced as ~((first << 2) | (count - 1)), triangles
// reordered into leaf order.  The per-frame TLAS keeps the GPU LBVH.
constexpr uint32_t BLAS_LEAF_MAX = VKB_BLAS_LEAF_MAX;
struct SahBlas {
    std::vector<SahNode> nodes;
    std::vector<uint32_t> order;  // leaf-ordered original triangle ids
    const float* lo; const float* hi; const float* c;
    std::vector<uint32_t> ids;
    std::vector<uint32_t>* shared_ids = nullptr;   // a sub-builder works on the root builder's ids
    std::vector<uint32_t>& I() { return shared_ids ? *shared_ids : ids; }
    struct Box { float lo[3], hi[3]; };
    static float area(const Box& b) {
        float x = std::max(b.hi[0] - b.lo[0], 0.f), y = std::max(b.hi[1] - b.lo[1], 0.f), z = std::max(b.hi[2] - b.lo[2], 0.f);
        return x * y + y * z + z * x;
    }
    static void grow(Box& a, const float* l, const float* h) { for (int k = 0; k < 3; ++k) { a.lo[k] = std::min(a.lo[k], l[k]); a.hi[k] = std::max(a.hi[k], h[k]); } }
    static Box empty() { Box b; for (int k = 0; k < 3; ++k) { b.lo[k] = INFINITY; b.hi[k] = -INFINITY; } return b; }
    static void set_child(SahNode& n, int side, const Box& b, int ref) {
        if (side == 0) { n.a = make_float4(b.lo[0], b.hi[0], b.lo[1], b.hi[1]); n.c.x = b.lo[2]; n.c.y = b.hi[2]; n.d.x = ref; }
        else { n.b = make_float4(b.lo[0], b.hi[0], b.lo[1], b.hi[1]); n.c.z = b.lo[2]; n.c.w = b.hi[2]; n.d.y = ref; }
    }
    // Returns the reference of the subtree over ids[first, first+count) and its box.
    static constexpr int BINS = 16;
    struct Bins { Box bb[3][BINS]; uint32_t cnt[3][BINS]; };
    // Boxes of the triangles and of their centroids over ids[a, e).
    void bounds_range(const std::vector<uint32_t>& ids, uint32_t a, uint32_t e, Box& b, Box& cb) const {
        b = empty(); cb = empty();
        for (uint32_t i = a; i < e; ++i) { grow(b, lo + 3 * ids[i], hi + 3 * ids[i]); grow(cb, c + 3 * ids[i], c + 3 * ids[i]); }
    }
    // One pass over ids[a, e) binning every axis at once.
    void bin_range(const std::vector<uint32_t>& ids, uint32_t a, uint32_t e, const Box& cb, const float* sc, Bins& out) const {
        for (int ax = 0; ax < 3; ++ax)
            for (int k = 0; k < BINS; ++k) { out.bb[ax][k] = empty(); out.cnt[ax][k] = 0; }
        for (uint32_t i = a; i < e; ++i) {
            const uint32_t t = ids[i];
            for (int ax = 0; ax < 3; ++ax) {
                if (!(sc[ax] > 0.f)) continue;
                const int k = std::min(BINS - 1, int((c[3 * t + ax] - cb.lo[ax]) * sc[ax]));
                grow(out.bb[ax][k], lo + 3 * t, hi + 3 * t);
                out.cnt[ax][k]++;
            }
        }
    }
    // Threads for the passes over one node: the node's share of the build's threads, for
    // nodes large enough to pay for them.  Box growth is min/max and counts are integers,
    // so chunk results merge to exactly the one-pass values.
    unsigned node_threads(uint32_t count, int depth) const {
        const unsigned share = std::max(1u, threads_total >> std::min(depth, 16));
        return std::max(1u, std::min<unsigned>(share, count / 65536u));
    }
    int build(uint32_t first, uint32_t count, Box& out, int depth) {
        std::vector<uint32_t>& ids = I();
        const unsigned nt = node_threads(count, depth);
        auto chunk = [&](unsigned j) { return first + uint32_t(uint64_t(count) * j / nt); };
        Box b = empty(), cb = empty();
        if (nt > 1) {
            std::vector<Box> pb(nt), pc(nt);
            std::vector<std::future<void>> jobs;
            for (unsigned j = 1; j < nt; ++j)
                jobs.push_back(std::async(std::launch::async, [&, j] { bounds_range(ids, chunk(j), chunk(j + 1), pb[j], pc[j]); }));
            bounds_range(ids, chunk(0), chunk(1), pb[0], pc[0]);
            for (auto& f : jobs) f.get();
            for (unsigned j = 0; j < nt; ++j) { grow(b, pb[j].lo, pb[j].hi); grow(cb, pc[j].lo, pc[j].hi); }
        } else {
            bounds_range(ids, first, first + count, b, cb);
        }
        out = b;
        float best = INFINITY; int best_axis = -1, best_bin = 0;
        if (count > 1 && depth < 60) {
            float sc[3];
            for (int axis = 0; axis < 3; ++axis) {
                const float l = cb.lo[axis], h = cb.hi[axis];
                sc[axis] = (h > l) ? float(BINS) / (h - l) : 0.f;
            }
            Bins bins;
            if (nt > 1) {
                std::vector<Bins> part(nt);
                std::vector<std::future<void>> jobs;
                for (unsigned j = 1; j < nt; ++j)
                    jobs.push_back(std::async(std::launch::async, [&, j] { bin_range(ids, chunk(j), chunk(j + 1), cb, sc, part[j]); }));
                bin_range(ids, chunk(0), chunk(1), cb, sc, part[0]);
                for (auto& f : jobs) f.get();
                bins = part[0];
                for (unsigned j = 1; j < nt; ++j)
                    for (int ax = 0; ax < 3; ++ax)
                        for (int k = 0; k < BINS; ++k) { grow(bins.bb[ax][k], part[j].bb[ax][k].lo, part[j].bb[ax][k].hi); bins.cnt[ax][k] += part[j].cnt[ax][k]; }
            } else {
                bin_range(ids, first, first + count, cb, sc, bins);
            }
            for (int axis = 0; axis < 3; ++axis) {
                if (!(sc[axis] > 0.f)) continue;
                const Box* bb = bins.bb[axis];
                const uint32_t* cnt = bins.cnt[axis];
                float la[BINS]; uint32_t lc[BINS];
                Box acc = empty(); uint32_t ac = 0;
                for (int k = 0; k < BINS; ++k) { grow(acc, bb[k].lo, bb[k].hi); ac += cnt[k]; la[k] = area(acc); lc[k] = ac; }
                acc = empty(); ac = 0;
                for (int k = BINS - 1; k > 0; --k) {
                    grow(acc, bb[k].lo, bb[k].hi); ac += cnt[k];
                    if (lc[k - 1] == 0 || ac == 0) continue;
                    float cost = la[k - 1] * float(lc[k - 1]) + area(acc) * float(ac);
                    if (cost < best) { best = cost; best_axis = axis; best_bin = k; }
                }
            }
        }
        float parent = area(b);
        // SAH with traversal cost 1 and triangle cost 1, relative to the parent's area.
        bool leaf = count == 1 || (count <= BLAS_LEAF_MAX && (best_axis < 0 || float(count) * parent <= parent + best));
        if (!leaf && best_axis < 0 && count > BLAS_LEAF_MAX) best_axis = -2;  // degenerate centroids: median split
        if (leaf) {
            uint32_t f = uint32_t(order.size());
            for (uint32_t i = first; i < first + count; ++i) order.push_back(ids[i]);
            return ~int((f << 2) | (count - 1));
        }
        uint32_t mid;
        if (best_axis >= 0) {
            float l = cb.lo[best_axis], sc = float(BINS) / (cb.hi[best_axis] - l);
            auto it = std::partition(ids.begin() + first, ids.begin() + first + count, [&](uint32_t p) {
                return std::min(BINS - 1, int((c[3 * p + best_axis] - l) * sc)) < best_bin; });
            mid = uint32_t(it - ids.begin());
            if (mid == first || mid == first + count) mid = first + count / 2;
        } else {
            mid = first + count / 2;
        }
        int index = int(nodes.size());
        nodes.push_back(SahNode{});
        Box lb, rb;
        int lref, rref;
        if (depth < spawn_depth && count >= SPAWN_MIN) {
            // Both halves on their own threads into their own buffers, then appended in
            // depth-first order (left subtree, then right) with node and leaf offsets:
            // the same tree, node numbering and leaf order as the one-thread build.
            SahBlas left = sub(), right = sub();
            auto job = std::async(std::launch::async, [&] { return left.build(first, mid - first, lb, depth + 1); });
            int r = right.build(mid, first + count - mid, rb, depth + 1);
            int l = job.get();
            lref = splice(left, l);
            rref = splice(right, r);
        } else {
            lref = build(first, mid - first, lb, depth + 1);
            rref = build(mid, first + count - mid, rb, depth + 1);
        }
        set_child(nodes[index], 0, lb, lref);
        set_child(nodes[index], 1, rb, rref);
        nodes[index].d.z = nodes[index].d.w = 0;
        return index;
    }
    // Subtrees of at least SPAWN_MIN triangles above spawn_depth build on their own threads.
    static constexpr uint32_t SPAWN_MIN = 32768;
    int spawn_depth = 0;
    unsigned threads_total = 1;
    SahBlas sub() {
        SahBlas t;
        t.lo = lo; t.hi = hi; t.c = c;
        t.spawn_depth = spawn_depth;
        t.threads_total = threads_total;
        t.shared_ids = shared_ids ? shared_ids : &ids;
        return t;
    }
    // Appends subtree t (root reference r in t's numbering) and returns r in this numbering.
    int splice(SahBlas& t, int r) {
        const int node_base = int(nodes.size());
        const uint32_t leaf_base = uint32_t(order.size());
        auto fix = [&](int ref) {
            if (ref >= 0) return ref + node_base;
            const uint32_t v = uint32_t(~ref);
            return ~int((((v >> 2) + leaf_base) << 2) | (v & 3u));
        };
        for (SahNode& n : t.nodes) { n.d.x = fix(n.d.x); n.d.y = fix(n.d.y); nodes.push_back(n); }
        order.insert(order.end(), t.order.begin(), t.order.end());
        return fix(r);
    }
    // threads: subtree threads to use (0: every hardware thread, 1: build on this thread).
    void run(uint32_t n, const float* l, const float* h, const float* cent, unsigned threads = 0) {
        lo = l; hi = h; c = cent;
        ids.resize(n);
        for (uint32_t i = 0; i < n; ++i) ids[i] = i;
        nodes.clear(); order.clear();
        nodes.push_back(SahNode{});  // root
        Box b = empty(), cb = empty();
        for (uint32_t i = 0; i < n; ++i) grow(b, l + 3 * i, h + 3 * i);
        (void)cb;
        if (n <= BLAS_LEAF_MAX) {
            order.assign(ids.begin(), ids.end());
            set_child(nodes[0], 0, b, ~int(n - 1));
            set_child(nodes[0], 1, empty(), ~int(n - 1));
            nodes[0].d.z = nodes[0].d.w = 0;
            return;
        }
        // The root is node 0: build its two halves under it.
        Box rb;
        nodes.pop_back();
        const unsigned hw = threads ? threads : std::max(1u, std::thread::hardware_concurrency());
        threads_total = hw;
        spawn_depth = 0;
        while ((1u << spawn_depth) < hw && spawn_depth < 8) ++spawn_depth;
        int r = build(0, n, rb, 0);
        (void)r;  // r == 0: the root node was allocated first
    }
};


}  // namespace vkb_host
