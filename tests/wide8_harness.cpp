// Test harness (tests only): builds the host SAH BLAS of a triangle soup, collapses it into
// compressed 8-wide nodes and checks, in double precision, that
//  - the leaf order is a permutation of the binary tree's leaves;
//  - every used child slot's decoded box (origin + q * step) contains every triangle under it;
//  - closest-hit traversal of the wide tree (nearest child first) finds the same triangle and
//    distance as a brute-force test of every triangle, for random rays.
#include <cstdio>
#include <cstring>
#include <random>
#include "vkb_wide8.h"

using vkb_host::Wide8Node;

struct Tri { double p[3][3]; };
static double decode(const Wide8Node& n, int axis, int k, bool hi) {
    uint32_t bits;
    std::memcpy(&bits, &n.h.w, 4);
    const int e = int((bits >> (8 * axis)) & 255u) - 127;
    const uint4 q = n.q[axis];
    const uint32_t w = hi ? (k < 4 ? q.z : q.w) : (k < 4 ? q.x : q.y);
    const double origin = axis == 0 ? n.h.x : (axis == 1 ? n.h.y : n.h.z);
    return origin + double((w >> (8 * (k & 3))) & 255u) * std::ldexp(1.0, e);
}
static bool hit_tri(const Tri& t, const double o[3], const double d[3], double& dist) {
    double e1[3], e2[3], pv[3], tv[3], qv[3];
    for (int a = 0; a < 3; ++a) { e1[a] = t.p[1][a] - t.p[0][a]; e2[a] = t.p[2][a] - t.p[0][a]; }
    pv[0] = d[1] * e2[2] - d[2] * e2[1]; pv[1] = d[2] * e2[0] - d[0] * e2[2]; pv[2] = d[0] * e2[1] - d[1] * e2[0];
    const double det = e1[0] * pv[0] + e1[1] * pv[1] + e1[2] * pv[2];
    if (std::fabs(det) < 1e-300) return false;
    for (int a = 0; a < 3; ++a) tv[a] = o[a] - t.p[0][a];
    const double u = (tv[0] * pv[0] + tv[1] * pv[1] + tv[2] * pv[2]) / det;
    if (u < 0 || u > 1) return false;
    qv[0] = tv[1] * e1[2] - tv[2] * e1[1]; qv[1] = tv[2] * e1[0] - tv[0] * e1[2]; qv[2] = tv[0] * e1[1] - tv[1] * e1[0];
    const double v = (d[0] * qv[0] + d[1] * qv[1] + d[2] * qv[2]) / det;
    if (v < 0 || u + v > 1) return false;
    dist = (e2[0] * qv[0] + e2[1] * qv[1] + e2[2] * qv[2]) / det;
    return dist >= 0;
}

int main(int argc, char** argv) {
    const uint32_t grid = argc > 1 ? uint32_t(std::atoi(argv[1])) : 60;
    const uint32_t soup = argc > 2 ? uint32_t(std::atoi(argv[2])) : 3000;
    const uint32_t rays = argc > 3 ? uint32_t(std::atoi(argv[3])) : 2000;
    std::mt19937 rng(11);
    std::uniform_real_distribution<float> U(0.f, 1.f);
    std::vector<Tri> tris;
    for (uint32_t z = 0; z < grid; ++z)
        for (uint32_t x = 0; x < grid; ++x) {
            const double h00 = U(rng), h10 = U(rng), h01 = U(rng), h11 = U(rng);
            tris.push_back({{{double(x), h00, double(z)}, {double(x), h01, double(z + 1)}, {double(x + 1), h10, double(z)}}});
            tris.push_back({{{double(x + 1), h10, double(z)}, {double(x), h01, double(z + 1)}, {double(x + 1), h11, double(z + 1)}}});
        }
    const double span = grid ? double(grid) : 10.0;
    for (uint32_t i = 0; i < soup; ++i) {
        Tri t;
        for (int a = 0; a < 3; ++a) t.p[0][a] = double(float(U(rng) * span));
        for (int k = 1; k < 3; ++k)
            for (int a = 0; a < 3; ++a) t.p[k][a] = double(float(t.p[0][a] + 0.3 * U(rng)));
        tris.push_back(t);
    }
    for (Tri& t : tris)
        for (auto& p : t.p)
            for (double& c : p) c = double(float(c));
    const uint32_t n = uint32_t(tris.size());
    std::vector<float> lo(3 * size_t(n)), hi(3 * size_t(n)), cen(3 * size_t(n));
    for (uint32_t t = 0; t < n; ++t)
        for (int a = 0; a < 3; ++a) {
            const float v0 = float(tris[t].p[0][a]), v1 = float(tris[t].p[1][a]), v2 = float(tris[t].p[2][a]);
            lo[3 * t + a] = std::min(v0, std::min(v1, v2)); hi[3 * t + a] = std::max(v0, std::max(v1, v2));
            cen[3 * t + a] = 0.5f * (lo[3 * t + a] + hi[3 * t + a]);
        }
    vkb_host::SahBlas sah;
    sah.run(n, lo.data(), hi.data(), cen.data(), 0);
    vkb_host::Wide8Blas w8;
    w8.run(sah.nodes, n);
    // Leaf order: a permutation.
    std::vector<int> seen(n, 0);
    if (w8.order.size() != n) { std::printf("FAIL order size %zu != %u\n", w8.order.size(), n); return 1; }
    for (uint32_t v : w8.order) { if (v >= n || seen[v]++) { std::printf("FAIL order not a permutation\n"); return 1; } }
    auto tri_of = [&](uint32_t leaf_pos) -> const Tri& { return tris[sah.order[w8.order[leaf_pos]]]; };
    // Containment: every triangle under a slot lies inside the slot's decoded box.
    size_t checked = 0;
    size_t max_depth = 0;
    std::vector<std::pair<uint32_t, size_t>> depth_stack{{0u, 1}};
    while (!depth_stack.empty()) {
        auto [ni, depth] = depth_stack.back();
        depth_stack.pop_back();
        max_depth = std::max(max_depth, depth);
        const Wide8Node& nd = w8.nodes[ni];
        uint32_t bits;
        std::memcpy(&bits, &nd.h.w, 4);
        const uint32_t imask = bits >> 24, internal = uint32_t(__builtin_popcount(imask));
        // Every reference stays inside the arrays: children below the node count, leaves
        // below the triangle count, internal slots first.
        if (nd.b.z < 1 || nd.b.z > 8 || imask != (1u << internal) - 1u || nd.b.x + internal > w8.nodes.size() ||
            nd.b.y + (nd.b.z - internal) > n) { std::printf("FAIL references of node %u\n", ni); return 1; }
        for (int k = 0; k < 8; ++k) {
            if (uint32_t(k) >= nd.b.z) continue;
            double blo[3], bhi[3];
            for (int a = 0; a < 3; ++a) { blo[a] = decode(nd, a, k, false); bhi[a] = decode(nd, a, k, true); }
            // Triangles under the slot.
            std::vector<uint32_t> under;
            if (imask >> k & 1u) {
                std::vector<uint32_t> sub{nd.b.x + uint32_t(k)};
                while (!sub.empty()) {
                    const Wide8Node& c = w8.nodes[sub.back()];
                    sub.pop_back();
                    uint32_t cb;
                    std::memcpy(&cb, &c.h.w, 4);
                    const uint32_t cm = cb >> 24, ci = uint32_t(__builtin_popcount(cm));
                    for (int j = 0; j < 8; ++j) {
                        if (uint32_t(j) >= c.b.z) continue;
                        if (cm >> j & 1u) sub.push_back(c.b.x + uint32_t(j));
                        else under.push_back(c.b.y + uint32_t(j) - ci);
                    }
                }
                depth_stack.push_back({nd.b.x + uint32_t(k), depth + 1});
            } else {
                under.push_back(nd.b.y + uint32_t(k) - internal);
            }
            for (uint32_t leaf : under) {
                const Tri& t = tri_of(leaf);
                for (auto& p : t.p)
                    for (int a = 0; a < 3; ++a)
                        if (p[a] < blo[a] || p[a] > bhi[a]) { std::printf("FAIL containment node %u slot %d\n", ni, k); return 1; }
                ++checked;
            }
        }
    }
    // Closest hits: wide traversal (nearest first, pruned by the best distance) vs brute force.
    std::uniform_real_distribution<double> R(-0.2, 1.2);
    uint32_t mismatches = 0, hits = 0;
    for (uint32_t r = 0; r < rays; ++r) {
        double o[3] = {R(rng) * span, 2.0 + 3.0 * R(rng), R(rng) * span}, tgt[3] = {R(rng) * span, 0.5 * R(rng), R(rng) * span}, d[3];
        double len = 0;
        for (int a = 0; a < 3; ++a) { d[a] = tgt[a] - o[a]; len += d[a] * d[a]; }
        len = std::sqrt(len);
        for (double& c : d) c /= len;
        double best = 1e300; int64_t best_tri = -1;
        for (uint32_t t = 0; t < n; ++t) { double dist; if (hit_tri(tris[t], o, d, dist) && dist < best) { best = dist; best_tri = t; } }
        double wbest = 1e300; int64_t wtri = -1;
        std::vector<uint32_t> st{0u};
        while (!st.empty()) {
            const Wide8Node& nd = w8.nodes[st.back()];
            st.pop_back();
            uint32_t bits;
            std::memcpy(&bits, &nd.h.w, 4);
            const uint32_t imask = bits >> 24, internal = uint32_t(__builtin_popcount(imask));
            for (int k = 0; k < int(nd.b.z); ++k) {
                double t0 = 0, t1 = wbest;
                for (int a = 0; a < 3; ++a) {
                    const double l = decode(nd, a, k, false), h = decode(nd, a, k, true);
                    if (d[a] == 0) { if (o[a] < l || o[a] > h) { t0 = 1; t1 = 0; } continue; }
                    // Near and far planes by the direction's sign, as the device reads them:
                    // an unused slot (lo > hi) is missed whatever the direction.
                    const double tn = ((d[a] > 0 ? l : h) - o[a]) / d[a], tf = ((d[a] > 0 ? h : l) - o[a]) / d[a];
                    t0 = std::max(t0, tn); t1 = std::min(t1, tf);
                }
                if (t0 > t1) continue;
                if (imask >> k & 1u) st.push_back(nd.b.x + uint32_t(k));
                else {
                    const uint32_t leaf = nd.b.y + uint32_t(k) - internal;
                    const uint32_t t = sah.order[w8.order[leaf]];
                    double dist;
                    if (hit_tri(tris[t], o, d, dist) && dist < wbest) { wbest = dist; wtri = t; }
                }
            }
        }
        if (best_tri >= 0) ++hits;
        if (wtri != best_tri && !(wtri >= 0 && best_tri >= 0 && std::fabs(wbest - best) <= 1e-9 * best)) ++mismatches;
    }
    std::printf("%s triangles=%u nodes=%zu depth=%zu slots_checked=%zu rays=%u hits=%u mismatches=%u\n", mismatches ? "FAIL" : "OK", n,
                w8.nodes.size(), max_depth, checked, rays, hits, mismatches);
    return mismatches ? 1 : 0;
}
