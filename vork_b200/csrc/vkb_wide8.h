// Host collapse of a BLAS's binary SAH tree into compressed 8-wide nodes (the layout of
// vkb::Bvh8Node), after Ylitie, Karras & Laine, "Efficient Incoherent Ray Traversal on
// GPUs Through Compressed Wide BVHs" (HPG 2017): each node keeps up to eight child boxes
// as bytes on a grid of its own (an origin and a power-of-two step per axis), rounded
// outward by one more step, its internal children stored together from child_base and
// its leaf triangles together from leaf_base.  Host-only: compiled into the library
// and, for its CPU tests, by a plain C++ compiler.
#pragma once
#include <algorithm>
#include <cmath>
#include <cstdint>
#include <cstring>
#include <vector>
#include "vkb_sah.h"

namespace vkb_host {

// h = (origin.x, origin.y, origin.z, bits: ex | ey << 8 | ez << 16 | internal-slot mask << 24),
//     e the biased exponent of the axis step 2^(e - 127);
// b = (child_base, leaf_base, used slots, 0): the internal children take the first slots
//     and are stored in slot order from child_base; the leaf children (one triangle each)
//     take the next slots, their triangles in slot order from leaf_base;
// q[a] = (lo bytes of slots 0-3, lo 4-7, hi 0-3, hi 4-7) of axis a; an unused slot
//     (after the used ones) has lo 255 > hi 0, and the traversal skips it by the count.
struct alignas(16) Wide8Node { float4 h; uint4 b; uint4 q[3]; };
static_assert(sizeof(Wide8Node) == 80, "80-byte compressed 8-wide node");

struct Wide8Blas {
    std::vector<Wide8Node> nodes;
    std::vector<uint32_t> order;   // leaf position in the wide tree -> leaf position in the binary tree

    struct Child { int ref; float lo[3], hi[3]; };
    static Child child_of(const SahNode& n, int side) {
        Child c;
        if (side == 0) { c.ref = n.d.x; c.lo[0] = n.a.x; c.hi[0] = n.a.y; c.lo[1] = n.a.z; c.hi[1] = n.a.w; c.lo[2] = n.c.x; c.hi[2] = n.c.y; }
        else { c.ref = n.d.y; c.lo[0] = n.b.x; c.hi[0] = n.b.y; c.lo[1] = n.b.z; c.hi[1] = n.b.w; c.lo[2] = n.c.z; c.hi[2] = n.c.w; }
        return c;
    }
    static bool empty_box(const Child& c) { return !(c.lo[0] <= c.hi[0]) || !(c.lo[1] <= c.hi[1]) || !(c.lo[2] <= c.hi[2]); }
    static double area(const Child& c) {
        const double x = double(c.hi[0]) - c.lo[0], y = double(c.hi[1]) - c.lo[1], z = double(c.hi[2]) - c.lo[2];
        return x * y + y * z + z * x;
    }
    // Smallest power-of-two step s >= extent / 250 and >= one float ulp of the axis's
    // coordinates, so that origin = lo - s is exact to a few ulps and every byte fits.
    static int axis_exponent(float lo, float hi) {
        const double extent = double(hi) - double(lo);
        const double mag = std::max(std::fabs(double(lo)), std::fabs(double(hi)));
        int e = -126;
        if (extent > 0.0) e = std::max(e, int(std::ceil(std::log2(extent / 250.0))));
        if (mag > 0.0) e = std::max(e, std::ilogb(mag) - 23);
        while (std::ldexp(250.0, e) < extent) ++e;
        return std::min(e, 127);
    }
    static float round_down(double v) {
        float f = float(v);
        while (double(f) > v) f = std::nextafter(f, -INFINITY);
        return f;
    }

    // Collapse `bin` (root 0, one-triangle leaves over `leaves` leaf positions); the
    // triangles move to the order they are met here, so a node's leaves are consecutive.
    void run(const std::vector<SahNode>& bin, uint32_t leaves) {
        static_assert(BLAS_LEAF_MAX == 1, "the 8-wide collapse takes one-triangle leaves");
        nodes.assign(1, Wide8Node{});
        order.clear();
        order.reserve(leaves);
        std::vector<std::pair<int, uint32_t>> todo{{0, 0u}};   // (binary node, wide node)
        while (!todo.empty()) {
            const auto [b, w] = todo.back();
            todo.pop_back();
            Child slot[8];
            int count = 0;
            for (int side = 0; side < 2; ++side) {
                Child c = child_of(bin[b], side);
                if (!empty_box(c)) slot[count++] = c;
            }
            // Open the internal child of largest surface area until eight slots are taken.
            while (count < 8) {
                int best = -1;
                double best_area = -1.0;
                for (int k = 0; k < count; ++k)
                    if (slot[k].ref >= 0 && area(slot[k]) > best_area) { best_area = area(slot[k]); best = k; }
                if (best < 0) break;
                const SahNode& n = bin[slot[best].ref];
                Child l = child_of(n, 0), r = child_of(n, 1);
                if (empty_box(r)) { slot[best] = l; continue; }
                if (empty_box(l)) { slot[best] = r; continue; }
                slot[best] = l;
                slot[count++] = r;
            }
            // Internal children first in slot order, then leaves: both keep their slot order.
            std::stable_partition(slot, slot + count, [](const Child& c) { return c.ref >= 0; });
            float lo[3] = {INFINITY, INFINITY, INFINITY}, hi[3] = {-INFINITY, -INFINITY, -INFINITY};
            for (int k = 0; k < count; ++k)
                for (int a = 0; a < 3; ++a) { lo[a] = std::min(lo[a], slot[k].lo[a]); hi[a] = std::max(hi[a], slot[k].hi[a]); }
            Wide8Node node;
            std::memset(&node, 0, sizeof(node));
            uint32_t qb[6][8];
            uint32_t bits = 0, imask = 0;
            float origin[3];
            for (int a = 0; a < 3; ++a) {
                const int e = count ? axis_exponent(lo[a], hi[a]) : 0;
                const double s = std::ldexp(1.0, e);
                origin[a] = count ? round_down(double(lo[a]) - s) : 0.f;
                bits |= uint32_t(e + 127) << (8 * a);
                for (int k = 0; k < 8; ++k) {
                    if (k >= count) { qb[a][k] = 255u; qb[3 + a][k] = 0u; continue; }
                    const double ql = std::floor((double(slot[k].lo[a]) - origin[a]) / s) - 1.0;
                    const double qh = std::ceil((double(slot[k].hi[a]) - origin[a]) / s) + 1.0;
                    qb[a][k] = uint32_t(std::clamp(ql, 0.0, 255.0));
                    qb[3 + a][k] = uint32_t(std::clamp(qh, 0.0, 255.0));
                }
            }
            const uint32_t child_base = uint32_t(nodes.size()), leaf_base = uint32_t(order.size());
            int internal = 0;
            for (int k = 0; k < count; ++k) {
                if (slot[k].ref >= 0) {
                    imask |= 1u << k;
                    todo.push_back({slot[k].ref, child_base + uint32_t(internal)});
                    ++internal;
                } else {
                    order.push_back(uint32_t(~slot[k].ref) >> 2);   // one-triangle leaves (BLAS_LEAF_MAX 1)
                }
            }
            nodes.resize(nodes.size() + size_t(internal));
            bits |= imask << 24;
            float hb;
            std::memcpy(&hb, &bits, 4);
            node.h = make_float4(origin[0], origin[1], origin[2], hb);
            node.b = make_uint4(child_base, leaf_base, uint32_t(count), 0u);
            auto pack = [&](int row, int half) {
                return qb[row][4 * half] | (qb[row][4 * half + 1] << 8) | (qb[row][4 * half + 2] << 16) | (qb[row][4 * half + 3] << 24);
            };
            for (int a = 0; a < 3; ++a) node.q[a] = make_uint4(pack(a, 0), pack(a, 1), pack(3 + a, 0), pack(3 + a, 1));
            nodes[w] = node;
        }
    }
};

}  // namespace vkb_host
