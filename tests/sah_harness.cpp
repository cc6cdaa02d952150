// Test harness (tests only): builds the host SAH BLAS of a triangle soup on one thread and
// on every hardware thread and reports whether the trees (nodes, leaf order) are identical.
#include <chrono>
#include <cstdio>
#include <cstring>
#include <random>
#include "vkb_sah.h"

int main(int argc, char** argv) {
    const uint32_t grid = argc > 1 ? uint32_t(std::atoi(argv[1])) : 300;   // terrain-like grid cells per side
    const uint32_t soup = argc > 2 ? uint32_t(std::atoi(argv[2])) : 50000;  // random triangles on top
    std::vector<float> lo, hi, c;
    auto add = [&](const float* p0, const float* p1, const float* p2) {
        for (int a = 0; a < 3; ++a) {
            float l = std::min(p0[a], std::min(p1[a], p2[a])), h = std::max(p0[a], std::max(p1[a], p2[a]));
            lo.push_back(l); hi.push_back(h); c.push_back(0.5f * (l + h));
        }
    };
    std::mt19937 rng(7);
    std::uniform_real_distribution<float> U(0.f, 1.f);
    for (uint32_t z = 0; z < grid; ++z)
        for (uint32_t x = 0; x < grid; ++x) {
            float h00 = U(rng), h10 = U(rng), h01 = U(rng), h11 = U(rng);
            float a[3] = {float(x), h00, float(z)}, b[3] = {float(x + 1), h10, float(z)}, d[3] = {float(x), h01, float(z + 1)}, e[3] = {float(x + 1), h11, float(z + 1)};
            add(a, d, b); add(b, d, e);
        }
    for (uint32_t i = 0; i < soup; ++i) {
        float p[3][3];
        for (int k = 0; k < 3; ++k) for (int a = 0; a < 3; ++a) p[k][a] = U(rng) * float(grid) + (k ? 0.3f * U(rng) : 0.f);
        add(p[0], p[1], p[2]);
    }
    const uint32_t n = uint32_t(lo.size() / 3);
    vkb_host::SahBlas one, many;
    auto t0 = std::chrono::steady_clock::now();
    one.run(n, lo.data(), hi.data(), c.data(), 1);
    auto t1 = std::chrono::steady_clock::now();
    many.run(n, lo.data(), hi.data(), c.data(), 0);
    auto t2 = std::chrono::steady_clock::now();
    const bool same = one.nodes.size() == many.nodes.size() && one.order == many.order &&
                      std::memcmp(one.nodes.data(), many.nodes.data(), one.nodes.size() * sizeof(vkb_host::SahNode)) == 0;
    std::printf("%s triangles=%u nodes=%zu one_ms=%.1f threads_ms=%.1f\n", same ? "SAME" : "DIFF", n, one.nodes.size(),
                std::chrono::duration<double, std::milli>(t1 - t0).count(), std::chrono::duration<double, std::milli>(t2 - t1).count());
    return same ? 0 : 1;
}
