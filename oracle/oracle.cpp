// ORACLE -- test infrastructure only, never part of the product path.
//
// CPU restatement of vork's `std/path` unidirectional path integrator
// (crates/vork-render/shaders/path.slang and the shaders it imports), used by the
// tests as the checker of the CUDA backend and by bench.py as the timed CPU
// baseline.  Only tests/, __graft_entry__.smoke() and bench.py's cpu_baseline leg
// load this library.  Templated on the real type: `double` is the FP64 oracle,
// `float` the FP32 restatement timed as the CPU baseline.
//
// Parity pins (reference tests this file is checked against by tests/):
//   * sampler bits: Sobol direction numbers and first points of
//     crates/vork-render/src/path_sampler.rs:81-93, net property :99-133, and the
//     table construction of path_sampler.rs:12-79 against the shader recurrence of
//     shaders/path_sampler.slang:74-95;
//   * BRDF atlas texels of crates/vork-render/src/environment/brdf_tests.rs:97-104;
//   * film table of crates/vork-render/src/sampling.rs:149-178 and its test :291;
//   * emitter pdf invariants of crates/vork-render/src/light_connection_tests.rs:8-84.
// The transport itself has no reference output available here (the reference is
// Rust + Slang + Vulkan ray queries; none can run in this image), so radiance
// parity against vork's own renders is unpinned; the restatement follows the
// reference line by line and is cited function by function below.
#include <algorithm>
#include <atomic>
#include <cmath>
#include <cstdint>
#include <cstring>
#include <limits>
#include <mutex>
#include <thread>
#include <vector>

#include "../include/vkb.h"

namespace {

// ---------------------------------------------------------------- constants
// crates/vork-slang/src/registry.rs:89,351,375-391; renderer_registry.rs:98-111,367.
constexpr uint32_t SAMPLE_HASH_MIX = 0x45d9f3bu;
constexpr uint32_t PIXEL_HASH_STREAM_STEP = 0x9e3779b9u;
constexpr uint32_t FILTER_INTERVALS = 1024;
constexpr uint32_t BRDF_SIZE = 128, BRDF_ALBEDO_SIZE = 64, BRDF_IOR_STEPS = 64;
constexpr uint32_t BRDF_HEIGHT = BRDF_SIZE + ((BRDF_IOR_STEPS + 2) / 2) * BRDF_ALBEDO_SIZE;  // 2240
constexpr uint32_t ENVIRONMENT_SAMPLES = 512, DIELECTRIC_ALBEDO_SAMPLES = 512;
constexpr double PI = 3.141592653589793, TAU = 2. * PI;
constexpr float MIN_ALPHA = 0.0001f;
constexpr float UINT_SCALE = 0.000000059604644775390625f;
constexpr float RADICAL_INVERSE_SCALE = 2.3283064365386963e-10f;
constexpr float POSITIVE_EPSILON = 1e-20f;
constexpr float FP32_MAX = 3.402823466e38f;
constexpr float FP32_EPS = 1.1920928955078125e-07f;
const float FP32_GAMMA7 = (7.f * (FP32_EPS * 0.5f)) / (1.f - 7.f * (FP32_EPS * 0.5f));
constexpr uint32_t ROULETTE_START = 3;
constexpr float ROULETTE_MIN = 0.05f, ROULETTE_MAX = 0.95f;
constexpr float LIGHT_TREE_UNIFORM_MIX = 0.25f;
constexpr float LIGHT_TREE_MIN_DISTANCE_SQUARED = 1e-12f;
constexpr double LUM[3] = {0.2126, 0.7152, 0.0722};

// ---------------------------------------------------------------- hashes + sampler (u32, bit-exact)
// vork_sampling.slang:3-15 (crates/vork-slang/src/vork_sampling.slang).
inline uint32_t pixel_hash(uint32_t s) {
    uint32_t v = (s ^ (s >> 16)) * SAMPLE_HASH_MIX;
    v = (v ^ (v >> 16)) * SAMPLE_HASH_MIX;
    return v ^ (v >> 16);
}
inline uint32_t screen_ray_hash(uint32_t px, uint32_t py, uint32_t index, uint32_t stream) {
    uint32_t spatial = pixel_hash((px * SAMPLE_HASH_MIX) ^ py);
    return pixel_hash(spatial ^ pixel_hash(index * PIXEL_HASH_STREAM_STEP + stream));
}
inline uint32_t rev(uint32_t x) {
    x = ((x >> 1) & 0x55555555u) | ((x & 0x55555555u) << 1);
    x = ((x >> 2) & 0x33333333u) | ((x & 0x33333333u) << 2);
    x = ((x >> 4) & 0x0f0f0f0fu) | ((x & 0x0f0f0f0fu) << 4);
    x = ((x >> 8) & 0x00ff00ffu) | ((x & 0x00ff00ffu) << 8);
    return (x >> 16) | (x << 16);
}
// path_sampler.slang:65-68 / path_sampler.rs:42-50.
inline uint32_t owen_reversed(uint32_t x, uint32_t seed) {
    seed = pixel_hash(seed);
    x ^= x * 0x3d20adeau;
    x += seed;
    x *= (seed >> 16) | 1u;
    x ^= x * 0x05526c56u;
    x ^= x * 0x53a22864u;
    return x;
}
inline float sample_unit(uint32_t x) { return (float(x >> 9) + 0.5f) * (1.f / 8388608.f); }

struct Sampler { uint32_t index, seed, mask, vertex; };
// path_sampler.slang:52-59; path_sampler.rs:55-58.
inline uint32_t sample_block(uint32_t count) {
    if (count <= 1) return 1u;
    uint32_t x = count - 1u;
    int hb = 31 - __builtin_clz(x);
    return 2u << hb;
}
inline Sampler make_sampler(uint32_t px, uint32_t py, uint32_t index, uint32_t count, uint32_t stream) {
    Sampler s;
    s.index = index;
    s.seed = screen_ray_hash(px, py, 0u, stream);
    s.vertex = 0;
    s.mask = sample_block(count) - 1u;
    return s;
}

// Sobol generator matrices built from Joe-Kuo's published primitive polynomials
// (path_sampler.rs:12-35), independently of the shader recurrence below.
struct SobolTable {
    uint32_t d[3][32];
    SobolTable() {
        const int s_[3] = {1, 2, 3};
        const uint32_t a_[3] = {0, 1, 1};
        const uint32_t m_[3][3] = {{1, 0, 0}, {1, 3, 0}, {1, 3, 1}};
        for (int k = 0; k < 3; ++k) {
            int s = s_[k];
            for (int i = 0; i < 32; ++i) {
                if (i < s) { d[k][i] = m_[k][i] << (31 - i); continue; }
                uint32_t v = d[k][i - s] ^ (d[k][i - s] >> s);
                for (int j = 1; j < s; ++j)
                    if ((a_[k] >> (s - 1 - j)) & 1u) v ^= d[k][i - j];
                d[k][i] = v;
            }
        }
    }
};
const SobolTable& sobol_table() { static SobolTable t; return t; }

// Group bits by the table form (path_sampler.rs:60-67).
inline void group_bits_table(const Sampler& s, uint32_t group, uint32_t out[4]) {
    uint32_t seed = pixel_hash(s.seed ^ pixel_hash(group + 1u));
    uint32_t index = rev(owen_reversed(rev(s.index), seed ^ 0x6c8e9cf5u)) & s.mask;
    uint32_t x[4] = {index, 0, 0, 0};
    const SobolTable& t = sobol_table();
    for (int k = 0; k < 32; ++k)
        if ((index >> k) & 1u)
            for (int d = 0; d < 3; ++d) x[d + 1] ^= t.d[d][k];
    for (int d = 1; d < 4; ++d) x[d] = rev(x[d]);
    const uint32_t seeds[4] = {0xa511e9b3u, 0x63d83595u, 0x2f7c4a1bu, 0x9e3779b9u};
    for (int c = 0; c < 4; ++c) out[c] = rev(owen_reversed(x[c], seed ^ seeds[c]));
}
// Group bits by the shader's generator recurrences (path_sampler.slang:74-95).
inline void group_bits_recurrence(const Sampler& s, uint32_t group, uint32_t out[4]) {
    uint32_t seed = pixel_hash(s.seed ^ pixel_hash(group + 1u));
    uint32_t index = rev(owen_reversed(rev(s.index), seed ^ 0x6c8e9cf5u)) & s.mask;
    uint32_t x0 = 0, x1 = 0, x2 = 0, p = 0x80000000u;
    uint32_t qx = 0x80000000u, qy = 0xc0000000u;
    uint32_t rx = 0x80000000u, ry = 0xc0000000u, rz = 0x20000000u;
    for (uint32_t bits = index; bits != 0u; bits >>= 1) {
        if (bits & 1u) { x0 ^= p; x1 ^= qx; x2 ^= rx; }
        p ^= p >> 1;
        uint32_t nqx = qy, nqy = qy ^ qx ^ (qx >> 2);
        qx = nqx; qy = nqy;
        uint32_t nrx = ry, nry = rz, nrz = ry ^ rx ^ (rx >> 3);
        rx = nrx; ry = nry; rz = nrz;
    }
    uint32_t sc[4] = {owen_reversed(index, seed ^ 0xa511e9b3u), owen_reversed(rev(x0), seed ^ 0x63d83595u),
                      owen_reversed(rev(x1), seed ^ 0x2f7c4a1bu), owen_reversed(rev(x2), seed ^ PIXEL_HASH_STREAM_STEP)};
    for (int c = 0; c < 4; ++c) out[c] = rev(sc[c]);
}
inline void sample_group(const Sampler& s, uint32_t group, float out[4]) {
    uint32_t b[4];
    group_bits_recurrence(s, group, b);
    for (int c = 0; c < 4; ++c) out[c] = sample_unit(b[c]);
}
// path_sampler.slang:96-112: group 0 camera; vertex v owns groups 1+5v .. 5+5v.
inline void vertex_group(const Sampler& s, uint32_t slot, float out[4]) { sample_group(s, 1u + s.vertex * 5u + slot, out); }
// path_sampler.slang:73.
inline float path_random(uint32_t& state) { state = pixel_hash(state + PIXEL_HASH_STREAM_STEP); return sample_unit(state); }

// ---------------------------------------------------------------- film table (sampling.rs:149-178)
double path_filter_cdf(double x) {
    double t = PI * x / 1.5;
    return 0.5 + (0.35875 * x + 1.5 / PI * (0.48829 * std::sin(t) + 0.14128 * std::sin(2. * t) / 2. + 0.01168 * std::sin(3. * t) / 3.)) / (3. * 0.35875);
}
const std::vector<float>& filter_table() {
    static std::vector<float> table = [] {
        std::vector<float> t(FILTER_INTERVALS + 1);
        for (uint32_t i = 0; i <= FILTER_INTERVALS; ++i) {
            if (i == 0) { t[i] = -1.5f; continue; }
            if (i == FILTER_INTERVALS) { t[i] = 1.5f; continue; }
            double u = double(i) / double(FILTER_INTERVALS), lo = -1.5, hi = 1.5;
            for (int k = 0; k < 48; ++k) {
                double mid = (lo + hi) * 0.5;
                if (path_filter_cdf(mid) < u) lo = mid; else hi = mid;
            }
            t[i] = float((lo + hi) * 0.5);
        }
        return t;
    }();
    return table;
}

// ---------------------------------------------------------------- fp16 storage of the BRDF atlas
uint16_t float_to_half(float f) {
    uint32_t x; std::memcpy(&x, &f, 4);
    uint32_t sign = (x >> 16) & 0x8000u;
    uint32_t mant = x & 0x7fffffu;
    int exp = int((x >> 23) & 0xffu);
    if (exp == 255) return uint16_t(sign | 0x7c00u | (mant ? 0x200u : 0u));
    int e = exp - 127 + 15;
    if (e >= 31) return uint16_t(sign | 0x7c00u);
    if (e <= 0) {
        if (e < -10) return uint16_t(sign);
        mant |= 0x800000u;
        int shift = 14 - e;
        uint32_t h = mant >> shift, rem = mant & ((1u << shift) - 1u), half = 1u << (shift - 1);
        if (rem > half || (rem == half && (h & 1u))) h++;
        return uint16_t(sign | h);
    }
    uint32_t h = (uint32_t(e) << 10) | (mant >> 13);
    uint32_t rem = mant & 0x1fffu;
    if (rem > 0x1000u || (rem == 0x1000u && (h & 1u))) h++;
    return uint16_t(sign | h);
}
float half_to_float(uint16_t h) {
    uint32_t sign = uint32_t(h & 0x8000u) << 16, exp = (h >> 10) & 0x1fu, mant = h & 0x3ffu, x;
    if (exp == 0) {
        if (mant == 0) x = sign;
        else { int e = -1; do { e++; mant <<= 1; } while (!(mant & 0x400u)); x = sign | (uint32_t(127 - 15 - e) << 23) | ((mant & 0x3ffu) << 13); }
    } else if (exp == 31) x = sign | 0x7f800000u | (mant << 13);
    else x = sign | ((exp + 112u) << 23) | (mant << 13);
    float f; std::memcpy(&f, &x, 4); return f;
}

// ---------------------------------------------------------------- vector math
template <class R> struct V3 {
    R x, y, z;
    V3() : x(0), y(0), z(0) {}
    V3(R a, R b, R c) : x(a), y(b), z(c) {}
    R& operator[](int i) { return i == 0 ? x : (i == 1 ? y : z); }
    R operator[](int i) const { return i == 0 ? x : (i == 1 ? y : z); }
};
template <class R> inline V3<R> operator+(V3<R> a, V3<R> b) { return {a.x + b.x, a.y + b.y, a.z + b.z}; }
template <class R> inline V3<R> operator-(V3<R> a, V3<R> b) { return {a.x - b.x, a.y - b.y, a.z - b.z}; }
template <class R> inline V3<R> operator-(V3<R> a) { return {-a.x, -a.y, -a.z}; }
template <class R> inline V3<R> operator*(V3<R> a, V3<R> b) { return {a.x * b.x, a.y * b.y, a.z * b.z}; }
template <class R> inline V3<R> operator*(V3<R> a, R s) { return {a.x * s, a.y * s, a.z * s}; }
template <class R> inline V3<R> operator*(R s, V3<R> a) { return {a.x * s, a.y * s, a.z * s}; }
template <class R> inline V3<R> operator/(V3<R> a, R s) { return {a.x / s, a.y / s, a.z / s}; }
template <class R> inline V3<R> operator/(V3<R> a, V3<R> b) { return {a.x / b.x, a.y / b.y, a.z / b.z}; }
template <class R> inline R dot(V3<R> a, V3<R> b) { return a.x * b.x + a.y * b.y + a.z * b.z; }
template <class R> inline V3<R> cross(V3<R> a, V3<R> b) { return {a.y * b.z - a.z * b.y, a.z * b.x - a.x * b.z, a.x * b.y - a.y * b.x}; }
template <class R> inline R length(V3<R> a) { return std::sqrt(dot(a, a)); }
template <class R> inline V3<R> normalize(V3<R> a) { return a / length(a); }
template <class R> inline V3<R> vabs(V3<R> a) { return {std::fabs(a.x), std::fabs(a.y), std::fabs(a.z)}; }
template <class R> inline V3<R> vmax(V3<R> a, V3<R> b) { return {std::max(a.x, b.x), std::max(a.y, b.y), std::max(a.z, b.z)}; }
template <class R> inline V3<R> vmin(V3<R> a, V3<R> b) { return {std::min(a.x, b.x), std::min(a.y, b.y), std::min(a.z, b.z)}; }
template <class R> inline R maxc(V3<R> a) { return std::max(a.x, std::max(a.y, a.z)); }
template <class R> inline bool finite3(V3<R> a) { return std::isfinite(a.x) && std::isfinite(a.y) && std::isfinite(a.z); }
template <class R> inline bool any_pos(V3<R> a) { return a.x > 0 || a.y > 0 || a.z > 0; }
template <class R> inline bool any_nonzero(V3<R> a) { return a.x != 0 || a.y != 0 || a.z != 0; }
template <class R> inline R lerp(R a, R b, R t) { return a + (b - a) * t; }
template <class R> inline V3<R> lerp3(V3<R> a, V3<R> b, R t) { return a + (b - a) * t; }
template <class R> inline R clampr(R x, R a, R b) { return std::min(std::max(x, a), b); }
template <class R> inline R lum(V3<R> c) { return c.x * R(LUM[0]) + c.y * R(LUM[1]) + c.z * R(LUM[2]); }
// reflect(i, n) = i - 2 dot(n, i) n (HLSL).
template <class R> inline V3<R> reflect(V3<R> i, V3<R> n) { return i - n * (R(2) * dot(n, i)); }
// stream.slang:416-427.
template <class R> inline V3<R> finite_unit_normal(V3<R> n, V3<R> fallback) {
    R s = maxc(vabs(n));
    if (finite3(n) && s > 0) return normalize(n / s);
    R fs = maxc(vabs(fallback));
    if (finite3(fallback) && fs > 0) return normalize(fallback / fs);
    return V3<R>(0, 0, 1);
}
// orthonormal_basis.slang (Duff et al. 2017).
template <class R> inline V3<R> basis_direction(V3<R> n, V3<R> v) {
    R s = n.z >= 0 ? R(1) : R(-1);
    R a = R(-1) / (s + n.z);
    R b = n.x * n.y * a;
    V3<R> r0(R(1) + s * n.x * n.x * a, s * b, -s * n.x);
    V3<R> r1(b, s + n.y * n.y * a, -n.y);
    return r0 * v.x + r1 * v.y + n * v.z;
}
template <class R> inline R next_float(R v, bool up) { return std::nextafter(v, up ? std::numeric_limits<R>::infinity() : -std::numeric_limits<R>::infinity()); }

// ---------------------------------------------------------------- OpenPBR core (libraries/std/openpbr_core.slang)
template <class R> inline R specular_alpha(R r) { return std::max(r * r, R(MIN_ALPHA)); }           // :5-7
template <class R> inline R modulated_ior(R eta, R weight) {                                         // :14-22
    if (weight == 1 || eta == 1) return eta;
    R contrast = (eta - 1) / (eta + 1);
    R limit = R(0.99999994039535522461);  // asfloat(0x3f7fffff)
    R e = clampr(std::sqrt(std::max(weight, R(0))) * contrast, -limit, limit);
    return (1 + e) / (1 - e);
}
template <class R> inline R fresnel(R c, R eta) {                                                    // :23-28
    c = clampr(c, R(0), R(1));
    if (eta == 1) return 0;
    R si2 = (1 - c * c) / (eta * eta);
    if (si2 >= 1) return 1;
    R ct = std::sqrt(std::max(R(0), 1 - si2));
    R rs = (c - eta * ct) / (c + eta * ct), rp = (eta * c - ct) / (eta * c + ct);
    return (rs * rs + rp * rp) * R(0.5);
}
template <class R> inline V3<R> metal_edge_correction(V3<R> f0, V3<R> tint) {                        // :31-35
    if (tint.x == 1 && tint.y == 1 && tint.z == 1) return V3<R>();
    R mu = R(1) / R(7);
    V3<R> edge = f0 + (V3<R>(1, 1, 1) - f0) * R(std::pow(1 - mu, R(5)));
    return edge * (V3<R>(1, 1, 1) - tint) / (mu * R(std::pow(1 - mu, R(6))));
}
template <class R> inline V3<R> reflection_fresnel_at_ior(V3<R> bc, R bw, R metal, R sw, V3<R> sc, R cosine, R eta) {  // :36-45
    cosine = clampr(cosine, R(0), R(1));
    V3<R> diel = sc * fresnel(cosine, eta);
    if (metal <= 0) return diel;
    V3<R> f0 = bc * bw;
    R f = R(std::pow(1 - cosine, R(5)));
    V3<R> m = f0 + (V3<R>(1, 1, 1) - f0) * f - metal_edge_correction(f0, sc) * (cosine * R(std::pow(1 - cosine, R(6))));
    m = vmax(m, V3<R>());
    return lerp3(diel, m * sw, metal);
}
template <class R> inline R distribution(R nh, R a) { R x = (1 - nh * nh) + nh * nh * a * a; return a * a / (R(PI) * x * x); }  // :113-117
template <class R> inline R smith_denominator(R no, R ni, R a) {                                      // :120-124
    R ci = std::fabs(ni), a2 = a * a;
    R po = std::sqrt(a2 + (1 - a2) * no * no), pi = std::sqrt(a2 + (1 - a2) * ci * ci);
    return ci * po + no * pi;
}
template <class R> inline R g2(R no, R ni, R a) { return 2 * no * std::fabs(ni) / smith_denominator(no, ni, a); }  // :128-130
template <class R> inline V3<R> ggx_visible_normal(V3<R> view, R alpha, R ux, R uy) {                 // :135-144
    V3<R> v = normalize(V3<R>(alpha * view.x, alpha * view.y, view.z));
    R ls = v.x * v.x + v.y * v.y;
    V3<R> t = ls > 0 ? V3<R>(-v.y, v.x, 0) / std::sqrt(ls) : V3<R>(1, 0, 0);
    V3<R> b = cross(v, t);
    R radius = std::sqrt(ux), phi = R(2 * PI) * uy;
    R x = radius * std::cos(phi);
    R y = lerp(std::sqrt(std::max(1 - x * x, R(0))), radius * std::sin(phi), R(0.5) * (1 + v.z));
    V3<R> p = t * x + b * y + v * std::sqrt(std::max(1 - x * x - y * y, R(0)));
    return normalize(V3<R>(alpha * p.x, alpha * p.y, std::max(p.z, R(0))));
}
template <class R> inline R ggx_visible_weight(R no, R ni, R a) {                                   // :147-151
    if (ni <= 0) return 0;
    R a2 = a * a;
    return ni * (no + std::sqrt(a2 + (1 - a2) * no * no)) / smith_denominator(no, ni, a);
}
template <class R> inline R ggx_visible_reflection(R no, R a, R ux, R uy, R& vh) {                  // :153-158
    V3<R> view(std::sqrt(std::max(1 - no * no, R(0))), 0, no);
    V3<R> h = ggx_visible_normal(view, a, ux, uy);
    V3<R> light = reflect(-view, h);
    vh = clampr(dot(view, h), R(0), R(1));
    return ggx_visible_weight(no, light.z, a);
}
template <class R> inline R dielectric_directional_albedo(R no, R r, R eta, uint32_t samples) {     // :160-171
    if (eta == 1) return 0;
    if (r == 0) return eta <= 0 ? R(1) : fresnel(no, eta);
    R a = specular_alpha(r), result = 0;
    for (uint32_t i = 0; i < samples; ++i) {
        R ux = (R(i) + R(0.5)) / R(samples);
        R uy = R(float(rev(i) >> 8u) * UINT_SCALE);
        R vh;
        R w = ggx_visible_reflection(no, a, ux, uy, vh);
        result += (eta <= 0 ? R(1) : fresnel(vh, eta)) * w;
    }
    return result / R(samples);
}
template <class R> inline V3<R> ggx_reflection(V3<R> refl, R no, R ni, R nh, R r) {                // :175-178
    R a = specular_alpha(r);
    return refl * (distribution(nh, a) * g2(no, ni, a) / (4 * no * ni));
}

// ---------------------------------------------------------------- BRDF atlas bake (shaders/environment.slang:14-108)
template <class R> R brdf_cosine(uint32_t col) { R t = R(col) / R(BRDF_SIZE - 1); R t2 = t * t; return t2 * t2; }
template <class R> R brdf_alpha(uint32_t row) {
    if (row == 0) return R(MIN_ALPHA);
    if (row == BRDF_SIZE - 1) return 1;
    return std::exp2(std::log2(R(MIN_ALPHA)) * (1 - R(row) / R(BRDF_SIZE - 1)));
}
template <class R> void bake_texel(uint32_t x, uint32_t y, float out[4]) {
    if (y >= BRDF_SIZE) {
        const uint32_t n = BRDF_ALBEDO_SIZE;
        uint32_t cx = x % n, cy = (y - BRDF_SIZE) % n;
        uint32_t slice = ((y - BRDF_SIZE) / n) * 2u + x / n;
        if (slice > BRDF_IOR_STEPS) { out[0] = out[1] = out[2] = out[3] = 0; return; }
        R no = std::max(R(cx) / R(n - 1), R(MIN_ALPHA));
        R r = R(cy) / R(n - 1);
        R q = R(slice) / R(BRDF_IOR_STEPS);
        R eta = slice == BRDF_IOR_STEPS ? R(0) : q / std::max(1 - q, R(POSITIVE_EPSILON));
        out[0] = float(dielectric_directional_albedo(no, r, eta, DIELECTRIC_ALBEDO_SAMPLES));
        out[1] = out[2] = 0; out[3] = 1;
        return;
    }
    R sum[3] = {0, 0, 0};
    R nv = brdf_cosine<R>(x), alpha = brdf_alpha<R>(y);
    for (uint32_t i = 0; i < ENVIRONMENT_SAMPLES; ++i) {
        R ux = (R(i) + R(0.5)) / R(ENVIRONMENT_SAMPLES), uy = R(float(rev(i)) * RADICAL_INVERSE_SCALE);
        R vh;
        R g = ggx_visible_reflection(nv, alpha, ux, uy, vh);
        R f = R(std::pow(1 - vh, R(5)));
        sum[0] += (1 - f) * g; sum[1] += f * g; sum[2] += vh * R(std::pow(1 - vh, R(6))) * g;
    }
    R average = 0;
    if (x == 0) {
        for (uint32_t j = 0; j < BRDF_SIZE; ++j) {
            R c = brdf_cosine<R>(j);
            R interval = R(0.5) * (brdf_cosine<R>(std::min(j + 1u, BRDF_SIZE - 1u)) - brdf_cosine<R>(j > 0 ? j - 1u : 0u));
            for (uint32_t i = 0; i < ENVIRONMENT_SAMPLES; ++i) {
                R ux = (R(i) + R(0.5)) / R(ENVIRONMENT_SAMPLES), uy = R(float(rev(i)) * RADICAL_INVERSE_SCALE);
                R vh;
                average += interval * 2 * c * ggx_visible_reflection(c, alpha, ux, uy, vh);
            }
        }
        average /= R(ENVIRONMENT_SAMPLES);
    }
    for (int c = 0; c < 3; ++c) out[c] = float(sum[c] / R(ENVIRONMENT_SAMPLES));
    out[3] = float(average);
}
template <class R> struct Lut {
    std::vector<float> texels;  // fp16-rounded values, BRDF_SIZE x BRDF_HEIGHT x 4
    Lut() {
        texels.resize(size_t(BRDF_SIZE) * BRDF_HEIGHT * 4);
        std::atomic<uint32_t> next{0};
        auto work = [&] {
            for (uint32_t y; (y = next.fetch_add(1)) < BRDF_HEIGHT;)
                for (uint32_t x = 0; x < BRDF_SIZE; ++x) {
                    float t[4];
                    bake_texel<R>(x, y, t);
                    for (int c = 0; c < 4; ++c) texels[(size_t(y) * BRDF_SIZE + x) * 4 + c] = half_to_float(float_to_half(t[c]));
                }
        };
        unsigned n = std::max(1u, std::thread::hardware_concurrency());
        std::vector<std::thread> ts;
        for (unsigned i = 0; i < n; ++i) ts.emplace_back(work);
        for (auto& t : ts) t.join();
    }
    // Bilinear, clamp-to-edge, texel-centred (a linear SamplerState).
    R fetch(R fx, R fy, int c) const {
        fx = clampr(fx, R(0), R(BRDF_SIZE - 1));
        fy = clampr(fy, R(0), R(BRDF_HEIGHT - 1));
        int x0 = int(std::floor(fx)), y0 = int(std::floor(fy));
        int x1 = std::min(x0 + 1, int(BRDF_SIZE) - 1), y1 = std::min(y0 + 1, int(BRDF_HEIGHT) - 1);
        R tx = fx - R(x0), ty = fy - R(y0);
        auto at = [&](int x, int y) { return R(texels[(size_t(y) * BRDF_SIZE + x) * 4 + c]); };
        return lerp(lerp(at(x0, y0), at(x1, y0), tx), lerp(at(x0, y1), at(x1, y1), tx), ty);
    }
    // frame.slang:158-168: fourth-power cosine / log-alpha grid, texel centred.
    void moments(R nv, R roughness, R out[3]) const {
        R u = std::sqrt(std::sqrt(clampr(nv, R(0), R(1))));
        R v = std::log2(clampr(roughness * roughness, R(MIN_ALPHA), R(1)) / R(MIN_ALPHA)) / std::log2(R(1) / R(MIN_ALPHA));
        for (int c = 0; c < 3; ++c) out[c] = fetch(u * R(BRDF_SIZE - 1), v * R(BRDF_SIZE - 1), c);
    }
    R average_albedo(R roughness) const {
        R v = std::log2(clampr(roughness * roughness, R(MIN_ALPHA), R(1)) / R(MIN_ALPHA)) / std::log2(R(1) / R(MIN_ALPHA));
        return fetch(0, v * R(BRDF_SIZE - 1), 3);
    }
    // frame.slang:169-181.
    R dielectric_albedo(R nv, R roughness, R eta) const {
        if (eta == 1) return 0;
        R at = eta / (1 + eta) * R(BRDF_IOR_STEPS);
        uint32_t first = std::min(uint32_t(at), BRDF_IOR_STEPS - 1u);
        const R n = BRDF_ALBEDO_SIZE;
        R lx = clampr(nv, R(0), R(1)) * (n - 1), ly = clampr(roughness, R(0), R(1)) * (n - 1);
        uint32_t second = first + 1;
        R ax = R((first % 2u) * BRDF_ALBEDO_SIZE), ay = R(BRDF_SIZE + (first / 2u) * BRDF_ALBEDO_SIZE);
        R bx = R((second % 2u) * BRDF_ALBEDO_SIZE), by = R(BRDF_SIZE + (second / 2u) * BRDF_ALBEDO_SIZE);
        return lerp(fetch(ax + lx, ay + ly, 0), fetch(bx + lx, by + ly, 0), at - R(first));
    }
};
template <class R> Lut<R>& lut_mut() { static Lut<R> l; return l; }
template <class R> const Lut<R>& lut() { return lut_mut<R>(); }
// Baked texels of each precision, kept while a caller's atlas replaces them.
template <class R> std::vector<float>& lut_baked() { static std::vector<float> b; return b; }

// ---------------------------------------------------------------- closure + BSDF (shaders/bsdf*.slang subset)
template <class R> struct Closure {
    V3<R> base_color; R base_weight, base_metalness;
    V3<R> specular_color; R specular_weight, specular_roughness, specular_ior, optical_ior;
    V3<R> n;  // geometry_normal
};
// dielectric_interface.slang:11-17.
template <class R> inline R dielectric_ior(const Closure<R>& c) { return c.optical_ior > 0 ? c.optical_ior : modulated_ior(c.specular_ior, c.specular_weight); }
// path_boundary.slang:41-50 with dielectric_interface.slang:18-35,49-58, air on both sides, not solid.
template <class R> inline void boundary_closure_air(Closure<R>& c) {
    R transmitted = c.specular_weight == 0 ? R(1) : (c.specular_weight == 1 ? c.specular_ior : modulated_ior(c.specular_ior, c.specular_weight));
    c.optical_ior = transmitted;  // optical_transmitted / optical_incident(1)
    // specular_ior = c.specular_ior / 1 (unchanged)
}
template <class R> struct Prepared {
    V3<R> p; V3<R> diffuse; V3<R> metal_comp; V3<R> smooth; R bump_a2; V3<R> interface_n;
};
// bsdf.slang:184-212 (no coat, fuzz, film, transmission, subsurface, thin wall).
template <class R> inline V3<R> transport_probabilities(const Closure<R>& c, V3<R> view) {
    R diffuse = std::max(lum(c.base_color) * c.base_weight * (1 - c.base_metalness) * (1 - R(0)) + R(0), R(0));
    R f = fresnel(std::max(dot(c.n, view), R(0)), dielectric_ior(c));
    R reflected = f;
    R dielectric = reflected * std::max(lum(c.specular_color), R(0));
    R reflection = std::max(lerp(dielectric, c.specular_weight, c.base_metalness), R(0));
    R total = diffuse + reflection;
    if (!(total > 0)) return V3<R>();
    return V3<R>(diffuse, reflection, 0) / std::max(total, R(POSITIVE_EPSILON));
}
// bsdf.slang:220-236.
template <class R> inline V3<R> valid_interface_normal(V3<R> normal, V3<R> geometric, V3<R> view) {
    R iz = dot(view, geometric);
    if (iz <= 0) return normal;
    if (dot(normal, geometric) < 0) normal = -normal;
    R threshold = std::min(R(0.9) * iz, R(0.01));
    if (dot(normal, view) > 0 && dot(reflect(-view, normal), geometric) >= threshold) return normal;
    V3<R> tangent = normal - geometric * dot(normal, geometric);
    R ts = dot(tangent, tangent);
    if (ts <= 0) return geometric;
    V3<R> axis = tangent * (R(1) / std::sqrt(ts));
    R ix = dot(view, axis), ls = ix * ix + iz * iz;
    R cs = clampr(R(0.5) * (1 + (iz * threshold - ix * std::sqrt(std::max(ls - threshold * threshold, R(0)))) / ls), R(0), R(1));
    return axis * std::sqrt(1 - cs) + geometric * std::sqrt(cs);
}
// bsdf_energy.slang:108-122 (white specular tint: closed-form branch).
template <class R> inline V3<R> metal_fresnel_average(const Closure<R>& c) {
    V3<R> f0 = c.base_color * c.base_weight;
    V3<R> b = metal_edge_correction(f0, c.specular_color);
    if (any_pos(b)) {
        V3<R> avg;
        for (uint32_t i = 0; i < BRDF_ALBEDO_SIZE; ++i) {
            R mu = (R(i) + R(0.5)) / R(BRDF_ALBEDO_SIZE);
            avg = avg + reflection_fresnel_at_ior(c.base_color, c.base_weight, R(1), R(1), c.specular_color, mu,
                                                 modulated_ior(c.specular_ior, R(1))) * (2 * mu / R(BRDF_ALBEDO_SIZE));
        }
        return vmin(vmax(avg, V3<R>()), V3<R>(1, 1, 1));
    }
    V3<R> v = f0 + (V3<R>(1, 1, 1) - f0) / R(21) - b / R(126);
    return vmin(vmax(v, V3<R>()), V3<R>(1, 1, 1));
}
// bsdf_response.slang:13-19 + bsdf_energy.slang:123-136.
template <class R> inline V3<R> metal_compensation(const Closure<R>& c, V3<R> view) {
    if (c.base_metalness <= 0 || c.specular_roughness == 0) return V3<R>();
    R m[3];
    lut<R>().moments(std::max(dot(c.n, view), R(0.0001)), c.specular_roughness, m);
    R avg_e = lut<R>().average_albedo(c.specular_roughness);
    R energy = m[0] + m[1];
    R missing = 1 / std::max(energy, R(1e-6)) - 1;
    V3<R> af = metal_fresnel_average(c);
    V3<R> den = vmax(V3<R>(1, 1, 1) - af * (1 - avg_e), V3<R>(1e-6, 1e-6, 1e-6));
    return (af * (missing * avg_e)) / den;
}
// bsdf_response.slang:82-96 (+ openpbr_core.slang:52-56).
template <class R> inline V3<R> direct_diffuse(const Closure<R>& c, V3<R> view) {
    if (!(c.base_weight > 0 && c.base_metalness < 1)) return V3<R>();
    R albedo_s = lut<R>().dielectric_albedo(std::max(dot(c.n, view), R(0.0001)), c.specular_roughness, dielectric_ior(c));
    V3<R> albedo = c.specular_color * albedo_s;
    V3<R> substrate = c.base_color * c.base_weight;
    return substrate * ((1 - c.base_metalness) * (1 - R(0))) * (V3<R>(1, 1, 1) - albedo) / R(PI);
}
// bsdf.slang:242-250.
template <class R> inline Prepared<R> transport_prepare(const Closure<R>& c, V3<R> view, V3<R> smooth, V3<R> geometric) {
    Prepared<R> pr;
    Closure<R> b = c;
    b.n = valid_interface_normal(c.n, geometric, view);
    pr.p = transport_probabilities(b, view);
    R dev = std::fabs(dot(smooth, c.n));
    pr.bump_a2 = clampr((1 - dev * dev) / std::max(8 * dev * dev, R(POSITIVE_EPSILON)), R(0), R(1));
    pr.diffuse = direct_diffuse(b, view);
    pr.metal_comp = metal_compensation(b, view);
    pr.smooth = smooth;
    pr.interface_n = b.n;
    return pr;
}
// bsdf.slang:255-265.
template <class R> inline R bump_shadow(const Closure<R>& c, V3<R> dir, const Prepared<R>& pr) {
    R cosine = dot(pr.smooth, dir);
    if (cosine * dot(pr.smooth, c.n) * dot(c.n, dir) < 0) return 0;
    if (pr.bump_a2 == 0) return 1;
    R mu = std::fabs(cosine);
    return mu > 0 ? 2 * mu / (mu + std::sqrt(pr.bump_a2 + (1 - pr.bump_a2) * mu * mu)) : R(0);
}
// bsdf_microfacet.slang:43-52 (isotropic).
template <class R> inline R visible_scale(R nv, R roughness) { R a = specular_alpha(roughness); return 2 / (nv + std::sqrt(a * a + (1 - a * a) * nv * nv)); }
// bsdf.slang:296-309 (coat probability 0; transmission weight 0).
template <class R> inline R pdf_mask(const Closure<R>& c, V3<R> view, V3<R> dir, uint32_t mask, const Prepared<R>& pr) {
    V3<R> n = pr.interface_n;
    R nl = dot(n, dir);
    R cd = dot(c.n, dir);
    R pdf = (mask & VKB_RAY_DIFFUSE) ? pr.p.x * (cd > 0 ? R(1) : R(0)) * std::fabs(cd) / R(PI) : R(0);
    if (nl <= 0) return pdf;
    V3<R> h = normalize(view + dir);
    R d = distribution(std::max(dot(n, h), R(0)), specular_alpha(c.specular_roughness));
    return pdf + ((mask & VKB_RAY_SPECULAR) ? pr.p.y * (d * visible_scale(dot(n, view), c.specular_roughness) / 4) : R(0));
}
// bsdf_energy.slang:138-149 + bsdf_film.slang:110-123 (no film, not thin).
template <class R> inline V3<R> compensated_reflection(const Closure<R>& c, R cosine, V3<R> comp) {
    V3<R> f = reflection_fresnel_at_ior(c.base_color, c.base_weight, c.base_metalness, c.specular_weight, c.specular_color, cosine, dielectric_ior(c));
    if (any_pos(comp)) {
        if (c.base_metalness == 1) f = f + comp * f;
        else {
            V3<R> cond = reflection_fresnel_at_ior(c.base_color, c.base_weight, R(1), c.specular_weight, c.specular_color, cosine,
                                                   modulated_ior(c.specular_ior, c.specular_weight));
            f = f + comp * cond * c.base_metalness;
        }
    }
    return f;
}
// bsdf.slang:356-375 with bsdf_response.slang:257-274.
template <class R> inline V3<R> eval_mask(const Closure<R>& c, V3<R> view, V3<R> dir, uint32_t mask, const Prepared<R>& pr) {
    R bump = bump_shadow(c, dir, pr);
    V3<R> specular;
    {
        V3<R> n = pr.interface_n;
        R nl = std::max(dot(n, dir), R(0)), nv = std::max(dot(n, view), R(0.0001));
        if (nl > 0 && (mask & VKB_RAY_SPECULAR)) {
            V3<R> h = normalize(view + dir);
            R nh = std::max(dot(n, h), R(0)), vh = std::max(dot(view, h), R(0));
            Closure<R> b = c; b.n = n;
            V3<R> f = compensated_reflection(b, vh, pr.metal_comp);
            specular = ggx_reflection(f, nv, nl, nh, c.specular_roughness) * nl;
        }
    }
    bool behind = dot(c.n, dir) <= 0;
    V3<R> diffuse;
    if ((mask & VKB_RAY_DIFFUSE) && !behind) diffuse = pr.diffuse * (bump * dot(c.n, dir));
    return specular + diffuse;
}
template <class R> struct BsdfSample { V3<R> dir, weight; R pdf = 0; uint32_t event = 0; };
// bsdf_microfacet.slang:53-62.
template <class R> inline V3<R> visible_normal(V3<R> n, R roughness, V3<R> view, R ux, R uy) {
    V3<R> x = basis_direction(n, V3<R>(1, 0, 0)), y = basis_direction(n, V3<R>(0, 1, 0));
    V3<R> local(dot(view, x), dot(view, y), dot(view, n));
    V3<R> s = ggx_visible_normal(local, specular_alpha(roughness), ux, uy);
    return x * s.x + y * s.y + n * s.z;
}
// bsdf.slang:446-511.
template <class R> inline BsdfSample<R> transport_sample(const Closure<R>& c, V3<R> view, R rx, R ry, R rz, const Prepared<R>& pr) {
    BsdfSample<R> r;
    V3<R> p = pr.p, n = pr.interface_n;
    if (rz < p.x) {
        R radius = std::sqrt(rx), phi = R(TAU) * ry;
        r.dir = basis_direction(c.n, V3<R>(radius * std::cos(phi), radius * std::sin(phi), std::sqrt(1 - rx)));
        r.event = VKB_RAY_DIFFUSE;
    } else if (rz < p.x + p.y) {
        V3<R> h = visible_normal(n, c.specular_roughness, view, rx, ry);
        r.dir = reflect(-view, h);
        r.event = VKB_RAY_SPECULAR;
    } else {
        return r;
    }
    if (r.event == VKB_RAY_SPECULAR && dot(n, r.dir) <= 0) return BsdfSample<R>();
    r.pdf = pdf_mask(c, view, r.dir, r.event, pr);
    if (r.pdf > 0) r.weight = eval_mask(c, view, r.dir, r.event, pr) / r.pdf;
    return r;
}
// path.slang:833-836, :837-840.
template <class R> inline R mis_power(R sampled, R other) {
    if (sampled <= 0) return 0;
    R ratio = other / sampled;
    return 1 / (1 + ratio * ratio);
}
template <class R> inline bool event_hemisphere(uint32_t event, V3<R> dir, V3<R> face, V3<R> smooth) {
    if (event == VKB_RAY_TRANSMISSION) return dot(face, dir) < 0 && dot(smooth, dir) < 0;
    return dot(smooth, dir) > 0;
}
// path.slang:841-850 (transmission lobe has zero response: no transmitting materials).
template <class R> inline V3<R> analytic_mis_response(const Closure<R>& c, V3<R> view, V3<R> dir, V3<R> face, uint32_t contribution, R light_pdf, const Prepared<R>& pr) {
    V3<R> value;
    const uint32_t events[2] = {VKB_RAY_DIFFUSE, VKB_RAY_SPECULAR};
    for (uint32_t e : events) {
        if (!(contribution & e) || !event_hemisphere(e, dir, face, pr.smooth)) continue;
        R w = light_pdf > 0 ? mis_power(light_pdf, pdf_mask(c, view, dir, e, pr)) : R(1);
        value = value + eval_mask(c, view, dir, e, pr) * w;
    }
    return value;
}

// ---------------------------------------------------------------- emitters (shaders/emitter.slang:70-170)
template <class R> struct LightV {
    V3<R> pos; R kind; V3<R> dir; R outer; V3<R> radiance; R inner; R size; V3<R> eu; R ellipse; V3<R> ev; R range, quad;
    uint32_t contribution, link, ray, ray_link;
};
template <class R> LightV<R> light_values(const vkb_light& l) {
    LightV<R> v;
    v.pos = V3<R>(l.position[0], l.position[1], l.position[2]); v.kind = l.position[3];
    v.dir = V3<R>(l.direction[0], l.direction[1], l.direction[2]); v.outer = l.direction[3];
    v.radiance = V3<R>(l.radiance[0], l.radiance[1], l.radiance[2]); v.inner = l.radiance[3];
    v.size = l.params[1];
    v.eu = V3<R>(l.emitter_u[0], l.emitter_u[1], l.emitter_u[2]); v.ellipse = l.emitter_u[3];
    v.ev = V3<R>(l.emitter_v[0], l.emitter_v[1], l.emitter_v[2]);
    v.range = l.projection[1]; v.quad = l.projection[2];
    v.contribution = l.shadow_offsets[VKB_LIGHT_CONTRIBUTION_WORD];
    v.link = l.shadow_offsets[VKB_LIGHT_LINK_WORD];
    v.ray = l.shadow_offsets[VKB_LIGHT_RAY_WORD];
    v.ray_link = l.shadow_offsets[VKB_LIGHT_RAY_LINK_WORD];
    return v;
}
template <class R> inline R saturate(R x) { return clampr(x, R(0), R(1)); }
// emitter.slang:54-67.
template <class R> inline R emitter_window(const LightV<R>& l, V3<R> world, V3<R> dir) {
    R value = 1;
    if (l.kind > 0 && l.range > 0) {
        V3<R> rel = (l.pos - world) / l.range;
        R ratio = dot(rel, rel);
        value = std::max(1 - ratio * ratio, R(0));
    }
    if (l.kind == 2) {
        R cosine = dot(-dir, normalize(l.dir));
        R cone = cosine >= l.outer ? R(1) : R(0);
        if (l.inner > l.outer) {
            R t = saturate((cosine - l.outer) / (l.inner - l.outer));
            cone = l.quad > 0 ? t * t : t * t * (3 - 2 * t);
        }
        value *= cone;
    }
    return value;
}
template <class R> inline V3<R> cone_direction(V3<R> axis, R omc, R u, R v) {  // :71-74
    R height = u * omc;
    R radius = std::sqrt(std::max(height * (2 - height), R(0)));
    return basis_direction(axis, V3<R>(radius * std::cos(R(TAU) * v), radius * std::sin(R(TAU) * v), 1 - height));
}
template <class R> inline V3<R> emitter_direction(const LightV<R>& l, V3<R> world, R ux, R uy, R& distance) {  // :75-96
    V3<R> axis = normalize(-l.dir);
    distance = R(FP32_MAX);
    if (l.kind == 0 && l.size > 0) {
        R s = std::sin(l.size * R(0.5));
        axis = cone_direction(axis, 2 * s * s, ux, uy);
    }
    if (l.kind > 0) {
        V3<R> point = l.pos, delta = point - world;
        distance = length(delta);
        axis = distance > 0 ? delta / distance : V3<R>();
        if (l.kind == 3) {
            R sx = ux - R(0.5), sy = uy - R(0.5);
            if (l.ellipse > 0) { R r = std::sqrt(ux) * R(0.5), phi = R(TAU) * uy; sx = r * std::cos(phi); sy = r * std::sin(phi); }
            point = point + l.eu * sx + l.ev * sy;
            distance = length(point - world);
            axis = distance > 0 ? (point - world) / distance : V3<R>();
        } else if (l.size > 0 && distance > l.size) {
            R ratio = l.size / distance, sq = ratio * ratio;
            axis = cone_direction(axis, sq / (1 + std::sqrt(1 - sq)), ux, uy);
            R along = dot(delta, axis);
            V3<R> perp = cross(delta, axis);
            distance = along - std::sqrt(std::max(l.size * l.size - dot(perp, perp), R(0)));
        }
    }
    return axis;
}
template <class R> struct EmitterEval { V3<R> radiance; R pdf = 0, distance = 0; };
template <class R> inline bool emitter_delta(const LightV<R>& l) { return l.kind != 3 && l.size == 0; }
template <class R> inline EmitterEval<R> emitter_eval(const LightV<R>& l, V3<R> world, V3<R> dir) {  // :104-146
    EmitterEval<R> r;
    if (emitter_delta(l)) return r;
    if (l.kind == 0) {
        V3<R> axis = normalize(-l.dir);
        R sine = std::sin(l.size);
        V3<R> perp = cross(axis, dir);
        if (dot(axis, dir) <= 0 || dot(perp, perp) > sine * sine) return r;
        R hs = std::sin(l.size * R(0.5));
        r.pdf = 1 / (4 * R(PI) * hs * hs);
        r.radiance = l.radiance / (R(PI) * sine * sine);
        r.distance = R(FP32_MAX);
        return r;
    }
    if (l.kind < 3) {
        V3<R> delta = l.pos - world;
        R sq = dot(delta, delta), radius = l.size;
        if (sq <= radius * radius) return r;
        R along = dot(delta, dir);
        V3<R> perp = cross(delta, dir);
        R disc = radius * radius - dot(perp, perp);
        if (along <= 0 || disc < 0) return r;
        R ratio = radius * radius / sq;
        r.pdf = (1 + std::sqrt(1 - ratio)) / (R(TAU) * ratio);
        r.radiance = l.radiance / (4 * R(PI) * R(PI) * radius * radius) * emitter_window(l, world, dir);
        r.distance = along - std::sqrt(disc);
        return r;
    }
    V3<R> center = l.pos - world;
    if (dot(l.dir, -center) <= 0) return r;
    V3<R> u = l.eu * R(0.5), v = l.ev * R(0.5);
    bool ellipse = l.ellipse > 0;
    V3<R> normal = cross(u, v);
    R square = dot(normal, normal);
    if (square <= 0) return r;
    R den = dot(normal, dir);
    if (den == 0) return r;
    R distance = dot(normal, center) / den;
    if (distance <= 0) return r;
    V3<R> q = dir * distance - center;
    R uu = dot(u, u), uv = dot(u, v), vv = dot(v, v), qu = dot(q, u), qv = dot(q, v);
    R cx = (qu * vv - qv * uv) / square, cy = (qv * uu - qu * uv) / square;
    if (ellipse ? (cx * cx + cy * cy > 1) : (std::fabs(cx) > 1 || std::fabs(cy) > 1)) return r;
    R area = 4 * std::sqrt(square) * (ellipse ? R(PI) * R(0.25) : R(1));
    r.pdf = distance * distance / (area * std::fabs(den) / std::sqrt(square));
    r.radiance = l.radiance / (R(PI) * area);
    r.distance = l.kind > 0 ? distance : R(FP32_MAX);
    if (l.kind > 0) r.radiance = r.radiance * emitter_window(l, world, dir);
    return r;
}
template <class R> struct LightSample { V3<R> dir, radiance; R distance = 0, pdf = 0; bool delta = false; };
template <class R> inline LightSample<R> emitter_sample(const LightV<R>& l, V3<R> world, R ux, R uy) {  // :151-167
    LightSample<R> s;
    s.delta = emitter_delta(l);
    s.dir = emitter_direction(l, world, ux, uy, s.distance);
    if (s.delta) {
        s.radiance = l.radiance;
        if (l.kind > 0) {
            R den = 4 * R(PI) * s.distance * s.distance;
            s.radiance = den > 0 ? s.radiance / den * emitter_window(l, world, s.dir) : V3<R>();
        }
    } else {
        EmitterEval<R> e = emitter_eval(l, world, s.dir);
        s.radiance = e.radiance; s.pdf = e.pdf;
    }
    return s;
}

// ---------------------------------------------------------------- light tree (src/lights/tree.rs:72-176; light_tree.slang)
struct TreeNode { float lower_power[4], upper_infinite[4]; uint32_t links[4], source[4]; };
std::vector<TreeNode> build_light_tree(const vkb_light* lights, uint32_t n) {
    struct Src { float lo[3], hi[3]; double power; bool infinite; uint32_t id; };
    std::vector<Src> src(n);
    for (uint32_t i = 0; i < n; ++i) {
        const vkb_light& l = lights[i];
        uint32_t kind = uint32_t(l.position[3]);
        float r[3];
        for (int c = 0; c < 3; ++c)
            r[c] = kind == 3 ? (std::fabs(l.emitter_u[c]) + std::fabs(l.emitter_v[c])) * 0.5f : (kind == 0 ? 0.f : l.params[1]);
        for (int c = 0; c < 3; ++c) { src[i].lo[c] = l.position[c] - r[c]; src[i].hi[c] = l.position[c] + r[c]; }
        double p = 0;
        for (int c = 0; c < 3; ++c) p += double(l.radiance[c]) * double(float(LUM[c]));
        src[i].power = std::max(p, 0.);
        src[i].infinite = kind == 0;
        src[i].id = i;
    }
    double scale = std::numeric_limits<double>::min();
    for (auto& s : src) scale = std::max(scale, s.power);
    std::vector<TreeNode> nodes;
    std::vector<uint32_t> ids(n);
    for (uint32_t i = 0; i < n; ++i) ids[i] = i;
    struct B {
        std::vector<Src>& src; std::vector<TreeNode>& nodes; double scale;
        uint32_t build(uint32_t* ids, uint32_t count, uint32_t parent) {
            uint32_t index = uint32_t(nodes.size());
            nodes.push_back(TreeNode{});
            float lo[3] = {INFINITY, INFINITY, INFINITY}, hi[3] = {-INFINITY, -INFINITY, -INFINITY};
            double power = 0; bool inf = false;
            for (uint32_t k = 0; k < count; ++k) {
                Src& s = src[ids[k]];
                for (int c = 0; c < 3; ++c) { lo[c] = std::min(lo[c], s.lo[c]); hi[c] = std::max(hi[c], s.hi[c]); }
                power += s.power / scale; inf |= s.infinite;
            }
            float pf = float(power);
            if (pf < std::numeric_limits<float>::min()) pf = 0;
            TreeNode node{};
            for (int c = 0; c < 3; ++c) { node.lower_power[c] = lo[c]; node.upper_infinite[c] = hi[c]; }
            node.lower_power[3] = pf; node.upper_infinite[3] = inf ? 1.f : 0.f;
            node.links[0] = node.links[1] = 0xffffffffu; node.links[2] = parent; node.links[3] = count;
            if (count == 1) {
                node.source[0] = 0; node.source[1] = src[ids[0]].id; node.source[2] = ids[0];
            } else {
                double ext[3];
                for (int c = 0; c < 3; ++c) ext[c] = double(hi[c]) - double(lo[c]);
                int axis = (ext[0] >= ext[1] && ext[0] >= ext[2]) ? 0 : (ext[1] >= ext[2] ? 1 : 2);
                uint32_t finite = 0;
                for (uint32_t k = 0; k < count; ++k) finite += src[ids[k]].infinite ? 0 : 1;
                uint32_t split;
                if (finite > 0 && finite < count) {
                    std::sort(ids, ids + count, [&](uint32_t a, uint32_t b) {
                        return std::make_pair(src[a].infinite, a) < std::make_pair(src[b].infinite, b); });
                    split = finite;
                } else {
                    uint32_t mid = count / 2;
                    std::nth_element(ids, ids + mid, ids + count, [&](uint32_t a, uint32_t b) {
                        double ca = double(src[a].lo[axis]) + double(src[a].hi[axis]);
                        double cb = double(src[b].lo[axis]) + double(src[b].hi[axis]);
                        return ca < cb || (ca == cb && a < b); });
                    split = mid;
                }
                node.links[0] = build(ids, split, index);
                node.links[1] = build(ids + split, count - split, index);
            }
            nodes[index] = node;
            return index;
        }
    } b{src, nodes, scale};
    if (n) b.build(ids.data(), n, 0xffffffffu);
    return nodes;
}
template <class R> inline R tree_log_importance(const TreeNode& node, V3<R> p) {  // light_tree.slang:18-28
    if (!(node.lower_power[3] > 0)) return -R(FP32_MAX);
    R power = std::log2(R(node.lower_power[3]));
    if (node.upper_infinite[3] != 0) return power;
    V3<R> lo(node.lower_power[0], node.lower_power[1], node.lower_power[2]);
    V3<R> hi(node.upper_infinite[0], node.upper_infinite[1], node.upper_infinite[2]);
    V3<R> center = lo * R(0.5) + hi * R(0.5), radius = hi * R(0.5) - lo * R(0.5), delta = p - center;
    R d = std::max(R(LIGHT_TREE_MIN_DISTANCE_SQUARED), std::max(dot(delta, delta), dot(radius, radius)));
    if (!std::isfinite(d)) return -R(FP32_MAX);
    return power - std::log2(d);
}
template <class R> inline R tree_branch(const TreeNode& a, const TreeNode& b, V3<R> p) {  // :29-36
    R x = tree_log_importance(a, p), y = tree_log_importance(b, p);
    R scale = std::max(x, y);
    R uniform = R(a.links[3]) / (R(a.links[3]) + R(b.links[3]));
    if (scale == -R(FP32_MAX)) return uniform;
    x = std::exp2(x - scale); y = std::exp2(y - scale);
    return x / (x + y);
}
template <class R> inline uint32_t tree_pick(const std::vector<TreeNode>& nodes, V3<R> p, R ux, R uy, R& probability) {  // :53-84
    probability = 0;
    if (nodes.empty()) return 0xffffffffu;
    uint32_t node = 0;
    R prob = 1;
    const R one_below = R(1) - R(FP32_EPS) * R(0.5);
    R choice = clampr(ux, R(0), one_below);
    bool uniform = uy < R(LIGHT_TREE_UNIFORM_MIX);
    uint32_t total = nodes[0].links[3];
    uint32_t rank = std::min(uint32_t(choice * R(total)), total - 1u);
    while (nodes[node].links[0] != 0xffffffffu) {
        uint32_t l = nodes[node].links[0], r = nodes[node].links[1];
        R pb = tree_branch(nodes[l], nodes[r], p);
        bool left;
        if (uniform) {
            uint32_t cnt = nodes[l].links[3];
            left = rank < cnt;
            if (!left) rank -= cnt;
        } else {
            left = choice < pb;
            choice = left ? choice / pb : (choice - pb) / (1 - pb);
            choice = std::min(choice, one_below);
        }
        prob *= left ? pb : 1 - pb;
        node = left ? l : r;
    }
    probability = R(LIGHT_TREE_UNIFORM_MIX) / R(total) + (1 - R(LIGHT_TREE_UNIFORM_MIX)) * prob;
    return nodes[node].source[1];
}

// ---------------------------------------------------------------- scene + CPU BVH (oracle of the hit IDs)
template <class R> struct Affine {  // rows of a 3x4 matrix
    R m[3][4];
    V3<R> point(V3<R> p) const { return {m[0][0] * p.x + m[0][1] * p.y + m[0][2] * p.z + m[0][3], m[1][0] * p.x + m[1][1] * p.y + m[1][2] * p.z + m[1][3], m[2][0] * p.x + m[2][1] * p.y + m[2][2] * p.z + m[2][3]}; }
    V3<R> vec(V3<R> p) const { return {m[0][0] * p.x + m[0][1] * p.y + m[0][2] * p.z, m[1][0] * p.x + m[1][1] * p.y + m[1][2] * p.z, m[2][0] * p.x + m[2][1] * p.y + m[2][2] * p.z}; }
    // transpose-applied linear part: M^T v
    V3<R> tvec(V3<R> p) const { return {m[0][0] * p.x + m[1][0] * p.y + m[2][0] * p.z, m[0][1] * p.x + m[1][1] * p.y + m[2][1] * p.z, m[0][2] * p.x + m[1][2] * p.y + m[2][2] * p.z}; }
    R det() const { return m[0][0] * (m[1][1] * m[2][2] - m[1][2] * m[2][1]) - m[0][1] * (m[1][0] * m[2][2] - m[1][2] * m[2][0]) + m[0][2] * (m[1][0] * m[2][1] - m[1][1] * m[2][0]); }
    Affine inverse() const {
        Affine r; R d = det(), id = R(1) / d;
        r.m[0][0] = (m[1][1] * m[2][2] - m[1][2] * m[2][1]) * id; r.m[0][1] = (m[0][2] * m[2][1] - m[0][1] * m[2][2]) * id; r.m[0][2] = (m[0][1] * m[1][2] - m[0][2] * m[1][1]) * id;
        r.m[1][0] = (m[1][2] * m[2][0] - m[1][0] * m[2][2]) * id; r.m[1][1] = (m[0][0] * m[2][2] - m[0][2] * m[2][0]) * id; r.m[1][2] = (m[0][2] * m[1][0] - m[0][0] * m[1][2]) * id;
        r.m[2][0] = (m[1][0] * m[2][1] - m[1][1] * m[2][0]) * id; r.m[2][1] = (m[0][1] * m[2][0] - m[0][0] * m[2][1]) * id; r.m[2][2] = (m[0][0] * m[1][1] - m[0][1] * m[1][0]) * id;
        for (int i = 0; i < 3; ++i) r.m[i][3] = -(r.m[i][0] * m[0][3] + r.m[i][1] * m[1][3] + r.m[i][2] * m[2][3]);
        return r;
    }
};
template <class R> struct Box { V3<R> lo{R(INFINITY), R(INFINITY), R(INFINITY)}, hi{-R(INFINITY), -R(INFINITY), -R(INFINITY)};
    void grow(V3<R> p) { lo = vmin(lo, p); hi = vmax(hi, p); }
    void grow(const Box& b) { lo = vmin(lo, b.lo); hi = vmax(hi, b.hi); }
    R area() const { V3<R> e = hi - lo; return e.x < 0 ? R(0) : 2 * (e.x * e.y + e.y * e.z + e.z * e.x); }
};
template <class R> struct BvhNode { Box<R> box; uint32_t left = 0, right = 0, first = 0, count = 0; };
// Binned-SAH BVH over boxes (a plain CPU build: the oracle of hit IDs, not of topology).
template <class R> struct Bvh {
    std::vector<BvhNode<R>> nodes;
    std::vector<uint32_t> prims;
    void build(const std::vector<Box<R>>& boxes) {
        uint32_t n = uint32_t(boxes.size());
        prims.resize(n);
        for (uint32_t i = 0; i < n; ++i) prims[i] = i;
        nodes.clear(); nodes.reserve(2 * n + 1);
        std::vector<V3<R>> cent(n);
        for (uint32_t i = 0; i < n; ++i) cent[i] = (boxes[i].lo + boxes[i].hi) * R(0.5);
        if (n == 0) return;
        nodes.push_back({});
        struct Item { uint32_t node, first, count; };
        std::vector<Item> stack{{0, 0, n}};
        while (!stack.empty()) {
            Item it = stack.back(); stack.pop_back();
            BvhNode<R>& nd = nodes[it.node];
            Box<R> b, cb;
            for (uint32_t k = it.first; k < it.first + it.count; ++k) { b.grow(boxes[prims[k]]); cb.grow(cent[prims[k]]); }
            nd.box = b;
            if (it.count <= 2) { nd.first = it.first; nd.count = it.count; continue; }
            const int BINS = 16;
            R best = R(INFINITY); int best_axis = -1, best_bin = 0;
            for (int axis = 0; axis < 3; ++axis) {
                R lo = cb.lo[axis], hi = cb.hi[axis];
                if (!(hi > lo)) continue;
                Box<R> bb[BINS]; uint32_t cnt[BINS] = {};
                R sc = R(BINS) / (hi - lo);
                for (uint32_t k = it.first; k < it.first + it.count; ++k) {
                    int bi = std::min(BINS - 1, int((cent[prims[k]][axis] - lo) * sc));
                    bb[bi].grow(boxes[prims[k]]); cnt[bi]++;
                }
                Box<R> lb[BINS]; uint32_t lc[BINS];
                Box<R> acc; uint32_t ac = 0;
                for (int i = 0; i < BINS; ++i) { acc.grow(bb[i]); ac += cnt[i]; lb[i] = acc; lc[i] = ac; }
                acc = Box<R>(); ac = 0;
                for (int i = BINS - 1; i > 0; --i) {
                    acc.grow(bb[i]); ac += cnt[i];
                    R cost = lb[i - 1].area() * R(lc[i - 1]) + acc.area() * R(ac);
                    if (lc[i - 1] > 0 && ac > 0 && cost < best) { best = cost; best_axis = axis; best_bin = i; }
                }
            }
            uint32_t mid;
            if (best_axis < 0) {
                mid = it.first + it.count / 2;
            } else {
                R lo = cb.lo[best_axis], sc = R(BINS) / (cb.hi[best_axis] - lo);
                auto pivot = std::partition(prims.begin() + it.first, prims.begin() + it.first + it.count, [&](uint32_t p) {
                    return std::min(BINS - 1, int((cent[p][best_axis] - lo) * sc)) < best_bin; });
                mid = uint32_t(pivot - prims.begin());
                if (mid == it.first || mid == it.first + it.count) mid = it.first + it.count / 2;
            }
            uint32_t l = uint32_t(nodes.size());
            nodes.push_back({}); nodes.push_back({});
            nodes[it.node].left = l; nodes[it.node].right = l + 1; nodes[it.node].count = 0;
            stack.push_back({l, it.first, mid - it.first});
            stack.push_back({l + 1, mid, it.first + it.count - mid});
        }
    }
};
template <class R> inline bool box_hit(const Box<R>& b, V3<R> o, V3<R> inv, R tmax) {
    R t0 = 0, t1 = tmax;
    for (int a = 0; a < 3; ++a) {
        R ta = (b.lo[a] - o[a]) * inv[a], tb = (b.hi[a] - o[a]) * inv[a];
        if (ta > tb) std::swap(ta, tb);
        if (std::isnan(ta)) ta = -R(INFINITY);
        if (std::isnan(tb)) tb = R(INFINITY);
        t0 = std::max(t0, ta); t1 = std::min(t1, tb);
    }
    return t0 <= t1;
}

template <class R> struct MeshData {
    std::vector<V3<R>> pos, nrm; std::vector<uint32_t> idx; bool has_normals = false;
    Bvh<R> bvh; Box<R> bounds;
};
template <class R> struct Scene {
    std::vector<MeshData<R>> meshes;
    std::vector<Affine<R>> model, inv;  // object->world, world->object
    std::vector<uint32_t> inst_mesh, inst_mat;
    std::vector<vkb_material> mats;
    std::vector<vkb_light> lights;
    std::vector<TreeNode> tree;
    Bvh<R> tlas;
    vkb_camera cam; vkb_environment env;
    // Image environment: texels as float (as stored on the device), strength, colour,
    // rotation (row-major, world direction d -> d R), and the proposal table (cumulative
    // mass, density) in float as the reference stores it.
    std::vector<float> env_rgba; uint32_t env_w = 0, env_h = 0; float env_strength = 0, env_color[3] = {0, 0, 0};
    double env_rot[9] = {1, 0, 0, 0, 1, 0, 0, 0, 1};
    std::vector<float> env_cdf, env_density;
    bool env_strategy() const { return env_w > 0 && env_strength > 0; }
    // Emissive-mesh sources (emitters.rs:22-44): per instance its source index (~0u: none);
    // per source its instance and the cumulative triangle count through it; the weight
    // tree over the padded leaves (float, node 1 the root, leaves from em_leaves on).
    std::vector<uint32_t> em_inst_source, em_src_inst, em_src_cum;
    uint32_t em_tris = 0, em_leaves = 0;
    std::vector<float> em_tree;
    bool mesh_strategy() const { return !em_src_inst.empty(); }
};
// The proposal of an environment image (crates/vork-render/src/environment.rs:573-620):
// per texel the 3x3 (1,2,1)^2/16 stencil of alpha-weighted RGB (columns wrap, rows clamp),
// its Rec.709 luminance times the texel's solid angle, accumulated in f64 row-major and
// normalised; a black image falls back to the uniform sphere.
void env_distribution(const float* rgba, uint32_t dw, uint32_t dh, std::vector<float>& cdf, std::vector<float>& density) {
    std::vector<double> cum(size_t(dw) * dh), lum_of(size_t(dw) * dh);
    double total = 0;
    for (uint32_t y = 0; y < dh; ++y) {
        const double solid = TAU / dw * (std::cos(PI * y / dh) - std::cos(PI * (y + 1) / dh));
        const int rows[3] = {std::clamp(int(y) - 1, 0, int(dh) - 1), int(y), std::clamp(int(y) + 1, 0, int(dh) - 1)};
        for (uint32_t x = 0; x < dw; ++x) {
            const int cols[3] = {(int(x) - 1 + int(dw)) % int(dw), int(x), (int(x) + 1) % int(dw)};
            double rgb[3] = {0, 0, 0};
            for (int dy = 0; dy < 3; ++dy)
                for (int dx = 0; dx < 3; ++dx) {
                    const size_t at = (size_t(rows[dy]) * dw + cols[dx]) * 4;
                    const double alpha = double(rgba[at + 3]), wx = dx == 1 ? 2. : 1., wy = dy == 1 ? 2. : 1.;
                    for (int c = 0; c < 3; ++c) rgb[c] += double(rgba[at + c]) * alpha * wx * wy;
                }
            double l = 0;
            for (int c = 0; c < 3; ++c) l += double(float(LUM[c])) * (rgb[c] / 16.);
            total += l * solid;
            cum[size_t(y) * dw + x] = total;
            lum_of[size_t(y) * dw + x] = l;
        }
    }
    cdf.resize(cum.size()); density.resize(cum.size());
    if (total > 0) {
        for (size_t i = 0; i < cum.size(); ++i) { cdf[i] = float(cum[i] / total); density[i] = float(lum_of[i] / total); }
        cdf.back() = 1.f;
    } else {
        for (size_t i = 0; i < cum.size(); ++i) {
            const uint32_t y = uint32_t(i / dw), x = uint32_t(i % dw);
            const float row = (1.f - std::cos(float(PI) * float(y) / float(dh))) / 2.f;
            const float next = (1.f - std::cos(float(PI) * float(y + 1) / float(dh))) / 2.f;
            cdf[i] = row + (next - row) * (float(x + 1) / float(dw));
            density[i] = 1.f / (4.f * float(PI));
        }
    }
}
// ---------------------------------------------------------------- emissive meshes
// A material emits when emission_luminance > 0 and its colour is not black
// (materials.rs:579-583); every instance drawn with such a material is a source, its
// triangles counted in instance order (emitters.rs:22-44, opaque materials only).
inline bool material_emits(const vkb_material& m) {
    return m.emission_luminance > 0.f && (m.emission_color[0] != 0.f || m.emission_color[1] != 0.f || m.emission_color[2] != 0.f);
}
inline uint32_t emitter_leaves(uint32_t count) {                          // emitter_mesh_proposal.slang:12
    uint32_t l = 1;
    while (l < count) l <<= 1;
    return l;
}
template <class R> void emitter_sources(Scene<R>& s) {
    const uint32_t n = uint32_t(s.inst_mesh.size());
    s.em_inst_source.assign(n, 0xffffffffu);
    s.em_src_inst.clear(); s.em_src_cum.clear(); s.em_tris = 0;
    for (uint32_t i = 0; i < n; ++i) {
        if (!material_emits(s.mats[s.inst_mat[i]])) continue;
        s.em_tris += uint32_t(s.meshes[s.inst_mesh[i]].idx.size() / 3);
        s.em_inst_source[i] = uint32_t(s.em_src_inst.size());
        s.em_src_inst.push_back(i);
        s.em_src_cum.push_back(s.em_tris);
    }
    s.em_leaves = s.em_src_inst.empty() ? 0u : emitter_leaves(s.em_tris);
}
// Source triangle -> (source, primitive) by binary search over the cumulative counts
// (emitter_mesh_proposal.slang:13-22); a triangle past the last source (reachable only
// through a zero-mass branch) maps to the last source.
template <class R> void emitter_triangle(const Scene<R>& s, uint32_t triangle, uint32_t& source, uint32_t& primitive) {
    uint32_t low = 0, high = uint32_t(s.em_src_inst.size());
    while (low < high) {
        const uint32_t mid = (low + high) / 2;
        if (triangle < s.em_src_cum[mid]) high = mid; else low = mid + 1;
    }
    source = std::min(low, uint32_t(s.em_src_inst.size()) - 1u);
    primitive = triangle - (source == 0 ? 0u : s.em_src_cum[source - 1]);
}
// Current world-space corners of a source triangle: the object corners, the edge vectors
// and the point at barycentrics (b1, b2) (hit_geometry.slang:121-124, 246-256).
template <class R> struct EmitterGeometry { V3<R> point, face; R area; };
template <class R> EmitterGeometry<R> emitter_geometry(const Scene<R>& s, uint32_t inst, uint32_t prim, R b1, R b2) {
    const MeshData<R>& m = s.meshes[s.inst_mesh[inst]];
    const Affine<R>& M = s.model[inst];
    const Affine<R>& I = s.inv[inst];
    const uint32_t i0 = m.idx[3 * prim], i1 = m.idx[3 * prim + 1], i2 = m.idx[3 * prim + 2];
    const V3<R> P[3] = {m.pos[i0], m.pos[i1], m.pos[i2]};
    const V3<R> raw = cross(P[1] - P[0], P[2] - P[0]);
    const V3<R> fobj = finite_unit_normal(raw, m.has_normals ? m.nrm[i0] : raw);
    EmitterGeometry<R> g;
    g.face = finite_unit_normal(I.tvec(fobj), V3<R>(0, 0, 1));
    g.point = M.point(P[0] * (R(1) - b1 - b2) + P[1] * b1 + P[2] * b2);
    g.area = length(cross(M.vec(P[1] - P[0]), M.vec(P[2] - P[0]))) * R(0.5);
    return g;
}
// The frame's weight tree (emitter_weights.slang:23-55): leaf = world area x the
// emission's Rec.709 luminance power (the area alone when that product is not finite),
// padded leaves 0; an inner node stores the mean of its children.
template <class R> void emitter_tree(Scene<R>& s) {
    s.em_tree.assign(s.em_leaves ? 2 * size_t(s.em_leaves) : 0, 0.f);
    if (!s.em_leaves) return;
    for (uint32_t t = 0; t < s.em_tris; ++t) {
        uint32_t src, prim;
        emitter_triangle(s, t, src, prim);
        const uint32_t inst = s.em_src_inst[src];
        float area = float(emitter_geometry(s, inst, prim, R(0), R(0)).area);
        if (area > 0.f) {
            const vkb_material& mt = s.mats[s.inst_mat[inst]];
            const float power = (std::max(mt.emission_color[0], 0.f) * float(LUM[0]) + std::max(mt.emission_color[1], 0.f) * float(LUM[1]) +
                                 std::max(mt.emission_color[2], 0.f) * float(LUM[2])) * std::max(mt.emission_luminance, 0.f);
            const float weight = area * power;
            if (std::isfinite(weight)) area = weight;
        }
        s.em_tree[s.em_leaves + t] = area;
    }
    for (uint32_t node = s.em_leaves - 1; node >= 1; --node) s.em_tree[node] = 0.5f * s.em_tree[2 * node] + 0.5f * s.em_tree[2 * node + 1];
}
// Ratio of sibling masses under a shared power-of-two scale (emitter_mesh_proposal.slang:25-35).
inline float emitter_left_probability(float left, float right) {
    uint32_t bits;
    const float top = std::max(left, right);
    std::memcpy(&bits, &top, 4);
    const int exponent = int((bits >> 23) & 255u) - 127;
    const uint32_t sb = uint32_t(127 - exponent / 2) << 23;
    float scale;
    std::memcpy(&scale, &sb, 4);
    left *= scale; right *= scale;
    if (left >= right) return left > 0.f ? 1.f / (1.f + right / left) : 0.f;
    const float ratio = left / right;
    return ratio / (1.f + ratio);
}
constexpr float MESH_SOURCE_UNIFORM_MIX = 0.5f;   // registry.rs MESH_SOURCE_UNIFORM_MIX
// The product of the branch probabilities from the leaf up, mixed half and half with the
// uniform choice over all source triangles (emitter_mesh_proposal.slang:37-57).
template <class R> float emitter_probability(const Scene<R>& s, uint32_t inst, uint32_t prim) {
    if (!s.mesh_strategy() || s.em_inst_source[inst] == 0xffffffffu || !(s.em_tree[1] > 0.f)) return 0.f;
    const uint32_t src = s.em_inst_source[inst];
    uint32_t node = s.em_leaves + prim + (src == 0 ? 0u : s.em_src_cum[src - 1]);
    float probability = 1.f;
    bool zero = false;
    while (node > 1) {
        const uint32_t parent = node / 2;
        const float left = s.em_tree[2 * parent], right = s.em_tree[2 * parent + 1];
        if (std::max(left, right) <= 0.f) { zero = true; break; }
        const float p = emitter_left_probability(left, right);
        probability *= (node & 1u) ? 1.f - p : p;
        node = parent;
    }
    const float weighted = zero ? 0.f : probability;
    return (1.f - MESH_SOURCE_UNIFORM_MIX) * weighted + MESH_SOURCE_UNIFORM_MIX / float(s.em_tris);
}
// emitter_mesh_sample (emitter_mesh_proposal.slang:59-83): u = path_triangle (the vertex's
// group 2 as .zxy): x picks the triangle, y the radius, z the strategy and the split.
template <class R> bool emitter_sample(const Scene<R>& s, const float u[3], uint32_t& inst, uint32_t& prim, float& b1, float& b2) {
    const float top = 0x1.fffffep-1f;
    float choice = std::min(u[0], top);
    uint32_t node = 1;
    if (!(s.em_tree[1] > 0.f)) return false;
    const bool uniform = u[2] < MESH_SOURCE_UNIFORM_MIX;
    const float point = (u[2] - (uniform ? 0.f : MESH_SOURCE_UNIFORM_MIX)) / (uniform ? MESH_SOURCE_UNIFORM_MIX : 1.f - MESH_SOURCE_UNIFORM_MIX);
    if (uniform) node = s.em_leaves + std::min(uint32_t(choice * float(s.em_tris)), s.em_tris - 1u);
    else
        while (node < s.em_leaves) {
            const float p = emitter_left_probability(s.em_tree[2 * node], s.em_tree[2 * node + 1]);
            if (choice < p) { choice /= p; node *= 2; }
            else { choice = (choice - p) / (1.f - p); node = 2 * node + 1; }
            choice = std::min(choice, top);
        }
    uint32_t src;
    emitter_triangle(s, node - s.em_leaves, src, prim);
    inst = s.em_src_inst[src];
    const float radius = std::sqrt(u[1]);
    b1 = radius * (1.f - point);
    b2 = radius - b1;
    return true;
}
// emitter_mesh_pdf x the triangle's probability (path.slang:996-1002, emitter_mesh_proposal.slang:86-92):
// the solid-angle density at `from` of the point on a source triangle.
template <class R> R mesh_pdf(const Scene<R>& s, uint32_t inst, uint32_t prim, R area, V3<R> from, V3<R> point, V3<R> face) {
    if (!s.mesh_strategy() || s.em_inst_source[inst] == 0xffffffffu) return 0;
    const V3<R> delta = point - from;
    const R squared = dot(delta, delta);
    const R cosine = std::fabs(dot(face, normalize(delta)));
    const R density = area > 0 && cosine > 0 ? squared / (area * cosine) : R(0);
    return density * R(emitter_probability(s, inst, prim));
}

template <class R> Scene<R>* make_scene(const vkb_scene_desc* d) {
    Scene<R>* s = new Scene<R>();
    s->meshes.resize(d->num_meshes);
    for (uint32_t m = 0; m < d->num_meshes; ++m) {
        const vkb_mesh& src = d->meshes[m];
        MeshData<R>& md = s->meshes[m];
        md.pos.resize(src.num_vertices);
        for (uint32_t i = 0; i < src.num_vertices; ++i) { md.pos[i] = V3<R>(src.positions[3 * i], src.positions[3 * i + 1], src.positions[3 * i + 2]); md.bounds.grow(md.pos[i]); }
        md.has_normals = src.normals != nullptr;
        if (md.has_normals) {
            md.nrm.resize(src.num_vertices);
            for (uint32_t i = 0; i < src.num_vertices; ++i) md.nrm[i] = V3<R>(src.normals[3 * i], src.normals[3 * i + 1], src.normals[3 * i + 2]);
        }
        md.idx.assign(src.indices, src.indices + size_t(src.num_triangles) * 3);
        std::vector<Box<R>> boxes(src.num_triangles);
        for (uint32_t t = 0; t < src.num_triangles; ++t)
            for (int k = 0; k < 3; ++k) boxes[t].grow(md.pos[md.idx[3 * t + k]]);
        md.bvh.build(boxes);
    }
    uint32_t n = d->num_instances;
    s->model.resize(n); s->inv.resize(n);
    s->inst_mesh.assign(d->instance_mesh, d->instance_mesh + n);
    s->inst_mat.assign(d->instance_material, d->instance_material + n);
    std::vector<Box<R>> boxes(n);
    for (uint32_t i = 0; i < n; ++i) {
        for (int r = 0; r < 3; ++r) for (int c = 0; c < 4; ++c) s->model[i].m[r][c] = R(d->instance_rows[12 * i + 4 * r + c]);
        s->inv[i] = s->model[i].inverse();
        const Box<R>& mb = s->meshes[s->inst_mesh[i]].bounds;
        for (int k = 0; k < 8; ++k) boxes[i].grow(s->model[i].point(V3<R>(k & 1 ? mb.hi.x : mb.lo.x, k & 2 ? mb.hi.y : mb.lo.y, k & 4 ? mb.hi.z : mb.lo.z)));
    }
    s->tlas.build(boxes);
    s->mats.assign(d->materials, d->materials + d->num_materials);
    s->lights.assign(d->lights, d->lights + d->num_lights);
    s->tree = build_light_tree(d->lights, d->num_lights);
    s->cam = d->camera; s->env = d->environment;
    if (d->environment_image && d->environment_image->rgba && d->environment_image->width && d->environment_image->height) {
        const vkb_environment_image& e = *d->environment_image;
        s->env_w = e.width; s->env_h = e.height; s->env_strength = e.strength;
        for (int c = 0; c < 3; ++c) s->env_color[c] = e.color[c];
        s->env_rgba.assign(e.rgba, e.rgba + size_t(e.width) * e.height * 4);
        bool any = false;
        for (int k = 0; k < 9; ++k) any = any || e.rotation[k] != 0.f;
        if (any) for (int k = 0; k < 9; ++k) s->env_rot[k] = double(e.rotation[k]);
        env_distribution(e.rgba, e.width, e.height, s->env_cdf, s->env_density);
    }
    emitter_sources(*s);
    emitter_tree(*s);
    return s;
}
struct Hit { double t = -1; uint32_t inst = 0xffffffffu, prim = 0xffffffffu; double u = 0, v = 0; };
// Moller-Trumbore in R; det > 0 is a front face (dot(n, d) < 0 with n = cross(e1, e2)).
template <class R> inline bool tri_hit(V3<R> o, V3<R> d, V3<R> p0, V3<R> p1, V3<R> p2, bool cull, R tmax, R& t, R& u, R& v) {
    V3<R> e1 = p1 - p0, e2 = p2 - p0, pv = cross(d, e2);
    R det = dot(e1, pv);
    if (cull ? !(det > 0) : det == 0) return false;
    R id = R(1) / det;
    V3<R> tv = o - p0;
    u = dot(tv, pv) * id;
    if (u < 0 || u > 1) return false;
    V3<R> qv = cross(tv, e1);
    v = dot(d, qv) * id;
    if (v < 0 || u + v > 1) return false;
    t = dot(e2, qv) * id;
    return t >= 0 && t <= tmax;
}
// Closest hit (back faces culled unless the material is double sided, path.slang:149)
// or any hit (no culling, path.slang:639) against the two-level scene.
template <class R> Hit trace(const Scene<R>& s, V3<R> o, V3<R> d, R tmax, bool any) {
    Hit h;
    R best = tmax;
    V3<R> inv(R(1) / d.x, R(1) / d.y, R(1) / d.z);
    if (s.tlas.nodes.empty()) return h;
    uint32_t st[256];
    int sp = 0;
    st[sp++] = 0;
    while (sp > 0) {
        const BvhNode<R>& nd = s.tlas.nodes[st[--sp]];
        if (!box_hit(nd.box, o, inv, best)) continue;
        if (nd.count == 0) { if (sp + 2 <= 256) { st[sp++] = nd.left; st[sp++] = nd.right; } continue; }
        for (uint32_t k = nd.first; k < nd.first + nd.count; ++k) {
            uint32_t inst = s.tlas.prims[k];
            const MeshData<R>& m = s.meshes[s.inst_mesh[inst]];
            if (m.bvh.nodes.empty()) continue;
            // Facing is decided in object space (hardware facing of the instance's own winding).
            bool cull = !any && !(s.mats[s.inst_mat[inst]].flags & 2u);
            V3<R> oo = s.inv[inst].point(o), od = s.inv[inst].vec(d);
            V3<R> oinv(R(1) / od.x, R(1) / od.y, R(1) / od.z);
            uint32_t bs[256];
            int bp = 0;
            bs[bp++] = 0;
            while (bp > 0) {
                const BvhNode<R>& bn = m.bvh.nodes[bs[--bp]];
                if (!box_hit(bn.box, oo, oinv, best)) continue;
                if (bn.count == 0) { if (bp + 2 <= 256) { bs[bp++] = bn.left; bs[bp++] = bn.right; } continue; }
                for (uint32_t q = bn.first; q < bn.first + bn.count; ++q) {
                    uint32_t tri = m.bvh.prims[q];
                    R t, u, v;
                    if (tri_hit(oo, od, m.pos[m.idx[3 * tri]], m.pos[m.idx[3 * tri + 1]], m.pos[m.idx[3 * tri + 2]], cull, best, t, u, v)) {
                        best = t; h.t = double(t); h.inst = inst; h.prim = tri; h.u = double(u); h.v = double(v);
                        if (any) return h;
                    }
                }
            }
        }
    }
    return h;
}

// ---------------------------------------------------------------- hit reconstruction (hit_geometry.slang, hit.slang, surface.slang)
template <class R> struct HitSurf {
    V3<R> world, face, geometric, error;  // face: toward the incoming ray; geometric: smooth normal
    V3<R> shadow_xyz; R shadow_cone = 0;
    bool entering = true;
};
// material.slang:69-79.
template <class R> V3<R> position_error(const Scene<R>& s, uint32_t inst, V3<R> world) {
    const Box<R>& b = s.meshes[s.inst_mesh[inst]].bounds;
    V3<R> mag = vmax(vabs(b.lo), vabs(b.hi)), span = vabs(b.hi - b.lo);
    R extent = maxc(span);
    const Affine<R>& M = s.model[inst];
    const Affine<R>& I = s.inv[inst];
    V3<R> aw = vabs(world), iw;
    for (int r = 0; r < 3; ++r) iw[r] = std::fabs(I.m[r][0]) * aw.x + std::fabs(I.m[r][1]) * aw.y + std::fabs(I.m[r][2]) * aw.z + std::fabs(I.m[r][3]);
    R g7 = R(FP32_GAMMA7);
    V3<R> local = (mag + V3<R>(extent, extent, extent) + iw) * g7;
    V3<R> out;
    for (int r = 0; r < 3; ++r) {
        R a = 0, m = 0;
        for (int c = 0; c < 3; ++c) { a += std::fabs(M.m[r][c]) * local[c]; m += std::fabs(M.m[r][c]) * mag[c]; }
        out[r] = a + g7 * (m + std::fabs(M.m[r][3]));
    }
    return out;
}
// hit_geometry.slang:174-205.
template <class R> void shadow_terminator(const V3<R> p[3], V3<R> n[3], V3<R> face, const R b[3], V3<R>& xyz, R& cone) {
    V3<R> smooth = n[0] * b[0] + n[1] * b[1] + n[2] * b[2];
    if (dot(smooth, face) < 0) { for (int i = 0; i < 3; ++i) n[i] = -n[i]; smooth = -smooth; }
    V3<R> point = p[0] * b[0] + p[1] * b[1] + p[2] * b[2];
    R envelope = 0, quadratic = 0; cone = 0;
    for (int i = 0; i < 3; ++i) {
        R support = 0;
        for (int j = 0; j < 3; ++j) support = std::max(support, dot(p[j] - point, n[i]));
        envelope = i == 0 ? support : std::min(envelope, support);
        cone = std::max(cone, length(n[i] - face));
        for (int j = i + 1; j < 3; ++j) quadratic += b[i] * b[j] * dot(n[j] - n[i], p[j] - p[i]);
    }
    xyz = smooth * std::max(envelope, R(0.5) * quadratic);
}
template <class R> HitSurf<R> hit_surface(const Scene<R>& s, const Hit& h, V3<R> dir) {
    HitSurf<R> hs;
    const MeshData<R>& m = s.meshes[s.inst_mesh[h.inst]];
    const Affine<R>& M = s.model[h.inst];
    const Affine<R>& I = s.inv[h.inst];
    uint32_t i0 = m.idx[3 * h.prim], i1 = m.idx[3 * h.prim + 1], i2 = m.idx[3 * h.prim + 2];
    V3<R> P[3] = {m.pos[i0], m.pos[i1], m.pos[i2]};
    V3<R> fobj_raw = cross(P[1] - P[0], P[2] - P[0]);
    V3<R> N[3];
    if (m.has_normals) { N[0] = m.nrm[i0]; N[1] = m.nrm[i1]; N[2] = m.nrm[i2]; }
    else N[0] = N[1] = N[2] = fobj_raw;
    V3<R> fobj = finite_unit_normal(fobj_raw, N[0]);
    R b[3] = {R(1) - R(h.u) - R(h.v), R(h.u), R(h.v)};
    V3<R> face = finite_unit_normal(I.tvec(fobj), V3<R>(0, 0, 1));      // hit_face
    hs.entering = dot(face, dir) < 0;
    hs.world = M.point(P[0] * b[0] + P[1] * b[1] + P[2] * b[2]);         // hit_point
    V3<R> nrm = I.tvec(N[0] * b[0] + N[1] * b[1] + N[2] * b[2]);
    V3<R> facew = I.tvec(fobj);
    V3<R> un = finite_unit_normal(nrm, facew);
    nrm = dot(un, facew) < 0 ? -un : un;                                 // winding_normal
    bool object_front = hs.entering != (M.det() < 0);                    // material_front
    hs.geometric = finite_unit_normal(nrm, V3<R>(0, 0, 1)) * (object_front ? R(1) : R(-1));
    // hit_shadow_offset (hit_geometry.slang:193-204), front = entering (hit.slang:36).
    R side = hs.entering ? R(1) : R(-1);
    V3<R> sf = face * side;
    V3<R> p[3], n[3];
    for (int k = 0; k < 3; ++k) { p[k] = M.vec(P[k] - P[0]); n[k] = finite_unit_normal(I.tvec(N[k]) * side, sf); }
    shadow_terminator(p, n, sf, b, hs.shadow_xyz, hs.shadow_cone);
    hs.face = hs.entering ? face : -face;
    hs.error = position_error(s, h.inst, hs.world);
    return hs;
}
// vork_prelude.slang:340-345.
template <class R> V3<R> shadow_offset(const HitSurf<R>& hs, V3<R> dir) {
    R cone = hs.shadow_cone;
    if (cone <= 0) return V3<R>();
    R nl = dot(hs.geometric, dir), ng = dot(hs.face, dir);
    R amount = nl < cone ? saturate(2 - (ng + nl) / cone) : saturate(1 - ng / cone);
    return hs.shadow_xyz * amount;
}
// vork_prelude.slang:170-181.
template <class R> V3<R> surface_ray_origin(V3<R> world, V3<R> error, V3<R> g, V3<R> dir) {
    R scale = maxc(vabs(g));
    if (scale == 0) return world;
    V3<R> n = g / scale;
    R amount = dot(vabs(n), error) / dot(n, n);
    amount = amount == 0 ? std::numeric_limits<R>::denorm_min() : next_float(amount, true);
    V3<R> offset = n * (amount * (dot(n, dir) >= 0 ? R(1) : R(-1)));
    V3<R> o = world + offset;
    for (int a = 0; a < 3; ++a)
        if (offset[a] != 0) {
            R v = o[a];
            o[a] = v == 0 ? (offset[a] > 0 ? std::numeric_limits<R>::denorm_min() : -std::numeric_limits<R>::denorm_min()) : next_float(v, offset[a] > 0);
        }
    return o;
}
// path.slang:771-784 (not hair).
template <class R> V3<R> path_origin(const HitSurf<R>& hs, V3<R> dir) {
    bool reflection = dot(hs.geometric, dir) > 0;
    V3<R> base = hs.world + (reflection ? shadow_offset(hs, dir) : V3<R>());
    return surface_ray_origin(base, hs.error, reflection ? hs.geometric : hs.face, dir);
}
// vork_prelude.slang:162-167.
template <class R> void ray_connection(V3<R> origin, V3<R> world, V3<R> dir, R distance, V3<R>& out_dir, R& out_dist) {
    if (distance == R(FP32_MAX) || (origin.x == world.x && origin.y == world.y && origin.z == world.z)) { out_dir = dir; out_dist = distance; return; }
    V3<R> delta = dir * distance - (origin - world);
    R rem = length(delta);
    out_dir = rem > 0 ? delta / rem : dir;
    out_dist = rem;
}
// sample_clamp.slang:7-17.
template <class R> V3<R> clamp_sample(V3<R> v, R limit, uint64_t& dropped) {
    R br = (std::fabs(v.x) + std::fabs(v.y) + std::fabs(v.z)) * (R(1) / R(3));
    if (!std::isfinite(br)) { dropped++; v = V3<R>(); br = 0; }
    return v * ((limit > 0 && br > limit) ? limit / std::max(br, R(POSITIVE_EPSILON)) : R(1));
}

// ---------------------------------------------------------------- image environment
// vork_prelude.slang:78-85.
template <class R> inline void equirect_uv(V3<R> d, R& u, R& v) {
    if (d.x == 0 && d.z == 0) { u = R(0.5); v = d.y > 0 ? R(0) : R(1); return; }
    u = std::atan2(d.z, d.x) / R(TAU) + R(0.5);
    v = std::atan2(std::sqrt(d.x * d.x + d.z * d.z), d.y) / R(PI);
}
// World -> environment (row vector times the rotation) and back (environment_uv,
// environment_direction: path.slang:985-992).
template <class R> inline V3<R> env_local(const Scene<R>& s, V3<R> d) {
    const double* m = s.env_rot;
    return normalize(V3<R>(d.x * R(m[0]) + d.y * R(m[3]) + d.z * R(m[6]), d.x * R(m[1]) + d.y * R(m[4]) + d.z * R(m[7]),
                           d.x * R(m[2]) + d.y * R(m[5]) + d.z * R(m[8])));
}
template <class R> inline V3<R> env_world(const Scene<R>& s, V3<R> l) {
    const double* m = s.env_rot;
    return normalize(V3<R>(R(m[0]) * l.x + R(m[1]) * l.y + R(m[2]) * l.z, R(m[3]) * l.x + R(m[4]) * l.y + R(m[5]) * l.z,
                           R(m[6]) * l.x + R(m[7]) * l.y + R(m[8]) * l.z));
}
template <class R> inline R fracr(R x) { return x - std::floor(x); }
// environment_radiance, wrap mode 0 (vork_prelude.slang:306-330): bilinear by differences.
template <class R> V3<R> env_lookup(const Scene<R>& s, R u, R v) {
    const int w = int(s.env_w), h = int(s.env_h);
    const R px = fracr(u) * R(w) - R(0.5), py = clampr(v, R(0), R(1)) * R(h) - R(0.5);
    const int cx = int(std::floor(px)), cy = int(std::floor(py));
    const R fx = fracr(px), fy = fracr(py);
    const int x0 = (cx + w) % w, x1 = (x0 + 1) % w, y0 = std::clamp(cy, 0, h - 1), y1 = std::clamp(cy + 1, 0, h - 1);
    auto at = [&](int x, int y) { const float* t = &s.env_rgba[(size_t(y) * w + x) * 4]; return V3<R>(t[0], t[1], t[2]); };
    const V3<R> a = at(x0, y0), b = at(x1, y0), c = at(x0, y1), d = at(x1, y1);
    const V3<R> top = a + (b - a) * fx, bottom = c + (d - c) * fx;
    return top + (bottom - top) * fy;
}
// The environment radiance of a non-camera direction (path.slang:961-983).
template <class R> V3<R> path_environment(const Scene<R>& s, V3<R> dir) {
    V3<R> r(s.env.radiance[0], s.env.radiance[1], s.env.radiance[2]);
    if (s.env_strategy()) {
        R u, v;
        equirect_uv(env_local(s, dir), u, v);
        const V3<R> img = env_lookup(s, u, v);
        r = r + img * R(s.env_strength) * V3<R>(s.env_color[0], s.env_color[1], s.env_color[2]);
    }
    return r;
}
// environment_proposal.slang:5-14, 17-24, 29-49.
template <class R> R env_solid_angle(const Scene<R>& s, uint32_t row) {
    const R angle = R(PI) / R(s.env_h);
    return R(TAU) / R(s.env_w) * 2 * std::sin(angle * (R(row) + R(0.5))) * std::sin(R(0.5) * angle);
}
template <class R> R env_pdf_local(const Scene<R>& s, V3<R> l) {
    R u, v;
    equirect_uv(l, u, v);
    const uint32_t cx = std::min(uint32_t(fracr(u) * R(s.env_w)), s.env_w - 1), cy = std::min(uint32_t(clampr(v, R(0), R(1)) * R(s.env_h)), s.env_h - 1);
    const uint32_t index = cy * s.env_w + cx;
    const R previous = index > 0 ? R(s.env_cdf[index - 1]) : R(0);
    return (R(s.env_cdf[index]) - previous) / env_solid_angle(s, cy);
}
inline uint32_t env_cdf_search(const std::vector<float>& cdf, uint32_t first, uint32_t stride, uint32_t count, float base, float target) {
    uint32_t low = 0, high = count - 1;
    while (low < high) {
        const uint32_t mid = (low + high) / 2;
        if (cdf[first + mid * stride] - base <= target) low = mid + 1; else high = mid;
    }
    return low;
}
template <class R> V3<R> env_sample_local(const Scene<R>& s, float ux, float uy, R& pdf) {
    const std::vector<float>& cdf = s.env_cdf;
    const uint32_t w = s.env_w, h = s.env_h;
    const uint32_t row = env_cdf_search(cdf, w - 1, w, h, 0.f, uy);
    const float row_start = row > 0 ? cdf[row * w - 1] : 0.f;
    const float row_mass = cdf[(row + 1) * w - 1] - row_start;
    const float target = std::min(ux * row_mass, std::nextafter(row_mass, -INFINITY));
    const uint32_t column = env_cdf_search(cdf, row * w, 1, w, row_start, target);
    const uint32_t at = row * w + column;
    const float previous = (at > 0 ? cdf[at - 1] : 0.f) - row_start;
    const R fraction = (R(target) - R(previous)) / (R(cdf[at]) - R(row_start) - R(previous));
    const R height = (R(uy) - R(row_start)) / R(row_mass);
    const R phi = R(TAU) * ((R(column) + fraction) / R(w) - R(0.5));
    const R cosine = lerp(std::cos(R(PI) * R(row) / R(h)), std::cos(R(PI) * R(row + 1) / R(h)), height);
    const R sine = std::sqrt(std::max(1 - cosine * cosine, R(0)));
    pdf = (R(cdf[at]) - (at > 0 ? R(cdf[at - 1]) : R(0))) / env_solid_angle(s, row);
    return V3<R>(sine * std::cos(phi), cosine, sine * std::sin(phi));
}
template <class R> R environment_density(const Scene<R>& s, V3<R> dir) { return env_pdf_local(s, env_local(s, dir)); }

template <class R> struct Ctx {
    const Scene<R>& s;
    const vkb_profile& prof;
    uint64_t dropped_light = 0, dropped_path = 0, ext_rays = 0, shadow_rays = 0;
};
template <class R> R filter_offset(R u) {  // path.slang:1712-1719
    const std::vector<float>& t = filter_table();
    R x = clampr(u, R(0), R(1)) * R(FILTER_INTERVALS);
    uint32_t i = std::min(uint32_t(x), FILTER_INTERVALS - 1u);
    return lerp(R(t[i]), R(t[i + 1]), x - R(i));
}
template <class R> void camera_ray(const vkb_camera& cam, uint32_t px, uint32_t py, const float cs[4], V3<R>& origin, V3<R>& dir, R& tmax) {
    // path.slang:1722-1774 with vork_prelude.slang:95-108 (pinhole, no lens, no jitter shift).
    R nx = (R(px) + R(0.5) + filter_offset(R(cs[0]))) / R(cam.width) * R(2) + R(-1);
    R ny = (R(py) + R(0.5) + filter_offset(R(cs[1]))) / R(cam.height) * R(-2) + R(1);
    V3<R> right(cam.right[0], cam.right[1], cam.right[2]), up(cam.up[0], cam.up[1], cam.up[2]), fwd(cam.forward[0], cam.forward[1], cam.forward[2]);
    V3<R> eye(cam.eye[0], cam.eye[1], cam.eye[2]);
    R cx = nx / R(cam.proj_x), cy = ny / R(cam.proj_y);
    dir = normalize(fwd + right * cx + up * cy);
    R near_d = R(cam.near_plane) / dot(dir, fwd), far_d = R(cam.far_plane) / dot(dir, fwd);
    origin = eye + dir * near_d;
    tmax = std::min(R(FP32_MAX), std::max(R(0), far_d - length(origin - eye)));
}
template <class R> bool occluded(Ctx<R>& cx, V3<R> o, V3<R> d, R dist) {
    cx.shadow_rays++;
    return trace(cx.s, o, d, dist, true).t >= 0;
}
template <class R> V3<R> next_event(Ctx<R>& cx, const HitSurf<R>& hs, const Closure<R>& c, V3<R> view, const Prepared<R>& pr,
                                    const BsdfSample<R>& smp, const Sampler& sm, uint32_t& rng, uint32_t groups) {
    const Scene<R>& s = cx.s;
    if (s.lights.empty()) return V3<R>();
    float u[4];
    vertex_group(sm, 1, u);                                               // path_light
    R probability;
    uint32_t i = tree_pick(s.tree, hs.world, R(u[2]), R(u[3]), probability);
    if (!(probability > 0)) return V3<R>();
    LightV<R> L = light_values<R>(s.lights[i]);
    if (!((L.contribution & VKB_LIGHT_LINK_ALL) || (L.link & groups))) return V3<R>();
    LightSample<R> src = emitter_sample(L, hs.world, R(u[0]), R(u[1]));
    R light_pdf = src.pdf;
    V3<R> power = src.delta ? src.radiance : (src.pdf > 0 ? src.radiance / src.pdf : V3<R>());
    V3<R> response = analytic_mis_response(c, view, src.dir, hs.face, L.contribution, light_pdf, pr);
    V3<R> value = response * power / probability;
    R threshold = R(cx.prof.light_threshold), importance = maxc(value);
    if (importance < threshold && threshold > 0) {
        R keep = importance / threshold;
        if (R(path_random(rng)) >= keep) value = V3<R>(); else value = value / keep;
    }
    if (any_nonzero(value) && (L.ray & VKB_LIGHT_RAY_SHADOWED)) {
        V3<R> o = path_origin(hs, src.dir), cd; R cl;
        ray_connection(o, hs.world, src.dir, src.distance, cd, cl);
        if (occluded(cx, o, cd, cl)) value = V3<R>();
    }
    bool continuation = (L.contribution & smp.event) && event_hemisphere(smp.event, smp.dir, hs.face, hs.geometric);
    if (continuation && dot(smp.dir, smp.dir) > 0) {
        EmitterEval<R> e = emitter_eval(L, hs.world, smp.dir);
        if (e.pdf > 0) {
            R w = smp.pdf > 0 ? mis_power(smp.pdf, e.pdf) : R(1);
            V3<R> second = smp.weight * e.radiance * (w / probability);
            R imp = maxc(second);
            if (imp < threshold && threshold > 0) {
                R keep = imp / threshold;
                if (R(path_random(rng)) >= keep) second = V3<R>(); else second = second / keep;
            }
            if (any_nonzero(second) && (L.ray & VKB_LIGHT_RAY_SHADOWED)) {
                V3<R> o = path_origin(hs, smp.dir), cd; R cl;
                ray_connection(o, hs.world, smp.dir, e.distance, cd, cl);
                if (occluded(cx, o, cd, cl)) second = V3<R>();
            }
            value = value + second;
        }
    }
    return value;
}
// Denoiser guide albedo of the camera hit (path.slang:1549-1571): the surface's response
// to a uniform white world, diffuse + reflected, from surface_radiance_at
// (surface_lighting.slang:260-300): diffuse = direct_diffuse * pi (bsdf_response.slang:
// 82-96), reflected = specular_reflectance(specular_response(c, view), brdf_moments(nv,
// roughness)) (bsdf_response.slang:47-77) with the closure's own normal; clamped to
// [0, 1] (the closure weight is 1: one closure, no opacity).
template <class R> V3<R> guide_albedo(const Closure<R>& c, V3<R> view) {
    V3<R> n = c.n;
    R nv = std::max(dot(n, view), R(0.0001));
    R m[3];
    lut<R>().moments(nv, c.specular_roughness, m);
    V3<R> diffuse = direct_diffuse(c, view) * R(PI);
    R f0 = fresnel(R(1), dielectric_ior(c));
    R grazing = f0 != 0 ? m[1] : R(0);
    V3<R> reflected = (V3<R>(f0, f0, f0) * m[0] + V3<R>(grazing, grazing, grazing)) * c.specular_color;
    if (c.base_metalness > 0) {
        V3<R> metal = c.base_color * c.base_weight;
        V3<R> corr = metal_edge_correction(metal, c.specular_color);
        V3<R> comp = metal_compensation(c, view);
        V3<R> mr = (V3<R>(1, 1, 1) + comp) * c.specular_weight * vmax(metal * m[0] + V3<R>(m[1], m[1], m[1]) - corr * m[2], V3<R>());
        reflected = lerp3(reflected, mr, c.base_metalness);
    }
    V3<R> a = diffuse + reflected;
    return V3<R>(clampr(a.x, R(0), R(1)), clampr(a.y, R(0), R(1)), clampr(a.z, R(0), R(1)));
}

// One camera sample: path_pixel (path.slang:1792-1968) + integrate (:1313-1709) for
// opaque OpenPBR surfaces, analytic lights and a constant environment.  guide (8 values,
// optional): the camera hit's guide albedo + coverage and guide normal + 0, zero on a
// miss or a dropped sample (path.slang:1946-1950).
template <class R> V3<R> integrate(Ctx<R>& cx, uint32_t px, uint32_t py, uint32_t index, uint32_t* ids, R* guide = nullptr) {
    const Scene<R>& s = cx.s;
    const vkb_profile& pf = cx.prof;
    Sampler sm = make_sampler(px, py, index, pf.samples, pf.seed);
    uint32_t rng = screen_ray_hash(px, py, index, pf.seed);
    float cs[4];
    sample_group(sm, 0, cs);
    V3<R> origin, dir; R cam_tmax;
    camera_ray<R>(s.cam, px, py, cs, origin, dir, cam_tmax);
    V3<R> throughput(1, 1, 1), radiance;
    uint32_t ray_event = VKB_RAY_CAMERA, diffuse = 0, glossy = 0, groups = 0;
    R previous_pdf = 0;                                                   // path.slang:1326,1699
    V3<R> previous_world = origin;
    bool nonfinite = false;
    uint64_t dropped = 0;
    const uint32_t B = pf.bounces[0];
    for (uint32_t bounce = 0; bounce <= B; sm.vertex++) {
        R tmax = ray_event == VKB_RAY_CAMERA ? cam_tmax : R(FP32_MAX);
        cx.ext_rays++;
        Hit h = trace(s, origin, dir, tmax, false);
        if (ids && bounce == 0) { ids[0] = h.inst; ids[1] = h.prim; }
        R limit = bounce == 0 ? R(pf.clamp_direct) : R(pf.clamp_indirect);
        if (h.t < 0) {
            V3<R> sky;
            if (ray_event == VKB_RAY_CAMERA && !s.env.camera_sees_environment) sky = V3<R>(s.env.background[0], s.env.background[1], s.env.background[2]);
            else {
                sky = path_environment(s, dir);
                if (ray_event == VKB_RAY_CAMERA)
                    for (const vkb_light& l : s.lights) {
                        LightV<R> L = light_values<R>(l);
                        if (L.kind != 0 || !(L.contribution & VKB_RAY_CAMERA)) continue;
                        sky = sky + emitter_eval(L, V3<R>(), dir).radiance;
                    }
            }
            // path.slang:1463: an escape after a BSDF sample is weighed against the
            // environment strategy.
            const R mis = (s.env_strategy() && previous_pdf > 0) ? mis_power(previous_pdf, environment_density(s, dir)) : R(1);
            radiance = radiance + clamp_sample(throughput * sky * mis, limit, dropped);
            break;
        }
        float sc[4];
        vertex_group(sm, 0, sc);                                          // path_scatter
        HitSurf<R> hs = hit_surface(s, h, dir);
        const vkb_material& mt = s.mats[s.inst_mat[h.inst]];
        Closure<R> c;
        c.base_color = V3<R>(mt.base_color[0], mt.base_color[1], mt.base_color[2]); c.base_weight = mt.base_weight;
        c.base_metalness = mt.base_metalness; c.specular_weight = mt.specular_weight;
        c.specular_color = V3<R>(mt.specular_color[0], mt.specular_color[1], mt.specular_color[2]);
        c.specular_roughness = mt.specular_roughness; c.specular_ior = mt.specular_ior; c.optical_ior = 0;
        c.n = hs.geometric;
        boundary_closure_air(c);
        groups = 0xffffffffu;                                             // objects[].metadata.x: every link group
        V3<R> view = -dir;
        if (guide && bounce == 0) {
            V3<R> a = guide_albedo(c, view);
            guide[0] = a.x; guide[1] = a.y; guide[2] = a.z; guide[3] = 1;
            guide[4] = c.n.x; guide[5] = c.n.y; guide[6] = c.n.z; guide[7] = 0;
        }
        if (material_emits(mt) && ((mt.flags & 2u) || hs.entering)) {
            // Surface emission (path.slang:1580-1591) on the side the material covers,
            // weighed against the mesh strategy after a BSDF sample.
            const V3<R> emitted = V3<R>(mt.emission_color[0], mt.emission_color[1], mt.emission_color[2]) * R(mt.emission_luminance);
            R mis = 1;
            if (previous_pdf > 0) {
                const R area = emitter_geometry(s, h.inst, h.prim, R(0), R(0)).area;
                mis = mis_power(previous_pdf, mesh_pdf(s, h.inst, h.prim, area, previous_world, hs.world, hs.face));
            }
            radiance = radiance + clamp_sample(throughput * emitted * mis, limit, dropped);
        }
        V3<R> iface = dot(hs.geometric, view) > 0 ? hs.geometric : hs.face;
        Prepared<R> pr = transport_prepare(c, view, hs.geometric, iface);
        BsdfSample<R> smp = transport_sample(c, view, R(sc[0]), R(sc[1]), R(sc[2]), pr);
        if (!finite3(smp.dir) || !finite3(smp.weight) || !std::isfinite(smp.pdf)) { nonfinite = true; break; }
        radiance = radiance + clamp_sample(throughput * next_event(cx, hs, c, view, pr, smp, sm, rng, groups), limit, dropped);
        if (s.env_strategy()) {
            // environment_next_event (path.slang:1096-1120): a proposal direction, the
            // diffuse and specular responses MIS-weighted against continuing there
            // (continuation_mask, path.slang:1003-1010), one visibility ray to infinity.
            uint32_t cont = 0;
            if (bounce < B) {
                if (diffuse < pf.bounces[1]) cont |= VKB_RAY_DIFFUSE;
                if (glossy < pf.bounces[2] && (diffuse == 0 || (pf.caustics & 1u))) cont |= VKB_RAY_SPECULAR;
            }
            float eu[4];
            vertex_group(sm, 3, eu);                                      // path_environment
            R epdf = 0;
            const V3<R> edir = env_world(s, env_sample_local(s, eu[0], eu[1], epdf));
            V3<R> env_value;
            if (epdf > 0) {
                for (uint32_t event : {uint32_t(VKB_RAY_DIFFUSE), uint32_t(VKB_RAY_SPECULAR)}) {
                    if (!event_hemisphere(event, edir, hs.face, hs.geometric)) continue;
                    const V3<R> emitted = path_environment(s, edir);
                    if (maxc(emitted) <= 0) continue;
                    const V3<R> response = eval_mask(c, view, edir, event, pr);
                    if (maxc(response) <= 0) continue;
                    const R bsdf_pdf = (cont & event) ? pdf_mask(c, view, edir, event, pr) : R(0);
                    env_value = env_value + emitted * response * (mis_power(epdf, bsdf_pdf) / epdf);
                }
                if (any_nonzero(env_value) && occluded(cx, path_origin(hs, edir), edir, R(FP32_MAX))) env_value = V3<R>();
            }
            radiance = radiance + clamp_sample(throughput * env_value, limit, dropped);
        }
        if (s.mesh_strategy()) {
            // mesh_next_event (path.slang:1121-1167), constant emission: a point on a source
            // triangle, the diffuse and specular responses MIS-weighted against continuing
            // there, one visibility ray between the offset end points; clamped on its own.
            uint32_t cont = 0;
            if (bounce < B) {
                if (diffuse < pf.bounces[1]) cont |= VKB_RAY_DIFFUSE;
                if (glossy < pf.bounces[2] && (diffuse == 0 || (pf.caustics & 1u))) cont |= VKB_RAY_SPECULAR;
            }
            float g[4];
            vertex_group(sm, 2, g);                                       // path_triangle (.zxy)
            const float u[3] = {g[2], g[0], g[1]};
            uint32_t ei, ep; float b1, b2;
            V3<R> mesh_value;
            if (emitter_sample(s, u, ei, ep, b1, b2)) {
                const EmitterGeometry<R> eg = emitter_geometry(s, ei, ep, R(b1), R(b2));
                const V3<R> delta = eg.point - hs.world;
                const R distance = length(delta);
                if (distance > 0) {
                    const V3<R> axis = delta / distance;
                    const R pdf = mesh_pdf(s, ei, ep, eg.area, hs.world, eg.point, eg.face);
                    const vkb_material& em = s.mats[s.inst_mat[ei]];
                    const bool entering = dot(eg.face, axis) < 0;
                    const V3<R> emitted = V3<R>(em.emission_color[0], em.emission_color[1], em.emission_color[2]) * R(em.emission_luminance);
                    if (pdf > 0 && ((em.flags & 2u) || entering) && maxc(emitted) > 0) {
                        const V3<R> start = path_origin(hs, axis);
                        const V3<R> end = surface_ray_origin(eg.point, position_error(s, ei, eg.point), entering ? eg.face : -eg.face, -axis);
                        const V3<R> connection = end - start;
                        const R extent = length(connection);
                        V3<R> response;
                        if (extent > 0)
                            for (uint32_t event : {uint32_t(VKB_RAY_DIFFUSE), uint32_t(VKB_RAY_SPECULAR)}) {
                                if (!event_hemisphere(event, axis, hs.face, hs.geometric)) continue;
                                const V3<R> f = eval_mask(c, view, axis, event, pr);
                                if (maxc(f) <= 0) continue;
                                const R bsdf_pdf = (cont & event) ? pdf_mask(c, view, axis, event, pr) : R(0);
                                response = response + f * mis_power(pdf, bsdf_pdf);
                            }
                        if (any_nonzero(response) && occluded(cx, start, connection / extent, extent)) response = V3<R>();
                        mesh_value = response * emitted / pdf;
                    }
                }
            }
            radiance = radiance + clamp_sample(throughput * mesh_value, limit, dropped);
        }
        if (bounce == B) break;
        uint32_t event = smp.event;
        ray_event = event;
        if (event == VKB_RAY_DIFFUSE) { if (diffuse++ >= pf.bounces[1]) break; }
        else if (event == VKB_RAY_SPECULAR) { if (glossy++ >= pf.bounces[2] || (diffuse > 0 && !(pf.caustics & 1u))) break; }
        else break;
        if (!event_hemisphere(event, smp.dir, hs.face, hs.geometric)) break;
        throughput = throughput * smp.weight;
        if (!finite3(throughput)) { nonfinite = true; break; }
        if (maxc(throughput) <= 0) break;
        if (bounce >= ROULETTE_START) {
            R survive = clampr(maxc(throughput), R(ROULETTE_MIN), R(ROULETTE_MAX));
            float dec[4];
            vertex_group(sm, 4, dec);
            if (R(dec[2]) > survive) break;
            throughput = throughput / survive;
        }
        dir = smp.dir;
        origin = path_origin(hs, dir);
        previous_pdf = smp.pdf;
        previous_world = hs.world;
        bounce++;
    }
    cx.dropped_light += dropped;
    V3<R> result = radiance * R(s.env.exposure);
    if (!finite3(result)) nonfinite = true;
    if (nonfinite) {
        cx.dropped_path++;
        if (guide) for (int k = 0; k < 8; ++k) guide[k] = 0;
        return V3<R>();
    }
    return result;
}

struct OracleScene { void* s32 = nullptr; void* s64 = nullptr; };

// Adaptive stopping (path.slang:1792-1837, 1963-1966), sample-major over the whole image:
// per pixel Welford moments of the RGBA sample values (a dropped sample is zero RGBA),
// settled once every channel's standard error of the mean is within threshold x
// max(|mean|, 0.01) from the minimum sample on, stopped once it and its 3x3
// neighbourhood were settled at the previous sample; a stopped pixel adds its mean to
// the accumulator for the remaining samples.  Arithmetic in float, as the shader's.
template <class R> void render_adaptive(const Scene<R>& s, const vkb_profile& pf, uint32_t w, uint32_t h, float* rgba, uint32_t threads,
                                        uint64_t* stats) {
    const uint32_t n = w * h, count = pf.samples;
    const float thr = pf.adaptive_threshold > 0.f ? pf.adaptive_threshold : 0.01f;
    const uint32_t minimum = pf.adaptive_min_samples ? pf.adaptive_min_samples : std::max(16u, uint32_t(std::sqrt(float(pf.samples))));
    std::vector<float> mean(4 * size_t(n), 0.f), m2(4 * size_t(n), 0.f);
    std::vector<double> sum(3 * size_t(n), 0.0);
    std::vector<uint32_t> state(n, 0u);
    std::vector<uint8_t> skip(n, 0);
    std::mutex mu;
    for (uint32_t i = 0; i < count; ++i) {
        // Decide (reads neighbours' previous parity bit only).
        std::vector<uint32_t> next = state;
        for (uint32_t p = 0; p < n; ++p) {
            uint32_t st = state[p];
            if (st & 4u) { skip[p] = 1; continue; }
            skip[p] = 0;
            bool settled = false;
            if (i >= minimum) {
                const float a1 = float(std::max(i - 1u, 1u)), a2 = float(i);
                settled = true;
                for (int c = 0; c < 4; ++c) {
                    const float e = std::sqrt(std::max(m2[4 * size_t(p) + c] / a1 / a2, 0.f));
                    settled = settled && e <= thr * std::max(std::fabs(mean[4 * size_t(p) + c]), .01f);
                }
            }
            const uint32_t bit = 1u << (i & 1u), prev = 1u << ((i & 1u) ^ 1u);
            bool done = settled;
            const int x = int(p % w), y = int(p / w);
            for (int dy = -1; dy <= 1 && done; ++dy)
                for (int dx = -1; dx <= 1 && done; ++dx) {
                    const int nx = std::min(std::max(x + dx, 0), int(w) - 1), ny = std::min(std::max(y + dy, 0), int(h) - 1);
                    done = (state[size_t(ny) * w + size_t(nx)] & prev) != 0u;
                }
            st = settled ? (st | bit) : (st & ~bit);
            if (done) { st |= 4u; skip[p] = 1; }
            next[p] = st;
        }
        state.swap(next);
        // Trace the live pixels of this sample.
        std::atomic<uint32_t> row{0};
        auto work = [&] {
            Ctx<R> cx{s, pf};
            for (uint32_t y; (y = row.fetch_add(1)) < h;)
                for (uint32_t x = 0; x < w; ++x) {
                    const size_t p = size_t(y) * w + x;
                    float* m = &mean[4 * p];
                    if (skip[p]) { for (int c = 0; c < 3; ++c) sum[3 * p + c] += m[c]; continue; }
                    const uint64_t before = cx.dropped_path;
                    const V3<R> v = integrate(cx, x, y, i, nullptr);
                    const float val[4] = {float(v.x), float(v.y), float(v.z), cx.dropped_path != before ? 0.f : 1.f};
                    for (int c = 0; c < 3; ++c) sum[3 * p + c] += val[c];
                    float* q = &m2[4 * p];
                    const float inv = 1.f / float(i + 1u);
                    for (int c = 0; c < 4; ++c) {
                        const float d = val[c] - m[c];
                        m[c] = m[c] + d * inv;
                        q[c] += d * (val[c] - m[c]);
                    }
                }
            std::lock_guard<std::mutex> g(mu);
            if (stats) { stats[0] += cx.ext_rays; stats[1] += cx.shadow_rays; stats[2] += cx.dropped_path; stats[3] += cx.dropped_light; }
        };
        if (threads <= 1) work();
        else {
            std::vector<std::thread> ts;
            for (uint32_t t = 0; t < threads; ++t) ts.emplace_back(work);
            for (auto& t : ts) t.join();
        }
    }
    for (uint32_t p = 0; p < n; ++p) {
        float* o = rgba + 4 * size_t(p);
        for (int c = 0; c < 3; ++c) o[c] = float(sum[3 * size_t(p) + c] / double(count));
        o[3] = 1.f;
    }
}

template <class R> void render_impl(const Scene<R>& s, const vkb_profile& pf, uint32_t x0, uint32_t y0, uint32_t w, uint32_t h,
                                    float* rgba, uint32_t* ids, uint32_t threads, uint64_t* stats, float* guides = nullptr) {
    if (pf.adaptive) {
        // Whole image, whole exposure: the stop rule reads image-edge-clamped neighbours.
        if (x0 != 0 || y0 != 0 || w != s.cam.width || h != s.cam.height || pf.first_sample != 0 ||
            (pf.sample_count && pf.sample_count != pf.samples))
        {   // refused (pyoracle checks first): the image reads NaN
            for (size_t k = 0; k < size_t(w) * h * 4; ++k) rgba[k] = std::numeric_limits<float>::quiet_NaN();
            return;
        }
        render_adaptive(s, pf, w, h, rgba, threads, stats);
        return;
    }
    uint32_t first = pf.first_sample, count = pf.sample_count ? pf.sample_count : pf.samples - pf.first_sample;
    std::atomic<uint32_t> next{0};
    std::mutex mu;
    auto work = [&] {
        Ctx<R> cx{s, pf};
        for (uint32_t row; (row = next.fetch_add(1)) < h;) {
            for (uint32_t x = 0; x < w; ++x) {
                V3<R> sum;
                R gsum[8] = {0, 0, 0, 0, 0, 0, 0, 0};
                uint32_t* pid = ids ? ids + (size_t(row) * w + x) * 2 : nullptr;
                for (uint32_t k = 0; k < count; ++k) {
                    R g[8] = {0, 0, 0, 0, 0, 0, 0, 0};
                    sum = sum + integrate(cx, x0 + x, y0 + row, first + k, k == 0 ? pid : nullptr, guides ? g : nullptr);
                    for (int c = 0; c < 8; ++c) gsum[c] += g[c];
                }
                float* o = rgba + (size_t(row) * w + x) * 4;
                o[0] = float(sum.x / R(count)); o[1] = float(sum.y / R(count)); o[2] = float(sum.z / R(count)); o[3] = 1.f;
                if (guides)
                    for (int c = 0; c < 8; ++c) guides[(size_t(row) * w + x) * 8 + c] = float(gsum[c] / R(count));
            }
        }
        std::lock_guard<std::mutex> g(mu);
        if (stats) { stats[0] += cx.ext_rays; stats[1] += cx.shadow_rays; stats[2] += cx.dropped_path; stats[3] += cx.dropped_light; }
    };
    if (threads <= 1) work();
    else {
        std::vector<std::thread> ts;
        for (uint32_t i = 0; i < threads; ++i) ts.emplace_back(work);
        for (auto& t : ts) t.join();
    }
}

// ---------------------------------------------------------------- Morton codes (fp32, no contraction: bit-exact restatement)
inline uint32_t expand_bits(uint32_t v) {
    v = (v * 0x00010001u) & 0xFF0000FFu;
    v = (v * 0x00000101u) & 0x0F00F00Fu;
    v = (v * 0x00000011u) & 0xC30C30C3u;
    v = (v * 0x00000005u) & 0x49249249u;
    return v;
}
inline uint32_t quantize10(float x) {
    float q = x * 1024.f;
    q = q < 0.f ? 0.f : q;
    q = q > 1023.f ? 1023.f : q;
    return uint32_t(q);
}
inline uint32_t morton3(const float c[3], const float lo[3], const float ext[3]) {
    uint32_t q[3];
    for (int a = 0; a < 3; ++a) {
        float n = ext[a] > 0.f ? (c[a] - lo[a]) / ext[a] : 0.5f;
        q[a] = quantize10(n);
    }
    return (expand_bits(q[0]) << 2) | (expand_bits(q[1]) << 1) | expand_bits(q[2]);
}
// split_large: bit 30 over the code of a box wider on some axis than a quarter of the
// centroid box's widest extent (the TLAS build's root split).
void box_morton(uint32_t n, const float* lo, const float* hi, uint32_t* out, bool split_large = false) {
    float slo[3] = {INFINITY, INFINITY, INFINITY}, shi[3] = {-INFINITY, -INFINITY, -INFINITY};
    for (uint32_t i = 0; i < n; ++i)
        for (int a = 0; a < 3; ++a) {
            float c = (lo[3 * i + a] + hi[3 * i + a]) * 0.5f;
            slo[a] = std::min(slo[a], c); shi[a] = std::max(shi[a], c);
        }
    float ext[3] = {shi[0] - slo[0], shi[1] - slo[1], shi[2] - slo[2]};
    const float big = std::max(ext[0], std::max(ext[1], ext[2])) * 0.25f;
    for (uint32_t i = 0; i < n; ++i) {
        float c[3];
        for (int a = 0; a < 3; ++a) c[a] = (lo[3 * i + a] + hi[3 * i + a]) * 0.5f;
        const float w = std::max(hi[3 * i] - lo[3 * i], std::max(hi[3 * i + 1] - lo[3 * i + 1], hi[3 * i + 2] - lo[3 * i + 2]));
        out[i] = morton3(c, slo, ext) | (split_large && w > big ? 1u << 30 : 0u);
    }
}
// World box of an instance: the 8 transformed corners of its mesh box, each
// component ((m0*x + m1*y) + m2*z) + m3 in fp32, intersected with the box of the
// transformed bounding sphere (centre ((m0*cx + m1*cy) + m2*cz) + m3, half extent
// r * sqrt((m0*m0 + m1*m1) + m2*m2) widened by 1e-5 relative plus 1e-6 of
// (|centre| + |m3| + extent)); sph[3] < 0 means no sphere.
void instance_box(const float* rows, const float mlo[3], const float mhi[3], const float sph[4], float lo[3], float hi[3]) {
    for (int a = 0; a < 3; ++a) { lo[a] = INFINITY; hi[a] = -INFINITY; }
    for (int k = 0; k < 8; ++k) {
        float p[3] = {k & 1 ? mhi[0] : mlo[0], k & 2 ? mhi[1] : mlo[1], k & 4 ? mhi[2] : mlo[2]};
        for (int a = 0; a < 3; ++a) {
            float v = rows[4 * a] * p[0];
            v = v + rows[4 * a + 1] * p[1];
            v = v + rows[4 * a + 2] * p[2];
            v = v + rows[4 * a + 3];
            lo[a] = std::min(lo[a], v); hi[a] = std::max(hi[a], v);
        }
    }
    if (sph[3] >= 0.f) {
        for (int a = 0; a < 3; ++a) {
            const float* m = rows + 4 * a;
            float cw = m[0] * sph[0];
            cw = cw + m[1] * sph[1];
            cw = cw + m[2] * sph[2];
            cw = cw + m[3];
            float nn = m[0] * m[0];
            nn = nn + m[1] * m[1];
            nn = nn + m[2] * m[2];
            const float ext = sph[3] * std::sqrt(nn);
            const float mag = (std::fabs(cw) + std::fabs(m[3])) + ext;
            const float half = ext * 1.00001f + mag * 1e-6f;
            lo[a] = std::max(lo[a], cw - half);
            hi[a] = std::min(hi[a], cw + half);
        }
    }
}
// Box and bounding sphere (about the box centre, radius = largest vertex distance in
// f64 rounded up to fp32; radius -1 without vertices) of a mesh.
void mesh_box(const vkb_mesh& m, float lo[3], float hi[3], float sph[4]) {
    for (int a = 0; a < 3; ++a) { lo[a] = INFINITY; hi[a] = -INFINITY; }
    for (uint32_t i = 0; i < m.num_vertices; ++i)
        for (int a = 0; a < 3; ++a) { lo[a] = std::min(lo[a], m.positions[3 * i + a]); hi[a] = std::max(hi[a], m.positions[3 * i + a]); }
    if (m.num_vertices == 0) { sph[0] = sph[1] = sph[2] = 0.f; sph[3] = -1.f; return; }
    float c[3];
    for (int a = 0; a < 3; ++a) c[a] = 0.5f * (lo[a] + hi[a]);
    double r2 = 0.0;
    for (uint32_t i = 0; i < m.num_vertices; ++i) {
        double dx = double(m.positions[3 * i]) - c[0], dy = double(m.positions[3 * i + 1]) - c[1], dz = double(m.positions[3 * i + 2]) - c[2];
        r2 = std::max(r2, dx * dx + dy * dy + dz * dz);
    }
    sph[0] = c[0]; sph[1] = c[1]; sph[2] = c[2];
    sph[3] = std::nextafter(float(std::sqrt(r2)), INFINITY);
}

}  // namespace

// Replace the atlas both precisions read with `texels` (BRDF_SIZE x BRDF_HEIGHT x 4
// floats, e.g. the device bake) so a transport comparison does not also measure the
// bake; NULL restores the oracle's own bake.
template <class R> void set_lut(const float* texels) {
    Lut<R>& l = lut_mut<R>();
    std::vector<float>& b = lut_baked<R>();
    if (texels) {
        if (b.empty()) b = l.texels;
        std::copy(texels, texels + l.texels.size(), l.texels.begin());
    } else if (!b.empty()) {
        l.texels = b;
        b.clear();
    }
}

extern "C" {

uint32_t oracle_version(void) { return 1u; }

// Sampler bits: mode 0 the shader recurrence, 1 the table form of path_sampler.rs.
void oracle_sampler_bits(uint32_t n, const uint32_t* px, const uint32_t* py, const uint32_t* index, const uint32_t* groups,
                         uint32_t count, uint32_t stream, uint32_t* out, int mode) {
    for (uint32_t i = 0; i < n; ++i) {
        Sampler s = make_sampler(px[i], py[i], index[i], count, stream);
        if (mode == 0) group_bits_recurrence(s, groups[i], out + 4 * i);
        else group_bits_table(s, groups[i], out + 4 * i);
    }
}
void oracle_sobol_directions(uint32_t* out) {
    const SobolTable& t = sobol_table();
    for (int d = 0; d < 3; ++d) for (int k = 0; k < 32; ++k) out[32 * d + k] = t.d[d][k];
}
// Unscrambled Sobol fractions of dimensions 0-3 (path_sampler.rs:71-79).
void oracle_sobol_points(uint32_t n, uint32_t* out) {
    const SobolTable& t = sobol_table();
    for (uint32_t i = 0; i < n; ++i) {
        uint32_t x[4] = {rev(i), 0, 0, 0};
        for (int k = 0; k < 32; ++k) if ((i >> k) & 1u) for (int d = 0; d < 3; ++d) x[d + 1] ^= t.d[d][k];
        for (int c = 0; c < 4; ++c) out[4 * i + c] = x[c];
    }
}
void oracle_filter_table(float* out) { const std::vector<float>& t = filter_table(); std::copy(t.begin(), t.end(), out); }
double oracle_filter_cdf(double x) { return path_filter_cdf(x); }
void oracle_brdf_lut(int fp64, float* out) {
    if (fp64) { const Lut<double>& l = lut<double>(); std::copy(l.texels.begin(), l.texels.end(), out); }
    else { const Lut<float>& l = lut<float>(); std::copy(l.texels.begin(), l.texels.end(), out); }
}
float oracle_half_round(float x) { return half_to_float(float_to_half(x)); }
void oracle_set_lut(const float* texels) { set_lut<float>(texels); set_lut<double>(texels); }
// Emitter evaluation (for the reference's light_connection_tests invariants).
void oracle_emitter_sample(const vkb_light* light, const double* world, const double* u, double* out_dir, double* out_radiance, double* out_pdf, double* out_distance) {
    LightV<double> L = light_values<double>(*light);
    LightSample<double> s = emitter_sample(L, V3<double>(world[0], world[1], world[2]), u[0], u[1]);
    out_dir[0] = s.dir.x; out_dir[1] = s.dir.y; out_dir[2] = s.dir.z;
    out_radiance[0] = s.radiance.x; out_radiance[1] = s.radiance.y; out_radiance[2] = s.radiance.z;
    *out_pdf = s.pdf; *out_distance = s.distance;
}
void oracle_emitter_eval(const vkb_light* light, const double* world, const double* dir, double* out_radiance, double* out_pdf, double* out_distance) {
    LightV<double> L = light_values<double>(*light);
    EmitterEval<double> e = emitter_eval(L, V3<double>(world[0], world[1], world[2]), V3<double>(dir[0], dir[1], dir[2]));
    out_radiance[0] = e.radiance.x; out_radiance[1] = e.radiance.y; out_radiance[2] = e.radiance.z;
    *out_pdf = e.pdf; *out_distance = e.distance;
}
// BSDF sample/eval/pdf on a bare closure (normal +z), for direct checks.
void oracle_bsdf(const vkb_material* m, const double* view, const double* u3, double* out_dir, double* out_weight, double* out_pdf, uint32_t* out_event) {
    Closure<double> c;
    c.base_color = V3<double>(m->base_color[0], m->base_color[1], m->base_color[2]); c.base_weight = m->base_weight;
    c.base_metalness = m->base_metalness; c.specular_weight = m->specular_weight;
    c.specular_color = V3<double>(m->specular_color[0], m->specular_color[1], m->specular_color[2]);
    c.specular_roughness = m->specular_roughness; c.specular_ior = m->specular_ior; c.optical_ior = 0; c.n = V3<double>(0, 0, 1);
    boundary_closure_air(c);
    V3<double> v(view[0], view[1], view[2]);
    Prepared<double> pr = transport_prepare(c, v, c.n, c.n);
    BsdfSample<double> s = transport_sample(c, v, u3[0], u3[1], u3[2], pr);
    out_dir[0] = s.dir.x; out_dir[1] = s.dir.y; out_dir[2] = s.dir.z;
    out_weight[0] = s.weight.x; out_weight[1] = s.weight.y; out_weight[2] = s.weight.z;
    *out_pdf = s.pdf; *out_event = s.event;
}

// precisions: bit 0 builds the FP32 restatement, bit 1 the FP64 one.
void* oracle_scene_create(const vkb_scene_desc* d, int precisions) {
    OracleScene* o = new OracleScene();
    if (precisions & 1) o->s32 = make_scene<float>(d);
    if (precisions & 2) o->s64 = make_scene<double>(d);
    return o;
}
void oracle_scene_destroy(void* h) {
    OracleScene* o = static_cast<OracleScene*>(h);
    delete static_cast<Scene<float>*>(o->s32);
    delete static_cast<Scene<double>*>(o->s64);
    delete o;
}
// Closest (any=0) or any (any=1) hits of world rays (origin, dir, tmax).
void oracle_trace(void* h, int fp64, uint32_t n, const float* rays7, int any, float* out_t, uint32_t* out_ids, float* out_uv) {
    OracleScene* o = static_cast<OracleScene*>(h);
    for (uint32_t i = 0; i < n; ++i) {
        const float* r = rays7 + 7 * i;
        Hit hit;
        if (fp64) hit = trace(*static_cast<Scene<double>*>(o->s64), V3<double>(r[0], r[1], r[2]), V3<double>(r[3], r[4], r[5]), double(r[6]), any != 0);
        else hit = trace(*static_cast<Scene<float>*>(o->s32), V3<float>(r[0], r[1], r[2]), V3<float>(r[3], r[4], r[5]), r[6], any != 0);
        out_t[i] = float(hit.t); out_ids[2 * i] = hit.inst; out_ids[2 * i + 1] = hit.prim;
        out_uv[2 * i] = float(hit.u); out_uv[2 * i + 1] = float(hit.v);
    }
}
// Image environment probes: n proposal samples (u2 pairs) -> world directions and pdfs;
// the proposal pdf and the radiance of n world directions.
void oracle_env_sample(void* h, int fp64, uint32_t n, const float* u2, float* dir3, float* pdf) {
    OracleScene* o = static_cast<OracleScene*>(h);
    for (uint32_t i = 0; i < n; ++i) {
        if (fp64) {
            const Scene<double>& s = *static_cast<Scene<double>*>(o->s64);
            double p; V3<double> d = env_world(s, env_sample_local(s, u2[2 * i], u2[2 * i + 1], p));
            dir3[3 * i] = float(d.x); dir3[3 * i + 1] = float(d.y); dir3[3 * i + 2] = float(d.z); pdf[i] = float(p);
        } else {
            const Scene<float>& s = *static_cast<Scene<float>*>(o->s32);
            float p; V3<float> d = env_world(s, env_sample_local(s, u2[2 * i], u2[2 * i + 1], p));
            dir3[3 * i] = d.x; dir3[3 * i + 1] = d.y; dir3[3 * i + 2] = d.z; pdf[i] = p;
        }
    }
}
// Emissive-mesh proposal of the fp32 scene: the weight tree (2 x leaves floats), source
// samples (instance, primitive, barycentrics, probability) and triangle probabilities.
uint32_t oracle_mesh_tree(void* h, float* out) {
    const Scene<float>& s = *static_cast<Scene<float>*>(static_cast<OracleScene*>(h)->s32);
    if (out) std::copy(s.em_tree.begin(), s.em_tree.end(), out);
    return s.em_leaves;
}
uint32_t oracle_mesh_triangles(void* h) { return static_cast<Scene<float>*>(static_cast<OracleScene*>(h)->s32)->em_tris; }
void oracle_mesh_sample(void* h, uint32_t n, const float* u3, uint32_t* inst, uint32_t* prim, float* bary2, float* probability) {
    const Scene<float>& s = *static_cast<Scene<float>*>(static_cast<OracleScene*>(h)->s32);
    for (uint32_t i = 0; i < n; ++i) {
        uint32_t a = 0xffffffffu, b = 0xffffffffu; float b1 = 0.f, b2 = 0.f;
        const bool ok = s.mesh_strategy() && emitter_sample(s, u3 + 3 * i, a, b, b1, b2);
        inst[i] = a; prim[i] = b; bary2[2 * i] = b1; bary2[2 * i + 1] = b2;
        probability[i] = ok ? emitter_probability(s, a, b) : 0.f;
    }
}
void oracle_mesh_probability(void* h, uint32_t n, const uint32_t* inst, const uint32_t* prim, float* out) {
    const Scene<float>& s = *static_cast<Scene<float>*>(static_cast<OracleScene*>(h)->s32);
    for (uint32_t i = 0; i < n; ++i) out[i] = emitter_probability(s, inst[i], prim[i]);
}
void oracle_env_eval(void* h, uint32_t n, const float* dir3, float* pdf, float* rgb) {
    const Scene<double>& s = *static_cast<Scene<double>*>(static_cast<OracleScene*>(h)->s64);
    for (uint32_t i = 0; i < n; ++i) {
        V3<double> d = normalize(V3<double>(dir3[3 * i], dir3[3 * i + 1], dir3[3 * i + 2]));
        if (pdf) pdf[i] = float(environment_density(s, d));
        V3<double> r = path_environment(s, d);
        rgb[3 * i] = float(r.x); rgb[3 * i + 1] = float(r.y); rgb[3 * i + 2] = float(r.z);
    }
}
// Camera rays of sample `index` for a crop, as path_camera_ray builds them (rays7 layout).
void oracle_camera_rays(void* h, const vkb_profile* pf, uint32_t index, uint32_t x0, uint32_t y0, uint32_t w, uint32_t hgt, float* rays7) {
    OracleScene* o = static_cast<OracleScene*>(h);
    const Scene<double>& s = *static_cast<Scene<double>*>(o->s64);
    for (uint32_t y = 0; y < hgt; ++y)
        for (uint32_t x = 0; x < w; ++x) {
            Sampler sm = make_sampler(x0 + x, y0 + y, index, pf->samples, pf->seed);
            float cs[4];
            sample_group(sm, 0, cs);
            V3<double> org, dir; double tmax;
            camera_ray<double>(s.cam, x0 + x, y0 + y, cs, org, dir, tmax);
            float* r = rays7 + 7 * (size_t(y) * w + x);
            r[0] = float(org.x); r[1] = float(org.y); r[2] = float(org.z);
            r[3] = float(dir.x); r[4] = float(dir.y); r[5] = float(dir.z); r[6] = float(tmax);
        }
}
// Render a crop. stats (optional, 4 u64): extension rays, shadow rays, dropped path samples, dropped light samples.
// guides (optional, w*hgt*8): per pixel the mean guide albedo + coverage and the mean
// guide normal + 0 over the rendered samples.
void oracle_render(void* h, int fp64, const vkb_profile* pf, uint32_t x0, uint32_t y0, uint32_t w, uint32_t hgt,
                   float* rgba, uint32_t* ids, uint32_t threads, uint64_t* stats, float* guides) {
    OracleScene* o = static_cast<OracleScene*>(h);
    if (guides && pf->adaptive) {   // refused (pyoracle checks first): guides read NaN
        for (size_t k = 0; k < size_t(w) * hgt * 8; ++k) guides[k] = std::numeric_limits<float>::quiet_NaN();
        guides = nullptr;
    }
    if (fp64) render_impl(*static_cast<Scene<double>*>(o->s64), *pf, x0, y0, w, hgt, rgba, ids, threads, stats, guides);
    else render_impl(*static_cast<Scene<float>*>(o->s32), *pf, x0, y0, w, hgt, rgba, ids, threads, stats, guides);
}
// Morton codes of the TLAS build (instance boxes) and of one mesh's BLAS build (triangle boxes).
// World boxes of the TLAS leaves (xyz lo, xyz hi per instance), as the build computes them.
void oracle_instance_boxes(const vkb_scene_desc* d, float* lo, float* hi) {
    std::vector<float> mlo(3 * size_t(d->num_meshes)), mhi(3 * size_t(d->num_meshes)), msph(4 * size_t(d->num_meshes));
    for (uint32_t m = 0; m < d->num_meshes; ++m) mesh_box(d->meshes[m], &mlo[3 * m], &mhi[3 * m], &msph[4 * m]);
    for (uint32_t i = 0; i < d->num_instances; ++i) {
        uint32_t m = d->instance_mesh[i];
        instance_box(d->instance_rows + 12 * size_t(i), &mlo[3 * m], &mhi[3 * m], &msph[4 * m], &lo[3 * i], &hi[3 * i]);
    }
}
void oracle_tlas_morton(const vkb_scene_desc* d, uint32_t* out) {
    std::vector<float> lo(3 * size_t(d->num_instances)), hi(3 * size_t(d->num_instances));
    oracle_instance_boxes(d, lo.data(), hi.data());
    box_morton(d->num_instances, lo.data(), hi.data(), out, true);
}
void oracle_blas_morton(const vkb_scene_desc* d, uint32_t mesh, uint32_t* out) {
    const vkb_mesh& m = d->meshes[mesh];
    std::vector<float> lo(3 * size_t(m.num_triangles)), hi(3 * size_t(m.num_triangles));
    for (uint32_t t = 0; t < m.num_triangles; ++t)
        for (int a = 0; a < 3; ++a) {
            float v0 = m.positions[3 * m.indices[3 * t] + a], v1 = m.positions[3 * m.indices[3 * t + 1] + a], v2 = m.positions[3 * m.indices[3 * t + 2] + a];
            lo[3 * t + a] = std::min(v0, std::min(v1, v2)); hi[3 * t + a] = std::max(v0, std::max(v1, v2));
        }
    box_morton(m.num_triangles, lo.data(), hi.data(), out);
}

}  // extern "C"
