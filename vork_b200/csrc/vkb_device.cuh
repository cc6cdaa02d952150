// Device-side path math for the B200 backend: hashing + Owen-scrambled Sobol sampler,
// OpenPBR 1.1.1 subset (Lambert with dielectric-albedo compensation, GGX VNDF, F82
// metal with multiple-scattering compensation), analytic emitters, light-tree pick,
// hit reconstruction and PBRT-style ray origins.  Every function cites the reference
// shader it restates; the subset (opaque, no coat/fuzz/film/transmission/subsurface)
// is what the std/path configurations install.
#pragma once
#include <cstdint>
#include <cuda_fp16.h>
#include "../../include/vkb.h"

namespace vkb {

// crates/vork-slang/src/registry.rs:89,351,375-391; renderer_registry.rs:98-111,367.
constexpr uint32_t SAMPLE_HASH_MIX = 0x45d9f3bu;
constexpr uint32_t PIXEL_HASH_STREAM_STEP = 0x9e3779b9u;
constexpr uint32_t FILTER_INTERVALS = 1024;
constexpr uint32_t BRDF_SIZE = 128, BRDF_ALBEDO_SIZE = 64, BRDF_IOR_STEPS = 64;
constexpr uint32_t BRDF_HEIGHT = BRDF_SIZE + ((BRDF_IOR_STEPS + 2) / 2) * BRDF_ALBEDO_SIZE;
constexpr uint32_t ENVIRONMENT_SAMPLES = 512, DIELECTRIC_ALBEDO_SAMPLES = 512;
constexpr float PI_F = 3.14159265358979323846f, TAU_F = 6.28318530717958647692f;
constexpr float MIN_ALPHA = 0.0001f;
constexpr float UINT_SCALE = 0.000000059604644775390625f;
constexpr float RADICAL_INVERSE_SCALE = 2.3283064365386963e-10f;
constexpr float POSITIVE_EPSILON = 1e-20f;
constexpr float FP32_MAX = 3.402823466e38f;
constexpr float FP32_EPS = 1.1920928955078125e-07f;
constexpr uint32_t ROULETTE_START = 3;
constexpr float ROULETTE_MIN = 0.05f, ROULETTE_MAX = 0.95f;
constexpr float LIGHT_TREE_UNIFORM_MIX = 0.25f;
constexpr float LIGHT_TREE_MIN_DISTANCE_SQUARED = 1e-12f;
constexpr float LUM_R = 0.2126f, LUM_G = 0.7152f, LUM_B = 0.0722f;
__host__ __device__ constexpr float fp32_gamma7() { return (7.f * (FP32_EPS * 0.5f)) / (1.f - 7.f * (FP32_EPS * 0.5f)); }

// ---------------------------------------------------------------- float3 helpers
__device__ __forceinline__ float3 f3(float a, float b, float c) { return make_float3(a, b, c); }
__device__ __forceinline__ float3 f3(float a) { return make_float3(a, a, a); }
__device__ __forceinline__ float3 operator+(float3 a, float3 b) { return f3(a.x + b.x, a.y + b.y, a.z + b.z); }
__device__ __forceinline__ float3 operator-(float3 a, float3 b) { return f3(a.x - b.x, a.y - b.y, a.z - b.z); }
__device__ __forceinline__ float3 operator-(float3 a) { return f3(-a.x, -a.y, -a.z); }
__device__ __forceinline__ float3 operator*(float3 a, float3 b) { return f3(a.x * b.x, a.y * b.y, a.z * b.z); }
__device__ __forceinline__ float3 operator*(float3 a, float s) { return f3(a.x * s, a.y * s, a.z * s); }
__device__ __forceinline__ float3 operator*(float s, float3 a) { return f3(a.x * s, a.y * s, a.z * s); }
__device__ __forceinline__ float3 operator/(float3 a, float s) { return f3(a.x / s, a.y / s, a.z / s); }
__device__ __forceinline__ float dot(float3 a, float3 b) { return a.x * b.x + a.y * b.y + a.z * b.z; }
__device__ __forceinline__ float3 cross(float3 a, float3 b) { return f3(a.y * b.z - a.z * b.y, a.z * b.x - a.x * b.z, a.x * b.y - a.y * b.x); }
__device__ __forceinline__ float length(float3 a) { return sqrtf(dot(a, a)); }
__device__ __forceinline__ float3 normalize(float3 a) { return a / length(a); }
__device__ __forceinline__ float3 vabs(float3 a) { return f3(fabsf(a.x), fabsf(a.y), fabsf(a.z)); }
__device__ __forceinline__ float3 vmax(float3 a, float3 b) { return f3(fmaxf(a.x, b.x), fmaxf(a.y, b.y), fmaxf(a.z, b.z)); }
__device__ __forceinline__ float3 vmin(float3 a, float3 b) { return f3(fminf(a.x, b.x), fminf(a.y, b.y), fminf(a.z, b.z)); }
__device__ __forceinline__ float maxc(float3 a) { return fmaxf(a.x, fmaxf(a.y, a.z)); }
__device__ __forceinline__ bool finite3(float3 a) { return isfinite(a.x) && isfinite(a.y) && isfinite(a.z); }
__device__ __forceinline__ bool any_pos(float3 a) { return a.x > 0.f || a.y > 0.f || a.z > 0.f; }
__device__ __forceinline__ bool any_nonzero(float3 a) { return a.x != 0.f || a.y != 0.f || a.z != 0.f; }
__device__ __forceinline__ float lerpf(float a, float b, float t) { return a + (b - a) * t; }
__device__ __forceinline__ float3 lerp3(float3 a, float3 b, float t) { return a + (b - a) * t; }
__device__ __forceinline__ float clampf(float x, float a, float b) { return fminf(fmaxf(x, a), b); }
__device__ __forceinline__ float saturatef(float x) { return clampf(x, 0.f, 1.f); }
__device__ __forceinline__ float lum(float3 c) { return c.x * LUM_R + c.y * LUM_G + c.z * LUM_B; }
__device__ __forceinline__ float3 reflect(float3 i, float3 n) { return i - n * (2.f * dot(n, i)); }
__device__ __forceinline__ float3 get3(const float* p) { return f3(p[0], p[1], p[2]); }
// stream.slang:416-427.
__device__ __forceinline__ float3 finite_unit_normal(float3 n, float3 fallback) {
    float s = maxc(vabs(n));
    if (finite3(n) && s > 0.f) return normalize(n / s);
    float fs = maxc(vabs(fallback));
    if (finite3(fallback) && fs > 0.f) return normalize(fallback / fs);
    return f3(0.f, 0.f, 1.f);
}
// orthonormal_basis.slang (Duff et al. 2017).
__device__ __forceinline__ float3 basis_direction(float3 n, float3 v) {
    float s = n.z >= 0.f ? 1.f : -1.f;
    float a = -1.f / (s + n.z);
    float b = n.x * n.y * a;
    float3 r0 = f3(1.f + s * n.x * n.x * a, s * b, -s * n.x);
    float3 r1 = f3(b, s + n.y * n.y * a, -n.y);
    return r0 * v.x + r1 * v.y + n * v.z;
}
// vork_prelude.slang screen_next_float: the adjacent float toward +/- infinity.
__device__ __forceinline__ float next_float(float v, bool up) {
    if (v == 0.f) return __uint_as_float(up ? 1u : 0x80000001u);
    bool increasing = (v > 0.f) == up;
    return __uint_as_float(__float_as_uint(v) + (increasing ? 1u : 0xffffffffu));
}

// ---------------------------------------------------------------- hashes + sampler (bit-exact)
// crates/vork-slang/src/vork_sampling.slang:3-15.
__device__ __forceinline__ uint32_t pixel_hash(uint32_t s) {
    uint32_t v = (s ^ (s >> 16)) * SAMPLE_HASH_MIX;
    v = (v ^ (v >> 16)) * SAMPLE_HASH_MIX;
    return v ^ (v >> 16);
}
__device__ __forceinline__ uint32_t screen_ray_hash(uint32_t px, uint32_t py, uint32_t index, uint32_t stream) {
    uint32_t spatial = pixel_hash((px * SAMPLE_HASH_MIX) ^ py);
    return pixel_hash(spatial ^ pixel_hash(index * PIXEL_HASH_STREAM_STEP + stream));
}
// path_sampler.slang:65-68 (Laine-Karras hash of a bit-reversed integer).
__device__ __forceinline__ uint32_t owen_reversed(uint32_t x, uint32_t seed) {
    seed = pixel_hash(seed);
    x ^= x * 0x3d20adeau;
    x += seed;
    x *= (seed >> 16) | 1u;
    x ^= x * 0x05526c56u;
    x ^= x * 0x53a22864u;
    return x;
}
__device__ __forceinline__ float sample_unit(uint32_t x) { return (float(x >> 9) + 0.5f) * (1.f / 8388608.f); }
// path_sampler.slang:52-59.
__device__ __forceinline__ uint32_t sample_mask(uint32_t count) {
    return count <= 1u ? 0u : (2u << (31 - __clz(count - 1u))) - 1u;
}
// path_sampler.slang:74-95: the four scrambled 32-bit fractions of one group.
__device__ __forceinline__ uint4 sample_group_bits(uint32_t pixel_seed, uint32_t index, uint32_t mask, uint32_t group) {
    uint32_t seed = pixel_hash(pixel_seed ^ pixel_hash(group + 1u));
    uint32_t idx = __brev(owen_reversed(__brev(index), seed ^ 0x6c8e9cf5u)) & mask;
    uint32_t x0 = 0, x1 = 0, x2 = 0, p = 0x80000000u;
    uint32_t qx = 0x80000000u, qy = 0xc0000000u;
    uint32_t rx = 0x80000000u, ry = 0xc0000000u, rz = 0x20000000u;
    for (uint32_t bits = idx; bits != 0u; bits >>= 1) {
        if (bits & 1u) { x0 ^= p; x1 ^= qx; x2 ^= rx; }
        p ^= p >> 1;
        uint32_t nqy = qy ^ qx ^ (qx >> 2);
        qx = qy; qy = nqy;
        uint32_t nrz = ry ^ rx ^ (rx >> 3);
        rx = ry; ry = rz; rz = nrz;
    }
    return make_uint4(__brev(owen_reversed(idx, seed ^ 0xa511e9b3u)), __brev(owen_reversed(__brev(x0), seed ^ 0x63d83595u)),
                      __brev(owen_reversed(__brev(x1), seed ^ 0x2f7c4a1bu)), __brev(owen_reversed(__brev(x2), seed ^ PIXEL_HASH_STREAM_STEP)));
}
__device__ __forceinline__ float4 sample_group(uint32_t pixel_seed, uint32_t index, uint32_t mask, uint32_t group) {
    uint4 b = sample_group_bits(pixel_seed, index, mask, group);
    return make_float4(sample_unit(b.x), sample_unit(b.y), sample_unit(b.z), sample_unit(b.w));
}
// Group 0 camera; vertex v owns groups 1+5v .. 5+5v (path_sampler.slang:96-112).
__device__ __forceinline__ uint32_t vertex_group(uint32_t vertex, uint32_t slot) { return 1u + vertex * 5u + slot; }
// path_sampler.slang:73.
__device__ __forceinline__ float path_random(uint32_t& state) { state = pixel_hash(state + PIXEL_HASH_STREAM_STEP); return sample_unit(state); }

// ---------------------------------------------------------------- OpenPBR core (libraries/std/openpbr_core.slang)
__device__ __forceinline__ float specular_alpha(float r) { return fmaxf(r * r, MIN_ALPHA); }
__device__ __forceinline__ float modulated_ior(float eta, float weight) {
    if (weight == 1.f || eta == 1.f) return eta;
    float contrast = (eta - 1.f) / (eta + 1.f);
    const float limit = __uint_as_float(0x3f7fffffu);
    float e = clampf(sqrtf(fmaxf(weight, 0.f)) * contrast, -limit, limit);
    return (1.f + e) / (1.f - e);
}
__device__ __forceinline__ float fresnel(float c, float eta) {
    c = clampf(c, 0.f, 1.f);
    if (eta == 1.f) return 0.f;
    float si2 = (1.f - c * c) / (eta * eta);
    if (si2 >= 1.f) return 1.f;
    float ct = sqrtf(fmaxf(0.f, 1.f - si2));
    float rs = (c - eta * ct) / (c + eta * ct), rp = (eta * c - ct) / (eta * c + ct);
    return (rs * rs + rp * rp) * 0.5f;
}
__device__ __forceinline__ float pow5(float x) { float x2 = x * x; return x2 * x2 * x; }
__device__ __forceinline__ float pow6(float x) { float x2 = x * x; return x2 * x2 * x2; }
__device__ __forceinline__ float3 metal_edge_correction(float3 f0, float3 tint) {
    if (tint.x == 1.f && tint.y == 1.f && tint.z == 1.f) return f3(0.f);
    const float mu = 1.f / 7.f;
    float3 edge = f0 + (f3(1.f) - f0) * powf(1.f - mu, 5.f);
    return edge * (f3(1.f) - tint) / (mu * powf(1.f - mu, 6.f));
}
__device__ __forceinline__ float3 reflection_fresnel_at_ior(float3 bc, float bw, float metal, float sw, float3 sc, float cosine, float eta) {
    cosine = clampf(cosine, 0.f, 1.f);
    float3 diel = sc * fresnel(cosine, eta);
    if (metal <= 0.f) return diel;
    float3 f0 = bc * bw;
    float3 m = f0 + (f3(1.f) - f0) * powf(1.f - cosine, 5.f) - metal_edge_correction(f0, sc) * (cosine * powf(1.f - cosine, 6.f));
    m = vmax(m, f3(0.f));
    return lerp3(diel, m * sw, metal);
}
__device__ __forceinline__ float distribution(float nh, float a) { float x = (1.f - nh * nh) + nh * nh * a * a; return a * a / (PI_F * x * x); }
__device__ __forceinline__ float smith_denominator(float no, float ni, float a) {
    float ci = fabsf(ni), a2 = a * a;
    float po = sqrtf(a2 + (1.f - a2) * no * no), pi = sqrtf(a2 + (1.f - a2) * ci * ci);
    return ci * po + no * pi;
}
__device__ __forceinline__ float g2(float no, float ni, float a) { return 2.f * no * fabsf(ni) / smith_denominator(no, ni, a); }
__device__ __forceinline__ float3 ggx_visible_normal(float3 view, float alpha, float ux, float uy) {
    float3 v = normalize(f3(alpha * view.x, alpha * view.y, view.z));
    float ls = v.x * v.x + v.y * v.y;
    float3 t = ls > 0.f ? f3(-v.y, v.x, 0.f) / sqrtf(ls) : f3(1.f, 0.f, 0.f);
    float3 b = cross(v, t);
    float radius = sqrtf(ux), phi = 2.f * PI_F * uy;
    float sphi, cphi;
    sincosf(phi, &sphi, &cphi);
    float x = radius * cphi;
    float y = lerpf(sqrtf(fmaxf(1.f - x * x, 0.f)), radius * sphi, 0.5f * (1.f + v.z));
    float3 p = t * x + b * y + v * sqrtf(fmaxf(1.f - x * x - y * y, 0.f));
    return normalize(f3(alpha * p.x, alpha * p.y, fmaxf(p.z, 0.f)));
}
__device__ __forceinline__ float ggx_visible_weight(float no, float ni, float a) {
    if (ni <= 0.f) return 0.f;
    float a2 = a * a;
    return ni * (no + sqrtf(a2 + (1.f - a2) * no * no)) / smith_denominator(no, ni, a);
}
__device__ __forceinline__ float ggx_visible_reflection(float no, float a, float ux, float uy, float& vh) {
    float3 view = f3(sqrtf(fmaxf(1.f - no * no, 0.f)), 0.f, no);
    float3 h = ggx_visible_normal(view, a, ux, uy);
    float3 light = reflect(-view, h);
    vh = clampf(dot(view, h), 0.f, 1.f);
    return ggx_visible_weight(no, light.z, a);
}
__device__ __forceinline__ float3 ggx_reflection(float3 refl, float no, float ni, float nh, float r) {
    float a = specular_alpha(r);
    return refl * (distribution(nh, a) * g2(no, ni, a) / (4.f * no * ni));
}

// ---------------------------------------------------------------- BRDF atlas lookup (frame.slang:158-181)
struct Lut { const ushort4* texels; };  // BRDF_SIZE x BRDF_HEIGHT RGBA fp16
__device__ __forceinline__ float4 lut_texel(const Lut& l, int x, int y) {
    ushort4 t = __ldg(&l.texels[y * BRDF_SIZE + x]);
    return make_float4(__half2float(__ushort_as_half(t.x)), __half2float(__ushort_as_half(t.y)),
                       __half2float(__ushort_as_half(t.z)), __half2float(__ushort_as_half(t.w)));
}
// Bilinear, clamp-to-edge, texel centred.
__device__ __forceinline__ float4 lut_fetch(const Lut& l, float fx, float fy) {
    fx = clampf(fx, 0.f, float(BRDF_SIZE - 1));
    fy = clampf(fy, 0.f, float(BRDF_HEIGHT - 1));
    int x0 = int(floorf(fx)), y0 = int(floorf(fy));
    int x1 = min(x0 + 1, int(BRDF_SIZE) - 1), y1 = min(y0 + 1, int(BRDF_HEIGHT) - 1);
    float tx = fx - float(x0), ty = fy - float(y0);
    float4 a = lut_texel(l, x0, y0), b = lut_texel(l, x1, y0), c = lut_texel(l, x0, y1), d = lut_texel(l, x1, y1);
    auto L = [&](float p, float q, float r, float s) { return lerpf(lerpf(p, q, tx), lerpf(r, s, tx), ty); };
    return make_float4(L(a.x, b.x, c.x, d.x), L(a.y, b.y, c.y, d.y), L(a.z, b.z, c.z, d.z), L(a.w, b.w, c.w, d.w));
}
__device__ __forceinline__ float lut_alpha_coord(float roughness) {
    return log2f(clampf(roughness * roughness, MIN_ALPHA, 1.f) / MIN_ALPHA) / log2f(1.f / MIN_ALPHA);
}
__device__ __forceinline__ float4 brdf_texel(const Lut& l, float nv, float roughness) {
    float u = sqrtf(sqrtf(clampf(nv, 0.f, 1.f)));
    return lut_fetch(l, u * float(BRDF_SIZE - 1), lut_alpha_coord(roughness) * float(BRDF_SIZE - 1));
}
__device__ __forceinline__ float dielectric_albedo(const Lut& l, float nv, float roughness, float eta) {
    if (eta == 1.f) return 0.f;
    float at = eta / (1.f + eta) * float(BRDF_IOR_STEPS);
    uint32_t first = min(uint32_t(at), BRDF_IOR_STEPS - 1u), second = first + 1u;
    const float n1 = float(BRDF_ALBEDO_SIZE - 1);
    float lx = clampf(nv, 0.f, 1.f) * n1, ly = clampf(roughness, 0.f, 1.f) * n1;
    float ax = float((first % 2u) * BRDF_ALBEDO_SIZE), ay = float(BRDF_SIZE + (first / 2u) * BRDF_ALBEDO_SIZE);
    float bx = float((second % 2u) * BRDF_ALBEDO_SIZE), by = float(BRDF_SIZE + (second / 2u) * BRDF_ALBEDO_SIZE);
    return lerpf(lut_fetch(l, ax + lx, ay + ly).x, lut_fetch(l, bx + lx, by + ly).x, at - float(first));
}

// ---------------------------------------------------------------- closure + BSDF (bsdf*.slang subset)
struct Closure {
    float3 base_color; float base_weight, base_metalness;
    float3 specular_color; float specular_weight, specular_roughness, specular_ior, optical_ior;
    float3 n;
};
__device__ __forceinline__ float dielectric_ior(const Closure& c) { return c.optical_ior > 0.f ? c.optical_ior : modulated_ior(c.specular_ior, c.specular_weight); }
// path_boundary.slang:41-50 with air on both sides of an opaque (non-solid) surface.
__device__ __forceinline__ void boundary_closure_air(Closure& c) {
    c.optical_ior = c.specular_weight == 0.f ? 1.f : (c.specular_weight == 1.f ? c.specular_ior : modulated_ior(c.specular_ior, c.specular_weight));
}
struct Prepared { float3 p, diffuse, metal_comp, smooth, interface_n; float bump_a2; };
// bsdf.slang:184-212.
__device__ __forceinline__ float3 transport_probabilities(const Closure& c, float3 n, float3 view) {
    float diffuse = fmaxf(lum(c.base_color) * c.base_weight * (1.f - c.base_metalness), 0.f);
    float f = fresnel(fmaxf(dot(n, view), 0.f), dielectric_ior(c));
    float dielectric = f * fmaxf(lum(c.specular_color), 0.f);
    float reflection = fmaxf(lerpf(dielectric, c.specular_weight, c.base_metalness), 0.f);
    float total = diffuse + reflection;
    if (!(total > 0.f)) return f3(0.f);
    return f3(diffuse, reflection, 0.f) / fmaxf(total, POSITIVE_EPSILON);
}
// bsdf.slang:220-236.
__device__ __forceinline__ float3 valid_interface_normal(float3 normal, float3 geometric, float3 view) {
    float iz = dot(view, geometric);
    if (iz <= 0.f) return normal;
    if (dot(normal, geometric) < 0.f) normal = -normal;
    float threshold = fminf(0.9f * iz, 0.01f);
    if (dot(normal, view) > 0.f && dot(reflect(-view, normal), geometric) >= threshold) return normal;
    float3 tangent = normal - geometric * dot(normal, geometric);
    float ts = dot(tangent, tangent);
    if (ts <= 0.f) return geometric;
    float3 axis = tangent * rsqrtf(ts);
    float ix = dot(view, axis), ls = ix * ix + iz * iz;
    float cs = clampf(0.5f * (1.f + (iz * threshold - ix * sqrtf(fmaxf(ls - threshold * threshold, 0.f))) / ls), 0.f, 1.f);
    return axis * sqrtf(1.f - cs) + geometric * sqrtf(cs);
}
// bsdf_energy.slang:108-122.
__device__ __forceinline__ float3 metal_fresnel_average(const Closure& c) {
    float3 f0 = c.base_color * c.base_weight;
    float3 b = metal_edge_correction(f0, c.specular_color);
    if (any_pos(b)) {
        float3 avg = f3(0.f);
        for (uint32_t i = 0; i < BRDF_ALBEDO_SIZE; ++i) {
            float mu = (float(i) + 0.5f) / float(BRDF_ALBEDO_SIZE);
            avg = avg + reflection_fresnel_at_ior(c.base_color, c.base_weight, 1.f, 1.f, c.specular_color, mu, modulated_ior(c.specular_ior, 1.f)) * (2.f * mu / float(BRDF_ALBEDO_SIZE));
        }
        return vmin(vmax(avg, f3(0.f)), f3(1.f));
    }
    return vmin(vmax(f0 + (f3(1.f) - f0) / 21.f - b / 126.f, f3(0.f)), f3(1.f));
}
// bsdf_response.slang:13-19 + bsdf_energy.slang:123-136.
__device__ __forceinline__ float3 metal_compensation(const Lut& l, const Closure& c, float3 n, float3 view) {
    if (c.base_metalness <= 0.f || c.specular_roughness == 0.f) return f3(0.f);
    float4 m = brdf_texel(l, fmaxf(dot(n, view), 0.0001f), c.specular_roughness);
    float avg_e = lut_fetch(l, 0.f, lut_alpha_coord(c.specular_roughness) * float(BRDF_SIZE - 1)).w;
    float missing = 1.f / fmaxf(m.x + m.y, 1e-6f) - 1.f;
    float3 af = metal_fresnel_average(c);
    float3 den = vmax(f3(1.f) - af * (1.f - avg_e), f3(1e-6f));
    float3 num = af * (missing * avg_e);
    return f3(num.x / den.x, num.y / den.y, num.z / den.z);
}
// bsdf_response.slang:82-96.
__device__ __forceinline__ float3 direct_diffuse(const Lut& l, const Closure& c, float3 n, float3 view) {
    if (!(c.base_weight > 0.f && c.base_metalness < 1.f)) return f3(0.f);
    float3 albedo = c.specular_color * dielectric_albedo(l, fmaxf(dot(n, view), 0.0001f), c.specular_roughness, dielectric_ior(c));
    return (c.base_color * c.base_weight) * (1.f - c.base_metalness) * (f3(1.f) - albedo) / PI_F;
}
// Denoiser guide albedo of a camera hit (path.slang:1549-1571): the response to a uniform
// white world from surface_radiance_at (surface_lighting.slang:260-300) -- diffuse =
// direct_diffuse * pi, reflected = specular_reflectance(specular_response(c, view),
// brdf_moments(nv, roughness)) (bsdf_response.slang:47-77) -- about the closure's own
// normal, clamped to [0, 1] (closure weight 1: one closure, opaque).
__device__ __forceinline__ float3 guide_albedo(const Lut& l, const Closure& c, float3 view) {
    const float3 n = c.n;
    const float nv = fmaxf(dot(n, view), 0.0001f);
    const float4 m = brdf_texel(l, nv, c.specular_roughness);
    const float3 diffuse = direct_diffuse(l, c, n, view) * PI_F;
    const float f0 = fresnel(1.f, dielectric_ior(c));
    const float grazing = f0 != 0.f ? m.y : 0.f;
    float3 reflected = (f3(f0) * m.x + f3(grazing)) * c.specular_color;
    if (c.base_metalness > 0.f) {
        const float3 metal = c.base_color * c.base_weight;
        const float3 corr = metal_edge_correction(metal, c.specular_color);
        const float3 comp = metal_compensation(l, c, n, view);
        const float3 mr = (f3(1.f) + comp) * c.specular_weight * vmax(metal * m.x + f3(m.y) - corr * m.z, f3(0.f));
        reflected = lerp3(reflected, mr, c.base_metalness);
    }
    const float3 a = diffuse + reflected;
    return f3(clampf(a.x, 0.f, 1.f), clampf(a.y, 0.f, 1.f), clampf(a.z, 0.f, 1.f));
}
// bsdf.slang:242-250.
__device__ __forceinline__ Prepared transport_prepare(const Lut& l, const Closure& c, float3 view, float3 smooth, float3 geometric) {
    Prepared pr;
    float3 n = valid_interface_normal(c.n, geometric, view);
    pr.p = transport_probabilities(c, n, view);
    float dev = fabsf(dot(smooth, c.n));
    pr.bump_a2 = clampf((1.f - dev * dev) / fmaxf(8.f * dev * dev, POSITIVE_EPSILON), 0.f, 1.f);
    pr.diffuse = direct_diffuse(l, c, n, view);
    pr.metal_comp = metal_compensation(l, c, n, view);
    pr.smooth = smooth;
    pr.interface_n = n;
    return pr;
}
// bsdf.slang:255-265.
__device__ __forceinline__ float bump_shadow(const Closure& c, float3 dir, const Prepared& pr) {
    float cosine = dot(pr.smooth, dir);
    if (cosine * dot(pr.smooth, c.n) * dot(c.n, dir) < 0.f) return 0.f;
    if (pr.bump_a2 == 0.f) return 1.f;
    float mu = fabsf(cosine);
    return mu > 0.f ? 2.f * mu / (mu + sqrtf(pr.bump_a2 + (1.f - pr.bump_a2) * mu * mu)) : 0.f;
}
// bsdf_microfacet.slang:43-52.
__device__ __forceinline__ float visible_scale(float nv, float roughness) { float a = specular_alpha(roughness); return 2.f / (nv + sqrtf(a * a + (1.f - a * a) * nv * nv)); }
// bsdf.slang:296-309 (coat probability 0, no transmission).
__device__ __forceinline__ float pdf_mask(const Closure& c, float3 view, float3 dir, uint32_t mask, const Prepared& pr) {
    float3 n = pr.interface_n;
    float nl = dot(n, dir), cd = dot(c.n, dir);
    float pdf = (mask & VKB_RAY_DIFFUSE) ? pr.p.x * (cd > 0.f ? 1.f : 0.f) * fabsf(cd) / PI_F : 0.f;
    if (nl <= 0.f) return pdf;
    float3 h = normalize(view + dir);
    float d = distribution(fmaxf(dot(n, h), 0.f), specular_alpha(c.specular_roughness));
    return pdf + ((mask & VKB_RAY_SPECULAR) ? pr.p.y * (d * visible_scale(dot(n, view), c.specular_roughness) / 4.f) : 0.f);
}
// bsdf_energy.slang:138-149.
__device__ __forceinline__ float3 compensated_reflection(const Closure& c, float cosine, float3 comp) {
    float3 f = reflection_fresnel_at_ior(c.base_color, c.base_weight, c.base_metalness, c.specular_weight, c.specular_color, cosine, dielectric_ior(c));
    if (any_pos(comp)) {
        if (c.base_metalness == 1.f) f = f + comp * f;
        else f = f + comp * reflection_fresnel_at_ior(c.base_color, c.base_weight, 1.f, c.specular_weight, c.specular_color, cosine,
                                                      modulated_ior(c.specular_ior, c.specular_weight)) * c.base_metalness;
    }
    return f;
}
// bsdf.slang:356-375 with bsdf_response.slang:257-274.
__device__ __forceinline__ float3 eval_mask(const Closure& c, float3 view, float3 dir, uint32_t mask, const Prepared& pr) {
    float bump = bump_shadow(c, dir, pr);
    float3 specular = f3(0.f);
    float3 n = pr.interface_n;
    float nl = fmaxf(dot(n, dir), 0.f), nv = fmaxf(dot(n, view), 0.0001f);
    if (nl > 0.f && (mask & VKB_RAY_SPECULAR)) {
        float3 h = normalize(view + dir);
        float nh = fmaxf(dot(n, h), 0.f), vh = fmaxf(dot(view, h), 0.f);
        specular = ggx_reflection(compensated_reflection(c, vh, pr.metal_comp), nv, nl, nh, c.specular_roughness) * nl;
    }
    float cd = dot(c.n, dir);
    float3 diffuse = f3(0.f);
    if ((mask & VKB_RAY_DIFFUSE) && !(cd <= 0.f)) diffuse = pr.diffuse * (bump * cd);
    return specular + diffuse;
}
struct BsdfSample { float3 dir, weight; float pdf; uint32_t event; };
// bsdf_microfacet.slang:53-62.
__device__ __forceinline__ float3 visible_normal(float3 n, float roughness, float3 view, float ux, float uy) {
    float3 x = basis_direction(n, f3(1.f, 0.f, 0.f)), y = basis_direction(n, f3(0.f, 1.f, 0.f));
    float3 s = ggx_visible_normal(f3(dot(view, x), dot(view, y), dot(view, n)), specular_alpha(roughness), ux, uy);
    return x * s.x + y * s.y + n * s.z;
}
// bsdf.slang:446-511.
__device__ __forceinline__ BsdfSample transport_sample(const Closure& c, float3 view, float rx, float ry, float rz, const Prepared& pr) {
    BsdfSample r;
    r.dir = f3(0.f); r.weight = f3(0.f); r.pdf = 0.f; r.event = 0u;
    float3 n = pr.interface_n;
    if (rz < pr.p.x) {
        float radius = sqrtf(rx), sphi, cphi;
        sincosf(TAU_F * ry, &sphi, &cphi);
        r.dir = basis_direction(c.n, f3(radius * cphi, radius * sphi, sqrtf(1.f - rx)));
        r.event = VKB_RAY_DIFFUSE;
    } else if (rz < pr.p.x + pr.p.y) {
        float3 h = visible_normal(n, c.specular_roughness, view, rx, ry);
        r.dir = reflect(-view, h);
        r.event = VKB_RAY_SPECULAR;
        if (dot(n, r.dir) <= 0.f) { r.dir = f3(0.f); r.event = 0u; return r; }
    } else {
        return r;
    }
    r.pdf = pdf_mask(c, view, r.dir, r.event, pr);
    if (r.pdf > 0.f) r.weight = eval_mask(c, view, r.dir, r.event, pr) / r.pdf;
    return r;
}
// path.slang:833-836, 837-840, 841-850.
__device__ __forceinline__ float mis_power(float sampled, float other) {
    if (sampled <= 0.f) return 0.f;
    float ratio = other / sampled;
    return 1.f / (1.f + ratio * ratio);
}
__device__ __forceinline__ bool event_hemisphere(uint32_t event, float3 dir, float3 face, float3 smooth) {
    if (event == VKB_RAY_TRANSMISSION) return dot(face, dir) < 0.f && dot(smooth, dir) < 0.f;
    return dot(smooth, dir) > 0.f;
}
__device__ __forceinline__ float3 analytic_mis_response(const Closure& c, float3 view, float3 dir, float3 face, uint32_t contribution, float light_pdf, const Prepared& pr) {
    float3 value = f3(0.f);
    if ((contribution & VKB_RAY_DIFFUSE) && event_hemisphere(VKB_RAY_DIFFUSE, dir, face, pr.smooth)) {
        float w = light_pdf > 0.f ? mis_power(light_pdf, pdf_mask(c, view, dir, VKB_RAY_DIFFUSE, pr)) : 1.f;
        value = value + eval_mask(c, view, dir, VKB_RAY_DIFFUSE, pr) * w;
    }
    if ((contribution & VKB_RAY_SPECULAR) && event_hemisphere(VKB_RAY_SPECULAR, dir, face, pr.smooth)) {
        float w = light_pdf > 0.f ? mis_power(light_pdf, pdf_mask(c, view, dir, VKB_RAY_SPECULAR, pr)) : 1.f;
        value = value + eval_mask(c, view, dir, VKB_RAY_SPECULAR, pr) * w;
    }
    return value;
}

// ---------------------------------------------------------------- emitters (emitter.slang:54-167)
__device__ __forceinline__ float emitter_window(const vkb_light& l, float3 world, float3 dir) {
    float value = 1.f;
    if (l.position[3] > 0.f && l.projection[1] > 0.f) {
        float3 rel = (get3(l.position) - world) / l.projection[1];
        float ratio = dot(rel, rel);
        value = fmaxf(1.f - ratio * ratio, 0.f);
    }
    if (l.position[3] == 2.f) {
        float cosine = dot(-dir, normalize(get3(l.direction)));
        float outer = l.direction[3], inner = l.radiance[3];
        float cone = cosine >= outer ? 1.f : 0.f;
        if (inner > outer) {
            float t = saturatef((cosine - outer) / (inner - outer));
            cone = l.projection[2] > 0.f ? t * t : t * t * (3.f - 2.f * t);
        }
        value *= cone;
    }
    return value;
}
__device__ __forceinline__ float3 cone_direction(float3 axis, float omc, float u, float v) {
    float height = u * omc;
    float radius = sqrtf(fmaxf(height * (2.f - height), 0.f));
    float s, c;
    sincosf(TAU_F * v, &s, &c);
    return basis_direction(axis, f3(radius * c, radius * s, 1.f - height));
}
__device__ __forceinline__ float3 emitter_direction(const vkb_light& l, float3 world, float ux, float uy, float& distance) {
    float kind = l.position[3], size = l.params[1];
    float3 axis = normalize(-get3(l.direction));
    distance = FP32_MAX;
    if (kind == 0.f && size > 0.f) {
        float s = sinf(size * 0.5f);
        axis = cone_direction(axis, 2.f * s * s, ux, uy);
    }
    if (kind > 0.f) {
        float3 point = get3(l.position), delta = point - world;
        distance = length(delta);
        axis = distance > 0.f ? delta / distance : f3(0.f);
        if (kind == 3.f) {
            float sx = ux - 0.5f, sy = uy - 0.5f;
            if (l.emitter_u[3] > 0.f) {
                float r = sqrtf(ux) * 0.5f, sphi, cphi;
                sincosf(TAU_F * uy, &sphi, &cphi);
                sx = r * cphi; sy = r * sphi;
            }
            point = point + get3(l.emitter_u) * sx + get3(l.emitter_v) * sy;
            distance = length(point - world);
            axis = distance > 0.f ? (point - world) / distance : f3(0.f);
        } else if (size > 0.f && distance > size) {
            float ratio = size / distance, sq = ratio * ratio;
            axis = cone_direction(axis, sq / (1.f + sqrtf(1.f - sq)), ux, uy);
            float along = dot(delta, axis);
            float3 perp = cross(delta, axis);
            distance = along - sqrtf(fmaxf(size * size - dot(perp, perp), 0.f));
        }
    }
    return axis;
}
struct EmitterEval { float3 radiance; float pdf, distance; };
__device__ __forceinline__ bool emitter_delta(const vkb_light& l) { return l.position[3] != 3.f && l.params[1] == 0.f; }
__device__ __forceinline__ EmitterEval emitter_eval(const vkb_light& l, float3 world, float3 dir) {
    EmitterEval r;
    r.radiance = f3(0.f); r.pdf = 0.f; r.distance = 0.f;
    if (emitter_delta(l)) return r;
    float kind = l.position[3], size = l.params[1];
    if (kind == 0.f) {
        float3 axis = normalize(-get3(l.direction));
        float sine = sinf(size);
        float3 perp = cross(axis, dir);
        if (dot(axis, dir) <= 0.f || dot(perp, perp) > sine * sine) return r;
        float hs = sinf(size * 0.5f);
        r.pdf = 1.f / (4.f * PI_F * hs * hs);
        r.radiance = get3(l.radiance) / (PI_F * sine * sine);
        r.distance = FP32_MAX;
        return r;
    }
    if (kind < 3.f) {
        float3 delta = get3(l.position) - world;
        float sq = dot(delta, delta), radius = size;
        if (sq <= radius * radius) return r;
        float along = dot(delta, dir);
        float3 perp = cross(delta, dir);
        float disc = radius * radius - dot(perp, perp);
        if (along <= 0.f || disc < 0.f) return r;
        float ratio = radius * radius / sq;
        r.pdf = (1.f + sqrtf(1.f - ratio)) / (TAU_F * ratio);
        r.radiance = get3(l.radiance) / (4.f * PI_F * PI_F * radius * radius) * emitter_window(l, world, dir);
        r.distance = along - sqrtf(disc);
        return r;
    }
    float3 center = get3(l.position) - world;
    if (dot(get3(l.direction), -center) <= 0.f) return r;
    float3 u = get3(l.emitter_u) * 0.5f, v = get3(l.emitter_v) * 0.5f;
    bool ellipse = l.emitter_u[3] > 0.f;
    float3 normal = cross(u, v);
    float square = dot(normal, normal);
    if (square <= 0.f) return r;
    float den = dot(normal, dir);
    if (den == 0.f) return r;
    float distance = dot(normal, center) / den;
    if (distance <= 0.f) return r;
    float3 q = dir * distance - center;
    float uu = dot(u, u), uv = dot(u, v), vv = dot(v, v), qu = dot(q, u), qv = dot(q, v);
    float cx = (qu * vv - qv * uv) / square, cy = (qv * uu - qu * uv) / square;
    if (ellipse ? (cx * cx + cy * cy > 1.f) : (fabsf(cx) > 1.f || fabsf(cy) > 1.f)) return r;
    float area = 4.f * sqrtf(square) * (ellipse ? PI_F * 0.25f : 1.f);
    r.pdf = distance * distance / (area * fabsf(den) / sqrtf(square));
    r.radiance = get3(l.radiance) / (PI_F * area) * emitter_window(l, world, dir);
    r.distance = distance;
    return r;
}
struct LightSample { float3 dir, radiance; float distance, pdf; bool delta; };
__device__ __forceinline__ LightSample emitter_sample(const vkb_light& l, float3 world, float ux, float uy) {
    LightSample s;
    s.delta = emitter_delta(l);
    s.dir = emitter_direction(l, world, ux, uy, s.distance);
    s.pdf = 0.f;
    if (s.delta) {
        s.radiance = get3(l.radiance);
        if (l.position[3] > 0.f) {
            float den = 4.f * PI_F * s.distance * s.distance;
            s.radiance = den > 0.f ? s.radiance / den * emitter_window(l, world, s.dir) : f3(0.f);
        }
    } else {
        EmitterEval e = emitter_eval(l, world, s.dir);
        s.radiance = e.radiance; s.pdf = e.pdf;
    }
    return s;
}

// ---------------------------------------------------------------- light tree (light_tree.slang:1-84; node = lights/tree.rs:27-36)
struct LightTreeNode { float4 lower_power, upper_infinite; uint4 links, source; };
__device__ __forceinline__ float tree_log_importance(const LightTreeNode& node, float3 p) {
    if (!(node.lower_power.w > 0.f)) return -FP32_MAX;
    float power = log2f(node.lower_power.w);
    if (node.upper_infinite.w != 0.f) return power;
    float3 lo = f3(node.lower_power.x, node.lower_power.y, node.lower_power.z);
    float3 hi = f3(node.upper_infinite.x, node.upper_infinite.y, node.upper_infinite.z);
    float3 center = lo * 0.5f + hi * 0.5f, radius = hi * 0.5f - lo * 0.5f, delta = p - center;
    float d = fmaxf(LIGHT_TREE_MIN_DISTANCE_SQUARED, fmaxf(dot(delta, delta), dot(radius, radius)));
    if (!isfinite(d)) return -FP32_MAX;
    return power - log2f(d);
}
__device__ __forceinline__ float tree_branch(const LightTreeNode& a, const LightTreeNode& b, float3 p) {
    float x = tree_log_importance(a, p), y = tree_log_importance(b, p);
    float scale = fmaxf(x, y);
    float uniform = float(a.links.w) / (float(a.links.w) + float(b.links.w));
    if (scale == -FP32_MAX) return uniform;
    x = exp2f(x - scale); y = exp2f(y - scale);
    return x / (x + y);
}
__device__ __forceinline__ uint32_t tree_pick(const LightTreeNode* nodes, uint32_t count, float3 p, float ux, float uy, float& probability) {
    probability = 0.f;
    if (count == 0u) return 0xffffffffu;
    uint32_t node = 0;
    float prob = 1.f;
    const float one_below = 1.f - FP32_EPS * 0.5f;
    float choice = clampf(ux, 0.f, one_below);
    bool uniform = uy < LIGHT_TREE_UNIFORM_MIX;
    uint32_t total = nodes[0].links.w;
    uint32_t rank = min(uint32_t(choice * float(total)), total - 1u);
    for (int guard = 0; guard < 64 && nodes[node].links.x != 0xffffffffu; ++guard) {
        uint32_t l = nodes[node].links.x, r = nodes[node].links.y;
        float pb = tree_branch(nodes[l], nodes[r], p);
        bool left;
        if (uniform) {
            uint32_t cnt = nodes[l].links.w;
            left = rank < cnt;
            if (!left) rank -= cnt;
        } else {
            left = choice < pb;
            choice = left ? choice / pb : (choice - pb) / (1.f - pb);
            choice = fminf(choice, one_below);
        }
        prob *= left ? pb : 1.f - pb;
        node = left ? l : r;
    }
    probability = LIGHT_TREE_UNIFORM_MIX / float(total) + (1.f - LIGHT_TREE_UNIFORM_MIX) * prob;
    return nodes[node].source.y;
}

// ---------------------------------------------------------------- ray origins (vork_prelude.slang:162-181,340-345)
__device__ __forceinline__ float3 surface_ray_origin(float3 world, float3 error, float3 g, float3 dir) {
    float scale = maxc(vabs(g));
    if (scale == 0.f) return world;
    float3 n = g / scale;
    float amount = next_float(dot(vabs(n), error) / dot(n, n), true);
    float3 offset = n * (amount * (dot(n, dir) >= 0.f ? 1.f : -1.f));
    float3 o = world + offset;
    if (offset.x != 0.f) o.x = next_float(o.x, offset.x > 0.f);
    if (offset.y != 0.f) o.y = next_float(o.y, offset.y > 0.f);
    if (offset.z != 0.f) o.z = next_float(o.z, offset.z > 0.f);
    return o;
}
__device__ __forceinline__ void ray_connection(float3 origin, float3 world, float3 dir, float distance, float3& od, float& ol) {
    if (distance == FP32_MAX || (origin.x == world.x && origin.y == world.y && origin.z == world.z)) { od = dir; ol = distance; return; }
    float3 delta = dir * distance - (origin - world);
    float rem = length(delta);
    od = rem > 0.f ? delta / rem : dir;
    ol = rem;
}
// sample_clamp.slang:7-17.
__device__ __forceinline__ float3 clamp_sample(float3 v, float limit, uint32_t& dropped) {
    float br = (fabsf(v.x) + fabsf(v.y) + fabsf(v.z)) * (1.f / 3.f);
    if (!isfinite(br)) { dropped++; v = f3(0.f); br = 0.f; }
    return v * ((limit > 0.f && br > limit) ? limit / fmaxf(br, POSITIVE_EPSILON) : 1.f);
}

}  // namespace vkb
