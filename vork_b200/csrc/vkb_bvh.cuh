// Acceleration structures for the B200 backend (B200 has no RT cores): a per-frame
// instance TLAS built as a linear BVH (Karras 2012) over 30-bit Morton codes, sorted
// with cub's radix sort and refitted bottom-up with atomic counters, and per-mesh BLAS
// built once at install with a binned SAH (host, vkb.cu) in the same node format.
// The reference builds these inside the Vulkan driver (crates/vork-render/src/rt.rs:
// Rays::new :1098-1289 for BLAS batches, FrameRays::new :1339-1385 and encode /
// rebuild_tlas :1387-1476 for the instance TLAS); its traversal is RayQuery::Proceed
// (shaders/path.slang:155-189, :641-684).  Both levels are built as binary trees and
// collapsed to 4-wide nodes of one 128-byte line (FP32 child boxes as planes); traversal
// is a two-level stack walk over those, nearest child first, with watertight triangle
// tests (Woop, Benthin & Wald, JCGT 2013), bounded stack and iteration count.
#pragma once
#include <cstdint>
#include "vkb_device.cuh"

namespace vkb {

// Both child boxes of a binary node in four 16-byte lanes: one 64-byte load per visit.
// a = (L.lo.x, L.hi.x, L.lo.y, L.hi.y), b = (R.lo.x, R.hi.x, R.lo.y, R.hi.y),
// c = (L.lo.z, L.hi.z, R.lo.z, R.hi.z), d = (left, right, -, -).  A child reference
// >= 0 is an internal node, < 0 is ~(sorted leaf index).
struct alignas(16) BvhNode { float4 a, b, c; int4 d; };

// Four child boxes of a 4-wide node as planes (component k = child slot k), one 128-byte
// line per node: plane 2a is the low face of axis a, plane 2a+1 the high face, so a ray
// reads its near face of axis a at 2a + (direction negative) and its far face at the
// other.  child = (c0, c1, c2, c3) as in BvhNode; an unused slot has the empty box
// lo = +inf, hi = -inf, which every ray misses.  Traversal runs on these nodes; they are
// collapsed from the binary trees (every internal node at even depth takes its children
// and the children of its internal children).
struct alignas(16) Bvh4Node { float4 plane[6]; int4 child; int4 pad; };
static_assert(sizeof(Bvh4Node) == 128, "one 128-byte line per 4-wide node");

// Compressed 8-wide BLAS node, 80 bytes (the layout of vkb_host::Wide8Node, built on the
// host in vkb_wide8.h): child boxes as bytes on the node's grid (origin + q * 2^(e-127)
// per axis, rounded outward), internal children from child_base in the first slots, leaf
// triangles from leaf_base in the next ones, unused slots (lo 255 > hi 0) last.
//   h = (origin.xyz, bits: ex | ey << 8 | ez << 16 | internal-slot mask << 24)
//   b = (child_base, leaf_base, used slots, -);  q[a] = (lo bytes 0-3, lo 4-7, hi 0-3, hi 4-7) of axis a
struct alignas(16) Bvh8Node { float4 h; uint4 b; uint4 q[3]; };
static_assert(sizeof(Bvh8Node) == 80, "80-byte compressed 8-wide node");

// One TLAS leaf, in Morton order: the instance's world->object rows and what its BLAS needs.
struct alignas(16) TlasLeaf { float4 w2o[3]; uint32_t instance, node_offset, tri_offset, flags; };
constexpr uint32_t LEAF_CULL_BACKFACES = 1u;

struct MeshInfo {
    uint32_t node_offset, tri_offset, index_offset, vertex_offset;
    uint32_t num_triangles, pad0, pad1, pad2;
    float lo[4], hi[4];      // object-space box (xyz)
    float sphere[4];         // bounding sphere about the box centre: centre xyz, radius (< 0: none)
};

#ifndef VKB_SMEM_STACK
#define VKB_SMEM_STACK 24
#endif
#ifndef VKB_SPILL_STACK
#define VKB_SPILL_STACK 40
#endif
// Traversal stacks: the first SMEM_STACK entries live in shared memory as
// [entry][thread] (lane l of a 128-thread block always touches bank l, whatever depth
// each lane is at: no bank conflicts); deeper entries go to a per-thread local array of
// SPILL_STACK entries.  Shared memory not taken by stacks serves as L1 for the nodes.
constexpr int SMEM_STACK = VKB_SMEM_STACK;
constexpr int SPILL_STACK = VKB_SPILL_STACK;
constexpr int STACK_CAP = SMEM_STACK + SPILL_STACK;
// An 8-wide BLAS visit pushes up to seven children: its traversals get a deeper local part.
constexpr int SPILL_STACK8 = 104;
constexpr int STACK_CAP8 = SMEM_STACK + SPILL_STACK8;
constexpr int TRACE_BLOCK = 128;
struct TraceStack {
    int* r;
    int* spill;
    __device__ __forceinline__ void put(int i, int v) {
        if (SPILL_STACK == 0 || i < SMEM_STACK) r[i * TRACE_BLOCK] = v;
        else spill[i - SMEM_STACK] = v;
    }
    __device__ __forceinline__ int get(int i) const {
        return (SPILL_STACK == 0 || i < SMEM_STACK) ? r[i * TRACE_BLOCK] : spill[i - SMEM_STACK];
    }
};
constexpr uint32_t TRACE_STEP_LIMIT = 1u << 16;
constexpr int SENTINEL = 0x7fffffff;

// ---------------------------------------------------------------- Morton codes (bit-exact with the CPU restatement)
__device__ __forceinline__ uint32_t expand_bits(uint32_t v) {
    v = (v * 0x00010001u) & 0xFF0000FFu;
    v = (v * 0x00000101u) & 0x0F00F00Fu;
    v = (v * 0x00000011u) & 0xC30C30C3u;
    v = (v * 0x00000005u) & 0x49249249u;
    return v;
}
__device__ __forceinline__ uint32_t quantize10(float x) {
    float q = __fmul_rn(x, 1024.f);
    q = q < 0.f ? 0.f : q;
    q = q > 1023.f ? 1023.f : q;
    return uint32_t(q);
}
// Centroid (lo+hi)/2 normalised over the centroid box, 10 bits per axis, x highest.
__device__ __forceinline__ uint32_t morton_code(float4 lo, float4 hi, float3 slo, float3 ext) {
    float c[3] = {__fmul_rn(__fadd_rn(lo.x, hi.x), 0.5f), __fmul_rn(__fadd_rn(lo.y, hi.y), 0.5f), __fmul_rn(__fadd_rn(lo.z, hi.z), 0.5f)};
    float l[3] = {slo.x, slo.y, slo.z}, e[3] = {ext.x, ext.y, ext.z};
    uint32_t q[3];
    for (int a = 0; a < 3; ++a) q[a] = quantize10(e[a] > 0.f ? __fdiv_rn(__fsub_rn(c[a], l[a]), e[a]) : 0.5f);
    return (expand_bits(q[0]) << 2) | (expand_bits(q[1]) << 1) | expand_bits(q[2]);
}
// Order-preserving float <-> uint for atomic min/max of the centroid box.
__device__ __forceinline__ uint32_t float_flip(float f) { uint32_t u = __float_as_uint(f); return (u & 0x80000000u) ? ~u : (u | 0x80000000u); }
__device__ __forceinline__ float float_unflip(uint32_t u) { return __uint_as_float((u & 0x80000000u) ? (u & 0x7fffffffu) : ~u); }

// ---------------------------------------------------------------- traversal
struct RaySpace {
    float3 o, idir, ood;        // origin, 1/d, o/d
    uint32_t k;                 // watertight shear permutation: kx | ky << 2 | kz << 4
    float sx, sy, sz;
};
__device__ __forceinline__ float safe_rcp(float x) { return 1.f / (fabsf(x) > 1e-20f ? x : copysignf(1e-20f, x)); }
__device__ __forceinline__ float comp(float3 v, int k) { return k == 0 ? v.x : (k == 1 ? v.y : v.z); }
__device__ __forceinline__ void make_space(RaySpace& r, float3 o, float3 d) {
    r.o = o;
    r.idir = f3(safe_rcp(d.x), safe_rcp(d.y), safe_rcp(d.z));
    r.ood = f3(o.x * r.idir.x, o.y * r.idir.y, o.z * r.idir.z);
    float ax = fabsf(d.x), ay = fabsf(d.y), az = fabsf(d.z);
    int kz = (ax > ay) ? (ax > az ? 0 : 2) : (ay > az ? 1 : 2);
    int kx = kz + 1 == 3 ? 0 : kz + 1;
    int ky = kx + 1 == 3 ? 0 : kx + 1;
    float dz = comp(d, kz);
    if (dz < 0.f) { int t = kx; kx = ky; ky = t; }
    r.k = uint32_t(kx) | uint32_t(ky) << 2 | uint32_t(kz) << 4;
    r.sx = comp(d, kx) / dz;
    r.sy = comp(d, ky) / dz;
    r.sz = 1.f / dz;
}
// Slab test of both children of a node; returns entry distances (or +inf on miss).
__device__ __forceinline__ void node_boxes(const BvhNode& n, const RaySpace& r, float tmax, float& tl, float& tr) {
    float lx0 = fmaf(n.a.x, r.idir.x, -r.ood.x), lx1 = fmaf(n.a.y, r.idir.x, -r.ood.x);
    float ly0 = fmaf(n.a.z, r.idir.y, -r.ood.y), ly1 = fmaf(n.a.w, r.idir.y, -r.ood.y);
    float lz0 = fmaf(n.c.x, r.idir.z, -r.ood.z), lz1 = fmaf(n.c.y, r.idir.z, -r.ood.z);
    float rx0 = fmaf(n.b.x, r.idir.x, -r.ood.x), rx1 = fmaf(n.b.y, r.idir.x, -r.ood.x);
    float ry0 = fmaf(n.b.z, r.idir.y, -r.ood.y), ry1 = fmaf(n.b.w, r.idir.y, -r.ood.y);
    float rz0 = fmaf(n.c.z, r.idir.z, -r.ood.z), rz1 = fmaf(n.c.w, r.idir.z, -r.ood.z);
    float lmin = fmaxf(fmaxf(fminf(lx0, lx1), fminf(ly0, ly1)), fmaxf(fminf(lz0, lz1), 0.f));
    float lmax = fminf(fminf(fmaxf(lx0, lx1), fmaxf(ly0, ly1)), fminf(fmaxf(lz0, lz1), tmax));
    float rmin = fmaxf(fmaxf(fminf(rx0, rx1), fminf(ry0, ry1)), fmaxf(fminf(rz0, rz1), 0.f));
    float rmax = fminf(fminf(fmaxf(rx0, rx1), fmaxf(ry0, ry1)), fminf(fmaxf(rz0, rz1), tmax));
    // Conservative widening by a few ulps keeps hits on box faces (exact-fit leaf boxes).
    tl = lmin <= lmax * 1.00000024f ? lmin : __int_as_float(0x7f800000);
    tr = rmin <= rmax * 1.00000024f ? rmin : __int_as_float(0x7f800000);
}
// Three-input float min / max (sm_100 instructions; no NaN reaches them here).
__device__ __forceinline__ float max3f(float a, float b, float c) { float r; asm("max.f32 %0, %1, %2, %3;" : "=f"(r) : "f"(a), "f"(b), "f"(c)); return r; }
__device__ __forceinline__ float min3f(float a, float b, float c) { float r; asm("min.f32 %0, %1, %2, %3;" : "=f"(r) : "f"(a), "f"(b), "f"(c)); return r; }
// Entry distance key of child slot k of a 4-wide node from the ray's near and far faces:
// float bits of the entry distance (>= 0, so unsigned order is distance order) with the
// slot in the two low bits, or ~0u on a miss.
__device__ __forceinline__ uint32_t slot_key(float nx, float ny, float nz, float fx, float fy, float fz, const RaySpace& r, float tmax, uint32_t k) {
    float tn = max3f(fmaf(nx, r.idir.x, -r.ood.x), fmaf(ny, r.idir.y, -r.ood.y), fmaxf(fmaf(nz, r.idir.z, -r.ood.z), 0.f));
    float tf = min3f(fmaf(fx, r.idir.x, -r.ood.x), fmaf(fy, r.idir.y, -r.ood.y), fminf(fmaf(fz, r.idir.z, -r.ood.z), tmax));
    return tn <= tf * 1.00000024f ? ((__float_as_uint(tn) & ~3u) | k) : 0xffffffffu;
}
// Far-first key (larger entry distance, smaller key; misses stay ~0u).  Occlusion rays
// visit children far to near: the near ones are mostly the surface the ray leaves, which
// cannot occlude it (measured on the flock frame: 45.5 -> 41.4 node visits per shadow ray).
__device__ __forceinline__ uint32_t far_key(uint32_t key) {
    return key == 0xffffffffu ? key : ((0x7ffffffcu - (key & ~3u)) | (key & 3u));
}
__device__ __forceinline__ void key_order(uint32_t& a, uint32_t& b) { uint32_t l = min(a, b); b = max(a, b); a = l; }
__device__ __forceinline__ int slot_child(const int4& c, uint32_t key) {
    const bool odd = (key & 1u) != 0u;
    const int lo = odd ? c.y : c.x, hi = odd ? c.w : c.z;
    return (key & 2u) ? hi : lo;
}
// Byte k (0-3) of w as a float: a byte permute builds 2^23 + byte, an exact subtract removes 2^23.
__device__ __forceinline__ float byte_f(uint32_t w, uint32_t k) {
    return __uint_as_float(__byte_perm(w, 0x4b000000u, k | 0x7440u)) - 8388608.f;
}
// Far-first key of an 8-wide slot (three slot bits).
__device__ __forceinline__ uint32_t far_key8(uint32_t key) {
    return key == 0xffffffffu ? key : ((0x7ffffff8u - (key & ~7u)) | (key & 7u));
}
// Batcher's odd-even merge network for eight keys (19 exchanges), ascending.
__device__ __forceinline__ void sort8(uint32_t (&k)[8]) {
    key_order(k[0], k[1]); key_order(k[2], k[3]); key_order(k[4], k[5]); key_order(k[6], k[7]);
    key_order(k[0], k[2]); key_order(k[1], k[3]); key_order(k[4], k[6]); key_order(k[5], k[7]);
    key_order(k[1], k[2]); key_order(k[5], k[6]);
    key_order(k[0], k[4]); key_order(k[1], k[5]); key_order(k[2], k[6]); key_order(k[3], k[7]);
    key_order(k[2], k[4]); key_order(k[3], k[5]);
    key_order(k[1], k[2]); key_order(k[3], k[4]); key_order(k[5], k[6]);
}
// Watertight ray/triangle test. cull: accept front faces only (counter-clockwise
// winding seen from the ray origin).  Returns t and barycentrics of vertices 1, 2.
__device__ __forceinline__ bool tri_test(const RaySpace& r, float3 v0, float3 v1, float3 v2, bool cull, float tbest, float& t, float& b1, float& b2) {
    const int kx = int(r.k & 3u), ky = int((r.k >> 2) & 3u), kz = int(r.k >> 4);
    float3 A = v0 - r.o, B = v1 - r.o, C = v2 - r.o;
    float Az = comp(A, kz), Bz = comp(B, kz), Cz = comp(C, kz);
    float Ax = comp(A, kx) - r.sx * Az, Ay = comp(A, ky) - r.sy * Az;
    float Bx = comp(B, kx) - r.sx * Bz, By = comp(B, ky) - r.sy * Bz;
    float Cx = comp(C, kx) - r.sx * Cz, Cy = comp(C, ky) - r.sy * Cz;
    float U = Cx * By - Cy * Bx, V = Ax * Cy - Ay * Cx, W = Bx * Ay - By * Ax;
    if (U == 0.f || V == 0.f || W == 0.f) {
        double cxby = double(Cx) * double(By), cybx = double(Cy) * double(Bx);
        double axcy = double(Ax) * double(Cy), aycx = double(Ay) * double(Cx);
        double bxay = double(Bx) * double(Ay), byax = double(By) * double(Ax);
        U = float(cxby - cybx); V = float(axcy - aycx); W = float(bxay - byax);
    }
    bool neg = U < 0.f || V < 0.f || W < 0.f, pos = U > 0.f || V > 0.f || W > 0.f;
    if (cull ? neg : (neg && pos)) return false;
    float det = U + V + W;
    if (det == 0.f) return false;
    float T = U * (r.sz * Az) + V * (r.sz * Bz) + W * (r.sz * Cz);
    float inv = 1.f / det;
    t = T * inv;
    if (!(t >= 0.f && t <= tbest)) return false;
    b1 = V * inv; b2 = W * inv;
    return true;
}

// Triangles per BLAS leaf (1..4; counts are stored in two bits).  One triangle per leaf
// measured fastest on the instanced flock frame (the SAH tree then has fewer box tests
// per ray than multi-triangle leaves save in node visits).
#ifndef VKB_BLAS_LEAF_MAX
#define VKB_BLAS_LEAF_MAX 1
#endif
static_assert(VKB_BLAS_LEAF_MAX >= 1 && VKB_BLAS_LEAF_MAX <= 4, "leaf counts are stored in two bits");

// tri: the hit triangle's position in BLAS leaf order (global index into blas_tris; its
// original id is blas_tris[3 * tri].w), inst: the original instance id.
struct HitRecord { float t, u, v; uint32_t tri, inst; };

// A world ray in global memory: entry i of an origin queue and a direction queue (xyz of
// float4).  Traversal re-reads it when it enters or leaves an instance instead of keeping
// six registers live across the loop; the volatile loads keep the compiler from caching
// the values, and the queue bases are the same for every thread (uniform registers).
struct RayRef {
    const float4* o;
    const float4* d;
    uint32_t i;
    __device__ __forceinline__ static float3 ld3(const float4* p) {
        float x, y, z;
        asm volatile("ld.global.nc.f32 %0, [%3];\n\tld.global.nc.f32 %1, [%3+4];\n\tld.global.nc.f32 %2, [%3+8];"
                     : "=f"(x), "=f"(y), "=f"(z) : "l"(p));
        return f3(x, y, z);
    }
    __device__ __forceinline__ float3 origin() const { return ld3(o + i); }
    __device__ __forceinline__ float3 dir() const { return ld3(d + i); }
};

struct SceneView {
    const Bvh4Node* tlas_nodes;
    const TlasLeaf* tlas_leaves;
    const Bvh4Node* blas_nodes;
    const Bvh8Node* blas8;       // compressed 8-wide BLAS nodes (scenes built with VKB_BLAS_WIDE8)
    const float4* blas_tris;     // 3 per triangle (Morton order within a mesh); v0.w = original triangle id
    uint32_t num_instances;
};

// Traversal work of one ray (instrumented builds only): node visits, triangle tests, instance entries.
struct TraceCount { uint32_t nodes = 0, tris = 0, instances = 0, blas_nodes = 0; };

// Traversal state of one ray: closest hit (ANY == false) or first hit (ANY == true) over
// the two-level BVH, advanced one step (a 4-wide node, an instance entry, a BLAS leaf,
// then a pop) at a time.  Error: overflow/step-limit exits set *err and end the ray with
// the best hit so far.  W8: the BLASes are compressed 8-wide (the TLAS stays 4-wide).
template <bool ANY, bool COUNT = false, bool W8 = false>
struct TraceLane {
    static constexpr int CAP = W8 ? STACK_CAP8 : STACK_CAP;
    RaySpace rs;
    float tbest;
    int node, sp;
    bool found, in_blas, cull;
    const Bvh4Node* nodes;
    const Bvh8Node* nodes8;
    uint32_t tri_base, cur_instance, steps;
    HitRecord hit;

    // Returns false when there is nothing to traverse.
    __device__ __forceinline__ bool start(const SceneView& s, RayRef ray, float tmax) {
        make_space(rs, ray.origin(), ray.dir());
        tbest = tmax; node = 0; sp = 0; steps = 0;
        found = false; in_blas = false; cull = false;
        nodes = s.tlas_nodes; tri_base = 0; cur_instance = 0;
        return s.num_instances != 0;
    }
    // One step; returns true when the ray is finished (hit/found hold the result).
    __device__ __forceinline__ bool step(const SceneView& s, RayRef ray, uint32_t* err, TraceCount* count, TraceStack stk) {
        if (++steps >= TRACE_STEP_LIMIT) { atomicOr(err, 2u); return true; }
        bool respace = false;
        float3 so, sd;
        if (W8 && in_blas && node >= 0) {
            // A compressed 8-wide BLAS node: decode the eight slots' planes on the ray's
            // grid (t = q * 2^e / d + (origin - o) / d), sort the hit slots' keys, descend
            // into the first and push the rest (farthest first).
            if (COUNT) { count->nodes++; count->blas_nodes++; }
            const float4* p = reinterpret_cast<const float4*>(nodes8 + node);
            const float4 h = __ldg(p);
            const uint4 b = __ldg(reinterpret_cast<const uint4*>(p + 1));
            const uint4 qx = __ldg(reinterpret_cast<const uint4*>(p + 2));
            const uint4 qy = __ldg(reinterpret_cast<const uint4*>(p + 3));
            const uint4 qz = __ldg(reinterpret_cast<const uint4*>(p + 4));
            const uint32_t bits = __float_as_uint(h.w);
            const float ax = __uint_as_float((bits & 0xffu) << 23) * rs.idir.x;
            const float ay = __uint_as_float(((bits >> 8) & 0xffu) << 23) * rs.idir.y;
            const float az = __uint_as_float(((bits >> 16) & 0xffu) << 23) * rs.idir.z;
            const float bx = fmaf(h.x, rs.idir.x, -rs.ood.x), by = fmaf(h.y, rs.idir.y, -rs.ood.y), bz = fmaf(h.z, rs.idir.z, -rs.ood.z);
            const bool nx = rs.idir.x < 0.f, ny = rs.idir.y < 0.f, nz = rs.idir.z < 0.f;
            const uint32_t nx0 = nx ? qx.z : qx.x, nx1 = nx ? qx.w : qx.y, fx0 = nx ? qx.x : qx.z, fx1 = nx ? qx.y : qx.w;
            const uint32_t ny0 = ny ? qy.z : qy.x, ny1 = ny ? qy.w : qy.y, fy0 = ny ? qy.x : qy.z, fy1 = ny ? qy.y : qy.w;
            const uint32_t nz0 = nz ? qz.z : qz.x, nz1 = nz ? qz.w : qz.y, fz0 = nz ? qz.x : qz.z, fz1 = nz ? qz.y : qz.w;
            uint32_t key[8];
            #pragma unroll
            for (uint32_t k = 0; k < 8u; ++k) {
                const uint32_t sel = k & 3u;
                const float tn = max3f(fmaf(byte_f(k < 4u ? nx0 : nx1, sel), ax, bx), fmaf(byte_f(k < 4u ? ny0 : ny1, sel), ay, by),
                                       fmaxf(fmaf(byte_f(k < 4u ? nz0 : nz1, sel), az, bz), 0.f));
                const float tf = min3f(fmaf(byte_f(k < 4u ? fx0 : fx1, sel), ax, bx), fmaf(byte_f(k < 4u ? fy0 : fy1, sel), ay, by),
                                       fminf(fmaf(byte_f(k < 4u ? fz0 : fz1, sel), az, bz), tbest));
                // Unused slots are skipped by the count: their inverted boxes could still pass
                // the widened test on a ray from very far away.
                key[k] = (k < b.z && tn <= tf * 1.00000024f) ? ((__float_as_uint(tn) & ~7u) | k) : 0xffffffffu;
                if (ANY) key[k] = far_key8(key[k]);
            }
            sort8(key);
            if (key[0] != 0xffffffffu) {
                const uint32_t imask = bits >> 24, internal = uint32_t(__popc(imask));
                auto child = [&](uint32_t kk) -> int {
                    const uint32_t slot = kk & 7u;
                    return ((imask >> slot) & 1u) ? int(b.x + slot) : ~int((b.y + slot - internal) << 2);
                };
                int pushes = 0;
                #pragma unroll
                for (int i = 1; i < 8; ++i) pushes += key[i] != 0xffffffffu ? 1 : 0;
                if (sp + pushes > CAP) { atomicOr(err, 1u); return true; }
                #pragma unroll
                for (int i = 7; i >= 1; --i)
                    if (key[i] != 0xffffffffu) { stk.put(sp, child(key[i])); ++sp; }
                node = child(key[0]);
                return false;
            }
        } else if (node >= 0) {
            if (COUNT) { count->nodes++; if (in_blas) count->blas_nodes++; }
            const float4* p = reinterpret_cast<const float4*>(nodes + node);
            const uint32_t sx = __float_as_uint(rs.idir.x) >> 31, sy = __float_as_uint(rs.idir.y) >> 31, sz = __float_as_uint(rs.idir.z) >> 31;
            const float4 nx = __ldg(p + sx), fx = __ldg(p + (sx ^ 1u));
            const float4 ny = __ldg(p + 2u + sy), fy = __ldg(p + (3u - sy));
            const float4 nz = __ldg(p + 4u + sz), fz = __ldg(p + (5u - sz));
            const int4 ch = __ldg(reinterpret_cast<const int4*>(p + 6));
            uint32_t k0 = slot_key(nx.x, ny.x, nz.x, fx.x, fy.x, fz.x, rs, tbest, 0u);
            uint32_t k1 = slot_key(nx.y, ny.y, nz.y, fx.y, fy.y, fz.y, rs, tbest, 1u);
            uint32_t k2 = slot_key(nx.z, ny.z, nz.z, fx.z, fy.z, fz.z, rs, tbest, 2u);
            uint32_t k3 = slot_key(nx.w, ny.w, nz.w, fx.w, fy.w, fz.w, rs, tbest, 3u);
            if (ANY) { k0 = far_key(k0); k1 = far_key(k1); k2 = far_key(k2); k3 = far_key(k3); }
            // Ascending keys (nearest first; farthest first for occlusion): a five-exchange
            // sorting network.
            key_order(k0, k1); key_order(k2, k3); key_order(k0, k2); key_order(k1, k3); key_order(k1, k2);
            if (k0 != 0xffffffffu) {
                if (k1 != 0xffffffffu) {
                    const int pushes = 1 + (k2 != 0xffffffffu) + (k3 != 0xffffffffu);
                    if (sp + pushes <= SMEM_STACK) {
                        // all in shared memory: one bound check for the three
                        if (k3 != 0xffffffffu) { stk.r[sp * TRACE_BLOCK] = slot_child(ch, k3); ++sp; }
                        if (k2 != 0xffffffffu) { stk.r[sp * TRACE_BLOCK] = slot_child(ch, k2); ++sp; }
                        stk.r[sp * TRACE_BLOCK] = slot_child(ch, k1); ++sp;
                    } else {
                        if (sp + pushes > CAP) { atomicOr(err, 1u); return true; }
                        if (k3 != 0xffffffffu) { stk.put(sp, slot_child(ch, k3)); ++sp; }
                        if (k2 != 0xffffffffu) { stk.put(sp, slot_child(ch, k2)); ++sp; }
                        stk.put(sp, slot_child(ch, k1)); ++sp;
                    }
                }
                node = slot_child(ch, k0);
                return false;
            }
        } else if (!in_blas) {
            if (COUNT) count->instances++;
            const TlasLeaf* lf = s.tlas_leaves + (~node);
            float4 r0 = __ldg(&lf->w2o[0]), r1 = __ldg(&lf->w2o[1]), r2 = __ldg(&lf->w2o[2]);
            uint4 info = __ldg(reinterpret_cast<const uint4*>(&lf->instance));
            const float3 o = ray.origin(), d = ray.dir();
            so = f3(r0.x * o.x + r0.y * o.y + r0.z * o.z + r0.w, r1.x * o.x + r1.y * o.y + r1.z * o.z + r1.w, r2.x * o.x + r2.y * o.y + r2.z * o.z + r2.w);
            sd = f3(r0.x * d.x + r0.y * d.y + r0.z * d.z, r1.x * d.x + r1.y * d.y + r1.z * d.z, r2.x * d.x + r2.y * d.y + r2.z * d.z);
            cur_instance = info.x;
            if (W8) nodes8 = s.blas8 + info.y;
            else nodes = s.blas_nodes + info.y;
            tri_base = info.z;
            cull = !ANY && (info.w & LEAF_CULL_BACKFACES);
            if (sp >= CAP) { atomicOr(err, 1u); return true; }
            stk.put(sp, SENTINEL);
            ++sp;
            in_blas = true;
            node = 0;
            respace = true;
        } else {
            // BLAS leaf: up to VKB_BLAS_LEAF_MAX triangles in leaf order, ~((first << 2) | (count - 1)).
            uint32_t v = uint32_t(~node), first = v >> 2, cnt = VKB_BLAS_LEAF_MAX == 1 ? 1u : (v & 3u) + 1u;
            for (uint32_t k = 0; k < cnt; ++k) {
                if (COUNT) count->tris++;
                const float4* tp = s.blas_tris + 3u * (tri_base + first + k);
                float4 v0 = __ldg(tp), v1 = __ldg(tp + 1), v2 = __ldg(tp + 2);
                float t, b1, b2;
                if (tri_test(rs, f3(v0.x, v0.y, v0.z), f3(v1.x, v1.y, v1.z), f3(v2.x, v2.y, v2.z), cull, tbest, t, b1, b2)) {
                    tbest = t; found = true;
                    hit.t = t; hit.u = b1; hit.v = b2; hit.tri = tri_base + first + k; hit.inst = cur_instance;
                    if (ANY) return true;
                }
            }
        }
        if (!respace) {
            // pop; leaving an instance (its sentinel) goes back to the world ray
            if (sp == 0) return true;
            --sp;
            node = stk.get(sp);
            if (node != SENTINEL) return false;
            while (node == SENTINEL) {
                in_blas = false;
                nodes = s.tlas_nodes;
                if (sp == 0) return true;
                --sp;
                node = stk.get(sp);
            }
            so = ray.origin();
            sd = ray.dir();
        }
        // the one ray-space set-up of a step (instance entry or exit)
        make_space(rs, so, sd);
        return false;
    }
};

template <bool ANY, bool COUNT = false, bool W8 = false>
__device__ __forceinline__ bool trace_ray(const SceneView& s, RayRef ray, float tmax, HitRecord& hit, uint32_t* err,
                                          TraceCount* count, TraceStack stk) {
    TraceLane<ANY, COUNT, W8> L;
    if (!L.start(s, ray, tmax)) return false;
    while (!L.step(s, ray, err, count, stk)) {}
    hit = L.hit;
    return L.found;
}

}  // namespace vkb
