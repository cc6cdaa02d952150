// Device kernels of the B200 backend: BRDF-atlas bake, LBVH build, and the path
// wavefront (camera -> closest-hit trace -> shade/NEE -> shadow trace -> accumulate).
#pragma once
#include <cstdint>
#include "vkb_device.cuh"
#include "vkb_bvh.cuh"
#include <cooperative_groups.h>

namespace vkb {

// ================================================================ BRDF atlas bake (shaders/environment.slang:14-108)
__device__ __forceinline__ float brdf_cosine(uint32_t col) { float t = float(col) / float(BRDF_SIZE - 1); float t2 = t * t; return t2 * t2; }
__device__ __forceinline__ float brdf_alpha(uint32_t row) {
    if (row == 0) return MIN_ALPHA;
    if (row == BRDF_SIZE - 1) return 1.f;
    return exp2f(log2f(MIN_ALPHA) * (1.f - float(row) / float(BRDF_SIZE - 1)));
}
// openpbr_core.slang:160-171.
__device__ __forceinline__ float dielectric_directional_albedo(float no, float r, float eta, uint32_t samples) {
    if (eta == 1.f) return 0.f;
    if (r == 0.f) return eta <= 0.f ? 1.f : fresnel(no, eta);
    float a = specular_alpha(r), result = 0.f;
    for (uint32_t i = 0; i < samples; ++i) {
        float ux = (float(i) + 0.5f) / float(samples), uy = float(__brev(i) >> 8u) * UINT_SCALE, vh;
        float w = ggx_visible_reflection(no, a, ux, uy, vh);
        result += (eta <= 0.f ? 1.f : fresnel(vh, eta)) * w;
    }
    return result / float(samples);
}
__global__ void k_bake_lut(ushort4* out) {
    uint32_t x = blockIdx.x * blockDim.x + threadIdx.x, y = blockIdx.y;
    if (x >= BRDF_SIZE || y >= BRDF_HEIGHT) return;
    float4 v;
    if (y >= BRDF_SIZE) {
        const uint32_t n = BRDF_ALBEDO_SIZE;
        uint32_t cx = x % n, cy = (y - BRDF_SIZE) % n, slice = ((y - BRDF_SIZE) / n) * 2u + x / n;
        if (slice > BRDF_IOR_STEPS) v = make_float4(0.f, 0.f, 0.f, 0.f);
        else {
            float no = fmaxf(float(cx) / float(n - 1), MIN_ALPHA), r = float(cy) / float(n - 1), q = float(slice) / float(BRDF_IOR_STEPS);
            float eta = slice == BRDF_IOR_STEPS ? 0.f : q / fmaxf(1.f - q, POSITIVE_EPSILON);
            v = make_float4(dielectric_directional_albedo(no, r, eta, DIELECTRIC_ALBEDO_SAMPLES), 0.f, 0.f, 1.f);
        }
    } else {
        float s0 = 0.f, s1 = 0.f, s2 = 0.f, nv = brdf_cosine(x), alpha = brdf_alpha(y), average = 0.f;
        for (uint32_t i = 0; i < ENVIRONMENT_SAMPLES; ++i) {
            float ux = (float(i) + 0.5f) / float(ENVIRONMENT_SAMPLES), uy = float(__brev(i)) * RADICAL_INVERSE_SCALE, vh;
            float g = ggx_visible_reflection(nv, alpha, ux, uy, vh);
            float f = powf(1.f - vh, 5.f);
            s0 += (1.f - f) * g; s1 += f * g; s2 += vh * powf(1.f - vh, 6.f) * g;
        }
        if (x == 0) {
            for (uint32_t j = 0; j < BRDF_SIZE; ++j) {
                float c = brdf_cosine(j);
                float interval = 0.5f * (brdf_cosine(min(j + 1u, BRDF_SIZE - 1u)) - brdf_cosine(j > 0 ? j - 1u : 0u));
                for (uint32_t i = 0; i < ENVIRONMENT_SAMPLES; ++i) {
                    float ux = (float(i) + 0.5f) / float(ENVIRONMENT_SAMPLES), uy = float(__brev(i)) * RADICAL_INVERSE_SCALE, vh;
                    average += interval * 2.f * c * ggx_visible_reflection(c, alpha, ux, uy, vh);
                }
            }
            average /= float(ENVIRONMENT_SAMPLES);
        }
        v = make_float4(s0 / float(ENVIRONMENT_SAMPLES), s1 / float(ENVIRONMENT_SAMPLES), s2 / float(ENVIRONMENT_SAMPLES), average);
    }
    out[y * BRDF_SIZE + x] = make_ushort4(__half_as_ushort(__float2half_rn(v.x)), __half_as_ushort(__float2half_rn(v.y)),
                                          __half_as_ushort(__float2half_rn(v.z)), __half_as_ushort(__float2half_rn(v.w)));
}

// ================================================================ LBVH build
// Object-space triangle boxes of one mesh (index buffer relative to the mesh's vertices).
__global__ void k_tri_boxes(uint32_t n, const uint32_t* idx, const float4* pos, float4* lo, float4* hi) {
    for (uint32_t t = blockIdx.x * blockDim.x + threadIdx.x; t < n; t += gridDim.x * blockDim.x) {
        float4 a = pos[idx[3 * t]], b = pos[idx[3 * t + 1]], c = pos[idx[3 * t + 2]];
        lo[t] = make_float4(fminf(a.x, fminf(b.x, c.x)), fminf(a.y, fminf(b.y, c.y)), fminf(a.z, fminf(b.z, c.z)), 0.f);
        hi[t] = make_float4(fmaxf(a.x, fmaxf(b.x, c.x)), fmaxf(a.y, fmaxf(b.y, c.y)), fmaxf(a.z, fmaxf(b.z, c.z)), 0.f);
    }
}
// Instance rows -> world->object rows and world boxes of the mesh box's 8 corners,
// each coordinate ((m0 x + m1 y) + m2 z) + m3 without contraction (bit-exact boxes).
__global__ void k_instances(uint32_t n, const float4* o2w, const uint4* info, const MeshInfo* meshes, float4* w2o, float4* lo, float4* hi) {
    for (uint32_t i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x) {
        float4 r0 = o2w[3 * i], r1 = o2w[3 * i + 1], r2 = o2w[3 * i + 2];
        const MeshInfo& m = meshes[info[i].x];
        float l[3] = {INFINITY, INFINITY, INFINITY}, h[3] = {-INFINITY, -INFINITY, -INFINITY};
        for (int k = 0; k < 8; ++k) {
            float p[3] = {k & 1 ? m.hi[0] : m.lo[0], k & 2 ? m.hi[1] : m.lo[1], k & 4 ? m.hi[2] : m.lo[2]};
            float4 rr[3] = {r0, r1, r2};
            for (int a = 0; a < 3; ++a) {
                float v = __fmul_rn(rr[a].x, p[0]);
                v = __fadd_rn(v, __fmul_rn(rr[a].y, p[1]));
                v = __fadd_rn(v, __fmul_rn(rr[a].z, p[2]));
                v = __fadd_rn(v, rr[a].w);
                l[a] = fminf(l[a], v); h[a] = fmaxf(h[a], v);
            }
        }
        // Intersected with the box of the transformed bounding sphere (centre c' = M c + t,
        // half extent r |row a| per axis, widened by 1e-5 relative plus 1e-6 of the
        // magnitudes for fp32 rounding): much tighter for round, rotated meshes.
        if (m.sphere[3] >= 0.f) {
            const float c[3] = {m.sphere[0], m.sphere[1], m.sphere[2]}, r = m.sphere[3];
            float4 rr[3] = {r0, r1, r2};
            for (int a = 0; a < 3; ++a) {
                float cw = __fmul_rn(rr[a].x, c[0]);
                cw = __fadd_rn(cw, __fmul_rn(rr[a].y, c[1]));
                cw = __fadd_rn(cw, __fmul_rn(rr[a].z, c[2]));
                cw = __fadd_rn(cw, rr[a].w);
                float nn = __fmul_rn(rr[a].x, rr[a].x);
                nn = __fadd_rn(nn, __fmul_rn(rr[a].y, rr[a].y));
                nn = __fadd_rn(nn, __fmul_rn(rr[a].z, rr[a].z));
                const float ext = __fmul_rn(r, __fsqrt_rn(nn));
                const float mag = __fadd_rn(__fadd_rn(fabsf(cw), fabsf(rr[a].w)), ext);
                const float half = __fadd_rn(__fmul_rn(ext, 1.00001f), __fmul_rn(mag, 1e-6f));
                l[a] = fmaxf(l[a], __fsub_rn(cw, half));
                h[a] = fminf(h[a], __fadd_rn(cw, half));
            }
        }
        lo[i] = make_float4(l[0], l[1], l[2], 0.f);
        hi[i] = make_float4(h[0], h[1], h[2], 0.f);
        // Affine inverse of the 3x4 rows.
        float a00 = r0.x, a01 = r0.y, a02 = r0.z, a10 = r1.x, a11 = r1.y, a12 = r1.z, a20 = r2.x, a21 = r2.y, a22 = r2.z;
        float c00 = a11 * a22 - a12 * a21, c01 = a02 * a21 - a01 * a22, c02 = a01 * a12 - a02 * a11;
        float c10 = a12 * a20 - a10 * a22, c11 = a00 * a22 - a02 * a20, c12 = a02 * a10 - a00 * a12;
        float c20 = a10 * a21 - a11 * a20, c21 = a01 * a20 - a00 * a21, c22 = a00 * a11 - a01 * a10;
        float det = a00 * c00 + a01 * c10 + a02 * c20, id = 1.f / det;
        float i00 = c00 * id, i01 = c01 * id, i02 = c02 * id, i10 = c10 * id, i11 = c11 * id, i12 = c12 * id, i20 = c20 * id, i21 = c21 * id, i22 = c22 * id;
        w2o[3 * i] = make_float4(i00, i01, i02, -(i00 * r0.w + i01 * r1.w + i02 * r2.w));
        w2o[3 * i + 1] = make_float4(i10, i11, i12, -(i10 * r0.w + i11 * r1.w + i12 * r2.w));
        w2o[3 * i + 2] = make_float4(i20, i21, i22, -(i20 * r0.w + i21 * r1.w + i22 * r2.w));
    }
}
// Changed object bytes of an instance update (rt.rs:1465-1476 counts the object bytes
// that differ): 48 for every 3x4 row block whose bits differ from the installed one.
__global__ void k_changed_rows(uint32_t n, const uint4* next, const uint4* cur, unsigned long long* changed) {
    unsigned long long local = 0;
    for (uint32_t i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x) {
        const uint4 a0 = next[3 * i], a1 = next[3 * i + 1], a2 = next[3 * i + 2];
        const uint4 b0 = cur[3 * i], b1 = cur[3 * i + 1], b2 = cur[3 * i + 2];
        const uint32_t d = (a0.x ^ b0.x) | (a0.y ^ b0.y) | (a0.z ^ b0.z) | (a0.w ^ b0.w) | (a1.x ^ b1.x) | (a1.y ^ b1.y) | (a1.z ^ b1.z) |
                           (a1.w ^ b1.w) | (a2.x ^ b2.x) | (a2.y ^ b2.y) | (a2.z ^ b2.z) | (a2.w ^ b2.w);
        if (d) local += 48ull;
    }
    for (int off = 16; off > 0; off >>= 1) local += __shfl_xor_sync(0xffffffffu, local, off);
    if ((threadIdx.x & 31u) == 0u && local) atomicAdd(changed, local);
}
// Centroid box: bounds[0..2] flipped minima, bounds[3..5] flipped maxima.
__global__ void k_centroid_box(uint32_t n, const float4* lo, const float4* hi, uint32_t* bounds) {
    uint32_t mn[3] = {0xffffffffu, 0xffffffffu, 0xffffffffu}, mx[3] = {0u, 0u, 0u};
    for (uint32_t i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x) {
        float4 a = lo[i], b = hi[i];
        float c[3] = {__fmul_rn(__fadd_rn(a.x, b.x), 0.5f), __fmul_rn(__fadd_rn(a.y, b.y), 0.5f), __fmul_rn(__fadd_rn(a.z, b.z), 0.5f)};
        for (int k = 0; k < 3; ++k) { uint32_t f = float_flip(c[k]); mn[k] = min(mn[k], f); mx[k] = max(mx[k], f); }
    }
    for (int k = 0; k < 3; ++k)
        for (int off = 16; off > 0; off >>= 1) {
            mn[k] = min(mn[k], __shfl_xor_sync(0xffffffffu, mn[k], off));
            mx[k] = max(mx[k], __shfl_xor_sync(0xffffffffu, mx[k], off));
        }
    if ((threadIdx.x & 31) == 0)
        for (int k = 0; k < 3; ++k) { atomicMin(&bounds[k], mn[k]); atomicMax(&bounds[3 + k], mx[k]); }
}
// split_large: a box wider on some axis than a quarter of the centroid box's widest
// extent gets bit 30 over its 30-bit code, so the hierarchy's root split separates such
// boxes (a terrain instance) from the rest and their size does not inflate the boxes
// of every node on their Morton path.
__global__ void k_morton(uint32_t n, const float4* lo, const float4* hi, const uint32_t* bounds, uint32_t* codes, uint32_t* ids, bool split_large) {
    float3 slo = f3(float_unflip(bounds[0]), float_unflip(bounds[1]), float_unflip(bounds[2]));
    float3 shi = f3(float_unflip(bounds[3]), float_unflip(bounds[4]), float_unflip(bounds[5]));
    float3 ext = f3(__fsub_rn(shi.x, slo.x), __fsub_rn(shi.y, slo.y), __fsub_rn(shi.z, slo.z));
    const float big = __fmul_rn(fmaxf(ext.x, fmaxf(ext.y, ext.z)), 0.25f);
    for (uint32_t i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x) {
        const float4 l = lo[i], h = hi[i];
        const float w = fmaxf(__fsub_rn(h.x, l.x), fmaxf(__fsub_rn(h.y, l.y), __fsub_rn(h.z, l.z)));
        codes[i] = morton_code(l, h, slo, ext) | (split_large && w > big ? 1u << 30 : 0u);
        ids[i] = i;
    }
}
__device__ __forceinline__ int lbvh_delta(const uint32_t* codes, int n, int i, int j) {
    if (j < 0 || j >= n) return -1;
    uint32_t a = codes[i], b = codes[j];
    if (a == b) return 32 + __clz(uint32_t(i ^ j));
    return __clz(a ^ b);
}
// Karras 2012, Algorithm 2: one internal node per thread; parents encoded node*2+side.
__global__ void k_karras(int n, const uint32_t* codes, BvhNode* nodes, uint32_t* leaf_parent, uint32_t* node_parent, uint32_t* counters) {
    for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < n - 1; i += gridDim.x * blockDim.x) {
        int d = lbvh_delta(codes, n, i, i + 1) - lbvh_delta(codes, n, i, i - 1) > 0 ? 1 : -1;
        int dmin = lbvh_delta(codes, n, i, i - d);
        int lmax = 2;
        while (lbvh_delta(codes, n, i, i + lmax * d) > dmin) lmax <<= 1;
        int l = 0;
        for (int t = lmax >> 1; t >= 1; t >>= 1)
            if (lbvh_delta(codes, n, i, i + (l + t) * d) > dmin) l += t;
        int j = i + l * d;
        int dnode = lbvh_delta(codes, n, i, j);
        int s = 0, t = l;
        do {
            t = (t + 1) >> 1;
            if (lbvh_delta(codes, n, i, i + (s + t) * d) > dnode) s += t;
        } while (t > 1);
        int gamma = i + s * d + min(d, 0);
        int left = min(i, j) == gamma ? ~gamma : gamma;
        int right = max(i, j) == gamma + 1 ? ~(gamma + 1) : gamma + 1;
        nodes[i].d = make_int4(left, right, 0, 0);
        if (left < 0) leaf_parent[~left] = uint32_t(i) * 2u; else node_parent[left] = uint32_t(i) * 2u;
        if (right < 0) leaf_parent[~right] = uint32_t(i) * 2u + 1u; else node_parent[right] = uint32_t(i) * 2u + 1u;
        counters[i] = 0u;
        if (i == 0) node_parent[0] = 0xffffffffu;
    }
}
__device__ __forceinline__ void store_child(BvhNode* nodes, uint32_t node, uint32_t side, float4 lo, float4 hi) {
    BvhNode& n = nodes[node];
    if (side == 0) { n.a = make_float4(lo.x, hi.x, lo.y, hi.y); n.c.x = lo.z; n.c.y = hi.z; }
    else { n.b = make_float4(lo.x, hi.x, lo.y, hi.y); n.c.z = lo.z; n.c.w = hi.z; }
}
// Bottom-up refit: the second child to arrive at a node merges both boxes upward.
__global__ void k_refit(int n, const uint32_t* sorted_ids, const float4* lo, const float4* hi, BvhNode* nodes,
                        const uint32_t* leaf_parent, const uint32_t* node_parent, uint32_t* counters) {
    for (int k = blockIdx.x * blockDim.x + threadIdx.x; k < n; k += gridDim.x * blockDim.x) {
        uint32_t id = sorted_ids[k];
        float4 blo = lo[id], bhi = hi[id];
        uint32_t pref = leaf_parent[k];
        for (int guard = 0; guard < 128 && pref != 0xffffffffu; ++guard) {
            uint32_t node = pref >> 1, side = pref & 1u;
            store_child(nodes, node, side, blo, bhi);
            __threadfence();
            if (atomicAdd(&counters[node], 1u) == 0u) break;
            __threadfence();
            const float4* p = reinterpret_cast<const float4*>(nodes + node);
            float4 a = __ldcg(p), b = __ldcg(p + 1), c = __ldcg(p + 2);
            blo = make_float4(fminf(a.x, b.x), fminf(a.z, b.z), fminf(c.x, c.z), 0.f);
            bhi = make_float4(fmaxf(a.y, b.y), fmaxf(a.w, b.w), fmaxf(c.y, c.w), 0.f);
            pref = node_parent[node];
        }
    }
}
// ---- PLOC (Meister & Bittner 2018, "Parallel Locally-Ordered Clustering for Bounding
// Volume Hierarchy Construction"): clusters in Morton order; each picks the neighbour
// within PLOC_RADIUS positions whose merged box has the least surface area; mutual
// pairs merge into a new node.  Ties are broken by a strict order on pairs, so the
// closest pair of every pass is mutual and every pass merges.  A cluster is (lo.xyz, ref) / (hi.xyz, -): ref ~k for the k-th leaf in Morton
// order, else an internal node index.
constexpr int PLOC_RADIUS = 16;
constexpr int PLOC_BLOCK = 256;
__device__ __forceinline__ float merged_area(float3 alo, float3 ahi, float3 blo, float3 bhi) {
    float dx = fmaxf(ahi.x, bhi.x) - fminf(alo.x, blo.x);
    float dy = fmaxf(ahi.y, bhi.y) - fminf(alo.y, blo.y);
    float dz = fmaxf(ahi.z, bhi.z) - fminf(alo.z, blo.z);
    float a = dx * dy + dy * dz + dz * dx;
    return a == a ? a : INFINITY;  // a NaN box sorts last, by index like every tie
}
__global__ void k_ploc_init(uint32_t n, const uint32_t* sorted_ids, const float4* lo, const float4* hi, float4* clo, float4* chi) {
    for (uint32_t k = blockIdx.x * blockDim.x + threadIdx.x; k < n; k += gridDim.x * blockDim.x) {
        uint32_t id = sorted_ids[k];
        float4 a = lo[id], b = hi[id];
        clo[k] = make_float4(a.x, a.y, a.z, __int_as_float(~int(k)));
        chi[k] = make_float4(b.x, b.y, b.z, 0.f);
    }
}
// Nearest neighbour of every cluster: one block covers PLOC_BLOCK clusters and stages
// their boxes plus PLOC_RADIUS on either side in shared memory.  Launch with
// blockDim.x == PLOC_BLOCK and one block per PLOC_BLOCK clusters.
__global__ void __launch_bounds__(PLOC_BLOCK) k_ploc_nn(uint32_t c, const float4* clo, const float4* chi, uint32_t* nn) {
    __shared__ float3 slo[PLOC_BLOCK + 2 * PLOC_RADIUS], shi[PLOC_BLOCK + 2 * PLOC_RADIUS];
    const int base = int(blockIdx.x) * PLOC_BLOCK - PLOC_RADIUS;
    for (int t = threadIdx.x; t < PLOC_BLOCK + 2 * PLOC_RADIUS; t += PLOC_BLOCK) {
        int g = base + t;
        if (g >= 0 && g < int(c)) {
            float4 a = clo[g], b = chi[g];
            slo[t] = f3(a.x, a.y, a.z); shi[t] = f3(b.x, b.y, b.z);
        }
    }
    __syncthreads();
    const int i = int(blockIdx.x) * PLOC_BLOCK + int(threadIdx.x);
    if (i >= int(c)) return;
    const int li = int(threadIdx.x) + PLOC_RADIUS;
    const float3 alo = slo[li], ahi = shi[li];
    const int j0 = max(0, i - PLOC_RADIUS), j1 = min(int(c) - 1, i + PLOC_RADIUS);
    float best = INFINITY;
    int best_j = -1, best_d = 0, best_m = 0;
    for (int j = j0; j <= j1; ++j) {
        if (j == i) continue;
        float a = merged_area(alo, ahi, slo[j - base], shi[j - base]);
        int d = abs(i - j), m = min(i, j);
        // Pair order (area, index distance, parity of the lower index, lower index): a
        // strict order that pairs equal neighbours as (0,1), (2,3), ... rather than
        // chaining them all to one cluster.
        bool better = best_j < 0 || a < best ||
                      (a == best && (d < best_d || (d == best_d && ((m & 1) < (best_m & 1) || ((m & 1) == (best_m & 1) && m < best_m)))));
        if (better) { best = a; best_j = j; best_d = d; best_m = m; }
    }
    nn[i] = uint32_t(best_j);
}
// Per cluster: bit 32 = merges (mutual pair, lower index), bit 0 = survives.
__global__ void k_ploc_flags(uint32_t c, const uint32_t* nn, unsigned long long* flags) {
    for (uint32_t i = blockIdx.x * blockDim.x + threadIdx.x; i < c; i += gridDim.x * blockDim.x) {
        uint32_t j = nn[i];
        bool mutual = nn[j] == i;
        flags[i] = ((mutual && i < j) ? (1ull << 32) : 0ull) | ((mutual && i > j) ? 0ull : 1ull);
    }
}
// Merge mutual pairs into nodes next_free-1, next_free-2, ... (by exclusive prefix of
// merges) and compact the surviving clusters; counts = {clusters left, merges}.
__global__ void k_ploc_merge(uint32_t c, const uint32_t* nn, const unsigned long long* offs, const float4* clo, const float4* chi,
                             uint32_t next_free, BvhNode* nodes, uint32_t* leaf_parent, uint32_t* node_parent, uint32_t* counters,
                             float4* clo2, float4* chi2, uint32_t* counts) {
    for (uint32_t i = blockIdx.x * blockDim.x + threadIdx.x; i < c; i += gridDim.x * blockDim.x) {
        uint32_t j = nn[i];
        bool mutual = nn[j] == i;
        bool merge = mutual && i < j, keep = !(mutual && i > j);
        unsigned long long o = offs[i];
        if (i == c - 1) {
            counts[0] = uint32_t(o & 0xffffffffull) + (keep ? 1u : 0u);
            counts[1] = uint32_t(o >> 32) + (merge ? 1u : 0u);
        }
        if (!keep) continue;
        uint32_t pos = uint32_t(o & 0xffffffffull);
        float4 alo = clo[i], ahi = chi[i];
        if (!merge) { clo2[pos] = alo; chi2[pos] = ahi; continue; }
        // next_free == c - 1 before every pass and a pass merges at most c / 2 pairs, so
        // the offset is below next_free; the test only keeps a broken caller in bounds.
        if (uint32_t(o >> 32) >= next_free) continue;
        float4 blo = clo[j], bhi = chi[j];
        uint32_t node = next_free - 1u - uint32_t(o >> 32);
        int ra = __float_as_int(alo.w), rb = __float_as_int(blo.w);
        BvhNode nd;
        nd.a = make_float4(alo.x, ahi.x, alo.y, ahi.y);
        nd.b = make_float4(blo.x, bhi.x, blo.y, bhi.y);
        nd.c = make_float4(alo.z, ahi.z, blo.z, bhi.z);
        nd.d = make_int4(ra, rb, 0, 0);
        nodes[node] = nd;
        if (ra < 0) leaf_parent[~ra] = node * 2u; else node_parent[ra] = node * 2u;
        if (rb < 0) leaf_parent[~rb] = node * 2u + 1u; else node_parent[rb] = node * 2u + 1u;
        counters[node] = 0u;
        if (node == 0u) node_parent[0] = 0xffffffffu;
        clo2[pos] = make_float4(fminf(alo.x, blo.x), fminf(alo.y, blo.y), fminf(alo.z, blo.z), __int_as_float(int(node)));
        chi2[pos] = make_float4(fmaxf(ahi.x, bhi.x), fmaxf(ahi.y, bhi.y), fmaxf(ahi.z, bhi.z), 0.f);
    }
}
// A one-primitive tree: root with the leaf on the left and an empty right box.
__global__ void k_single_leaf(const float4* lo, const float4* hi, BvhNode* nodes) {
    BvhNode n;
    n.a = make_float4(lo[0].x, hi[0].x, lo[0].y, hi[0].y);
    n.b = make_float4(INFINITY, -INFINITY, INFINITY, -INFINITY);
    n.c = make_float4(lo[0].z, hi[0].z, INFINITY, -INFINITY);
    n.d = make_int4(~0, ~0, 0, 0);
    nodes[0] = n;
}
// ---- 4-wide traversal nodes from a binary tree (parent links, root 0 with parent ~0u).
// Depth parity of every internal node, by walking its parent links to the root.
__global__ void k_bvh_parity(uint32_t n_internal, const uint32_t* node_parent, uint8_t* odd) {
    for (uint32_t i = blockIdx.x * blockDim.x + threadIdx.x; i < n_internal; i += gridDim.x * blockDim.x) {
        uint32_t d = 0, j = i;
        for (uint32_t guard = 0; guard < n_internal; ++guard) {
            uint32_t pr = node_parent[j];
            if (pr == 0xffffffffu) break;
            j = pr >> 1;
            ++d;
        }
        odd[i] = uint8_t(d & 1u);
    }
}
// Child slot k of a 4-wide node: box planes and reference.
__device__ __host__ __forceinline__ void set_slot(Bvh4Node& q, int k, float lx, float hx, float ly, float hy, float lz, float hz, int ref) {
    float* pl = reinterpret_cast<float*>(q.plane);
    pl[0 * 4 + k] = lx; pl[1 * 4 + k] = hx; pl[2 * 4 + k] = ly; pl[3 * 4 + k] = hy; pl[4 * 4 + k] = lz; pl[5 * 4 + k] = hz;
    reinterpret_cast<int*>(&q.child)[k] = ref;
}
// The slots of the 4-wide node for binary node b: each leaf child keeps its slot, each
// internal child gives its own two children (internal references stay binary indices).
__device__ __host__ __forceinline__ Bvh4Node collapse_node(const BvhNode* n2, const BvhNode& b) {
    Bvh4Node q;
    int k = 0;
    const int refs[2] = {b.d.x, b.d.y};
    const float box[2][6] = {{b.a.x, b.a.y, b.a.z, b.a.w, b.c.x, b.c.y}, {b.b.x, b.b.y, b.b.z, b.b.w, b.c.z, b.c.w}};
    for (int side = 0; side < 2; ++side) {
        if (refs[side] >= 0) {
            const BvhNode c = n2[refs[side]];
            set_slot(q, k++, c.a.x, c.a.y, c.a.z, c.a.w, c.c.x, c.c.y, c.d.x);
            set_slot(q, k++, c.b.x, c.b.y, c.b.z, c.b.w, c.c.z, c.c.w, c.d.y);
        } else {
            set_slot(q, k++, box[side][0], box[side][1], box[side][2], box[side][3], box[side][4], box[side][5], refs[side]);
        }
    }
    for (; k < 4; ++k) set_slot(q, k, INFINITY, -INFINITY, INFINITY, -INFINITY, INFINITY, -INFINITY, ~0);
    q.pad = make_int4(0, 0, 0, 0);
    return q;
}
// Every even-depth internal node i of the binary tree becomes 4-wide node i (the odd
// depths are folded into their parents; their slots stay unused).
__global__ void k_collapse4(uint32_t n_internal, const BvhNode* n2, const uint8_t* odd, Bvh4Node* n4) {
    for (uint32_t i = blockIdx.x * blockDim.x + threadIdx.x; i < n_internal; i += gridDim.x * blockDim.x) {
        if (odd[i]) continue;
        n4[i] = collapse_node(n2, n2[i]);
    }
}
// Triangles of one mesh in Morton order, v0.w = original triangle id.
__global__ void k_sorted_tris(uint32_t n, const uint32_t* sorted_ids, const uint32_t* idx, const float4* pos, float4* tris) {
    for (uint32_t k = blockIdx.x * blockDim.x + threadIdx.x; k < n; k += gridDim.x * blockDim.x) {
        uint32_t t = sorted_ids[k];
        float4 a = pos[idx[3 * t]], b = pos[idx[3 * t + 1]], c = pos[idx[3 * t + 2]];
        tris[3 * k] = make_float4(a.x, a.y, a.z, __uint_as_float(t));
        tris[3 * k + 1] = make_float4(b.x, b.y, b.z, 0.f);
        tris[3 * k + 2] = make_float4(c.x, c.y, c.z, 0.f);
    }
}
// Vertex normals of one mesh's triangles in the same order (zeros where the mesh has none).
__global__ void k_sorted_nrm(uint32_t n, const uint32_t* sorted_ids, const uint32_t* idx, const float4* nrm, float4* out) {
    for (uint32_t k = blockIdx.x * blockDim.x + threadIdx.x; k < n; k += gridDim.x * blockDim.x) {
        uint32_t t = sorted_ids[k];
        out[3 * k] = nrm[idx[3 * t]]; out[3 * k + 1] = nrm[idx[3 * t + 1]]; out[3 * k + 2] = nrm[idx[3 * t + 2]];
    }
}
// A GPU-built BLAS's leaf references in the traversal's BLAS encoding: the binary builders
// reference leaf k as ~k, the BLAS step reads ~(first << 2 | count - 1) (one triangle each).
__global__ void k_blas_leaf_refs(uint32_t n_internal, BvhNode* nodes) {
    for (uint32_t i = blockIdx.x * blockDim.x + threadIdx.x; i < n_internal; i += gridDim.x * blockDim.x) {
        int4 d = nodes[i].d;
        if (d.x < 0) d.x = ~int(uint32_t(~d.x) << 2);
        if (d.y < 0) d.y = ~int(uint32_t(~d.y) << 2);
        nodes[i].d = d;
    }
}
__global__ void k_tlas_leaves(uint32_t n, const uint32_t* sorted_ids, const float4* w2o, const uint4* info, const MeshInfo* meshes,
                              const vkb_material* materials, TlasLeaf* leaves) {
    for (uint32_t k = blockIdx.x * blockDim.x + threadIdx.x; k < n; k += gridDim.x * blockDim.x) {
        uint32_t i = sorted_ids[k];
        TlasLeaf lf;
        lf.w2o[0] = w2o[3 * i]; lf.w2o[1] = w2o[3 * i + 1]; lf.w2o[2] = w2o[3 * i + 2];
        uint4 in = info[i];
        lf.instance = i;
        lf.node_offset = meshes[in.x].node_offset;
        lf.tri_offset = meshes[in.x].tri_offset;
        lf.flags = (materials[in.y].flags & 2u) ? 0u : LEAF_CULL_BACKFACES;
        leaves[k] = lf;
    }
}

// ================================================================ path wavefront
// One render job: an installed scene, its profile and outputs.  A wave holds, for
// every job scheduled in it, `wave_samples` consecutive samples of all its pixels in
// path slots [slot_base, slot_base + npix*wave_samples).  A plain render is a batch
// of one job; batched renders share every wave among many jobs.
struct Job {
    SceneView sv;
    const float4* o2w; const float4* w2o; const uint4* inst_info; const MeshInfo* meshes;
    const float4* tri_nrm;   // vertex normals of every triangle in BLAS leaf order (3 per triangle, beside sv.blas_tris)
    const vkb_material* materials; const vkb_light* lights; uint32_t num_lights;
    const LightTreeNode* tree; uint32_t tree_nodes;
    vkb_camera cam; vkb_environment env;
    uint32_t spp, seed, bounces[4], caustics, sample_mask;
    float clamp_direct, clamp_indirect, light_threshold;
    uint32_t npix, first_sample;
    uint32_t wave_first, wave_samples, slot_base, pixel_base;  // this wave
    float4* accum; uint32_t* primary_ids; float4* out;
    // Adaptive sampling (path.slang:1792-1837,1963-1966): per-pixel moments (mean, M2 of
    // the accumulated RGBA values) and a state word (bit 0/1: settled at an even/odd
    // sample, bit 2: stopped); one sample per wave.
    uint32_t adaptive, adaptive_min;
    float adaptive_threshold;
    float4* ad_mean; float4* ad_m2; uint32_t* ad_state;
    // Denoiser guides (path.slang:1549-1571,1956-1963), single-job renders only: per-pixel
    // sums (albedo + coverage, normal) in sample order and the mean planes written at resolve.
    float4* guide_accum; float4* guide_albedo; float4* guide_normal;
    // Image environment (env_w == 0: none): RGBA texels, the proposal (cumulative mass,
    // density), strength x colour, and the rotation (world d -> d R, row-major).
    const float4* env_img; const float2* env_dist;
    uint32_t env_w, env_h;
    float env_scale[3];
    float env_rot[9];
    // Emissive meshes (em_tris == 0: none): per instance its source (~0u: none), per source
    // its instance and the cumulative triangle count through it, the weight tree (node 1
    // the root, leaves from em_leaves on), and the meshes' own index order (indices
    // relative to the mesh's vertices) for the corners of a sampled triangle.
    const uint32_t* em_inst_source; const uint2* em_sources; const float* em_tree;
    const uint32_t* indices; const float4* vpos;
    uint32_t em_count, em_tris, em_leaves;
};
constexpr uint32_t AD_STOPPED = 4u;
// Radiance-cache hooks of a wave.  mode 1 (query): a path reaching vertex `vertex`
// (0 = camera hit) appends a cache record (counters[9] counts them, `capacity` bounds
// them) and stops; the query kernel adds throughput x the cached outgoing radiance.
// mode 2 (record): vertex v >= 1 of the path in slot s writes its record, throughput and
// radiance at position s * vmax + v - 1 and sets flag[position]; the training set is
// compacted from the flags in position order, so it does not depend on thread timing.
struct CacheParams {
    uint32_t mode, vertex, capacity, vmax;
    float4 box_lo, box_scale;      // world -> [0,1]^3
    float4* rec;                   // 4 float4 per record
    uint32_t* slot;                // mode 1: path slot of each record
    float4* aux;                   // mode 2: throughput, radiance at the vertex (2 float4 per record)
    uint32_t* flag;                // mode 2: position holds a record
};

struct PathParams {
    Job job0;             // single-job waves read their job from the kernel parameters
    const Job* jobs; uint32_t njobs;
    uint32_t* slot_job;   // batched waves: job index of each path slot
    Lut lut; const float* filter;
    float4* ray_o[2]; float4* ray_d[2];
    float4* hit; uint32_t* hit_inst;
    float4* thr; float4* rad; uint2* rng;
    float4* sa_o; float4* sa_d; float4* sa_c;
    float4* sb_o; float4* sb_d; float4* sb_c;
    // [0],[1] ray counts, [2] shadow count, [3] ext rays, [4] shadow rays, [5] dropped light,
    // [6] dropped paths, [7] path slots of this wave, [8] pixels of this wave's jobs
    // [9] radiance-cache records of this wave, [10] adaptive pixel-samples skipped
    uint32_t* counters;
    unsigned long long* work;  // instrumented traversal: closest nodes, tris, instances, blas nodes; shadow nodes, tris, blas nodes
    uint32_t* err;
    CacheParams cache;
    float4* guide;        // guide renders: the camera hit's guide albedo and normal per path slot (2 float4)
    // Waves with an image environment or emissive meshes: each slot's environment and
    // mesh shadow rays (origin+tmax, direction, contribution), and the vertex and pdf of
    // the BSDF sample that made its current ray (xyz, w).
    float4* sc_o; float4* sc_d; float4* sc_c;
    float4* sd_o; float4* sd_d; float4* sd_c;
    float4* prev;
};
constexpr uint32_t META_NONFINITE = 0x80000000u;
constexpr uint32_t SH_TRACE_A = 1u, SH_HAS_B = 2u, SH_TRACE_B = 4u, SH_DIRECT = 8u, SH_HAS_C = 16u, SH_HAS_D = 32u;

// ---------------------------------------------------------------- image environment
// vork_prelude.slang:78-85.
__device__ __forceinline__ float2 equirect_uv(float3 d) {
    if (d.x == 0.f && d.z == 0.f) return make_float2(0.5f, d.y > 0.f ? 0.f : 1.f);
    return make_float2(atan2f(d.z, d.x) / TAU_F + 0.5f, atan2f(sqrtf(d.x * d.x + d.z * d.z), d.y) / PI_F);
}
// World -> environment (row vector times the rotation) and back (path.slang:985-992).
__device__ __forceinline__ float3 env_local(const Job& J, float3 d) {
    const float* m = J.env_rot;
    return normalize(f3(d.x * m[0] + d.y * m[3] + d.z * m[6], d.x * m[1] + d.y * m[4] + d.z * m[7], d.x * m[2] + d.y * m[5] + d.z * m[8]));
}
__device__ __forceinline__ float3 env_world(const Job& J, float3 l) {
    const float* m = J.env_rot;
    return normalize(f3(m[0] * l.x + m[1] * l.y + m[2] * l.z, m[3] * l.x + m[4] * l.y + m[5] * l.z, m[6] * l.x + m[7] * l.y + m[8] * l.z));
}
__device__ __forceinline__ float fracf(float x) { return x - floorf(x); }
// environment_radiance, wrap mode 0 (vork_prelude.slang:306-330): bilinear by differences.
__device__ float3 env_lookup(const Job& J, float2 uv) {
    const int w = int(J.env_w), h = int(J.env_h);
    const float px = fracf(uv.x) * float(w) - 0.5f, py = clampf(uv.y, 0.f, 1.f) * float(h) - 0.5f;
    const int cx = int(floorf(px)), cy = int(floorf(py));
    const float fx = fracf(px), fy = fracf(py);
    const int x0 = (cx + w) % w, x1 = (x0 + 1) % w, y0 = min(max(cy, 0), h - 1), y1 = min(max(cy + 1, 0), h - 1);
    const float4 a = __ldg(J.env_img + y0 * w + x0), b = __ldg(J.env_img + y0 * w + x1);
    const float4 c = __ldg(J.env_img + y1 * w + x0), d = __ldg(J.env_img + y1 * w + x1);
    const float3 top = f3(a.x, a.y, a.z) + (f3(b.x, b.y, b.z) - f3(a.x, a.y, a.z)) * fx;
    const float3 bottom = f3(c.x, c.y, c.z) + (f3(d.x, d.y, d.z) - f3(c.x, c.y, c.z)) * fx;
    return top + (bottom - top) * fy;
}
// Radiance of a direction: the constant environment plus the image term (path.slang:961-983).
__device__ __forceinline__ float3 env_radiance(const Job& J, float3 dir) {
    float3 r = get3(J.env.radiance);
    if (J.env_w) {
        const float3 img = env_lookup(J, equirect_uv(env_local(J, dir)));
        r = r + f3(img.x * J.env_scale[0], img.y * J.env_scale[1], img.z * J.env_scale[2]);
    }
    return r;
}
// environment_proposal.slang:5-14, 17-24, 29-49.
__device__ __forceinline__ float env_solid_angle(const Job& J, uint32_t row) {
    const float angle = PI_F / float(J.env_h);
    return TAU_F / float(J.env_w) * 2.f * sinf(angle * (float(row) + 0.5f)) * sinf(0.5f * angle);
}
__device__ float env_density(const Job& J, float3 dir) {
    const float2 uv = equirect_uv(env_local(J, dir));
    const uint32_t cx = min(uint32_t(fracf(uv.x) * float(J.env_w)), J.env_w - 1u);
    const uint32_t cy = min(uint32_t(clampf(uv.y, 0.f, 1.f) * float(J.env_h)), J.env_h - 1u);
    const uint32_t index = cy * J.env_w + cx;
    const float previous = index > 0u ? __ldg(&J.env_dist[index - 1u].x) : 0.f;
    return (__ldg(&J.env_dist[index].x) - previous) / env_solid_angle(J, cy);
}
__device__ __forceinline__ uint32_t env_cdf_search(const float2* dist, uint32_t first, uint32_t stride, uint32_t count, float base, float target) {
    uint32_t low = 0u, high = count - 1u;
    while (low < high) {
        const uint32_t mid = (low + high) >> 1;
        if (__ldg(&dist[first + mid * stride].x) - base <= target) low = mid + 1u; else high = mid;
    }
    return low;
}
__device__ float3 env_sample(const Job& J, float ux, float uy, float& pdf) {
    const float2* cdf = J.env_dist;
    const uint32_t w = J.env_w, h = J.env_h;
    const uint32_t row = env_cdf_search(cdf, w - 1u, w, h, 0.f, uy);
    const float row_start = row > 0u ? __ldg(&cdf[row * w - 1u].x) : 0.f;
    const float row_mass = __ldg(&cdf[(row + 1u) * w - 1u].x) - row_start;
    const float target = fminf(ux * row_mass, __uint_as_float(__float_as_uint(row_mass) - 1u));
    const uint32_t column = env_cdf_search(cdf, row * w, 1u, w, row_start, target);
    const uint32_t at = row * w + column;
    const float at_mass = __ldg(&cdf[at].x), before = at > 0u ? __ldg(&cdf[at - 1u].x) : 0.f;
    const float previous = before - row_start;
    const float fraction = (target - previous) / (at_mass - row_start - previous);
    const float height = (uy - row_start) / row_mass;
    const float phi = TAU_F * ((float(column) + fraction) / float(w) - 0.5f);
    const float cosine = lerpf(cosf(PI_F * float(row) / float(h)), cosf(PI_F * float(row + 1u) / float(h)), height);
    const float sine = sqrtf(fmaxf(1.f - cosine * cosine, 0.f));
    pdf = (at_mass - before) / env_solid_angle(J, row);
    return env_world(J, f3(sine * cosf(phi), cosine, sine * sinf(phi)));
}

__device__ __forceinline__ float filter_offset(const float* table, float u) {
    float x = clampf(u, 0.f, 1.f) * float(FILTER_INTERVALS);
    uint32_t i = min(uint32_t(x), FILTER_INTERVALS - 1u);
    return lerpf(__ldg(table + i), __ldg(table + i + 1), x - float(i));
}
// Warp-aggregated queue append: one atomic per warp.
__device__ __forceinline__ uint32_t warp_append(uint32_t* counter, bool want) {
    uint32_t mask = __ballot_sync(0xffffffffu, want);
    if (!want) return 0xffffffffu;
    uint32_t lane = threadIdx.x & 31u, leader = __ffs(mask) - 1u;
    uint32_t base = 0;
    if (lane == leader) base = atomicAdd(counter, __popc(mask));
    base = __shfl_sync(mask, base, leader);
    return base + __popc(mask & ((1u << lane) - 1u));
}
// Queue append by the threads of a warp that reach it together (one atomic per group).
__device__ __forceinline__ uint32_t group_append(uint32_t* counter) {
    const uint32_t mask = __activemask(), lane = threadIdx.x & 31u, leader = __ffs(mask) - 1u;
    uint32_t base = 0;
    if (lane == leader) base = atomicAdd(counter, uint32_t(__popc(mask)));
    base = __shfl_sync(mask, base, leader);
    return base + uint32_t(__popc(mask & ((1u << lane) - 1u)));
}
// Shade appends a new extension ray or shadow entry where it makes it (the threads of a
// warp that get there together share one atomic) instead of carrying five float4s to a
// warp-wide append at the end of the loop body: 128 registers with 12/16 B of spill
// instead of 108/156 B (measured: 618 vs 623 ms per large frame).
// The same, with the group's slots ordered by key (0..7; ties by lane): the entries a
// trace warp later takes together then share their direction octant where they can.
__device__ __forceinline__ uint32_t group_append_by_key(uint32_t* counter, uint32_t key) {
    const uint32_t mask = __activemask(), lane = threadIdx.x & 31u, leader = __ffs(mask) - 1u;
    const uint32_t k0 = __ballot_sync(mask, key & 1u), k1 = __ballot_sync(mask, key & 2u), k2 = __ballot_sync(mask, key & 4u);
    uint32_t below = 0, same = 0;
    #pragma unroll
    for (uint32_t k = 0; k < 8; ++k) {
        const uint32_t with = mask & ((k & 1u) ? k0 : ~k0) & ((k & 2u) ? k1 : ~k1) & ((k & 4u) ? k2 : ~k2);
        if (k < key) below += uint32_t(__popc(with));
        if (k == key) same = with;
    }
    uint32_t base = 0;
    if (lane == leader) base = atomicAdd(counter, uint32_t(__popc(mask)));
    base = __shfl_sync(mask, base, leader);
    return base + below + uint32_t(__popc(same & ((1u << lane) - 1u)));
}
#ifndef VKB_SHADE_OCTANT_APPEND
#define VKB_SHADE_OCTANT_APPEND 0
#endif
#ifndef VKB_SHADE_EARLY_APPEND
#define VKB_SHADE_EARLY_APPEND 1
#endif
// The job owning a slot (BATCH) or job 0.
template <bool BATCH>
__device__ __forceinline__ uint32_t job_of_slot(const PathParams& p, uint32_t slot) { return BATCH ? __ldg(&p.slot_job[slot]) : 0u; }
// Largest job whose base (slot_base or pixel_base) is <= x: binary search over the table.
template <bool PIXELS>
__device__ __forceinline__ uint32_t find_job(const PathParams& p, uint32_t x) {
    uint32_t lo = 0, hi = p.njobs;
    while (hi - lo > 1) {
        uint32_t mid = (lo + hi) >> 1;
        uint32_t b = PIXELS ? p.jobs[mid].pixel_base : p.jobs[mid].slot_base;
        if (b <= x) lo = mid; else hi = mid;
    }
    return lo;
}

// path.slang:1792-1866 up to integrate: sampler, film-filtered pinhole camera ray.
template <bool BATCH>
__global__ void k_camera(PathParams p) {
    const uint32_t n = p.counters[7];
    for (uint32_t slot = blockIdx.x * blockDim.x + threadIdx.x; slot < n; slot += gridDim.x * blockDim.x) {
        uint32_t j = BATCH ? find_job<false>(p, slot) : 0u;
        const Job& J = BATCH ? p.jobs[j] : p.job0;
        if (BATCH) p.slot_job[slot] = j;
        uint32_t local = slot - J.slot_base;
        uint32_t pixel = local % J.npix, sidx = J.wave_first + local / J.npix;
        uint32_t px = pixel % J.cam.width, py = pixel / J.cam.width;
        uint32_t pseed = screen_ray_hash(px, py, 0u, J.seed);
        uint32_t rng = screen_ray_hash(px, py, sidx, J.seed);
        float4 cs = sample_group(pseed, sidx, J.sample_mask, 0u);
        float nx = (float(px) + 0.5f + filter_offset(p.filter, cs.x)) / float(J.cam.width) * 2.f + -1.f;
        float ny = (float(py) + 0.5f + filter_offset(p.filter, cs.y)) / float(J.cam.height) * -2.f + 1.f;
        float3 fwd = get3(J.cam.forward), eye = get3(J.cam.eye);
        float3 dir = normalize(fwd + get3(J.cam.right) * (nx / J.cam.proj_x) + get3(J.cam.up) * (ny / J.cam.proj_y));
        float near_d = J.cam.near_plane / dot(dir, fwd), far_d = J.cam.far_plane / dot(dir, fwd);
        float3 o = eye + dir * near_d;
        float tmax = fminf(FP32_MAX, fmaxf(0.f, far_d - length(o - eye)));
        p.thr[slot] = make_float4(1.f, 1.f, 1.f, __uint_as_float(0u));
        p.rad[slot] = make_float4(0.f, 0.f, 0.f, __uint_as_float(0u));
        p.rng[slot] = make_uint2(rng, pseed);
        if (!BATCH && J.adaptive) {
            // Stopped pixels trace nothing: the camera rays of the others are compacted.
            const bool live = (J.ad_state[pixel] & AD_STOPPED) == 0u;
            namespace cg = cooperative_groups;
            if (live) {
                cg::coalesced_group g = cg::coalesced_threads();
                uint32_t base = 0;
                if (g.thread_rank() == 0) base = atomicAdd(&p.counters[0], g.size());
                const uint32_t ri = g.shfl(base, 0) + g.thread_rank();
                p.ray_o[0][ri] = make_float4(o.x, o.y, o.z, tmax);
                p.ray_d[0][ri] = make_float4(dir.x, dir.y, dir.z, __uint_as_float(slot));
            }
            continue;
        }
        p.ray_o[0][slot] = make_float4(o.x, o.y, o.z, tmax);
        p.ray_d[0][slot] = make_float4(dir.x, dir.y, dir.z, __uint_as_float(slot));
    }
}
__device__ __forceinline__ void flush_count(unsigned long long* dst, uint32_t v) {
    unsigned long long x = v;
    for (int off = 16; off > 0; off >>= 1) x += __shfl_xor_sync(0xffffffffu, x, off);
    if ((threadIdx.x & 31u) == 0u && x) atomicAdd(dst, x);
}
#ifndef VKB_TRACE_MIN_BLOCKS
#define VKB_TRACE_MIN_BLOCKS 8
#endif
template <bool ANY, bool COUNT, bool W8 = false>
__device__ __forceinline__ bool trace_any(const SceneView& sv, RayRef ray, float tmax, HitRecord& h, uint32_t* err, TraceCount* tc,
                                          TraceStack stk) {
    return trace_ray<ANY, COUNT, W8>(sv, ray, tmax, h, err, tc, stk);
}
// This thread's column of the block's shared-memory traversal stack (W8: the deeper local
// part of the 8-wide BLAS traversal).
#define VKB_STACK_DECL_W(W8)                                                                             \
    __shared__ int stack_r_[SMEM_STACK * TRACE_BLOCK];                                                  \
    int stack_spill_[(W8) ? SPILL_STACK8 : (SPILL_STACK > 0 ? SPILL_STACK : 1)];                         \
    TraceStack stk{stack_r_ + threadIdx.x, stack_spill_};
#define VKB_STACK_DECL VKB_STACK_DECL_W(false)
// Lanes of a warp refill together once at most this many are still tracing.
#ifndef VKB_TRACE_REFILL
#define VKB_TRACE_REFILL 20
#endif
static_assert(VKB_TRACE_REFILL >= 1 && VKB_TRACE_REFILL <= 31, "refill threshold in lanes");
// Closest hits of the queued rays with lane refill: each lane carries one ray's
// traversal state; once at most VKB_TRACE_REFILL lanes of a warp are still tracing, the
// idle lanes take the next rays of the queue together (one atomic per warp), so a warp
// does not run on with a few long rays while its other lanes wait (measured: a warp's
// lanes otherwise spend ~60% of its steps idle behind its longest ray).  Refilling
// each lane as soon as it finishes is slower: the refill code then runs on single lanes.
template <bool COUNT, bool BATCH, bool W8 = false>
__global__ void __launch_bounds__(TRACE_BLOCK, VKB_TRACE_MIN_BLOCKS) k_trace(PathParams p, int cur) {
    VKB_STACK_DECL_W(W8)
    const uint32_t n = p.counters[cur];
    if (blockIdx.x == 0 && threadIdx.x == 0) atomicAdd(&p.counters[3], n);
    const uint32_t lane = threadIdx.x & 31u;
    TraceCount tc;
    TraceLane<false, COUNT, W8> L;
    constexpr uint32_t NONE = 0xffffffffu;
    uint32_t ray = NONE, job = 0;
    bool drained = false;
    for (;;) {
        uint32_t act = __ballot_sync(0xffffffffu, ray != NONE);
        if (!drained && uint32_t(__popc(act)) <= uint32_t(VKB_TRACE_REFILL)) {
            const uint32_t idle = ~act;
            uint32_t base = 0;
            if (lane == 0u) base = atomicAdd(&p.counters[11], uint32_t(__popc(idle)));
            base = __shfl_sync(0xffffffffu, base, 0);
            drained = base + uint32_t(__popc(idle)) >= n;
            if (ray == NONE) {
                const uint32_t r = base + uint32_t(__popc(idle & ((1u << lane) - 1u)));
                if (r < n) {
                    if (BATCH) job = job_of_slot<true>(p, __float_as_uint(p.ray_d[cur][r].w));
                    if (L.start(BATCH ? p.jobs[job].sv : p.job0.sv, RayRef{p.ray_o[cur], p.ray_d[cur], r}, p.ray_o[cur][r].w)) {
                        ray = r;
                    } else {
                        p.hit[r] = make_float4(-1.f, 0.f, 0.f, __uint_as_float(0xffffffffu));
                        p.hit_inst[r] = 0xffffffffu;
                    }
                }
            }
            act = __ballot_sync(0xffffffffu, ray != NONE);
        }
        if (act == 0u) {
            if (drained) break;
            continue;
        }
        bool done = false;
        if (ray != NONE) {
            if constexpr (BATCH) done = L.step(p.jobs[job].sv, RayRef{p.ray_o[cur], p.ray_d[cur], ray}, p.err, &tc, stk);
            else done = L.step(p.job0.sv, RayRef{p.ray_o[cur], p.ray_d[cur], ray}, p.err, &tc, stk);
        }
        if (done) {
            p.hit[ray] = L.found ? make_float4(L.hit.t, L.hit.u, L.hit.v, __uint_as_float(L.hit.tri)) : make_float4(-1.f, 0.f, 0.f, __uint_as_float(0xffffffffu));
            p.hit_inst[ray] = L.found ? L.hit.inst : 0xffffffffu;
            ray = NONE;
        }
    }
    if (COUNT) {
        flush_count(&p.work[0], tc.nodes);
        flush_count(&p.work[1], tc.tris);
        flush_count(&p.work[2], tc.instances);
        flush_count(&p.work[5], tc.blas_nodes);
    }
}

// Shadow entries with lane refill (as k_trace): a lane carries one entry through its
// ray A, then its ray B (the second estimator's, when present and traced), then adds
// the unoccluded contributions to the slot's radiance.
// EXT: waves with an image environment or emissive meshes, whose entries may carry an
// environment ray (phase 2) and a mesh ray (phase 3) after the light rays A and B.
template <bool COUNT, bool BATCH, bool EXT, bool W8 = false>
__global__ void __launch_bounds__(TRACE_BLOCK, VKB_TRACE_MIN_BLOCKS) k_trace_shadow(PathParams p) {
    VKB_STACK_DECL_W(W8)
    const uint32_t n = p.counters[2];
    if (blockIdx.x == 0 && threadIdx.x == 0) atomicAdd(&p.counters[4], n);
    const uint32_t lane = threadIdx.x & 31u;
    TraceCount tc;
    TraceLane<true, COUNT, W8> L;
    constexpr uint32_t NONE = 0xffffffffu;
    uint32_t e = NONE, rid = 0, phase = 0, occ = 0, job = 0;
    // Starts entry e's next ray from phase ph on; false when the entry has no ray left.
    auto begin = [&](uint32_t ph) -> bool {
        const uint32_t flags = __float_as_uint(p.sa_c[e].w);
        if (ph == 0u) {
            if ((flags & SH_TRACE_A) && L.start(BATCH ? p.jobs[job].sv : p.job0.sv, RayRef{p.sa_o, p.sa_d, e}, p.sa_o[e].w)) { phase = 0u; rid = e; return true; }
        }
        if (ph <= 1u && (flags & SH_HAS_B) && (flags & SH_TRACE_B)) {
            const uint32_t slot = __float_as_uint(p.sa_d[e].w);
            if (L.start(BATCH ? p.jobs[job].sv : p.job0.sv, RayRef{p.sb_o, p.sb_d, slot}, p.sb_o[slot].w)) { phase = 1u; rid = slot; return true; }
        }
        if constexpr (EXT) {
            const uint32_t slot = __float_as_uint(p.sa_d[e].w);
            if (ph <= 2u && (flags & SH_HAS_C)) {
                if (L.start(BATCH ? p.jobs[job].sv : p.job0.sv, RayRef{p.sc_o, p.sc_d, slot}, p.sc_o[slot].w)) { phase = 2u; rid = slot; return true; }
            }
            if (flags & SH_HAS_D) {
                if (L.start(BATCH ? p.jobs[job].sv : p.job0.sv, RayRef{p.sd_o, p.sd_d, slot}, p.sd_o[slot].w)) { phase = 3u; rid = slot; return true; }
            }
        }
        return false;
    };
    auto finish = [&]() {
        const float4 sc = p.sa_c[e];
        const uint32_t slot = __float_as_uint(p.sa_d[e].w), flags = __float_as_uint(sc.w);
        float3 total = (occ & 1u) ? f3(0.f) : f3(sc.x, sc.y, sc.z);
        if (flags & SH_HAS_B) {
            const float4 bc = p.sb_c[slot];
            if (!(occ & 2u)) total = total + f3(bc.x, bc.y, bc.z);
        }
        const float4 r = p.rad[slot];
        uint32_t dropped = __float_as_uint(r.w);
        const Job& J = BATCH ? p.jobs[job] : p.job0;
        const float limit = (flags & SH_DIRECT) ? J.clamp_direct : J.clamp_indirect;
        float3 add = clamp_sample(total, limit, dropped);
        if constexpr (EXT) {
            // The environment and mesh estimates are clamped on their own (path.slang:1660-1661).
            if ((flags & SH_HAS_C) && !(occ & 4u)) {
                const float4 cc = p.sc_c[slot];
                add = add + clamp_sample(f3(cc.x, cc.y, cc.z), limit, dropped);
            }
            if ((flags & SH_HAS_D) && !(occ & 8u)) {
                const float4 dc = p.sd_c[slot];
                add = add + clamp_sample(f3(dc.x, dc.y, dc.z), limit, dropped);
            }
        }
        p.rad[slot] = make_float4(r.x + add.x, r.y + add.y, r.z + add.z, __uint_as_float(dropped));
        e = NONE;
    };
    bool drained = false;
    for (;;) {
        uint32_t act = __ballot_sync(0xffffffffu, e != NONE);
        if (!drained && uint32_t(__popc(act)) <= uint32_t(VKB_TRACE_REFILL)) {
            const uint32_t idle = ~act;
            uint32_t base = 0;
            if (lane == 0u) base = atomicAdd(&p.counters[12], uint32_t(__popc(idle)));
            base = __shfl_sync(0xffffffffu, base, 0);
            drained = base + uint32_t(__popc(idle)) >= n;
            if (e == NONE) {
                const uint32_t r = base + uint32_t(__popc(idle & ((1u << lane) - 1u)));
                if (r < n) {
                    e = r;
                    occ = 0u;
                    if (BATCH) job = job_of_slot<true>(p, __float_as_uint(p.sa_d[r].w));
                    if (!begin(0u)) finish();
                }
            }
            act = __ballot_sync(0xffffffffu, e != NONE);
        }
        if (act == 0u) {
            if (drained) break;
            continue;
        }
        bool done = false;
        if (e != NONE) {
            // The traversal re-reads its ray (instance entry, return to world space):
            // phase 0 the light ray A, 1 the light ray B, 2 the environment ray, 3 the mesh ray.
            RayRef ray{phase ? p.sb_o : p.sa_o, phase ? p.sb_d : p.sa_d, rid};
            if constexpr (EXT) {
                if (phase == 2u) ray = RayRef{p.sc_o, p.sc_d, rid};
                else if (phase == 3u) ray = RayRef{p.sd_o, p.sd_d, rid};
            }
            if constexpr (BATCH) done = L.step(p.jobs[job].sv, ray, p.err, &tc, stk);
            else done = L.step(p.job0.sv, ray, p.err, &tc, stk);
        }
        if (done) {
            if (L.found) occ |= 1u << phase;
            if constexpr (EXT) { if (phase == 3u || !begin(phase + 1u)) finish(); }
            else { if (phase != 0u || !begin(1u)) finish(); }
        }
    }
    if (COUNT) {
        flush_count(&p.work[3], tc.nodes);
        flush_count(&p.work[4], tc.tris);
        flush_count(&p.work[6], tc.blas_nodes);
    }
}

struct Surface { float3 world, face, geometric, error, shadow_xyz; float shadow_cone; bool entering; };
__device__ __forceinline__ float3 tvec(const float4 I[3], float3 x) {
    return f3(I[0].x * x.x + I[1].x * x.y + I[2].x * x.z, I[0].y * x.x + I[1].y * x.y + I[2].y * x.z, I[0].z * x.x + I[1].z * x.y + I[2].z * x.z);
}
__device__ __forceinline__ float3 mvec(const float4 M[3], float3 x) { return f3(M[0].x * x.x + M[0].y * x.y + M[0].z * x.z, M[1].x * x.x + M[1].y * x.y + M[1].z * x.z, M[2].x * x.x + M[2].y * x.y + M[2].z * x.z); }
// surface_position_error: the rounding bound of a world point on an instance of mesh m.
__device__ __forceinline__ float3 position_error(const MeshInfo& m, const float4 M[3], const float4 I[3], float3 world) {
    float3 lo = f3(m.lo[0], m.lo[1], m.lo[2]), hi = f3(m.hi[0], m.hi[1], m.hi[2]);
    float3 mag = vmax(vabs(lo), vabs(hi));
    float extent = maxc(vabs(hi - lo));
    float3 aw = vabs(world);
    float3 iw = f3(fabsf(I[0].x) * aw.x + fabsf(I[0].y) * aw.y + fabsf(I[0].z) * aw.z + fabsf(I[0].w),
                   fabsf(I[1].x) * aw.x + fabsf(I[1].y) * aw.y + fabsf(I[1].z) * aw.z + fabsf(I[1].w),
                   fabsf(I[2].x) * aw.x + fabsf(I[2].y) * aw.y + fabsf(I[2].z) * aw.z + fabsf(I[2].w));
    const float g7 = fp32_gamma7();
    float3 local = (mag + f3(extent) + iw) * g7;
    float e[3];
    for (int r = 0; r < 3; ++r) {
        float4 row = M[r];
        e[r] = fabsf(row.x) * local.x + fabsf(row.y) * local.y + fabsf(row.z) * local.z + g7 * (fabsf(row.x) * mag.x + fabsf(row.y) * mag.y + fabsf(row.z) * mag.z + fabsf(row.w));
    }
    return f3(e[0], e[1], e[2]);
}
// hit_geometry.slang:64-138,174-205; hit.slang:86-114; surface.slang:290-333; material.slang:69-79.
// The triangle's corners come from the BLAS leaf-order copies (positions in blas_tris,
// normals in tri_nrm, the index buffer's vertex order), so they need no index lookup
// first: the same values as indices -> vertices, one dependent load fewer.
__device__ __forceinline__ Surface hit_surface(const Job& p, uint32_t inst, uint32_t tri, float u, float v, float3 dir) {
    Surface s;
    uint4 info = __ldg(&p.inst_info[inst]);
    const MeshInfo& m = p.meshes[info.x];
    float4 M[3] = {__ldg(&p.o2w[3 * inst]), __ldg(&p.o2w[3 * inst + 1]), __ldg(&p.o2w[3 * inst + 2])};
    float4 I[3] = {__ldg(&p.w2o[3 * inst]), __ldg(&p.w2o[3 * inst + 1]), __ldg(&p.w2o[3 * inst + 2])};
    const float4* tp = p.sv.blas_tris + 3u * size_t(tri);
    const float4* np = p.tri_nrm + 3u * size_t(tri);
    float4 q0 = __ldg(tp), q1 = __ldg(tp + 1), q2 = __ldg(tp + 2);
    float4 m0 = __ldg(np), m1 = __ldg(np + 1), m2 = __ldg(np + 2);
    float3 P[3] = {f3(q0.x, q0.y, q0.z), f3(q1.x, q1.y, q1.z), f3(q2.x, q2.y, q2.z)};
    float3 N[3] = {f3(m0.x, m0.y, m0.z), f3(m1.x, m1.y, m1.z), f3(m2.x, m2.y, m2.z)};
    float b[3] = {1.f - u - v, u, v};
    float3 fobj = finite_unit_normal(cross(P[1] - P[0], P[2] - P[0]), N[0]);
    float3 face = finite_unit_normal(tvec(I, fobj), f3(0.f, 0.f, 1.f));
    bool entering = dot(face, dir) < 0.f;
    float3 lp = P[0] * b[0] + P[1] * b[1] + P[2] * b[2];
    s.world = mvec(M, lp) + f3(M[0].w, M[1].w, M[2].w);
    float3 facew = tvec(I, fobj);
    float3 un = finite_unit_normal(tvec(I, N[0] * b[0] + N[1] * b[1] + N[2] * b[2]), facew);
    float3 nrm = dot(un, facew) < 0.f ? -un : un;
    float det = M[0].x * (M[1].y * M[2].z - M[1].z * M[2].y) - M[0].y * (M[1].x * M[2].z - M[1].z * M[2].x) + M[0].z * (M[1].x * M[2].y - M[1].y * M[2].x);
    bool object_front = entering != (det < 0.f);
    s.geometric = finite_unit_normal(nrm, f3(0.f, 0.f, 1.f)) * (object_front ? 1.f : -1.f);
    // Shadow-terminator envelope (hit_geometry.slang:174-205), front = entering.
    float side = entering ? 1.f : -1.f;
    float3 sf = face * side, pr[3], nr[3];
    for (int k = 0; k < 3; ++k) { pr[k] = mvec(M, P[k] - P[0]); nr[k] = finite_unit_normal(tvec(I, N[k]) * side, sf); }
    float3 smooth = nr[0] * b[0] + nr[1] * b[1] + nr[2] * b[2];
    if (dot(smooth, sf) < 0.f) { for (int k = 0; k < 3; ++k) nr[k] = -nr[k]; smooth = -smooth; }
    float3 point = pr[0] * b[0] + pr[1] * b[1] + pr[2] * b[2];
    float envelope = 0.f, quadratic = 0.f, cone = 0.f;
    for (int i = 0; i < 3; ++i) {
        float support = 0.f;
        for (int j = 0; j < 3; ++j) support = fmaxf(support, dot(pr[j] - point, nr[i]));
        envelope = i == 0 ? support : fminf(envelope, support);
        cone = fmaxf(cone, length(nr[i] - sf));
        for (int j = i + 1; j < 3; ++j) quadratic += b[i] * b[j] * dot(nr[j] - nr[i], pr[j] - pr[i]);
    }
    s.shadow_xyz = smooth * fmaxf(envelope, 0.5f * quadratic);
    s.shadow_cone = cone;
    s.face = entering ? face : -face;
    s.entering = entering;
    s.error = position_error(m, M, I, s.world);
    return s;
}
// path.slang:771-784 with vork_prelude.slang:340-345.
__device__ __forceinline__ float3 path_origin(const Surface& s, float3 dir) {
    bool reflection = dot(s.geometric, dir) > 0.f;
    float3 base = s.world;
    if (reflection && s.shadow_cone > 0.f) {
        float nl = dot(s.geometric, dir), ng = dot(s.face, dir), cone = s.shadow_cone;
        float amount = nl < cone ? saturatef(2.f - (ng + nl) / cone) : saturatef(1.f - ng / cone);
        base = base + s.shadow_xyz * amount;
    }
    return surface_ray_origin(base, s.error, reflection ? s.geometric : s.face, dir);
}
// ---------------------------------------------------------------- emissive meshes
// Ratio of sibling masses under a shared power-of-two scale (emitter_mesh_proposal.slang:25-35).
__device__ __forceinline__ float em_left_probability(float left, float right) {
    const int exponent = int((__float_as_uint(fmaxf(left, right)) >> 23) & 255u) - 127;
    const float scale = __uint_as_float(uint32_t(127 - exponent / 2) << 23);
    left *= scale; right *= scale;
    if (left >= right) return left > 0.f ? 1.f / (1.f + right / left) : 0.f;
    const float ratio = left / right;
    return ratio / (1.f + ratio);
}
constexpr float MESH_SOURCE_UNIFORM_MIX = 0.5f;
// Source triangle -> (source, primitive) over the cumulative counts (emitter_mesh_proposal.slang:13-22);
// past the last source (only through a zero-mass branch) it stays on the last one.
__device__ __forceinline__ void em_triangle(const Job& J, uint32_t triangle, uint32_t& src, uint32_t& prim) {
    uint32_t low = 0u, high = J.em_count;
    while (low < high) {
        const uint32_t mid = (low + high) >> 1;
        if (triangle < __ldg(&J.em_sources[mid].y)) high = mid; else low = mid + 1u;
    }
    src = min(low, J.em_count - 1u);
    prim = triangle - (src == 0u ? 0u : __ldg(&J.em_sources[src - 1u].y));
}
// The branch probabilities from the leaf up, mixed half and half with the uniform choice
// (emitter_mesh_proposal.slang:37-57); 0 for a triangle that is not a source.
__device__ float em_probability(const Job& J, uint32_t inst, uint32_t prim) {
    const uint32_t src = __ldg(&J.em_inst_source[inst]);
    if (src == 0xffffffffu || !(__ldg(&J.em_tree[1]) > 0.f)) return 0.f;
    uint32_t node = J.em_leaves + prim + (src == 0u ? 0u : __ldg(&J.em_sources[src - 1u].y));
    float probability = 1.f;
    while (node > 1u) {
        const uint32_t parent = node >> 1;
        const float left = __ldg(&J.em_tree[2u * parent]), right = __ldg(&J.em_tree[2u * parent + 1u]);
        if (fmaxf(left, right) <= 0.f) { probability = 0.f; break; }
        const float q = em_left_probability(left, right);
        probability *= (node & 1u) ? 1.f - q : q;
        node = parent;
    }
    return (1.f - MESH_SOURCE_UNIFORM_MIX) * probability + MESH_SOURCE_UNIFORM_MIX / float(J.em_tris);
}
// emitter_mesh_sample (emitter_mesh_proposal.slang:59-83); u = path_triangle (group 2 as .zxy).
__device__ bool em_sample(const Job& J, float ux, float uy, float uz, uint32_t& inst, uint32_t& prim, float& b1, float& b2) {
    const float top = __uint_as_float(0x3f7fffffu);
    float choice = fminf(ux, top);
    if (!(__ldg(&J.em_tree[1]) > 0.f)) return false;
    const bool uniform = uz < MESH_SOURCE_UNIFORM_MIX;
    const float point = (uz - (uniform ? 0.f : MESH_SOURCE_UNIFORM_MIX)) / (uniform ? MESH_SOURCE_UNIFORM_MIX : 1.f - MESH_SOURCE_UNIFORM_MIX);
    uint32_t node = 1u;
    if (uniform) node = J.em_leaves + min(uint32_t(choice * float(J.em_tris)), J.em_tris - 1u);
    else
        while (node < J.em_leaves) {
            const float q = em_left_probability(__ldg(&J.em_tree[2u * node]), __ldg(&J.em_tree[2u * node + 1u]));
            if (choice < q) { choice /= q; node *= 2u; }
            else { choice = (choice - q) / (1.f - q); node = 2u * node + 1u; }
            choice = fminf(choice, top);
        }
    uint32_t src;
    em_triangle(J, node - J.em_leaves, src, prim);
    inst = __ldg(&J.em_sources[src].x);
    const float radius = sqrtf(uy);
    b1 = radius * (1.f - point);
    b2 = radius - b1;
    return true;
}
// World point at (b1, b2), face normal and area of a source triangle in the mesh's own
// index order (hit_geometry.slang:116-124,246-256).
struct EmGeometry { float3 point, face, error; float area; };
__device__ EmGeometry em_geometry(const Job& J, uint32_t inst, uint32_t prim, float b1, float b2) {
    const MeshInfo& m = J.meshes[__ldg(&J.inst_info[inst]).x];
    const float4 M[3] = {__ldg(&J.o2w[3 * inst]), __ldg(&J.o2w[3 * inst + 1]), __ldg(&J.o2w[3 * inst + 2])};
    const float4 I[3] = {__ldg(&J.w2o[3 * inst]), __ldg(&J.w2o[3 * inst + 1]), __ldg(&J.w2o[3 * inst + 2])};
    const uint32_t* ix = J.indices + m.index_offset + 3u * prim;
    const float4* vp = J.vpos + m.vertex_offset;
    const float4 q0 = __ldg(vp + __ldg(ix)), q1 = __ldg(vp + __ldg(ix + 1)), q2 = __ldg(vp + __ldg(ix + 2));
    const float3 P0 = f3(q0.x, q0.y, q0.z), P1 = f3(q1.x, q1.y, q1.z), P2 = f3(q2.x, q2.y, q2.z);
    const float3 raw = cross(P1 - P0, P2 - P0);
    // A degenerate face (whose vertex-normal fallback the hit uses) has no area, hence no
    // probability and no contribution, so the face's own cross product stands in for it.
    EmGeometry g;
    g.face = finite_unit_normal(tvec(I, finite_unit_normal(raw, raw)), f3(0.f, 0.f, 1.f));
    g.point = mvec(M, P0 * (1.f - b1 - b2) + P1 * b1 + P2 * b2) + f3(M[0].w, M[1].w, M[2].w);
    g.area = length(cross(mvec(M, P1 - P0), mvec(M, P2 - P0))) * 0.5f;
    g.error = position_error(m, M, I, g.point);
    return g;
}
// Solid-angle density at `from` of a point on a source triangle, times the triangle's
// probability (path.slang:996-1002, emitter_mesh_proposal.slang:86-92).
__device__ __forceinline__ float mesh_pdf(const Job& J, uint32_t inst, uint32_t prim, float area, float3 from, float3 point, float3 face) {
    const float3 delta = point - from;
    const float squared = dot(delta, delta);
    const float cosine = fabsf(dot(face, normalize(delta)));
    const float density = area > 0.f && cosine > 0.f ? squared / (area * cosine) : 0.f;
    return density * em_probability(J, inst, prim);
}

// The frame's mesh-source weights (emitter_weights.slang:23-47): leaf t = world area x the
// emission's Rec.709 luminance power of source triangle t (the area alone when that
// product is not finite), 0 on the padded leaves.  J carries the topology and geometry.
__global__ void k_em_leaves(const __grid_constant__ Job J, float* tree) {
    for (uint32_t t = blockIdx.x * blockDim.x + threadIdx.x; t < J.em_leaves; t += gridDim.x * blockDim.x) {
        float area = 0.f;
        if (t < J.em_tris) {
            uint32_t src, prim;
            em_triangle(J, t, src, prim);
            const uint32_t inst = __ldg(&J.em_sources[src].x);
            area = em_geometry(J, inst, prim, 0.f, 0.f).area;
            if (area > 0.f) {
                const vkb_material& m = J.materials[__ldg(&J.inst_info[inst]).y];
                const float power = (fmaxf(m.emission_color[0], 0.f) * LUM_R + fmaxf(m.emission_color[1], 0.f) * LUM_G +
                                     fmaxf(m.emission_color[2], 0.f) * LUM_B) * fmaxf(m.emission_luminance, 0.f);
                const float weight = area * power;
                if (isfinite(weight)) area = weight;
            }
        }
        tree[J.em_leaves + t] = area;
    }
}
// Inner nodes [first, 2 first): the mean of their two children (emitter_weights.slang:48-55).
__global__ void k_em_reduce(float* tree, uint32_t first) {
    for (uint32_t i = blockIdx.x * blockDim.x + threadIdx.x; i < first; i += gridDim.x * blockDim.x) {
        const uint32_t node = first + i;
        tree[node] = 0.5f * tree[2u * node] + 0.5f * tree[2u * node + 1u];
    }
}
// The levels from `first` up to the root in one block (a barrier between levels).
__global__ void k_em_reduce_top(float* tree, uint32_t first) {
    for (uint32_t level = first; level >= 1u; level >>= 1) {
        for (uint32_t i = threadIdx.x; i < level; i += blockDim.x) {
            const uint32_t node = level + i;
            tree[node] = 0.5f * tree[2u * node] + 0.5f * tree[2u * node + 1u];
        }
        __syncthreads();
    }
}

__device__ __forceinline__ float3 light_threshold(float3 value, float threshold, uint32_t& rng) {
    float importance = maxc(value);
    if (importance < threshold && threshold > 0.f) {
        float keep = importance / threshold;
        if (path_random(rng) >= keep) return f3(0.f);
        return value / keep;
    }
    return value;
}

// One radiance-cache record of this vertex: queries append (warp-aggregated on
// counters[9]); training records go to their fixed position.
// The closure values it stores come by value, so the caller's closure need not have an
// address (a reference to it kept the closure in local memory).
__device__ __noinline__ void cache_append(const PathParams& p, float3 world, float3 view, float3 normal, float roughness, float metalness,
                                          float3 base_color, uint32_t slot, uint32_t vertex, float3 thr, float3 rad) {
    uint32_t idx;
    if (p.cache.mode == 1u) {
        namespace cg = cooperative_groups;
        cg::coalesced_group g = cg::coalesced_threads();
        uint32_t base = 0;
        if (g.thread_rank() == 0) base = atomicAdd(&p.counters[9], g.size());
        base = g.shfl(base, 0);
        idx = base + g.thread_rank();
    } else {
        if (vertex < 1u || vertex > p.cache.vmax) return;
        idx = slot * p.cache.vmax + vertex - 1u;
    }
    if (idx >= p.cache.capacity) return;
    const float3 q = f3((world.x - p.cache.box_lo.x) * p.cache.box_scale.x, (world.y - p.cache.box_lo.y) * p.cache.box_scale.y,
                        (world.z - p.cache.box_lo.z) * p.cache.box_scale.z);
    float4* r = p.cache.rec + 4 * size_t(idx);
    r[0] = make_float4(q.x, q.y, q.z, view.x);
    r[1] = make_float4(view.y, view.z, normal.x, normal.y);
    r[2] = make_float4(normal.z, roughness, metalness, base_color.x);
    r[3] = make_float4(base_color.y, base_color.z, 0.f, 0.f);
    if (p.cache.mode == 1u) {
        p.cache.slot[idx] = slot;
    } else {
        p.cache.aux[2 * size_t(idx)] = make_float4(thr.x, thr.y, thr.z, 0.f);
        p.cache.aux[2 * size_t(idx) + 1] = make_float4(rad.x, rad.y, rad.z, 0.f);
        p.cache.flag[idx] = 1u;
    }
}

// integrate's per-vertex body (path.slang:1340-1709) for one queued extension hit.
// The parameter block is __grid_constant__: `J = p.job0` then refers to it in place
// (a plain by-value parameter that is referenced gets copied to a 736-byte local frame
// per thread); one block of 512 per SM (128 registers, a small spill) measured faster
// than 3 blocks of 128 at 158 registers, 4 blocks of 128 and 2 blocks of 256.
#ifndef VKB_SHADE_BLOCK
#define VKB_SHADE_BLOCK 512
#endif
#ifndef VKB_SHADE_MIN_BLOCKS
#define VKB_SHADE_MIN_BLOCKS 1
#endif
constexpr int SHADE_BLOCK = VKB_SHADE_BLOCK;
// EXT: waves with an image environment or emissive meshes (their strategies and the
// per-slot previous vertex); the plain instantiation carries none of it.
template <bool BATCH, bool EXT>
__global__ void __launch_bounds__(VKB_SHADE_BLOCK, VKB_SHADE_MIN_BLOCKS) k_shade(const __grid_constant__ PathParams p, int cur) {
    const int nxt = cur ^ 1;
    uint32_t n = p.counters[cur];
    uint32_t loop_end = (n + blockDim.x - 1) / blockDim.x * blockDim.x;  // whole warps stay in the loop for ballots
    for (uint32_t i = blockIdx.x * blockDim.x + threadIdx.x; i < loop_end; i += gridDim.x * blockDim.x) {
        bool active = i < n;
        bool push_ray = false, push_shadow = false;
        float4 new_o, new_d, sh_o, sh_d, sh_c;
        uint32_t slot = 0;
        if (active) {
            float4 ro = p.ray_o[cur][i], rd = p.ray_d[cur][i];
            slot = __float_as_uint(rd.w);
            const Job& J = BATCH ? p.jobs[job_of_slot<true>(p, slot)] : p.job0;
            float3 dir = f3(rd.x, rd.y, rd.z);
            float4 hh = p.hit[i];
            uint32_t inst = p.hit_inst[i];
            float4 T = p.thr[slot], R = p.rad[slot];
            uint2 rg = p.rng[slot];
            uint32_t meta = __float_as_uint(T.w);
            uint32_t bounce = meta & 0xffu, diffuse = (meta >> 8) & 0xffu, glossy = (meta >> 16) & 0xffu;
            uint32_t ray_event = bounce == 0 ? VKB_RAY_CAMERA : ((meta >> 24) & 0x3fu);
            float3 thr = f3(T.x, T.y, T.z), rad = f3(R.x, R.y, R.z);
            uint32_t dropped = __float_as_uint(R.w), rng = rg.x, pseed = rg.y;
            uint32_t local = slot - J.slot_base;
            uint32_t pixel = local % J.npix, sidx = J.wave_first + local / J.npix;
            float limit = bounce == 0 ? J.clamp_direct : J.clamp_indirect;
            if (J.primary_ids && bounce == 0 && sidx == J.first_sample) {
                J.primary_ids[2 * pixel] = hh.x >= 0.f ? inst : 0xffffffffu;
                J.primary_ids[2 * pixel + 1] = hh.x >= 0.f ? __float_as_uint(__ldg(&J.sv.blas_tris[3u * size_t(__float_as_uint(hh.w))]).w) : 0xffffffffu;
            }
            if (!(hh.x >= 0.f)) {
                // Miss: path.slang:1484-1512 with the constant world light and camera-visible suns.
                float3 sky;
                if (ray_event == VKB_RAY_CAMERA && !J.env.camera_sees_environment) sky = get3(J.env.background);
                else {
                    sky = EXT ? env_radiance(J, dir) : get3(J.env.radiance);
                    if (ray_event == VKB_RAY_CAMERA)
                        for (uint32_t l = 0; l < J.num_lights; ++l) {
                            const vkb_light& L = J.lights[l];
                            if (L.position[3] != 0.f || !(L.shadow_offsets[0] & VKB_RAY_CAMERA)) continue;
                            sky = sky + emitter_eval(L, f3(0.f), dir).radiance;
                        }
                }
                if (EXT && J.env_w && bounce > 0u) {
                    // path.slang:1463: an escape after a BSDF sample, weighed against the
                    // environment strategy.
                    const float prev = p.prev[slot].w;
                    if (prev > 0.f) sky = sky * mis_power(prev, env_density(J, dir));
                }
                rad = rad + clamp_sample(thr * sky, limit, dropped);
            } else {
                uint32_t vtx = bounce;
                float4 sc = sample_group(pseed, sidx, J.sample_mask, vertex_group(vtx, 0));   // path_scatter
                Surface s = hit_surface(J, inst, __float_as_uint(hh.w), hh.y, hh.z, dir);
                const vkb_material& mt = J.materials[__ldg(&J.inst_info[inst]).y];
                Closure c;
                c.base_color = get3(mt.base_color); c.base_weight = mt.base_weight; c.base_metalness = mt.base_metalness;
                c.specular_color = get3(mt.specular_color); c.specular_weight = mt.specular_weight;
                c.specular_roughness = mt.specular_roughness; c.specular_ior = mt.specular_ior; c.optical_ior = 0.f;
                c.n = s.geometric;
                boundary_closure_air(c);
                float3 view = -dir;
                if (EXT && mt.emission_luminance > 0.f && ((mt.flags & 2u) || s.entering)) {
                    // Surface emission (path.slang:1580-1591) on the side the material covers,
                    // weighed against the mesh strategy after a BSDF sample.
                    const float3 emitted = get3(mt.emission_color) * mt.emission_luminance;
                    float mis = 1.f;
                    if (bounce > 0u && J.em_tris) {
                        const float4 pv = p.prev[slot];
                        if (pv.w > 0.f) {
                            const uint32_t tri = __float_as_uint(hh.w);
                            const float4* tp = J.sv.blas_tris + 3u * size_t(tri);
                            const float4 q0 = __ldg(tp), q1 = __ldg(tp + 1), q2 = __ldg(tp + 2);
                            const float4 M[3] = {__ldg(&J.o2w[3 * inst]), __ldg(&J.o2w[3 * inst + 1]), __ldg(&J.o2w[3 * inst + 2])};
                            const float3 e1 = mvec(M, f3(q1.x - q0.x, q1.y - q0.y, q1.z - q0.z)), e2 = mvec(M, f3(q2.x - q0.x, q2.y - q0.y, q2.z - q0.z));
                            const float area = length(cross(e1, e2)) * 0.5f;
                            mis = mis_power(pv.w, mesh_pdf(J, inst, __float_as_uint(q0.w), area, f3(pv.x, pv.y, pv.z), s.world, s.face));
                        }
                    }
                    rad = rad + clamp_sample(thr * emitted * mis, limit, dropped);
                }
                // Radiance cache: record this vertex, and at the query vertex stop the path
                // here (the query kernel adds thr x the cached outgoing radiance).
                const bool cache_query = p.cache.mode == 1u && bounce >= p.cache.vertex;
                if (cache_query || (p.cache.mode == 2u && bounce >= 1u)) cache_append(p, s.world, view, s.geometric, c.specular_roughness, c.base_metalness, c.base_color, slot, bounce, thr, rad);
                if (!cache_query) {
                float3 iface = dot(s.geometric, view) > 0.f ? s.geometric : s.face;
                Prepared pr = transport_prepare(p.lut, c, view, s.geometric, iface);
                BsdfSample smp = transport_sample(c, view, sc.x, sc.y, sc.z, pr);
                if (!finite3(smp.dir) || !finite3(smp.weight) || !isfinite(smp.pdf)) {
                    meta |= META_NONFINITE;
                } else {
                    // The image-environment and mesh strategies first: their shadow rays go
                    // to the slot's own buffers at once, so nothing of theirs stays live
                    // across the analytic estimate (the sample groups and the order of the
                    // sums in the shadow kernel do not depend on this order).
                    // environment_next_event (path.slang:1096-1120): a proposal direction,
                    // the diffuse and specular responses MIS-weighted against continuing
                    // there (continuation_mask, path.slang:1003-1010), one visibility ray
                    // to infinity; clamped on its own.
                    bool trace_c = false, trace_d = false;
                    uint32_t cont = 0u;
                    if (EXT && bounce < J.bounces[0]) {
                        if (diffuse < J.bounces[1]) cont |= VKB_RAY_DIFFUSE;
                        if (glossy < J.bounces[2] && (diffuse == 0u || (J.caustics & 1u))) cont |= VKB_RAY_SPECULAR;
                    }
                    if (EXT && J.env_w) {
                        const float4 eu = sample_group(pseed, sidx, J.sample_mask, vertex_group(vtx, 3));   // path_environment
                        float epdf = 0.f;
                        const float3 edir = env_sample(J, eu.x, eu.y, epdf);
                        float3 ev = f3(0.f);
                        if (epdf > 0.f) {
                            const float3 emitted = env_radiance(J, edir);
                            if (maxc(emitted) > 0.f) {
                                #pragma unroll
                                for (int k = 0; k < 2; ++k) {
                                    const uint32_t event = k == 0 ? VKB_RAY_DIFFUSE : VKB_RAY_SPECULAR;
                                    if (!event_hemisphere(event, edir, s.face, s.geometric)) continue;
                                    const float3 response = eval_mask(c, view, edir, event, pr);
                                    if (maxc(response) <= 0.f) continue;
                                    const float bpdf = (cont & event) ? pdf_mask(c, view, edir, event, pr) : 0.f;
                                    ev = ev + emitted * response * (mis_power(epdf, bpdf) / epdf);
                                }
                            }
                        }
                        if (any_nonzero(ev)) {
                            const float3 oc = path_origin(s, edir), cc = thr * ev;
                            p.sc_o[slot] = make_float4(oc.x, oc.y, oc.z, FP32_MAX);
                            p.sc_d[slot] = make_float4(edir.x, edir.y, edir.z, 0.f);
                            p.sc_c[slot] = make_float4(cc.x, cc.y, cc.z, 0.f);
                            trace_c = true;
                        }
                    }
                    if (EXT && J.em_tris) {
                        // mesh_next_event (path.slang:1121-1167), constant emission: a point on a
                        // source triangle, the diffuse and specular responses MIS-weighted against
                        // continuing there, one visibility ray between the offset end points.
                        const float4 g = sample_group(pseed, sidx, J.sample_mask, vertex_group(vtx, 2));   // path_triangle
                        uint32_t ei, ep; float b1, b2;
                        if (em_sample(J, g.z, g.x, g.y, ei, ep, b1, b2)) {
                            const EmGeometry eg = em_geometry(J, ei, ep, b1, b2);
                            const float3 delta = eg.point - s.world;
                            const float distance = length(delta);
                            if (distance > 0.f) {
                                const float3 axis = delta / distance;
                                const float mpdf = mesh_pdf(J, ei, ep, eg.area, s.world, eg.point, eg.face);
                                const vkb_material& em = J.materials[__ldg(&J.inst_info[ei]).y];
                                const bool front = dot(eg.face, axis) < 0.f;
                                const float3 emitted = get3(em.emission_color) * em.emission_luminance;
                                if (mpdf > 0.f && ((em.flags & 2u) || front) && maxc(emitted) > 0.f) {
                                    const float3 start = path_origin(s, axis);
                                    const float3 end = surface_ray_origin(eg.point, eg.error, front ? eg.face : -eg.face, -axis);
                                    const float3 connection = end - start;
                                    const float extent = length(connection);
                                    float3 response = f3(0.f);
                                    if (extent > 0.f) {
                                        #pragma unroll
                                        for (int k = 0; k < 2; ++k) {
                                            const uint32_t event = k == 0 ? VKB_RAY_DIFFUSE : VKB_RAY_SPECULAR;
                                            if (!event_hemisphere(event, axis, s.face, s.geometric)) continue;
                                            const float3 f = eval_mask(c, view, axis, event, pr);
                                            if (maxc(f) <= 0.f) continue;
                                            const float bpdf = (cont & event) ? pdf_mask(c, view, axis, event, pr) : 0.f;
                                            response = response + f * mis_power(mpdf, bpdf);
                                        }
                                    }
                                    if (any_nonzero(response)) {
                                        const float3 md = thr * (response * emitted / mpdf), cdir = connection / extent;
                                        p.sd_o[slot] = make_float4(start.x, start.y, start.z, extent);
                                        p.sd_d[slot] = make_float4(cdir.x, cdir.y, cdir.z, 0.f);
                                        p.sd_c[slot] = make_float4(md.x, md.y, md.z, 0.f);
                                        trace_d = true;
                                    }
                                }
                            }
                        }
                    }
                    // next_event (path.slang:851-951): one analytic light, two estimators.
                    float3 va = f3(0.f), vb = f3(0.f);
                    bool trace_a = false, has_b = false, trace_b = false;
                    float3 oa, da, ob, db; float la = 0.f, lb = 0.f;
                    if (J.num_lights > 0) {
                        float4 u = sample_group(pseed, sidx, J.sample_mask, vertex_group(vtx, 1));   // path_light
                        float probability;
                        uint32_t li = tree_pick(J.tree, J.tree_nodes, s.world, u.z, u.w, probability);
                        if (probability > 0.f && li < J.num_lights) {
                            const vkb_light& L = J.lights[li];
                            uint32_t contribution = L.shadow_offsets[VKB_LIGHT_CONTRIBUTION_WORD];
                            bool shadowed = (L.shadow_offsets[VKB_LIGHT_RAY_WORD] & VKB_LIGHT_RAY_SHADOWED) != 0u;
                            if ((contribution & VKB_LIGHT_LINK_ALL) || L.shadow_offsets[VKB_LIGHT_LINK_WORD]) {
                                LightSample src = emitter_sample(L, s.world, u.x, u.y);
                                float3 power = src.delta ? src.radiance : (src.pdf > 0.f ? src.radiance / src.pdf : f3(0.f));
                                va = analytic_mis_response(c, view, src.dir, s.face, contribution, src.pdf, pr) * power / probability;
                                va = light_threshold(va, J.light_threshold, rng);
                                if (any_nonzero(va) && shadowed) {
                                    oa = path_origin(s, src.dir);
                                    ray_connection(oa, s.world, src.dir, src.distance, da, la);
                                    trace_a = true;
                                }
                                bool continuation = (contribution & smp.event) && event_hemisphere(smp.event, smp.dir, s.face, s.geometric);
                                if (continuation && dot(smp.dir, smp.dir) > 0.f) {
                                    EmitterEval e = emitter_eval(L, s.world, smp.dir);
                                    if (e.pdf > 0.f) {
                                        float w = smp.pdf > 0.f ? mis_power(smp.pdf, e.pdf) : 1.f;
                                        vb = light_threshold(smp.weight * e.radiance * (w / probability), J.light_threshold, rng);
                                        if (any_nonzero(vb)) {
                                            has_b = true;
                                            if (shadowed) {
                                                ob = path_origin(s, smp.dir);
                                                ray_connection(ob, s.world, smp.dir, e.distance, db, lb);
                                                trace_b = true;
                                            }
                                        }
                                    }
                                }
                            }
                        }
                    }
                    float3 ca = thr * va, cb = thr * vb;
                    if (trace_a || trace_b || trace_c || trace_d) {
                        push_shadow = true;
                        uint32_t flags = (trace_a ? SH_TRACE_A : 0u) | (has_b ? SH_HAS_B : 0u) | (trace_b ? SH_TRACE_B : 0u) | (bounce == 0 ? SH_DIRECT : 0u) |
                                         (trace_c ? SH_HAS_C : 0u) | (trace_d ? SH_HAS_D : 0u);
                        sh_o = make_float4(oa.x, oa.y, oa.z, la);
                        sh_d = make_float4(da.x, da.y, da.z, __uint_as_float(slot));
                        sh_c = make_float4(ca.x, ca.y, ca.z, __uint_as_float(flags));
                        if (!trace_a) sh_o = make_float4(0.f, 0.f, 0.f, 0.f);
#if VKB_SHADE_EARLY_APPEND
                        {
                            const uint32_t si = group_append(&p.counters[2]);
                            p.sa_o[si] = sh_o; p.sa_d[si] = sh_d; p.sa_c[si] = sh_c;
                            push_shadow = false;
                        }
#endif
                        if (has_b) {
                            p.sb_c[slot] = make_float4(cb.x, cb.y, cb.z, 0.f);
                            if (trace_b) { p.sb_o[slot] = make_float4(ob.x, ob.y, ob.z, lb); p.sb_d[slot] = make_float4(db.x, db.y, db.z, 0.f); }
                        }
                    } else {
                        rad = rad + clamp_sample(ca + cb, limit, dropped);
                    }
                    // Continuation (path.slang:1683-1708).
                    bool go = bounce < J.bounces[0];
                    uint32_t event = smp.event;
                    if (go) {
                        if (event == VKB_RAY_DIFFUSE) { if (diffuse++ >= J.bounces[1]) go = false; }
                        else if (event == VKB_RAY_SPECULAR) { if (glossy++ >= J.bounces[2] || (diffuse > 0 && !(J.caustics & 1u))) go = false; }
                        else go = false;
                    }
                    if (go && !event_hemisphere(event, smp.dir, s.face, s.geometric)) go = false;
                    if (go) {
                        thr = thr * smp.weight;
                        if (!finite3(thr)) { meta |= META_NONFINITE; go = false; }
                        else if (maxc(thr) <= 0.f) go = false;
                    }
                    if (go && bounce >= ROULETTE_START) {
                        float survive = clampf(maxc(thr), ROULETTE_MIN, ROULETTE_MAX);
                        float4 dec = sample_group(pseed, sidx, J.sample_mask, vertex_group(vtx, 4));
                        if (dec.z > survive) go = false;
                        else thr = thr / survive;
                    }
                    if (go) {
                        float3 o = path_origin(s, smp.dir);
                        new_o = make_float4(o.x, o.y, o.z, FP32_MAX);
                        new_d = make_float4(smp.dir.x, smp.dir.y, smp.dir.z, __uint_as_float(slot));
                        push_ray = true;
                        if (EXT) p.prev[slot] = make_float4(s.world.x, s.world.y, s.world.z, smp.pdf);
#if VKB_SHADE_EARLY_APPEND
                        {
#if VKB_SHADE_OCTANT_APPEND
                            const uint32_t oct = (smp.dir.x < 0.f ? 1u : 0u) | (smp.dir.y < 0.f ? 2u : 0u) | (smp.dir.z < 0.f ? 4u : 0u);
                            const uint32_t ri = group_append_by_key(&p.counters[nxt], oct);
#else
                            const uint32_t ri = group_append(&p.counters[nxt]);
#endif
                            p.ray_o[nxt][ri] = new_o; p.ray_d[nxt][ri] = new_d;
                            push_ray = false;
                        }
#endif
                        meta = (meta & META_NONFINITE) | ((bounce + 1u) & 0xffu) | ((diffuse & 0xffu) << 8) | ((glossy & 0xffu) << 16) | ((event & 0x3fu) << 24);
                    }
                }
                }  // !cache_query
            }
            p.thr[slot] = make_float4(thr.x, thr.y, thr.z, __uint_as_float(meta));
            p.rad[slot] = make_float4(rad.x, rad.y, rad.z, __uint_as_float(dropped));
            p.rng[slot] = make_uint2(rng, pseed);
        }
        uint32_t ri = warp_append(&p.counters[nxt], push_ray);
        if (push_ray) { p.ray_o[nxt][ri] = new_o; p.ray_d[nxt][ri] = new_d; }
        uint32_t si = warp_append(&p.counters[2], push_shadow);
        if (push_shadow) { p.sa_o[si] = sh_o; p.sa_d[si] = sh_d; p.sa_c[si] = sh_c; }
    }
}
// Seed the first ray queue's count from the wave's path-slot count.
__global__ void k_start_wave(uint32_t* counters, uint32_t append_camera) {
    counters[0] = append_camera ? 0u : counters[7];
    counters[9] = 0u;
    counters[11] = 0u;   // trace fetch counters (closest, shadow)
    counters[12] = 0u;
}
// Adaptive sampling, before the wave of sample index i = wave_first (path.slang:1797-1835):
// reset at i = 0; from the minimum on a pixel is settled when every channel's standard
// error of the mean is within threshold x max(|mean|, 0.01); it publishes that in its
// parity slot (i & 1) and stops once it and its whole 3x3 neighbourhood were settled at
// the previous sample (slot (i & 1) ^ 1, which nothing writes during this kernel).
__global__ void k_adaptive_decide(PathParams p) {
    const Job& J = p.job0;
    const uint32_t i = J.wave_first, w = J.cam.width, h = J.cam.height;
    uint32_t skipped = 0;
    for (uint32_t px = blockIdx.x * blockDim.x + threadIdx.x; px < J.npix; px += gridDim.x * blockDim.x) {
        uint32_t st = J.ad_state[px];
        if (i == 0u) {
            st &= ~AD_STOPPED;
            J.ad_mean[px] = make_float4(0.f, 0.f, 0.f, 0.f);
            J.ad_m2[px] = make_float4(0.f, 0.f, 0.f, 0.f);
        }
        if (st & AD_STOPPED) { ++skipped; continue; }
        bool settled = false;
        if (i >= J.adaptive_min) {
            const float4 m = J.ad_mean[px], v = J.ad_m2[px];
            const float a1 = float(max(i - 1u, 1u)), a2 = float(i);
            const float e[4] = {sqrtf(fmaxf(v.x / a1 / a2, 0.f)), sqrtf(fmaxf(v.y / a1 / a2, 0.f)), sqrtf(fmaxf(v.z / a1 / a2, 0.f)),
                                sqrtf(fmaxf(v.w / a1 / a2, 0.f))};
            const float a[4] = {m.x, m.y, m.z, m.w};
            settled = true;
            for (int c = 0; c < 4; ++c) settled = settled && e[c] <= J.adaptive_threshold * fmaxf(fabsf(a[c]), .01f);
        }
        const uint32_t bit = 1u << (i & 1u), prev = 1u << ((i & 1u) ^ 1u);
        bool done = settled;
        const int x = int(px % w), y = int(px / w);
        for (int dy = -1; dy <= 1 && done; ++dy)
            for (int dx = -1; dx <= 1 && done; ++dx) {
                const int nx = min(max(x + dx, 0), int(w) - 1), ny = min(max(y + dy, 0), int(h) - 1);
                done = (J.ad_state[uint32_t(ny) * w + uint32_t(nx)] & prev) != 0u;
            }
        st = settled ? (st | bit) : (st & ~bit);
        if (done) { st |= AD_STOPPED; ++skipped; }
        J.ad_state[px] = st;   // neighbours read only the other parity bit of this word
    }
    for (int off = 16; off > 0; off >>= 1) skipped += __shfl_xor_sync(0xffffffffu, skipped, off);
    if ((threadIdx.x & 31u) == 0u && skipped) atomicAdd(&p.counters[10], skipped);
}
// Zero the next ray queue and the shadow queue before a shade pass.
__global__ void k_reset_queues(uint32_t* counters, int nxt) { counters[nxt] = 0u; counters[2] = 0u; counters[11] = 0u; counters[12] = 0u; }
// Denoiser guides of this wave's camera hits (path.slang:1549-1571): per path slot the
// hit's guide albedo (w = 1: coverage) and shading normal, zero on a miss.  Runs between
// the bounce-0 closest-hit trace and the shade pass of single-job guide renders.
__global__ void k_guides(PathParams p) {
    const uint32_t n = p.counters[0];
    const Job& J = p.job0;
    for (uint32_t i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x) {
        const float4 rd = p.ray_d[0][i], hh = p.hit[i];
        const uint32_t slot = __float_as_uint(rd.w);
        float4 ga = make_float4(0.f, 0.f, 0.f, 0.f), gn = ga;
        if (hh.x >= 0.f) {
            const uint32_t inst = p.hit_inst[i];
            const float3 dir = f3(rd.x, rd.y, rd.z);
            const Surface s = hit_surface(J, inst, __float_as_uint(hh.w), hh.y, hh.z, dir);
            const vkb_material& mt = J.materials[__ldg(&J.inst_info[inst]).y];
            Closure c;
            c.base_color = get3(mt.base_color); c.base_weight = mt.base_weight; c.base_metalness = mt.base_metalness;
            c.specular_color = get3(mt.specular_color); c.specular_weight = mt.specular_weight;
            c.specular_roughness = mt.specular_roughness; c.specular_ior = mt.specular_ior; c.optical_ior = 0.f;
            c.n = s.geometric;
            boundary_closure_air(c);
            const float3 a = guide_albedo(p.lut, c, -dir);
            ga = make_float4(a.x, a.y, a.z, 1.f);
            gn = make_float4(c.n.x, c.n.y, c.n.z, 0.f);
        }
        p.guide[2 * size_t(slot)] = ga;
        p.guide[2 * size_t(slot) + 1] = gn;
    }
}
// resolve.slang:162-191: add this wave's finished samples to each job's accumulator,
// one sample at a time in sample order (any wave size gives the same sums).
template <bool BATCH>
__global__ void k_accumulate(PathParams p) {
    const uint32_t n = p.counters[8];
    for (uint32_t g = blockIdx.x * blockDim.x + threadIdx.x; g < n; g += gridDim.x * blockDim.x) {
        const Job& J = BATCH ? p.jobs[find_job<true>(p, g)] : p.job0;
        uint32_t pixel = g - J.pixel_base;
        if (pixel >= J.npix || J.wave_samples == 0) continue;
        float4 sum = J.accum[pixel];
        uint32_t dl = 0, dp = 0;
        if (!BATCH && J.adaptive) {
            // One sample per wave: a stopped pixel adds its stopped mean; a live one its
            // value, which also updates its moments (Welford, path.slang:1963-1965; a
            // dropped non-finite sample is the zero RGBA value).
            const uint32_t slot = J.slot_base + pixel;
            const float4 m = J.ad_mean[pixel];
            if (J.ad_state[pixel] & AD_STOPPED) {
                sum.x += m.x; sum.y += m.y; sum.z += m.z; sum.w += 1.f;
            } else {
                float4 T = p.thr[slot], R = p.rad[slot];
                dl += __float_as_uint(R.w);
                float3 v = f3(R.x, R.y, R.z) * J.env.exposure;
                float alpha = 1.f;
                if ((__float_as_uint(T.w) & META_NONFINITE) || !finite3(v)) { v = f3(0.f); alpha = 0.f; dp++; }
                sum.x += v.x; sum.y += v.y; sum.z += v.z; sum.w += 1.f;
                const float inv = 1.f / float(J.wave_first + 1u);
                const float4 d = make_float4(v.x - m.x, v.y - m.y, v.z - m.z, alpha - m.w);
                const float4 nm = make_float4(m.x + d.x * inv, m.y + d.y * inv, m.z + d.z * inv, m.w + d.w * inv);
                float4 m2 = J.ad_m2[pixel];
                m2.x += d.x * (v.x - nm.x); m2.y += d.y * (v.y - nm.y); m2.z += d.z * (v.z - nm.z); m2.w += d.w * (alpha - nm.w);
                J.ad_mean[pixel] = nm;
                J.ad_m2[pixel] = m2;
            }
        } else if (!BATCH && J.guide_accum) {
            // Guide renders: the guides of a dropped sample are zero too (path.slang:1946-1950).
            float4 ga = J.guide_accum[2 * pixel], gn = J.guide_accum[2 * pixel + 1];
            for (uint32_t k = 0; k < J.wave_samples; ++k) {
                uint32_t slot = J.slot_base + k * J.npix + pixel;
                float4 T = p.thr[slot], R = p.rad[slot];
                dl += __float_as_uint(R.w);
                float3 v = f3(R.x, R.y, R.z) * J.env.exposure;
                const bool drop = (__float_as_uint(T.w) & META_NONFINITE) || !finite3(v);
                if (drop) { v = f3(0.f); dp++; }
                sum.x += v.x; sum.y += v.y; sum.z += v.z; sum.w += 1.f;
                if (!drop) {
                    const float4 a = p.guide[2 * size_t(slot)], nn = p.guide[2 * size_t(slot) + 1];
                    ga.x += a.x; ga.y += a.y; ga.z += a.z; ga.w += a.w;
                    gn.x += nn.x; gn.y += nn.y; gn.z += nn.z;
                }
            }
            J.guide_accum[2 * pixel] = ga;
            J.guide_accum[2 * pixel + 1] = gn;
        } else
        for (uint32_t k = 0; k < J.wave_samples; ++k) {
            uint32_t slot = J.slot_base + k * J.npix + pixel;
            float4 T = p.thr[slot], R = p.rad[slot];
            dl += __float_as_uint(R.w);
            float3 v = f3(R.x, R.y, R.z) * J.env.exposure;
            if ((__float_as_uint(T.w) & META_NONFINITE) || !finite3(v)) { v = f3(0.f); dp++; }
            sum.x += v.x; sum.y += v.y; sum.z += v.z; sum.w += 1.f;
        }
        J.accum[pixel] = sum;
        if (dl) atomicAdd(&p.counters[5], dl);
        if (dp) atomicAdd(&p.counters[6], dp);
    }
}
// Mean image of every job (pixels numbered across jobs by pixel_base).
template <bool BATCH>
__global__ void k_resolve(PathParams p, uint32_t total_pixels) {
    for (uint32_t g = blockIdx.x * blockDim.x + threadIdx.x; g < total_pixels; g += gridDim.x * blockDim.x) {
        const Job& J = BATCH ? p.jobs[find_job<true>(p, g)] : p.job0;
        uint32_t i = g - J.pixel_base;
        if (i >= J.npix) continue;
        float4 a = J.accum[i];
        float inv = a.w > 0.f ? 1.f / a.w : 0.f;
        J.out[i] = make_float4(a.x * inv, a.y * inv, a.z * inv, a.w > 0.f ? 1.f : 0.f);
        if (!BATCH && J.guide_accum) {
            const float4 ga = J.guide_accum[2 * i], gn = J.guide_accum[2 * i + 1];
            if (J.guide_albedo) J.guide_albedo[i] = make_float4(ga.x * inv, ga.y * inv, ga.z * inv, ga.w * inv);
            if (J.guide_normal) J.guide_normal[i] = make_float4(gn.x * inv, gn.y * inv, gn.z * inv, 0.f);
        }
    }
}
// Test entry: sampler groups for arbitrary (pixel, index, group).
__global__ void k_sampler_groups(uint32_t n, const uint32_t* px, const uint32_t* py, const uint32_t* index, const uint32_t* groups,
                                 uint32_t mask, uint32_t stream, uint4* out) {
    for (uint32_t i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x) {
        uint32_t seed = screen_ray_hash(px[i], py[i], 0u, stream);
        out[i] = sample_group_bits(seed, index[i], mask, groups[i]);
    }
}
// Test entry: closest hits of arbitrary world rays.
template <bool W8>
__global__ void __launch_bounds__(TRACE_BLOCK) k_debug_trace(SceneView sv, uint32_t n, const float4* rays, float* t, uint32_t* ids, float* uv, uint32_t* err) {
    VKB_STACK_DECL_W(W8)
    for (uint32_t i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x) {
        HitRecord h;
        bool f = trace_any<false, false, W8>(sv, RayRef{rays, rays + n, i}, rays[i].w, h, err, nullptr, stk);
        t[i] = f ? h.t : -1.f;
        ids[2 * i] = f ? h.inst : 0xffffffffu; ids[2 * i + 1] = f ? __float_as_uint(__ldg(&sv.blas_tris[3u * size_t(h.tri)]).w) : 0xffffffffu;
        uv[2 * i] = f ? h.u : 0.f; uv[2 * i + 1] = f ? h.v : 0.f;
    }
}
// Occlusion of n world rays by the shadow rays' any-hit traversal (first hit ends the
// walk, no back-face culling): occluded[i] = 1 when anything lies within (0, tmax).
template <bool W8>
__global__ void __launch_bounds__(TRACE_BLOCK) k_debug_occluded(SceneView sv, uint32_t n, const float4* rays, uint32_t* occluded, uint32_t* err) {
    VKB_STACK_DECL_W(W8)
    for (uint32_t i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x) {
        HitRecord h;
        occluded[i] = trace_any<true, false, W8>(sv, RayRef{rays, rays + n, i}, rays[i].w, h, err, nullptr, stk) ? 1u : 0u;
    }
}

}  // namespace vkb
