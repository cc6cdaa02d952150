// Eight-wide BVH with quantized child boxes, collapsed on the device from the binary
// LBVH (in the spirit of Ylitie, Karras & Laine, "Efficient Incoherent Ray Traversal on
// GPUs Through Compressed Wide BVHs", HPG 2017: 8-bit child planes relative to a node
// origin with a power-of-two scale per axis).  One 128-byte node per visit replaces
// about three dependent BVH2 visits; the traversal is latency-bound, so fewer dependent
// fetches is the lever.
#pragma once
#include <cstdint>
#include "vkb_bvh.cuh"

namespace vkb {

// 128 bytes: origin + packed exponents/count, 8 child references, 48 bytes of planes.
//   h    = (origin.x, origin.y, origin.z, bits: ex | ey<<8 | ez<<16 | count<<24), exponents biased by 127
//   r0,r1= child references: >= 0 wide node, < 0 ~leaf (sorted primitive index)
//   q0   = (lo.x[0..3], lo.x[4..7], lo.y[0..3], lo.y[4..7]) bytes
//   q1   = (lo.z[0..3], lo.z[4..7], hi.x[0..3], hi.x[4..7])
//   q2   = (hi.y[0..3], hi.y[4..7], hi.z[0..3], hi.z[4..7])
struct alignas(128) WideNode { float4 h; int4 r0, r1; uint4 q0, q1, q2; uint4 pad[2]; };

struct WideBox { float lo[3], hi[3]; };
__device__ __forceinline__ float box_area(const WideBox& b) {
    float x = fmaxf(b.hi[0] - b.lo[0], 0.f), y = fmaxf(b.hi[1] - b.lo[1], 0.f), z = fmaxf(b.hi[2] - b.lo[2], 0.f);
    return x * y + y * z + z * x;
}
__device__ __forceinline__ WideBox child_box(const BvhNode& n, int side) {
    WideBox b;
    if (side == 0) { b.lo[0] = n.a.x; b.hi[0] = n.a.y; b.lo[1] = n.a.z; b.hi[1] = n.a.w; b.lo[2] = n.c.x; b.hi[2] = n.c.y; }
    else { b.lo[0] = n.b.x; b.hi[0] = n.b.y; b.lo[1] = n.b.z; b.hi[1] = n.b.w; b.lo[2] = n.c.z; b.hi[2] = n.c.w; }
    return b;
}

// One collapse step per work item (binary node -> wide node): grow a frontier of up
// to 8 subtrees by repeatedly opening the internal element of largest area, quantize
// the frontier into the wide node, allocate wide nodes for internal elements and
// queue them.  work[i] = (binary node, wide node).
// Levels run back to back with three rotating counters: level L reads counter L%3,
// appends to counter (L+1)%3 and clears counter (L+2)%3 for level L+1 (no host sync).
__global__ void k_collapse(const BvhNode* bin, WideNode* wide, const uint2* work_in, const uint32_t* n_in, uint2* work_out,
                           uint32_t* n_out, uint32_t* wide_count, uint32_t* n_clear) {
    if (blockIdx.x == 0 && threadIdx.x == 0) *n_clear = 0u;
    uint32_t n = *n_in;
    for (uint32_t i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x) {
        uint2 w = work_in[i];
        BvhNode root = bin[w.x];
        int ref[8];
        WideBox box[8];
        int count = 2;
        ref[0] = root.d.x; box[0] = child_box(root, 0);
        ref[1] = root.d.y; box[1] = child_box(root, 1);
        // An empty right box (a one-primitive tree) has lo > hi: drop it.
        if (box[1].lo[0] > box[1].hi[0]) count = 1;
        while (count < 8) {
            int best = -1;
            float best_area = -1.f;
            for (int k = 0; k < count; ++k)
                if (ref[k] >= 0) { float a = box_area(box[k]); if (a > best_area) { best_area = a; best = k; } }
            if (best < 0) break;
            BvhNode c = bin[ref[best]];
            ref[best] = c.d.x; box[best] = child_box(c, 0);
            ref[count] = c.d.y; box[count] = child_box(c, 1);
            ++count;
        }
        float lo[3] = {INFINITY, INFINITY, INFINITY}, hi[3] = {-INFINITY, -INFINITY, -INFINITY};
        for (int k = 0; k < count; ++k)
            for (int a = 0; a < 3; ++a) { lo[a] = fminf(lo[a], box[k].lo[a]); hi[a] = fmaxf(hi[a], box[k].hi[a]); }
        int e[3];
        float scale[3];
        for (int a = 0; a < 3; ++a) {
            float ext = __fsub_ru(hi[a], lo[a]);
            int ex = ext > 0.f ? int(ceilf(log2f(ext / 255.f))) : -100;
            // Guard the float log: the scale must cover the extent in 255 steps.
            while (ex < 127 && ldexpf(255.f, ex) < ext) ++ex;
            ex = max(ex, -100);
            e[a] = ex;
            scale[a] = ldexpf(1.f, ex);
        }
        uint8_t q[6][8];
        for (int k = 0; k < 8; ++k)
            for (int a = 0; a < 3; ++a) {
                if (k < count) {
                    float l = floorf(__fsub_rd(box[k].lo[a], lo[a]) / scale[a]);
                    float h = ceilf(__fsub_ru(box[k].hi[a], lo[a]) / scale[a]);
                    q[a][k] = uint8_t(fminf(fmaxf(l, 0.f), 255.f));
                    q[3 + a][k] = uint8_t(fminf(fmaxf(h, 0.f), 255.f));
                } else {
                    q[a][k] = 255; q[3 + a][k] = 0;  // empty: lo > hi never hits
                }
            }
        int refs[8];
        uint32_t internal = 0;
        for (int k = 0; k < count; ++k) internal += ref[k] >= 0 ? 1u : 0u;
        uint32_t base = internal ? atomicAdd(wide_count, internal) : 0u;
        uint32_t qbase = internal ? atomicAdd(n_out, internal) : 0u;
        uint32_t j = 0;
        for (int k = 0; k < 8; ++k) {
            if (k >= count) { refs[k] = SENTINEL; continue; }
            if (ref[k] >= 0) {
                refs[k] = int(base + j);
                work_out[qbase + j] = make_uint2(uint32_t(ref[k]), base + j);
                ++j;
            } else {
                refs[k] = ref[k];
            }
        }
        auto pack = [&](int row, int half) {
            return uint32_t(q[row][4 * half]) | (uint32_t(q[row][4 * half + 1]) << 8) | (uint32_t(q[row][4 * half + 2]) << 16) |
                   (uint32_t(q[row][4 * half + 3]) << 24);
        };
        WideNode node;
        node.h = make_float4(lo[0], lo[1], lo[2],
                             __uint_as_float(uint32_t(e[0] + 127) | (uint32_t(e[1] + 127) << 8) | (uint32_t(e[2] + 127) << 16) | (uint32_t(count) << 24)));
        node.r0 = make_int4(refs[0], refs[1], refs[2], refs[3]);
        node.r1 = make_int4(refs[4], refs[5], refs[6], refs[7]);
        node.q0 = make_uint4(pack(0, 0), pack(0, 1), pack(1, 0), pack(1, 1));
        node.q1 = make_uint4(pack(2, 0), pack(2, 1), pack(3, 0), pack(3, 1));
        node.q2 = make_uint4(pack(4, 0), pack(4, 1), pack(5, 0), pack(5, 1));
        node.pad[0] = node.pad[1] = make_uint4(0u, 0u, 0u, 0u);
        wide[w.y] = node;
    }
}
// A one-primitive binary tree becomes a wide root with one leaf child.
__global__ void k_collapse_seed(uint2* work, uint32_t* n_work, uint32_t* wide_count) {
    work[0] = make_uint2(0u, 0u);
    *n_work = 1u;
    *wide_count = 1u;
}

// Byte k of w as a float: one byte permute builds 2^23 + byte, one exact subtract removes 2^23.
__device__ __forceinline__ float byte_f(uint32_t w, int k) {
    return __uint_as_float(__byte_perm(w, 0x4b000000u, uint32_t(k) | 0x7440u)) - 8388608.f;
}
__device__ __forceinline__ int pick8(const int r[8], int k) {
    int v = r[0];
#pragma unroll
    for (int i = 1; i < 8; ++i) v = k == i ? r[i] : v;
    return v;
}

// Closest hit (ANY = false) or first hit (ANY = true) over the two-level wide BVH.
// A node visit tests all children into a hit mask (unrolled, registers only), tests
// BLAS triangle leaves at once, descends into the nearest hit child and pushes the
// others with their entry distances; a popped entry farther than the current closest
// hit is skipped.
template <bool ANY, bool COUNT = false>
__device__ __forceinline__ bool trace_wide(const WideNode* tlas, const TlasLeaf* leaves, const WideNode* blas, const float4* tris,
                                           uint32_t num_instances, float3 o, float3 d, float tmax, HitRecord& hit, uint32_t* err,
                                           TraceCount* count, TraceStack stk) {
    constexpr int STACK = SMEM_STACK;
    if (num_instances == 0) return false;
    RaySpace rs;
    make_space(rs, o, d);
    int sp = 0;
    float tbest = tmax;
    bool found = false, in_blas = false, cull = false;
    const WideNode* nodes = tlas;
    uint32_t tri_base = 0, cur_instance = 0;
    int node = 0;
    for (uint32_t steps = 0;; ++steps) {
        if (steps >= TRACE_STEP_LIMIT) { atomicOr(err, 2u); return found; }
        if (node >= 0) {
            if (COUNT) { count->nodes++; if (in_blas) count->blas_nodes++; }
            const uint4* p = reinterpret_cast<const uint4*>(nodes + node);
            uint4 hb = __ldg(p);
            int4 r0 = __ldg(reinterpret_cast<const int4*>(p + 1)), r1 = __ldg(reinterpret_cast<const int4*>(p + 2));
            uint4 q0 = __ldg(p + 3), q1 = __ldg(p + 4), q2 = __ldg(p + 5);
            uint32_t meta = hb.w;
            int cnt = int(meta >> 24);
            // t = (origin + q*scale - o)/d = q*(scale/d) + (origin - o)/d; scale = 2^(e-127) from the exponent byte.
            float ax = __uint_as_float((meta & 0xffu) << 23) * rs.idir.x;
            float ay = __uint_as_float(((meta >> 8) & 0xffu) << 23) * rs.idir.y;
            float az = __uint_as_float(((meta >> 16) & 0xffu) << 23) * rs.idir.z;
            float bx = (__uint_as_float(hb.x) - rs.o.x) * rs.idir.x;
            float by = (__uint_as_float(hb.y) - rs.o.y) * rs.idir.y;
            float bz = (__uint_as_float(hb.z) - rs.o.z) * rs.idir.z;
            const int refs[8] = {r0.x, r0.y, r0.z, r0.w, r1.x, r1.y, r1.z, r1.w};
            float tn[8];
            uint32_t mask = 0u, leafmask = 0u;
#pragma unroll
            for (int k = 0; k < 8; ++k) {
                const int kk = k & 3;
                uint32_t wlx = k < 4 ? q0.x : q0.y, wly = k < 4 ? q0.z : q0.w, wlz = k < 4 ? q1.x : q1.y;
                uint32_t whx = k < 4 ? q1.z : q1.w, why = k < 4 ? q2.x : q2.y, whz = k < 4 ? q2.z : q2.w;
                float x0 = fmaf(byte_f(wlx, kk), ax, bx), x1 = fmaf(byte_f(whx, kk), ax, bx);
                float y0 = fmaf(byte_f(wly, kk), ay, by), y1 = fmaf(byte_f(why, kk), ay, by);
                float z0 = fmaf(byte_f(wlz, kk), az, bz), z1 = fmaf(byte_f(whz, kk), az, bz);
                float a = fmaxf(fmaxf(fminf(x0, x1), fminf(y0, y1)), fmaxf(fminf(z0, z1), 0.f));
                float b = fminf(fminf(fmaxf(x0, x1), fmaxf(y0, y1)), fminf(fmaxf(z0, z1), tbest));
                tn[k] = a;
                bool h = k < cnt && a <= b * 1.0000005f;
                mask |= h ? (1u << k) : 0u;
                leafmask |= (h && refs[k] < 0) ? (1u << k) : 0u;
            }
            if (in_blas) {
                // Triangle leaves: test now, nearest first is not needed (tbest prunes).
                uint32_t lm = leafmask;
                mask &= ~leafmask;
                while (lm) {
                    int k = __ffs(lm) - 1;
                    lm &= lm - 1u;
                    if (COUNT) count->tris++;
                    const float4* tp = tris + 3u * (tri_base + uint32_t(~pick8(refs, k)));
                    float4 v0 = __ldg(tp), v1 = __ldg(tp + 1), v2 = __ldg(tp + 2);
                    float t, b1, b2;
                    if (tri_test(rs, f3(v0.x, v0.y, v0.z), f3(v1.x, v1.y, v1.z), f3(v2.x, v2.y, v2.z), cull, tbest, t, b1, b2)) {
                        tbest = t; found = true;
                        hit.t = t; hit.u = b1; hit.v = b2; hit.prim = __float_as_uint(v0.w); hit.inst = cur_instance;
                        if (ANY) return true;
                    }
                }
            }
            if (mask) {
                // Nearest hit child next; the rest onto the stack with their entry distances.
                int nearest = 0;
                float best = INFINITY;
#pragma unroll
                for (int k = 0; k < 8; ++k)
                    if (((mask >> k) & 1u) && tn[k] < best) { best = tn[k]; nearest = k; }
                if (sp + __popc(mask) - 1 > STACK) { atomicOr(err, 1u); return found; }
#pragma unroll
                for (int k = 0; k < 8; ++k)
                    if (((mask >> k) & 1u) && k != nearest) { stk.r[sp * TRACE_BLOCK] = refs[k]; stk.t[sp * TRACE_BLOCK] = tn[k]; ++sp; }
                node = pick8(refs, nearest);
                if (!(in_blas && node < 0)) continue;
            }
        } else if (!in_blas) {
            // Instance leaf of the TLAS: enter its BLAS in object space.
            if (COUNT) count->instances++;
            const TlasLeaf* lf = leaves + (~node);
            float4 m0 = __ldg(&lf->w2o[0]), m1 = __ldg(&lf->w2o[1]), m2 = __ldg(&lf->w2o[2]);
            uint4 info = __ldg(reinterpret_cast<const uint4*>(&lf->instance));
            float3 oo = f3(m0.x * o.x + m0.y * o.y + m0.z * o.z + m0.w, m1.x * o.x + m1.y * o.y + m1.z * o.z + m1.w, m2.x * o.x + m2.y * o.y + m2.z * o.z + m2.w);
            float3 od = f3(m0.x * d.x + m0.y * d.y + m0.z * d.z, m1.x * d.x + m1.y * d.y + m1.z * d.z, m2.x * d.x + m2.y * d.y + m2.z * d.z);
            make_space(rs, oo, od);
            cur_instance = info.x;
            nodes = blas + info.y;
            tri_base = info.z;
            cull = !ANY && (info.w & LEAF_CULL_BACKFACES);
            if (sp >= STACK) { atomicOr(err, 1u); return found; }
            stk.r[sp * TRACE_BLOCK] = SENTINEL; stk.t[sp * TRACE_BLOCK] = 0.f; ++sp;
            in_blas = true;
            node = 0;
            continue;
        }
        // pop
        for (;;) {
            if (sp == 0) return found;
            --sp;
            node = stk.r[sp * TRACE_BLOCK];
            if (node == SENTINEL) {
                in_blas = false;
                make_space(rs, o, d);
                nodes = tlas;
                continue;
            }
            if (stk.t[sp * TRACE_BLOCK] <= tbest) break;
        }
    }
}

}  // namespace vkb
