// Learned radiance cache (neural radiance caching, Mueller et al. 2021, "Real-time
// Neural Radiance Caching for Path Tracing"): a multiresolution hash encoding of the
// hit position (Mueller et al. 2022, "Instant Neural Graphics Primitives") plus the
// outgoing direction and surface features, fed to a 5-layer, 64-wide MLP.  BF16
// operands, FP32 accumulation in tensor memory: every layer is a tcgen05.mma issued by
// one thread of the CTA, operands staged in shared memory in the no-swizzle canonical
// layout, accumulators read back with tcgen05.ld.
//
// Network:
//   input  x[64]: [0,32) hash grid, 16 levels x 2 features (trilinear); [32,48) real
//          spherical harmonics of the outgoing direction, bands 0..3; [48,51) shading
//          normal * 0.5 + 0.5; [51] roughness; [52,55) base colour; [55] metalness;
//          [56] 1 (bias input); [57,64) 0.
//   h1 = relu(W0 x), h2 = relu(W1 h1), h3 = relu(W2 h2), h4 = relu(W3 h3)  (64x64 each)
//   y  = W4 h4 (W4 16x64, rows 3..15 zero): outgoing radiance (RGB); queries use max(y, 0).
//   loss (training) = mean over rows and the 3 channels of (y - t)^2 / (sg(y)^2 + 0.01).
#pragma once
#include <cuda_bf16.h>
#include <cuda_fp16.h>
#include <stdint.h>

namespace vkb {
namespace nrc {

constexpr int WIDTH = 64;            // MLP width and input width
constexpr int OUT_ROWS = 16;         // output layer rows (N of the last MMA), 3 used
constexpr int LAYERS = 5;
constexpr int TILE = 128;            // rows per CTA tile (M of the MMAs)
constexpr int HASH_LEVELS = 16;
constexpr int HASH_FEATURES = 2;
constexpr uint32_t HASH_LOG2_T = 19;
constexpr uint32_t HASH_T = 1u << HASH_LOG2_T;
constexpr float HASH_BASE_RES = 16.f;
constexpr float HASH_MAX_RES = 2048.f;
// MLP parameters, row-major [out][in] per layer: 4 x 64x64 + 16x64.
constexpr uint32_t MLP_PARAMS = 4u * WIDTH * WIDTH + OUT_ROWS * WIDTH;
constexpr uint64_t HASH_PARAMS = uint64_t(HASH_LEVELS) * HASH_T * HASH_FEATURES;
constexpr float LOSS_EPS = 0.01f;

// ---------------------------------------------------------------- tile layout
// A 128 x 64 (or 64 x 64) BF16 tile in shared memory as 8x8 core matrices (8 rows x 16
// bytes): row r, 8-element chunk c at (r / 8) * 1024 + c * 128 + (r % 8) * 16 bytes.
// Read K-major (rows = M or N, chunks along K): SBO = 1024 (row groups), LBO = 128
// (K chunks), K step s of 16 at +256 s.  Read MN-major (chunks along M/N, rows = K):
// SBO = 128 (MN chunks), LBO = 1024 (K groups), K step s of 16 rows at +2048 s.
__host__ __device__ constexpr uint32_t tile_offset(uint32_t row, uint32_t chunk) { return (row >> 3) * 1024u + chunk * 128u + (row & 7u) * 16u; }
constexpr uint32_t TILE_BYTES = TILE * WIDTH * 2;       // 16 KiB
constexpr uint32_t W_BYTES = WIDTH * WIDTH * 2;         // 8 KiB
constexpr uint32_t W4_BYTES = OUT_ROWS * WIDTH * 2;     // 2 KiB

// Shared-memory matrix descriptor (no swizzle, sm_100 version 1).
__device__ __forceinline__ uint64_t smem_desc(uint32_t saddr, uint32_t lbo, uint32_t sbo) {
    return uint64_t((saddr >> 4) & 0x3fffu) | (uint64_t((lbo >> 4) & 0x3fffu) << 16) | (uint64_t((sbo >> 4) & 0x3fffu) << 32) |
           (uint64_t(1) << 46);
}
// Instruction descriptor, kind::f16: BF16 x BF16 -> F32, M, N, majors (0 = K, 1 = MN).
__host__ __device__ constexpr uint32_t instr_desc(uint32_t m, uint32_t n, uint32_t a_mn, uint32_t b_mn) {
    return (1u << 4) | (1u << 7) | (1u << 10) | (a_mn << 15) | (b_mn << 16) | ((n >> 3) << 17) | ((m >> 4) << 24);
}

__device__ __forceinline__ uint32_t smem_u32(const void* p) { return static_cast<uint32_t>(__cvta_generic_to_shared(p)); }

// ---------------------------------------------------------------- tcgen05 primitives
__device__ __forceinline__ void tmem_alloc(uint32_t dst_smem, uint32_t cols) {
    asm volatile("tcgen05.alloc.cta_group::1.sync.aligned.shared::cta.b32 [%0], %1;" ::"r"(dst_smem), "r"(cols));
    asm volatile("tcgen05.relinquish_alloc_permit.cta_group::1.sync.aligned;" ::);
}
__device__ __forceinline__ void tmem_dealloc(uint32_t taddr, uint32_t cols) {
    asm volatile("tcgen05.dealloc.cta_group::1.sync.aligned.b32 %0, %1;" ::"r"(taddr), "r"(cols));
}
__device__ __forceinline__ void tc_fence_before() { asm volatile("tcgen05.fence::before_thread_sync;" ::: "memory"); }
__device__ __forceinline__ void tc_fence_after() { asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory"); }
__device__ __forceinline__ void fence_async_smem() { asm volatile("fence.proxy.async.shared::cta;" ::: "memory"); }
__device__ __forceinline__ void mma_bf16(uint32_t d_tmem, uint64_t a, uint64_t b, uint32_t idesc, uint32_t accumulate) {
    asm volatile(
        "{\n\t.reg .pred p;\n\tsetp.ne.b32 p, %4, 0;\n\t"
        "tcgen05.mma.cta_group::1.kind::f16 [%0], %1, %2, %3, {%5, %6, %7, %8}, p;\n\t}\n" ::"r"(d_tmem),
        "l"(a), "l"(b), "r"(idesc), "r"(accumulate), "r"(0u), "r"(0u), "r"(0u), "r"(0u));
}
__device__ __forceinline__ void mma_commit(uint32_t mbar) {
    asm volatile("tcgen05.commit.cta_group::1.mbarrier::arrive::one.shared::cluster.b64 [%0];" ::"r"(mbar) : "memory");
}
__device__ __forceinline__ void mbar_init(uint32_t mbar, uint32_t count) {
    asm volatile("mbarrier.init.shared::cta.b64 [%0], %1;" ::"r"(mbar), "r"(count));
    asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
}
// Bounded wait for the barrier phase `parity`; false when the limit ran out.
__device__ __forceinline__ bool mbar_wait(uint32_t mbar, uint32_t parity) {
    for (uint32_t it = 0; it < (1u << 24); ++it) {
        uint32_t done;
        asm volatile("{\n\t.reg .pred p;\n\tmbarrier.try_wait.parity.shared::cta.b64 p, [%1], %2;\n\tselp.u32 %0, 1, 0, p;\n\t}\n"
                     : "=r"(done)
                     : "r"(mbar), "r"(parity)
                     : "memory");
        if (done) return true;
    }
    return false;
}
// 16 consecutive FP32 columns of this thread's TMEM lane.
__device__ __forceinline__ void tmem_ld16(uint32_t taddr, float (&v)[16]) {
    uint32_t r[16];
    asm volatile(
        "tcgen05.ld.sync.aligned.32x32b.x16.b32 {%0, %1, %2, %3, %4, %5, %6, %7, %8, %9, %10, %11, %12, %13, %14, %15}, [%16];"
        : "=r"(r[0]), "=r"(r[1]), "=r"(r[2]), "=r"(r[3]), "=r"(r[4]), "=r"(r[5]), "=r"(r[6]), "=r"(r[7]), "=r"(r[8]), "=r"(r[9]),
          "=r"(r[10]), "=r"(r[11]), "=r"(r[12]), "=r"(r[13]), "=r"(r[14]), "=r"(r[15])
        : "r"(taddr));
    asm volatile("tcgen05.wait::ld.sync.aligned;" ::: "memory");
#pragma unroll
    for (int i = 0; i < 16; ++i) v[i] = __uint_as_float(r[i]);
}

// Eight floats -> eight BF16 in one 16-byte chunk.
__device__ __forceinline__ uint4 pack8(const float* v) {
    uint4 q;
    __nv_bfloat162 a = __floats2bfloat162_rn(v[0], v[1]), b = __floats2bfloat162_rn(v[2], v[3]);
    __nv_bfloat162 c = __floats2bfloat162_rn(v[4], v[5]), d = __floats2bfloat162_rn(v[6], v[7]);
    q.x = *reinterpret_cast<uint32_t*>(&a); q.y = *reinterpret_cast<uint32_t*>(&b);
    q.z = *reinterpret_cast<uint32_t*>(&c); q.w = *reinterpret_cast<uint32_t*>(&d);
    return q;
}
__device__ __forceinline__ void unpack8(uint4 q, float* v) {
    const __nv_bfloat162* h = reinterpret_cast<const __nv_bfloat162*>(&q);
#pragma unroll
    for (int i = 0; i < 4; ++i) { float2 f = __bfloat1622float2(h[i]); v[2 * i] = f.x; v[2 * i + 1] = f.y; }
}

// ---------------------------------------------------------------- encoding
// Real spherical harmonics, bands 0..3 (16 values) of a unit vector (the standard
// Cartesian polynomials with their normalisation constants).
__host__ __device__ inline void sh16(float x, float y, float z, float* o) {
    const float xx = x * x, yy = y * y, zz = z * z;
    o[0] = 0.28209479177387814f;
    o[1] = -0.48860251190291987f * y;
    o[2] = 0.48860251190291987f * z;
    o[3] = -0.48860251190291987f * x;
    o[4] = 1.0925484305920792f * x * y;
    o[5] = -1.0925484305920792f * y * z;
    o[6] = 0.94617469575755997f * zz - 0.31539156525251999f;
    o[7] = -1.0925484305920792f * x * z;
    o[8] = 0.54627421529603959f * (xx - yy);
    o[9] = 0.59004358992664352f * y * (-3.f * xx + yy);
    o[10] = 2.8906114426405538f * x * y * z;
    o[11] = 0.45704579946446572f * y * (1.f - 5.f * zz);
    o[12] = 0.3731763325901154f * z * (5.f * zz - 3.f);
    o[13] = 0.45704579946446572f * x * (1.f - 5.f * zz);
    o[14] = 1.4453057213202769f * z * (xx - yy);
    o[15] = 0.59004358992664352f * x * (-xx + 3.f * yy);
}

// Grid resolution of level l: floor(16 * (2048/16)^(l/15)), evaluated in double once
// (a float evaluation can land either side of an integer at the finest level).
__constant__ uint32_t kLevelRes[HASH_LEVELS] = {16, 22, 30, 42, 58, 80, 111, 153, 212, 294, 406, 561, 776, 1072, 1482, 2048};
__device__ __forceinline__ float level_scale(int l) { return float(kLevelRes[l]); }
// Table index of grid vertex (x, y, z) at a level with `res` cells per axis: dense when
// (res + 1)^3 fits the table, else the spatial hash of the instant-NGP paper.
__host__ __device__ inline uint32_t grid_index(uint32_t x, uint32_t y, uint32_t z, uint32_t res) {
    const uint64_t side = uint64_t(res) + 1u;
    if (side * side * side <= HASH_T) return uint32_t(x + side * (y + side * z));
    return (x * 1u ^ y * 2654435761u ^ z * 805459861u) & (HASH_T - 1u);
}

// One cache record: where the query or training vertex is and what it looks like.
struct Record {
    float3 pos;        // normalised to [0,1]^3 by the scene box
    float3 wo;         // unit outgoing direction
    float3 normal;     // unit shading normal
    float roughness, metalness;
    float3 albedo;
};

// The 64 inputs of one record (hash features from the FP16 table).
__device__ __forceinline__ void encode(const Record& r, const __half* __restrict__ table, float* x) {
#pragma unroll 1
    for (int l = 0; l < HASH_LEVELS; ++l) {
        const float s = level_scale(l);
        const uint32_t res = uint32_t(s);
        const float px = fminf(fmaxf(r.pos.x, 0.f), 1.f) * s, py = fminf(fmaxf(r.pos.y, 0.f), 1.f) * s, pz = fminf(fmaxf(r.pos.z, 0.f), 1.f) * s;
        const uint32_t cx = min(uint32_t(px), res - 1u), cy = min(uint32_t(py), res - 1u), cz = min(uint32_t(pz), res - 1u);
        const float fx = px - float(cx), fy = py - float(cy), fz = pz - float(cz);
        float f0 = 0.f, f1 = 0.f;
        const __half2* lvl = reinterpret_cast<const __half2*>(table) + size_t(l) * HASH_T;
#pragma unroll
        for (int c = 0; c < 8; ++c) {
            const uint32_t dx = c & 1u, dy = (c >> 1) & 1u, dz = (c >> 2) & 1u;
            const float w = (dx ? fx : 1.f - fx) * (dy ? fy : 1.f - fy) * (dz ? fz : 1.f - fz);
            const float2 v = __half22float2(__ldg(lvl + grid_index(cx + dx, cy + dy, cz + dz, res)));
            f0 = fmaf(w, v.x, f0);
            f1 = fmaf(w, v.y, f1);
        }
        x[2 * l] = f0;
        x[2 * l + 1] = f1;
    }
    sh16(r.wo.x, r.wo.y, r.wo.z, x + 32);
    x[48] = r.normal.x * 0.5f + 0.5f; x[49] = r.normal.y * 0.5f + 0.5f; x[50] = r.normal.z * 0.5f + 0.5f;
    x[51] = r.roughness;
    x[52] = r.albedo.x; x[53] = r.albedo.y; x[54] = r.albedo.z;
    x[55] = r.metalness;
    x[56] = 1.f;
#pragma unroll
    for (int i = 57; i < 64; ++i) x[i] = 0.f;
}

// Records are stored SoA-free as 16 floats: pos(3) wo(3) normal(3) roughness metalness albedo(3) pad(2).
constexpr int RECORD_FLOATS = 16;
__device__ __forceinline__ Record load_record(const float4* __restrict__ rec, uint32_t i) {
    const float4 a = rec[4 * i], b = rec[4 * i + 1], c = rec[4 * i + 2], d = rec[4 * i + 3];
    Record r;
    r.pos = make_float3(a.x, a.y, a.z);
    r.wo = make_float3(a.w, b.x, b.y);
    r.normal = make_float3(b.z, b.w, c.x);
    r.roughness = c.y; r.metalness = c.z;
    r.albedo = make_float3(c.w, d.x, d.y);
    return r;
}

// ---------------------------------------------------------------- shared building blocks
// Copy one row-major [rows][64] BF16 weight matrix into a core-matrix tile.
__device__ __forceinline__ void stage_weights(const __nv_bfloat16* __restrict__ w, uint32_t rows, unsigned char* tile) {
    for (uint32_t k = threadIdx.x; k < rows * 8u; k += blockDim.x) {
        const uint32_t row = k >> 3, chunk = k & 7u;
        *reinterpret_cast<uint4*>(tile + tile_offset(row, chunk)) = __ldg(reinterpret_cast<const uint4*>(w + row * WIDTH) + chunk);
    }
}
// Store this thread's 64 floats as row `row` of a tile (BF16).
__device__ __forceinline__ void store_row(unsigned char* tile, uint32_t row, const float* v) {
#pragma unroll
    for (int c = 0; c < 8; ++c) *reinterpret_cast<uint4*>(tile + tile_offset(row, c)) = pack8(v + 8 * c);
}
__device__ __forceinline__ void load_row(const unsigned char* tile, uint32_t row, float* v) {
#pragma unroll
    for (int c = 0; c < 8; ++c) unpack8(*reinterpret_cast<const uint4*>(tile + tile_offset(row, c)), v + 8 * c);
}

// D[128 x n] = A[128 x k] * B[n x k]^T with A and B K-major tiles (forward layers, and
// delta * W with W read MN-major).  Issued by the calling (single) thread.
__device__ __forceinline__ void mma_rows(uint32_t d_tmem, uint32_t a_saddr, uint32_t b_saddr, uint32_t n, uint32_t k, bool b_mn) {
    const uint32_t idesc = instr_desc(128, n, 0, b_mn ? 1u : 0u);
    for (uint32_t s = 0; s < k / 16; ++s) {
        const uint64_t a = smem_desc(a_saddr + 256u * s, 128u, 1024u);
        const uint64_t b = b_mn ? smem_desc(b_saddr + 2048u * s, 1024u, 128u) : smem_desc(b_saddr + 256u * s, 128u, 1024u);
        mma_bf16(d_tmem, a, b, idesc, s > 0 ? 1u : 0u);
    }
}
// D[64 x 64] = A^T B over the 128 tile rows, A and B read MN-major (weight gradients:
// A = delta tile, B = layer-input tile).  D uses the M = 64 TMEM layout.
__device__ __forceinline__ void mma_wgrad(uint32_t d_tmem, uint32_t a_saddr, uint32_t b_saddr) {
    const uint32_t idesc = instr_desc(64, 64, 1, 1);
    for (uint32_t s = 0; s < TILE / 16; ++s) {
        const uint64_t a = smem_desc(a_saddr + 2048u * s, 1024u, 128u);
        const uint64_t b = smem_desc(b_saddr + 2048u * s, 1024u, 128u);
        mma_bf16(d_tmem, a, b, idesc, s > 0 ? 1u : 0u);
    }
}

}  // namespace nrc
}  // namespace vkb

namespace vkb {
namespace nrc {

// ---------------------------------------------------------------- kernels
// Shared memory of the forward kernel: W0..W3, W4, one activation tile, barrier, TMEM slot.
constexpr uint32_t FWD_W4 = 4u * W_BYTES;                     // 32768
constexpr uint32_t FWD_TILE = 36864u;                         // 1 KiB aligned
constexpr uint32_t FWD_BAR = FWD_TILE + TILE_BYTES;           // 53248
constexpr uint32_t FWD_SMEM = FWD_BAR + 16u;
// Training kernel: weights, the five layer-input tiles (x, h1..h4), the delta tile.
constexpr uint32_t TRN_ACT = 36864u;
constexpr uint32_t TRN_DELTA = TRN_ACT + 5u * TILE_BYTES;     // 118784
constexpr uint32_t TRN_BAR = TRN_DELTA + TILE_BYTES;          // 135168
constexpr uint32_t TRN_SMEM = TRN_BAR + 32u;           // barrier, TMEM slot, 4 per-warp loss sums
constexpr uint32_t TMEM_COLS_FWD = 64, TMEM_COLS_TRN = 128;
// Fixed-point scale of the hash-table gradient accumulators (int64 atomics keep the
// sum independent of the order in which threads add).
constexpr double HASH_GRAD_SCALE = 1099511627776.0;   // 2^40

__device__ __forceinline__ uint32_t layer_rows(int l) { return l == LAYERS - 1 ? OUT_ROWS : WIDTH; }
__device__ __forceinline__ const __nv_bfloat16* layer_weights(const __nv_bfloat16* w, int l) { return w + size_t(l) * WIDTH * WIDTH; }

// Error bits written to *err: 1 = a tensor-core wait ran out.
__device__ __forceinline__ bool all_ok(bool ok) { return __syncthreads_and(ok ? 1 : 0) != 0; }

// Input/output policies of the forward kernel.
struct DebugIO {         // records in, encoded inputs and raw outputs out
    static constexpr bool kDebug = true;
    const float4* rec; uint32_t n; float* x_out; float* y_out;
};
struct QueryIO {         // cache queries of a wave: rad[slot] += throughput * max(y, 0)
    static constexpr bool kDebug = false;
    const float4* rec; const uint32_t* count; uint32_t cap; const uint32_t* slot; const float4* thr; float4* rad;
    unsigned long long* queries;   // += queries answered
};

// Fused query kernel: 128 rows per tile, persistent over tiles.  blockDim.x == TILE.
template <class IO>
__global__ void __launch_bounds__(TILE) k_nrc_forward(IO io, const __nv_bfloat16* __restrict__ w, const __half* __restrict__ table,
                                                      uint32_t* err) {
    extern __shared__ __align__(1024) unsigned char smem[];
    unsigned char* act = smem + FWD_TILE;
    const uint32_t mbar = smem_u32(smem + FWD_BAR), tslot = smem_u32(smem + FWD_BAR + 8);
    const uint32_t warp = threadIdx.x >> 5, row = threadIdx.x;
    if (warp == 0) tmem_alloc(tslot, TMEM_COLS_FWD);
    if (threadIdx.x == 0) mbar_init(mbar, 1);
    for (int l = 0; l < LAYERS; ++l) stage_weights(layer_weights(w, l), layer_rows(l), smem + l * W_BYTES);
    tc_fence_before();
    __syncthreads();
    tc_fence_after();
    const uint32_t tmem = *reinterpret_cast<volatile uint32_t*>(smem + FWD_BAR + 8);
    const uint32_t lane_addr = tmem + ((warp * 32u) << 16);
    uint32_t n;
    if constexpr (IO::kDebug) n = io.n; else n = min(*io.count, io.cap);
    if constexpr (!IO::kDebug) {
        if (blockIdx.x == 0 && threadIdx.x == 0) atomicAdd(io.queries, (unsigned long long)n);
    }
    const uint32_t tiles = (n + TILE - 1) / TILE;
    uint32_t phase = 0;
    bool ok = true;
    for (uint32_t t = blockIdx.x; t < tiles && ok; t += gridDim.x) {
        const uint32_t i = t * TILE + row;
        const bool valid = i < n;
        float v[64];
        if (valid) encode(load_record(io.rec, i), table, v);
        else for (int k = 0; k < 64; ++k) v[k] = 0.f;
        if constexpr (IO::kDebug) {
            if (valid) for (int k = 0; k < 64; ++k) io.x_out[size_t(i) * 64 + k] = __bfloat162float(__float2bfloat16_rn(v[k]));
        }
        store_row(act, row, v);
        fence_async_smem();
        tc_fence_before();
        __syncthreads();
        tc_fence_after();
        for (int l = 0; l < LAYERS && ok; ++l) {
            if (threadIdx.x == 0) {
                mma_rows(tmem, smem_u32(act), smem_u32(smem + l * W_BYTES), layer_rows(l), WIDTH, false);
                mma_commit(mbar);
            }
            ok = all_ok(mbar_wait(mbar, phase));
            phase ^= 1u;
            if (!ok) break;
            tc_fence_after();
            if (l < LAYERS - 1) {
#pragma unroll
                for (int q = 0; q < 4; ++q) {
                    tmem_ld16(lane_addr + 16u * q, *reinterpret_cast<float(*)[16]>(v + 16 * q));
                }
#pragma unroll
                for (int k = 0; k < 64; ++k) v[k] = fmaxf(v[k], 0.f);
                store_row(act, row, v);
                fence_async_smem();
            } else {
                float y[16];
                tmem_ld16(lane_addr, y);
                if (valid) {
                    if constexpr (IO::kDebug) {
                        io.y_out[3 * size_t(i)] = y[0]; io.y_out[3 * size_t(i) + 1] = y[1]; io.y_out[3 * size_t(i) + 2] = y[2];
                    } else {
                        const uint32_t s = io.slot[i];
                        const float4 th = io.thr[s];
                        float4 r = io.rad[s];
                        r.x += th.x * fmaxf(y[0], 0.f); r.y += th.y * fmaxf(y[1], 0.f); r.z += th.z * fmaxf(y[2], 0.f);
                        io.rad[s] = r;
                    }
                }
            }
            tc_fence_before();
            __syncthreads();
            tc_fence_after();
        }
    }
    if (!ok && threadIdx.x == 0) atomicOr(err, 1u);
    __syncthreads();
    if (warp == 0) tmem_dealloc(tmem, TMEM_COLS_FWD);
}

// Training: one tile of 128 records per CTA.  Forward with every layer input kept in
// shared memory, relative-L2 loss gradient, backward through the layers on the tensor
// cores (delta * W row GEMMs and delta^T * input weight-gradient GEMMs), per-tile
// weight-gradient partials (summed in tile order by the optimizer: deterministic), and
// the hash-table gradient scattered as fixed-point int64 atomics.  blockDim.x == TILE.
// Rows i < n of this step are records offset + i * stride (interleaved minibatches).
__global__ void __launch_bounds__(TILE) k_nrc_train(const float4* __restrict__ rec, const float* __restrict__ target, uint32_t n,
                                                   uint32_t offset, uint32_t stride,
                                                   float inv_count, const __nv_bfloat16* __restrict__ w, const __half* __restrict__ table,
                                                   float* __restrict__ wgrad_partial, long long* __restrict__ hash_grad,
                                                   float* __restrict__ loss_partial, uint32_t* err) {
    extern __shared__ __align__(1024) unsigned char smem[];
    unsigned char* tiles = smem + TRN_ACT;
    unsigned char* delta = smem + TRN_DELTA;
    const uint32_t mbar = smem_u32(smem + TRN_BAR), tslot = smem_u32(smem + TRN_BAR + 8);
    const uint32_t warp = threadIdx.x >> 5, lane = threadIdx.x & 31u, row = threadIdx.x;
    if (warp == 0) tmem_alloc(tslot, TMEM_COLS_TRN);
    if (threadIdx.x == 0) mbar_init(mbar, 1);
    for (int l = 0; l < LAYERS; ++l) stage_weights(layer_weights(w, l), layer_rows(l), smem + l * W_BYTES);
    const uint32_t i = blockIdx.x * TILE + row;
    const size_t ri = size_t(offset) + size_t(i) * stride;
    const bool valid = i < n;
    Record r{};
    float v[64];
    if (valid) { r = load_record(rec, uint32_t(ri)); encode(r, table, v); }
    else for (int k = 0; k < 64; ++k) v[k] = 0.f;
    store_row(tiles, row, v);
    fence_async_smem();
    tc_fence_before();
    __syncthreads();
    tc_fence_after();
    const uint32_t tmem = *reinterpret_cast<volatile uint32_t*>(smem + TRN_BAR + 8);
    const uint32_t lane_addr = tmem + ((warp * 32u) << 16);
    uint32_t phase = 0;
    bool ok = true;
    float y[16];
    // Forward.
    for (int l = 0; l < LAYERS && ok; ++l) {
        if (threadIdx.x == 0) {
            mma_rows(tmem, smem_u32(tiles + l * TILE_BYTES), smem_u32(smem + l * W_BYTES), layer_rows(l), WIDTH, false);
            mma_commit(mbar);
        }
        ok = all_ok(mbar_wait(mbar, phase));
        phase ^= 1u;
        if (!ok) break;
        tc_fence_after();
        if (l < LAYERS - 1) {
#pragma unroll
            for (int q = 0; q < 4; ++q) tmem_ld16(lane_addr + 16u * q, *reinterpret_cast<float(*)[16]>(v + 16 * q));
#pragma unroll
            for (int k = 0; k < 64; ++k) v[k] = fmaxf(v[k], 0.f);
            store_row(tiles + (l + 1) * TILE_BYTES, row, v);
            fence_async_smem();
        } else {
            tmem_ld16(lane_addr, y);
        }
        tc_fence_before();
        __syncthreads();
        tc_fence_after();
    }
    // Loss and its gradient with respect to y (columns 3..63 zero).
    float g[64];
#pragma unroll
    for (int k = 0; k < 64; ++k) g[k] = 0.f;
    float loss = 0.f;
    if (valid && ok) {
        for (int c = 0; c < 3; ++c) {
            const float t = target[3 * ri + c], d = y[c] - t, den = y[c] * y[c] + LOSS_EPS;
            loss += d * d / den;
            g[c] = 2.f * d / den * inv_count;
        }
    }
    for (int off = 16; off > 0; off >>= 1) loss += __shfl_xor_sync(0xffffffffu, loss, off);
    float* wloss = reinterpret_cast<float*>(smem + TRN_BAR + 16);
    if (lane == 0) wloss[warp] = loss;
    store_row(delta, row, g);
    fence_async_smem();
    tc_fence_before();
    __syncthreads();
    tc_fence_after();
    if (threadIdx.x == 0) loss_partial[blockIdx.x] = (wloss[0] + wloss[1]) + (wloss[2] + wloss[3]);
    // Backward: layer l has input tile l and output delta in `delta`.
    float* part = wgrad_partial + size_t(blockIdx.x) * MLP_PARAMS;
    for (int l = LAYERS - 1; l >= 0 && ok; --l) {
        if (threadIdx.x == 0) {
            mma_wgrad(tmem + 64u, smem_u32(delta), smem_u32(tiles + l * TILE_BYTES));
            mma_rows(tmem, smem_u32(delta), smem_u32(smem + l * W_BYTES), WIDTH, layer_rows(l), true);
            mma_commit(mbar);
        }
        ok = all_ok(mbar_wait(mbar, phase));
        phase ^= 1u;
        if (!ok) break;
        tc_fence_after();
        // Weight gradient (M = 64 layout: row o in lane (o % 16) + 32 (o / 16)).
        {
            float d[64];
#pragma unroll
            for (int q = 0; q < 4; ++q) tmem_ld16(lane_addr + 64u + 16u * q, *reinterpret_cast<float(*)[16]>(d + 16 * q));
            const uint32_t o = warp * 16u + lane;
            if (lane < 16 && o < layer_rows(l)) {
                float4* dst = reinterpret_cast<float4*>(part + size_t(l) * WIDTH * WIDTH + size_t(o) * WIDTH);
#pragma unroll
                for (int q = 0; q < 16; ++q) dst[q] = make_float4(d[4 * q], d[4 * q + 1], d[4 * q + 2], d[4 * q + 3]);
            }
        }
        // Input gradient: delta of the previous layer (relu mask from its output), or dx.
#pragma unroll
        for (int q = 0; q < 4; ++q) tmem_ld16(lane_addr + 16u * q, *reinterpret_cast<float(*)[16]>(v + 16 * q));
        if (l > 0) {
            float h[64];
            load_row(tiles + l * TILE_BYTES, row, h);
#pragma unroll
            for (int k = 0; k < 64; ++k) v[k] = h[k] > 0.f ? v[k] : 0.f;
            store_row(delta, row, v);
            fence_async_smem();
        }
        tc_fence_before();
        __syncthreads();
        tc_fence_after();
    }
    // Hash-table gradient: dL/dfeature scattered to the 8 corners of each level.
    if (valid && ok) {
        for (int l = 0; l < HASH_LEVELS; ++l) {
            const float s = level_scale(l);
            const uint32_t res = uint32_t(s);
            const float px = fminf(fmaxf(r.pos.x, 0.f), 1.f) * s, py = fminf(fmaxf(r.pos.y, 0.f), 1.f) * s, pz = fminf(fmaxf(r.pos.z, 0.f), 1.f) * s;
            const uint32_t cx = min(uint32_t(px), res - 1u), cy = min(uint32_t(py), res - 1u), cz = min(uint32_t(pz), res - 1u);
            const float fx = px - float(cx), fy = py - float(cy), fz = pz - float(cz);
            long long* lvl = hash_grad + size_t(l) * HASH_T * HASH_FEATURES;
            for (int c = 0; c < 8; ++c) {
                const uint32_t dx = c & 1u, dy = (c >> 1) & 1u, dz = (c >> 2) & 1u;
                const float wgt = (dx ? fx : 1.f - fx) * (dy ? fy : 1.f - fy) * (dz ? fz : 1.f - fz);
                const uint32_t idx = grid_index(cx + dx, cy + dy, cz + dz, res);
                // |gradient| is clamped to 2^20 so the scaled value stays inside int64.
                const double q0 = fmin(fmax(double(wgt * v[2 * l]), -1048576.0), 1048576.0);
                const double q1 = fmin(fmax(double(wgt * v[2 * l + 1]), -1048576.0), 1048576.0);
                const long long g0 = llrint(q0 * HASH_GRAD_SCALE), g1 = llrint(q1 * HASH_GRAD_SCALE);
                if (g0) atomicAdd(reinterpret_cast<unsigned long long*>(lvl + 2 * idx), static_cast<unsigned long long>(g0));
                if (g1) atomicAdd(reinterpret_cast<unsigned long long*>(lvl + 2 * idx + 1), static_cast<unsigned long long>(g1));
            }
        }
    }
    if (!ok && threadIdx.x == 0) atomicOr(err, 1u);
    __syncthreads();
    if (warp == 0) tmem_dealloc(tmem, TMEM_COLS_TRN);
}

// Training set of a recording wave, in position order (indices from the flags): the
// record itself and its target, the outgoing radiance = (the path's final radiance - its
// radiance at the vertex) / its throughput at the vertex, per channel.
__global__ void k_nrc_gather(const uint32_t* __restrict__ count, uint32_t cap, const uint32_t* __restrict__ index, uint32_t vmax,
                             const float4* __restrict__ rec, const float4* __restrict__ aux, const float4* __restrict__ rad,
                             float4* __restrict__ out_rec, float* __restrict__ targets) {
    const uint32_t n = min(*count, cap);
    for (uint32_t i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x) {
        const uint32_t q = index[i];
        for (int k = 0; k < 4; ++k) out_rec[4 * size_t(i) + k] = rec[4 * size_t(q) + k];
        const float4 t = aux[2 * size_t(q)], r0 = aux[2 * size_t(q) + 1], rf = rad[q / vmax];
        const float tt[3] = {t.x, t.y, t.z}, d[3] = {rf.x - r0.x, rf.y - r0.y, rf.z - r0.z};
        for (int c = 0; c < 3; ++c) {
            float v = tt[c] > 0.f ? d[c] / tt[c] : 0.f;
            targets[3 * size_t(i) + c] = isfinite(v) ? fminf(fmaxf(v, 0.f), 1e4f) : 0.f;
        }
    }
}

// Adam over the MLP: gradient = sum of the tile partials in tile order; FP32 master
// weights, BF16 copy for the kernels.  Rows 3..15 of the output layer stay zero.
struct AdamParams { float lr, beta1, beta2, eps, bc1, bc2; };
__global__ void k_nrc_adam_mlp(uint32_t tiles, const float* __restrict__ partial, float* __restrict__ master, float* __restrict__ m1,
                               float* __restrict__ m2, __nv_bfloat16* __restrict__ w, AdamParams a, float* __restrict__ grad_out) {
    for (uint32_t p = blockIdx.x * blockDim.x + threadIdx.x; p < MLP_PARAMS; p += gridDim.x * blockDim.x) {
        const bool fixed_zero = p >= 4u * WIDTH * WIDTH && (p - 4u * WIDTH * WIDTH) / WIDTH >= 3u;
        float g = 0.f;
        for (uint32_t t = 0; t < tiles; ++t) g += partial[size_t(t) * MLP_PARAMS + p];
        if (fixed_zero) g = 0.f;
        if (grad_out) grad_out[p] = g;
        if (a.lr == 0.f || fixed_zero) continue;
        const float mm = a.beta1 * m1[p] + (1.f - a.beta1) * g, vv = a.beta2 * m2[p] + (1.f - a.beta2) * g * g;
        m1[p] = mm; m2[p] = vv;
        const float x = master[p] - a.lr * (mm / a.bc1) / (sqrtf(vv / a.bc2) + a.eps);
        master[p] = x;
        w[p] = __float2bfloat16_rn(x);
    }
}
// Adam over the hash table from the fixed-point gradients (which it clears).
__global__ void k_nrc_adam_hash(uint64_t count, long long* __restrict__ grad, float* __restrict__ master, float* __restrict__ m1,
                                float* __restrict__ m2, __half* __restrict__ table, AdamParams a, float* __restrict__ grad_out) {
    for (uint64_t p = blockIdx.x * uint64_t(blockDim.x) + threadIdx.x; p < count; p += uint64_t(gridDim.x) * blockDim.x) {
        const long long q = grad[p];
        const float g = float(double(q) / HASH_GRAD_SCALE);
        if (grad_out) grad_out[p] = g;
        if (q) grad[p] = 0;
        if (a.lr == 0.f) continue;
        const float mm = a.beta1 * m1[p] + (1.f - a.beta1) * g, vv = a.beta2 * m2[p] + (1.f - a.beta2) * g * g;
        m1[p] = mm; m2[p] = vv;
        const float x = master[p] - a.lr * (mm / a.bc1) / (sqrtf(vv / a.bc2) + a.eps);
        master[p] = x;
        table[p] = __float2half_rn(x);
    }
}

}  // namespace nrc
}  // namespace vkb
