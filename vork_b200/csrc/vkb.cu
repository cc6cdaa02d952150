// Host runtime and C ABI of the B200 render backend (include/vkb.h).
//
// One vkb_ctx per device: a CUDA stream, the BRDF atlas baked on the device
// (Renderer::new + environment bake, crates/vork-render/src/lib.rs:726,
// src/environment.rs:312-323) and the film table (src/sampling.rs:149-178).
// One vkb_scene per installed scene: meshes, per-mesh BLAS, instance TLAS, material
// and light tables (Renderer::install, lib.rs:1322-1470; rt.rs:1098-1385), plus the
// wavefront buffers its renders reuse.
#include <cuda_runtime.h>
#include <cub/device/device_radix_sort.cuh>
#include <cub/device/device_scan.cuh>
#include <cub/device/device_select.cuh>
#include <thrust/iterator/counting_iterator.h>

#include <algorithm>
#include <chrono>
#include <deque>
#include <map>
#include <memory>
#include <cmath>
#include <cstdio>
#include <cstring>
#include <mutex>
#include <thread>
#include <future>
#include <string>
#include <vector>

#include "vkb_kernels.cuh"
#include "vkb_sah.h"
#include "vkb_wide8.h"
#include "vkb_nrc.cuh"
#include "vkb_display.cuh"

using namespace vkb;

namespace {

thread_local std::string g_error;

struct CudaError {
    cudaError_t code;
    const char* what;
};
#define VKB_CUDA(x)                                                    \
    do {                                                               \
        cudaError_t e_ = (x);                                          \
        if (e_ != cudaSuccess) throw CudaError{e_, #x};                \
    } while (0)

struct ArgError { std::string msg; };
struct Unsupported { std::string msg; };
struct InternalError { std::string msg; };
struct DeviceTimeout { std::string msg; };

template <class T> struct DBuf {
    T* p = nullptr;
    size_t n = 0;
    void alloc(size_t count) {
        if (count <= n && p) return;
        release();
        if (count == 0) return;
        VKB_CUDA(cudaMalloc(&p, count * sizeof(T)));
        n = count;
    }
    void release() { if (p) cudaFree(p); p = nullptr; n = 0; }
    void upload(const T* src, size_t count, cudaStream_t s) { alloc(count); if (count) VKB_CUDA(cudaMemcpyAsync(p, src, count * sizeof(T), cudaMemcpyHostToDevice, s)); }
};

int grid_for(uint32_t n, int block, int sm_count, int per_sm = 8) {
    int need = int((uint64_t(n) + block - 1) / block);
    return std::max(1, std::min(need, sm_count * per_sm));
}

// Film table: inverse CDF of Cycles' 1.5 px Blackman-Harris kernel, bisected in f64
// (crates/vork-render/src/sampling.rs:151-178).
std::vector<float> film_table() {
    auto cdf = [](double x) {
        const double pi = 3.141592653589793;
        double t = pi * x / 1.5;
        return 0.5 + (0.35875 * x + 1.5 / pi * (0.48829 * std::sin(t) + 0.14128 * std::sin(2. * t) / 2. + 0.01168 * std::sin(3. * t) / 3.)) / (3. * 0.35875);
    };
    std::vector<float> t(FILTER_INTERVALS + 1);
    for (uint32_t i = 0; i <= FILTER_INTERVALS; ++i) {
        if (i == 0) { t[i] = -1.5f; continue; }
        if (i == FILTER_INTERVALS) { t[i] = 1.5f; continue; }
        double u = double(i) / FILTER_INTERVALS, lo = -1.5, hi = 1.5;
        for (int k = 0; k < 48; ++k) { double mid = (lo + hi) * 0.5; if (cdf(mid) < u) lo = mid; else hi = mid; }
        t[i] = float((lo + hi) * 0.5);
    }
    return t;
}

// Light tree over analytic sources (crates/vork-render/src/lights/tree.rs:43-176).
std::vector<LightTreeNode> light_tree(const vkb_light* lights, uint32_t n) {
    struct Src { float lo[3], hi[3]; double power; bool inf; };
    std::vector<Src> src(n);
    const float lumc[3] = {0.2126f, 0.7152f, 0.0722f};
    for (uint32_t i = 0; i < n; ++i) {
        const vkb_light& l = lights[i];
        uint32_t kind = uint32_t(l.position[3]);
        for (int c = 0; c < 3; ++c) {
            float r = kind == 3 ? (std::fabs(l.emitter_u[c]) + std::fabs(l.emitter_v[c])) * 0.5f : (kind == 0 ? 0.f : l.params[1]);
            src[i].lo[c] = l.position[c] - r; src[i].hi[c] = l.position[c] + r;
        }
        double p = 0;
        for (int c = 0; c < 3; ++c) p += double(l.radiance[c]) * double(lumc[c]);
        src[i].power = std::max(p, 0.);
        src[i].inf = kind == 0;
    }
    double scale = 2.2250738585072014e-308;
    for (auto& s : src) scale = std::max(scale, s.power);
    std::vector<LightTreeNode> nodes;
    std::vector<uint32_t> ids(n);
    for (uint32_t i = 0; i < n; ++i) ids[i] = i;
    struct Builder {
        std::vector<Src>& src; std::vector<LightTreeNode>& nodes; double scale;
        uint32_t go(uint32_t* id, uint32_t count, uint32_t parent) {
            uint32_t index = uint32_t(nodes.size());
            nodes.push_back(LightTreeNode{});
            float lo[3] = {INFINITY, INFINITY, INFINITY}, hi[3] = {-INFINITY, -INFINITY, -INFINITY};
            double power = 0; bool inf = false;
            for (uint32_t k = 0; k < count; ++k) {
                const Src& s = src[id[k]];
                for (int c = 0; c < 3; ++c) { lo[c] = std::min(lo[c], s.lo[c]); hi[c] = std::max(hi[c], s.hi[c]); }
                power += s.power / scale; inf |= s.inf;
            }
            float pf = float(power);
            if (pf < 1.17549435e-38f) pf = 0.f;
            LightTreeNode nd{};
            nd.lower_power = make_float4(lo[0], lo[1], lo[2], pf);
            nd.upper_infinite = make_float4(hi[0], hi[1], hi[2], inf ? 1.f : 0.f);
            nd.links = make_uint4(0xffffffffu, 0xffffffffu, parent, count);
            if (count == 1) {
                nd.source = make_uint4(0u, id[0], id[0], 0u);
            } else {
                double ext[3];
                for (int c = 0; c < 3; ++c) ext[c] = double(hi[c]) - double(lo[c]);
                int axis = (ext[0] >= ext[1] && ext[0] >= ext[2]) ? 0 : (ext[1] >= ext[2] ? 1 : 2);
                uint32_t finite = 0;
                for (uint32_t k = 0; k < count; ++k) finite += src[id[k]].inf ? 0u : 1u;
                uint32_t split;
                if (finite > 0 && finite < count) {
                    std::sort(id, id + count, [&](uint32_t a, uint32_t b) { return std::make_pair(src[a].inf, a) < std::make_pair(src[b].inf, b); });
                    split = finite;
                } else {
                    split = count / 2;
                    std::nth_element(id, id + split, id + count, [&](uint32_t a, uint32_t b) {
                        double ca = double(src[a].lo[axis]) + double(src[a].hi[axis]), cb = double(src[b].lo[axis]) + double(src[b].hi[axis]);
                        return ca < cb || (ca == cb && a < b);
                    });
                }
                uint32_t l = go(id, split, index);
                uint32_t r = go(id + split, count - split, index);
                nd.links.x = l; nd.links.y = r;
            }
            nodes[index] = nd;
            return index;
        }
    } b{src, nodes, scale};
    if (n) b.go(ids.data(), n, 0xffffffffu);
    return nodes;
}

// Bounding sphere of a mesh about its box centre (c = (lo + hi) / 2 in fp32): the radius
// is the largest vertex distance, in f64, rounded up to fp32; radius -1 for no vertices.
void mesh_sphere(const float* pos, uint32_t nv, const float lo[3], const float hi[3], float out[4]) {
    if (nv == 0) { out[0] = out[1] = out[2] = 0.f; out[3] = -1.f; return; }
    float c[3];
    for (int a = 0; a < 3; ++a) c[a] = 0.5f * (lo[a] + hi[a]);
    double r2 = 0.0;
    for (uint32_t i = 0; i < nv; ++i) {
        double dx = double(pos[3 * i]) - c[0], dy = double(pos[3 * i + 1]) - c[1], dz = double(pos[3 * i + 2]) - c[2];
        r2 = std::max(r2, dx * dx + dy * dy + dz * dz);
    }
    out[0] = c[0]; out[1] = c[1]; out[2] = c[2];
    out[3] = std::nextafter(float(std::sqrt(r2)), INFINITY);
}

// 4-wide BLAS from the binary SAH tree (root 0): the 4-wide children of one node are
// allocated together, depth first.
std::vector<Bvh4Node> collapse_blas(const std::vector<BvhNode>& n2) {
    std::vector<Bvh4Node> out(1);
    std::vector<std::pair<int, int>> todo{{0, 0}};  // (binary node, 4-wide node)
    while (!todo.empty()) {
        auto [b, q] = todo.back();
        todo.pop_back();
        Bvh4Node node = collapse_node(n2.data(), n2[b]);
        int* child = reinterpret_cast<int*>(&node.child);
        for (int k = 0; k < 4; ++k) {
            if (child[k] < 0) continue;
            const int idx = int(out.size());
            out.emplace_back();
            todo.push_back({child[k], idx});
            child[k] = idx;
        }
        out[q] = node;
    }
    return out;
}

// Scratch of one LBVH build, reused across builds.
struct LbvhScratch {
    DBuf<uint32_t> codes, codes_sorted, ids, ids_sorted, leaf_parent, node_parent, counters, bounds;
    DBuf<unsigned char> cub_temp;
    void reserve(size_t n, cudaStream_t s) {
        codes.alloc(n); codes_sorted.alloc(n); ids.alloc(n); ids_sorted.alloc(n);
        leaf_parent.alloc(n); node_parent.alloc(std::max<size_t>(n, 1)); counters.alloc(std::max<size_t>(n, 1)); bounds.alloc(6);
        size_t bytes = 0;
        cub::DeviceRadixSort::SortPairs(nullptr, bytes, codes.p, codes_sorted.p, ids.p, ids_sorted.p, int(n), 0, 31, s);
        cub_temp.alloc(std::max<size_t>(bytes, 1));
    }
};

// Morton codes of n boxes (sc.codes, input order) and the sorted order (sc.ids_sorted).
void morton_sort(uint32_t n, const float4* lo, const float4* hi, LbvhScratch& sc, cudaStream_t s, int sms, uint64_t& launches) {
    launches += 3;
    sc.reserve(n, s);
    VKB_CUDA(cudaMemsetAsync(sc.bounds.p, 0xff, 3 * sizeof(uint32_t), s));
    VKB_CUDA(cudaMemsetAsync(sc.bounds.p + 3, 0x00, 3 * sizeof(uint32_t), s));
    k_centroid_box<<<grid_for(n, 256, sms), 256, 0, s>>>(n, lo, hi, sc.bounds.p);
    k_morton<<<grid_for(n, 256, sms), 256, 0, s>>>(n, lo, hi, sc.bounds.p, sc.codes.p, sc.ids.p, true);
    size_t bytes = sc.cub_temp.n;
    VKB_CUDA(cub::DeviceRadixSort::SortPairs(sc.cub_temp.p, bytes, sc.codes.p, sc.codes_sorted.p, sc.ids.p, sc.ids_sorted.p, int(n), 0, 31, s));
}

// Build one LBVH over n boxes into nodes (n-1 internal nodes, or 1 for n == 1).
// On return scratch.ids_sorted holds the leaf order and scratch.codes the codes in input order.
void build_lbvh(uint32_t n, const float4* lo, const float4* hi, BvhNode* nodes, LbvhScratch& sc, cudaStream_t s, int sms, uint64_t& launches) {
    if (n == 0) return;
    morton_sort(n, lo, hi, sc, s, sms, launches);
    launches += n == 1 ? 0 : 1;
    if (n == 1) {
        k_single_leaf<<<1, 1, 0, s>>>(lo, hi, nodes);
        return;
    }
    k_karras<<<grid_for(n - 1, 256, sms), 256, 0, s>>>(int(n), sc.codes_sorted.p, nodes, sc.leaf_parent.p, sc.node_parent.p, sc.counters.p);
    k_refit<<<grid_for(n, 256, sms), 256, 0, s>>>(int(n), sc.ids_sorted.p, lo, hi, nodes, sc.leaf_parent.p, sc.node_parent.p, sc.counters.p);
    VKB_CUDA(cudaGetLastError());
}

// Cluster arrays of the PLOC builder (double-buffered) and its prefix-sum scratch.
struct PlocScratch {
    DBuf<float4> clo, chi, clo2, chi2;
    DBuf<uint32_t> nn, counts;
    DBuf<unsigned long long> flags, offs;
    DBuf<unsigned char> cub_temp;
    void reserve(size_t n, cudaStream_t s) {
        clo.alloc(n); chi.alloc(n); clo2.alloc(n); chi2.alloc(n); nn.alloc(n); counts.alloc(2); flags.alloc(n); offs.alloc(n);
        size_t bytes = 0;
        cub::DeviceScan::ExclusiveSum(nullptr, bytes, flags.p, offs.p, int(n), s);
        cub_temp.alloc(std::max<size_t>(bytes, 1));
    }
};

// Build a PLOC tree over n boxes (n >= 2) into nodes[0, n-1), root 0, leaves ~k in
// Morton order (sc.ids_sorted, from the same sort as the LBVH), with parent links and
// zeroed counters for refits.  One host round trip per pass (cluster count).
void build_ploc(uint32_t n, const float4* lo, const float4* hi, BvhNode* nodes, uint32_t* leaf_parent, uint32_t* node_parent,
                uint32_t* counters, LbvhScratch& sc, PlocScratch& pc, cudaStream_t s, int sms, uint64_t& launches) {
    pc.reserve(n, s);
    k_ploc_init<<<grid_for(n, 256, sms), 256, 0, s>>>(n, sc.ids_sorted.p, lo, hi, pc.clo.p, pc.chi.p);
    launches += 1;
    uint32_t c = n, next_free = n - 1;
    float4 *a_lo = pc.clo.p, *a_hi = pc.chi.p, *b_lo = pc.clo2.p, *b_hi = pc.chi2.p;
    for (uint32_t pass = 0; c > 1; ++pass) {
        if (pass >= n) throw InternalError{"PLOC made no progress"};
        k_ploc_nn<<<(c + PLOC_BLOCK - 1) / PLOC_BLOCK, PLOC_BLOCK, 0, s>>>(c, a_lo, a_hi, pc.nn.p);
        k_ploc_flags<<<grid_for(c, 256, sms), 256, 0, s>>>(c, pc.nn.p, pc.flags.p);
        size_t bytes = pc.cub_temp.n;
        VKB_CUDA(cub::DeviceScan::ExclusiveSum(pc.cub_temp.p, bytes, pc.flags.p, pc.offs.p, int(c), s));
        k_ploc_merge<<<grid_for(c, 256, sms), 256, 0, s>>>(c, pc.nn.p, pc.offs.p, a_lo, a_hi, next_free, nodes, leaf_parent, node_parent,
                                                           counters, b_lo, b_hi, pc.counts.p);
        launches += 4;
        uint32_t counts[2] = {0u, 0u};
        VKB_CUDA(cudaMemcpyAsync(counts, pc.counts.p, sizeof(counts), cudaMemcpyDeviceToHost, s));
        VKB_CUDA(cudaStreamSynchronize(s));
        if (counts[1] == 0 || counts[1] > next_free || counts[0] != c - counts[1]) throw InternalError{"PLOC pass merged no pair"};
        c = counts[0];
        next_free -= counts[1];
        std::swap(a_lo, b_lo); std::swap(a_hi, b_hi);
    }
    if (next_free != 0) throw InternalError{"PLOC left unused nodes"};
}

}  // namespace

// Device pointers of one wavefront: queues and path state for `capacity` path slots,
// the counters, and the job table of `job_capacity` entries.
struct WaveBuffers {
    size_t capacity = 0;
    uint32_t job_capacity = 0;
    float4 *ray_o0 = nullptr, *ray_d0 = nullptr, *ray_o1 = nullptr, *ray_d1 = nullptr, *hit = nullptr, *thr = nullptr, *rad = nullptr;
    float4 *sa_o = nullptr, *sa_d = nullptr, *sa_c = nullptr, *sb_o = nullptr, *sb_d = nullptr, *sb_c = nullptr;
    uint32_t *hit_inst = nullptr, *slot_job = nullptr, *counters = nullptr, *err = nullptr;
    uint2* rng = nullptr;
    unsigned long long* work = nullptr;
    Job* jobs = nullptr;
    float4* guide = nullptr;   // guide renders: 2 float4 per path slot
    // Waves with an image environment or emissive meshes: the environment and mesh shadow
    // rays of every slot and its previous vertex + BSDF pdf.
    float4 *sc_o = nullptr, *sc_d = nullptr, *sc_c = nullptr, *sd_o = nullptr, *sd_d = nullptr, *sd_c = nullptr;
    float4* prev = nullptr;
};
// The context's own wavefront storage (grown on demand, reused by every render).
struct Wavefront {
    DBuf<float4> ray_o0, ray_d0, ray_o1, ray_d1, hit, thr, rad, sa_o, sa_d, sa_c, sb_o, sb_d, sb_c;
    DBuf<uint32_t> hit_inst, slot_job, counters, err;
    DBuf<uint2> rng;
    DBuf<unsigned long long> work;
    DBuf<Job> jobs;
    DBuf<float4> sc_o, sc_d, sc_c, sd_o, sd_d, sd_c, prev;   // EXT waves only (allocated on first need)
    uint64_t generation = 0;  // bumps when a buffer moves (captured graphs refer to the old ones)
    // The environment and mesh shadow rays and the previous vertex of every slot, for waves
    // with an image environment or emissive meshes (112 B per slot).
    void reserve_ext(size_t slots) {
        if (slots > sc_o.n) {
            DBuf<float4>* f4[] = {&sc_o, &sc_d, &sc_c, &sd_o, &sd_d, &sd_c, &prev};
            for (auto* b : f4) b->alloc(slots);
            generation++;
        }
    }
    WaveBuffers view() const {
        WaveBuffers w;
        w.sc_o = sc_o.p; w.sc_d = sc_d.p; w.sc_c = sc_c.p; w.sd_o = sd_o.p; w.sd_d = sd_d.p; w.sd_c = sd_c.p; w.prev = prev.p;
        w.capacity = ray_o0.n; w.job_capacity = uint32_t(jobs.n);
        w.ray_o0 = ray_o0.p; w.ray_d0 = ray_d0.p; w.ray_o1 = ray_o1.p; w.ray_d1 = ray_d1.p; w.hit = hit.p; w.thr = thr.p; w.rad = rad.p;
        w.sa_o = sa_o.p; w.sa_d = sa_d.p; w.sa_c = sa_c.p; w.sb_o = sb_o.p; w.sb_d = sb_d.p; w.sb_c = sb_c.p;
        w.hit_inst = hit_inst.p; w.slot_job = slot_job.p; w.counters = counters.p; w.err = err.p; w.rng = rng.p; w.work = work.p; w.jobs = jobs.p;
        return w;
    }
    void reserve(size_t slots, uint32_t njobs) {
        if (slots > ray_o0.n) {
            DBuf<float4>* f4[] = {&ray_o0, &ray_d0, &ray_o1, &ray_d1, &hit, &thr, &rad, &sa_o, &sa_d, &sa_c, &sb_o, &sb_d, &sb_c};
            for (auto* b : f4) b->alloc(slots);
            hit_inst.alloc(slots); slot_job.alloc(slots); rng.alloc(slots);
            if (sc_o.p) reserve_ext(slots);
            generation++;
        }
        if (!counters.p) { counters.alloc(16); err.alloc(1); work.alloc(8); generation++; }
        if (njobs > jobs.n) { jobs.alloc(std::max<size_t>(njobs, 16)); generation++; }
    }
    void release() {
        DBuf<float4>* f4[] = {&ray_o0, &ray_d0, &ray_o1, &ray_d1, &hit, &thr, &rad, &sa_o, &sa_d, &sa_c, &sb_o, &sb_d, &sb_c,
                              &sc_o, &sc_d, &sc_c, &sd_o, &sd_d, &sd_c, &prev};
        for (auto* b : f4) b->release();
        hit_inst.release(); slot_job.release(); rng.release(); counters.release(); err.release(); work.release(); jobs.release();
    }
};
struct GraphEntry { uint64_t key; cudaGraphExec_t exec; };

constexpr size_t SINGLE_JOB_WAVE_SLOTS = size_t(64) << 20;   // 14.8 GB of queues per wavefront when full
struct vkb_ctx {
    int device = 0;
    int sms = 148;
    cudaStream_t stream = nullptr;
    DBuf<ushort4> lut;
    DBuf<float> filter;
    Wavefront wave;
    DBuf<float4> accum, staging;        // per-render accumulators and host-output staging (all jobs of a call)
    DBuf<uint32_t> ids;                 // primary ids of the jobs that asked for them
    size_t wave_capacity = 32u << 20;   // path slots per wave (autotuned); 7.4 GB of queues when full
    int trace_blocks_per_sm = 128;      // trace/shade grid = SMs x this (autotuned)
    uint64_t launches = 0;
    cudaEvent_t ev0 = nullptr, ev1 = nullptr;
    std::vector<cudaEvent_t> kernel_events;
    std::vector<cudaEvent_t> cache_events;    // timed renders: around each radiance-cache query launch
    DBuf<float4> ad_mean, ad_m2;              // adaptive stopping: per-pixel moments
    DBuf<uint32_t> ad_state;                  // and parity/stop bits
    DBuf<float4> guide_slots, guide_accum, guide_staging;   // denoiser-guide renders
    // Overlapped waves of single-job renders: a second stream and wavefront; consecutive
    // waves alternate between the two, their accumulations kept in wave order by events.
    cudaStream_t stream2 = nullptr;
    Wavefront wave2;
    cudaEvent_t fork_ev = nullptr, join_ev = nullptr, acc_ev[2] = {nullptr, nullptr};
};

struct vkb_scene {
    vkb_ctx* ctx = nullptr;
    // host copies of the descriptor
    uint32_t num_meshes = 0, num_instances = 0, total_tris = 0;
    std::vector<MeshInfo> mesh_info;
    std::vector<uint32_t> inst_mesh, inst_mat;
    std::vector<vkb_material> materials;
    std::vector<vkb_light> lights;
    vkb_camera camera{};
    vkb_environment env{};
    uint32_t tree_nodes = 0;
    DBuf<float4> o2w_next;                    // rows of an update, compared with o2w on the device
    DBuf<unsigned long long> changed;         // its changed-bytes count
    // device scene
    DBuf<float4> vpos, vnrm, blas_tris, tri_nrm, o2w, w2o, inst_lo, inst_hi, tri_lo, tri_hi;
    DBuf<uint32_t> indices, tlas_codes;
    DBuf<uint32_t> tlas_order, tlas_leaf_parent, tlas_node_parent, tlas_counters;  // TLAS topology kept for refits
    uint64_t motion_bytes = 0, tlas_rebuilds = 0, tlas_refits = 0;
    DBuf<uint4> inst_info;
    DBuf<MeshInfo> meshes;
    DBuf<BvhNode> tlas_nodes;                 // binary TLAS (built, refitted; SAH statistics)
    DBuf<Bvh4Node> blas4, tlas4;              // 4-wide traversal nodes (TLAS sparse: index = binary node)
    DBuf<Bvh8Node> blas8;                     // compressed 8-wide BLAS nodes (VKB_BLAS_WIDE8 scenes; blas4 then unused)
    uint32_t blas_format = VKB_BLAS_WIDE4;
    uint32_t blas_builder = VKB_BLAS_BUILD_SAH;
    DBuf<uint8_t> tlas_odd;                   // depth parity of the binary TLAS nodes
    DBuf<TlasLeaf> tlas_leaves;
    DBuf<vkb_material> d_materials;
    DBuf<vkb_light> d_lights;
    DBuf<LightTreeNode> tree;
    LbvhScratch scratch;
    PlocScratch ploc;
    uint32_t tlas_builder = VKB_TLAS_LBVH;
    float build_ms = 0.f;
    cudaEvent_t ev0 = nullptr, ev1 = nullptr;
    uint64_t launches = 0;                    // kernels launched for this scene so far
    // A fork (vkb_scene_fork) shares its base's meshes, BLASes, materials, lights and light
    // tree and owns only its instances and TLAS; a base counts its live forks.
    vkb_scene* base = nullptr;
    uint32_t forks = 0;
    float install_ms = 0.f, blas_host_ms = 0.f, upload_ms = 0.f, tlas_ms = 0.f;   // install cost
    // Image environment (env_w == 0: none): texels, proposal, strength x colour, rotation.
    DBuf<float4> env_img;
    DBuf<float2> env_dist;
    uint32_t env_w = 0, env_h = 0;
    float env_scale[3] = {0.f, 0.f, 0.f};
    float env_rot[9] = {1.f, 0.f, 0.f, 0.f, 1.f, 0.f, 0.f, 0.f, 1.f};
    // Emissive meshes (em_tris == 0: none): the source topology (shared with forks) and
    // the weight tree (each scene's own: it follows its instance rows).
    DBuf<uint32_t> em_inst_source;
    DBuf<uint2> em_sources;
    DBuf<float> em_tree;
    uint32_t em_count = 0, em_tris = 0, em_leaves = 0;
};

namespace {

vkb_status fail(vkb_status st, const std::string& msg) { g_error = msg; return st; }
template <class F> vkb_status guarded(F&& f) {
    try {
        f();
        return VKB_OK;
    } catch (const CudaError& e) {
        return fail(e.code == cudaErrorMemoryAllocation ? VKB_OUT_OF_MEMORY : VKB_INTERNAL, std::string(e.what) + ": " + cudaGetErrorString(e.code));
    } catch (const ArgError& e) {
        return fail(VKB_INVALID_ARG, e.msg);
    } catch (const Unsupported& e) {
        return fail(VKB_UNSUPPORTED, e.msg);
    } catch (const InternalError& e) {
        return fail(VKB_INTERNAL, e.msg);
    } catch (const DeviceTimeout& e) {
        return fail(VKB_DEVICE_TIMEOUT, e.msg);
    } catch (const std::bad_alloc&) {
        return fail(VKB_OUT_OF_MEMORY, "host allocation failed");
    }
}

SceneView scene_view(const vkb_scene* s) {
    SceneView v;
    v.tlas_nodes = s->tlas4.p; v.tlas_leaves = s->tlas_leaves.p;
    v.blas_nodes = s->blas4.p; v.blas_tris = s->blas_tris.p;
    v.blas8 = s->blas8.p;   // null unless the scene was built with compressed 8-wide BLASes
    v.num_instances = s->num_instances;
    return v;
}

// The proposal of an environment image (crates/vork-render/src/environment.rs:573-620):
// per texel the 3x3 (1,2,1)^2/16 stencil of alpha-weighted RGB (columns wrap, rows clamp),
// its Rec.709 luminance times the texel's solid angle, accumulated in f64 row-major and
// normalised to (cumulative mass, density) in f32; a black image gets the uniform sphere.
std::vector<float2> env_proposal(const float* rgba, uint32_t dw, uint32_t dh) {
    const double PI_D = 3.141592653589793, TAU_D = 2.0 * PI_D;
    const float lum[3] = {0.2126f, 0.7152f, 0.0722f};
    std::vector<double> cum(size_t(dw) * dh), dens(size_t(dw) * dh);
    double total = 0.0;
    for (uint32_t y = 0; y < dh; ++y) {
        const double solid = TAU_D / dw * (std::cos(PI_D * y / dh) - std::cos(PI_D * (y + 1) / dh));
        const int rows[3] = {std::max(int(y) - 1, 0), int(y), std::min(int(y) + 1, int(dh) - 1)};
        for (uint32_t x = 0; x < dw; ++x) {
            const int cols[3] = {(int(x) - 1 + int(dw)) % int(dw), int(x), (int(x) + 1) % int(dw)};
            double rgb[3] = {0.0, 0.0, 0.0};
            for (int dy = 0; dy < 3; ++dy)
                for (int dx = 0; dx < 3; ++dx) {
                    const size_t at = (size_t(rows[dy]) * dw + cols[dx]) * 4;
                    const double w = double(rgba[at + 3]) * (dx == 1 ? 2.0 : 1.0) * (dy == 1 ? 2.0 : 1.0);
                    for (int c = 0; c < 3; ++c) rgb[c] += double(rgba[at + c]) * w;
                }
            double l = 0.0;
            for (int c = 0; c < 3; ++c) l += double(lum[c]) * (rgb[c] / 16.0);
            total += l * solid;
            cum[size_t(y) * dw + x] = total;
            dens[size_t(y) * dw + x] = l;
        }
    }
    std::vector<float2> out(cum.size());
    if (total > 0.0) {
        for (size_t i = 0; i < cum.size(); ++i) out[i] = make_float2(float(cum[i] / total), float(dens[i] / total));
        out.back().x = 1.f;
    } else {
        for (size_t i = 0; i < cum.size(); ++i) {
            const uint32_t y = uint32_t(i / dw), x = uint32_t(i % dw);
            const float row = (1.f - std::cos(float(PI_D) * float(y) / float(dh))) / 2.f;
            const float next = (1.f - std::cos(float(PI_D) * float(y + 1) / float(dh))) / 2.f;
            out[i] = make_float2(row + (next - row) * (float(x + 1) / float(dw)), 1.f / (4.f * float(PI_D)));
        }
    }
    return out;
}

// Instance rows -> w2o, world boxes, TLAS and its leaf records.  The TLAS is the
// Karras LBVH or a PLOC tree over the instance boxes in Morton order (the scene's
// tlas_builder); both keep parent links for refits.
void build_emitter_tree(vkb_scene* s);
void build_tlas(vkb_scene* s) {
    cudaStream_t st = s->ctx->stream;
    int sms = s->ctx->sms;
    uint32_t n = s->num_instances;
    if (n == 0) return;
    VKB_CUDA(cudaEventRecord(s->ev0, st));
    k_instances<<<grid_for(n, 256, sms), 256, 0, st>>>(n, s->o2w.p, s->inst_info.p, s->meshes.p, s->w2o.p, s->inst_lo.p, s->inst_hi.p);
    s->tlas_order.alloc(n); s->tlas_leaf_parent.alloc(n); s->tlas_node_parent.alloc(std::max(1u, n)); s->tlas_counters.alloc(std::max(1u, n));
    if (s->tlas_builder == VKB_TLAS_LBVH || n == 1) {
        build_lbvh(n, s->inst_lo.p, s->inst_hi.p, s->tlas_nodes.p, s->scratch, st, sms, s->launches);
        // Keep the topology for later refits (the LBVH scratch is shared with other builds).
        if (n > 1) {
            VKB_CUDA(cudaMemcpyAsync(s->tlas_leaf_parent.p, s->scratch.leaf_parent.p, n * sizeof(uint32_t), cudaMemcpyDeviceToDevice, st));
            VKB_CUDA(cudaMemcpyAsync(s->tlas_node_parent.p, s->scratch.node_parent.p, (n - 1) * sizeof(uint32_t), cudaMemcpyDeviceToDevice, st));
        }
    } else {
        morton_sort(n, s->inst_lo.p, s->inst_hi.p, s->scratch, st, sms, s->launches);
        build_ploc(n, s->inst_lo.p, s->inst_hi.p, s->tlas_nodes.p, s->tlas_leaf_parent.p, s->tlas_node_parent.p, s->tlas_counters.p,
                   s->scratch, s->ploc, st, sms, s->launches);
    }
    s->launches += 4;
    k_tlas_leaves<<<grid_for(n, 256, sms), 256, 0, st>>>(n, s->scratch.ids_sorted.p, s->w2o.p, s->inst_info.p, s->meshes.p, s->d_materials.p, s->tlas_leaves.p);
    const uint32_t ni = n > 1 ? n - 1 : 1u;
    if (n > 1) k_bvh_parity<<<grid_for(ni, 256, sms), 256, 0, st>>>(ni, s->tlas_node_parent.p, s->tlas_odd.p);
    else VKB_CUDA(cudaMemsetAsync(s->tlas_odd.p, 0, 1, st));
    k_collapse4<<<grid_for(ni, 256, sms), 256, 0, st>>>(ni, s->tlas_nodes.p, s->tlas_odd.p, s->tlas4.p);
    VKB_CUDA(cudaMemcpyAsync(s->tlas_codes.p, s->scratch.codes.p, n * sizeof(uint32_t), cudaMemcpyDeviceToDevice, st));
    VKB_CUDA(cudaMemcpyAsync(s->tlas_order.p, s->scratch.ids_sorted.p, n * sizeof(uint32_t), cudaMemcpyDeviceToDevice, st));
    s->tlas_rebuilds++;
    build_emitter_tree(s);
    VKB_CUDA(cudaEventRecord(s->ev1, st));
    VKB_CUDA(cudaEventSynchronize(s->ev1));
    VKB_CUDA(cudaEventElapsedTime(&s->build_ms, s->ev0, s->ev1));
}

// The mesh-source weight tree at the scene's current instance rows: the leaves, the
// large inner levels one launch each, the top levels (<= 1024 nodes) in one block.
void build_emitter_tree(vkb_scene* s) {
    if (!s->em_tris) return;
    cudaStream_t st = s->ctx->stream;
    const int sms = s->ctx->sms;
    Job j{};
    j.o2w = s->o2w.p; j.w2o = s->w2o.p; j.inst_info = s->inst_info.p; j.meshes = s->meshes.p; j.materials = s->d_materials.p;
    j.em_inst_source = s->em_inst_source.p; j.em_sources = s->em_sources.p; j.indices = s->indices.p; j.vpos = s->vpos.p;
    j.em_count = s->em_count; j.em_tris = s->em_tris; j.em_leaves = s->em_leaves;
    k_em_leaves<<<grid_for(s->em_leaves, 256, sms), 256, 0, st>>>(j, s->em_tree.p);
    s->launches++;
    uint32_t first = s->em_leaves / 2u;
    for (; first > 1024u; first >>= 1) { k_em_reduce<<<grid_for(first, 256, sms), 256, 0, st>>>(s->em_tree.p, first); s->launches++; }
    if (first >= 1u) { k_em_reduce_top<<<1, 1024, 0, st>>>(s->em_tree.p, first); s->launches++; }
    VKB_CUDA(cudaGetLastError());
}
// Emissive-mesh sources (emitters.rs:22-44): every instance drawn with a material whose
// emission_luminance > 0 and colour is not black, its triangles counted in instance order.
void emitter_topology(vkb_scene* s, cudaStream_t str) {
    std::vector<uint32_t> inst_source(s->num_instances, 0xffffffffu);
    std::vector<uint2> sources;
    uint64_t tris = 0;
    for (uint32_t i = 0; i < s->num_instances; ++i) {
        const vkb_material& m = s->materials[s->inst_mat[i]];
        if (!(m.emission_luminance > 0.f && (m.emission_color[0] != 0.f || m.emission_color[1] != 0.f || m.emission_color[2] != 0.f))) continue;
        const uint32_t nt = s->mesh_info[s->inst_mesh[i]].num_triangles;
        if (!nt) continue;
        tris += nt;
        if (tris > (uint64_t(1) << 30)) throw Unsupported{"more than 2^30 emissive triangles"};
        inst_source[i] = uint32_t(sources.size());
        sources.push_back(make_uint2(i, uint32_t(tris)));
    }
    if (sources.empty()) return;
    s->em_count = uint32_t(sources.size());
    s->em_tris = uint32_t(tris);
    s->em_leaves = 1u;
    while (s->em_leaves < s->em_tris) s->em_leaves <<= 1;
    s->em_inst_source.upload(inst_source.data(), inst_source.size(), str);
    s->em_sources.upload(sources.data(), sources.size(), str);
    s->em_tree.alloc(2 * size_t(s->em_leaves));
}

// Refit the TLAS in place: new instance boxes and world->object rows, same topology.
void refit_tlas(vkb_scene* s) {
    cudaStream_t st = s->ctx->stream;
    int sms = s->ctx->sms;
    uint32_t n = s->num_instances;
    if (n == 0) return;
    VKB_CUDA(cudaEventRecord(s->ev0, st));
    k_instances<<<grid_for(n, 256, sms), 256, 0, st>>>(n, s->o2w.p, s->inst_info.p, s->meshes.p, s->w2o.p, s->inst_lo.p, s->inst_hi.p);
    if (n == 1) {
        k_single_leaf<<<1, 1, 0, st>>>(s->inst_lo.p, s->inst_hi.p, s->tlas_nodes.p);
    } else {
        VKB_CUDA(cudaMemsetAsync(s->tlas_counters.p, 0, (n - 1) * sizeof(uint32_t), st));
        k_refit<<<grid_for(n, 256, sms), 256, 0, st>>>(int(n), s->tlas_order.p, s->inst_lo.p, s->inst_hi.p, s->tlas_nodes.p, s->tlas_leaf_parent.p,
                                                       s->tlas_node_parent.p, s->tlas_counters.p);
    }
    k_tlas_leaves<<<grid_for(n, 256, sms), 256, 0, st>>>(n, s->tlas_order.p, s->w2o.p, s->inst_info.p, s->meshes.p, s->d_materials.p, s->tlas_leaves.p);
    const uint32_t ni = n > 1 ? n - 1 : 1u;
    k_collapse4<<<grid_for(ni, 256, sms), 256, 0, st>>>(ni, s->tlas_nodes.p, s->tlas_odd.p, s->tlas4.p);
    s->launches += 4;
    VKB_CUDA(cudaGetLastError());
    build_emitter_tree(s);
    VKB_CUDA(cudaEventRecord(s->ev1, st));
    VKB_CUDA(cudaEventSynchronize(s->ev1));
    VKB_CUDA(cudaEventElapsedTime(&s->build_ms, s->ev0, s->ev1));
    s->tlas_refits++;
}

// rt.rs:1465-1476: accumulate the changed object bytes; rebuild once they reach a
// quarter of the object buffer, otherwise refit (policy 0).  1 rebuilds, 2 refits.
// A server wave on the second stream may still read a scene's rows and TLAS: an update on
// the context's stream starts after it.
void after_second_stream(vkb_ctx* c) {
    VKB_CUDA(cudaEventRecord(c->join_ev, c->stream2));
    VKB_CUDA(cudaStreamWaitEvent(c->stream, c->join_ev, 0));
}
void update_tlas(vkb_scene* s, uint64_t changed_bytes, int policy) {
    uint64_t total = uint64_t(s->num_instances) * 48u;
    uint64_t threshold = std::max<uint64_t>(1, (total + 3) / 4);
    s->motion_bytes += changed_bytes;
    bool rebuild = policy == 1 || (policy == 0 && s->motion_bytes >= threshold);
    if (rebuild) { s->motion_bytes = 0; build_tlas(s); }
    else refit_tlas(s);
}

void validate_desc(const vkb_scene_desc* d) {
    if (!d) throw ArgError{"null scene descriptor"};
    if (d->num_meshes && !d->meshes) throw ArgError{"meshes pointer is null"};
    for (uint32_t m = 0; m < d->num_meshes; ++m) {
        const vkb_mesh& me = d->meshes[m];
        if (me.num_triangles && (!me.positions || !me.indices)) throw ArgError{"mesh " + std::to_string(m) + " has no positions or indices"};
        for (size_t i = 0; i < size_t(me.num_triangles) * 3; ++i)
            if (me.indices[i] >= me.num_vertices) throw ArgError{"mesh " + std::to_string(m) + " index out of range"};
        for (size_t i = 0; i < size_t(me.num_vertices) * 3; ++i)
            if (!std::isfinite(me.positions[i])) throw ArgError{"mesh " + std::to_string(m) + " has a non-finite position"};
    }
    if (d->num_instances && (!d->instance_rows || !d->instance_mesh || !d->instance_material)) throw ArgError{"instance arrays are null"};
    for (uint32_t i = 0; i < d->num_instances; ++i) {
        if (d->instance_mesh[i] >= d->num_meshes) throw ArgError{"instance mesh index out of range"};
        if (d->instance_material[i] >= d->num_materials) throw ArgError{"instance material index out of range"};
    }
    for (uint32_t m = 0; m < d->num_materials; ++m) {
        const vkb_material& mt = d->materials[m];
        if (!(mt.emission_luminance >= 0.f) || !std::isfinite(mt.emission_luminance)) throw ArgError{"emission luminance must be finite and non-negative"};
        for (int k = 0; k < 3; ++k)
            if (!std::isfinite(mt.emission_color[k])) throw ArgError{"emission colour must be finite"};
    }
    for (uint32_t l = 0; l < d->num_lights; ++l) {
        float k = d->lights[l].position[3];
        if (!(k == 0.f || k == 1.f || k == 2.f || k == 3.f)) throw ArgError{"light kind must be 0..3"};
    }
    if (d->camera.width == 0 || d->camera.height == 0) throw ArgError{"camera resolution is zero"};
    if (d->tlas_builder > VKB_TLAS_PLOC) throw ArgError{"unknown TLAS builder"};
    if (d->blas_format > VKB_BLAS_WIDE8) throw ArgError{"unknown BLAS format"};
    if (d->blas_builder > VKB_BLAS_BUILD_PLOC) throw ArgError{"unknown BLAS builder"};
    if (d->blas_builder != VKB_BLAS_BUILD_SAH && d->blas_format == VKB_BLAS_WIDE8)
        throw Unsupported{"compressed 8-wide BLASes are collapsed from the host SAH tree"};
    if (const vkb_environment_image* e = d->environment_image) {
        if (!e->rgba || e->width == 0 || e->height == 0) throw ArgError{"environment image has no texels"};
        if (uint64_t(e->width) * e->height > (uint64_t(1) << 26)) throw ArgError{"environment image above 2^26 texels"};
        if (!(e->strength >= 0.f) || !std::isfinite(e->strength)) throw ArgError{"environment strength must be finite and non-negative"};
        for (size_t i = 0; i < size_t(e->width) * e->height * 4; ++i)
            if (!std::isfinite(e->rgba[i]) || e->rgba[i] < 0.f) throw ArgError{"environment image texels must be finite and non-negative"};
    }
}


void validate_camera(const vkb_camera& cam) {
    if (cam.width == 0 || cam.height == 0) throw ArgError{"camera resolution is zero"};
    if (uint64_t(cam.width) * cam.height > (uint64_t(1) << 28)) throw ArgError{"camera resolution above 2^28 pixels"};
    const float* f = &cam.eye[0];
    for (int k = 0; k < 16; ++k) if (!std::isfinite(f[k])) throw ArgError{"camera has a non-finite field"};
}


// ================================================================ wave engine
double host_seconds() { return std::chrono::duration<double>(std::chrono::steady_clock::now().time_since_epoch()).count(); }
// One job of a render call: a scene, its profile, and where its mean image goes.
struct EngineJob {
    vkb_scene* s = nullptr;
    vkb_profile pf{};
    bool own_camera = false;        // render through `camera` instead of the scene's
    vkb_camera camera{};
    float4* ad_mean = nullptr;      // adaptive stopping: per-pixel moments and state
    float4* ad_m2 = nullptr;
    uint32_t* ad_state = nullptr;
    float4* out_dev = nullptr;      // device destination of the mean image
    uint32_t* ids_dev = nullptr;    // device primary ids (first sample) or null
    float4* accum = nullptr;        // device accumulator, npix
    float4* guide_accum = nullptr;  // guide renders: 2 x npix sums; mean planes (device) or null
    float4* guide_albedo = nullptr;
    float4* guide_normal = nullptr;
    uint32_t npix = 0, count = 0, done = 0, pixel_base = 0;
    double admitted_s = 0.0;        // serving: host clock at admission (aging of the shortest-first order)
};
struct WaveTotals {
    uint32_t launches = 0, trace_launches = 0, cache_launches = 0;
    float trace_ms = 0.f, render_ms = 0.f, cache_ms = 0.f;
    uint32_t counters[16] = {};
    unsigned long long work[8] = {};
    uint32_t err = 0;
};

void validate_profile(const vkb_profile* pf) {
    if (pf->adaptive > 1u) throw ArgError{"adaptive must be 0 or 1"};
    if (pf->adaptive && !(pf->adaptive_threshold >= 0.f)) throw ArgError{"adaptive_threshold must be non-negative"};
    if (pf->samples == 0) throw ArgError{"samples must be positive"};
    if (pf->first_sample >= pf->samples) throw ArgError{"first_sample beyond samples"};
    uint32_t count = pf->sample_count ? pf->sample_count : pf->samples - pf->first_sample;
    if (pf->first_sample + count > pf->samples) throw ArgError{"sample range beyond samples"};
    if (pf->bounces[0] > 250) throw ArgError{"bounce budget above 250"};
}
uint32_t sample_mask_of(uint32_t samples) { return samples <= 1 ? 0u : ((2u << (31 - __builtin_clz(samples - 1u))) - 1u); }

// The static part of a job's device record (the wave fields are set per wave).
Job make_job(const EngineJob& e) {
    const vkb_scene* s = e.s;
    const vkb_profile& pf = e.pf;
    Job j{};
    j.sv = scene_view(s);
    j.o2w = s->o2w.p; j.w2o = s->w2o.p; j.inst_info = s->inst_info.p; j.meshes = s->meshes.p;
    j.tri_nrm = s->tri_nrm.p;
    j.materials = s->d_materials.p; j.lights = s->d_lights.p; j.num_lights = uint32_t(s->lights.size());
    j.tree = s->tree.p; j.tree_nodes = s->tree_nodes;
    j.cam = e.own_camera ? e.camera : s->camera; j.env = s->env;
    j.spp = pf.samples; j.seed = pf.seed;
    for (int k = 0; k < 4; ++k) j.bounces[k] = pf.bounces[k];
    j.caustics = pf.caustics;
    j.sample_mask = sample_mask_of(pf.samples);
    j.clamp_direct = pf.clamp_direct; j.clamp_indirect = pf.clamp_indirect; j.light_threshold = pf.light_threshold;
    j.npix = e.npix; j.first_sample = pf.first_sample;
    j.pixel_base = e.pixel_base;
    j.accum = e.accum; j.primary_ids = e.ids_dev; j.out = e.out_dev;
    j.adaptive = (pf.adaptive && e.ad_state) ? 1u : 0u;   // only where the caller gave it moment buffers
    j.adaptive_threshold = pf.adaptive_threshold > 0.f ? pf.adaptive_threshold : 0.01f;
    j.adaptive_min = pf.adaptive_min_samples ? pf.adaptive_min_samples : std::max(16u, uint32_t(std::sqrt(float(pf.samples))));
    j.ad_mean = e.ad_mean; j.ad_m2 = e.ad_m2; j.ad_state = e.ad_state;
    j.guide_accum = e.guide_accum; j.guide_albedo = e.guide_albedo; j.guide_normal = e.guide_normal;
    j.env_img = s->env_img.p; j.env_dist = s->env_dist.p; j.env_w = s->env_w; j.env_h = s->env_h;
    for (int k = 0; k < 3; ++k) j.env_scale[k] = s->env_scale[k];
    for (int k = 0; k < 9; ++k) j.env_rot[k] = s->env_rot[k];
    j.em_inst_source = s->em_inst_source.p; j.em_sources = s->em_sources.p; j.em_tree = s->em_tree.p;
    j.indices = s->indices.p; j.vpos = s->vpos.p;
    j.em_count = s->em_count; j.em_tris = s->em_tris; j.em_leaves = s->em_leaves;
    return j;
}

PathParams path_params(const vkb_ctx* c, const WaveBuffers& w, uint32_t njobs) {
    PathParams p{};
    p.jobs = w.jobs; p.njobs = njobs; p.slot_job = w.slot_job;
    p.lut.texels = c->lut.p; p.filter = c->filter.p;
    p.ray_o[0] = w.ray_o0; p.ray_d[0] = w.ray_d0; p.ray_o[1] = w.ray_o1; p.ray_d[1] = w.ray_d1;
    p.hit = w.hit; p.hit_inst = w.hit_inst; p.thr = w.thr; p.rad = w.rad; p.rng = w.rng;
    p.sa_o = w.sa_o; p.sa_d = w.sa_d; p.sa_c = w.sa_c; p.sb_o = w.sb_o; p.sb_d = w.sb_d; p.sb_c = w.sb_c;
    p.counters = w.counters; p.work = w.work; p.err = w.err;
    p.guide = w.guide;
    p.sc_o = w.sc_o; p.sc_d = w.sc_d; p.sc_c = w.sc_c; p.sd_o = w.sd_o; p.sd_d = w.sd_d; p.sd_c = w.sd_c; p.prev = w.prev;
    return p;
}

// A render's radiance-cache hooks: the device side (copied into PathParams) and what
// the query kernel after the bounce loop (mode 1) needs.
struct CacheLaunch {
    CacheParams dev{};
    const __nv_bfloat16* w = nullptr;
    const __half* table = nullptr;
    uint32_t* err = nullptr;
};

// The kernels of one wave: camera, then per bounce closest-hit trace, shade, shadow trace;
// then the radiance-cache queries, if any; then accumulation.  Timed
// mode records events around every closest-hit trace.
// The closest-hit and shadow traces of one bounce, instantiated for the counters (COUNT),
// the EXT shadow entries and the BLAS format (W8: compressed 8-wide).
template <bool BATCH, bool W8>
void launch_trace(bool counted, int grid, cudaStream_t st, const PathParams& p, int cur) {
    if (counted) k_trace<true, BATCH, W8><<<grid, TRACE_BLOCK, 0, st>>>(p, cur);
    else k_trace<false, BATCH, W8><<<grid, TRACE_BLOCK, 0, st>>>(p, cur);
}
template <bool BATCH, bool EXT, bool W8>
void launch_shadow(bool counted, int grid, cudaStream_t st, const PathParams& p) {
    if (counted) k_trace_shadow<true, BATCH, EXT, W8><<<grid, TRACE_BLOCK, 0, st>>>(p);
    else k_trace_shadow<false, BATCH, EXT, W8><<<grid, TRACE_BLOCK, 0, st>>>(p);
}
// st: the wave's stream; acc_wait / acc_done: events that order the accumulation after
// the previous wave's and mark this one's (overlapped waves), or null.
template <bool BATCH>
void wave_kernels(vkb_ctx* c, const PathParams& p, uint32_t bounces, bool counted, bool timed, WaveTotals& tot,
                  const CacheLaunch* cache = nullptr, bool ext = false, bool w8 = false, cudaStream_t st = nullptr,
                  cudaEvent_t acc_wait = nullptr, cudaEvent_t acc_done = nullptr) {
    if (!st) st = c->stream;
    const int sms = c->sms, tgrid = sms * c->trace_blocks_per_sm, sgrid = sms * c->trace_blocks_per_sm;
    const bool adaptive = !BATCH && p.job0.adaptive;
    if (adaptive) k_adaptive_decide<<<grid_for(p.job0.npix, 256, sms), 256, 0, st>>>(p);
    k_start_wave<<<1, 1, 0, st>>>(p.counters, adaptive ? 1u : 0u);
    k_camera<BATCH><<<sms * 8, 256, 0, st>>>(p);
    for (uint32_t b = 0; b <= bounces; ++b) {
        int cur = int(b & 1u);
        if (timed) {
            while (c->kernel_events.size() < 2 * (tot.trace_launches + 1)) {
                cudaEvent_t e;
                VKB_CUDA(cudaEventCreate(&e));
                c->kernel_events.push_back(e);
            }
            VKB_CUDA(cudaEventRecord(c->kernel_events[2 * tot.trace_launches], st));
        }
        if (w8) launch_trace<BATCH, true>(counted, tgrid, st, p, cur);
        else launch_trace<BATCH, false>(counted, tgrid, st, p, cur);
        if (timed) VKB_CUDA(cudaEventRecord(c->kernel_events[2 * tot.trace_launches + 1], st));
        tot.trace_launches++;
        if (!BATCH && b == 0u && p.guide) { k_guides<<<sms * 8, 256, 0, st>>>(p); tot.launches += 1; }
        k_reset_queues<<<1, 1, 0, st>>>(p.counters, cur ^ 1);
        // Waves with an image environment or emissive meshes run the kernels with their
        // strategies (two more shadow rays per vertex); the others keep the plain ones.
        if (ext) {
            k_shade<BATCH, true><<<sgrid, SHADE_BLOCK, 0, st>>>(p, cur);
            if (w8) launch_shadow<BATCH, true, true>(counted, tgrid, st, p);
            else launch_shadow<BATCH, true, false>(counted, tgrid, st, p);
        } else {
            k_shade<BATCH, false><<<sgrid, SHADE_BLOCK, 0, st>>>(p, cur);
            if (w8) launch_shadow<BATCH, false, true>(counted, tgrid, st, p);
            else launch_shadow<BATCH, false, false>(counted, tgrid, st, p);
        }
    }
    if (cache && cache->dev.mode == 1u) {
        if (timed) {
            while (c->cache_events.size() < 2 * (tot.cache_launches + 1)) {
                cudaEvent_t e;
                VKB_CUDA(cudaEventCreate(&e));
                c->cache_events.push_back(e);
            }
            VKB_CUDA(cudaEventRecord(c->cache_events[2 * tot.cache_launches], st));
        }
        nrc::QueryIO io{cache->dev.rec, p.counters + 9, cache->dev.capacity, cache->dev.slot, p.thr, p.rad, p.work + 7};
        nrc::k_nrc_forward<nrc::QueryIO><<<sms * 4, nrc::TILE, nrc::FWD_SMEM, st>>>(io, cache->w, cache->table, cache->err);
        if (timed) VKB_CUDA(cudaEventRecord(c->cache_events[2 * tot.cache_launches + 1], st));
        tot.cache_launches++;
        tot.launches += 1;
    }
    if (acc_wait) VKB_CUDA(cudaStreamWaitEvent(st, acc_wait, 0));
    k_accumulate<BATCH><<<sms * 8, 256, 0, st>>>(p);
    if (acc_done) VKB_CUDA(cudaEventRecord(acc_done, st));
    tot.launches += 3 + 4 * (bounces + 1) + (adaptive ? 1 : 0);
}

// A wavefront that runs jobs wave by wave.  Each wave gives one sample to every
// unfinished job that fits (in admission order), then more samples while path slots
// remain; uploads the job table; and runs the wave, replayed from a captured CUDA
// graph when several jobs share it.  Jobs may be added between waves (continuous
// batching) and are resolved into their out_dev when finished.
struct WaveEngine {
    vkb_ctx* c;
    WaveBuffers w;
    WaveBuffers w2;                     // overlapped waves: the second wavefront (on c->stream2)
    bool overlap = false;
    uint32_t waves = 0;
    cudaEvent_t* acc_ev = nullptr;      // overlapped waves: the accumulation-order events (default: the context's)
    cudaStream_t last_stream = nullptr; // the stream of the latest wave
    // A long-lived engine (the server's) clears admitted jobs' accumulators on the stream of
    // the next wave instead of the context's stream, which may still be running the other
    // stream's work: a later wave's accumulation waits for that wave's by the event chain.
    bool defer_clears = false;
    std::vector<std::pair<float4*, size_t>> pending_clears;
    size_t capacity;
    uint32_t flags;
    bool graphs;
    std::vector<EngineJob> jobs;
    std::vector<Job> table;
    std::vector<Job> wave_table;        // the jobs of the current wave (uploaded)
    WaveTotals tot;
    std::vector<GraphEntry> captured;   // this engine's wave graphs (they point at its buffers)
    // Scheduling: fair (one sample of every unfinished job per wave, then more), packed
    // (each job's remaining samples before the next job: fewer scenes per wave, so their
    // BVHs stay in L2 -- batch throughput), or shortest remaining work first (the jobs
    // with the fewest paths left take their samples first -- serving latency).
    bool packed = false, srpt = false;
    double aging_rate = 0.0;              // shortest-first aging, paths per second waited
    const CacheLaunch* cache = nullptr;   // radiance-cache hooks (single-job renders)
    ~WaveEngine() { for (auto& g : captured) cudaGraphExecDestroy(g.exec); }
    WaveEngine(vkb_ctx* ctx, const WaveBuffers& wb, size_t cap, uint32_t fl, bool use_graphs) : c(ctx), w(wb), capacity(cap), flags(fl), graphs(use_graphs) {
        cudaStream_t st = c->stream;
        VKB_CUDA(cudaMemsetAsync(w.counters, 0, 16 * sizeof(uint32_t), st));
        VKB_CUDA(cudaMemsetAsync(w.err, 0, sizeof(uint32_t), st));
        VKB_CUDA(cudaMemsetAsync(w.work, 0, 8 * sizeof(unsigned long long), st));
    }
    void add(EngineJob e) {
        if (defer_clears) pending_clears.push_back({e.accum, size_t(e.npix)});
        else VKB_CUDA(cudaMemsetAsync(e.accum, 0, size_t(e.npix) * sizeof(float4), c->stream));
        jobs.push_back(e);
        table.push_back(make_job(jobs.back()));
    }
    bool finished(size_t k) const { return jobs[k].done >= jobs[k].count; }
    // Drop finished jobs (after resolve) from the front of the table.
    void compact() {
        size_t o = 0;
        for (size_t k = 0; k < jobs.size(); ++k)
            if (!finished(k)) { jobs[o] = jobs[k]; table[o] = table[k]; ++o; }
        jobs.resize(o); table.resize(o);
    }
    // One wave; false when no job has work left.
    bool step() {
        // Overlapped waves alternate between the two wavefronts and streams.
        const bool second = overlap && (waves & 1u);
        const WaveBuffers& w = second ? this->w2 : this->w;
        cudaStream_t st = second ? c->stream2 : c->stream;
        cudaEvent_t* order_ev = acc_ev ? acc_ev : c->acc_ev;
        cudaEvent_t acc_wait = (overlap && waves > 0) ? order_ev[(waves - 1) & 1u] : nullptr;
        cudaEvent_t acc_done = overlap ? order_ev[waves & 1u] : nullptr;
        const uint32_t njobs = uint32_t(jobs.size());
        if (njobs == 0) return false;
        if (njobs > w.job_capacity) throw ArgError{"more active jobs than the job table holds"};
        const bool timed = (flags & VKB_PROFILE_TIME_KERNELS) != 0, counted = (flags & VKB_PROFILE_COUNT_TRAVERSAL) != 0;
        std::vector<uint32_t> take(njobs, 0u);
        size_t left = capacity;
        bool any = false;
        if (srpt) {
            // Shortest remaining work first: every job, in order of the paths it has left
            // (admission order on ties), takes as many samples as still fit.
            // With aging, the paths left count as reduced by aging_rate x seconds waited.
            std::vector<uint32_t> order;
            std::vector<double> key(njobs, 0.0);
            const double now = aging_rate > 0.0 ? host_seconds() : 0.0;
            for (uint32_t k = 0; k < njobs; ++k) {
                if (finished(k)) continue;
                order.push_back(k);
                key[k] = double(jobs[k].count - jobs[k].done) * double(jobs[k].npix) - aging_rate * (now - jobs[k].admitted_s);
            }
            std::stable_sort(order.begin(), order.end(), [&](uint32_t a, uint32_t b) { return key[a] < key[b]; });
            for (uint32_t k : order) {
                EngineJob& e = jobs[k];
                uint32_t n = uint32_t(std::min<size_t>(e.count - e.done, left / e.npix));
                if (n == 0 && !any) n = 1;
                if (n == 0) continue;
                take[k] = n; any = true;
                left = size_t(n) * e.npix <= left ? left - size_t(n) * e.npix : 0;
            }
        } else if (packed) {
            // A job whose remaining samples fill at least half a wave takes the wave alone
            // (the plain single-job kernels, its scene alone in L2).  Otherwise first fit in
            // admission order over the small jobs: one that does not fit what is left is
            // skipped for this wave and later ones fill the slots.
            auto big = [&](uint32_t k) { return size_t(jobs[k].count - jobs[k].done) * jobs[k].npix >= capacity / 2; };
            uint32_t first = 0;
            while (first < njobs && finished(first)) ++first;
            if (first < njobs && big(first)) {
                EngineJob& e = jobs[first];
                take[first] = uint32_t(std::max<size_t>(1, std::min<size_t>(e.count - e.done, capacity / e.npix)));
                any = true;
            } else {
                for (uint32_t k = 0; k < njobs && left > 0; ++k) {
                    EngineJob& e = jobs[k];
                    if (finished(k) || big(k)) continue;
                    uint32_t n = uint32_t(std::min<size_t>(e.count - e.done, left / e.npix));
                    if (n == 0) continue;
                    take[k] = n; any = true;
                    left -= size_t(n) * e.npix;
                }
                if (!any)   // only big jobs are left: the first of them alone
                    for (uint32_t k = 0; k < njobs && !any; ++k)
                        if (!finished(k)) {
                            take[k] = uint32_t(std::max<size_t>(1, std::min<size_t>(jobs[k].count - jobs[k].done, capacity / jobs[k].npix)));
                            any = true;
                        }
            }
        } else {
            for (uint32_t k = 0; k < njobs; ++k) {
                EngineJob& e = jobs[k];
                if (finished(k)) continue;
                if (size_t(e.npix) <= left || !any) { take[k] = 1; left = size_t(e.npix) <= left ? left - e.npix : 0; any = true; }
            }
            for (uint32_t k = 0; k < njobs; ++k) {
                if (!take[k]) continue;
                EngineJob& e = jobs[k];
                uint32_t more = uint32_t(std::min<size_t>(e.count - e.done - 1, left / e.npix));
                take[k] += more;
                left -= size_t(more) * e.npix;
            }
        }
        if (!any) return false;
        // The wave's table holds only the jobs that take samples in it, so the camera and
        // accumulate passes see no idle jobs' pixels.
        uint32_t n_paths = 0, bounces = 0, total_pixels = 0;
        wave_table.clear();
        for (uint32_t k = 0; k < njobs; ++k) {
            if (!take[k]) continue;
            EngineJob& e = jobs[k];
            Job& j = table[k];
            e.pixel_base = total_pixels; j.pixel_base = total_pixels; total_pixels += e.npix;
            j.wave_first = e.pf.first_sample + e.done;
            j.wave_samples = take[k];
            j.slot_base = n_paths;
            n_paths += take[k] * e.npix;
            e.done += take[k];
            bounces = std::max(bounces, e.pf.bounces[0]);
            wave_table.push_back(j);
        }
        const uint32_t wave_jobs = uint32_t(wave_table.size());
        const bool batch = wave_jobs > 1;
        // Overlapped waves launch directly: a captured graph would bake in one stream's
        // events and buffers, and the second stream hides the launch gaps a graph saves.
        const bool use_graph = graphs && batch && !timed && !overlap;
        uint32_t wave_counts[2] = {n_paths, total_pixels};
        for (const auto& pc : pending_clears) VKB_CUDA(cudaMemsetAsync(pc.first, 0, pc.second * sizeof(float4), st));
        pending_clears.clear();
        last_stream = st;
        VKB_CUDA(cudaMemcpyAsync(w.jobs, wave_table.data(), wave_jobs * sizeof(Job), cudaMemcpyHostToDevice, st));
        VKB_CUDA(cudaMemcpyAsync(w.counters + 7, wave_counts, sizeof(wave_counts), cudaMemcpyHostToDevice, st));
        PathParams p = path_params(c, w, wave_jobs);
        p.job0 = wave_table[0];
        bool ext = false;
        const bool w8 = wave_table[0].sv.blas8 != nullptr;
        for (const Job& j : wave_table) {
            ext = ext || j.env_w != 0u || j.em_tris != 0u;
            if ((j.sv.blas8 != nullptr) != w8) throw ArgError{"the jobs of one wave share a BLAS format"};
        }
        if (ext && !w.sc_o) throw InternalError{"environment or emissive-mesh wave without its shadow buffers"};
        if (cache) {
            if (batch) throw ArgError{"radiance-cache renders take one job"};
            p.cache = cache->dev;
        }
        if (use_graph) {
            uint64_t key = (uint64_t(bounces) << 1) | 1u;
            key = key * 1315423911ull + (counted ? 7u : 3u) + (ext ? 11u : 0u) + (w8 ? 17u : 0u);
            key = key * 40503ull + wave_jobs;
            key = key * 97ull + uint64_t(c->trace_blocks_per_sm);
            cudaGraphExec_t exec = nullptr;
            for (auto& g : captured) if (g.key == key) exec = g.exec;
            if (!exec) {
                cudaGraph_t g;
                VKB_CUDA(cudaStreamBeginCapture(st, cudaStreamCaptureModeThreadLocal));
                WaveTotals scratch;
                wave_kernels<true>(c, p, bounces, counted, false, scratch, nullptr, ext, w8);
                VKB_CUDA(cudaStreamEndCapture(st, &g));
                VKB_CUDA(cudaGraphInstantiate(&exec, g, 0));
                VKB_CUDA(cudaGraphDestroy(g));
                captured.push_back({key, exec});
            }
            VKB_CUDA(cudaGraphLaunch(exec, st));
            tot.launches += 3 + 4 * (bounces + 1);
            tot.trace_launches += bounces + 1;
        } else if (batch) {
            wave_kernels<true>(c, p, bounces, counted, timed, tot, nullptr, ext, w8, st, acc_wait, acc_done);
        } else {
            wave_kernels<false>(c, p, bounces, counted, timed, tot, cache, ext, w8, st, acc_wait, acc_done);
        }
        VKB_CUDA(cudaGetLastError());
        ++waves;
        return true;
    }
    // Mean image of job k into its out_dev (on `st`, default the context's stream).
    void resolve(size_t k, cudaStream_t st = nullptr) {
        PathParams p = path_params(c, w, 1);
        p.job0 = table[k];
        p.job0.pixel_base = 0;
        k_resolve<false><<<grid_for(jobs[k].npix, 256, c->sms), 256, 0, st ? st : c->stream>>>(p, jobs[k].npix);
        tot.launches += 1;
    }
    // Counters, traversal work and device time of everything run so far (synchronises).
    void collect(float ms_since_ev0) {
        cudaStream_t st = c->stream;
        VKB_CUDA(cudaMemcpyAsync(tot.counters, w.counters, sizeof(tot.counters), cudaMemcpyDeviceToHost, st));
        VKB_CUDA(cudaMemcpyAsync(tot.work, w.work, sizeof(tot.work), cudaMemcpyDeviceToHost, st));
        VKB_CUDA(cudaMemcpyAsync(&tot.err, w.err, sizeof(tot.err), cudaMemcpyDeviceToHost, st));
        uint32_t counters2[16] = {};
        unsigned long long work2[8] = {};
        uint32_t err2 = 0;
        if (overlap) {
            // c->stream has joined c->stream2: the second wavefront's totals are final.
            VKB_CUDA(cudaMemcpyAsync(counters2, w2.counters, sizeof(counters2), cudaMemcpyDeviceToHost, st));
            VKB_CUDA(cudaMemcpyAsync(work2, w2.work, sizeof(work2), cudaMemcpyDeviceToHost, st));
            VKB_CUDA(cudaMemcpyAsync(&err2, w2.err, sizeof(err2), cudaMemcpyDeviceToHost, st));
        }
        VKB_CUDA(cudaStreamSynchronize(st));
        if (overlap) {
            static_assert(sizeof(tot.counters) == sizeof(counters2) && sizeof(tot.work) == sizeof(work2), "per-wavefront totals");
            for (int k = 0; k < 16; ++k) tot.counters[k] += counters2[k];
            for (int k = 0; k < 8; ++k) tot.work[k] += work2[k];
            tot.err |= err2;
        }
        tot.render_ms = ms_since_ev0;
        if (flags & VKB_PROFILE_TIME_KERNELS)
            for (uint32_t k = 0; k < tot.trace_launches; ++k) {
                float e = 0.f;
                VKB_CUDA(cudaEventElapsedTime(&e, c->kernel_events[2 * k], c->kernel_events[2 * k + 1]));
                tot.trace_ms += e;
            }
        if (flags & VKB_PROFILE_TIME_KERNELS)
            for (uint32_t k = 0; k < tot.cache_launches; ++k) {
                float e = 0.f;
                VKB_CUDA(cudaEventElapsedTime(&e, c->cache_events[2 * k], c->cache_events[2 * k + 1]));
                tot.cache_ms += e;
            }
    }
};

// Run `jobs` to completion on the wavefront `w` and resolve each into its out_dev.
// w2 (non-null: overlapped waves): the second wavefront, used on c->stream2.
void run_engine(vkb_ctx* c, std::vector<EngineJob>& jobs, const WaveBuffers& w, size_t capacity, uint32_t flags, bool graphs, WaveTotals& tot,
                bool packed = false, const CacheLaunch* cache = nullptr, const WaveBuffers* w2 = nullptr) {
    WaveEngine eng(c, w, capacity, flags, graphs);
    eng.packed = packed;
    eng.cache = cache;
    for (auto& e : jobs) eng.add(e);
    if (w2) {
        eng.overlap = true;
        eng.w2 = *w2;
        VKB_CUDA(cudaMemsetAsync(w2->counters, 0, 16 * sizeof(uint32_t), c->stream));
        VKB_CUDA(cudaMemsetAsync(w2->err, 0, sizeof(uint32_t), c->stream));
        VKB_CUDA(cudaMemsetAsync(w2->work, 0, 8 * sizeof(unsigned long long), c->stream));
    }
    VKB_CUDA(cudaEventRecord(c->ev0, c->stream));
    if (w2) {
        // c->stream2 starts after everything queued so far (scene builds, cleared accumulators).
        VKB_CUDA(cudaEventRecord(c->fork_ev, c->stream));
        VKB_CUDA(cudaStreamWaitEvent(c->stream2, c->fork_ev, 0));
    }
    while (eng.step()) {}
    if (w2) {
        VKB_CUDA(cudaEventRecord(c->join_ev, c->stream2));
        VKB_CUDA(cudaStreamWaitEvent(c->stream, c->join_ev, 0));
    }
    VKB_CUDA(cudaEventRecord(c->ev1, c->stream));
    for (size_t k = 0; k < eng.jobs.size(); ++k) eng.resolve(k);
    VKB_CUDA(cudaEventSynchronize(c->ev1));
    float ms = 0.f;
    VKB_CUDA(cudaEventElapsedTime(&ms, c->ev0, c->ev1));
    eng.collect(ms);
    tot = eng.tot;
    for (size_t k = 0; k < jobs.size(); ++k) jobs[k] = eng.jobs[k];
}

void fill_stats(vkb_stats* stats, const WaveTotals& t, uint64_t paths, float build_ms) {
    if (!stats) return;
    std::memset(stats, 0, sizeof(*stats));
    stats->paths = paths;
    stats->extension_rays = t.counters[3];
    stats->shadow_rays = t.counters[4];
    stats->dropped_light_samples = t.counters[5];
    stats->dropped_path_samples = t.counters[6];
    stats->traversal_overflows = t.err;
    stats->render_ms = t.render_ms;
    stats->build_ms = build_ms;
    stats->trace_ms = t.trace_ms;
    stats->trace_launches = t.trace_launches;
    stats->kernel_launches = t.launches;
    stats->nodes_visited = t.work[0];
    stats->triangles_tested = t.work[1];
    stats->instances_entered = t.work[2];
    stats->shadow_nodes_visited = t.work[3];
    stats->shadow_triangles_tested = t.work[4];
    stats->blas_nodes_visited = t.work[5];
    stats->cache_ms = t.cache_ms;
    stats->cache_queries = t.work[7];
    stats->samples_skipped = t.counters[10];
}

// Render jobs with the context's own buffers (grown on demand).
void render_jobs(vkb_ctx* c, const std::vector<std::pair<vkb_scene*, vkb_profile>>& in, std::vector<vkb_output*>& outs, uint32_t flags,
                 uint32_t wave_samples_hint, WaveTotals& tot, uint64_t& paths, const CacheLaunch* cache = nullptr,
                 const std::vector<const vkb_camera*>* cams = nullptr) {
    cudaStream_t st = c->stream;
    auto camera_of = [&](size_t k) -> const vkb_camera& { return (cams && (*cams)[k]) ? *(*cams)[k] : in[k].first->camera; };
    size_t total_pixels = 0, max_pix = 0, ids_words = 0, staged = 0;
    for (size_t k = 0; k < in.size(); ++k) {
        const vkb_camera& cam = camera_of(k);
        size_t npix = size_t(cam.width) * cam.height;
        total_pixels += npix; max_pix = std::max(max_pix, npix);
        if (outs[k]->primary_ids) ids_words += 2 * npix;
        if (!outs[k]->on_device) staged += npix;
    }
    for (const auto& job : in)
        if ((job.first->blas8.p != nullptr) != (in[0].first->blas8.p != nullptr))
            throw ArgError{"the scenes of one batch share a BLAS format"};
    bool adaptive = false, guides = false;
    for (const auto& job : in) adaptive = adaptive || job.second.adaptive;
    for (size_t k = 0; k < in.size(); ++k) guides = guides || outs[k]->guide_albedo || outs[k]->guide_normal;
    if (guides && (in.size() != 1 || cache || adaptive))
        throw Unsupported{"denoiser guides render one job through vkb_render / vkb_render_view, without adaptive stopping"};
    if (adaptive) {
        // path.slang stops pixels sample by sample against their neighbours' previous
        // sample: one job, one sample per wave, the whole exposure in this call.
        const vkb_profile& pf = in[0].second;
        if (in.size() != 1 || cache) throw Unsupported{"adaptive stopping renders one job through vkb_render"};
        if (pf.first_sample != 0 || (pf.sample_count && pf.sample_count != pf.samples))
            throw Unsupported{"adaptive stopping renders a whole exposure (first_sample 0, every sample)"};
        wave_samples_hint = 1;
        c->ad_mean.alloc(max_pix); c->ad_m2.alloc(max_pix); c->ad_state.alloc(max_pix);
        VKB_CUDA(cudaMemsetAsync(c->ad_state.p, 0, max_pix * sizeof(uint32_t), st));
    }
    // Path slots per wave: the context's (autotuned) capacity for batches; for one job the
    // profile's samples per wave, else up to 64 Mi slots, but no more than the job's paths
    // (measured on 1080p, 64-spp flock frames with overlapped waves: 2 waves of 32 samples
    // 218.1 / 216.3 vs 4 of 16 215.8 / 214.2 M paths/s on two frame ranges; one wave of 64: 217.2).
    size_t capacity = c->wave_capacity;
    if (in.size() == 1) {
        const uint64_t job_paths = uint64_t(max_pix) * (in[0].second.sample_count ? in[0].second.sample_count
                                                                                   : in[0].second.samples - in[0].second.first_sample);
        capacity = wave_samples_hint ? max_pix * wave_samples_hint
                                     : size_t(std::min<uint64_t>(std::max<size_t>(capacity, SINGLE_JOB_WAVE_SLOTS), job_paths));
    }
    capacity = std::max(capacity, max_pix);
    c->wave.reserve(capacity, uint32_t(in.size()));
    for (const auto& job : in)
        if (job.first->env_w || job.first->em_tris) { c->wave.reserve_ext(std::max(capacity, c->wave.ray_o0.n)); break; }
    c->accum.alloc(std::max<size_t>(1, total_pixels));
    WaveBuffers wb = c->wave.view();
    if (guides) {
        c->guide_slots.alloc(2 * capacity);
        c->guide_accum.alloc(2 * max_pix);
        VKB_CUDA(cudaMemsetAsync(c->guide_accum.p, 0, 2 * max_pix * sizeof(float4), st));
        if (!outs[0]->on_device) c->guide_staging.alloc(2 * max_pix);
        wb.guide = c->guide_slots.p;
    }
    if (staged) c->staging.alloc(staged);
    if (ids_words) c->ids.alloc(ids_words);
    std::vector<EngineJob> jobs(in.size());
    size_t acc = 0, stg = 0, idw = 0;
    for (size_t k = 0; k < in.size(); ++k) {
        EngineJob& e = jobs[k];
        e.s = in[k].first; e.pf = in[k].second;
        if (cams && (*cams)[k]) { e.own_camera = true; e.camera = *(*cams)[k]; }
        e.npix = camera_of(k).width * camera_of(k).height;
        e.count = e.pf.sample_count ? e.pf.sample_count : e.pf.samples - e.pf.first_sample;
        e.accum = c->accum.p + acc; acc += e.npix;
        if (outs[k]->on_device) e.out_dev = reinterpret_cast<float4*>(outs[k]->rgba);
        else { e.out_dev = c->staging.p + stg; stg += e.npix; }
        if (outs[k]->primary_ids) { e.ids_dev = c->ids.p + idw; idw += 2 * size_t(e.npix); }
        if (adaptive) { e.ad_mean = c->ad_mean.p; e.ad_m2 = c->ad_m2.p; e.ad_state = c->ad_state.p; }
        if (guides) {
            e.guide_accum = c->guide_accum.p;
            if (outs[k]->on_device) {
                e.guide_albedo = reinterpret_cast<float4*>(outs[k]->guide_albedo);
                e.guide_normal = reinterpret_cast<float4*>(outs[k]->guide_normal);
            } else {
                e.guide_albedo = outs[k]->guide_albedo ? c->guide_staging.p : nullptr;
                e.guide_normal = outs[k]->guide_normal ? c->guide_staging.p + e.npix : nullptr;
            }
        }
        paths += uint64_t(e.npix) * e.count;
    }
    // Renders of more than one wave overlap their waves on two streams (not with the
    // adaptive, guide or radiance-cache hooks: adaptive stopping reads one wave's moments in the
    // next, the guide and cache hooks fill buffers shared by all waves).
    // Timed renders keep one stream too: an event pair around a kernel would also count the
    // other stream's kernels sharing the SMs.
    uint64_t all_paths = 0;
    bool any_ext = false;
    for (size_t k = 0; k < jobs.size(); ++k) {
        all_paths += uint64_t(jobs[k].npix) * jobs[k].count;
        any_ext = any_ext || in[k].first->env_w || in[k].first->em_tris;
    }
    const bool overlap = !adaptive && !guides && !cache && !(flags & (VKB_PROFILE_SERIAL_WAVES | VKB_PROFILE_TIME_KERNELS)) &&
                         all_paths > capacity;
    WaveBuffers wb2;
    if (overlap) {
        c->wave2.reserve(capacity, uint32_t(in.size()));
        if (any_ext) c->wave2.reserve_ext(std::max(capacity, c->wave2.ray_o0.n));
        wb2 = c->wave2.view();
    }
    run_engine(c, jobs, wb, capacity, flags, true, tot, (flags & VKB_BATCH_FAIR) == 0, cache, overlap ? &wb2 : nullptr);
    for (size_t k = 0; k < in.size(); ++k) {
        if (guides && !outs[k]->on_device) {
            const size_t bytes = size_t(jobs[k].npix) * sizeof(float4);
            if (outs[k]->guide_albedo) VKB_CUDA(cudaMemcpyAsync(outs[k]->guide_albedo, jobs[k].guide_albedo, bytes, cudaMemcpyDeviceToHost, st));
            if (outs[k]->guide_normal) VKB_CUDA(cudaMemcpyAsync(outs[k]->guide_normal, jobs[k].guide_normal, bytes, cudaMemcpyDeviceToHost, st));
        }
        if (!outs[k]->on_device) VKB_CUDA(cudaMemcpyAsync(outs[k]->rgba, jobs[k].out_dev, size_t(jobs[k].npix) * sizeof(float4), cudaMemcpyDeviceToHost, st));
        if (outs[k]->primary_ids) VKB_CUDA(cudaMemcpyAsync(outs[k]->primary_ids, jobs[k].ids_dev, size_t(jobs[k].npix) * 2 * sizeof(uint32_t), cudaMemcpyDeviceToHost, st));
    }
    VKB_CUDA(cudaStreamSynchronize(st));
    c->launches += tot.launches;
}
}  // namespace

extern "C" {

uint32_t vkb_abi_version(void) { return VKB_ABI_VERSION; }
const char* vkb_last_error(void) { return g_error.c_str(); }

vkb_status vkb_open(int device, vkb_ctx** out) {
    if (!out) return fail(VKB_INVALID_ARG, "null output pointer");
    *out = nullptr;
    vkb_ctx* c = new vkb_ctx();
    vkb_status st = guarded([&] {
        c->device = device;
        VKB_CUDA(cudaSetDevice(device));
        VKB_CUDA(cudaDeviceGetAttribute(&c->sms, cudaDevAttrMultiProcessorCount, device));
        VKB_CUDA(cudaStreamCreateWithFlags(&c->stream, cudaStreamNonBlocking));
        VKB_CUDA(cudaStreamCreateWithFlags(&c->stream2, cudaStreamNonBlocking));
        VKB_CUDA(cudaEventCreate(&c->ev0));
        VKB_CUDA(cudaEventCreate(&c->ev1));
        VKB_CUDA(cudaEventCreateWithFlags(&c->fork_ev, cudaEventDisableTiming));
        VKB_CUDA(cudaEventCreateWithFlags(&c->join_ev, cudaEventDisableTiming));
        VKB_CUDA(cudaEventCreateWithFlags(&c->acc_ev[0], cudaEventDisableTiming));
        VKB_CUDA(cudaEventCreateWithFlags(&c->acc_ev[1], cudaEventDisableTiming));
        c->lut.alloc(size_t(BRDF_SIZE) * BRDF_HEIGHT);
        k_bake_lut<<<dim3(1, BRDF_HEIGHT), BRDF_SIZE, 0, c->stream>>>(c->lut.p);
        VKB_CUDA(cudaGetLastError());
        std::vector<float> ft = film_table();
        c->filter.upload(ft.data(), ft.size(), c->stream);
        VKB_CUDA(cudaStreamSynchronize(c->stream));
    });
    if (st != VKB_OK) { delete c; return st; }
    *out = c;
    return VKB_OK;
}

vkb_status vkb_close(vkb_ctx* c) {
    if (!c) return VKB_OK;
    cudaSetDevice(c->device);
    if (c->stream) cudaStreamSynchronize(c->stream);
    if (c->stream2) cudaStreamSynchronize(c->stream2);
    for (cudaEvent_t e : {c->fork_ev, c->join_ev, c->acc_ev[0], c->acc_ev[1]})
        if (e) cudaEventDestroy(e);
    for (cudaEvent_t e : c->kernel_events) cudaEventDestroy(e);
    for (cudaEvent_t e : c->cache_events) cudaEventDestroy(e);
    if (c->ev0) cudaEventDestroy(c->ev0);
    if (c->ev1) cudaEventDestroy(c->ev1);
    c->wave.release();
    c->wave2.release();
    c->accum.release(); c->staging.release(); c->ids.release(); c->ad_mean.release(); c->ad_m2.release(); c->ad_state.release();
    c->guide_slots.release(); c->guide_accum.release(); c->guide_staging.release();
    c->lut.release(); c->filter.release();
    if (c->stream) cudaStreamDestroy(c->stream);
    if (c->stream2) cudaStreamDestroy(c->stream2);
    delete c;
    return VKB_OK;
}

// Every mesh's BLAS on the GPU with the TLAS's builders (Morton order, then Karras LBVH or
// PLOC), its leaf references in the BLAS encoding, collapsed to 4-wide nodes indexed like
// the binary nodes (even depths used), and the triangles and normals in leaf order.
void build_blas_gpu(vkb_scene* s, uint32_t builder, cudaStream_t st) {
    const int sms = s->ctx->sms;
    uint32_t total = 0, max_tris = 1;
    for (auto& mi : s->mesh_info) {
        mi.node_offset = total;
        total += mi.num_triangles > 1 ? mi.num_triangles - 1 : 1u;
        max_tris = std::max(max_tris, mi.num_triangles);
    }
    s->blas4.alloc(std::max(1u, total));
    s->tri_nrm.alloc(std::max<size_t>(1, size_t(s->total_tris) * 3));
    DBuf<BvhNode> bin;
    DBuf<uint8_t> odd;
    DBuf<uint32_t> leaf_parent, node_parent, counters;
    bin.alloc(max_tris); odd.alloc(max_tris);
    if (builder == VKB_BLAS_BUILD_PLOC) { leaf_parent.alloc(max_tris); node_parent.alloc(max_tris); counters.alloc(max_tris); }
    // Every scratch buffer at the largest mesh's size before the first launch: growing one
    // between meshes would free memory that the previous mesh's kernels, still queued on
    // this non-blocking stream, read.
    s->scratch.reserve(max_tris, st);
    if (builder == VKB_BLAS_BUILD_PLOC) s->ploc.reserve(max_tris, st);
    VKB_CUDA(cudaStreamSynchronize(st));
    for (const MeshInfo& mi : s->mesh_info) {
        const uint32_t n = mi.num_triangles;
        if (n == 0) continue;
        const uint32_t* idx = s->indices.p + mi.index_offset;
        k_tri_boxes<<<grid_for(n, 256, sms), 256, 0, st>>>(n, idx, s->vpos.p + mi.vertex_offset, s->tri_lo.p, s->tri_hi.p);
        const uint32_t* parents = s->scratch.node_parent.p;
        if (builder == VKB_BLAS_BUILD_PLOC && n > 1) {
            morton_sort(n, s->tri_lo.p, s->tri_hi.p, s->scratch, st, sms, s->launches);
            build_ploc(n, s->tri_lo.p, s->tri_hi.p, bin.p, leaf_parent.p, node_parent.p, counters.p, s->scratch, s->ploc, st, sms, s->launches);
            parents = node_parent.p;
        } else {
            build_lbvh(n, s->tri_lo.p, s->tri_hi.p, bin.p, s->scratch, st, sms, s->launches);
        }
        const uint32_t ni = n > 1 ? n - 1 : 1u;
        k_blas_leaf_refs<<<grid_for(ni, 256, sms), 256, 0, st>>>(ni, bin.p);
        if (n > 1) k_bvh_parity<<<grid_for(ni, 256, sms), 256, 0, st>>>(ni, parents, odd.p);
        else VKB_CUDA(cudaMemsetAsync(odd.p, 0, 1, st));
        k_collapse4<<<grid_for(ni, 256, sms), 256, 0, st>>>(ni, bin.p, odd.p, s->blas4.p + mi.node_offset);
        k_sorted_tris<<<grid_for(n, 256, sms), 256, 0, st>>>(n, s->scratch.ids_sorted.p, idx, s->vpos.p + mi.vertex_offset,
                                                             s->blas_tris.p + 3 * size_t(mi.tri_offset));
        k_sorted_nrm<<<grid_for(n, 256, sms), 256, 0, st>>>(n, s->scratch.ids_sorted.p, idx, s->vnrm.p + mi.vertex_offset,
                                                            s->tri_nrm.p + 3 * size_t(mi.tri_offset));
        s->launches += 6;
        VKB_CUDA(cudaGetLastError());
    }
    VKB_CUDA(cudaStreamSynchronize(st));
    bin.release(); odd.release(); leaf_parent.release(); node_parent.release(); counters.release();
}

vkb_status vkb_scene_create(vkb_ctx* ctx, const vkb_scene_desc* d, vkb_scene** out) {
    if (!ctx || !out) return fail(VKB_INVALID_ARG, "null context or output pointer");
    *out = nullptr;
    vkb_scene* s = new vkb_scene();
    s->ctx = ctx;
    const auto t_start = std::chrono::steady_clock::now();
    double blas_host = 0.0;
    vkb_status st = guarded([&] {
        validate_desc(d);
        VKB_CUDA(cudaSetDevice(ctx->device));
        cudaStream_t str = ctx->stream;
        int sms = ctx->sms;
        VKB_CUDA(cudaEventCreate(&s->ev0));
        VKB_CUDA(cudaEventCreate(&s->ev1));
        s->num_meshes = d->num_meshes;
        s->num_instances = d->num_instances;
        s->tlas_builder = d->tlas_builder;
        s->blas_format = d->blas_format;
        s->blas_builder = d->blas_builder;
        const bool wide8 = s->blas_format == VKB_BLAS_WIDE8;
        // Concatenate meshes.
        uint32_t nv = 0, nt = 0;
        s->mesh_info.resize(d->num_meshes);
        for (uint32_t m = 0; m < d->num_meshes; ++m) {
            MeshInfo& mi = s->mesh_info[m];
            std::memset(&mi, 0, sizeof(mi));
            mi.vertex_offset = nv; mi.index_offset = 3u * nt; mi.tri_offset = nt; mi.num_triangles = d->meshes[m].num_triangles;
            float lo[3] = {INFINITY, INFINITY, INFINITY}, hi[3] = {-INFINITY, -INFINITY, -INFINITY};
            for (uint32_t i = 0; i < d->meshes[m].num_vertices; ++i)
                for (int a = 0; a < 3; ++a) { lo[a] = std::min(lo[a], d->meshes[m].positions[3 * i + a]); hi[a] = std::max(hi[a], d->meshes[m].positions[3 * i + a]); }
            for (int a = 0; a < 3; ++a) { mi.lo[a] = lo[a]; mi.hi[a] = hi[a]; }
            mesh_sphere(d->meshes[m].positions, d->meshes[m].num_vertices, lo, hi, mi.sphere);
            nv += d->meshes[m].num_vertices; nt += d->meshes[m].num_triangles;
        }
        s->total_tris = nt;
        std::vector<float4> pos(nv), nrm(nv);
        std::vector<uint32_t> idx(size_t(nt) * 3);
        for (uint32_t m = 0; m < d->num_meshes; ++m) {
            const vkb_mesh& me = d->meshes[m];
            const MeshInfo& mi = s->mesh_info[m];
            for (uint32_t i = 0; i < me.num_vertices; ++i) {
                pos[mi.vertex_offset + i] = make_float4(me.positions[3 * i], me.positions[3 * i + 1], me.positions[3 * i + 2], 0.f);
                nrm[mi.vertex_offset + i] = me.normals ? make_float4(me.normals[3 * i], me.normals[3 * i + 1], me.normals[3 * i + 2], 0.f) : make_float4(0.f, 0.f, 0.f, 0.f);
            }
            std::copy(me.indices, me.indices + size_t(me.num_triangles) * 3, idx.begin() + mi.index_offset);
        }
        s->vpos.upload(pos.data(), pos.size(), str);
        s->vnrm.upload(nrm.data(), nrm.size(), str);
        s->indices.upload(idx.data(), idx.size(), str);
        // BLAS per mesh: binary SAH tree, collapsed to 4-wide nodes (mesh node_offset into those).
        s->blas_tris.alloc(std::max<size_t>(1, size_t(nt) * 3));
        uint32_t max_tris = 0;
        for (auto& mi : s->mesh_info) max_tris = std::max(max_tris, mi.num_triangles);
        s->tri_lo.alloc(std::max(1u, max_tris)); s->tri_hi.alloc(std::max(1u, max_tris));
        VKB_CUDA(cudaEventRecord(s->ev0, str));
        const auto t_blas = std::chrono::steady_clock::now();
        if (s->blas_builder != VKB_BLAS_BUILD_SAH) {
            build_blas_gpu(s, s->blas_builder, str);
        } else {
            std::vector<Bvh4Node> all_nodes;
            std::vector<Bvh8Node> all_nodes8;
            std::vector<float4> all_tris(std::max<size_t>(1, size_t(nt) * 3)), all_nrm(std::max<size_t>(1, size_t(nt) * 3));
            for (uint32_t m = 0; m < d->num_meshes; ++m) {
                MeshInfo& mi = s->mesh_info[m];
                const vkb_mesh& me = d->meshes[m];
                uint32_t n = mi.num_triangles;
                mi.node_offset = uint32_t(wide8 ? all_nodes8.size() : all_nodes.size());
                if (n == 0) continue;
                std::vector<float> lo(3 * size_t(n)), hi(3 * size_t(n)), cen(3 * size_t(n));
                for (uint32_t t = 0; t < n; ++t)
                    for (int a = 0; a < 3; ++a) {
                        float v0 = me.positions[3 * me.indices[3 * t] + a], v1 = me.positions[3 * me.indices[3 * t + 1] + a], v2 = me.positions[3 * me.indices[3 * t + 2] + a];
                        lo[3 * t + a] = std::min(v0, std::min(v1, v2)); hi[3 * t + a] = std::max(v0, std::max(v1, v2));
                        cen[3 * t + a] = 0.5f * (lo[3 * t + a] + hi[3 * t + a]);
                    }
                vkb_host::SahBlas sah;
                sah.run(n, lo.data(), hi.data(), cen.data());
                if (sah.nodes.size() > std::max(1u, n > 1 ? n - 1 : 1u)) throw ArgError{"BLAS node count above its bound"};
                static_assert(sizeof(vkb_host::SahNode) == sizeof(BvhNode), "host SAH nodes have the device layout");
                // Leaf position k of this mesh's BLAS -> its original triangle.
                std::vector<uint32_t> leaf_tri(sah.order);
                if (wide8) {
                    static_assert(sizeof(vkb_host::Wide8Node) == sizeof(Bvh8Node), "host 8-wide nodes have the device layout");
                    vkb_host::Wide8Blas w8;
                    w8.run(sah.nodes, n);
                    if (all_nodes8.size() + w8.nodes.size() > size_t(INT32_MAX)) throw ArgError{"BLAS node count above its bound"};
                    const size_t at = all_nodes8.size();
                    all_nodes8.resize(at + w8.nodes.size());
                    std::memcpy(all_nodes8.data() + at, w8.nodes.data(), w8.nodes.size() * sizeof(Bvh8Node));
                    for (uint32_t k = 0; k < n; ++k) leaf_tri[k] = sah.order[w8.order[k]];
                } else {
                    std::vector<BvhNode> bin(sah.nodes.size());
                    std::memcpy(bin.data(), sah.nodes.data(), bin.size() * sizeof(BvhNode));
                    std::vector<Bvh4Node> wide = collapse_blas(bin);
                    if (all_nodes.size() + wide.size() > size_t(INT32_MAX)) throw ArgError{"BLAS node count above its bound"};
                    all_nodes.insert(all_nodes.end(), wide.begin(), wide.end());
                }
                for (uint32_t k = 0; k < n; ++k) {
                    uint32_t t = leaf_tri[k];
                    const float* p0 = me.positions + 3 * me.indices[3 * t];
                    const float* p1 = me.positions + 3 * me.indices[3 * t + 1];
                    const float* p2 = me.positions + 3 * me.indices[3 * t + 2];
                    size_t o = 3 * (size_t(mi.tri_offset) + k);
                    float tid;
                    std::memcpy(&tid, &t, sizeof(tid));
                    all_tris[o] = make_float4(p0[0], p0[1], p0[2], tid);
                    all_tris[o + 1] = make_float4(p1[0], p1[1], p1[2], 0.f);
                    all_tris[o + 2] = make_float4(p2[0], p2[1], p2[2], 0.f);
                    for (int c = 0; c < 3; ++c) {
                        const float* nv = me.normals ? me.normals + 3 * me.indices[3 * t + c] : nullptr;
                        all_nrm[o + c] = nv ? make_float4(nv[0], nv[1], nv[2], 0.f) : make_float4(0.f, 0.f, 0.f, 0.f);
                    }
                }
            }
            if (all_nodes.empty()) all_nodes.emplace_back();
            if (wide8) {
                if (all_nodes8.empty()) all_nodes8.emplace_back();
                s->blas8.upload(all_nodes8.data(), all_nodes8.size(), str);
            }
            blas_host = std::chrono::duration<double, std::milli>(std::chrono::steady_clock::now() - t_blas).count();
            s->blas4.alloc(all_nodes.size());
            VKB_CUDA(cudaMemcpyAsync(s->blas4.p, all_nodes.data(), all_nodes.size() * sizeof(Bvh4Node), cudaMemcpyHostToDevice, str));
            VKB_CUDA(cudaMemcpyAsync(s->blas_tris.p, all_tris.data(), all_tris.size() * sizeof(float4), cudaMemcpyHostToDevice, str));
            s->tri_nrm.upload(all_nrm.data(), all_nrm.size(), str);
        }
        VKB_CUDA(cudaStreamSynchronize(str));
        VKB_CUDA(cudaEventRecord(s->ev1, str));
        s->meshes.upload(s->mesh_info.data(), s->mesh_info.size(), str);
        // Materials, lights, light tree.
        s->materials.assign(d->materials, d->materials + d->num_materials);
        s->lights.assign(d->lights, d->lights + d->num_lights);
        s->d_materials.upload(s->materials.data(), s->materials.size(), str);
        s->d_lights.upload(s->lights.data(), std::max<size_t>(s->lights.size(), 0), str);
        std::vector<LightTreeNode> tree = light_tree(d->lights, d->num_lights);
        s->tree_nodes = uint32_t(tree.size());
        s->tree.upload(tree.data(), tree.size(), str);
        s->camera = d->camera;
        s->env = d->environment;
        if (const vkb_environment_image* e = d->environment_image) {
            if (e->strength > 0.f) {
                s->env_w = e->width; s->env_h = e->height;
                for (int c = 0; c < 3; ++c) s->env_scale[c] = e->strength * e->color[c];
                bool any = false;
                for (int k = 0; k < 9; ++k) any = any || e->rotation[k] != 0.f;
                if (any) for (int k = 0; k < 9; ++k) s->env_rot[k] = e->rotation[k];
                s->env_img.upload(reinterpret_cast<const float4*>(e->rgba), size_t(e->width) * e->height, str);
                std::vector<float2> dist = env_proposal(e->rgba, e->width, e->height);
                s->env_dist.upload(dist.data(), dist.size(), str);
                VKB_CUDA(cudaStreamSynchronize(str));
            }
        }
        // Instances + TLAS.
        uint32_t n = d->num_instances;
        s->inst_mesh.assign(d->instance_mesh, d->instance_mesh + n);
        s->inst_mat.assign(d->instance_material, d->instance_material + n);
        std::vector<uint4> info(n);
        for (uint32_t i = 0; i < n; ++i) info[i] = make_uint4(d->instance_mesh[i], d->instance_material[i], 0u, 0u);
        s->inst_info.upload(info.data(), n, str);
        s->o2w.upload(reinterpret_cast<const float4*>(d->instance_rows), size_t(n) * 3, str);
        s->w2o.alloc(size_t(n) * 3);
        s->inst_lo.alloc(n); s->inst_hi.alloc(n);
        s->tlas_nodes.alloc(std::max(1u, n > 1 ? n - 1 : 1u));
        s->tlas4.alloc(std::max(1u, n > 1 ? n - 1 : 1u));
        s->tlas_odd.alloc(std::max(1u, n > 1 ? n - 1 : 1u));
        s->tlas_leaves.alloc(std::max(1u, n));
        s->tlas_codes.alloc(std::max(1u, n));
        emitter_topology(s, str);
        VKB_CUDA(cudaStreamSynchronize(str));
        float blas_ms = 0.f;
        VKB_CUDA(cudaEventElapsedTime(&blas_ms, s->ev0, s->ev1));
        build_tlas(s);
        s->tlas_ms = s->build_ms;
        s->build_ms += blas_ms;
        s->install_ms = float(std::chrono::duration<double, std::milli>(std::chrono::steady_clock::now() - t_start).count());
        s->blas_host_ms = float(blas_host);
        s->upload_ms = std::max(0.f, s->install_ms - s->blas_host_ms - s->tlas_ms);
    });
    if (st != VKB_OK) { vkb_scene_destroy(s); return st; }
    *out = s;
    return VKB_OK;
}

vkb_status vkb_scene_fork(vkb_scene* b, vkb_scene** out) {
    if (!b || !out) return fail(VKB_INVALID_ARG, "null scene or output pointer");
    if (b->base) return fail(VKB_INVALID_ARG, "fork of a fork: fork the base scene");
    *out = nullptr;
    vkb_scene* s = new vkb_scene();
    s->ctx = b->ctx;
    const auto t_start = std::chrono::steady_clock::now();
    vkb_status st = guarded([&] {
        VKB_CUDA(cudaSetDevice(b->ctx->device));
        cudaStream_t str = b->ctx->stream;
        VKB_CUDA(cudaEventCreate(&s->ev0));
        VKB_CUDA(cudaEventCreate(&s->ev1));
        s->num_meshes = b->num_meshes; s->num_instances = b->num_instances; s->total_tris = b->total_tris;
        s->mesh_info = b->mesh_info; s->inst_mesh = b->inst_mesh; s->inst_mat = b->inst_mat;
        s->materials = b->materials; s->lights = b->lights; s->camera = b->camera; s->env = b->env;
        s->tree_nodes = b->tree_nodes; s->tlas_builder = b->tlas_builder;
        // Shared, read-only: geometry, BLASes, materials, lights, light tree.
        s->vpos = b->vpos; s->vnrm = b->vnrm; s->blas_tris = b->blas_tris; s->tri_nrm = b->tri_nrm;
        s->indices = b->indices; s->meshes = b->meshes; s->blas4 = b->blas4; s->blas8 = b->blas8; s->blas_format = b->blas_format; s->blas_builder = b->blas_builder;
        s->d_materials = b->d_materials; s->d_lights = b->d_lights; s->tree = b->tree;
        s->env_img = b->env_img; s->env_dist = b->env_dist; s->env_w = b->env_w; s->env_h = b->env_h;
        std::copy(b->env_scale, b->env_scale + 3, s->env_scale); std::copy(b->env_rot, b->env_rot + 9, s->env_rot);
        s->em_inst_source = b->em_inst_source; s->em_sources = b->em_sources;
        s->em_count = b->em_count; s->em_tris = b->em_tris; s->em_leaves = b->em_leaves;
        if (s->em_leaves) s->em_tree.alloc(2 * size_t(s->em_leaves));
        s->base = b;
        b->forks++;
        // Owned: the base's current instance rows and records, and a TLAS over them.
        uint32_t n = b->num_instances;
        s->inst_info.alloc(std::max(1u, n));
        s->o2w.alloc(std::max<size_t>(1, size_t(n) * 3));
        if (n) {
            VKB_CUDA(cudaMemcpyAsync(s->inst_info.p, b->inst_info.p, n * sizeof(uint4), cudaMemcpyDeviceToDevice, str));
            VKB_CUDA(cudaMemcpyAsync(s->o2w.p, b->o2w.p, size_t(n) * 3 * sizeof(float4), cudaMemcpyDeviceToDevice, str));
        }
        s->w2o.alloc(std::max<size_t>(1, size_t(n) * 3));
        s->inst_lo.alloc(std::max(1u, n)); s->inst_hi.alloc(std::max(1u, n));
        s->tlas_nodes.alloc(std::max(1u, n > 1 ? n - 1 : 1u));
        s->tlas4.alloc(std::max(1u, n > 1 ? n - 1 : 1u));
        s->tlas_odd.alloc(std::max(1u, n > 1 ? n - 1 : 1u));
        s->tlas_leaves.alloc(std::max(1u, n));
        s->tlas_codes.alloc(std::max(1u, n));
        build_tlas(s);
        s->tlas_ms = s->build_ms;
        s->install_ms = float(std::chrono::duration<double, std::milli>(std::chrono::steady_clock::now() - t_start).count());
        s->upload_ms = std::max(0.f, s->install_ms - s->tlas_ms);
    });
    if (st != VKB_OK) { vkb_scene_destroy(s); return st; }
    *out = s;
    return VKB_OK;
}

vkb_status vkb_scene_destroy(vkb_scene* s) {
    if (!s) return VKB_OK;
    if (s->forks) return fail(VKB_INVALID_ARG, "scene has live forks: destroy them first");
    cudaSetDevice(s->ctx->device);
    cudaStreamSynchronize(s->ctx->stream);
    cudaStreamSynchronize(s->ctx->stream2);
    if (s->base) {
        // Shared with the base scene: not this fork's to free.
        DBuf<float4>* shared4[] = {&s->vpos, &s->vnrm, &s->blas_tris, &s->tri_nrm};
        for (auto* b : shared4) { b->p = nullptr; b->n = 0; }
        s->indices.p = nullptr; s->indices.n = 0;
        s->meshes.p = nullptr; s->meshes.n = 0;
        s->blas4.p = nullptr; s->blas4.n = 0;
        s->blas8.p = nullptr; s->blas8.n = 0;
        s->d_materials.p = nullptr; s->d_materials.n = 0;
        s->d_lights.p = nullptr; s->d_lights.n = 0;
        s->tree.p = nullptr; s->tree.n = 0;
        s->env_img.p = nullptr; s->env_img.n = 0;
        s->env_dist.p = nullptr; s->env_dist.n = 0;
        s->em_inst_source.p = nullptr; s->em_inst_source.n = 0;
        s->em_sources.p = nullptr; s->em_sources.n = 0;
        s->base->forks--;
    }
    s->env_img.release(); s->env_dist.release();
    s->em_inst_source.release(); s->em_sources.release(); s->em_tree.release();
    DBuf<float4>* f4[] = {&s->vpos, &s->vnrm, &s->blas_tris, &s->tri_nrm, &s->o2w, &s->o2w_next, &s->w2o, &s->inst_lo, &s->inst_hi, &s->tri_lo, &s->tri_hi};
    for (auto* b : f4) b->release();
    s->changed.release();
    s->indices.release(); s->tlas_codes.release();
    s->tlas_order.release(); s->tlas_leaf_parent.release(); s->tlas_node_parent.release(); s->tlas_counters.release(); s->inst_info.release(); s->meshes.release();
    s->blas4.release(); s->blas8.release(); s->tlas4.release(); s->tlas_odd.release(); s->tlas_nodes.release(); s->tlas_leaves.release(); s->d_materials.release(); s->d_lights.release();
    s->tree.release();
    s->scratch.codes.release(); s->scratch.codes_sorted.release(); s->scratch.ids.release(); s->scratch.ids_sorted.release();
    s->scratch.leaf_parent.release(); s->scratch.node_parent.release(); s->scratch.counters.release(); s->scratch.bounds.release(); s->scratch.cub_temp.release();
    DBuf<float4>* pf4[] = {&s->ploc.clo, &s->ploc.chi, &s->ploc.clo2, &s->ploc.chi2};
    for (auto* b : pf4) b->release();
    s->ploc.nn.release(); s->ploc.counts.release(); s->ploc.flags.release(); s->ploc.offs.release(); s->ploc.cub_temp.release();
    if (s->ev0) cudaEventDestroy(s->ev0);
    if (s->ev1) cudaEventDestroy(s->ev1);
    delete s;
    return VKB_OK;
}

vkb_status vkb_scene_update_instances(vkb_scene* s, const float* rows, uint32_t n, int policy) {
    if (!s || !rows) return fail(VKB_INVALID_ARG, "null scene or rows");
    if (n != s->num_instances) return fail(VKB_INVALID_ARG, "instance count differs from the installed scene");
    if (policy < 0 || policy > 2) return fail(VKB_INVALID_ARG, "policy must be 0, 1 or 2");
    return guarded([&] {
        VKB_CUDA(cudaSetDevice(s->ctx->device));
        after_second_stream(s->ctx);
        // Changed bytes: rows that differ from the installed ones, counted on the device
        // (the new rows go up once; only the count comes back).
        cudaStream_t st = s->ctx->stream;
        s->o2w_next.alloc(size_t(n) * 3);
        s->changed.alloc(1);
        VKB_CUDA(cudaMemcpyAsync(s->o2w_next.p, rows, size_t(n) * 3 * sizeof(float4), cudaMemcpyHostToDevice, st));
        VKB_CUDA(cudaMemsetAsync(s->changed.p, 0, sizeof(unsigned long long), st));
        k_changed_rows<<<grid_for(n, 256, s->ctx->sms), 256, 0, st>>>(n, reinterpret_cast<const uint4*>(s->o2w_next.p),
                                                                      reinterpret_cast<const uint4*>(s->o2w.p), s->changed.p);
        s->launches += 1;
        unsigned long long changed = 0;
        VKB_CUDA(cudaMemcpyAsync(&changed, s->changed.p, sizeof(changed), cudaMemcpyDeviceToHost, st));
        VKB_CUDA(cudaStreamSynchronize(st));
        if (changed == 0 && policy == 0) return;
        VKB_CUDA(cudaMemcpyAsync(s->o2w.p, s->o2w_next.p, size_t(n) * 3 * sizeof(float4), cudaMemcpyDeviceToDevice, st));
        update_tlas(s, changed, policy);
    });
}

vkb_status vkb_scene_update_instances_device(vkb_scene* s, const float* rows, uint32_t n, int policy) {
    if (!s || !rows) return fail(VKB_INVALID_ARG, "null scene or rows");
    if (n != s->num_instances) return fail(VKB_INVALID_ARG, "instance count differs from the installed scene");
    if (policy < 0 || policy > 2) return fail(VKB_INVALID_ARG, "policy must be 0, 1 or 2");
    return guarded([&] {
        VKB_CUDA(cudaSetDevice(s->ctx->device));
        after_second_stream(s->ctx);
        VKB_CUDA(cudaMemcpyAsync(s->o2w.p, rows, size_t(n) * 3 * sizeof(float4), cudaMemcpyDeviceToDevice, s->ctx->stream));
        // device rows: every row counts as changed
        update_tlas(s, uint64_t(n) * 48u, policy);
    });
}

vkb_status vkb_render(vkb_scene* s, const vkb_profile* pf, vkb_output* out, vkb_stats* stats) {
    if (!s || !pf || !out || !out->rgba) return fail(VKB_INVALID_ARG, "null scene, profile or output");
    return guarded([&] {
        validate_profile(pf);
        vkb_ctx* c = s->ctx;
        VKB_CUDA(cudaSetDevice(c->device));
        std::vector<std::pair<vkb_scene*, vkb_profile>> in{{s, *pf}};
        std::vector<vkb_output*> outs{out};
        WaveTotals tot;
        uint64_t paths = 0;
        uint32_t hint = pf->wave_samples;
        if (!hint) {
            uint32_t count = pf->sample_count ? pf->sample_count : pf->samples - pf->first_sample;
            size_t npix = size_t(s->camera.width) * s->camera.height;
            hint = uint32_t(std::max<size_t>(1, std::min<size_t>(count, std::max(c->wave_capacity, SINGLE_JOB_WAVE_SLOTS) / std::max<size_t>(1, npix))));
        }
        render_jobs(c, in, outs, pf->flags, hint, tot, paths);
        s->launches += tot.launches;
        fill_stats(stats, tot, paths, s->build_ms);
    });
}

vkb_status vkb_render_view(vkb_scene* s, const vkb_camera* cam, const vkb_profile* pf, vkb_output* out, vkb_stats* stats) {
    if (!cam) return vkb_render(s, pf, out, stats);
    if (!s || !pf || !out || !out->rgba) return fail(VKB_INVALID_ARG, "null scene, profile or output");
    return guarded([&] {
        validate_profile(pf);
        validate_camera(*cam);
        vkb_ctx* c = s->ctx;
        VKB_CUDA(cudaSetDevice(c->device));
        std::vector<std::pair<vkb_scene*, vkb_profile>> in{{s, *pf}};
        std::vector<vkb_output*> outs{out};
        std::vector<const vkb_camera*> cams{cam};
        WaveTotals tot;
        uint64_t paths = 0;
        uint32_t hint = pf->wave_samples;
        if (!hint) {
            uint32_t count = pf->sample_count ? pf->sample_count : pf->samples - pf->first_sample;
            size_t npix = size_t(cam->width) * cam->height;
            hint = uint32_t(std::max<size_t>(1, std::min<size_t>(count, std::max(c->wave_capacity, SINGLE_JOB_WAVE_SLOTS) / std::max<size_t>(1, npix))));
        }
        render_jobs(c, in, outs, pf->flags, hint, tot, paths, nullptr, &cams);
        s->launches += tot.launches;
        fill_stats(stats, tot, paths, s->build_ms);
    });
}

vkb_status vkb_render_batch(vkb_ctx* c, vkb_job* jobs, uint32_t njobs, uint32_t flags, vkb_stats* stats) {
    if (!c || (njobs && !jobs)) return fail(VKB_INVALID_ARG, "null context or jobs");
    return guarded([&] {
        if (njobs == 0) { if (stats) std::memset(stats, 0, sizeof(*stats)); return; }
        VKB_CUDA(cudaSetDevice(c->device));
        std::vector<std::pair<vkb_scene*, vkb_profile>> in(njobs);
        std::vector<vkb_output*> outs(njobs);
        for (uint32_t k = 0; k < njobs; ++k) {
            if (!jobs[k].scene || !jobs[k].out.rgba) throw ArgError{"job " + std::to_string(k) + " has a null scene or output"};
            if (jobs[k].scene->ctx != c) throw ArgError{"job " + std::to_string(k) + " belongs to another context"};
            validate_profile(&jobs[k].profile);
            in[k] = {jobs[k].scene, jobs[k].profile};
            outs[k] = &jobs[k].out;
        }
        WaveTotals tot;
        uint64_t paths = 0;
        render_jobs(c, in, outs, flags, 0, tot, paths);
        fill_stats(stats, tot, paths, 0.f);
    });
}

vkb_status vkb_autotune(vkb_ctx* c, vkb_job* jobs, uint32_t njobs, vkb_tune_result* out) {
    if (!c || !jobs || njobs == 0) return fail(VKB_INVALID_ARG, "null context or no jobs");
    return guarded([&] {
        VKB_CUDA(cudaSetDevice(c->device));
        // Candidates: wave capacity (queue slots) x trace/shade blocks per SM, each timed on
        // one sample of every job (same work for every candidate).
        const size_t caps[] = {size_t(2) << 20, size_t(4) << 20, size_t(8) << 20, size_t(16) << 20, size_t(32) << 20};
        const int grids[] = {32, 64, 128};
        std::vector<std::pair<vkb_scene*, vkb_profile>> in(njobs);
        std::vector<vkb_output> o(njobs);
        std::vector<vkb_output*> outs(njobs);
        size_t max_pix = 0;
        for (uint32_t k = 0; k < njobs; ++k) {
            vkb_profile pf = jobs[k].profile;
            validate_profile(&pf);
            pf.sample_count = 1;
            pf.adaptive = 0;   // timing one sample of every job
            in[k] = {jobs[k].scene, pf};
            max_pix = std::max(max_pix, size_t(jobs[k].scene->camera.width) * jobs[k].scene->camera.height);
        }
        c->staging.alloc(1);
        size_t best_cap = c->wave_capacity;
        int best_grid = c->trace_blocks_per_sm;
        float best_ms = INFINITY;
        uint32_t tried = 0;
        for (size_t cap : caps)
            for (int g : grids) {
                c->wave_capacity = std::max(cap, max_pix);
                c->trace_blocks_per_sm = g;
                // Device outputs into the staging buffer region (results are discarded).
                size_t total = 0;
                for (uint32_t k = 0; k < njobs; ++k) total += size_t(in[k].first->camera.width) * in[k].first->camera.height;
                c->staging.alloc(total);
                size_t off = 0;
                for (uint32_t k = 0; k < njobs; ++k) {
                    o[k] = vkb_output{};
                    o[k].rgba = reinterpret_cast<float*>(c->staging.p + off);
                    o[k].on_device = 1;
                    outs[k] = &o[k];
                    off += size_t(in[k].first->camera.width) * in[k].first->camera.height;
                }
                WaveTotals warm, tot;
                uint64_t paths = 0;
                render_jobs(c, in, outs, 0, 0, warm, paths);  // warm-up: buffer sizes, caches
                render_jobs(c, in, outs, 0, 0, tot, paths);
                if (out && tried < 16) {
                    out->capacity[tried] = uint64_t(c->wave_capacity);
                    out->blocks_per_sm[tried] = uint32_t(g);
                    out->ms[tried] = tot.render_ms;
                }
                ++tried;
                if (tot.render_ms < best_ms) { best_ms = tot.render_ms; best_cap = c->wave_capacity; best_grid = g; }
            }
        c->wave_capacity = best_cap;
        c->trace_blocks_per_sm = best_grid;
        if (out) {
            out->tried = tried;
            out->best_capacity = uint64_t(best_cap);
            out->best_blocks_per_sm = uint32_t(best_grid);
            out->best_ms = best_ms;
        }
    });
}

vkb_status vkb_scene_info(vkb_scene* s, vkb_scene_info_t* out) {
    if (!s || !out) return fail(VKB_INVALID_ARG, "null argument");
    std::memset(out, 0, sizeof(*out));
    out->num_instances = s->num_instances;
    out->num_triangles = s->total_tris;
    out->tlas_rebuilds = s->tlas_rebuilds;
    out->tlas_refits = s->tlas_refits;
    out->motion_bytes = s->motion_bytes;
    size_t dev = 0;
    dev += s->vpos.n * sizeof(float4) + s->vnrm.n * sizeof(float4) + s->indices.n * 4 + s->blas4.n * sizeof(Bvh4Node) + s->blas8.n * sizeof(Bvh8Node) +
           (s->blas_tris.n + s->tri_nrm.n) * sizeof(float4);
    dev += s->tlas_nodes.n * sizeof(BvhNode) + s->tlas4.n * sizeof(Bvh4Node) + s->tlas_odd.n + s->tlas_leaves.n * sizeof(TlasLeaf) + (s->o2w.n + s->w2o.n) * sizeof(float4);
    dev += s->env_img.n * sizeof(float4) + s->env_dist.n * sizeof(float2) + s->em_inst_source.n * 4 + s->em_sources.n * sizeof(uint2) + s->em_tree.n * sizeof(float);
    out->scene_bytes = dev;
    out->build_ms = s->build_ms;
    out->install_ms = s->install_ms; out->blas_host_ms = s->blas_host_ms; out->upload_ms = s->upload_ms; out->tlas_ms = s->tlas_ms;
    return VKB_OK;
}

vkb_status vkb_display(vkb_ctx* c, const vkb_display_params* prm, const float* rgba, int rgba_on_device, uint32_t width, uint32_t height,
                       void* out, int out_on_device) {
    if (!c || !prm || !rgba || !out) return fail(VKB_INVALID_ARG, "null argument");
    if (prm->display > VKB_DISPLAY_REC2100_HLG) return fail(VKB_INVALID_ARG, "unknown display");
    if (prm->bits != 8 && prm->bits != 16 && prm->bits != 32) return fail(VKB_INVALID_ARG, "bits must be 8, 16 or 32");
    if (!(prm->gamma > 0.f) || !std::isfinite(prm->exposure)) return fail(VKB_INVALID_ARG, "gamma must be positive and exposure finite");
    if (prm->display >= VKB_DISPLAY_REC2100_PQ && !(prm->peak_luminance > 0.f && prm->reference_white > 0.f))
        return fail(VKB_INVALID_ARG, "Rec.2100 needs a positive peak luminance and reference white");
    uint32_t bad = 0;
    vkb_status st = guarded([&] {
        VKB_CUDA(cudaSetDevice(c->device));
        cudaStream_t s = c->stream;
        const size_t n = size_t(width) * height;
        if (n == 0) return;
        const size_t out_bytes = n * (prm->bits / 8u) * 4u;
        DBuf<float4> in;
        DBuf<unsigned char> o;
        DBuf<uint32_t> flag;
        const float4* src = reinterpret_cast<const float4*>(rgba);
        if (!rgba_on_device) { in.upload(reinterpret_cast<const float4*>(rgba), n, s); src = in.p; }
        void* dst = out;
        if (!out_on_device) { o.alloc(out_bytes); dst = o.p; }
        flag.alloc(1);
        VKB_CUDA(cudaMemsetAsync(flag.p, 0, sizeof(uint32_t), s));
        DisplayParams d;
        d.display = prm->display; d.bits = prm->bits; d.unassociate = prm->unassociate ? 1u : 0u;
        d.exposure_scale = std::exp2(prm->exposure); d.inv_gamma = 1.f / prm->gamma;
        d.peak = prm->peak_luminance > 0.f ? prm->peak_luminance : 1000.f;
        d.white = prm->reference_white > 0.f ? prm->reference_white : 100.f;
        const double rel = std::log2(double(d.peak) / 1000.0);
        d.hlg_gamma = float(d.peak >= 400.f && d.peak <= 2000.f ? 1.2 + .42 * .30102999566 * rel : 1.2 * std::pow(1.111, rel));
        k_display<<<grid_for(uint32_t(n), 256, c->sms), 256, 0, s>>>(uint32_t(n), src, d, dst, flag.p);
        VKB_CUDA(cudaGetLastError());
        if (!out_on_device) VKB_CUDA(cudaMemcpyAsync(out, o.p, out_bytes, cudaMemcpyDeviceToHost, s));
        VKB_CUDA(cudaMemcpyAsync(&bad, flag.p, sizeof(bad), cudaMemcpyDeviceToHost, s));
        VKB_CUDA(cudaStreamSynchronize(s));
        c->launches += 1;
    });
    if (st != VKB_OK) return st;
    if (bad) return fail(VKB_NONFINITE, "non-finite pixels were written as zero");
    return VKB_OK;
}

vkb_status vkb_debug_tlas_stats(vkb_scene* s, double* sah_cost, uint32_t* max_depth, uint32_t* valid) {
    if (!s || !sah_cost || !max_depth || !valid) return fail(VKB_INVALID_ARG, "null argument");
    return guarded([&] {
        VKB_CUDA(cudaSetDevice(s->ctx->device));
        VKB_CUDA(cudaStreamSynchronize(s->ctx->stream));
        const uint32_t n = s->num_instances;
        *sah_cost = 0.0; *max_depth = 0; *valid = 1;
        if (n == 0) return;
        const uint32_t nn = std::max(1u, n - 1);
        std::vector<BvhNode> nodes(nn);
        VKB_CUDA(cudaMemcpy(nodes.data(), s->tlas_nodes.p, nn * sizeof(BvhNode), cudaMemcpyDeviceToHost));
        auto area = [](const float lo[3], const float hi[3]) {
            double dx = double(hi[0]) - lo[0], dy = double(hi[1]) - lo[1], dz = double(hi[2]) - lo[2];
            return dx * dy + dy * dz + dz * dx;
        };
        struct Item { int ref; uint32_t depth; float lo[3], hi[3]; };
        auto child = [&](const BvhNode& b, int side, Item& it) {
            const float4 q = side ? b.b : b.a;
            it.lo[0] = q.x; it.hi[0] = q.y; it.lo[1] = q.z; it.hi[1] = q.w;
            it.lo[2] = side ? b.c.z : b.c.x; it.hi[2] = side ? b.c.w : b.c.y;
            it.ref = side ? b.d.y : b.d.x;
        };
        std::vector<uint8_t> seen_leaf(n, 0), seen_node(nn, 0);
        std::vector<Item> stack;
        Item root;
        root.ref = 0; root.depth = 0;
        for (int k = 0; k < 3; ++k) { root.lo[k] = INFINITY; root.hi[k] = -INFINITY; }
        {
            Item a, b;
            child(nodes[0], 0, a); child(nodes[0], 1, b);
            for (int k = 0; k < 3; ++k) { root.lo[k] = std::min(a.lo[k], n > 1 ? b.lo[k] : a.lo[k]); root.hi[k] = std::max(a.hi[k], n > 1 ? b.hi[k] : a.hi[k]); }
        }
        const double root_area = std::max(area(root.lo, root.hi), 1e-30);
        stack.push_back(root);
        double cost = 0.0;
        while (!stack.empty()) {
            Item it = stack.back(); stack.pop_back();
            *max_depth = std::max(*max_depth, it.depth);
            cost += area(it.lo, it.hi) / root_area;
            if (it.ref < 0) {
                uint32_t leaf = uint32_t(~it.ref);
                if (leaf >= n || seen_leaf[leaf]) { *valid = 0; continue; }
                seen_leaf[leaf] = 1;
                continue;
            }
            if (uint32_t(it.ref) >= nn || seen_node[it.ref] || it.depth > n) { *valid = 0; continue; }
            seen_node[it.ref] = 1;
            const BvhNode& b = nodes[it.ref];
            for (int side = 0; side < (n > 1 ? 2 : 1); ++side) {
                Item c;
                child(b, side, c);
                c.depth = it.depth + 1;
                for (int k = 0; k < 3; ++k)
                    if (!(c.lo[k] >= it.lo[k] && c.hi[k] <= it.hi[k])) *valid = 0;
                stack.push_back(c);
            }
        }
        for (uint32_t k = 0; k < n; ++k) if (!seen_leaf[k]) *valid = 0;
        *sah_cost = cost;
    });
}

void* vkb_ctx_stream(vkb_ctx* c) { return c ? reinterpret_cast<void*>(c->stream) : nullptr; }
uint64_t vkb_scene_launch_count(vkb_scene* s) { return s ? s->launches : 0; }

vkb_status vkb_debug_sampler_groups(vkb_ctx* c, uint32_t n, const uint32_t* px, const uint32_t* py, const uint32_t* index,
                                    const uint32_t* groups, uint32_t count, uint32_t stream, uint32_t* out_bits) {
    if (!c || (n && (!px || !py || !index || !groups || !out_bits))) return fail(VKB_INVALID_ARG, "null argument");
    return guarded([&] {
        VKB_CUDA(cudaSetDevice(c->device));
        DBuf<uint32_t> a, b, i, g;
        DBuf<uint4> o;
        a.upload(px, n, c->stream); b.upload(py, n, c->stream); i.upload(index, n, c->stream); g.upload(groups, n, c->stream);
        o.alloc(n);
        uint32_t mask = count <= 1 ? 0u : ((2u << (31 - __builtin_clz(count - 1u))) - 1u);
        if (n) k_sampler_groups<<<grid_for(n, 256, c->sms), 256, 0, c->stream>>>(n, a.p, b.p, i.p, g.p, mask, stream, o.p);
        if (n) VKB_CUDA(cudaMemcpyAsync(out_bits, o.p, size_t(n) * sizeof(uint4), cudaMemcpyDeviceToHost, c->stream));
        VKB_CUDA(cudaStreamSynchronize(c->stream));
        a.release(); b.release(); i.release(); g.release(); o.release();
    });
}

vkb_status vkb_debug_brdf_lut(vkb_ctx* c, float* out) {
    if (!c || !out) return fail(VKB_INVALID_ARG, "null argument");
    return guarded([&] {
        VKB_CUDA(cudaSetDevice(c->device));
        std::vector<ushort4> h(size_t(BRDF_SIZE) * BRDF_HEIGHT);
        VKB_CUDA(cudaMemcpyAsync(h.data(), c->lut.p, h.size() * sizeof(ushort4), cudaMemcpyDeviceToHost, c->stream));
        VKB_CUDA(cudaStreamSynchronize(c->stream));
        for (size_t i = 0; i < h.size(); ++i) {
            uint16_t v[4] = {h[i].x, h[i].y, h[i].z, h[i].w};
            for (int k = 0; k < 4; ++k) out[4 * i + k] = __half2float(__ushort_as_half(v[k]));
        }
    });
}

vkb_status vkb_debug_tlas_morton(vkb_scene* s, uint32_t* out) {
    if (!s || !out) return fail(VKB_INVALID_ARG, "null argument");
    return guarded([&] {
        VKB_CUDA(cudaSetDevice(s->ctx->device));
        if (s->num_instances) VKB_CUDA(cudaMemcpyAsync(out, s->tlas_codes.p, s->num_instances * sizeof(uint32_t), cudaMemcpyDeviceToHost, s->ctx->stream));
        VKB_CUDA(cudaStreamSynchronize(s->ctx->stream));
    });
}

vkb_status vkb_debug_blas_morton(vkb_scene* s, uint32_t mesh, uint32_t* out) {
    if (!s || !out) return fail(VKB_INVALID_ARG, "null argument");
    if (mesh >= s->num_meshes) return fail(VKB_INVALID_ARG, "mesh index out of range");
    return guarded([&] {
        VKB_CUDA(cudaSetDevice(s->ctx->device));
        const MeshInfo& mi = s->mesh_info[mesh];
        uint32_t n = mi.num_triangles;
        if (n == 0) return;
        cudaStream_t st = s->ctx->stream;
        int sms = s->ctx->sms;
        s->tri_lo.alloc(n); s->tri_hi.alloc(n);
        s->scratch.reserve(n, st);
        k_tri_boxes<<<grid_for(n, 256, sms), 256, 0, st>>>(n, s->indices.p + mi.index_offset, s->vpos.p + mi.vertex_offset, s->tri_lo.p, s->tri_hi.p);
        VKB_CUDA(cudaMemsetAsync(s->scratch.bounds.p, 0xff, 3 * sizeof(uint32_t), st));
        VKB_CUDA(cudaMemsetAsync(s->scratch.bounds.p + 3, 0x00, 3 * sizeof(uint32_t), st));
        k_centroid_box<<<grid_for(n, 256, sms), 256, 0, st>>>(n, s->tri_lo.p, s->tri_hi.p, s->scratch.bounds.p);
        k_morton<<<grid_for(n, 256, sms), 256, 0, st>>>(n, s->tri_lo.p, s->tri_hi.p, s->scratch.bounds.p, s->scratch.codes.p, s->scratch.ids.p, false);
        VKB_CUDA(cudaMemcpyAsync(out, s->scratch.codes.p, n * sizeof(uint32_t), cudaMemcpyDeviceToHost, st));
        VKB_CUDA(cudaStreamSynchronize(st));
    });
}

vkb_status vkb_debug_trace(vkb_scene* s, uint32_t n, const float* rays7, float* out_t, uint32_t* out_ids, float* out_uv) {
    if (!s || (n && (!rays7 || !out_t || !out_ids || !out_uv))) return fail(VKB_INVALID_ARG, "null argument");
    return guarded([&] {
        VKB_CUDA(cudaSetDevice(s->ctx->device));
        cudaStream_t st = s->ctx->stream;
        DBuf<float4> r;
        DBuf<float> t, uv;
        DBuf<uint32_t> ids, err;
        // origins (xyz, tmax) in [0, n), directions in [n, 2n)
        std::vector<float4> rays4(2 * size_t(n));
        for (uint32_t i = 0; i < n; ++i) {
            const float* q = rays7 + 7 * size_t(i);
            rays4[i] = make_float4(q[0], q[1], q[2], q[6]);
            rays4[n + i] = make_float4(q[3], q[4], q[5], 0.f);
        }
        r.upload(rays4.data(), rays4.size(), st);
        t.alloc(n); uv.alloc(size_t(n) * 2); ids.alloc(size_t(n) * 2); err.alloc(1);
        VKB_CUDA(cudaMemsetAsync(err.p, 0, sizeof(uint32_t), st));
        if (n && s->blas8.p) k_debug_trace<true><<<grid_for(n, 128, s->ctx->sms), 128, 0, st>>>(scene_view(s), n, r.p, t.p, ids.p, uv.p, err.p);
        else if (n) k_debug_trace<false><<<grid_for(n, 128, s->ctx->sms), 128, 0, st>>>(scene_view(s), n, r.p, t.p, ids.p, uv.p, err.p);
        if (n) {
            VKB_CUDA(cudaMemcpyAsync(out_t, t.p, n * sizeof(float), cudaMemcpyDeviceToHost, st));
            VKB_CUDA(cudaMemcpyAsync(out_ids, ids.p, size_t(n) * 2 * sizeof(uint32_t), cudaMemcpyDeviceToHost, st));
            VKB_CUDA(cudaMemcpyAsync(out_uv, uv.p, size_t(n) * 2 * sizeof(float), cudaMemcpyDeviceToHost, st));
        }
        VKB_CUDA(cudaStreamSynchronize(st));
        r.release(); t.release(); uv.release(); ids.release(); err.release();
    });
}

vkb_status vkb_debug_occluded(vkb_scene* s, uint32_t n, const float* rays7, uint32_t* out_occluded) {
    if (!s || (n && (!rays7 || !out_occluded))) return fail(VKB_INVALID_ARG, "null argument");
    return guarded([&] {
        VKB_CUDA(cudaSetDevice(s->ctx->device));
        cudaStream_t st = s->ctx->stream;
        DBuf<float4> r;
        DBuf<uint32_t> occ, err;
        std::vector<float4> rays4(2 * size_t(n));
        for (uint32_t i = 0; i < n; ++i) {
            const float* q = rays7 + 7 * size_t(i);
            rays4[i] = make_float4(q[0], q[1], q[2], q[6]);
            rays4[n + i] = make_float4(q[3], q[4], q[5], 0.f);
        }
        r.upload(rays4.data(), rays4.size(), st);
        occ.alloc(n); err.alloc(1);
        VKB_CUDA(cudaMemsetAsync(err.p, 0, sizeof(uint32_t), st));
        if (n) {
            if (s->blas8.p) k_debug_occluded<true><<<grid_for(n, 128, s->ctx->sms), 128, 0, st>>>(scene_view(s), n, r.p, occ.p, err.p);
            else k_debug_occluded<false><<<grid_for(n, 128, s->ctx->sms), 128, 0, st>>>(scene_view(s), n, r.p, occ.p, err.p);
            VKB_CUDA(cudaMemcpyAsync(out_occluded, occ.p, n * sizeof(uint32_t), cudaMemcpyDeviceToHost, st));
        }
        uint32_t e = 0;
        VKB_CUDA(cudaMemcpyAsync(&e, err.p, sizeof(uint32_t), cudaMemcpyDeviceToHost, st));
        VKB_CUDA(cudaStreamSynchronize(st));
        r.release(); occ.release(); err.release();
        if (e) throw InternalError{"any-hit traversal overflowed its stack or step cap"};
    });
}

}  // extern "C"


// ================================================================ serving
// Continuous batching: requests queue on the host; at every wave boundary the server
// admits queued requests (FIFO) while the job table has room and the device-memory
// budget holds (resident scenes + shared wavefront + every admitted job's accumulator
// and output staging), runs one wave over all admitted jobs, and returns finished
// images.  vork's own kept-alive session serves one request at a time
// (crates/vork-cli/src/session.rs:1-60, crates/vork-render/src/shot/worker.rs).
struct vkb_server {
    vkb_ctx* c = nullptr;
    uint64_t budget = 0;
    uint32_t max_jobs = 0;
    size_t capacity = 0;
    Wavefront wave;                                   // the server's own queues (renders on the context keep theirs)
    Wavefront wave2;                                  // overlapped waves: the second wavefront (on the context's stream2)
    cudaEvent_t acc_ev[2] = {nullptr, nullptr};       // and the events that keep its accumulations in wave order
    std::unique_ptr<WaveEngine> eng;
    struct Pending { uint64_t id; vkb_scene* s; vkb_profile pf; float* host_out; bool own_camera; vkb_camera cam; };
    // A request's device accumulator and mean image, taken from (and returned to) a pool
    // keyed by pixel capacity, so steady serving calls neither cudaMalloc nor cudaFree.
    struct Buffers { float4* accum = nullptr; float4* out = nullptr; size_t npix = 0; };
    struct Live { uint64_t id; float* host_out; Buffers buf; uint32_t npix; uint64_t bytes; };
    std::deque<Pending> queue;
    std::map<uint64_t, std::unique_ptr<Live>> live;   // admitted, keyed by id
    std::map<uint64_t, int> state;                    // 0 queued, 1 running, 2 done
    uint64_t next_id = 1, used_bytes = 0, peak_bytes = 0, wave_bytes = 0, pool_bytes = 0;
    std::map<vkb_scene*, uint64_t> resident;           // scene -> device bytes
    std::multimap<size_t, Buffers> pool;               // idle request buffers by pixel capacity
    // Waves in flight: the event after a wave and the copies of its finished requests' images,
    // with those requests' ids.  A step enqueues its wave without waiting for the previous
    // one, so the device always has the next wave queued while the host admits and reaps.
    struct Completion { cudaEvent_t ev; std::vector<uint64_t> ids; };
    std::deque<Completion> inflight;
    std::vector<cudaEvent_t> spare_events;
    cudaStream_t copy_stream = nullptr;               // device->host copies of finished images
};

namespace {
// Device bytes a scene holds itself (a fork: its instances and TLAS only).
uint64_t scene_bytes(const vkb_scene* s) {
    uint64_t own = s->tlas_nodes.n * sizeof(BvhNode) + s->tlas4.n * sizeof(Bvh4Node) + s->tlas_odd.n + s->tlas_leaves.n * sizeof(TlasLeaf) +
                   (s->o2w.n + s->w2o.n) * sizeof(float4) + s->inst_info.n * sizeof(uint4) + s->em_tree.n * sizeof(float);
    if (s->base) return own;
    return own + s->vpos.n * sizeof(float4) + s->vnrm.n * sizeof(float4) + s->indices.n * 4 + s->blas4.n * sizeof(Bvh4Node) + s->blas8.n * sizeof(Bvh8Node) +
           (s->blas_tris.n + s->tri_nrm.n) * sizeof(float4) + s->env_img.n * sizeof(float4) + s->env_dist.n * sizeof(float2) +
           s->em_inst_source.n * 4 + s->em_sources.n * sizeof(uint2);
}
uint64_t resident_bytes(const vkb_server* v) {
    uint64_t b = 0;
    for (auto& kv : v->resident) b += kv.second;
    return b;
}
constexpr uint64_t SERVER_BYTES_PER_PIXEL = 2 * sizeof(float4);   // accumulator + mean image
// Buffers for npix pixels: the smallest idle ones that hold them (and are not more than
// twice as large), else new ones.
constexpr uint64_t SERVER_DEVICE_RESERVE = uint64_t(1) << 30;   // device memory left to the driver and other users
vkb_server::Buffers take_buffers(vkb_server* v, size_t npix) {
    auto it = v->pool.lower_bound(npix);
    if (it != v->pool.end() && it->first <= 2 * npix) {
        vkb_server::Buffers b = it->second;
        v->pool.erase(it);
        v->pool_bytes -= b.npix * SERVER_BYTES_PER_PIXEL;
        return b;
    }
    vkb_server::Buffers b;
    b.npix = npix;
    VKB_CUDA(cudaMalloc(&b.accum, npix * sizeof(float4)));
    cudaError_t e = cudaMalloc(&b.out, npix * sizeof(float4));
    if (e != cudaSuccess) { cudaFree(b.accum); throw CudaError{e, "cudaMalloc(request image)"}; }
    return b;
}
void free_pool(vkb_server* v) {
    for (auto& kv : v->pool) { cudaFree(kv.second.accum); cudaFree(kv.second.out); }
    v->pool.clear();
    v->pool_bytes = 0;
}
// Finished requests of the waves whose events have completed (all of them with wait):
// copy each image to its host buffer on the copy stream (the next wave keeps running),
// return the buffers to the pool and mark the request done.
uint32_t reap(vkb_server* v, bool wait_all, bool wait_oldest) {
    uint32_t done = 0;
    while (!v->inflight.empty()) {
        vkb_server::Completion& cpl = v->inflight.front();
        if (wait_all || (wait_oldest && done == 0)) VKB_CUDA(cudaEventSynchronize(cpl.ev));
        else {
            cudaError_t q = cudaEventQuery(cpl.ev);
            if (q == cudaErrorNotReady) break;
            if (q != cudaSuccess) throw CudaError{q, "cudaEventQuery(wave)"};
        }
        for (uint64_t id : cpl.ids) {
            vkb_server::Live& l = *v->live[id];
            VKB_CUDA(cudaMemcpyAsync(l.host_out, l.buf.out, size_t(l.npix) * sizeof(float4), cudaMemcpyDeviceToHost, v->copy_stream));
        }
        VKB_CUDA(cudaStreamSynchronize(v->copy_stream));
        for (uint64_t id : cpl.ids) {
            vkb_server::Live& l = *v->live[id];
            v->pool.emplace(l.buf.npix, l.buf);
            v->pool_bytes += l.buf.npix * SERVER_BYTES_PER_PIXEL;
            v->used_bytes -= l.bytes;
            v->live.erase(id);
            v->state[id] = 2;
            ++done;
        }
        v->spare_events.push_back(cpl.ev);
        v->inflight.pop_front();
    }
    return done;
}
}  // namespace

extern "C" {

vkb_status vkb_server_create(vkb_ctx* c, const vkb_server_config* cfg, vkb_server** out) {
    if (!c || !cfg || !out) return fail(VKB_INVALID_ARG, "null argument");
    *out = nullptr;
    auto v = std::make_unique<vkb_server>();
    vkb_status st = guarded([&] {
        if (cfg->max_jobs == 0 || cfg->max_jobs > 4096) throw ArgError{"max_jobs must be 1..4096"};
        VKB_CUDA(cudaSetDevice(c->device));
        v->c = c;
        v->budget = cfg->memory_budget_bytes;
        v->max_jobs = cfg->max_jobs;
        v->capacity = cfg->wave_capacity ? size_t(cfg->wave_capacity) : c->wave_capacity;
        v->wave_bytes = uint64_t(v->capacity) * 220u + uint64_t(v->max_jobs) * sizeof(Job);
        if (v->budget && v->wave_bytes >= v->budget) throw ArgError{"memory budget below the wavefront's own footprint"};
        v->wave.reserve(v->capacity, v->max_jobs);
        VKB_CUDA(cudaStreamCreateWithFlags(&v->copy_stream, cudaStreamNonBlocking));
        v->eng = std::make_unique<WaveEngine>(c, v->wave.view(), v->capacity, cfg->flags, true);
        // Consecutive waves alternate between two wavefronts and streams (as single renders
        // do) when the budget holds both wavefronts and the flags do not ask for one stream;
        // the second wavefront counts against the budget like the first, and the accumulator
        // clears of admitted requests then go with the waves.
        const uint64_t second = uint64_t(v->capacity) * 220u + uint64_t(v->max_jobs) * sizeof(Job);
        if (!(cfg->flags & (VKB_PROFILE_SERIAL_WAVES | VKB_PROFILE_TIME_KERNELS)) && (!v->budget || v->wave_bytes + second < v->budget)) {
            v->wave2.reserve(v->capacity, v->max_jobs);
            VKB_CUDA(cudaEventCreateWithFlags(&v->acc_ev[0], cudaEventDisableTiming));
            VKB_CUDA(cudaEventCreateWithFlags(&v->acc_ev[1], cudaEventDisableTiming));
            WaveBuffers w2 = v->wave2.view();
            VKB_CUDA(cudaMemsetAsync(w2.counters, 0, 16 * sizeof(uint32_t), c->stream));
            VKB_CUDA(cudaMemsetAsync(w2.err, 0, sizeof(uint32_t), c->stream));
            VKB_CUDA(cudaMemsetAsync(w2.work, 0, 8 * sizeof(unsigned long long), c->stream));
            VKB_CUDA(cudaStreamSynchronize(c->stream));
            v->eng->overlap = true;
            v->eng->w2 = w2;
            v->eng->acc_ev = v->acc_ev;
            v->eng->defer_clears = true;
            v->wave_bytes += second;
        }
        v->eng->packed = (cfg->flags & VKB_BATCH_PACKED) != 0;
        v->eng->srpt = !v->eng->packed && (cfg->flags & VKB_BATCH_FAIR) == 0;
        if (!(cfg->aging_paths_per_s >= 0.0)) throw ArgError{"aging_paths_per_s must be non-negative"};
        v->eng->aging_rate = cfg->aging_paths_per_s;
    });
    if (st != VKB_OK) return st;
    *out = v.release();
    return VKB_OK;
}

vkb_status vkb_server_submit_view(vkb_server* v, vkb_scene* s, const vkb_camera* cam, const vkb_profile* pf, float* host_rgba, uint64_t* id) {
    if (!v || !s || !pf || !host_rgba || !id) return fail(VKB_INVALID_ARG, "null argument");
    if (s->ctx != v->c) return fail(VKB_INVALID_ARG, "scene belongs to another context");
    return guarded([&] {
        validate_profile(pf);
        if (cam) validate_camera(*cam);
        if (pf->adaptive) throw Unsupported{"adaptive stopping renders through vkb_render"};
        if (s->blas8.p) throw Unsupported{"compressed 8-wide BLAS scenes render through vkb_render and vkb_render_batch"};
        const vkb_camera& c = cam ? *cam : s->camera;
        uint64_t need = uint64_t(c.width) * c.height * 32u;
        const uint64_t sb = scene_bytes(s) + (s->base ? scene_bytes(s->base) : 0u);
        if (v->budget && v->wave_bytes + sb + need > v->budget) throw ArgError{"request can never fit the memory budget"};
        if (uint64_t(c.width) * c.height > v->capacity) throw ArgError{"request image larger than a wave"};
        *id = v->next_id++;
        v->queue.push_back({*id, s, *pf, host_rgba, cam != nullptr, c});
        v->state[*id] = 0;
    });
}

vkb_status vkb_server_submit(vkb_server* v, vkb_scene* s, const vkb_profile* pf, float* host_rgba, uint64_t* id) {
    return vkb_server_submit_view(v, s, nullptr, pf, host_rgba, id);
}

vkb_status vkb_server_step(vkb_server* v, vkb_server_status* status) {
    if (!v) return fail(VKB_INVALID_ARG, "null server");
    return guarded([&] {
        vkb_ctx* c = v->c;
        VKB_CUDA(cudaSetDevice(c->device));
        WaveEngine& eng = *v->eng;
        uint32_t finished = reap(v, false, false);
        // Scenes held under the budget: those of the admitted requests (and a fork's base).
        v->resident.clear();
        for (const EngineJob& e : eng.jobs) {
            v->resident[e.s] = scene_bytes(e.s);
            if (e.s->base) v->resident[e.s->base] = scene_bytes(e.s->base);
        }
        // Admit at the wave boundary.  Budget: the wavefront, resident scenes, every live
        // request's buffers and the idle pool (emptied first when a request needs the room).
        while (!v->queue.empty() && eng.jobs.size() < v->max_jobs) {
            auto& q = v->queue.front();
            uint64_t npix = uint64_t(q.cam.width) * q.cam.height;
            uint64_t need = npix * SERVER_BYTES_PER_PIXEL;
            uint64_t scene = v->resident.count(q.s) ? 0u : scene_bytes(q.s);
            if (q.s->base && !v->resident.count(q.s->base)) scene += scene_bytes(q.s->base);
            auto held = [&] { return v->wave_bytes + resident_bytes(v) + v->used_bytes + v->pool_bytes; };
            auto fit = v->pool.lower_bound(npix);
            uint64_t extra = (fit != v->pool.end() && fit->first <= 2 * npix) ? 0u : need;   // reused buffers add nothing
            // The first request with an image environment or emissive meshes: the
            // wavefront's environment and mesh shadow rays and previous vertices (112 B per
            // path slot), kept for every later wave.
            const bool ext = (q.s->env_w || q.s->em_tris) && !v->wave.sc_o.p;
            const uint64_t ext_bytes = ext ? uint64_t(v->capacity) * 112u * (eng.overlap ? 2u : 1u) : 0u;
            if (v->budget && held() + scene + extra + ext_bytes > v->budget && v->pool_bytes) {
                finished += reap(v, true, false);
                free_pool(v);
                extra = need;
            }
            if (v->budget && held() + scene + extra + ext_bytes > v->budget) break;
            // The budget counts the server's own memory only: a request that needs new
            // device memory also waits for the device to have it (other renders on the
            // context hold their own wavefronts), unless nothing else is running.
            if (extra + ext_bytes > 0) {
                auto device_free = [] {
                    size_t f = 0, t = 0;
                    return cudaMemGetInfo(&f, &t) == cudaSuccess ? uint64_t(f) : ~uint64_t(0);
                };
                if (device_free() < extra + ext_bytes + SERVER_DEVICE_RESERVE && v->pool_bytes) {
                    finished += reap(v, true, false);
                    free_pool(v);
                    extra = need;
                }
                if (device_free() < extra + ext_bytes + SERVER_DEVICE_RESERVE && (!eng.jobs.empty() || !v->inflight.empty())) break;
            }
            if (ext) {
                v->wave.reserve_ext(v->capacity);
                v->wave_bytes += ext_bytes;
                eng.w = v->wave.view();
                if (eng.overlap) {   // ext_bytes counts both wavefronts
                    v->wave2.reserve_ext(v->capacity);
                    eng.w2 = v->wave2.view();
                }
            }
            auto live = std::make_unique<vkb_server::Live>();
            live->id = q.id; live->host_out = q.host_out; live->npix = uint32_t(npix);
            live->buf = take_buffers(v, npix);
            live->bytes = live->buf.npix * SERVER_BYTES_PER_PIXEL;
            EngineJob e;
            e.s = q.s; e.pf = q.pf; e.npix = uint32_t(npix);
            e.own_camera = q.own_camera; e.camera = q.cam;
            e.count = q.pf.sample_count ? q.pf.sample_count : q.pf.samples - q.pf.first_sample;
            e.accum = live->buf.accum; e.out_dev = live->buf.out;
            e.admitted_s = host_seconds();
            eng.add(e);
            v->resident[q.s] = scene_bytes(q.s);
            if (q.s->base) v->resident[q.s->base] = scene_bytes(q.s->base);
            v->used_bytes += live->bytes;
            v->peak_bytes = std::max(v->peak_bytes, held());
            v->state[q.id] = 1;
            v->live[q.id] = std::move(live);
            v->queue.pop_front();
        }
        if (!eng.jobs.empty()) {
            eng.step();
            // Requests whose last samples are in this wave: resolve behind it (on its stream);
            // they are done once the wave's event has completed and their images are copied (reap).
            cudaStream_t ws = eng.last_stream ? eng.last_stream : c->stream;
            vkb_server::Completion cpl;
            for (size_t k = 0; k < eng.jobs.size(); ++k) {
                if (!eng.finished(k)) continue;
                eng.resolve(k, ws);
                for (auto& kv : v->live)
                    if (kv.second->buf.out == eng.jobs[k].out_dev) cpl.ids.push_back(kv.first);
            }
            eng.compact();
            if (v->spare_events.empty()) {
                cudaEvent_t ev;
                VKB_CUDA(cudaEventCreateWithFlags(&ev, cudaEventDisableTiming));
                v->spare_events.push_back(ev);
            }
            cpl.ev = v->spare_events.back();
            v->spare_events.pop_back();
            VKB_CUDA(cudaEventRecord(cpl.ev, ws));
            v->inflight.push_back(std::move(cpl));
            // At most two waves in flight: wait for the older one before returning.
            if (v->inflight.size() > 2) finished += reap(v, false, true);
        } else if (!v->inflight.empty()) {
            finished += reap(v, false, true);             // nothing new to run: deliver the oldest
        }
        if (status) {
            uint32_t completing = 0;
            for (const auto& cp : v->inflight) completing += uint32_t(cp.ids.size());
            status->queued = uint32_t(v->queue.size());
            status->running = uint32_t(eng.jobs.size()) + completing;
            status->finished = finished;
            status->used_bytes = v->wave_bytes + resident_bytes(v) + v->used_bytes + v->pool_bytes;
            status->peak_bytes = v->peak_bytes;
        }
    });
}

vkb_status vkb_server_poll(vkb_server* v, uint64_t id, int* state) {
    if (!v || !state) return fail(VKB_INVALID_ARG, "null argument");
    auto it = v->state.find(id);
    if (it == v->state.end()) return fail(VKB_INVALID_ARG, "unknown request id");
    if (it->second == 1) {
        vkb_status st = guarded([&] { VKB_CUDA(cudaSetDevice(v->c->device)); reap(v, false, false); });
        if (st != VKB_OK) return st;
    }
    *state = it->second;
    return VKB_OK;
}

vkb_status vkb_server_destroy(vkb_server* v) {
    if (!v) return VKB_OK;
    cudaSetDevice(v->c->device);
    cudaStreamSynchronize(v->c->stream);
    cudaStreamSynchronize(v->c->stream2);
    for (auto& cp : v->inflight) cudaEventDestroy(cp.ev);
    for (cudaEvent_t e : v->acc_ev) if (e) cudaEventDestroy(e);
    for (cudaEvent_t e : v->spare_events) cudaEventDestroy(e);
    if (v->copy_stream) { cudaStreamSynchronize(v->copy_stream); cudaStreamDestroy(v->copy_stream); }
    for (auto& kv : v->live) { cudaFree(kv.second->buf.accum); cudaFree(kv.second->buf.out); }
    v->live.clear();
    free_pool(v);
    v->eng.reset();
    v->wave.release();
    v->wave2.release();
    delete v;
    return VKB_OK;
}

}  // extern "C"

// ================================================================ render without allocation
//
// Some callers cannot allocate device memory while they render: a host renderer
// that owns every device allocation through its own memory manager and residency
// budget (vork's gpu_memory / residency model), a serving loop that must not change
// its footprint after admission, or code running while the device allocator is
// locked.  vkb_render_noalloc serves them: it renders an installed scene with every
// wavefront queue, accumulator and counter carved from one fixed device array that
// the library holds for the life of the process, and calls no cudaMalloc/cudaFree.
namespace {

constexpr size_t NOALLOC_SCRATCH_BYTES = size_t(VKB_NOALLOC_SCRATCH_MIB) << 20;
// Every GPU that loads this library holds this array until the process exits.
static __device__ __align__(256) unsigned char g_noalloc_scratch[NOALLOC_SCRATCH_BYTES];

// Device address of g_noalloc_scratch on the current device, looked up on every call
// (the host-side symbol is only a stand-in, never a device address; a per-process cache
// would go stale if the caller reset the device and its context were recreated).
unsigned char* noalloc_scratch() {
    void* p = nullptr;
    VKB_CUDA(cudaGetSymbolAddress(&p, g_noalloc_scratch));
    return static_cast<unsigned char*>(p);
}

struct Carver {
    unsigned char* base;
    size_t used = 0, cap;
    template <class T> T* take(size_t count) {
        size_t off = (used + 255) & ~size_t(255);
        size_t bytes = count * sizeof(T);
        if (off + bytes > cap) return nullptr;
        used = off + bytes;
        return reinterpret_cast<T*>(base + off);
    }
};

}  // namespace

extern "C" vkb_status vkb_render_noalloc(vkb_scene* s, const vkb_profile* pf, vkb_output* out, vkb_stats* stats) {
    if (!s || !pf || !out || !out->rgba) return fail(VKB_INVALID_ARG, "null scene, profile or output");
    return guarded([&] {
        validate_profile(pf);
        if (pf->adaptive) throw Unsupported{"adaptive stopping renders through vkb_render"};
        if (out->guide_albedo || out->guide_normal) throw Unsupported{"denoiser guides render through vkb_render"};
        if (s->env_w || s->em_tris) throw Unsupported{"image environments and emissive meshes render through vkb_render"};
        uint32_t count = pf->sample_count ? pf->sample_count : pf->samples - pf->first_sample;
        vkb_ctx* c = s->ctx;
        VKB_CUDA(cudaSetDevice(c->device));
        unsigned char* base = noalloc_scratch();
        cudaStream_t st = c->stream;
        const uint32_t W = s->camera.width, H = s->camera.height, npix = W * H;
        // Fixed part: counters, error word, traversal counters, job table, accumulator,
        // optional ids and host-output staging.
        Carver cv{base, 0, NOALLOC_SCRATCH_BYTES};
        WaveBuffers w;
        w.counters = cv.take<uint32_t>(16);
        w.err = cv.take<uint32_t>(1);
        w.work = cv.take<unsigned long long>(8);
        w.jobs = cv.take<Job>(1);
        w.job_capacity = 1;
        float4* accum = cv.take<float4>(npix);
        uint32_t* ids = out->primary_ids ? cv.take<uint32_t>(size_t(npix) * 2) : nullptr;
        float4* staging = out->on_device ? reinterpret_cast<float4*>(out->rgba) : cv.take<float4>(npix);
        // Per-slot part: 13 float4 queues/state + hit instance + rng = 220 bytes per path slot.
        const size_t per_slot = 13 * sizeof(float4) + sizeof(uint32_t) + sizeof(uint2);
        const size_t fixed = (cv.used + 255) & ~size_t(255);
        size_t free_bytes = fixed < NOALLOC_SCRATCH_BYTES ? NOALLOC_SCRATCH_BYTES - fixed : 0;
        // 15 regions, each rounded up to 256 bytes.
        size_t slots_fit = free_bytes > 15 * 256 ? (free_bytes - 15 * 256) / per_slot : 0;
        if (!w.counters || !w.err || !w.work || !w.jobs || !accum || (out->primary_ids && !ids) || !staging || slots_fit < npix)
            throw ArgError{"vkb_render_noalloc: a " + std::to_string(W) + "x" + std::to_string(H) + " image needs " +
                           std::to_string((fixed + size_t(npix) * per_slot + 15 * 256) >> 10) + " KiB of scratch for one sample per wave; the fixed array holds " +
                           std::to_string(NOALLOC_SCRATCH_BYTES >> 10) + " KiB (use vkb_render)"};
        uint32_t wave = uint32_t(std::min<size_t>(slots_fit / npix, count));
        if (pf->wave_samples) wave = std::min(wave, pf->wave_samples);
        wave = std::max(1u, wave);
        size_t slots = size_t(npix) * wave;
        w.capacity = slots;
        w.ray_o0 = cv.take<float4>(slots); w.ray_d0 = cv.take<float4>(slots);
        w.ray_o1 = cv.take<float4>(slots); w.ray_d1 = cv.take<float4>(slots);
        w.hit = cv.take<float4>(slots); w.hit_inst = cv.take<uint32_t>(slots);
        w.thr = cv.take<float4>(slots); w.rad = cv.take<float4>(slots); w.rng = cv.take<uint2>(slots);
        w.sa_o = cv.take<float4>(slots); w.sa_d = cv.take<float4>(slots); w.sa_c = cv.take<float4>(slots);
        w.sb_o = cv.take<float4>(slots); w.sb_d = cv.take<float4>(slots); w.sb_c = cv.take<float4>(slots);
        w.slot_job = nullptr;  // one job: no per-slot job index
        if (!w.sb_c) throw ArgError{"vkb_render_noalloc: scratch layout overflow"};
        // The array keeps the previous call's contents: the engine clears the counters,
        // the accumulator and the traversal counters before the first wave.
        std::vector<EngineJob> jobs(1);
        EngineJob& e = jobs[0];
        e.s = s; e.pf = *pf; e.npix = npix; e.count = count;
        e.accum = accum; e.out_dev = staging; e.ids_dev = ids;
        WaveTotals tot;
        run_engine(c, jobs, w, slots, pf->flags & VKB_PROFILE_COUNT_TRAVERSAL, false, tot);
        if (!out->on_device) VKB_CUDA(cudaMemcpyAsync(out->rgba, staging, npix * sizeof(float4), cudaMemcpyDeviceToHost, st));
        if (out->primary_ids) VKB_CUDA(cudaMemcpyAsync(out->primary_ids, ids, size_t(npix) * 2 * sizeof(uint32_t), cudaMemcpyDeviceToHost, st));
        VKB_CUDA(cudaStreamSynchronize(st));
        s->launches += tot.launches;
        c->launches += tot.launches;
        fill_stats(stats, tot, uint64_t(npix) * count, s->build_ms);
    });
}

// ================================================================ learned radiance cache
#include "vkb_cache.cuh"
