// Host side of the learned radiance cache: parameters, Adam state, training buffers and
// the C ABI (included at the end of vkb.cu, inside its translation unit).
#pragma once

struct vkb_cache {
    vkb_scene* s = nullptr;
    vkb_cache_config cfg{};
    uint64_t steps = 0;
    float last_loss = 0.f, last_train_ms = 0.f;
    uint64_t last_records = 0;
    DBuf<float> mlp_master, mlp_m1, mlp_m2;
    DBuf<__nv_bfloat16> mlp_w;
    DBuf<float> hash_master, hash_m1, hash_m2;
    DBuf<__half> table;
    DBuf<long long> hash_grad;
    DBuf<float> wpartial, loss_partial, targets, scratch;
    DBuf<float4> records;
    DBuf<uint32_t> err;
    // Training paths: records, (throughput, radiance) and flags at fixed positions, the
    // compacted indices and count; the low-resolution training render's accumulator and image.
    DBuf<uint32_t> rec_flag, rec_index, rec_count;
    DBuf<float4> rec_sparse, aux, train_accum, train_out;
    DBuf<unsigned char> select_temp;
    // Render queries: one record and path slot per path slot of a wave.
    DBuf<float4> qrec;
    DBuf<uint32_t> qslot;
    float4 box_lo{}, box_scale{};   // world -> [0,1]^3, fixed at creation (5% margin)
    uint64_t train_calls = 0;
    // Training round: compaction start/end, optimizer steps start/end (no host
    // synchronisation inside either pair, so they measure device work only).
    cudaEvent_t ev[4] = {nullptr, nullptr, nullptr, nullptr};
    float last_paths_ms = 0.f, last_steps_ms = 0.f, last_host_ms = 0.f;
};

namespace {

using namespace vkb::nrc;

__global__ void k_nrc_init_hash(uint64_t count, uint32_t seed, float* master, __half* table) {
    for (uint64_t p = blockIdx.x * uint64_t(blockDim.x) + threadIdx.x; p < count; p += uint64_t(gridDim.x) * blockDim.x) {
        uint32_t h = uint32_t(p) * 0x9e3779b9u ^ uint32_t(p >> 32) * 0x85ebca6bu ^ seed * 0xc2b2ae35u;
        h ^= h >> 16; h *= 0x7feb352du; h ^= h >> 15; h *= 0x846ca68bu; h ^= h >> 16;
        const float x = (float(h >> 8) * (1.f / 16777216.f) * 2.f - 1.f) * 1e-4f;
        master[p] = x;
        table[p] = __float2half_rn(x);
    }
}
__global__ void k_nrc_from_master(uint64_t count, const float* master, __half* table) {
    for (uint64_t p = blockIdx.x * uint64_t(blockDim.x) + threadIdx.x; p < count; p += uint64_t(gridDim.x) * blockDim.x)
        table[p] = __float2half_rn(master[p]);
}
__global__ void k_nrc_mlp_from_master(uint32_t count, const float* master, __nv_bfloat16* w) {
    for (uint32_t p = blockIdx.x * blockDim.x + threadIdx.x; p < count; p += gridDim.x * blockDim.x) w[p] = __float2bfloat16_rn(master[p]);
}

void cache_defaults(vkb_cache_config& c) {
    if (!c.train_records) c.train_records = 65536;
    if (!c.train_steps) c.train_steps = 4;
    if (!c.query_vertex) c.query_vertex = 2;
    if (c.lr_mlp == 0.f) c.lr_mlp = 2e-3f;
    if (c.lr_hash == 0.f) c.lr_hash = 1e-2f;
    if (c.beta1 == 0.f) c.beta1 = 0.9f;
    if (c.beta2 == 0.f) c.beta2 = 0.99f;
    if (c.eps == 0.f) c.eps = 1e-10f;
}

// Xavier-uniform MLP weights from a PCG32 stream (rows 3..15 of the output layer zero).
std::vector<float> mlp_init(uint32_t seed) {
    std::vector<float> w(MLP_PARAMS, 0.f);
    uint64_t state = 0x853c49e6748fea9bull + seed, inc = 0xda3e39cb94b95bdbull | 1u;
    auto next = [&]() {
        uint64_t old = state;
        state = old * 6364136223846793005ull + inc;
        uint32_t xs = uint32_t(((old >> 18u) ^ old) >> 27u), rot = uint32_t(old >> 59u);
        return (xs >> rot) | (xs << ((32u - rot) & 31u));
    };
    for (int l = 0; l < LAYERS; ++l) {
        const int rows = l == LAYERS - 1 ? 3 : WIDTH;
        const float a = std::sqrt(6.f / float(WIDTH + rows));
        for (int o = 0; o < rows; ++o)
            for (int i = 0; i < WIDTH; ++i) w[size_t(l) * WIDTH * WIDTH + size_t(o) * WIDTH + i] = (float(next() >> 8) * (1.f / 16777216.f) * 2.f - 1.f) * a;
    }
    return w;
}

void nrc_kernel_attributes() {
    static std::once_flag once;
    std::call_once(once, [] {
        VKB_CUDA(cudaFuncSetAttribute(k_nrc_forward<DebugIO>, cudaFuncAttributeMaxDynamicSharedMemorySize, int(FWD_SMEM)));
        VKB_CUDA(cudaFuncSetAttribute(k_nrc_forward<QueryIO>, cudaFuncAttributeMaxDynamicSharedMemorySize, int(FWD_SMEM)));
        VKB_CUDA(cudaFuncSetAttribute(k_nrc_train, cudaFuncAttributeMaxDynamicSharedMemorySize, int(TRN_SMEM)));
    });
}

void check_nrc_err(vkb_cache* k) {
    uint32_t e = 0;
    VKB_CUDA(cudaMemcpyAsync(&e, k->err.p, sizeof(e), cudaMemcpyDeviceToHost, k->s->ctx->stream));
    VKB_CUDA(cudaStreamSynchronize(k->s->ctx->stream));
    if (e) {
        VKB_CUDA(cudaMemsetAsync(k->err.p, 0, sizeof(uint32_t), k->s->ctx->stream));
        throw DeviceTimeout{"a tensor-core wait of the radiance cache ran out"};
    }
}

// Mean loss of the last step (over its n records) from the per-tile partials; also
// raises a timed-out tensor-core wait.  Synchronises.
float nrc_read_loss(vkb_cache* k, uint32_t n) {
    cudaStream_t st = k->s->ctx->stream;
    const uint32_t tiles = (n + TILE - 1) / TILE;
    std::vector<float> lp(tiles);
    VKB_CUDA(cudaMemcpyAsync(lp.data(), k->loss_partial.p, tiles * sizeof(float), cudaMemcpyDeviceToHost, st));
    check_nrc_err(k);
    double sum = 0.0;
    for (float x : lp) sum += x;
    k->last_loss = float(sum / (3.0 * n));
    return k->last_loss;
}

// Gradients of the loss over the device records offset, offset + stride, ... below
// `total` (already in k->records / k->targets); with `update` also one Adam step.  With
// `read_loss` returns the step's mean loss (one host round trip), else 0.
float nrc_step(vkb_cache* k, uint32_t total, bool update, float* mlp_grad_dev, float* hash_grad_dev, uint32_t offset = 0,
               uint32_t stride = 1, bool read_loss = true) {
    vkb_ctx* c = k->s->ctx;
    cudaStream_t st = c->stream;
    nrc_kernel_attributes();
    const uint32_t n = offset < total ? (total - offset + stride - 1) / stride : 0u;
    if (n == 0) return 0.f;
    const uint32_t tiles = (n + TILE - 1) / TILE;
    k->wpartial.alloc(size_t(tiles) * MLP_PARAMS);
    k->loss_partial.alloc(tiles);
    k_nrc_train<<<tiles, TILE, TRN_SMEM, st>>>(k->records.p, k->targets.p, n, offset, stride, 1.f / float(3u * n), k->mlp_w.p, k->table.p,
                                               k->wpartial.p, k->hash_grad.p, k->loss_partial.p, k->err.p);
    AdamParams am{0.f, k->cfg.beta1, k->cfg.beta2, k->cfg.eps, 1.f, 1.f}, ah = am;
    if (update) {
        k->steps++;
        const float bc1 = 1.f - std::pow(k->cfg.beta1, float(k->steps)), bc2 = 1.f - std::pow(k->cfg.beta2, float(k->steps));
        am = AdamParams{k->cfg.lr_mlp, k->cfg.beta1, k->cfg.beta2, k->cfg.eps, bc1, bc2};
        ah = AdamParams{k->cfg.lr_hash, k->cfg.beta1, k->cfg.beta2, k->cfg.eps, bc1, bc2};
    }
    k_nrc_adam_mlp<<<grid_for(MLP_PARAMS, 256, c->sms), 256, 0, st>>>(tiles, k->wpartial.p, k->mlp_master.p, k->mlp_m1.p, k->mlp_m2.p, k->mlp_w.p,
                                                                       am, mlp_grad_dev);
    k_nrc_adam_hash<<<c->sms * 8, 256, 0, st>>>(HASH_PARAMS, k->hash_grad.p, k->hash_master.p, k->hash_m1.p, k->hash_m2.p, k->table.p, ah,
                                                hash_grad_dev);
    k->s->launches += 3;
    VKB_CUDA(cudaGetLastError());
    if (!read_loss) return 0.f;
    return nrc_read_loss(k, n);
}

void upload_records(vkb_cache* k, uint32_t n, const float* records, const float* targets) {
    cudaStream_t st = k->s->ctx->stream;
    k->records.alloc(size_t(n) * 4);
    VKB_CUDA(cudaMemcpyAsync(k->records.p, records, size_t(n) * RECORD_FLOATS * sizeof(float), cudaMemcpyHostToDevice, st));
    if (targets) {
        k->targets.alloc(size_t(n) * 3);
        VKB_CUDA(cudaMemcpyAsync(k->targets.p, targets, size_t(n) * 3 * sizeof(float), cudaMemcpyHostToDevice, st));
    }
}

}  // namespace

extern "C" {

vkb_status vkb_cache_create(vkb_scene* s, const vkb_cache_config* config, vkb_cache** out) {
    if (!s || !out) return fail(VKB_INVALID_ARG, "null scene or output pointer");
    *out = nullptr;
    auto* k = new vkb_cache();
    k->s = s;
    if (config) k->cfg = *config;
    cache_defaults(k->cfg);
    vkb_status st = guarded([&] {
        if (k->cfg.query_vertex < 1 || k->cfg.query_vertex > 16) throw ArgError{"query_vertex must be 1..16"};
        VKB_CUDA(cudaSetDevice(s->ctx->device));
        cudaStream_t str = s->ctx->stream;
        for (auto& e : k->ev) VKB_CUDA(cudaEventCreate(&e));
        k->mlp_master.alloc(MLP_PARAMS); k->mlp_m1.alloc(MLP_PARAMS); k->mlp_m2.alloc(MLP_PARAMS); k->mlp_w.alloc(MLP_PARAMS);
        k->hash_master.alloc(HASH_PARAMS); k->hash_m1.alloc(HASH_PARAMS); k->hash_m2.alloc(HASH_PARAMS);
        k->table.alloc(HASH_PARAMS); k->hash_grad.alloc(HASH_PARAMS); k->err.alloc(1);
        VKB_CUDA(cudaMemsetAsync(k->mlp_m1.p, 0, MLP_PARAMS * sizeof(float), str));
        VKB_CUDA(cudaMemsetAsync(k->mlp_m2.p, 0, MLP_PARAMS * sizeof(float), str));
        VKB_CUDA(cudaMemsetAsync(k->hash_m1.p, 0, HASH_PARAMS * sizeof(float), str));
        VKB_CUDA(cudaMemsetAsync(k->hash_m2.p, 0, HASH_PARAMS * sizeof(float), str));
        VKB_CUDA(cudaMemsetAsync(k->hash_grad.p, 0, HASH_PARAMS * sizeof(long long), str));
        VKB_CUDA(cudaMemsetAsync(k->err.p, 0, sizeof(uint32_t), str));
        // Normalisation box: the TLAS root box at creation, 5% margin on every side.
        BvhNode root{};
        VKB_CUDA(cudaMemcpyAsync(&root, s->tlas_nodes.p, sizeof(BvhNode), cudaMemcpyDeviceToHost, str));
        VKB_CUDA(cudaStreamSynchronize(str));
        float lo[3] = {root.a.x, root.a.z, root.c.x}, hi[3] = {root.a.y, root.a.w, root.c.y};
        if (s->num_instances > 1) {
            lo[0] = std::min(lo[0], root.b.x); hi[0] = std::max(hi[0], root.b.y);
            lo[1] = std::min(lo[1], root.b.z); hi[1] = std::max(hi[1], root.b.w);
            lo[2] = std::min(lo[2], root.c.z); hi[2] = std::max(hi[2], root.c.w);
        }
        float ext = 0.f;
        for (int a = 0; a < 3; ++a) ext = std::max(ext, hi[a] - lo[a]);
        if (!(ext > 0.f) || !std::isfinite(ext)) throw ArgError{"the scene has no finite extent for the radiance cache"};
        for (int a = 0; a < 3; ++a) {
            const float m = 0.05f * std::max(hi[a] - lo[a], 1e-3f * ext);
            lo[a] -= m; hi[a] += m;
        }
        k->box_lo = make_float4(lo[0], lo[1], lo[2], 0.f);
        k->box_scale = make_float4(1.f / (hi[0] - lo[0]), 1.f / (hi[1] - lo[1]), 1.f / (hi[2] - lo[2]), 0.f);
        std::vector<float> w = mlp_init(k->cfg.seed);
        VKB_CUDA(cudaMemcpyAsync(k->mlp_master.p, w.data(), MLP_PARAMS * sizeof(float), cudaMemcpyHostToDevice, str));
        k_nrc_mlp_from_master<<<grid_for(MLP_PARAMS, 256, s->ctx->sms), 256, 0, str>>>(MLP_PARAMS, k->mlp_master.p, k->mlp_w.p);
        k_nrc_init_hash<<<s->ctx->sms * 8, 256, 0, str>>>(HASH_PARAMS, k->cfg.seed, k->hash_master.p, k->table.p);
        VKB_CUDA(cudaGetLastError());
        VKB_CUDA(cudaStreamSynchronize(str));
    });
    if (st != VKB_OK) { delete k; return st; }
    *out = k;
    return VKB_OK;
}

vkb_status vkb_cache_destroy(vkb_cache* k) {
    if (!k) return VKB_OK;
    cudaSetDevice(k->s->ctx->device);
    cudaStreamSynchronize(k->s->ctx->stream);
    k->mlp_master.release(); k->mlp_m1.release(); k->mlp_m2.release(); k->mlp_w.release();
    k->hash_master.release(); k->hash_m1.release(); k->hash_m2.release(); k->table.release(); k->hash_grad.release();
    k->wpartial.release(); k->loss_partial.release(); k->targets.release(); k->scratch.release(); k->records.release(); k->err.release();
    for (auto& e : k->ev) if (e) cudaEventDestroy(e);
    k->rec_flag.release(); k->rec_index.release(); k->rec_count.release(); k->rec_sparse.release(); k->aux.release();
    k->train_accum.release(); k->train_out.release(); k->select_temp.release(); k->qrec.release(); k->qslot.release();
    delete k;
    return VKB_OK;
}

vkb_status vkb_cache_train(vkb_cache* k, const vkb_profile* pf, vkb_cache_stats* stats) {
    if (!k || !pf) return fail(VKB_INVALID_ARG, "null cache or profile");
    return guarded([&] {
        validate_profile(pf);
        vkb_scene* s = k->s;
        vkb_ctx* c = s->ctx;
        VKB_CUDA(cudaSetDevice(c->device));
        cudaStream_t st = c->stream;
        nrc_kernel_attributes();
        const auto host0 = std::chrono::steady_clock::now();
        // Training paths: the scene's camera at a resolution of about train_records / 2
        // pixels, one sample of a fresh seed per call, full path depth.
        const vkb_camera& cam = s->camera;
        const double px = std::max(256.0, double(k->cfg.train_records) / 2.0);
        const double aspect = double(cam.width) / double(cam.height);
        const uint32_t tw = std::max(8u, uint32_t(std::lround(std::sqrt(px * aspect)))), th = std::max(8u, uint32_t(std::lround(px / tw)));
        std::vector<EngineJob> jobs(1);
        EngineJob& e = jobs[0];
        e.s = s; e.pf = *pf;
        e.pf.samples = 1; e.pf.first_sample = 0; e.pf.sample_count = 1; e.pf.wave_samples = 1; e.pf.adaptive = 0;
        e.pf.seed = pf->seed ^ (0x9e3779b9u * uint32_t(k->train_calls + 1) + k->cfg.seed);
        e.own_camera = true; e.camera = cam; e.camera.width = tw; e.camera.height = th;
        e.npix = tw * th; e.count = 1;
        k->train_accum.alloc(e.npix); k->train_out.alloc(e.npix);
        e.accum = k->train_accum.p; e.out_dev = k->train_out.p;
        // Record positions: path slot x vmax + vertex - 1 (vertices 1..bounces[0]).
        const uint32_t vmax = std::max(1u, pf->bounces[0]);
        const uint32_t cap = e.npix * vmax;
        k->rec_sparse.alloc(size_t(cap) * 4); k->aux.alloc(size_t(cap) * 2); k->rec_flag.alloc(cap); k->rec_index.alloc(cap);
        k->rec_count.alloc(1); k->records.alloc(size_t(cap) * 4); k->targets.alloc(size_t(cap) * 3);
        VKB_CUDA(cudaMemsetAsync(k->rec_flag.p, 0, size_t(cap) * sizeof(uint32_t), st));
        c->wave.reserve(e.npix, 1);
        if (s->env_w || s->em_tris) c->wave.reserve_ext(c->wave.ray_o0.n);
        CacheLaunch cl;
        cl.dev.mode = 2; cl.dev.vertex = 0; cl.dev.capacity = cap; cl.dev.vmax = vmax;
        cl.dev.box_lo = k->box_lo; cl.dev.box_scale = k->box_scale;
        cl.dev.rec = k->rec_sparse.p; cl.dev.slot = nullptr; cl.dev.aux = k->aux.p; cl.dev.flag = k->rec_flag.p;
        cl.w = k->mlp_w.p; cl.table = k->table.p; cl.err = k->err.p;
        WaveTotals tot;
        run_engine(c, jobs, c->wave.view(), e.npix, 0, false, tot, false, &cl);
        // The wave's radiance is still in place: compact the flagged positions in order
        // and gather records and targets.
        VKB_CUDA(cudaEventRecord(k->ev[0], st));
        thrust::counting_iterator<uint32_t> positions(0u);
        size_t bytes = 0;
        VKB_CUDA(cub::DeviceSelect::Flagged(nullptr, bytes, positions, k->rec_flag.p, k->rec_index.p, k->rec_count.p, int(cap), st));
        k->select_temp.alloc(std::max<size_t>(bytes, 1));
        bytes = k->select_temp.n;
        VKB_CUDA(cub::DeviceSelect::Flagged(k->select_temp.p, bytes, positions, k->rec_flag.p, k->rec_index.p, k->rec_count.p, int(cap), st));
        k_nrc_gather<<<c->sms * 8, 256, 0, st>>>(k->rec_count.p, cap, k->rec_index.p, vmax, k->rec_sparse.p, k->aux.p, c->wave.view().rad,
                                                 k->records.p, k->targets.p);
        tot.launches += 2;
        VKB_CUDA(cudaGetLastError());
        VKB_CUDA(cudaEventRecord(k->ev[1], st));
        uint32_t count = 0;
        VKB_CUDA(cudaMemcpyAsync(&count, k->rec_count.p, sizeof(count), cudaMemcpyDeviceToHost, st));
        VKB_CUDA(cudaStreamSynchronize(st));
        count = std::min(count, cap);
        s->launches += tot.launches;
        k->train_calls++;
        // train_steps interleaved minibatches: step i takes records i, i + steps, ... (each
        // spread over the whole image), so one round visits every record once.
        const uint32_t steps = std::min(k->cfg.train_steps, std::max(1u, count));
        {
            // Per-tile partials of the largest step, grown here (a power of two of tiles, so
            // rarely) rather than inside the timed steps: a reallocation synchronises.
            const size_t tiles = (size_t((count + steps - 1) / steps) + TILE - 1) / TILE;
            size_t t2 = 1;
            while (t2 < tiles) t2 <<= 1;
            k->wpartial.alloc(t2 * MLP_PARAMS);
            k->loss_partial.alloc(t2);
        }
        VKB_CUDA(cudaEventRecord(k->ev[2], st));
        for (uint32_t i = 0; i < steps && count > 0; ++i) nrc_step(k, count, true, nullptr, nullptr, i, steps, false);
        VKB_CUDA(cudaEventRecord(k->ev[3], st));
        VKB_CUDA(cudaEventSynchronize(k->ev[3]));
        if (count > 0) nrc_read_loss(k, (count - (steps - 1) + steps - 1) / steps);   // records of the last step (offset steps - 1)
        float compact_ms = 0.f;
        VKB_CUDA(cudaEventElapsedTime(&compact_ms, k->ev[0], k->ev[1]));
        VKB_CUDA(cudaEventElapsedTime(&k->last_steps_ms, k->ev[2], k->ev[3]));
        k->last_paths_ms = tot.render_ms + compact_ms;
        k->last_train_ms = k->last_paths_ms + k->last_steps_ms;
        k->last_host_ms = std::chrono::duration<float, std::milli>(std::chrono::steady_clock::now() - host0).count();
        k->last_records = count;
        if (stats) {
            stats->steps = k->steps; stats->records = count; stats->loss = k->last_loss; stats->train_ms = k->last_train_ms;
            stats->paths_ms = k->last_paths_ms; stats->steps_ms = k->last_steps_ms; stats->host_ms = k->last_host_ms;
        }
    });
}

vkb_status vkb_render_cached(vkb_cache* k, const vkb_profile* pf, vkb_output* out, vkb_stats* stats) {
    if (!k || !pf || !out || !out->rgba) return fail(VKB_INVALID_ARG, "null cache, profile or output");
    return guarded([&] {
        validate_profile(pf);
        vkb_scene* s = k->s;
        vkb_ctx* c = s->ctx;
        VKB_CUDA(cudaSetDevice(c->device));
        nrc_kernel_attributes();
        const uint32_t count = pf->sample_count ? pf->sample_count : pf->samples - pf->first_sample;
        const size_t npix = size_t(s->camera.width) * s->camera.height;
        uint32_t hint = pf->wave_samples;
        if (!hint) hint = uint32_t(std::max<size_t>(1, std::min<size_t>(count, c->wave_capacity / std::max<size_t>(1, npix))));
        const size_t capacity = std::max(npix * hint, npix);   // the wave size render_jobs picks for one job
        k->qrec.alloc(capacity * 4); k->qslot.alloc(capacity);
        CacheLaunch cl;
        cl.dev.mode = 1; cl.dev.vertex = k->cfg.query_vertex; cl.dev.capacity = uint32_t(capacity);
        cl.dev.box_lo = k->box_lo; cl.dev.box_scale = k->box_scale;
        cl.dev.rec = k->qrec.p; cl.dev.slot = k->qslot.p; cl.dev.aux = nullptr;
        cl.w = k->mlp_w.p; cl.table = k->table.p; cl.err = k->err.p;
        std::vector<std::pair<vkb_scene*, vkb_profile>> in{{s, *pf}};
        std::vector<vkb_output*> outs{out};
        WaveTotals tot;
        uint64_t paths = 0;
        render_jobs(c, in, outs, pf->flags, hint, tot, paths, &cl);
        check_nrc_err(k);
        s->launches += tot.launches;
        fill_stats(stats, tot, paths, s->build_ms);
    });
}

vkb_status vkb_debug_nrc_set_params(vkb_cache* k, const float* mlp, const float* hash) {
    if (!k) return fail(VKB_INVALID_ARG, "null cache");
    return guarded([&] {
        VKB_CUDA(cudaSetDevice(k->s->ctx->device));
        cudaStream_t st = k->s->ctx->stream;
        if (mlp) {
            VKB_CUDA(cudaMemcpyAsync(k->mlp_master.p, mlp, MLP_PARAMS * sizeof(float), cudaMemcpyHostToDevice, st));
            k_nrc_mlp_from_master<<<grid_for(MLP_PARAMS, 256, k->s->ctx->sms), 256, 0, st>>>(MLP_PARAMS, k->mlp_master.p, k->mlp_w.p);
        }
        if (hash) {
            VKB_CUDA(cudaMemcpyAsync(k->hash_master.p, hash, HASH_PARAMS * sizeof(float), cudaMemcpyHostToDevice, st));
            k_nrc_from_master<<<k->s->ctx->sms * 8, 256, 0, st>>>(HASH_PARAMS, k->hash_master.p, k->table.p);
        }
        VKB_CUDA(cudaGetLastError());
        VKB_CUDA(cudaStreamSynchronize(st));
    });
}

vkb_status vkb_debug_nrc_get_params(vkb_cache* k, float* mlp, float* hash) {
    if (!k) return fail(VKB_INVALID_ARG, "null cache");
    return guarded([&] {
        VKB_CUDA(cudaSetDevice(k->s->ctx->device));
        cudaStream_t st = k->s->ctx->stream;
        if (mlp) VKB_CUDA(cudaMemcpyAsync(mlp, k->mlp_master.p, MLP_PARAMS * sizeof(float), cudaMemcpyDeviceToHost, st));
        if (hash) VKB_CUDA(cudaMemcpyAsync(hash, k->hash_master.p, HASH_PARAMS * sizeof(float), cudaMemcpyDeviceToHost, st));
        VKB_CUDA(cudaStreamSynchronize(st));
    });
}

vkb_status vkb_debug_nrc_forward(vkb_cache* k, uint32_t n, const float* records, float* x_out, float* y_out) {
    if (!k || (n && (!records || !y_out))) return fail(VKB_INVALID_ARG, "null argument");
    return guarded([&] {
        if (n == 0) return;
        VKB_CUDA(cudaSetDevice(k->s->ctx->device));
        cudaStream_t st = k->s->ctx->stream;
        nrc_kernel_attributes();
        upload_records(k, n, records, nullptr);
        DBuf<float> x, y;
        x.alloc(size_t(n) * 64); y.alloc(size_t(n) * 3);
        DebugIO io{k->records.p, n, x.p, y.p};
        const uint32_t tiles = (n + TILE - 1) / TILE;
        k_nrc_forward<DebugIO><<<std::min<uint32_t>(tiles, uint32_t(k->s->ctx->sms) * 4u), TILE, FWD_SMEM, st>>>(io, k->mlp_w.p, k->table.p, k->err.p);
        VKB_CUDA(cudaGetLastError());
        check_nrc_err(k);
        if (x_out) VKB_CUDA(cudaMemcpyAsync(x_out, x.p, size_t(n) * 64 * sizeof(float), cudaMemcpyDeviceToHost, st));
        VKB_CUDA(cudaMemcpyAsync(y_out, y.p, size_t(n) * 3 * sizeof(float), cudaMemcpyDeviceToHost, st));
        VKB_CUDA(cudaStreamSynchronize(st));
        x.release(); y.release();
    });
}

vkb_status vkb_debug_nrc_gradients(vkb_cache* k, uint32_t n, const float* records, const float* targets, float* mlp_grad, float* hash_grad,
                                   float* loss) {
    if (!k || !records || !targets || !mlp_grad || n == 0) return fail(VKB_INVALID_ARG, "null argument or no records");
    return guarded([&] {
        VKB_CUDA(cudaSetDevice(k->s->ctx->device));
        cudaStream_t st = k->s->ctx->stream;
        upload_records(k, n, records, targets);
        DBuf<float> g, h;
        g.alloc(MLP_PARAMS);
        if (hash_grad) h.alloc(HASH_PARAMS);
        float l = nrc_step(k, n, false, g.p, hash_grad ? h.p : nullptr);
        VKB_CUDA(cudaMemcpyAsync(mlp_grad, g.p, MLP_PARAMS * sizeof(float), cudaMemcpyDeviceToHost, st));
        if (hash_grad) VKB_CUDA(cudaMemcpyAsync(hash_grad, h.p, HASH_PARAMS * sizeof(float), cudaMemcpyDeviceToHost, st));
        VKB_CUDA(cudaStreamSynchronize(st));
        if (loss) *loss = l;
        g.release(); h.release();
    });
}

vkb_status vkb_debug_nrc_step(vkb_cache* k, uint32_t n, const float* records, const float* targets, float* loss) {
    if (!k || !records || !targets || n == 0) return fail(VKB_INVALID_ARG, "null argument or no records");
    return guarded([&] {
        VKB_CUDA(cudaSetDevice(k->s->ctx->device));
        upload_records(k, n, records, targets);
        float l = nrc_step(k, n, true, nullptr, nullptr);
        if (loss) *loss = l;
    });
}

}  // extern "C"
