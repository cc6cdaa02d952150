/*
 * vkb.h -- C ABI of the B200 render backend for vork's `std/path` integrator.
 *
 * The reference has no FFI or plugin registry for its integrator: the path pass is
 * recorded by `passes::path::record` (crates/vork-render/src/passes/path.rs:539-559)
 * over a 30-binding wgpu layout (passes/path.rs:323-384), after the acceleration
 * structures are built by `rt::Rays::new` / `FrameRays::new` / `rt::encode`
 * (crates/vork-render/src/rt.rs:1098,1339,1387).  The entry points below are what a
 * Rust shim in `passes::path` would bind instead of that dispatch.  Plain C types
 * only: pointers, sizes and POD structs.  No call traps on the device; every device
 * wait and traversal loop is bounded and reports through vkb_status / vkb_stats.
 */
#ifndef VKB_H
#define VKB_H

#include <stdint.h>
#include <stddef.h>

#ifdef __cplusplus
extern "C" {
#endif

#define VKB_ABI_VERSION 7u

/* Error model: FailureKind exit categories of crates/vork-render/src/failure.rs:21-100,
 * reduced to what a render call can report. */
typedef enum vkb_status {
    VKB_OK = 0,
    VKB_INVALID_ARG = 1,      /* malformed descriptor or profile (failure.rs "scene") */
    VKB_OUT_OF_MEMORY = 2,    /* device allocation refused (gpu_memory.rs device_limit) */
    VKB_DEVICE_TIMEOUT = 3,   /* a bounded device loop or host wait ran out */
    VKB_NONFINITE = 4,        /* non-finite input (an image given to vkb_display) */
    VKB_INTERNAL = 5,         /* CUDA runtime error; message via vkb_last_error() */
    VKB_UNSUPPORTED = 6       /* a profile feature outside the built subset */
} vkb_status;

/* Ray-event bits, crates/vork-slang/src/registry.rs:186-191. */
#define VKB_RAY_CAMERA 1u
#define VKB_RAY_SHADOW 2u
#define VKB_RAY_DIFFUSE 4u
#define VKB_RAY_SPECULAR 8u
#define VKB_RAY_TRANSMISSION 16u
#define VKB_RAY_VOLUME 32u
/* Light record words, registry.rs:161,322-328,344. */
#define VKB_LIGHT_CONTRIBUTION_WORD 0
#define VKB_LIGHT_LINK_WORD 1
#define VKB_LIGHT_RAY_WORD 2
#define VKB_LIGHT_RAY_LINK_WORD 3
#define VKB_LIGHT_RAY_SHADOWED 1u
#define VKB_LIGHT_RAY_SHADOWED_BY_ALL 2u
#define VKB_LIGHT_LINK_ALL 64u

/* One triangle mesh in object space (the BLAS input of rt.rs:1098-1289). */
typedef struct vkb_mesh {
    const float* positions;    /* num_vertices*3 */
    const float* normals;      /* num_vertices*3 smooth normals (NULL: face normals) */
    const uint32_t* indices;   /* num_triangles*3, counter-clockwise = front */
    uint32_t num_vertices;
    uint32_t num_triangles;
} vkb_mesh;

/* OpenPBR 1.1.1 inputs used by the path subset (crates/vork-scene/openpbr-params.md:22-30);
 * every other OpenPBR input is held at its specification default. */
typedef struct vkb_material {
    float base_weight;
    float base_color[3];
    float base_metalness;
    float specular_weight;
    float specular_color[3];
    float specular_roughness;
    float specular_ior;
    /* Emission: radiance emission_color x emission_luminance on the front side (both sides
     * when double sided), finite and >= 0.  Every instance drawn with emission_luminance > 0
     * and a non-black colour is a mesh light source: its triangles are sampled by the mesh
     * next-event strategy (area x luminance power, half uniform; emitters.rs:22-44,
     * emitter_mesh_proposal.slang) and its hits are weighed against it by MIS
     * (path.slang:1121-1167,1580-1591). */
    float emission_luminance;
    float emission_color[3];
    uint32_t flags;            /* bit 1: double sided (registry FLAG_DOUBLE_SIDED) */
} vkb_material;

/* Analytic light record, byte-for-byte `Light` of crates/vork-render/src/lights.rs:13-24
 * (8 shadow words + 8 float4 = 160 B). kind = position[3]: 0 sun, 1 point, 2 spot, 3 area. */
typedef struct vkb_light {
    uint32_t shadow_offsets[8];
    float position[4];
    float direction[4];
    float radiance[4];
    float params[4];
    float emitter_u[4];
    float emitter_v[4];
    float emission[4];
    float projection[4];
} vkb_light;

/* Pinhole camera: the Frame uniform subset path_camera_ray reads
 * (crates/vork-render/src/lib.rs:288-320; shaders/vork_prelude.slang:95-108). */
typedef struct vkb_camera {
    float eye[3];
    float right[3];
    float up[3];
    float forward[3];
    float proj_x;       /* projection[0][0]: Frame.projection.y */
    float proj_y;       /* projection[1][1]: Frame.projection.x */
    float near_plane;   /* Frame.params.x */
    float far_plane;    /* Frame.params.y */
    uint32_t width;
    uint32_t height;
} vkb_camera;

/* Constant world light (Frame.radiance / background, path.slang:961-983). */
typedef struct vkb_environment {
    float radiance[3];         /* constant environment radiance seen by every ray */
    float exposure;            /* Frame.radiance.w, multiplies the finished sample */
    float background[3];       /* camera-miss colour when camera_sees_environment == 0 */
    uint32_t camera_sees_environment;
} vkb_environment;

/* Image environment (the image term of path_environment, path.slang:961-983; the
 * proposal of crates/vork-render/src/environment.rs:573-620 and
 * shaders/environment_proposal.slang:1-49; environment_next_event, path.slang:1096-1120).
 * A lat-long linear RGBA image: direction d (after the rotation) maps to
 * equirect_uv(d) = (atan2(d.z, d.x)/2pi + 1/2, atan2(|d.xz|, d.y)/pi) (vork_prelude.slang:78-85),
 * texel row 0 at the +y pole, sampled bilinearly, wrapping in longitude
 * (vork_prelude.slang:306-330).  Radiance of a direction = environment.radiance +
 * image x strength x color.  With strength > 0 every surface vertex also samples the
 * environment (next-event estimation from a proposal proportional to the image's 3x3
 * smoothed, alpha-weighted luminance times texel solid angle), MIS-weighted against the
 * BSDF, and escaping rays are weighted the other way. */
typedef struct vkb_environment_image {
    const float* rgba;         /* width*height*4 (copied at vkb_scene_create) */
    uint32_t width, height;    /* each >= 1 */
    float strength;            /* Frame.environment.x: 0 turns the image and its strategy off */
    float color[3];            /* Frame.environment_color.rgb */
    float rotation[9];         /* row-major 3x3 R: a world direction d looks up equirect_uv(normalize(d R));
                                  all zero means the identity */
} vkb_environment_image;

typedef struct vkb_scene_desc {
    const vkb_mesh* meshes;
    uint32_t num_meshes;
    uint32_t num_instances;
    const float* instance_rows;       /* num_instances*12: rows of the 3x4 object->world matrix (Object.model, lib.rs:226-240) */
    const uint32_t* instance_mesh;    /* num_instances */
    const uint32_t* instance_material;/* num_instances */
    const vkb_material* materials;
    uint32_t num_materials;
    const vkb_light* lights;
    uint32_t num_lights;
    vkb_camera camera;
    vkb_environment environment;
    uint32_t tlas_builder;            /* VKB_TLAS_LBVH or VKB_TLAS_PLOC (no reference counterpart: the
                                         reference's TLAS is built by the graphics driver) */
    const vkb_environment_image* environment_image;   /* NULL: the constant environment alone */
    uint32_t blas_format;             /* VKB_BLAS_WIDE4 (default) or VKB_BLAS_WIDE8 */
    uint32_t blas_builder;            /* VKB_BLAS_BUILD_SAH (default), _LBVH or _PLOC */
} vkb_scene_desc;

/* BLAS builders: a binned-SAH tree on the host threads (the trees that trace fastest), or
 * on the GPU the TLAS's own Morton-ordered builders, LBVH or PLOC (install in milliseconds
 * for scenes that must start rendering at once; 4-wide nodes only). */
#define VKB_BLAS_BUILD_SAH 0u
#define VKB_BLAS_BUILD_LBVH 1u
#define VKB_BLAS_BUILD_PLOC 2u

/* BLAS node formats (the TLAS is 4-wide in both): 4-wide FP32 child planes (one 128-byte
 * line per node), or compressed 8-wide nodes (80 bytes: child boxes as bytes on a per-node
 * grid; Ylitie, Karras & Laine, HPG 2017).  Scenes of the two formats render alone or in
 * batches of their own format; the server takes 4-wide scenes. */
#define VKB_BLAS_WIDE4 0u
#define VKB_BLAS_WIDE8 1u

/* TLAS builders, both over the instance boxes in Morton order and both refittable:
 * Karras LBVH (fast build, siblings adjacent in memory) or PLOC (lower surface area
 * cost; Meister & Bittner 2018). */
#define VKB_TLAS_LBVH 0u
#define VKB_TLAS_PLOC 1u

/* PathSettings (path.slang:54; passes/path.rs:16-28,576-607). */
typedef struct vkb_profile {
    uint32_t samples;          /* exposure sample count (Frame.temporal.y) */
    uint32_t first_sample;     /* first exposure index rendered by this call (resume/progressive) */
    uint32_t sample_count;     /* samples rendered by this call (0 = samples - first_sample) */
    uint32_t seed;             /* sampling.y */
    uint32_t bounces[4];       /* max, diffuse, glossy, transmission */
    uint32_t transparent;      /* limits.z */
    uint32_t caustics;         /* limits.w bits: 1 glossy after diffuse, 2 transmission after diffuse */
    float clamp_direct;        /* clamp.x (0 = off) */
    float clamp_indirect;      /* clamp.y (0 = off) */
    float light_threshold;     /* adaptive.z: stochastic light-sample kill */
    uint32_t adaptive;         /* 1: adaptive stopping (path.slang:1792-1837), vkb_render of a whole exposure only */
    uint32_t wave_samples;     /* samples per wavefront wave (0 = automatic: as many as up to 64 Mi path
                                  slots hold for one render, the context's capacity in a batch; 1 with
                                  adaptive stopping) */
    uint32_t flags;            /* VKB_PROFILE_* measurement switches (0 for production renders) */
    float adaptive_threshold;  /* adaptive.x: relative standard error to stop at (0 = 0.01) */
    uint32_t adaptive_min_samples; /* sampling.w: samples before stopping (0 = max(16, sqrt(samples))) */
} vkb_profile;

/* Measurement switches of vkb_profile.flags (no reference counterpart: timing hooks). */
#define VKB_PROFILE_TIME_KERNELS 1u        /* CUDA events around every closest-hit trace launch
                                              (its waves then run one after another) */
#define VKB_PROFILE_COUNT_TRAVERSAL 2u     /* instrumented traversal: node and triangle visits */
#define VKB_PROFILE_SERIAL_WAVES 16u       /* one wave after another on one stream (default: the
                                              waves of a single-job render alternate between two
                                              streams and wavefronts, so one wave's sparse last
                                              bounces overlap the next wave's first ones; the
                                              image is the same either way) */
/* Wave scheduling of several jobs (vkb_render_batch flags / vkb_server_config.flags):
 * batches pack each job's remaining samples before the next job (throughput: fewer
 * scenes per wave keep their BVHs in L2) unless VKB_BATCH_FAIR; servers give the waves to
 * the admitted requests with the least remaining work first (latency), or one sample of
 * every request per wave with VKB_BATCH_FAIR, or pack like batches with VKB_BATCH_PACKED. */
#define VKB_BATCH_FAIR 4u
#define VKB_BATCH_PACKED 8u

/* Render output: linear RGBA32F mean image (resolve.slang:162-191). */
typedef struct vkb_output {
    float* rgba;               /* width*height*4 */
    uint32_t on_device;        /* 1: rgba (and the guide planes) are device pointers on the context's GPU */
    uint32_t* primary_ids;     /* optional, width*height*2 (instance, triangle) of sample first_sample; 0xffffffff on miss */
    /* Optional denoiser guides (path.slang:1549-1571 written per sample, summed per pixel as
     * path.slang:1956-1963 does), as means over the rendered samples, width*height*4 each:
     * guide_albedo = the camera hit's response to a uniform white world (diffuse + reflected,
     * clamped to [0,1]) in rgb and its coverage (fraction of samples that hit) in w;
     * guide_normal = the camera hit's shading normal in xyz, 0 in w.  A miss or a dropped
     * sample adds zero.  vkb_render / vkb_render_view without adaptive stopping only. */
    float* guide_albedo;
    float* guide_normal;
} vkb_output;

typedef struct vkb_stats {
    uint64_t paths;            /* camera samples traced */
    uint64_t extension_rays;   /* closest-hit rays */
    uint64_t shadow_rays;      /* any-hit rays */
    uint64_t dropped_path_samples;  /* non-finite samples zeroed (path.slang:1946-1955) */
    uint64_t dropped_light_samples; /* non-finite contributions dropped (sample_clamp.slang) */
    uint64_t traversal_overflows;   /* bounded-stack or iteration-cap exits (error, never a trap) */
    float render_ms;           /* device time of the wavefront, CUDA events */
    float build_ms;            /* device time of the last acceleration-structure build */
    float trace_ms;            /* VKB_PROFILE_TIME_KERNELS: summed closest-hit trace kernel time */
    uint32_t trace_launches;   /* closest-hit trace launches in this render */
    uint32_t kernel_launches;  /* every kernel this library launched for this render */
    uint64_t nodes_visited;    /* VKB_PROFILE_COUNT_TRAVERSAL: closest-hit BVH node visits */
    uint64_t triangles_tested; /* closest-hit triangle tests */
    uint64_t instances_entered;/* closest-hit TLAS leaf (instance) entries */
    uint64_t shadow_nodes_visited;
    uint64_t shadow_triangles_tested;
    uint64_t blas_nodes_visited;   /* closest-hit node visits inside instance BLASes (the rest are TLAS) */
    float cache_ms;            /* VKB_PROFILE_TIME_KERNELS, vkb_render_cached: radiance-cache query kernel time */
    uint64_t cache_queries;    /* vkb_render_cached: paths answered by the radiance cache */
    uint64_t samples_skipped;  /* adaptive stopping: pixel samples not traced (stopped pixels) */
} vkb_stats;

typedef struct vkb_ctx vkb_ctx;
typedef struct vkb_scene vkb_scene;

/* Library identity and the last error message of this thread. */
uint32_t vkb_abi_version(void);
const char* vkb_last_error(void);

/* Renderer::new (crates/vork-render/src/lib.rs:726) for one CUDA device.  Also bakes
 * the BRDF lookup atlas (shaders/environment.slang:28-108, src/environment.rs:312-323). */
vkb_status vkb_open(int device, vkb_ctx** out);
vkb_status vkb_close(vkb_ctx* ctx);

/* Renderer::install + FrameRays::new (lib.rs:1322-1470; rt.rs:1098-1385): uploads the
 * descriptor (copied; the caller may free it on return) and builds every BLAS and the TLAS. */
vkb_status vkb_scene_create(vkb_ctx* ctx, const vkb_scene_desc* desc, vkb_scene** out);
vkb_status vkb_scene_destroy(vkb_scene* scene);

/* rt::encode / rebuild_tlas (rt.rs:1387-1476): new object->world rows for every
 * instance (host pointer, num_instances*12 floats). policy 0: refit, or rebuild once
 * the changed object bytes accumulated since the last rebuild reach a quarter of the
 * object buffer (the reference's rule); 1: always rebuild; 2: always refit (the
 * topology of the last rebuild is kept; boxes and matrices are replaced). */
vkb_status vkb_scene_update_instances(vkb_scene* scene, const float* rows, uint32_t num_instances, int policy);
/* The same with rows already in device memory of the context's GPU (no host copy). */
vkb_status vkb_scene_update_instances_device(vkb_scene* scene, const float* device_rows, uint32_t num_instances, int policy);

/* A frame slot over an installed scene (FrameRays::new per frame, rt.rs:1339-1385, over the
 * BLASes of one install; InstalledScene::create_frame_slot, crates/vork-render/src/install.rs:3303):
 * a scene that shares `base`'s meshes, BLASes, materials, lights and light tree and owns its
 * own instance rows and TLAS, starting from base's current rows.  Updating a fork's
 * instances (vkb_scene_update_instances*) leaves base and other forks unchanged, so frames
 * of an animated sequence render while other requests use base.  Forks of forks are
 * refused; base must outlive its forks (vkb_scene_destroy refuses a scene with live forks). */
vkb_status vkb_scene_fork(vkb_scene* base, vkb_scene** out);

/* passes::path::record + resolve (passes/path.rs:539-724; resolve.slang:162-191): renders
 * samples [first_sample, first_sample+sample_count) of `profile` and writes the mean
 * over them. stats may be NULL. */
vkb_status vkb_render(vkb_scene* scene, const vkb_profile* profile, vkb_output* out, vkb_stats* stats);
/* vkb_render through `camera` (its resolution included) instead of the scene's own camera
 * (the per-shot camera of Shot::render, crates/vork-render/src/shot.rs:31-72); NULL = the
 * scene's camera.  out->rgba holds camera->width * camera->height * 4 floats. */
vkb_status vkb_render_view(vkb_scene* scene, const vkb_camera* camera, const vkb_profile* profile, vkb_output* out,
                           vkb_stats* stats);

/* Batched previews: many render jobs (each its own installed scene of this context,
 * profile and output) share every wavefront wave; each wave's kernel sequence is
 * replayed from a captured CUDA graph.  No reference counterpart: vork renders one
 * shot per Renderer at a time (crates/vork-render/src/shot.rs:374).  Per-job results
 * equal vkb_render's for the same scene and profile.  flags: VKB_PROFILE_* switches. */
typedef struct vkb_job {
    vkb_scene* scene;
    vkb_profile profile;
    vkb_output out;
} vkb_job;
vkb_status vkb_render_batch(vkb_ctx* ctx, vkb_job* jobs, uint32_t njobs, uint32_t flags, vkb_stats* stats);

/* Autotuner of the wavefront: times one sample of `jobs` for every candidate wave
 * capacity (path slots per wave: 2, 4, 8, 16, 32 Mi) and trace/shade grid (32, 64, 128
 * blocks per SM) and keeps the fastest for this context's later renders. */
typedef struct vkb_tune_result {
    uint32_t tried;
    uint32_t best_blocks_per_sm;
    uint64_t best_capacity;
    float best_ms;
    uint32_t blocks_per_sm[16];
    uint64_t capacity[16];
    float ms[16];
} vkb_tune_result;
vkb_status vkb_autotune(vkb_ctx* ctx, vkb_job* jobs, uint32_t njobs, vkb_tune_result* out);

/* Serving with continuous batching (vkb_job_submit/poll of the boundary plan): requests
 * queue on the host; every vkb_server_step admits queued requests at the wave boundary
 * (FIFO) while `max_jobs` and the device-memory budget allow (resident scenes + the
 * shared wavefront + 32 bytes per pixel of every admitted request), runs one wave over
 * all admitted requests, and copies finished images to their host buffers.  No
 * reference counterpart beyond vork's one-request-at-a-time session
 * (crates/vork-cli/src/session.rs:1-60). */
typedef struct vkb_server vkb_server;
typedef struct vkb_server_config {
    uint64_t memory_budget_bytes;  /* 0: unbounded */
    uint32_t max_jobs;             /* admitted requests at once (job-table entries) */
    uint32_t flags;                /* VKB_PROFILE_* switches for every wave */
    uint64_t wave_capacity;        /* path slots per wave (0: the context's autotuned value) */
    double aging_paths_per_s;      /* shortest-remaining-work waves: a request's remaining paths count as
                                      reduced by this rate times the seconds since its admission, so a
                                      large request is not overtaken forever (0: pure shortest first) */
} vkb_server_config;
typedef struct vkb_server_status {
    uint32_t queued, running, finished;   /* finished: requests completed by this step */
    uint32_t reserved;
    uint64_t used_bytes, peak_bytes;      /* device bytes under the budget now / at peak */
} vkb_server_status;
vkb_status vkb_server_create(vkb_ctx* ctx, const vkb_server_config* cfg, vkb_server** out);
/* host_rgba (width*height*4 floats) must stay valid until the request is done. */
vkb_status vkb_server_submit(vkb_server* server, vkb_scene* scene, const vkb_profile* profile, float* host_rgba, uint64_t* id);
/* vkb_server_submit through `camera` (NULL: the scene's camera); host_rgba holds
 * camera->width * camera->height * 4 floats.  The scene (and a fork's base) must stay
 * installed until the request is done. */
vkb_status vkb_server_submit_view(vkb_server* server, vkb_scene* scene, const vkb_camera* camera, const vkb_profile* profile,
                                  float* host_rgba, uint64_t* id);
vkb_status vkb_server_step(vkb_server* server, vkb_server_status* status);
/* state: 0 queued, 1 running, 2 done (its host_rgba holds the mean image). */
vkb_status vkb_server_poll(vkb_server* server, uint64_t id, int* state);
vkb_status vkb_server_destroy(vkb_server* server);

/* Installed-scene facts: sizes, device bytes of the scene structures, and the TLAS
 * update history of vkb_scene_update_instances (rebuilds vs refits, rt.rs:1465-1476). */
typedef struct vkb_scene_info_t {
    uint64_t num_instances;
    uint64_t num_triangles;
    uint64_t scene_bytes;      /* device bytes of meshes, BLAS, TLAS and instance records */
    uint64_t tlas_rebuilds;
    uint64_t tlas_refits;
    uint64_t motion_bytes;     /* changed object bytes accumulated since the last rebuild */
    float build_ms;            /* device time of the last TLAS build or refit */
    uint32_t reserved;
    /* Install cost (Renderer::install + Rays::new, lib.rs:1322-1470, rt.rs:1098-1289) of
     * vkb_scene_create (of vkb_scene_fork for a fork): */
    float install_ms;          /* wall time of the whole call */
    float blas_host_ms;        /* of which the host binned-SAH builds and 4-wide collapses of every BLAS */
    float upload_ms;           /* of which the host->device copies (meshes, BLAS, records, instances) */
    float tlas_ms;             /* of which the first TLAS build (device time) */
} vkb_scene_info_t;
vkb_status vkb_scene_info(vkb_scene* scene, vkb_scene_info_t* out);

/* The CUDA stream (cudaStream_t) every kernel of this context is launched on, so a
 * caller can record its own events on it. */
void* vkb_ctx_stream(vkb_ctx* ctx);
/* Kernel launches issued so far for this scene (renders and acceleration-structure builds). */
uint64_t vkb_scene_launch_count(vkb_scene* scene);

/* Render without allocating (no counterpart in the reference: it exists for callers
 * that cannot allocate device memory while they render, e.g. a host renderer whose
 * own memory manager owns every device allocation, or a serving loop with a fixed
 * footprint).  Same semantics, results and stats as vkb_render, but every wavefront
 * queue, accumulator and counter lives in one fixed device array of
 * VKB_NOALLOC_SCRATCH_MIB MiB that each GPU loading the library holds until process
 * exit; no cudaMalloc or cudaFree is called.  One sample per wave needs about 252 bytes
 * per pixel with host output (16 accumulator + 220 queue + 16 staging; ~133k pixels),
 * 260 with host output and primary_ids (~129k), 236 with device output (~142k), 244
 * with device output and primary_ids (~137k); larger images are rejected with
 * VKB_INVALID_ARG.  Each call looks up the array's device address with the device
 * current: make the first call on a device before any stream capture.  All calls share
 * the array and it keeps the previous call's contents: calls that overlap on the GPU
 * (another stream, another thread) race, so serialise them.  VKB_PROFILE_TIME_KERNELS
 * is ignored (no events). */
#define VKB_NOALLOC_SCRATCH_MIB 32u
vkb_status vkb_render_noalloc(vkb_scene* scene, const vkb_profile* profile, vkb_output* out, vkb_stats* stats);

/* --- Test and measurement entry points (no reference counterpart beyond the cited tests) --- */

/* Sampler groups, bit-exact with path_sampler.slang:53-95 (the harness of
 * src/path_sampler.rs:266-276): for each i, the four 32-bit scrambled fractions of
 * group groups[i] at pixel (px[i],py[i]), index[i], count, stream. out: n*4 u32 (host). */
vkb_status vkb_debug_sampler_groups(vkb_ctx* ctx, uint32_t n, const uint32_t* px, const uint32_t* py,
                                    const uint32_t* index, const uint32_t* groups, uint32_t count,
                                    uint32_t stream, uint32_t* out_bits);
/* The BRDF atlas as baked on the device: 128*2240*4 floats (host), fp16 values widened. */
vkb_status vkb_debug_brdf_lut(vkb_ctx* ctx, float* out);
/* 30-bit Morton codes of the scene's TLAS build (instance AABB centroids over the scene
 * box), in instance order: num_instances u32 (host). */
vkb_status vkb_debug_tlas_morton(vkb_scene* scene, uint32_t* out);
/* 30-bit Morton codes of one mesh's BLAS build (triangle centroids over the mesh box). */
vkb_status vkb_debug_blas_morton(vkb_scene* scene, uint32_t mesh, uint32_t* out);
/* ---- Display stage (crates/vork-render/shaders/resolve.slang:13,140-160 and the std/standard
 * view, libraries/std/standard.slang:1-33 with libraries/std/view.slang:3-25): linear Rec.709
 * RGBA (a vkb_render result) -> display code values for an sRGB, Display P3, Rec.2100 PQ or
 * Rec.2100 HLG destination, quantised to 8 or 16 bits like the resolve stage's unorm store
 * (no dither, as the reference's Render::dither = false) or returned as float codes. */
#define VKB_DISPLAY_SRGB 0u
#define VKB_DISPLAY_P3 1u
#define VKB_DISPLAY_REC2100_PQ 2u
#define VKB_DISPLAY_REC2100_HLG 3u
typedef struct vkb_display_params {
    uint32_t display;          /* VKB_DISPLAY_* */
    float exposure;            /* stops (std/standard `exposure`, default 0) */
    float gamma;               /* creative gamma on the code values (std/standard `gamma`, default 1) */
    float peak_luminance;      /* Rec.2100 destinations: display peak, cd/m^2 (1000) */
    float reference_white;     /* Rec.2100 destinations: cd/m^2 of unit scene white (100) */
    uint32_t bits;             /* 8 (uchar4), 16 (ushort4) or 32 (float4 code values) per pixel */
    uint32_t unassociate;      /* 1: colour divided by alpha first (resolve.slang:140-145) */
    uint32_t reserved;
} vkb_display_params;
/* width x height RGBA float pixels (host or device) -> `out` (host or device), row-major.
 * Non-finite input pixels are written as zero and the call returns VKB_NONFINITE. */
vkb_status vkb_display(vkb_ctx* ctx, const vkb_display_params* params, const float* rgba, int rgba_on_device, uint32_t width,
                       uint32_t height, void* out, int out_on_device);

/* ---- Learned radiance cache (no reference counterpart: vork has no learned path
 * component).  A multiresolution hash encoding (16 levels x 2^19 entries x 2 FP16
 * features) and a 5-layer, 64-wide BF16 MLP with FP32 accumulation on the tensor cores,
 * trained online on the tracer's own path vertices; renders through it stop each path at
 * `query_vertex` and add throughput x the cached outgoing radiance there.  One cache per
 * installed scene; it owns its parameters, optimizer state and training buffers. */
typedef struct vkb_cache vkb_cache;
typedef struct vkb_cache_config {
    uint32_t train_records;    /* training vertices per vkb_cache_train call (default 65536) */
    uint32_t train_steps;      /* optimizer steps per vkb_cache_train call, over interleaved minibatches of its records (default 4) */
    uint32_t query_vertex;     /* path vertex (0 = camera hit) answered by the cache (default 2) */
    uint32_t seed;             /* parameter initialisation and training-path sampling */
    float lr_mlp, lr_hash;     /* Adam learning rates (defaults 2e-3, 1e-2) */
    float beta1, beta2, eps;   /* Adam moments (defaults 0.9, 0.99, 1e-10) */
} vkb_cache_config;
typedef struct vkb_cache_stats {
    uint64_t steps;            /* optimizer steps taken so far */
    uint64_t records;          /* training vertices of the last call */
    float loss;                /* mean relative-L2 loss of the last step */
    float train_ms;            /* device time of the last call (paths + steps) */
    float paths_ms;            /* of which the training paths and the training-set compaction */
    float steps_ms;            /* of which the optimizer steps */
    float host_ms;             /* wall time of the call on the host */
} vkb_cache_stats;
vkb_status vkb_cache_create(vkb_scene* scene, const vkb_cache_config* config, vkb_cache** out);
vkb_status vkb_cache_destroy(vkb_cache* cache);
/* One online training round: trace about train_records / 2 training paths through the
 * scene's camera at reduced resolution (one sample, a fresh seed each call, the
 * profile's bounce limits), take every vertex from 1 on as a training record whose
 * target is the path's radiance from there on, and run train_steps optimizer steps,
 * step i over records i, i + train_steps, ... (every record once per round). */
vkb_status vkb_cache_train(vkb_cache* cache, const vkb_profile* profile, vkb_cache_stats* stats);
/* vkb_render through the cache: paths stop at query_vertex and add throughput x the
 * cached outgoing radiance there (the plain render is the fallback and the judge of its
 * error).  Same output and stats as vkb_render. */
vkb_status vkb_render_cached(vkb_cache* cache, const vkb_profile* profile, vkb_output* out, vkb_stats* stats);
/* Test hooks of the network itself.  Parameters as FP32: MLP row-major [out][in] per
 * layer (4 x 64x64 then 16x64, rows 3..15 of the last zero), hash table [level][entry][feature]. */
#define VKB_NRC_MLP_PARAMS 17408u
#define VKB_NRC_HASH_PARAMS 16777216u
vkb_status vkb_debug_nrc_set_params(vkb_cache* cache, const float* mlp, const float* hash);
vkb_status vkb_debug_nrc_get_params(vkb_cache* cache, float* mlp, float* hash);
/* records: n x 16 floats (position normalised to [0,1]^3, outgoing direction, shading
 * normal, roughness, metalness, base colour, 2 pad).  x_out: n x 64 network inputs (as
 * BF16 values), y_out: n x 3 raw outputs. */
vkb_status vkb_debug_nrc_forward(vkb_cache* cache, uint32_t n, const float* records, float* x_out, float* y_out);
/* Gradients of the mean relative-L2 loss over n records against targets (n x 3), no
 * update: mlp_grad (VKB_NRC_MLP_PARAMS), hash_grad (VKB_NRC_HASH_PARAMS, may be NULL), loss. */
vkb_status vkb_debug_nrc_gradients(vkb_cache* cache, uint32_t n, const float* records, const float* targets, float* mlp_grad,
                                   float* hash_grad, float* loss);
/* One optimizer step over n records (the same step vkb_cache_train takes). */
vkb_status vkb_debug_nrc_step(vkb_cache* cache, uint32_t n, const float* records, const float* targets, float* loss);

/* TLAS check (test hook, no reference counterpart): walks the installed TLAS from its
 * root and reports whether every instance leaf is reached exactly once and every stored
 * child box contains its subtree (*valid = 1), the deepest leaf, and the tree's surface
 * area cost (sum of node and leaf box areas over the root box area, unit costs). */
vkb_status vkb_debug_tlas_stats(vkb_scene* scene, double* sah_cost, uint32_t* max_depth, uint32_t* valid);
/* Closest hits of n world rays (origin xyz, dir xyz, tmax per ray; host arrays):
 * out_t[n], out_ids[n*2] (instance, triangle; 0xffffffff on miss), out_uv[n*2]. */
vkb_status vkb_debug_trace(vkb_scene* scene, uint32_t n, const float* rays7, float* out_t,
                           uint32_t* out_ids, float* out_uv);
/* Occlusion of n world rays by the shadow-ray traversal (straight_shadow_transmittance's
 * ACCEPT_FIRST_HIT_AND_END_SEARCH query, shaders/path.slang:630-684: first hit ends the
 * walk, no back-face culling): out_occluded[n] = 1 when a surface lies within tmax. */
vkb_status vkb_debug_occluded(vkb_scene* scene, uint32_t n, const float* rays7, uint32_t* out_occluded);

#ifdef __cplusplus
}
#endif
#endif
