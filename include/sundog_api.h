/* sundog_api.h — C ABI of the B200 path tracer (libsundog.so).
 *
 * The first block is the drop-in surface: the 27 entry points and four
 * structs that sundog's scene library (scenes/scenelib.py) binds with ctypes.
 * Names, argument meaning, return codes and struct layouts are identical to
 * sundog's src/sundog_api.h (cited per declaration), so existing scene files
 * run against this library unchanged.
 *
 * Conventions kept from the reference ABI (src/sundog_api.h:1-15):
 *   - scalars cross as double and are narrowed to float once, at entry;
 *   - "unset, use the renderer default" is NaN for doubles, NULL for
 *     vectors and -1 for tri-state ints;
 *   - set_* / validate / probe / render return 0 on success, 1 on error;
 *     add_* return an id >= 0, or -1 on error; scene_create returns NULL on
 *     error; the message of the last error on the calling thread is
 *     available from sundog_last_error();
 *   - call order is config/registries -> objects -> flames -> explicit
 *     lights -> render, which freezes the light list as
 *     [auto NEE area lights in object order][2 per flame][explicit lights].
 *
 * The second block holds additive entry points with no counterpart in the
 * reference; they extend, and never change, the layouts above.
 */
#ifndef SUNDOG_B200_API_H
#define SUNDOG_B200_API_H

#include <stddef.h>
#include <stdint.h>

#ifdef __cplusplus
#define SUNDOG_API extern "C" __attribute__((visibility("default")))
#else
#define SUNDOG_API __attribute__((visibility("default")))
#endif

#define SUNDOG_OK 0
#define SUNDOG_ERROR 1

/* ======================= drop-in surface (27 symbols) ===================== */

/* src/sundog_api.h:30 — thread-local message of the last failed call. */
SUNDOG_API const char* sundog_last_error(void);

typedef struct sundog_scene sundog_scene;
/* src/sundog_api.h:34-35 — handle lifetime; base_dir resolves relative asset
 * paths ("." when NULL or empty). */
SUNDOG_API sundog_scene* sundog_scene_create(const char* base_dir);
SUNDOG_API void sundog_scene_destroy(sundog_scene*);

/* src/sundog_api.h:38-52 — geometry kinds and transform-step kinds. */
enum {
  SUNDOG_GK_SPHERE = 0,
  SUNDOG_GK_RECT = 1,
  SUNDOG_GK_DISK = 2,
  SUNDOG_GK_CYLINDER = 3,
  SUNDOG_GK_PARABOLA = 4,
  SUNDOG_GK_MESH = 5,
};
enum {
  SUNDOG_XF_SCALE = 0,
  SUNDOG_XF_TRANSLATE = 1,
  SUNDOG_XF_ROTATE_X = 2,
  SUNDOG_XF_ROTATE_Y = 3,
  SUNDOG_XF_ROTATE_Z = 4,
};
#define SUNDOG_MAT_NONE (-1)    /* src/sundog_api.h:53 face passes rays through */
#define SUNDOG_MAT_DEFAULT (-2) /* src/sundog_api.h:54 back face = front face */

/* src/sundog_api.h:57-76 — configuration blocks. */
SUNDOG_API int sundog_set_render(sundog_scene*, int width, int height, int spp,
                                 int max_depth, double clamp, int64_t seed,
                                 double exposure, int transparent_shadows);
SUNDOG_API int sundog_set_camera(sundog_scene*, const double lookfrom[3],
                                 const double lookat[3], const double up[3],
                                 double vfov, double aperture, double focus_dist);
SUNDOG_API int sundog_set_background_solid(sundog_scene*, const double color[3]);
SUNDOG_API int sundog_set_background_gradient(sundog_scene*, const double horizon[3],
                                              const double zenith[3]);
SUNDOG_API int sundog_set_background_envmap(sundog_scene*, const char* file,
                                            double rotate_deg, double intensity,
                                            int importance);
SUNDOG_API int sundog_set_physics(sundog_scene*, const double gravity[3],
                                  double timestep, double max_time, double friction,
                                  double restitution, int pos_iters, int vel_iters,
                                  double sleep_threshold, double stop_time);

/* src/sundog_api.h:79-111 — texture / material / mesh registries. */
SUNDOG_API int sundog_add_texture_solid(sundog_scene*, const double color[3]);
SUNDOG_API int sundog_add_texture_checker(sundog_scene*, const double a[3],
                                          const double b[3], const double scale[2]);
SUNDOG_API int sundog_add_texture_grid(sundog_scene*, const double a[3],
                                       const double b[3], const double scale[2],
                                       double width);
SUNDOG_API int sundog_add_texture_image(sundog_scene*, const char* file, int srgb);
SUNDOG_API int sundog_add_material_lambert(sundog_scene*, const double color[3],
                                           int tex_id);
SUNDOG_API int sundog_add_material_metal(sundog_scene*, const double color[3],
                                         int tex_id, double roughness);
SUNDOG_API int sundog_add_material_dielectric(sundog_scene*, double ior,
                                              const double absorb[3],
                                              const double color[3], int tex_id,
                                              double roughness);
SUNDOG_API int sundog_add_material_emissive(sundog_scene*, const double color[3],
                                            int tex_id, double intensity,
                                            int two_sided);
SUNDOG_API int sundog_add_material_water(sundog_scene*, double ior,
                                         const double absorb[3], double wave_amp,
                                         double wave_freq, const double color[3]);
SUNDOG_API int sundog_add_material_plastic(sundog_scene*, const double color[3],
                                           int tex_id, double roughness);
SUNDOG_API int sundog_add_mesh(sundog_scene*, const char* obj_file,
                               int smooth_normals, const char* usemtl);

/* src/sundog_api.h:117-138 — objects. Byte layouts are load-bearing: the
 * ctypes mirrors in scenes/scenelib.py:724-734 must match. */
typedef struct {
  int32_t kind; /* SUNDOG_XF_* */
  double a, b, c;
} sundog_xform_step;

typedef struct {
  int32_t dynamic;
  double density;
  int32_t has_velocity, has_angular_velocity;
  double velocity[3], angular_velocity[3];
  double friction, restitution;
  double thickness;
} sundog_physics_body;

SUNDOG_API int sundog_add_object(sundog_scene*, int geom_kind, int mesh_id,
                                 int mat_front, int mat_back, int cutout_tex_id,
                                 const sundog_xform_step* steps, int num_steps,
                                 int nee, const sundog_physics_body* physics);

/* src/sundog_api.h:141-152 — flames and explicit lights. */
SUNDOG_API int sundog_add_flame(sundog_scene*, const double base[3], double height,
                                double radius, double intensity, double sigma,
                                double noise_scale, int64_t seed,
                                double light_intensity);
SUNDOG_API int sundog_add_point_light(sundog_scene*, const double position[3],
                                      const double intensity[3], double radius);
SUNDOG_API int sundog_add_distant_light(sundog_scene*, const double direction[3],
                                        const double radiance[3]);

/* src/sundog_api.h:155 — GPU-free checks (camera present). */
SUNDOG_API int sundog_scene_validate(sundog_scene*);

/* src/sundog_api.h:157-165 — device probe. This library has no OptiX: both
 * OptiX fields are reported as 0. */
typedef struct {
  char name[256];
  int32_t cc_major, cc_minor;
  int32_t driver_version, runtime_version;
  uint64_t total_mem_mb;
  uint32_t optix_header_version;
  uint32_t rtcore_version;
} sundog_device_info;
SUNDOG_API int sundog_probe(sundog_device_info* out);

/* src/sundog_api.h:167-179 — synchronous render of the scene. */
typedef struct {
  const char* out_path;
  const char* stats_path;
  const char* aov_albedo_path, *aov_normal_path;
  const char* scene_name;
  int32_t spp, width, height;
  int64_t seed;
  int32_t denoise, transparent_shadows;
  double clamp;
  double physics_time;
  int32_t quiet;
} sundog_render_options;
SUNDOG_API int sundog_render(sundog_scene*, const sundog_render_options*);

/* ===================== additive entry points (no reference) =============== */

/* Flame ray-march step count. The reference hard-codes 32 steps in both the
 * radiance and the shadow marcher; this sets a per-flame count (1..1024) that
 * both marchers use, default 32. Flames phase; returns 0/1. */
SUNDOG_API int sundog_set_flame_steps(sundog_scene*, int flame_id, int steps);

/* Extended render: same scene, same options, plus host buffers to receive the
 * film and a result record. Any pointer may be NULL. film_rgba receives
 * width*height float4 (linear radiance, running mean over all samples);
 * aov_albedo / aov_normal likewise (AOVs are accumulated only when one of the
 * two is non-NULL or the options name AOV paths). out_path may be NULL here,
 * in which case no image file is written. */
typedef struct {
  float* film_rgba;
  float* aov_albedo;
  float* aov_normal;
  int32_t chunk_spp;     /* samples per chunk (one persistent launch, or one
                            pass of the wavefront engine); <= 0 = automatic */
  int32_t repeat;        /* >1: re-render the film this many times and report
                            the fastest render loop (timing aid); 0/1 = once */
  int32_t guiding;       /* 1 = learned path guiding (see sundog_guiding_*) */
  int32_t sample_offset; /* first sample index: the render folds samples
                            [sample_offset, sample_offset + spp) */
  int32_t frame_spp;     /* samples of the whole frame this render is one block
                            of: the pixel strata follow it, so blocks rendered
                            apart (one per GPU) hold exactly the frame's
                            samples; <= 0 = this render's spp */
  int32_t engine;        /* path-tracing kernels: 0 = automatic (the
                            wavefront engine, guiding's training passes
                            included), 1 = persistent megakernel throughout,
                            2 = same as 0. Both engines give the same
                            samples. */
  int32_t shard_count;   /* > 1: render one tile shard of the frame, for one
                            GPU of shard_count: the 64x64 film tiles t
                            (row-major) with t % shard_count == shard_index.
                            Those pixels equal the whole-frame render's bit
                            for bit; the others stay 0. <= 1 = whole frame */
  int32_t shard_index;
} sundog_render_ext;

typedef struct {
  uint64_t rays_traced;      /* radiance + shadow traces (reference definition) */
  uint64_t paths;            /* camera samples traced */
  double render_ms;          /* render loop only (device work, synchronised) */
  double build_ms;           /* acceleration-structure + CDF build */
  double load_ms;            /* asset load (OBJ / HDR) */
  double total_ms;
  double mrays_per_sec;
  double samples_per_sec;
  uint64_t kernel_launches;  /* kernels this library launched in the render loop */
  double kernel_ms;          /* CUDA-event time of the path-tracing kernels only */
} sundog_render_result;

SUNDOG_API int sundog_render_ex(sundog_scene*, const sundog_render_options*,
                                const sundog_render_ext*, sundog_render_result*);

/* Resident render session: the load-time work of sundog_render (asset load,
 * CDFs, BVH build, uploads) done once, then any number of device-resident
 * renders of the same film. session_render runs on the given CUDA stream
 * (NULL = the session's own) and returns when the render is complete;
 * reset != 0 clears the film first. session_read copies film / AOVs
 * (width*height float4 each) to host memory. */
typedef struct sundog_session sundog_session;
typedef struct {
  int32_t width, height, spp, chunk_spp;
  int32_t grid, block;           /* persistent launch shape */
  uint64_t device_bytes;         /* device memory held by the session */
  uint64_t bvh_nodes, triangles, instances;
  int32_t tlas_depth, blas_depth;
  double load_ms, build_ms, setup_ms;
} sundog_session_stats;

SUNDOG_API sundog_session* sundog_session_create(sundog_scene*, const sundog_render_options*,
                                                 const sundog_render_ext*);
SUNDOG_API int sundog_session_render(sundog_session*, void* cuda_stream, int reset,
                                     sundog_render_result*);
SUNDOG_API int sundog_session_read(sundog_session*, float* film_rgba, float* aov_albedo,
                                   float* aov_normal);
SUNDOG_API int sundog_session_info(sundog_session*, sundog_session_stats*);
/* Device-to-device copy of the session's film (width*height float4 running
 * means, device memory the caller owns) on cuda_stream (NULL = default
 * stream); returns once the copy is queued. For gathering the tile shards of
 * a frame rendered on several GPUs (shard_count in sundog_render_ext) with
 * the caller's collective library. Returns 0/1. */
SUNDOG_API int sundog_session_copy_film(sundog_session*, void* film_device, void* cuda_stream);
SUNDOG_API void sundog_session_destroy(sundog_session*);

/* Traversal visit counts over one full render of the session (a counting
 * build of the path kernel, for the roofline's algorithmic bytes; never the
 * timed path). Leaves the film holding that render. */
typedef struct {
  uint64_t rays;          /* radiance + shadow traces */
  uint64_t box_tests;     /* child-box slab tests (2 per binary node visit) */
  uint64_t tri_tests;     /* ray/triangle tests */
  uint64_t quadric_tests; /* analytic quadric instance tests */
  uint64_t blas_entries;  /* mesh instances entered (object-space rays) */
  uint64_t trav_iters;    /* warp iterations of the traversal loop */
  uint64_t trav_lanes;    /* active lanes summed over those iterations */
  uint64_t loop_iters;    /* warp iterations of the path loop */
  uint64_t loop_lanes;    /* lanes running a path segment in them */
} sundog_trace_counts;
SUNDOG_API int sundog_session_trace_counts(sundog_session*, sundog_trace_counts*);
/* The same counting render with the two ray kinds apart: radiance rays
 * (camera and bounce rays, closest hit) in *radiance and shadow rays (any hit,
 * transparent crossings) in *shadow; `rays` of each is its traversal count and
 * loop_* are only filled for the radiance set (the path loop). No counterpart
 * in the reference. Returns 0/1. */
SUNDOG_API int sundog_session_trace_counts_split(sundog_session*, sundog_trace_counts* radiance,
                                                 sundog_trace_counts* shadow);

/* Per-stage device time of a session's wavefront renders (no counterpart in
 * the reference). With stage timing on, each later session_render records
 * CUDA events around every stage launch on its stream (read at the
 * synchronisation the engine makes once per iteration) and keeps, for the
 * last render: the summed milliseconds of the start, trace (radiance rays),
 * shade-A, shadow-ray and shade-B stages, the iterations, the radiance and
 * shadow rays traced and the stage launches. Megakernel renders leave it
 * zero. Returns 0/1. */
/* Denoised copy of the session's film (the replacement of the reference's
 * OptiX AI denoiser pass, src/denoise.cpp:18-53, with the same albedo and
 * normal guides): an edge-avoiding a-trous wavelet filter on the GPU. The
 * session must render AOVs (sundog_render_ext.aov_albedo or aov_normal set
 * at creation). out: width*height float4, host memory. sundog_render and
 * sundog_render_ex run the same filter when the scene or the options ask for
 * denoise, and write / return the denoised film. Returns 0/1. */
SUNDOG_API int sundog_session_denoise(sundog_session*, float* out);

/* The session's film as sundog's HDR output codes (no counterpart in the
 * reference; src/film.cpp:96-115 computes the same codes on the host before
 * its AVIF encode): x 2^exposure (exposure NaN = the scene's), BT.709 ->
 * BT.2020, linear 1.0 at 203 cd/m^2, SMPTE ST 2084 PQ, 12-bit code, encoded
 * on the device. out: width*height*3 uint16 (RGB, row 0 = top). sundog_render
 * writes the same codes for a ".png" out_path (16-bit, cICP BT.2020/PQ), and
 * for an ".avif" out_path beside it as ".png" (no AVIF encoder is linked).
 * Returns 0/1. */
SUNDOG_API int sundog_session_read_pq12(sundog_session*, double exposure, uint16_t* out);

/* Which builder makes the binary BVHs of later scene uploads (no counterpart
 * in the reference, whose optixAccelBuild runs on the device,
 * src/accel.cpp:46-121): device != 0 (the default) builds every mesh's BVH and
 * the instance BVH on the GPU; 0 uses the host binned-SAH builder. Both apply
 * the same split rules; the trees differ only in tie-breaking. Returns 0/1. */
SUNDOG_API int sundog_set_bvh_builder(int device);

/* Device-memory cache between calls (no counterpart in the reference).
 * Off by default: sundog_render / sundog_render_ex free every device buffer
 * they allocated before returning, and a destroyed session frees its own.
 * keep != 0: the per-sample radiance buffer (about 1 GiB) and the wavefront
 * path pool of a finished render stay allocated on their device for the next
 * render (saves their allocation and free per one-shot call) until
 * sundog_release_device_memory() or sundog_set_device_memory_cache(0), which
 * free them. Returns 0/1. */
SUNDOG_API int sundog_set_device_memory_cache(int keep);
SUNDOG_API int sundog_release_device_memory(void);

/* A sampling table of the session's scene as the device holds it (no
 * counterpart in the reference): which = 0 the environment's marginal CDF
 * (H + 1 floats), 1 its conditional CDFs (H rows of W + 1 floats), 2 + k the
 * area CDF of light k (triangles + 1 floats; empty unless light k is an
 * emissive mesh). Copies min(cap, length) floats to out (may be NULL) and
 * sets *count to the length. Returns 0/1. */
SUNDOG_API int sundog_session_table(sundog_session*, int which, float* out, size_t cap,
                                    size_t* count);

typedef struct {
  double start_ms, trace_ms, shade_a_ms, shadow_ms, shade_b_ms;
  uint64_t iterations, radiance_rays, shadow_rays, launches;
} sundog_stage_times;
SUNDOG_API int sundog_session_set_stage_timing(sundog_session*, int enable);
SUNDOG_API int sundog_session_stage_times(sundog_session*, sundog_stage_times*);

/* Allocation-free tile render (no counterpart in the reference). For callers
 * that cannot allocate device memory when they render, such as a serving
 * worker whose device memory is owned by another allocator or held to a fixed
 * budget: renders samples [sample_begin, sample_begin + sample_count) of the
 * pixel rectangle (x0, y0, w, h) of a resident session's image and folds them
 * in sample order into film_device, w*h float4 running means in device memory
 * the caller owns (zeros for sample_begin 0). Sample indices count from the
 * session's first sample (its sample_offset), so the pixels equal the same
 * pixels of a full render of the session. Sessions with learned guiding
 * enabled are rejected (plain samples only). Calls no cudaMalloc/cudaFree:
 * its scratch is a static 16 MiB device array in the library (held by every
 * GPU that loads it until exit), so w*h*sample_count may not exceed 1048576
 * (64x64 at 256 spp); larger requests fail. All calls share that array and it
 * keeps the last call's contents: calls that overlap on the GPU race,
 * serialise them. The first call on a device looks the array up (with that
 * device current) and should come before any stream capture. rays_out (host,
 * may be NULL): radiance + shadow traces; when given, the call waits for
 * completion. cuda_stream NULL = default stream. Returns 0/1. */
SUNDOG_API int sundog_session_render_tile_noalloc(sundog_session*, int x0, int y0, int w, int h,
                                                  int sample_begin, int sample_count,
                                                  float* film_device, uint64_t* rays_out,
                                                  void* cuda_stream);

/* Host<->device bytes moved by the library since load (uploads, downloads);
 * bench.py reads the per-step difference for its end-to-end record. */
SUNDOG_API void sundog_transfer_bytes(uint64_t* h2d, uint64_t* d2h);

/* Derived scene state as JSON (lights after NEE registration, object
 * transforms, materials, flames, settings). Writes at most cap bytes including
 * the terminating NUL; *needed receives the full length + 1. Returns 0/1. */
SUNDOG_API int sundog_scene_debug_json(sundog_scene*, char* buf, size_t cap,
                                       size_t* needed);

/* Device self-test of one hot-path function over a batch of inputs, for
 * parity tests against the CPU oracle. `which` selects the function (see
 * sundog_b200/csrc/selftest.cu); in/out are host arrays of documented
 * per-item layout; n is the item count. Returns 0/1. */
SUNDOG_API int sundog_selftest(int which, const void* in, int n, void* out,
                               size_t out_bytes);

/* ---- Learned path guiding (no counterpart in the reference) -------------
 * A small network (48 inputs: frequency-encoded position + normal; 3 hidden
 * layers of 64, ReLU; 8 von Mises-Fisher lobes out), trained on the GPU from
 * the renderer's own radiance samples and mixed into BSDF sampling by MIS,
 * so a guided render stays unbiased. A guided render traces its first
 * train_spp samples in passes of pass_spp; after each pass the network takes
 * steps_per_pass Adam steps and its mixture table is re-baked; the rest of
 * the samples use the final guide. Every sample goes to the film. */
typedef struct {
  int32_t train_spp;      /* samples whose paths train the network (32) */
  int32_t pass_spp;       /* samples per training pass (8) */
  int32_t steps_per_pass; /* Adam steps after each pass (64) */
  int32_t batch;          /* training records per step (16384) */
  float learning_rate;    /* Adam step size (5e-3) */
  float mix;              /* probability of drawing from the guide, [0, 1) (0.7) */
  uint64_t seed;          /* network initialisation and batch draws (1) */
  uint64_t record_cap;    /* training records kept per pass (4194304) */
} sundog_guiding_config;

typedef struct {
  uint64_t records;       /* records the last pass produced (may exceed the cap) */
  int32_t passes;         /* training passes so far */
  int32_t train_steps;    /* Adam steps so far */
  double train_ms;        /* CUDA-event time of training, summed */
  double bake_ms;         /* CUDA-event time of the mixture-table bakes, summed */
  double last_loss;       /* mean batch loss of the last pass */
  float box_lo[3], box_hi[3]; /* region the guide's grid covers */
} sundog_guiding_stats;

/* Fills *config with the defaults above. */
SUNDOG_API void sundog_guiding_defaults(sundog_guiding_config* config);
/* Turns guiding on (config NULL = defaults; the network starts untrained) or
 * off (enable 0) for the session's later renders. A render with reset != 0
 * retrains from scratch. sundog_render_ext.guiding = 1 at session creation
 * (or in sundog_render_ex) is the same as enabling it with the defaults.
 * Returns 0/1. */
SUNDOG_API int sundog_session_set_guiding(sundog_session*, int enable,
                                          const sundog_guiding_config* config);
SUNDOG_API int sundog_session_guiding_stats(sundog_session*, sundog_guiding_stats*);
/* The session's current network parameters (14576 floats, layout below). */
SUNDOG_API int sundog_session_guide_params(sundog_session*, float* params);
/* Training records of the last training pass (12 floats each: x, F/p, n, 0,
 * wi, 0): *count receives how many the pass kept; at most max_records are
 * copied to out (may be NULL). */
SUNDOG_API int sundog_session_guide_records(sundog_session*, float* out, uint64_t max_records,
                                            uint64_t* count);

/* The network's kernels on caller-given parameters, for parity checks
 * against a CPU restatement. params: 14576 floats (weight matrices row-major
 * [out][in]: W0 64x48, W1 64x64, W2 64x64, W3 48x64; then biases 64, 64, 64,
 * 48), rounded to BF16 for the weights. */
/* Initial parameters for a seed. */
SUNDOG_API int sundog_guide_init_params(uint64_t seed, float* params);
/* Raw network outputs (n x 40) for queries (n x 6: position in [0,1]^3,
 * normal). */
SUNDOG_API int sundog_guide_outputs(const float* params, const float* queries, int n,
                                    float* outputs);
/* Loss and its gradient (14576 floats, parameter layout) over n training
 * records (n x 12 floats: x, F/p, n, 0, wi, 0), all in one batch; box: guide
 * box origin (3) and 1/extent (3). */
SUNDOG_API int sundog_guide_gradients(const float* params, const float* records, int n,
                                      const float* box, float* grads, float* loss);

/* ---- Render server (no counterpart in the reference) ----------------------
 * Jobs (a scene, its size, spp and seed) are submitted from any thread. A
 * server thread admits them in arrival order when a job slot and enough free
 * device memory are available (jobs that fit pass one that does not), keeps
 * each scene's device data (BVH, CDFs, textures, meshes) resident and shared
 * by all jobs of that scene, and renders all admitted jobs together: each
 * iteration renders one batch of tile-passes (a tile x tile pixel rectangle
 * and a range of its samples) drawn from every active job, then folds those
 * samples into each job's film. Jobs arriving while others run
 * join at the next iteration. A job's film is the same alone or in any mix
 * of jobs, bit for bit; with engine 1 it is bit-identical to a
 * sundog_session_render of the same scene, size, spp and seed with the
 * megakernel engine (sundog_render_ext.engine = 1), and with engine 0 it
 * equals the wavefront engine's session render up to FP32 rounding (the same
 * per-path code compiled into other kernels). */
typedef struct sundog_server sundog_server;
typedef struct {
  int32_t max_jobs;            /* jobs on the device at once, 1..32 (16) */
  int32_t tile;                /* tile edge in pixels, a multiple of 8 (64) */
  int32_t pass_spp;            /* samples of a tile per tile-pass (8) */
  int32_t engine;              /* path-tracing kernels: 0 = wavefront (default),
                                  1 = persistent megakernel, 2 = same as 0 */
  uint64_t iteration_paths;    /* camera paths per batch (8388608) */
  uint64_t reserve_bytes;      /* device memory left free at admission (1 GiB) */
  uint64_t scene_cache_bytes;  /* scene data kept resident with no job using it (8 GiB) */
} sundog_server_config;

enum {
  SUNDOG_JOB_QUEUED = 0,
  SUNDOG_JOB_RUNNING = 1,
  SUNDOG_JOB_DONE = 2,
  SUNDOG_JOB_FAILED = 3,
  SUNDOG_JOB_CANCELLED = 4
};

typedef struct {
  int32_t state;               /* SUNDOG_JOB_* */
  int32_t width, height, spp;
  uint64_t paths_done, paths_total;
  double queued_ms;            /* submission -> admission */
  double latency_ms;           /* submission -> film on the host (final states) */
  char error[256];             /* reason for FAILED */
} sundog_job_status;

typedef struct {
  uint64_t jobs_submitted, jobs_done, jobs_failed, jobs_cancelled;
  uint64_t iterations;         /* batches rendered */
  uint64_t rays;               /* radiance + shadow traces of all jobs */
  uint64_t paths;              /* camera paths of all jobs */
  double busy_ms;              /* CUDA-event time of the iterations */
  double wall_ms;              /* since sundog_server_create */
  int32_t active_jobs, queued_jobs;
  uint64_t scenes_resident;
  uint64_t scene_bytes;        /* device memory held by resident scenes */
} sundog_server_statistics;

SUNDOG_API void sundog_server_defaults(sundog_server_config* config);
/* config NULL = defaults. Returns NULL on error (sundog_last_error). */
SUNDOG_API sundog_server* sundog_server_create(const sundog_server_config* config);
/* The same on a given device (0 .. sundog_device_count() - 1): the server's
 * thread, stream, pool and scene cache live there. One server per device is
 * how several GPUs serve together (sundog_b200/serve.py MultiServer places
 * each job on the device with the least queued work); servers and sessions
 * may share a device (a per-device lock orders their launches). Returns NULL
 * on failure. */
SUNDOG_API sundog_server* sundog_server_create_on_device(const sundog_server_config*,
                                                        int device);
/* CUDA devices visible to the library, or -1 when the runtime cannot tell. */
SUNDOG_API int sundog_device_count(void);
/* Queues a render of the scene (copied: the handle may be destroyed after the
 * call). options: width / height / spp / seed / transparent_shadows / clamp
 * overrides as in sundog_render (NULL = the scene's). film_rgba: host buffer
 * of width*height float4 receiving the film when the job is done (NULL = none;
 * must stay valid until the job ends). Returns the job id, or -1. */
SUNDOG_API int64_t sundog_server_submit(sundog_server*, sundog_scene*,
                                        const sundog_render_options* options, float* film_rgba);
SUNDOG_API int sundog_server_status(sundog_server*, int64_t job, sundog_job_status*);
/* Waits until the job is DONE, FAILED or CANCELLED (timeout_ms < 0: no
 * limit). Returns 0 when it is, 1 on timeout or error. */
SUNDOG_API int sundog_server_wait(sundog_server*, int64_t job, double timeout_ms,
                                  sundog_job_status*);
/* Cancels a queued or running job (between iterations); its film is not
 * written. Returns 0, or 1 if the job is unknown or already final. */
SUNDOG_API int sundog_server_cancel(sundog_server*, int64_t job);
SUNDOG_API int sundog_server_stats(sundog_server*, sundog_server_statistics*);
/* Cancels what is left, stops the server thread, frees device memory. */
SUNDOG_API void sundog_server_destroy(sundog_server*);

#endif /* SUNDOG_B200_API_H */
