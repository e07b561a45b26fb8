/* nd_march.h - C ABI of the B200 distance-estimator sphere-tracing pass.
 *
 * This header is the drop-in boundary between NumericDream's host code and the
 * CUDA kernels.  It is plain C (no CUDA or torch types) so that Zig can import it
 * with addTranslateC exactly like the reference's own translate-C shims
 * (build.zig:379-423, e.g. src/bindings/webgpu_shim.h), and Python with ctypes.
 *
 * What each entry point replaces in the reference:
 *   nd_formula_register / nd_formula_find
 *       FractalRenderer.rebuild / rebuildAsync  (src/gpu/fractal_renderer.zig:2927, :2951)
 *       + assembleShaderSource (fractal_renderer.zig:725-760) + stampFormulaCodes (:2882):
 *       a formula source becomes an integer formula code.  Formula files are
 *       translated from WGSL to CUDA at build time; registering a source looks up
 *       its compiled code by the source hash, as CodeTable.find does (:585-590), and
 *       a source the build did not compile is translated and compiled then, as the
 *       reference's compileWorker does (:1609).
 *   nd_formula_params
 *       formula.parseFormulaParams / CustomParam  (src/app/formula.zig:6-13, :147-157)
 *   nd_view_desc
 *       the per-view part of `Uniforms` (fractal_renderer.zig:228-346): camera
 *       basis, resolution, tile_scale/tile_bias (tileTransform :852-863), max_steps,
 *       max_dist, epsilon_coefficient/floor, refine_fast/hq, march_verify,
 *       high_quality, and one FractalInstance (code, params, orbit trap).
 *   nd_march_forward
 *       FractalRenderer.renderToImage -> renderTile -> drawSlot(fs_simple)
 *       (fractal_renderer.zig:3548, :3741-3828; template.wgsl:4522-4538): march every
 *       pixel of every view and write the G-buffer (frag_out, template.wgsl:3768-3774:
 *       depth = t or 0 on a miss, normal xyz with w = hit).
 *   nd_last_stats
 *       the hot-spot DE-evaluation counter (template.wgsl:363-378) and the wavefront
 *       per-pass profile (src/gpu/wavefront.zig:280-411), as totals.
 *   nd_autotune, nd_graph_*
 *       no reference counterpart; the reference picks sub-tile sizes by a pacing
 *       heuristic (ExportPacer, fractal_renderer.zig:991) instead.
 *   nd_orbit_view
 *       FreeCamera's basis (src/app/camera.zig:98-112) for an orbit pose.
 *   nd_march_backward
 *       no reference counterpart (the reference has no gradients).
 *
 * Conventions: every call returns an nd_status and never aborts.  The caller owns
 * every buffer; G-buffer pointers are DEVICE pointers, descriptors are HOST
 * pointers.  Work is enqueued on the given CUDA stream (a cudaStream_t passed as
 * void*, NULL = legacy default stream) and is asynchronous with respect to the
 * host unless the call says otherwise.  A context is not thread-safe; distinct
 * contexts are.
 */
#ifndef ND_MARCH_H
#define ND_MARCH_H

#include <stddef.h>
#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

#define ND_ABI_VERSION 4
#define ND_MAX_PARAMS 16          /* fractal_renderer.zig:47 */
#define ND_PARAM_NAME_LEN 24      /* CustomParam.name [24:0]u8, formula.zig:7 */

typedef int32_t nd_status;
enum {
  ND_OK = 0,
  ND_ERR_INVALID = 1,      /* bad argument or descriptor */
  ND_ERR_COMPILE = 2,      /* formula source rejected or not compiled into this build */
  ND_ERR_OOM = 3,          /* device allocation failed */
  ND_ERR_TIMEOUT = 4,      /* the device watchdog stopped a launch */
  ND_ERR_CUDA = 5,         /* any other CUDA error */
  ND_ERR_UNSUPPORTED = 6,  /* valid request this build cannot serve */
  ND_ERR_NOT_FOUND = 7     /* unknown formula name or id */
};

typedef int32_t nd_formula_id;
typedef struct nd_ctx nd_ctx;
typedef struct nd_graph nd_graph;

/* One @param slider (CustomParam, src/app/formula.zig:6-13). */
typedef struct nd_param_info {
  char name[ND_PARAM_NAME_LEN];
  float min_value;
  float max_value;
  float default_value;
  int32_t integral;
} nd_param_info;

/* Orbit trap of one instance (OrbitTrap template.wgsl:1207-1214, enums
 * src/app/scene_state.zig:134-189) and its colour-strip mapping
 * (orbit_trap_to_strip template.wgsl:2025-2035). */
enum { ND_TRAP_POINT = 0, ND_TRAP_SPHERE = 1, ND_TRAP_BOX = 2, ND_TRAP_CROSS = 3, ND_TRAP_TORUS = 4 };
enum { ND_TRAP_MIN = 0, ND_TRAP_MAX = 1, ND_TRAP_AVERAGE = 2, ND_TRAP_LAST = 3, ND_TRAP_ITERATION = 4 };
typedef struct nd_trap_desc {
  float center[3];
  int32_t shape;
  float box[3];
  int32_t mode;
  float radius;
  float tube;
  float span;     /* strip mapping: x = v / max(span, 1e-4) + offset */
  float offset;
  int32_t repeat; /* 0 clamp, 1 repeat, 2 mirror */
  int32_t reserved;
} nd_trap_desc;

enum { ND_NORMAL_TETRA = 0, ND_NORMAL_CENTRAL = 1 };

/* nd_view_desc.flags: ND_VIEW_DIR64 keeps ray directions in FP64 (set
 * automatically when |right| or |up| < 1e-3, i.e. fields of view under ~0.1 deg).
 * ND_VIEW_EXACT_HIT runs the hit bisection for its whole refine budget instead of
 * stopping once the bracket is narrower than eps(t) (the reference's stop): the hit
 * distance then follows the root of DE = eps(t) to bracket / 2^budget and is a
 * smooth function of the view and the parameters, which gradients need. */
enum { ND_VIEW_DIR64 = 1, ND_VIEW_EXACT_HIT = 2 };

/* One view: a camera, a frame (or a tile of it) and one fractal instance. */
typedef struct nd_view_desc {
  double cam_pos[3];      /* ray origin, FP64 (u.camera_pos) */
  double fwd[3];          /* u.camera_forward */
  double right[3];        /* u.camera_right, already scaled by tan(fov_y/2) */
  double up[3];           /* u.camera_up, already scaled by tan(fov_y/2) */
  int32_t width;          /* full frame size: aspect = width / height */
  int32_t height;
  int32_t tile_x;         /* rendered rectangle of the frame (tileTransform) */
  int32_t tile_y;
  int32_t tile_w;
  int32_t tile_h;
  nd_formula_id formula;  /* from nd_formula_find / nd_formula_register */
  int32_t spp;            /* primary rays per pixel; 1 = pixel centre, >1 = jittered */
  uint64_t seed;          /* jitter seed (counter-based, per ray) */
  float params[ND_MAX_PARAMS]; /* packed @param values (packParams, formula.zig:104) */
  nd_trap_desc trap;
  int32_t max_steps;      /* u.max_steps */
  float max_dist;         /* u.max_dist (24 in the reference UI) */
  float eps_coef;         /* u.epsilon_coefficient: eps(t) = coef * t + floor */
  float eps_floor;        /* u.epsilon_floor */
  int32_t refine_budget;  /* u.refine_fast or u.refine_hq (bisection / verify budget) */
  int32_t march_verify;   /* u.march_verify */
  int32_t high_quality;   /* u.high_quality */
  float hq_footprint_px;  /* u.hq_footprint_budget_px */
  int32_t normal_mode;    /* ND_NORMAL_TETRA (template.wgsl:1783) or ND_NORMAL_CENTRAL */
  float normal_h_coef;    /* central differences: h = coef * t (0 -> eps(t)) */
  int32_t shadow;         /* 1: one shadow ray per hit toward light_dir */
  float light_dir[3];     /* direction TO a LIGHT_GLOBAL light (normalised by the library) */
  float shadow_k;         /* soft-shadow sharpness k */
  float step_safety;      /* instance step safety, clamped to [0.001, 1] */
  int32_t flags;          /* ND_VIEW_* bits */
  /* Empty-space accelerator (cs_build_accel template.wgsl:5412-5431, accel_skip
   * :428-447, cascade placement src/gpu/accel.zig:32-56): a camera-centred cascade of
   * accel_levels grids of accel_res^3 safe skip distances, built by the library for
   * this view before its march.  accel_res 0 = off; otherwise clamped to 16..160 and
   * rounded down to a multiple of 4, levels to 1..8 (reference defaults 64, 6, 0.92). */
  int32_t accel_res;
  int32_t accel_levels;
  float accel_safety;     /* every recorded skip is multiplied by this */
  /* The formula image of a formula that declares `// @image` (read through
   * image_info / image_sample, template.wgsl:1111-1191; HeightMaps, src/gpu/height_maps.zig):
   * DEVICE pointer to image_width x image_height texels of 4 words as nd_image_prepare
   * writes them, and the image's per-channel slope bound from nd_image_prepare.
   * NULL: no image (the formula sees size 0, as the reference does with none loaded). */
  const uint32_t* image_texels;
  int32_t image_width;
  int32_t image_height;
  float image_slope[4];
} nd_view_desc;

/* A scene of up to four fractal instances combined by distance (scene_de,
 * template.wgsl:1756-1779), each with its own formula, parameters, placement
 * (instance_local: transpose(frame) * (p - offset) / scale, tpl:1611-1615; DE factor
 * min|scale| * clamp(step_safety), tpl:1617-1620), combine mode with the previous
 * instances (combine_de, tpl:1708-1730) and optional hybrid mixins (eval_mixed,
 * tpl:1321-1392: iterations cycle through hybrid_base_iters steps of the base formula,
 * then each mixin's steps; the base formula finalises), plus up to 16 spherical carves
 * (apply_carves, tpl:1741-1753).  Mirrors FractalInstance / MixinParams
 * (tpl:106-141); the per-instance colours are a shading concern and not here. */
#define ND_MAX_INSTANCES 4  /* MAX_INSTANCES tpl:22 */
#define ND_MAX_MIXINS 3     /* MAX_MIXINS tpl:23 */
#define ND_MAX_CARVES 16    /* MAX_CARVES tpl:32 */
enum {
  ND_COMBINE_UNION = 0,
  ND_COMBINE_SMOOTH_MIN = 1,
  ND_COMBINE_SMOOTH_MAX = 2,
  ND_COMBINE_SMOOTH_INV_MAX = 3,
  ND_COMBINE_SMOOTH_MIN_LIN = 4,
  ND_COMBINE_SMOOTH_MIN_NLIN = 5,
  ND_COMBINE_SMOOTH_MIX = 6
};

typedef struct nd_mixin_desc {
  nd_formula_id formula;
  int32_t iterations;              /* steps of this mixin per hybrid cycle */
  float params[ND_MAX_PARAMS];
} nd_mixin_desc;

typedef struct nd_instance_desc {
  nd_formula_id formula;
  int32_t hidden;                  /* 1: skipped by scene_de */
  float params[ND_MAX_PARAMS];
  float offset[3];
  float scale[3];                  /* per axis; |scale| floored at 0.001 */
  float frame[9];                  /* rotation matrix, three columns (u.instances[i].frame) */
  float step_safety;
  float blend_k;                   /* combine blend radius (<= 1e-4: hard) */
  int32_t combine_mode;            /* ND_COMBINE_*, with the instances before it */
  int32_t mixin_count;             /* 0: the plain formula; 1..3: hybrid */
  int32_t hybrid_base_iters;
  int32_t hybrid_total_iters;
  nd_mixin_desc mixins[ND_MAX_MIXINS];
  nd_trap_desc trap;
} nd_instance_desc;

typedef struct nd_scene_desc {
  int32_t instance_count;          /* 1..4 */
  int32_t carve_count;             /* 0..16 */
  nd_instance_desc instances[ND_MAX_INSTANCES];
  float carves[ND_MAX_CARVES][4];  /* sphere centre xyz, radius w */
} nd_scene_desc;

/* G-buffer of one forward call.  Rays of view v occupy [ray_offset(v), +rays(v)),
 * views in call order; rays(v) = spp * tile_w * tile_h and the ray index inside a
 * view is sample * tile_w * tile_h + y * tile_w + x.  Every pointer may be NULL
 * except depth. */
typedef struct nd_gbuffer {
  float* depth;       /* t at the hit, 0 on a miss (R32F depth target) */
  float* normal;      /* 4 floats per ray: unit normal, w = 1 on a hit */
  float* trap;        /* orbit-trap value of the DE evaluation at the hit point */
  uint32_t* steps;    /* probe steps (MarchResult.steps; max_steps on a miss) */
  uint32_t* iters;    /* formula iterations that changed the carry, at the hit */
  float* shade;       /* Lambert grey level (simple_geometry, template.wgsl:4492) */
  float* shadow;      /* shadow-ray visibility in [0, 1] (1 without a shadow ray) */
  double* depth64;    /* t in FP64 */
  uint32_t* evals;    /* DE evaluations spent on this ray */
  uint16_t* normal_half; /* the normal as the reference's RGBA16F target: 4 IEEE halves per ray,
                            w = 1 on a hit (8-byte aligned) */
} nd_gbuffer;

enum { ND_KERNEL_AUTO = 0, ND_KERNEL_PLAIN = 1, ND_KERNEL_PERSISTENT = 2 };

typedef struct nd_march_opts {
  int32_t kernel;            /* ND_KERNEL_*; AUTO = the tuned kernel, else the persistent one, but
                                the plain launch for one view with no more rays than the
                                persistent grid has threads (nothing to refill) */
  int32_t block;             /* persistent march: threads per block, 64, 128 or 256 (0 = tuned, else 128) */
  int32_t blocks_per_sm;     /* persistent kernel residency: > 0 that many (at most what fits), < 0 that
                                many fewer than fit, 0 = tuned default (as many as fit) */
  int32_t refill_threshold;  /* persistent: refill a warp once this many lanes idle (0 = tuned, else 6;
                                2 for an FP64 DE) */
  int32_t de_precision;      /* 32 (default) or 64: float type of the DE itself */
  int32_t watchdog_ms;       /* device watchdog per launch (0 = 10000 ms) */
  int32_t accel_chain;       /* accelerator jumps a ray takes per pass of the persistent
                                march before it waits for the next pass (0 = 4, < 0 = no
                                limit); the march itself is unchanged */
  int32_t reserved;
} nd_march_opts;

typedef struct nd_stats {
  uint64_t rays;
  uint64_t de_evals;        /* all DE evaluations: march, normals, shadows and trap pass */
  uint64_t march_evals;     /* primary march probes + refinement */
  uint64_t normal_evals;
  uint64_t shadow_evals;
  uint64_t trap_evals;      /* one DE with the orbit trap per hit (when trap/iters are requested) */
  uint64_t hits;
  uint64_t refills;         /* persistent kernel: warp refills */
  uint32_t timeouts;        /* watchdog expiries */
  uint32_t kernel;          /* kernel that ran (ND_KERNEL_PLAIN / _PERSISTENT) */
  double march_ms;          /* device time of the march kernels of the last nd_march_forward
                               (CUDA events on its stream; 0 after a graph launch) */
  double shade_ms;          /* device time of its shade passes (normals, shadows, orbit trap) */
  uint64_t accel_voxels;    /* accelerator grid cells built (one DE evaluation each, not in de_evals) */
  double accel_ms;          /* device time of the accelerator grid builds */
} nd_stats;

typedef struct nd_tune_result {
  int32_t block;
  int32_t blocks_per_sm;
  int32_t refill_threshold;
  int32_t kernel;
  double rays_per_s;
} nd_tune_result;

/* ---- library ---- */
int32_t nd_abi_version(void);
const char* nd_status_string(nd_status s);

/* ---- formulas (build-time translated) ---- */
nd_status nd_formula_count(int32_t* n);
nd_status nd_formula_find(const char* name, nd_formula_id* out);
nd_status nd_formula_name(nd_formula_id id, char* out, size_t out_len);
/* A formula source (WGSL) to a formula id.  A source compiled into the build (same
 * bytes) is found by its hash.  Any other source is compiled now: the build's
 * translator and nvcc turn it into a small library of its forward kernels (march,
 * surface and shadow passes, DE at points; FP32 and FP64 DE; no accelerator, lite
 * shading or adjoint for it), which is loaded and gets the next id (name
 * "user_<hash>"); this takes seconds, like the reference's shader compile, so call it
 * from a worker thread as the reference does.  Needs a Python interpreter with this
 * package (ND_PYTHON, default python3) and nvcc; temporary files go under ND_RTC_DIR
 * (default /tmp).  A source the translator or nvcc refuses returns ND_ERR_COMPILE
 * with the message in err.  Thread-safe (one compile at a time). */
nd_status nd_formula_register(const char* wgsl_src, size_t len, nd_formula_id* out, char* err, size_t err_len);
nd_status nd_formula_params(nd_formula_id id, nd_param_info* out, int32_t* n);
nd_status nd_view_defaults(nd_formula_id id, nd_view_desc* out);

/* ---- context ---- */
nd_status nd_ctx_create(int32_t device, nd_ctx** out);
nd_status nd_ctx_destroy(nd_ctx* ctx);
nd_status nd_last_error(const nd_ctx* ctx, char* out, size_t out_len);
nd_status nd_last_stats(nd_ctx* ctx, nd_stats* out); /* synchronises the last forward's stream */

/* ---- marching ---- */
nd_status nd_count_rays(const nd_view_desc* views, int32_t nviews, int64_t* total);
/* Returns once the call's work is enqueued on `stream`.  A context keeps two calls'
 * view tables, so a call blocks the host only until the call two back has finished on
 * the device; calls on different streams run one after the other on the device. */
nd_status nd_march_forward(nd_ctx* ctx, const nd_view_desc* views, int32_t nviews,
                           const nd_march_opts* opts, const nd_gbuffer* out, void* stream);
/* Times the launch configurations of the march on these views (writing into
 * scratch_out): the plain per-view launch, and the persistent march at 64, 128 and
 * 256 threads per block x as many resident blocks per SM as fit or two fewer x
 * refill thresholds 3..12; each candidate's time is the median of three runs with
 * the L2 cache flushed before each.  The candidates run the FP32 DE; the winner is
 * kept for the call's formula sets on this GPU and the FP32 DE (later FP32 forwards
 * with opts fields 0 use it; FP64-DE forwards keep the defaults).
 * result->blocks_per_sm is the resident count the march runs with. */
nd_status nd_autotune(nd_ctx* ctx, const nd_view_desc* views, int32_t nviews,
                      const nd_gbuffer* scratch_out, nd_tune_result* result);
/* The autotuner's winners on disk: a JSON array of entries keyed by GPU name, formula
 * set, a hash of the formula sources and the DE precision, so that a later process
 * starts tuned.  No
 * counterpart in the reference (it paces sub-tiles by a heuristic instead, ExportPacer,
 * fractal_renderer.zig:991).  load: ND_ERR_NOT_FOUND when the file does not exist;
 * *loaded (nullable) receives the number of entries read. */
nd_status nd_tune_cache_save(const char* path);
nd_status nd_tune_cache_load(const char* path, int32_t* loaded);
nd_status nd_graph_capture(nd_ctx* ctx, const nd_view_desc* views, int32_t nviews,
                           const nd_march_opts* opts, const nd_gbuffer* out, void* stream, nd_graph** graph);
nd_status nd_graph_launch(nd_graph* graph, void* stream);
nd_status nd_graph_destroy(nd_graph* graph);

/* An orbit camera: position = target + dist * (cos(pitch) sin(yaw), sin(pitch),
 * -cos(pitch) cos(yaw)) (angles in radians), looking at target, with FreeCamera's
 * basis (src/app/camera.zig:98-112: right = normalize(forward x up), up = right x
 * forward) scaled by tan(fov_y/2).  The pose the adjoint differentiates. */
typedef struct nd_orbit_camera {
  double target[3];
  double yaw;
  double pitch;
  double dist;
  double world_up[3];
  double fov_y_deg;
} nd_orbit_camera;

/* Fill view->cam_pos/fwd/right/up from an orbit camera. */
nd_status nd_orbit_view(const nd_orbit_camera* cam, nd_view_desc* view);

/* nd_march_forward for scenes of several instances.  view_scene[i] >= 0 marches
 * views[i] against scenes[view_scene[i]] (HOST array of nscenes); -1 uses the view's
 * own single instance (formula, params, trap, step_safety).  Every formula of a call
 * (instances, mixins and the single-instance views) must lie in one compiled formula
 * group (ND_ERR_UNSUPPORTED otherwise; ND_GROUPS at build time adds groups); scenes run
 * on the persistent kernel.  At a hit the G-buffer's trap and iteration count are those
 * of the visible instance with the smallest DE there.  Replaces renderTile with a
 * multi-instance Uniforms write (fractal_renderer.zig:3063, instances at tpl:114-141). */
nd_status nd_march_forward_scenes(nd_ctx* ctx, const nd_view_desc* views, int32_t nviews,
                                  const int32_t* view_scene, const nd_scene_desc* scenes, int32_t nscenes,
                                  const nd_march_opts* opts, const nd_gbuffer* out, void* stream);
/* nd_graph_capture for a scene call: the graph owns device copies of the view and
 * scene tables, so the caller may change or free views, view_scene and scenes after
 * the capture; replays march the captured scenes. */
nd_status nd_graph_capture_scenes(nd_ctx* ctx, const nd_view_desc* views, int32_t nviews,
                                  const int32_t* view_scene, const nd_scene_desc* scenes, int32_t nscenes,
                                  const nd_march_opts* opts, const nd_gbuffer* out, void* stream,
                                  nd_graph** graph);

/* Gradient of an image loss with respect to formula @params and the orbit pose.
 * No counterpart in the reference (it has no gradients).  views/cams (HOST) are the
 * forward call's views and their orbit cameras (view i must have been filled from
 * cams[i]); fwd (DEVICE) the forward's G-buffer, of which depth64 and normal are
 * read; dL_dshade (DEVICE, one float per ray) is dLoss/d(shade) for the Lambert
 * grey level the forward wrote.  For each view the call ADDS to dL_dtheta (DEVICE,
 * nviews x (nparams + 3) doubles) the gradient with respect to
 * params[param_idx[0..nparams-1]] (nparams <= 4), then yaw, pitch, dist.
 * dshade_dtheta (DEVICE, nullable) receives per G-buffer slot the nparams + 3
 * derivatives of that ray's shade (0 for misses and back-lit rays); when it is
 * given, dL_dtheta and dL_dshade may be NULL.
 * Implicit differentiation at each hit: dt/dtheta = -(dDE/dtheta) / (grad DE . d - eps
 * coef), through the central-difference normal and the Lambert term; visibility
 * (silhouette) changes are not differentiated.  opts (nullable) selects the dual
 * numbers' precision, de_precision 32 (default) or 64; its other fields are unused.
 * Needs a directional light (light_dir), central-difference normals and no shadow
 * ray; other views return ND_ERR_UNSUPPORTED.  Synchronises the stream. */
nd_status nd_march_backward(nd_ctx* ctx, const nd_view_desc* views, const nd_orbit_camera* cams, int32_t nviews,
                            const int32_t* param_idx, int32_t nparams, const nd_gbuffer* fwd,
                            const float* dL_dshade, double* dL_dtheta, double* dshade_dtheta,
                            const nd_march_opts* opts, void* stream);

/* Forward march that allocates nothing: no cudaMalloc, no cudaFree, no context.
 * No counterpart in the reference.  For callers that cannot allocate device
 * memory (a host whose allocator owns the device, a render thread where an
 * allocation may synchronise the device, loops that must not allocate after
 * start-up).  Runs the persistent kernel on the current device and the given
 * stream; its scratch (view table, work counters, statistics) is a fixed array of
 * about 28 KB inside the library, present on every GPU that loads it.
 * Limits: at most 64 views and 2^31-1 rays per call; trap and iters outputs are
 * not available here (they need per-ray scratch) and return ND_ERR_UNSUPPORTED.
 * The call cannot be captured into a CUDA graph (it copies the view table from its
 * own stack frame): on a capturing stream it returns ND_ERR_UNSUPPORTED.  The first
 * call in a CUDA context looks up the array's device address.  Every call shares the one array: calls
 * that overlap on the GPU (different streams, or host threads) race, so serialise
 * them.  views is a HOST array; the G-buffer pointers are DEVICE pointers.  The
 * call returns once the work is enqueued; a failure's message is kept per host
 * thread (nd_march_forward_noalloc_stats reads it). */
nd_status nd_march_forward_noalloc(const nd_view_desc* views, int32_t nviews, const nd_march_opts* opts,
                                   const nd_gbuffer* out, void* stream);

/* Statistics of the last nd_march_forward_noalloc call on the current device (rays,
 * DE evaluations, hits, refills, watchdog expiries), read from the library's
 * scratch array once `stream`'s work is done (synchronises the stream; allocates
 * nothing).  Returns ND_ERR_TIMEOUT when the device watchdog stopped the march
 * (opts->watchdog_ms): the G-buffer slots of the rays it did not finish are then
 * not written.  err (nullable) receives the message of the calling thread's last
 * failed nd_march_forward_noalloc call, or of the timeout.  No counterpart in the
 * reference, like the entry point it reports on. */
nd_status nd_march_forward_noalloc_stats(void* stream, nd_stats* out, char* err, size_t err_len);

/* DE of view->formula (with view->params and view->trap) at n points: pts is a
 * DEVICE array of 3n doubles; de, trap (nullable) and iters (nullable) are DEVICE
 * arrays of n.  Each point runs the formula wrapper of the reference (carry =
 * (pos, 1), de_iterations() x de_step with the orbit trap, de_finalize;
 * fractal_renderer.zig:490-512) in FP32 (de_precision 32) or FP64 (64). */
nd_status nd_de_points(nd_ctx* ctx, const nd_view_desc* view, int64_t n, const double* pts, double* de,
                       double* trap, uint32_t* iters, int32_t de_precision, void* stream);

/* Lite shading of a forward call's hits (shade_lite, template.wgsl:4424-4444, as
 * render_lite draws a hit :4446-4458): the material from the view's colour strip
 * (sample_gradient :2003-2023 at orbit_trap_to_strip :2025-2035 of the ray's orbit
 * trap), ambient occlusion (calc_ao :1825-1840), and every light's Lambert and
 * Blinn-Phong terms (light_sample_ex :2178-2190 for point and global lights),
 * times 1 - Fresnel (fresnel_schlick :3424-3430).  No shadows, as in the reference's
 * lite pass.  Misses take the background colour (the reference's sky is out of
 * this pass's scope).  Colour stops are sorted by position, as the reference's
 * host does (sortedColorOrder, scene_state.zig:98-108). */
#define ND_MAX_COLOR_STOPS 16  /* MAX_COLOR_STOPS tpl:24 */
#define ND_MAX_LIGHTS 8        /* MAX_LIGHTS tpl:27 */
enum { ND_LIGHT_POINT = 0, ND_LIGHT_GLOBAL = 1 };
typedef struct nd_color_stop {
  float color[3];
  float position;    /* along the strip, 0..1 */
  float glossiness;  /* 0..1: specular weight and power mix(4, 128, g) */
  float ior;         /* Fresnel index (>= 1 used) */
  float reserved[2];
} nd_color_stop;
typedef struct nd_light {
  float color[3];
  float brightness;
  float position_or_direction[3]; /* point: position; global: direction to the light */
  int32_t type;                   /* ND_LIGHT_POINT / ND_LIGHT_GLOBAL */
} nd_light;
typedef struct nd_lite_desc {
  int32_t color_count;            /* 0: the default material */
  int32_t light_count;
  int32_t ambient_occlusion;      /* 1: calc_ao (5 DE evaluations per hit); 0: none */
  int32_t specular;               /* 1: Blinn-Phong term on */
  float background[3];
  int32_t reserved;
  nd_color_stop colors[ND_MAX_COLOR_STOPS];
  nd_light lights[ND_MAX_LIGHTS];
} nd_lite_desc;

/* Lite shading of the views of an earlier nd_march_forward with the same views:
 * in holds its depth64, normal and trap (device); lite one descriptor per view
 * (host); rgba (device, 4 floats per ray in G-buffer order) receives the colour
 * and w = 1 on a hit, 0 on a miss.  Views without a scene (see below for scenes). */
nd_status nd_shade_lite(nd_ctx* ctx, const nd_view_desc* views, int32_t nviews, const nd_lite_desc* lite,
                        const nd_gbuffer* in, float* rgba, void* stream);

/* Lite shading after nd_march_forward_scenes (the same views, view_scene and
 * scenes): a scene view's material is hit_material's (template.wgsl:2128-2155):
 * each visible instance's colour stops at its own trap strip, blended instance by
 * instance with combine_de's weight; its ambient occlusion samples the scene.
 * instance_colors holds ND_MAX_INSTANCES descriptors per scene (scene-major; only
 * their colour stops are read); lite[i] gives view i's lights, switches and
 * background (and the colours of a view without a scene). */
nd_status nd_shade_lite_scenes(nd_ctx* ctx, const nd_view_desc* views, int32_t nviews, const int32_t* view_scene,
                               const nd_scene_desc* scenes, int32_t nscenes, const nd_lite_desc* lite,
                               const nd_lite_desc* instance_colors, const nd_gbuffer* in, float* rgba, void* stream);

/* The empty-space accelerator grid of one view (its own formula; accel_res > 0),
 * as nd_march_forward builds it before the view's march (cs_build_accel,
 * template.wgsl:5412-5431): grid is a DEVICE array of capacity floats that receives
 * levels * res^3 safe skip distances ([level][z][y][x]); prm (HOST, 32 floats)
 * receives the cascade placement (corner xyz, cell size per cascade, zeros past the
 * last); *count the number of floats.  Synchronous. */
nd_status nd_accel_grid(nd_ctx* ctx, const nd_view_desc* view, int32_t de_precision, float* grid, int64_t capacity,
                        float* prm, int64_t* count);

/* A scene file (.dream JSON, version <= 12; src/app/scene_file.zig) as one view and
 * one scene: the camera (FreeCamera position / forward / up; right = forward x up,
 * 90 degree vertical field of view), the march settings of the bench export
 * (render_settings: max_steps, max_dist and MarchPrecision, high quality on), and up
 * to four instances with their formulas (by file stem; an empty path is the built-in
 * Mandelbulb), @param values (by name, over the formula's defaults), placement,
 * combine mode, mixins and orbit trap.  width / height <= 0 take the file's
 * export size.  *needs_scene = 0 when the view alone describes the scene (one
 * visible instance at the identity placement, no mixins): render it with
 * nd_march_forward; otherwise with nd_march_forward_scenes (view_scene = {0}).
 * Lights, fog, sky, materials, warps and particles are not read.  The message of a
 * failure goes to err. */
nd_status nd_scene_file_load(const char* json, size_t len, int32_t width, int32_t height, nd_view_desc* view,
                             nd_scene_desc* scene, int32_t* needs_scene, char* err, size_t err_len);

/* The lite-shading descriptor of a scene file: instance `instance`'s colour stops
 * (position, color, glossiness, ior), the visible point and global lights (a global
 * light's direction, a point light's position; ray lights are left out), ambient
 * occlusion and specular on, the simple pass's background colour. */
nd_status nd_scene_file_lite(const char* json, size_t len, int32_t instance, nd_lite_desc* lite, char* err,
                             size_t err_len);

/* Measures the device's FP32 FMA throughput (the roofline of the march, whose DE
 * code is scalar FP32): a resident grid of independent fused multiply-add chains for
 * about `ms` milliseconds; *tflops = 2 x FMAs / CUDA-event time. */
nd_status nd_measure_fp32_peak(nd_ctx* ctx, double ms, double* tflops);

/* A formula image from its pixels, as the reference prepares a height map after
 * decoding it (height_maps.zig:264-320): rgba (HOST, width x height x 4 floats, row
 * major, top row first) holds R, G, B premultiplied by alpha and alpha, each in [0, 1]
 * (the reference's 8- and 16-bit decode; HDR images normalised to [0, 1] with alpha 1).
 * Each channel is quantised to 16 bits; per texel the change to its right and lower
 * neighbours bounds the slope, its running maximum within 8 + 2 and 64 + 2 texels
 * (max-filter dilation) becomes the near and far slope codes.  texels (HOST, 4 words
 * per texel) receives the layout image_sample reads; slope (HOST, 4 floats) the
 * largest slope per channel (times 1.001).  Copy texels to the device and set the
 * view's image fields.  Sizes up to 2048 x 2048 (the reference's max_edge). */
nd_status nd_image_prepare(const float* rgba, int32_t width, int32_t height, uint32_t* texels, float* slope);

/* Size of a public struct by name ("nd_view_desc", ...), for binding layout checks. */
size_t nd_sizeof(const char* name);

#ifdef __cplusplus
}
#endif

#endif /* ND_MARCH_H */
