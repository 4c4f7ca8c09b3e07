/*
 * hpmvs.h - C ABI of the B200 PatchMatch multi-view-stereo engine.
 *
 * The engine fills the dense-reconstruction stage of the Hemiphoto3D pipeline.
 * Its call surface follows the reference's
 *     std::vector<DepthMap> runPatchMatchMVS(images, cameras, sfm, config)
 * (src/dense_recon/patchmatch_mvs.h:39-44, defined at patchmatch_mvs.cu:1028):
 * images and cameras in, one depth / normal / cost map per reference view out.
 * Source views and the depth range, which the reference derives from the SfM
 * result (selectSourceViews, patchmatch_mvs.cu:74-157), are explicit job inputs.
 *
 * Conventions
 *  - Every entry point returns hp_status; nothing exits the process and no C++
 *    exception crosses the boundary (the reference calls exit() through
 *    CUDA_CHECK, src/utils/cuda_utils.cuh:7-15).  hp_ctx_last_error() gives text.
 *  - Cameras are FP64, row-major, world-to-camera: P_cam = R * P_world + t
 *    (CameraPose, include/types.h:55-74).
 *  - Maps are row-major H x W.  Normals are camera-frame, 3 floats per pixel
 *    (the frame the reference's kernels produce, patchmatch_mvs.cu:213-215).
 *  - A pointer argument lives in host or device memory as its hp_memory flag
 *    says; device pointers must belong to the context's device.
 *  - One context per host thread, or external locking: a context is not
 *    internally synchronised.  Work is issued on the context's own stream.
 */
#ifndef HPMVS_H_
#define HPMVS_H_

#include <stddef.h>
#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

#define HP_MAX_SOURCES 8   /* MAX_SRC_VIEWS, patchmatch_mvs.cu:18 */
#define HP_MAX_RADIUS 7    /* the reference clamps to 5 (patchmatch_mvs.cu:24, :1065-1070) */
#define HP_MAX_TOP_K 3     /* NCC_TOP_K, patchmatch_mvs.cu:26 */

typedef enum hp_status {
    HP_OK = 0,
    HP_ERR_INVALID_ARG = 1,
    HP_ERR_CUDA = 2,
    HP_ERR_OUT_OF_MEMORY = 3,
    HP_ERR_NOT_FOUND = 4,
    HP_ERR_TIMEOUT = 5,
    HP_ERR_UNSUPPORTED = 6,
    HP_ERR_IO = 7,
    HP_ERR_BUSY = 8,
    HP_ERR_CANCELLED = 9
} hp_status;

typedef enum hp_dtype {
    HP_DTYPE_U8 = 0,   /* 0..255, scaled by 1/255 on upload */
    HP_DTYPE_F16 = 1,  /* IEEE half in [0,1] */
    HP_DTYPE_F32 = 2   /* float in [0,1]: ImageData.gray, include/types.h:17 */
} hp_dtype;

typedef enum hp_precision {
    /* Plain FP32: per-tap arithmetic and hardware bilinear sampling as in the
     * reference's computePixelCost (patchmatch_mvs.cu:222-343). */
    HP_PRECISION_F32 = 0,
    /* FP16 image storage, FP16 window products with FP32 accumulation and
     * mean-subtracted variance; FP64 homography setup. */
    HP_PRECISION_F16ACC = 1
} hp_precision;

typedef enum hp_memory { HP_MEMORY_HOST = 0, HP_MEMORY_DEVICE = 1 } hp_memory;

typedef struct hp_ctx hp_ctx;

/* World-to-camera pinhole camera; all matrices row-major. */
typedef struct hp_camera {
    double K[9];
    double R[9];
    double t[3];
} hp_camera;

/* Solver parameters.  hp_params_default() gives the reference's constants:
 * radius 5 (mvs_patch_size 11, include/types.h:151), stride 1, top-3 view
 * selection, 2 refinement steps, ranges x0.6 per iteration and x0.5 per step
 * (patchmatch_mvs.cu:598-607, :645-646). */
typedef struct hp_params {
    int radius;          /* window radius, 1..HP_MAX_RADIUS */
    int stride;          /* window sampling stride, 1 or 2 */
    int top_k;           /* sources averaged per pixel, 1..HP_MAX_TOP_K */
    int precision;       /* hp_precision */
    int refine_steps;    /* random perturbations per pixel visit, 0..4 */
    float iter_decay;    /* perturbation range factor per iteration */
    float step_decay;    /* perturbation range factor per refinement step */
    int tile_w;          /* pixels per CTA row: 0 or 64 (a warp per row of 32 same-colour pixels) */
    int tile_h;          /* rows per CTA tile: 8, or 4 (FP16-acc path only: 128-thread CTAs); 0 = 8,
                          * or for plans the autotuner's pick.  Others: HP_ERR_UNSUPPORTED.
                          * Every tile shape gives the same bits */
    /* FP16-acc path only: bit s set = source s is sampled by the software
     * bilinear sampler (quad-packed FP16 texels, fixed-point weights, FP16
     * interpolation) instead of the texture unit.  The software sampler
     * runs on the load/store and FP16 pipes, which sustain more taps per SM
     * clock than the texture filter (B200: ~500 vs ~400 Mpix*iter/s at
     * 20 x 1920x1080, r 7, s 2, 6 sources).
     * -1 = engine default (every source), 0 = texture unit only. */
    int soft_sources;
    /* Geometric-consistency filter as the final stage of hp_solve and of
     * plans (geometric_consistency_filter_kernel with runPatchMatchMVS's view
     * loop, patchmatch_mvs.cu:668-781, :1267-1384).  0 = off (the default
     * here); the reference stage uses 2.  When on and a solve has at least
     * two jobs, each job with iterations > 0 is checked, in job order and in
     * place, against the jobs that solved its source images (a job whose
     * ref_image is one of its src_images, the last such job when several are,
     * of the same size, itself excluded): a pixel with fewer than
     * filter_min_consistent agreeing sources gets depth 0 and cost 2
     * (confidence 0).  A job with fewer such sources than that is left as
     * solved.  Later jobs see earlier jobs' filtered depths, as in the
     * reference's loop.  The check uses the jobs' cameras (also when
     * use_coeffs is set). */
    int filter_min_consistent;
    float filter_depth_tol;     /* relative depth tolerance (reference 0.12) */
    float filter_normal_cos;    /* min cosine of the two world normals (reference cos(180 deg) = -1: off) */
    /* FP16-acc path: quad loads in flight per window row (the staging depth):
     * 4 or 8; 0 = 4, or for plans the autotuner's pick.  Same bits either way. */
    int staging;
    /* Tests only (0 = off; the self-checking build alone accepts 1, others
     * return HP_ERR_UNSUPPORTED): 1 turns the FP16-acc path's corner-test
     * shortcuts off, so every window takes the per-tap checked form and
     * wholly-outside sources are sampled too.  The results are the same bits;
     * the switch exists to test that. */
    int debug_checked_taps;
} hp_params;

/* One SfM seed in a reference view: pixel, depth and camera-frame normal. */
typedef struct hp_seed {
    int x, y;
    float depth;
    float normal[3];
} hp_seed;

/* One reference view to solve. */
typedef struct hp_job {
    int ref_image;                     /* id from hp_image_upload */
    int num_sources;                   /* 1..HP_MAX_SOURCES */
    int src_images[HP_MAX_SOURCES];
    hp_camera ref_cam;
    hp_camera src_cams[HP_MAX_SOURCES];
    float depth_min, depth_max;
    uint64_t seed;                     /* RNG key; with view_id keys Philox streams */
    uint32_t view_id;
    int iterations;                    /* red-black iterations (mvs_iterations) */
    /* When use_coeffs != 0 the per-source homography coefficients below are
     * used as given instead of the FP64 setup from the cameras: kinv = K_ref^-1
     * and ab[s] = {A (9), b (3)} with A = K_s R_rel K_ref^-1, b = K_s t_rel
     * (GPUSourceView, patchmatch_mvs.cu:31-34).  This lets a caller feed the
     * exact coefficients another implementation used. */
    int use_coeffs;
    float kinv[9];
    float ab[HP_MAX_SOURCES][12];
    /* SfM-seeded initialisation (runPatchMatchMVS, patchmatch_mvs.cu:1111-1177):
     * after the random initialisation every pixel within seed_radius (per axis)
     * of a seed's pixel takes that seed's depth and normal; where squares
     * overlap, the seed listed last wins.  Host memory, num_seeds records, as
     * hp_project_seeds makes them; NULL / 0 for none.  The reference's radius
     * is 50.  hp_solve, hp_init_hypotheses, plans and the server apply them
     * (the list is copied; it need not outlive the call). */
    const hp_seed* seeds;
    int num_seeds;
    int seed_radius;
} hp_job;

/* Per-view maps, caller-owned. */
typedef struct hp_maps {
    int memory;       /* hp_memory of the pointers */
    float* depth;     /* H*W */
    float* normal;    /* H*W*3, camera frame */
    float* cost;      /* H*W, mean of the top_k lowest 1-NCC, 2 = invalid */
    float* confidence; /* H*W or NULL: 1 - cost/2, DepthMap.confidence (patchmatch_mvs.cu:1246-1252),
                        * written on the device by the solve's unpack; hp_solve, plans and the
                        * server fill it when given */
} hp_maps;

const char* hp_status_string(hp_status s);
void hp_params_default(hp_params* p);
/* Library version as "major.minor.patch". */
const char* hp_version(void);

/* Context: owns a CUDA stream, the uploaded images and solver scratch. */
hp_status hp_ctx_create(int device, hp_ctx** out);
hp_status hp_ctx_destroy(hp_ctx* ctx);
const char* hp_ctx_last_error(const hp_ctx* ctx);
hp_status hp_ctx_synchronize(hp_ctx* ctx);
/* Free device memory and the device total, in bytes. */
hp_status hp_ctx_mem_info(hp_ctx* ctx, size_t* free_bytes, size_t* total_bytes);
/* The context's CUDA stream (a cudaStream_t), for callers that order their own
 * work or timing events against the engine's.  No reference counterpart: the
 * reference runs everything on the default stream. */
hp_status hp_ctx_stream(hp_ctx* ctx, void** stream);

/* Kernel kinds counted by the context profiler. */
typedef enum hp_kernel_kind {
    HP_KERNEL_INIT = 0,      /* hypothesis initialisation */
    HP_KERNEL_COST = 1,      /* full-map cost */
    HP_KERNEL_PROPAGATE = 2, /* red-black propagate + refine half-pass */
    HP_KERNEL_OTHER = 3,     /* layout, conversion and filter kernels */
    HP_KERNEL_PERSISTENT = 4, /* whole-solve persistent launches (plans, server) */
    HP_KERNEL_KINDS = 5
} hp_kernel_kind;

typedef struct hp_profile {
    uint64_t launches[HP_KERNEL_KINDS];  /* every kernel launch the context issued */
    double device_ms[HP_KERNEL_KINDS];   /* summed CUDA-event time, while profiling was on */
    uint64_t timed[HP_KERNEL_KINDS];     /* launches that device_ms covers */
} hp_profile;

/* Tracing: with profiling on, every init / cost / propagate launch is
 * bracketed by CUDA events on the context stream and its device time summed.
 * Launch counts are kept always.  The reference has only printf progress
 * lines (patchmatch_mvs.cu:1083-1087). */
hp_status hp_ctx_set_profiling(hp_ctx* ctx, int enable);
hp_status hp_ctx_profile(hp_ctx* ctx, hp_profile* out);
hp_status hp_ctx_profile_reset(hp_ctx* ctx);

/* Replaces createGrayscaleTexture (patchmatch_mvs.cu:789-814): copies a W x H
 * grayscale image (tightly packed rows) to the device, where it stays until
 * released.  The FP32 and FP16 device copies the solver needs are made here. */
hp_status hp_image_upload(hp_ctx* ctx, const void* data, int memory, int width, int height,
                          int dtype, int* image_id);
hp_status hp_image_release(hp_ctx* ctx, int image_id);
/* Released images keep their device buffers (planes, texture arrays and
 * objects, quad plane) in a per-context cache, up to limit_bytes (default
 * 4 GiB, oldest evicted first), and the next upload of the same size reuses
 * them instead of allocating: a stream of per-request uploads then costs
 * copies and conversions only.  0 disables the cache and frees what it holds.
 * No reference counterpart (the reference creates and destroys its textures
 * on every call, patchmatch_mvs.cu:789-819). */
hp_status hp_ctx_set_image_cache(hp_ctx* ctx, uint64_t limit_bytes);
hp_status hp_image_size(hp_ctx* ctx, int image_id, int* width, int* height);

/* FP64 homography setup, replacing eigenToGPUCamera + precomputeSourceViews
 * (patchmatch_mvs.cu:832-884): kinv9 = K_ref^-1, ab[s] = {A, b} per source. */
hp_status hp_setup_homographies(const hp_camera* ref, const hp_camera* srcs, int num_sources,
                                double* kinv9, double* ab);

/* Replaces runPatchMatchMVS's per-view body (patchmatch_mvs.cu:1076-1260,
 * without SfM seeding): random init, initial cost, `iterations` red-black
 * propagate + refine passes.  out[j] receives job j's maps.  All jobs are
 * solved as one batch: each half-pass is one launch over every job's pixels. */
hp_status hp_solve(hp_ctx* ctx, const hp_job* jobs, int num_jobs, const hp_params* params,
                   hp_maps* out);

/* Replaces launchInitKernel (patchmatch_mvs.cu:890-902): Philox-keyed random
 * depth in [depth_min, depth_max] and camera-facing unit normal per pixel.
 * Fills out->depth and out->normal. */
hp_status hp_init_hypotheses(hp_ctx* ctx, const hp_job* job, const hp_params* params,
                             hp_maps* out);

/* Replaces launchNCCCostKernel (patchmatch_mvs.cu:904-934): NCC cost with
 * top-k view selection of the given (depth, normal) hypotheses; writes
 * maps->cost.  maps->depth / maps->normal are read only. */
hp_status hp_ncc_cost(hp_ctx* ctx, const hp_job* job, const hp_params* params, hp_maps* maps);

/* Replaces launchPropagateRefineKernel (patchmatch_mvs.cu:936-961): one
 * red-black half-pass (color 0: (x+y) even, 1: odd) of iteration `iteration`,
 * in place on maps (depth, normal, cost). */
hp_status hp_propagate_pass(hp_ctx* ctx, const hp_job* job, const hp_params* params,
                            hp_maps* maps, int iteration, int color);

/* Replaces geometric_consistency_filter_kernel + its host packing
 * (patchmatch_mvs.cu:668-781, :1267-1384) for maps the caller holds; a solve
 * runs the same check itself with hp_params.filter_min_consistent.  depth
 * and confidence are updated in place: a pixel with fewer than
 * min_consistent agreeing sources gets 0 in both, and a pixel without a
 * positive depth gets confidence 0.  All maps are width x height (the
 * reference's rule: sources of another size are not passed).  A source
 * agrees when the pixel's point lies in front of it, inside it at the
 * nearest pixel, that pixel's depth is positive and within depth_tol of the
 * point's depth in the source camera (relative), and the world-frame normals
 * have a cosine of at least normal_tol_cos.  Reference defaults: depth_tol
 * 0.12, normal_tol_cos cos(180 deg), min_consistent 2.  The transforms are
 * composed in FP64 from the cameras; a source map must not be the depth map
 * being filtered.  All map pointers are in `memory`. */
hp_status hp_geometric_filter(hp_ctx* ctx, const hp_camera* ref_cam, int width, int height,
                              float* depth, const float* normal, float* confidence,
                              int num_sources, const hp_camera* src_cams,
                              const float* const* src_depths, const float* const* src_normals,
                              int memory, float depth_tol, float normal_tol_cos,
                              int min_consistent);

/* Largest view hp_solve_static accepts (width * height), fixed by its
 * statically sized device scratch: 20 bytes per pixel, 26.2 MB in all. */
#define HP_STATIC_MAX_PIXELS (1280 * 1024)

/* No counterpart in the reference.  The single-view FP32 solve of hp_solve
 * (random init, initial cost, `iterations` red-black passes, same kernels and
 * results) for callers that must not have the library allocate device memory:
 * applications whose device memory is owned by their own pool or budget, or
 * latency-critical loops that cannot afford cudaMalloc/cudaFree and the
 * synchronisation they bring.  It calls no allocation routine: the plane
 * state, costs and launch descriptors live in one file-scope device array of
 * fixed size that every GPU loading the library holds until exit, so views
 * larger than HP_STATIC_MAX_PIXELS are rejected with HP_ERR_UNSUPPORTED.
 *   device, stream    where to run (stream may be NULL); waits for completion
 *   job               cameras or use_coeffs, depth range, seed, view_id,
 *                     iterations, num_sources (its image ids are ignored)
 *   ref_image         device FP32 reference image, values in [0,1], row pitch
 *                     ref_pitch floats
 *   src_textures      num_sources cudaTextureObject_t over the FP32 source
 *                     images (same size): linear filter, clamp addressing,
 *                     unnormalised coordinates, element read mode
 *   params            precision must be HP_PRECISION_F32
 *   out               device maps (memory HP_MEMORY_DEVICE)
 * The first call in a CUDA context looks up the scratch array's address in
 * that context and caches it; make it before any stream capture.  The cache is
 * keyed by the context's id, so after cudaDeviceReset (or with another context
 * made current) the next call looks the address up again: the address a
 * previous context had is never reused.  Completion: the call waits for every
 * copy and kernel it queued, on success and on failure alike.  All calls share
 * the one array, so calls that overlap in time (several host threads) race:
 * serialise them. */
hp_status hp_solve_static(int device, void* stream, const hp_job* job, const float* ref_image, int ref_pitch,
                          int width, int height, const unsigned long long* src_textures, const hp_params* params,
                          hp_maps* out);

/* ---------------------------------------------------------------------------
 * Plans: a batched solve prepared once and run many times.  No counterpart in
 * the reference, which solves one view at a time with a device
 * synchronisation after every launch (runPatchMatchMVS,
 * patchmatch_mvs.cu:1199-1232).  A plan owns the device state of its jobs
 * (views of any size and source count, each with its own iteration count) and
 * the output binding, and replays its launch sequence as one CUDA graph.
 * Every schedule gives bit-identical results (the per-pixel arithmetic does
 * not depend on how tiles are scheduled); they differ only in speed.
 * ------------------------------------------------------------------------- */
typedef enum hp_schedule_kind {
    HP_SCHEDULE_AUTO = 0,       /* persistent until hp_plan_tune has chosen */
    HP_SCHEDULE_PER_PASS = 1,   /* init, cost, one launch per red-black half-pass over all views, unpack */
    HP_SCHEDULE_PERSISTENT = 2  /* one launch for the whole solve: CTAs take (view, stage, tile) tickets */
} hp_schedule_kind;

typedef struct hp_plan_options {
    int schedule;         /* hp_schedule_kind */
    int ctas_per_sm;      /* persistent: resident CTAs per SM, 0 = the occupancy maximum */
    int use_graph;        /* 1: capture the launch sequence once and replay it as a CUDA graph */
    int wait_limit_ms;    /* persistent: bound on one inter-tile dependency wait (0 = 2000 ms) */
    int debug_stall_view; /* tests only: tile (view, tile) never reports completion, so its */
    int debug_stall_tile; /*   dependants' bounded waits run out (-1 = off) */
} hp_plan_options;

typedef struct hp_plan_info {
    int schedule;            /* the schedule a run uses (never AUTO) */
    int ctas_per_sm;         /* persistent: resident CTAs per SM in use */
    int grid;                /* persistent: CTAs launched */
    int max_ctas_per_sm;     /* persistent: occupancy maximum of the kernel */
    int tickets;             /* persistent: (view, stage, tile) work items */
    int launches_per_run;    /* kernel launches one run issues */
    int views;
    int use_graph;
    uint64_t state_bytes;    /* device memory the plan holds */
    double pixel_iterations; /* sum over views of W * H * iterations */
    float tuned_ms;          /* hp_plan_tune: the chosen candidate's median solve time (0 before) */
    int tile_h;              /* rows per CTA tile in use (8, or 4 on the FP16-acc path) */
    int staging;             /* FP16-acc: quad loads in flight per window row in use (4 or 8) */
} hp_plan_info;

typedef struct hp_plan hp_plan;

void hp_plan_options_default(hp_plan_options* o);
/* Validates the jobs, allocates their state and binds `out` (one hp_maps per
 * job, host or device memory; host maps are filled when a run finishes). */
hp_status hp_plan_create(hp_ctx* ctx, const hp_job* jobs, int num_jobs, const hp_params* params,
                         const hp_plan_options* options, const hp_maps* out, hp_plan** plan);
/* One full solve into the bound maps; returns when they are written.
 * HP_ERR_TIMEOUT when a persistent dependency wait ran out (the kernel then
 * stops taking work and the context stays usable). */
hp_status hp_plan_run(hp_plan* plan);
/* Enqueue one solve on the context stream without waiting (device maps
 * only); hp_plan_wait completes it and reports its status. */
hp_status hp_plan_launch(hp_plan* plan);
hp_status hp_plan_wait(hp_plan* plan);
/* Autotuner: times candidates `repeats` times each on the plan's own jobs and
 * keeps the fastest by median, reporting it in `best`.  On the FP16-acc path
 * it first picks the tile height (64x8 or 64x4 pixels per CTA) and the
 * staging depth (4 or 8 quad loads in flight per window row) with the
 * per-pass graph, where params left them at 0; then the schedule: the
 * per-pass graph, or the persistent kernel at each resident-CTA count up to
 * its occupancy maximum.  Every candidate gives the same bits.  The bound maps
 * hold a valid solve afterwards. */
hp_status hp_plan_tune(hp_plan* plan, int repeats, hp_plan_info* best);
hp_status hp_plan_get_info(const hp_plan* plan, hp_plan_info* info);
hp_status hp_plan_destroy(hp_plan* plan);

/* The persistent ticket order, computed on the host (no device needed): view
 * v runs stages [stage_begin[v], stage_end[v]) of its stage sequence (0 init +
 * cost, 1 + 2*it + color the half-passes, 2*iterations + 1 the unpack) and
 * entry e covers tickets [entry_ticket[e], entry_ticket[e + 1]) of view
 * entry_view[e] at stage entry_stage[e].  Entries are ordered by the stage's
 * offset from its view's stage_begin, then by view.  `capacity` bounds the
 * entries; entry_ticket needs capacity + 1 slots. */
hp_status hp_schedule_build(int num_views, const int* tiles, const int* stage_begin, const int* stage_end,
                            int capacity, int* entry_ticket, int* entry_view, int* entry_stage, int* num_entries);

/* ---------------------------------------------------------------------------
 * Server: continuous batching of depth-map solves.  No counterpart in the
 * reference, which solves one view at a time, synchronously
 * (runPatchMatchMVS, patchmatch_mvs.cu:1076-1260).  Requests - one hp_job
 * each, with its own size, sources and iteration count, over images already
 * uploaded to the context - are submitted from any host thread.  A worker
 * thread admits queued requests in arrival order while request slots and
 * device memory allow, and runs steps: each step advances every admitted
 * request by `passes_per_step` stages (initialisation + cost, red-black
 * half-passes, unpacking into its maps) in the persistent kernel, all
 * requests together.  A request that arrives while others are on the GPU
 * joins at the next step.  Its result does not depend on what it was
 * batched with: it equals hp_solve of the same job bit for bit.
 * While a server runs, the context's images must stay uploaded until the
 * requests that read them have completed; other work on the context may
 * proceed from the caller's thread (the server uses its own stream).
 * ------------------------------------------------------------------------- */
typedef struct hp_server hp_server;

/* How a step divides its stages among the admitted requests. */
typedef enum hp_server_policy {
    /* Every admitted request advances passes_per_step stages per step. */
    HP_SERVER_POLICY_ROUND_ROBIN = 0,
    /* Oldest first within a work budget: in admission order, each request
     * takes as many of its next stages (up to passes_per_step) as the step's
     * budget of step_budget_mpix million pixel x source stage units still
     * covers, and at least one, so the oldest requests finish first and none
     * stalls. */
    HP_SERVER_POLICY_BUDGET = 1
} hp_server_policy;

typedef struct hp_server_options {
    int max_active;         /* request slots (admitted, not yet completed); 0 = 64 */
    float mem_fraction;     /* admit while device memory in use stays <= this fraction
                             * of the device total (0 = 0.8) */
    uint64_t mem_limit;     /* if nonzero: byte budget for request state instead */
    int passes_per_step;    /* stages per request per step, 1..64 (0 = 8); with the budget
                             * policy the most a request takes in one step */
    int split_launches;     /* 1: one launch per stage offset of a step (no waits between
                             * tiles); 0: one persistent launch per step */
    int ctas_per_sm;        /* resident CTAs per SM (0 = the occupancy maximum) */
    int inflight_steps;     /* steps enqueued ahead of the oldest unfinished one, 1..4 (0 = 2) */
    int wait_limit_ms;      /* bound on one inter-tile dependency wait (0 = 2000) */
    int policy;             /* hp_server_policy (0 = round robin).  hp_server_options_default
                             * sets the budget policy with 32 stages and 1200 M units a step:
                             * on B200 with mixed 0.3-12 Mpix requests at 10/s it lowered p50
                             * and p90 latency by 15-20% against round robin with 8 stages
                             * a step; p99 moved by -20% to +5% over the runs measured */
    double step_budget_mpix; /* HP_SERVER_POLICY_BUDGET: work per step, in 1e6 pixel x source stage
                              * units (0 = 1200, ~0.2 s of FP16-acc r 7 s 2 work on a B200) */
    uint64_t debug_stall_request; /* tests only: in the request with this id (0 = off), tile */
    int debug_stall_tile;         /*   debug_stall_tile never reports completion, so the step's
                                   *   bounded waits run out and the failure is contained */
    int debug_fail_step;          /* tests only: step n (1-based; 0 = off) fails to launch on the
                                   *   host, as a launch error would (its requests: HP_ERR_CUDA) */
} hp_server_options;

/* One finished request. */
typedef struct hp_completion {
    uint64_t request_id;
    int status;             /* hp_status: HP_OK, or why the request failed */
    double latency_ms;      /* hp_submit to completion, host clock */
    double queue_ms;        /* hp_submit to admission */
} hp_completion;

typedef struct hp_server_stats {
    uint64_t submitted, admitted, completed, failed;
    uint64_t steps, launches;
    int queued, active, peak_active;
    double p50_ms, p99_ms, mean_ms, max_ms;   /* latency of the completed requests */
    double pixel_iterations;                  /* sum of W * H * iterations, completed */
    double device_ms;                         /* device time of all finished steps */
    uint64_t state_bytes, peak_state_bytes;   /* request state held now / at most */
    uint64_t budget_bytes;                    /* admission budget at the last admission */
    uint64_t failed_steps;                    /* steps that failed (each fails the requests admitted
                                               * at the time; hp_server_last_error says where) */
    uint64_t pool_reserved_bytes;             /* the server's memory pool at the last admission check */
    uint64_t device_free_bytes;               /* free device memory at the last admission check */
} hp_server_stats;

void hp_server_options_default(hp_server_options* o);
/* params apply to every request (radius, stride, precision, ...). */
hp_status hp_server_create(hp_ctx* ctx, const hp_params* params, const hp_server_options* options,
                           hp_server** server);
/* Queue one solve.  `out` (depth, normal, cost; host or device memory) must
 * stay valid until the request completes.  HP_ERR_OUT_OF_MEMORY when the
 * request alone exceeds the admission budget. */
hp_status hp_submit(hp_server* s, const hp_job* job, const hp_maps* out, uint64_t* request_id);
/* Completed requests, oldest first: up to `capacity` into `done`, waiting up
 * to timeout_ms (0: no wait, < 0: until one completes) for the first. */
hp_status hp_poll(hp_server* s, hp_completion* done, int capacity, int* num_done, int timeout_ms);
/* Waits until no request is queued or running (HP_ERR_TIMEOUT after timeout_ms, < 0 = no limit). */
hp_status hp_server_drain(hp_server* s, int timeout_ms);
hp_status hp_server_stats_get(hp_server* s, hp_server_stats* stats);
hp_status hp_server_stats_reset(hp_server* s);
const char* hp_server_last_error(hp_server* s);
/* The worker's first error since the server was created ("" if none): a later
 * error (say, admissions refused after a device fault) does not replace it. */
const char* hp_server_first_error(hp_server* s);
/* Stops the worker after the requests already admitted finish; queued
 * requests complete with HP_ERR_CANCELLED (their completions are dropped). */
hp_status hp_server_destroy(hp_server* s);

/* The server's admission and step-composition policy run without a device,
 * for tests: requests k = 0..n-1 arrive before steps arrive_step[k], need
 * state_bytes[k] and have stages[k] stages (2 * iterations + 2).  With the
 * given slots, byte budget and stages per step, admit_step[k] and
 * finish_step[k] receive the step in which request k is admitted and the one
 * in which its last stage runs; *steps the number of steps run. */
hp_status hp_server_simulate(int n, const int* arrive_step, const uint64_t* state_bytes, const int* stages,
                             int max_active, uint64_t budget, int passes_per_step, int* admit_step,
                             int* finish_step, int* steps);
/* The same with a step policy: work[k] is request k's work per stage (pixel x
 * source units, W * H * num_sources), step_work the budget policy's work per
 * step in the same units. */
hp_status hp_server_simulate_policy(int n, const int* arrive_step, const uint64_t* state_bytes, const int* stages,
                                    const double* work, int max_active, uint64_t budget, int passes_per_step,
                                    int policy, double step_work, int* admit_step, int* finish_step, int* steps);

/* ---------------------------------------------------------------------------
 * SfM front of the stage: what runPatchMatchMVS derives from the sparse
 * reconstruction before solving.
 * ------------------------------------------------------------------------- */
/* Sparse points with their tracks: point p is seen by cameras
 * track_images[track_offset[p] .. track_offset[p + 1]) (SparsePoint,
 * include/types.h:76-83). */
typedef struct hp_sparse_points {
    int num_points;
    const double* position;      /* 3 per point, world frame */
    const int* track_offset;     /* num_points + 1 */
    const int* track_images;     /* camera indices */
} hp_sparse_points;

/* Sources and depth range of one reference view (MVSViewParams, patchmatch_mvs.h:16-28). */
typedef struct hp_view_selection {
    int ref_image;                       /* camera index */
    int num_sources;
    int sources[HP_MAX_SOURCES];         /* camera indices, best first */
    float scores[HP_MAX_SOURCES];        /* shared points * baseline score */
    float baseline_deg[HP_MAX_SOURCES];
    float depth_min, depth_max;
} hp_view_selection;

/* Replaces selectSourceViews (patchmatch_mvs.cu:74-157).  For every
 * registered camera, in index order: the other registered cameras whose
 * baseline angle at the points' centroid lies in [5, 90] degrees and that
 * share points with it, scored shared * sin(clamp(angle, 5, 30)) and sorted
 * best first (equal scores: lower camera index first; the reference's sort
 * leaves their order unspecified), at most num_sources (1..HP_MAX_SOURCES).
 * Depth range: the 5th and 95th percentile of the camera-frame depths of the
 * points it sees, x0.5 and x1.5 (fewer than two: the centroid depth x0.3 and
 * x3).  Shared counts come from one pass over the tracks.  out needs one entry
 * per registered camera; *num_out receives the count. */
hp_status hp_select_sources(const hp_camera* cams, const int* registered, int num_cams,
                            const hp_sparse_points* points, int num_sources, hp_view_selection* out,
                            int* num_out);

/* The seeds of reference camera `ref` (patchmatch_mvs.cu:1122-1160): every
 * point whose track contains `ref` and whose camera-frame depth is positive
 * and inside [depth_min, depth_max], at the rounded pixel of its projection,
 * with the unit normal towards the camera centre in the camera frame, in
 * point order.  FP64 throughout, as the reference.  Returns up to capacity
 * seeds; *num_seeds receives how many there are. */
hp_status hp_project_seeds(const hp_camera* cam, int ref, float depth_min, float depth_max,
                           const hp_sparse_points* points, hp_seed* out, int capacity, int* num_seeds);

/* ---- Depth-map fusion: the stage's consumer ------------------------------
 * Fills the reference's fuseDepthMaps(depth_maps, poses, images)
 * (src/dense_recon/point_cloud.h:7, a stub returning an empty cloud at
 * src/dense_recon/point_cloud.cu:4-8) and its DensePointCloud output
 * (include/types.h:93-106: positions, normals, colours as float3 arrays).
 *
 * A pixel of view i with depth > 0 (and confidence >= min_confidence) is
 * back-projected to X with its normal rotated to the world frame.  Each
 * neighbour j takes X to its pixel q (rounded projection), and agrees when
 *   q is inside view j with depth > 0 (and confidence >= min_confidence),
 *   |z_j(X) - depth_j(q)| <= max_depth_rel * depth_j(q),
 *   q's back-projection lands within max_reproj_px of the pixel in view i,
 *   the two world normals have cosine >= min_normal_cos.
 * The point is emitted when at least min_views views agree (the view itself
 * counts) and no agreeing neighbour has a lower index than i; that lowest view
 * emits the surface point instead, so with symmetric neighbour lists each is
 * emitted once.  Position, normal and colour are the means over the agreeing
 * views (the normal renormalised; the colour the gray value, replicated to
 * three channels).  Points come in (view, row, column) order; FP32 arithmetic
 * with every operation rounded as written (no contraction), so results do not
 * depend on the launch configuration. */
typedef struct hp_fuse_view {
    hp_camera cam;
    const float* depth;       /* H*W, 0 = invalid (e.g. after hp_geometric_filter) */
    const float* normal;      /* H*W*3, camera frame, as hp_solve writes them */
    const float* confidence;  /* H*W, or NULL: every pixel eligible */
    const float* gray;        /* H*W intensity in [0, 1] for the colour, or NULL: colour 0 */
    const int* neighbors;     /* host array of view indices to check, or NULL: every other view */
    int num_neighbors;
    int width, height;
} hp_fuse_view;

typedef struct hp_fuse_params {
    int memory;               /* hp_memory of every view's map pointers */
    int min_views;            /* agreeing views, the view itself included (default 2) */
    float min_confidence;     /* default 0 */
    float max_depth_rel;      /* default 0.01 */
    float max_reproj_px;      /* default 2 */
    float min_normal_cos;     /* default cos(10 deg); -1 turns the normal test off */
} hp_fuse_params;

typedef struct hp_point_cloud {
    int memory;               /* hp_memory of the three arrays */
    float* positions;         /* capacity*3 world-frame points, or NULL */
    float* normals;           /* capacity*3 unit world-frame normals, or NULL */
    float* colors;            /* capacity*3, or NULL */
    int64_t capacity;         /* points the arrays hold */
    int64_t count;            /* out: points fused; those at index >= capacity are not written */
} hp_point_cloud;

void hp_fuse_params_default(hp_fuse_params* p);
/* Fuses num_views depth maps into out (see above).  With capacity 0 it only
 * counts, so a caller can size the arrays and call again. */
hp_status hp_fuse_depth_maps(hp_ctx* ctx, const hp_fuse_view* views, int num_views,
                             const hp_fuse_params* params, hp_point_cloud* out);

/* Replaces saveDepthMapPFM / loadDepthMapPFM (patchmatch_mvs.cu:990-1022):
 * 'Pf' (channels 1) or 'PF' (channels 3) little-endian PFM, rows bottom-up. */
hp_status hp_pfm_write(const char* path, const float* data, int width, int height, int channels);
/* Reads into `data` (capacity floats); width/height/channels receive the header. */
hp_status hp_pfm_read(const char* path, float* data, size_t capacity, int* width, int* height,
                      int* channels);

#ifdef __cplusplus
}
#endif

#endif /* HPMVS_H_ */
