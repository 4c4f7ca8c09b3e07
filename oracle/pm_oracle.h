/*
 * pm_oracle.h - CPU restatement of the reference's PatchMatch MVS path.
 *
 * TEST INFRASTRUCTURE.  This is the checker the engine's CUDA kernels are
 * compared against, and the timed CPU baseline.  Only tests/, the smoke check
 * and the bench's CPU-baseline leg load it; the engine never does.
 *
 * Two arithmetic flavours:
 *  - f32: the reference's FP32 per-tap arithmetic (computePixelCost,
 *    src/dense_recon/patchmatch_mvs.cu:222-343) with the texture unit's
 *    linear filter emulated in software (8-bit fractional weights, clamp
 *    addressing, unnormalised coordinates, cudaFilterModeLinear as configured
 *    at patchmatch_mvs.cu:805-811).
 *  - f64: the same cost in double precision with exact bilinear weights (or,
 *    optionally, the texture unit's 8-bit weights) - the FP64 oracle.
 *
 * Random streams are the engine's own keyed Philox4x32-10 (Salmon et al.,
 * SC'11), not cuRAND's: see orc_philox4x32_10 for the keying.
 */
#ifndef PM_ORACLE_H_
#define PM_ORACLE_H_

#include <stdint.h>
#include <stddef.h>

#ifdef __cplusplus
extern "C" {
#endif

#define ORC_MAX_SOURCES 8

typedef struct orc_camera {
    double K[9], R[9], t[3];
} orc_camera;

/* One reference view with up to 8 sources, FP32 images (W*H each). */
typedef struct orc_view {
    int W, H, S;
    const float* ref;
    const float* src[ORC_MAX_SOURCES];
    float kinv[9];
    float ab[ORC_MAX_SOURCES][12];
    double kinv64[9];
    double ab64[ORC_MAX_SOURCES][12];
    int radius, stride, top_k;
} orc_view;

/* Texture-filter emulation: how a coordinate becomes 8-bit fixed point.
 * 0 = round half up (measured on B200, the default), 1 = truncate. */
void orc_set_tex_rounding(int mode);
int orc_get_tex_rounding(void);

/* FP64 cost with quantized weights: sources whose bit is set use the FP16
 * path's software-sampler model (separable 8-bit weights, coordinates rounded
 * to nearest) instead of the texture unit's.  Default 0. */
void orc_set_soft_sources(unsigned mask);
unsigned orc_get_soft_sources(void);

void orc_philox4x32_10(const uint32_t ctr[4], const uint32_t key[2], uint32_t out[4]);
float orc_u01(uint32_t x);

/* FP64 setup: kinv = K_ref^-1, ab[s] = {A = K_s R_s R_ref^T K_ref^-1, b = K_s (t_s - R_rel t_ref)}. */
int orc_setup_f64(const orc_camera* ref, const orc_camera* srcs, int S, double* kinv9, double* ab);
/* Fill view->kinv/ab (float) and kinv64/ab64 (double) from cameras. */
int orc_view_set_cameras(orc_view* v, const orc_camera* ref, const orc_camera* srcs);

float orc_tex_linear(const float* img, int W, int H, float xc, float yc);

float orc_pixel_cost_f32(const orc_view* v, int x, int y, float d, float nx, float ny, float nz);
double orc_pixel_cost_f64(const orc_view* v, int x, int y, double d, double nx, double ny, double nz,
                          int quantized_weights);
/* Per-source NCC (before view selection), FP64; out_ncc[S], returns valid mask bits. */
int orc_source_ncc_f64(const orc_view* v, int x, int y, double d, double nx, double ny, double nz,
                       int quantized_weights, double* out_ncc);

/* Whole-map costs of fixed hypotheses.  normal is AoS (3 floats per pixel). */
void orc_cost_map_f32(const orc_view* v, const float* depth, const float* normal, float* cost);
/* Rows [y0, y1) only (bounded samples for the CPU baseline). */
void orc_cost_rows_f32(const orc_view* v, const float* depth, const float* normal, float* cost, int y0, int y1);
void orc_cost_map_f64(const orc_view* v, const float* depth, const float* normal, int quantized_weights,
                      double* cost);
void orc_cost_rows_f64(const orc_view* v, const float* depth, const float* normal, int quantized_weights,
                       double* cost, int y0, int y1);

void orc_init(const orc_view* v, float dmin, float dmax, uint64_t seed, uint32_t view_id,
              float* depth, float* normal);

typedef struct orc_refine {
    int refine_steps;     /* 2 */
    float iter_decay;     /* 0.6 */
    float step_decay;     /* 0.5 */
} orc_refine;

void orc_propagate_pass(const orc_view* v, float* depth, float* normal, float* cost, float dmin, float dmax,
                        int iteration, int color, uint64_t seed, uint32_t view_id, const orc_refine* rf);

void orc_propagate_rows(const orc_view* v, float* depth, float* normal, float* cost, float dmin, float dmax,
                        int iteration, int color, uint64_t seed, uint32_t view_id, const orc_refine* rf, int y0,
                        int y1);

/* init + initial cost + `iterations` red-black iterations. */
void orc_solve_view(const orc_view* v, float dmin, float dmax, uint64_t seed, uint32_t view_id,
                    int iterations, const orc_refine* rf, float* depth, float* normal, float* cost);

/* geometric_consistency_filter_kernel (patchmatch_mvs.cu:668-781), FP32 camera
 * parameters cast from FP64 as the reference's eigenToGPUCamera does. */
void orc_geometric_filter(const orc_camera* ref, int W, int H, float* depth, const float* normal,
                          float* confidence, int S, const orc_camera* srcs, const float* const* src_depths,
                          const float* const* src_normals, float depth_tol, float normal_tol_cos,
                          int min_consistent);

/* Depth-map fusion into a point cloud, the rule hp_fuse_depth_maps states in
 * include/hpmvs.h (the reference's fuseDepthMaps, src/dense_recon/point_cloud.h:7,
 * is a stub): a pixel's world point, checked in each neighbour for depth,
 * reprojection and normal agreement, emitted as the mean of the agreeing
 * points by the lowest-index agreeing view, in (view, row, column) order.
 * Same FP32 operation order as the engine's kernel.  Returns the number of
 * points; writes the first `capacity` of them (any output may be NULL). */
typedef struct orc_fuse_view {
    orc_camera cam;
    const float* depth;
    const float* normal;      /* camera frame */
    const float* confidence;  /* or NULL */
    const float* gray;        /* or NULL */
    const int* neighbors;     /* or NULL: every other view */
    int num_neighbors;
    int W, H;
} orc_fuse_view;

long long orc_fuse(const orc_fuse_view* views, int num_views, int min_views, float min_confidence,
                   float max_depth_rel, float max_reproj_px, float min_normal_cos, float* positions,
                   float* normals, float* colors, long long capacity);

int orc_num_threads(void);
void orc_set_num_threads(int n);

#ifdef __cplusplus
}
#endif

#endif
