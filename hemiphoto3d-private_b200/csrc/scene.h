// Synthetic scene renderer (host only): planes and spheres with one blurred
// uniform-noise albedo texture, analytic depth and normal ground truth.
#pragma once
#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

enum { HPS_PLANE = 0, HPS_SPHERE = 1 };

typedef struct hps_object {
    int kind;              // HPS_PLANE or HPS_SPHERE
    double p[3];           // plane: a point on it (its centre if bounded); sphere: centre
    double n[3];           // plane unit normal
    double u[3], v[3];     // plane unit in-plane axes (texture axes and bounds)
    double half_u, half_v; // plane half extents along u / v; <= 0 means unbounded
    double radius;         // sphere radius
    double tex_offset[2];  // texture offset in metres
} hps_object;

// n x n albedo: uniform noise, Gaussian blur of std `sigma` texels (wrap),
// rescaled to mean 0.5 and std `contrast_std`, clipped to [0.02, 0.98].
int hps_make_albedo(int n, double sigma, uint64_t seed, float contrast_std, float* out);

// Render one W x H view (spp x spp samples per pixel).  K, R, t row-major,
// world-to-camera.  depth (camera z, 0 = miss) and normal (camera frame, 3 per
// pixel, facing the camera) are optional ground truth at pixel centres.
int hps_render(const hps_object* objs, int n_objs, const float* tex, int tex_n, double texels_per_meter,
               const double* K, const double* R, const double* t, int W, int H, int spp, float background,
               float* img, float* depth, float* normal);

#ifdef __cplusplus
}
#endif
