// GPU reference harness: the reference's own PatchMatch translation unit
// (src/dense_recon/patchmatch_mvs.cu), compiled unmodified from where it lies
// and wrapped in a flat C ABI so tests can drive its kernels on fixed inputs.
//
// TEST INFRASTRUCTURE ONLY.  Nothing in the engine links or loads this; only
// tests/ and the bench's reference-GPU leg call it, as a checker.  The include
// of the reference source is supplied by the build recipe (PMREF_SOURCE), and
// the data-model types it needs come from the stand-in headers under shim/.
//
// Entry points and the reference code they drive:
//   pmref_setup_views   eigenToGPUCamera + precomputeSourceViews  (patchmatch_mvs.cu:832-884)
//   pmref_ncc_cost      launchNCCCostKernel -> compute_ncc_cost_kernel (:904-934, :349-513)
//   pmref_pixel_cost    computePixelCost, one thread per pixel     (:222-343)
//   pmref_init          launchInitKernel -> init_depth_normal_kernel (:890-902, :164-216)
//   pmref_propagate     launchPropagateRefineKernel               (:936-961, :519-655)
//   pmref_solve_view    the per-view body of runPatchMatchMVS without SfM seeding
//                       (:1094-1107, :1189-1232)
//   pmref_geometric_filter launchGeometricFilterKernel            (:963-988, :668-781)
//   pmref_select_sources selectSourceViews (host only)            (:74-157)
//   pmref_run_stage     runPatchMatchMVS itself with mvs_iterations = 0: random
//                       init, SfM seeding, initial cost, download (:1028-1260)

#ifndef PMREF_SOURCE
#error "PMREF_SOURCE must name the reference patchmatch_mvs.cu"
#endif
#include PMREF_SOURCE

#include <cstring>
#include <vector>

namespace {

struct TexSet {
    cudaTextureObject_t ref_tex = 0;
    cudaArray_t ref_arr = nullptr;
    std::vector<cudaTextureObject_t> src_tex;
    std::vector<cudaArray_t> src_arr;
    ~TexSet() {
        destroyTexture(ref_tex, ref_arr);
        for (size_t i = 0; i < src_tex.size(); ++i) destroyTexture(src_tex[i], src_arr[i]);
    }
};

void make_textures(TexSet& t, const float* ref_img, const float* const* src_imgs, int S, int W, int H) {
    createGrayscaleTexture(ref_img, W, H, t.ref_tex, t.ref_arr);
    t.src_tex.assign(S, 0);
    t.src_arr.assign(S, nullptr);
    for (int s = 0; s < S; ++s) createGrayscaleTexture(src_imgs[s], W, H, t.src_tex[s], t.src_arr[s]);
}

std::vector<GPUSourceView> unpack_views(const float* ab, int S) {
    std::vector<GPUSourceView> v(S);
    for (int s = 0; s < S; ++s) {
        std::memcpy(v[s].A, ab + 12 * s, 9 * sizeof(float));
        std::memcpy(v[s].b, ab + 12 * s + 9, 3 * sizeof(float));
    }
    return v;
}

__global__ void pixel_cost_wrapper_kernel(cudaTextureObject_t ref, const cudaTextureObject_t* src,
                                          const float* depth, const float* normal, const float* kinv,
                                          const GPUSourceView* views, float* cost, int radius,
                                          int W, int H, int S) {
    int x = blockIdx.x * blockDim.x + threadIdx.x;
    int y = blockIdx.y * blockDim.y + threadIdx.y;
    if (x >= W || y >= H) return;
    int idx = y * W + x;
    cost[idx] = computePixelCost(ref, src, depth[idx], normal[3 * idx], normal[3 * idx + 1],
                                 normal[3 * idx + 2], kinv, views, x, y, radius, W, H, S);
}

// A flat SfM description: camera c is K R t (21 doubles) at cams_krt + 21 c; point p
// at pos + 3 p, seen by cameras timg[toff[p] .. toff[p + 1]).
SfMResult make_sfm(const double* cams_krt, const int* registered, int n_cams, const double* pos, const int* toff,
                   const int* timg, int n_pts);

CameraPose to_pose(const double* krt) {
    CameraPose c;
    for (int i = 0; i < 9; ++i) c.K(i / 3, i % 3) = krt[i];
    for (int i = 0; i < 9; ++i) c.R(i / 3, i % 3) = krt[9 + i];
    for (int i = 0; i < 3; ++i) c.t(i) = krt[18 + i];
    c.is_registered = true;
    return c;
}

SfMResult make_sfm(const double* cams_krt, const int* registered, int n_cams, const double* pos, const int* toff,
                   const int* timg, int n_pts) {
    SfMResult sfm;
    sfm.num_registered = 0;
    for (int c = 0; c < n_cams; ++c) {
        CameraPose cp = to_pose(cams_krt + 21 * c);
        cp.image_id = c;
        cp.is_registered = registered[c] != 0;
        sfm.num_registered += cp.is_registered ? 1 : 0;
        sfm.cameras.push_back(cp);
    }
    for (int p = 0; p < n_pts; ++p) {
        SparsePoint sp;
        sp.position(0) = pos[3 * p];
        sp.position(1) = pos[3 * p + 1];
        sp.position(2) = pos[3 * p + 2];
        for (int k = toff[p]; k < toff[p + 1]; ++k) sp.image_ids.push_back(timg[k]);
        sp.track_length = toff[p + 1] - toff[p];
        sfm.points.push_back(sp);
    }
    return sfm;
}

}  // namespace

extern "C" {

// selectSourceViews: per returned view its reference id, source count, sources
// (HP 8 slots each), scores, baseline angles and depth range.
int pmref_select_sources(const double* cams_krt, const int* registered, int n_cams, const double* pos,
                         const int* toff, const int* timg, int n_pts, int num_sources, int* out_ref, int* out_n,
                         int* out_src, float* out_score, float* out_angle, float* out_dmin, float* out_dmax,
                         int* n_out) {
    SfMResult sfm = make_sfm(cams_krt, registered, n_cams, pos, toff, timg, n_pts);
    std::vector<MVSViewParams> v = selectSourceViews(sfm, num_sources);
    for (size_t i = 0; i < v.size(); ++i) {
        out_ref[i] = v[i].ref_image_id;
        out_n[i] = static_cast<int>(v[i].source_views.size());
        for (size_t k = 0; k < v[i].source_views.size() && k < 8; ++k) {
            out_src[8 * i + k] = v[i].source_views[k].image_id;
            out_score[8 * i + k] = v[i].source_views[k].score;
            out_angle[8 * i + k] = v[i].source_views[k].baseline_deg;
        }
        out_dmin[i] = v[i].depth_min;
        out_dmax[i] = v[i].depth_max;
    }
    *n_out = static_cast<int>(v.size());
    return 0;
}

// runPatchMatchMVS with mvs_iterations = 0 and the given patch size on W x H
// grayscale images (one per camera): each returned view's id, depth and
// normal (the random init with the SfM seeds painted over it).
int pmref_run_stage(const float* const* grays, int W, int H, const double* cams_krt, const int* registered,
                    int n_cams, const double* pos, const int* toff, const int* timg, int n_pts, int patch_size,
                    int* out_ids, float* out_depth, float* out_normal, int* n_out) {
    SfMResult sfm = make_sfm(cams_krt, registered, n_cams, pos, toff, timg, n_pts);
    std::vector<ImageData> images(n_cams);
    for (int c = 0; c < n_cams; ++c) {
        images[c].gray = cv::Mat(H, W, CV_32F);
        std::memcpy(images[c].gray.data, grays[c], static_cast<size_t>(W) * H * sizeof(float));
        images[c].width = W;
        images[c].height = H;
        images[c].id = c;
    }
    PipelineConfig config;
    config.mvs_iterations = 0;
    config.mvs_patch_size = patch_size;
    config.verbose = false;
    config.save_intermediate = false;
    std::vector<DepthMap> maps = runPatchMatchMVS(images, sfm.cameras, sfm, config);
    const size_t n = static_cast<size_t>(W) * H;
    for (size_t i = 0; i < maps.size(); ++i) {
        out_ids[i] = maps[i].image_id;
        std::memcpy(out_depth + i * n, maps[i].depth.data, n * sizeof(float));
        std::memcpy(out_normal + i * 3 * n, maps[i].normal.data, 3 * n * sizeof(float));
    }
    *n_out = static_cast<int>(maps.size());
    return 0;
}


// Per-view homography coefficients exactly as the reference computes them:
// K^-1 in FP64 cast to FP32, then A = K_s R_rel K_ref^-1, b = K_s t_rel in FP32.
// Cameras are packed as K(9) R(9) t(3) doubles, row-major.
int pmref_setup_views(const double* ref_krt, const double* src_krt, int S, float* kinv9, float* ab) {
    GPUCameraParams ref = eigenToGPUCamera(to_pose(ref_krt));
    std::vector<GPUCameraParams> srcs;
    for (int s = 0; s < S; ++s) srcs.push_back(eigenToGPUCamera(to_pose(src_krt + 21 * s)));
    std::vector<GPUSourceView> v = precomputeSourceViews(ref, srcs);
    std::memcpy(kinv9, ref.K_inv, 9 * sizeof(float));
    for (int s = 0; s < S; ++s) {
        std::memcpy(ab + 12 * s, v[s].A, 9 * sizeof(float));
        std::memcpy(ab + 12 * s + 9, v[s].b, 3 * sizeof(float));
    }
    return 0;
}

// compute_ncc_cost_kernel on fixed (depth, normal[AoS]) maps.  radius <= 5.
int pmref_ncc_cost(const float* ref_img, const float* const* src_imgs, int S, int W, int H,
                   const float* kinv9, const float* ab, const float* depth, const float* normal,
                   int radius, float* cost) {
    if (radius < 1 || radius > NCC_PATCH_RADIUS || S < 1 || S > MAX_SRC_VIEWS) return 1;
    TexSet t;
    make_textures(t, ref_img, src_imgs, S, W, H);
    size_t n = static_cast<size_t>(W) * H;
    DeviceBuffer<float> d_depth, d_normal, d_cost, d_kinv;
    d_depth.upload(depth, n);
    d_normal.upload(normal, 3 * n);
    d_cost.alloc(n);
    d_kinv.upload(kinv9, 9);
    launchNCCCostKernel(t.ref_tex, t.src_tex, d_depth.ptr, d_normal.ptr, d_kinv.ptr,
                        unpack_views(ab, S), d_cost.ptr, radius, W, H);
    d_cost.download(cost, n);
    return 0;
}

// computePixelCost on fixed maps, one thread per pixel; any radius (texture reads only).
int pmref_pixel_cost(const float* ref_img, const float* const* src_imgs, int S, int W, int H,
                     const float* kinv9, const float* ab, const float* depth, const float* normal,
                     int radius, float* cost) {
    if (radius < 1 || S < 1 || S > MAX_SRC_VIEWS) return 1;
    TexSet t;
    make_textures(t, ref_img, src_imgs, S, W, H);
    size_t n = static_cast<size_t>(W) * H;
    DeviceBuffer<float> d_depth, d_normal, d_cost, d_kinv;
    d_depth.upload(depth, n);
    d_normal.upload(normal, 3 * n);
    d_cost.alloc(n);
    d_kinv.upload(kinv9, 9);
    DeviceBuffer<cudaTextureObject_t> d_tex;
    d_tex.upload(t.src_tex.data(), S);
    std::vector<GPUSourceView> views = unpack_views(ab, S);
    DeviceBuffer<GPUSourceView> d_views;
    d_views.upload(views.data(), S);
    dim3 block(16, 16), grid((W + 15) / 16, (H + 15) / 16);
    pixel_cost_wrapper_kernel<<<grid, block>>>(t.ref_tex, d_tex.ptr, d_depth.ptr, d_normal.ptr, d_kinv.ptr,
                                               d_views.ptr, d_cost.ptr, radius, W, H, S);
    CUDA_CHECK_KERNEL();
    d_cost.download(cost, n);
    return 0;
}

int pmref_init(const float* kinv9, int W, int H, float dmin, float dmax, unsigned long long seed,
               float* depth, float* normal) {
    size_t n = static_cast<size_t>(W) * H;
    DeviceBuffer<float> d_depth, d_normal, d_kinv;
    d_depth.alloc(n);
    d_normal.alloc(3 * n);
    d_kinv.upload(kinv9, 9);
    launchInitKernel(d_depth.ptr, d_normal.ptr, dmin, dmax, d_kinv.ptr, W, H, seed);
    d_depth.download(depth, n);
    d_normal.download(normal, 3 * n);
    return 0;
}

// One propagate_and_refine_kernel pass, in place on (depth, normal, cost).
int pmref_propagate(const float* ref_img, const float* const* src_imgs, int S, int W, int H,
                    const float* kinv9, const float* ab, float* depth, float* normal, float* cost,
                    float dmin, float dmax, int radius, int iteration, int red_black,
                    unsigned long long seed) {
    if (radius < 1 || S < 1 || S > MAX_SRC_VIEWS) return 1;
    TexSet t;
    make_textures(t, ref_img, src_imgs, S, W, H);
    size_t n = static_cast<size_t>(W) * H;
    DeviceBuffer<float> d_depth, d_normal, d_cost, d_kinv;
    d_depth.upload(depth, n);
    d_normal.upload(normal, 3 * n);
    d_cost.upload(cost, n);
    d_kinv.upload(kinv9, 9);
    DeviceBuffer<cudaTextureObject_t> d_tex;
    d_tex.upload(t.src_tex.data(), S);
    std::vector<GPUSourceView> views = unpack_views(ab, S);
    DeviceBuffer<GPUSourceView> d_views;
    d_views.upload(views.data(), S);
    launchPropagateRefineKernel(t.ref_tex, d_tex.ptr, d_depth.ptr, d_normal.ptr, d_cost.ptr, d_kinv.ptr,
                                d_views.ptr, dmin, dmax, radius, W, H, S, iteration, red_black, seed);
    d_depth.download(depth, n);
    d_normal.download(normal, 3 * n);
    d_cost.download(cost, n);
    return 0;
}

// The per-view solve of runPatchMatchMVS (random init, initial cost, red-black
// iterations with the reference's seed schedule), without the SfM seeding step.
// gpu_ms receives the device time from the init launch to the last pass (CUDA
// events; the reference's own per-launch device synchronisations included).
int pmref_solve_view(const float* ref_img, const float* const* src_imgs, int S, int W, int H,
                     const float* kinv9, const float* ab, float dmin, float dmax, int radius,
                     int iterations, int ref_id, float* depth, float* normal, float* cost,
                     float* gpu_ms) {
    if (radius < 1 || radius > NCC_PATCH_RADIUS || S < 1 || S > MAX_SRC_VIEWS) return 1;
    TexSet t;
    make_textures(t, ref_img, src_imgs, S, W, H);
    size_t n = static_cast<size_t>(W) * H;
    DeviceBuffer<float> d_depth, d_normal, d_cost, d_kinv;
    d_depth.alloc(n);
    d_normal.alloc(3 * n);
    d_cost.alloc(n);
    d_kinv.upload(kinv9, 9);
    std::vector<GPUSourceView> views = unpack_views(ab, S);
    DeviceBuffer<cudaTextureObject_t> d_tex;
    d_tex.upload(t.src_tex.data(), S);
    DeviceBuffer<GPUSourceView> d_views;
    d_views.upload(views.data(), S);
    cudaEvent_t e0, e1;
    cudaEventCreate(&e0);
    cudaEventCreate(&e1);
    cudaEventRecord(e0);
    unsigned long long seed = 42ull + static_cast<unsigned long long>(ref_id) * 1000000ull;
    launchInitKernel(d_depth.ptr, d_normal.ptr, dmin, dmax, d_kinv.ptr, W, H, seed);
    launchNCCCostKernel(t.ref_tex, t.src_tex, d_depth.ptr, d_normal.ptr, d_kinv.ptr, views, d_cost.ptr,
                        radius, W, H);
    for (int iter = 0; iter < iterations; ++iter) {
        launchPropagateRefineKernel(t.ref_tex, d_tex.ptr, d_depth.ptr, d_normal.ptr, d_cost.ptr, d_kinv.ptr,
                                    d_views.ptr, dmin, dmax, radius, W, H, S, iter, 0, seed + 100ull * iter);
        launchPropagateRefineKernel(t.ref_tex, d_tex.ptr, d_depth.ptr, d_normal.ptr, d_cost.ptr, d_kinv.ptr,
                                    d_views.ptr, dmin, dmax, radius, W, H, S, iter, 1,
                                    seed + 100ull * iter + 50ull);
    }
    cudaEventRecord(e1);
    cudaEventSynchronize(e1);
    float ms = 0.f;
    cudaEventElapsedTime(&ms, e0, e1);
    if (gpu_ms) *gpu_ms = ms;
    cudaEventDestroy(e0);
    cudaEventDestroy(e1);
    d_depth.download(depth, n);
    d_normal.download(normal, 3 * n);
    d_cost.download(cost, n);
    return 0;
}

// geometric_consistency_filter_kernel.  ref_depth / ref_conf are updated in place.
// src_krt packs K(9) R(9) t(3) doubles per source, cast to float as the reference does.
int pmref_geometric_filter(float* ref_depth, const float* ref_normal, float* ref_conf,
                           const double* ref_krt, const float* src_depths, const float* src_normals,
                           const double* src_krt, int S, int W, int H, float depth_tol,
                           float normal_tol_cos, int min_consistent) {
    GPUCameraParams ref = eigenToGPUCamera(to_pose(ref_krt));
    std::vector<GeomFilterSrcView> fsv(S);
    for (int s = 0; s < S; ++s) {
        GPUCameraParams g = eigenToGPUCamera(to_pose(src_krt + 21 * s));
        std::memcpy(fsv[s].K, g.K, sizeof g.K);
        std::memcpy(fsv[s].R, g.R, sizeof g.R);
        std::memcpy(fsv[s].t, g.t, sizeof g.t);
    }
    size_t n = static_cast<size_t>(W) * H;
    DeviceBuffer<float> d_depth, d_normal, d_conf, d_kinv, d_R, d_t, d_sd, d_sn;
    d_depth.upload(ref_depth, n);
    d_normal.upload(ref_normal, 3 * n);
    d_conf.upload(ref_conf, n);
    d_kinv.upload(ref.K_inv, 9);
    d_R.upload(ref.R, 9);
    d_t.upload(ref.t, 3);
    d_sd.upload(src_depths, S * n);
    d_sn.upload(src_normals, 3 * S * n);
    DeviceBuffer<GeomFilterSrcView> d_views;
    d_views.upload(fsv.data(), S);
    launchGeometricFilterKernel(d_depth.ptr, d_normal.ptr, d_conf.ptr, d_kinv.ptr, d_R.ptr, d_t.ptr, d_sd.ptr,
                                d_sn.ptr, d_views.ptr, depth_tol, normal_tol_cos, min_consistent, S, W, H);
    d_depth.download(ref_depth, n);
    d_conf.download(ref_conf, n);
    return 0;
}

}  // extern "C"
