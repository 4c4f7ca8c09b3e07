// Runs the engine's C++ stage adapter, include/hpmvs_stage.hpp, the way the
// reference would: inside the reference's own PatchMatch translation unit
// (src/dense_recon/patchmatch_mvs.cu, compiled unmodified from where it lies),
// whose data model and selectSourceViews the adapter uses, linked against the
// engine library.  A flat C ABI lets tests drive it on the same images,
// cameras and sparse points they give the Python stage mirror.
//
// TEST INFRASTRUCTURE ONLY: it exists to execute the adapter, which outside
// this harness is only compiled.  The data-model types come from the
// stand-in headers under shim/.

#ifndef PMREF_SOURCE
#error "PMREF_SOURCE must name the reference patchmatch_mvs.cu"
#endif
#include PMREF_SOURCE

#include <cstring>
#include <string>
#include <vector>

#include "hpmvs_stage.hpp"

namespace {

CameraPose pose_of(const double* krt) {
    CameraPose c;
    for (int i = 0; i < 9; ++i) c.K(i / 3, i % 3) = krt[i];
    for (int i = 0; i < 9; ++i) c.R(i / 3, i % 3) = krt[9 + i];
    for (int i = 0; i < 3; ++i) c.t(i) = krt[18 + i];
    c.is_registered = true;
    return c;
}

}  // namespace

extern "C" {

// hpmvs_stage::runPatchMatchMVS on W x H grayscale images (one per camera;
// camera c is K R t, 21 doubles, at cams_krt + 21 c) and sparse points (point
// p at pos + 3 p, seen by cameras timg[toff[p] .. toff[p + 1])).  Per returned
// view: its image id, depth, normal (AoS) and confidence.  *status receives
// the adapter's hp_status; the return value is 0.  output_dir, when not null,
// turns on save_intermediate with output_path inside it.
int pmstage_run(const float* const* grays, int W, int H, const double* cams_krt, int n_cams, const double* pos,
                const int* toff, const int* timg, int n_pts, int patch_size, int iterations, const char* output_dir,
                int* out_ids, float* out_depth, float* out_normal, float* out_conf, int* n_out, int* status) {
    SfMResult sfm;
    sfm.num_registered = n_cams;
    for (int c = 0; c < n_cams; ++c) {
        CameraPose cp = pose_of(cams_krt + 21 * c);
        cp.image_id = c;
        sfm.cameras.push_back(cp);
    }
    for (int p = 0; p < n_pts; ++p) {
        SparsePoint sp;
        for (int i = 0; i < 3; ++i) sp.position(i) = pos[3 * p + i];
        for (int k = toff[p]; k < toff[p + 1]; ++k) sp.image_ids.push_back(timg[k]);
        sp.track_length = toff[p + 1] - toff[p];
        sfm.points.push_back(sp);
    }
    std::vector<ImageData> images(n_cams);
    for (int c = 0; c < n_cams; ++c) {
        images[c].gray = cv::Mat(H, W, CV_32F);
        std::memcpy(images[c].gray.data, grays[c], static_cast<size_t>(W) * H * sizeof(float));
        images[c].width = W;
        images[c].height = H;
        images[c].id = c;
    }
    PipelineConfig config;
    config.mvs_iterations = iterations;
    config.mvs_patch_size = patch_size;
    config.verbose = false;
    config.save_intermediate = output_dir != nullptr;
    if (output_dir) config.output_path = std::string(output_dir) + "/cloud.ply";
    hp_status st = HP_OK;
    std::vector<DepthMap> maps = hpmvs_stage::runPatchMatchMVS(images, sfm.cameras, sfm, config, &st);
    *status = static_cast<int>(st);
    const size_t n = static_cast<size_t>(W) * H;
    for (size_t i = 0; i < maps.size(); ++i) {
        out_ids[i] = maps[i].image_id;
        std::memcpy(out_depth + i * n, maps[i].depth.data, n * sizeof(float));
        std::memcpy(out_normal + i * 3 * n, maps[i].normal.data, 3 * n * sizeof(float));
        std::memcpy(out_conf + i * n, maps[i].confidence.data, n * sizeof(float));
    }
    *n_out = static_cast<int>(maps.size());
    return 0;
}

}  // extern "C"
