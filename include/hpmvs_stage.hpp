// hpmvs_stage.hpp - header-only C++ adapter: the reference's dense stage
//     std::vector<DepthMap> runPatchMatchMVS(images, cameras, sfm, config)
// (src/dense_recon/patchmatch_mvs.h:39-44), and its consumer fuseDepthMaps
// (src/dense_recon/point_cloud.h:7), implemented on the B200 engine's C ABI
// (hpmvs.h).  It is meant to be included by the reference's
// patchmatch_mvs.cu, whose data model (types.h: ImageData, CameraPose,
// DepthMap, PipelineConfig; sfm/camera_pose.h: SfMResult) and host-side
// selectSourceViews it uses; it compiles wherever those headers do.
//
// Behaviour follows runPatchMatchMVS (:1028-1388): sources and depth range from
// selectSourceViews, radius (mvs_patch_size - 1) / 2 (clamped to the engine's
// 1..7 instead of the reference's 1..5), per-view seed 42 + 1e6 * ref_id,
// confidence 1 - cost / 2 (formed on the device), then the in-place geometric
// filter (tolerance 0.12, normal check off, 2 agreeing views) when iterations
// > 0 and >= 2 maps, as the solve's last stage on the device.  With
// save_intermediate the PFM depth of each view is written before the filter,
// as the reference does, so the filter then runs on the host maps through
// hp_geometric_filter (the same check, the same bits).  The initial hypotheses are seeded
// from the SfM points each view sees (:1111-1177, radius 50) through
// hp_project_seeds.  Errors are reported by return value (an empty vector and
// `*status`), never by exit().
#pragma once

#include <algorithm>
#include <cmath>
#include <cstring>
#include <string>
#include <vector>

#include "hpmvs.h"

namespace hpmvs_stage {

inline hp_camera to_hp_camera(const CameraPose& c) {
    hp_camera h;
    for (int r = 0; r < 3; ++r) {
        for (int k = 0; k < 3; ++k) {
            h.K[3 * r + k] = c.K(r, k);
            h.R[3 * r + k] = c.R(r, k);
        }
        h.t[r] = c.t(r);
    }
    return h;
}

inline std::vector<DepthMap> runPatchMatchMVS(const std::vector<ImageData>& images,
                                              const std::vector<CameraPose>& cameras, const SfMResult& sfm,
                                              const PipelineConfig& config, hp_status* status = nullptr) {
    hp_status st_local = HP_OK;
    hp_status& st = status ? *status : st_local;
    std::vector<DepthMap> maps;
    const int num_sources = std::min(HP_MAX_SOURCES, std::max(3, sfm.num_registered - 1));
    std::vector<MVSViewParams> views = selectSourceViews(sfm, num_sources);

    hp_ctx* ctx = nullptr;
    if ((st = hp_ctx_create(config.gpu_id, &ctx)) != HP_OK) return maps;
    std::vector<int> ids(images.size(), -1);
    auto upload = [&](int i) -> bool {
        if (ids[i] >= 0) return true;
        const cv::Mat& g = images[i].gray;  // CV_32F in [0, 1]
        st = hp_image_upload(ctx, g.data, HP_MEMORY_HOST, g.cols, g.rows, HP_DTYPE_F32, &ids[i]);
        return st == HP_OK;
    };

    hp_params params;
    hp_params_default(&params);
    params.radius = std::min(HP_MAX_RADIUS, std::max(1, (config.mvs_patch_size - 1) / 2));
    const bool want_pfm = config.save_intermediate && !config.output_path.empty();
    if (!want_pfm) {  // the geometric filter as the solve's last stage (:1273-1276 constants)
        params.filter_min_consistent = 2;
        params.filter_depth_tol = 0.12f;
        params.filter_normal_cos = -1.0f;  // cos(180 deg): normal check off
    }

    // The sparse points and their tracks, flattened once for hp_project_seeds.
    std::vector<double> pos;
    std::vector<int> toff(1, 0), timg;
    for (const SparsePoint& p : sfm.points) {
        for (int i = 0; i < 3; ++i) pos.push_back(p.position(i));
        for (int id : p.image_ids) timg.push_back(id);
        toff.push_back(static_cast<int>(timg.size()));
    }
    hp_sparse_points pts;
    pts.num_points = static_cast<int>(sfm.points.size());
    pts.position = pos.data();
    pts.track_offset = toff.data();
    pts.track_images = timg.data();
    std::vector<std::vector<hp_seed>> seeds;
    seeds.reserve(views.size());

    std::vector<hp_job> jobs;
    std::vector<const MVSViewParams*> solved;
    for (const MVSViewParams& vp : views) {
        if (vp.source_views.empty()) continue;  // :1089-1092
        if (!upload(vp.ref_image_id)) break;
        hp_job j;
        std::memset(&j, 0, sizeof j);
        j.ref_image = ids[vp.ref_image_id];
        j.ref_cam = to_hp_camera(cameras[vp.ref_image_id]);
        j.num_sources = static_cast<int>(std::min<size_t>(vp.source_views.size(), HP_MAX_SOURCES));
        for (int s = 0; s < j.num_sources; ++s) {
            const int id = vp.source_views[s].image_id;
            if (!upload(id)) break;
            j.src_images[s] = ids[id];
            j.src_cams[s] = to_hp_camera(cameras[id]);
        }
        if (st != HP_OK) break;
        j.depth_min = vp.depth_min;
        j.depth_max = vp.depth_max;
        j.seed = 42ull + static_cast<uint64_t>(vp.ref_image_id) * 1000000ull;  // :1106
        j.view_id = static_cast<uint32_t>(vp.ref_image_id);
        j.iterations = config.mvs_iterations;
        // SfM seeding (:1111-1177): the points this view sees, painted over the random init.
        const hp_camera seed_cam = to_hp_camera(cameras[vp.ref_image_id]);
        int n_seeds = 0;
        st = hp_project_seeds(&seed_cam, vp.ref_image_id, vp.depth_min, vp.depth_max, &pts, nullptr, 0, &n_seeds);
        if (st != HP_OK) break;
        seeds.emplace_back(static_cast<size_t>(n_seeds));
        if (n_seeds > 0 &&
            (st = hp_project_seeds(&seed_cam, vp.ref_image_id, vp.depth_min, vp.depth_max, &pts,
                                   seeds.back().data(), n_seeds, &n_seeds)) != HP_OK)
            break;
        j.seeds = seeds.back().data();
        j.num_seeds = n_seeds;
        j.seed_radius = 50;  // SEED_RADIUS, :1123
        jobs.push_back(j);
        solved.push_back(&vp);
    }
    std::vector<hp_maps> out(jobs.size());
    std::vector<std::vector<float>> costs(jobs.size());
    for (size_t k = 0; st == HP_OK && k < jobs.size(); ++k) {
        const ImageData& img = images[solved[k]->ref_image_id];
        DepthMap dm;
        dm.image_id = solved[k]->ref_image_id;
        dm.width = img.width;
        dm.height = img.height;
        dm.depth = cv::Mat(img.height, img.width, CV_32F);
        dm.normal = cv::Mat(img.height, img.width, CV_32FC3);
        dm.confidence = cv::Mat(img.height, img.width, CV_32F);
        maps.push_back(dm);
        costs[k].resize(static_cast<size_t>(img.width) * img.height);
        out[k].memory = HP_MEMORY_HOST;
        out[k].depth = reinterpret_cast<float*>(maps.back().depth.data);
        out[k].normal = reinterpret_cast<float*>(maps.back().normal.data);
        out[k].cost = costs[k].data();
        out[k].confidence = reinterpret_cast<float*>(maps.back().confidence.data);  // 1 - cost / 2 (:1246-1252)
    }
    if (st == HP_OK && !jobs.empty())
        st = hp_solve(ctx, jobs.data(), static_cast<int>(jobs.size()), &params, out.data());
    if (st == HP_OK && want_pfm) {
        const std::string dir = config.output_path.substr(0, config.output_path.find_last_of('/'));
        for (const DepthMap& dm : maps)
            hp_pfm_write((dir + "/depth_" + std::to_string(dm.image_id) + ".pfm").c_str(),
                         reinterpret_cast<const float*>(dm.depth.data), dm.width, dm.height, 1);
        if (config.mvs_iterations > 0 && maps.size() >= 2) {  // :1267-1384, in place, in view order
            for (size_t k = 0; st == HP_OK && k < maps.size(); ++k) {
                std::vector<hp_camera> cams;
                std::vector<const float*> sd, sn;
                for (const SourceViewInfo& sv : solved[k]->source_views) {
                    int m_last = -1;  // the last map of that image, as the reference's id lookup
                    for (size_t m = 0; m < maps.size(); ++m)
                        if (maps[m].image_id == sv.image_id) m_last = static_cast<int>(m);
                    if (m_last < 0 || m_last == static_cast<int>(k) || maps[m_last].width != maps[k].width ||
                        maps[m_last].height != maps[k].height || cams.size() >= HP_MAX_SOURCES)
                        continue;
                    cams.push_back(to_hp_camera(cameras[sv.image_id]));
                    sd.push_back(reinterpret_cast<const float*>(maps[m_last].depth.data));
                    sn.push_back(reinterpret_cast<const float*>(maps[m_last].normal.data));
                }
                if (cams.size() < 2) continue;
                hp_camera ref = to_hp_camera(cameras[maps[k].image_id]);
                st = hp_geometric_filter(ctx, &ref, maps[k].width, maps[k].height,
                                         reinterpret_cast<float*>(maps[k].depth.data),
                                         reinterpret_cast<const float*>(maps[k].normal.data),
                                         reinterpret_cast<float*>(maps[k].confidence.data),
                                         static_cast<int>(cams.size()), cams.data(), sd.data(), sn.data(),
                                         HP_MEMORY_HOST, 0.12f, -1.0f /* cos(180 deg): normal check off */, 2);
            }
        }
    }
    hp_ctx_destroy(ctx);
    if (st != HP_OK) maps.clear();
    return maps;
}

// fuseDepthMaps(depth_maps, poses, images) (src/dense_recon/point_cloud.h:7, a
// stub at point_cloud.cu:4-8) on hp_fuse_depth_maps: poses and images are
// indexed by each map's image_id, every other map is a neighbour, and the
// tolerances are the engine's defaults.  The colour is the gray value.
inline DensePointCloud fuseDepthMaps(const std::vector<DepthMap>& depth_maps, const std::vector<CameraPose>& poses,
                                     const std::vector<ImageData>& images, hp_status* status = nullptr,
                                     int gpu_id = 0) {
    static_assert(sizeof(Eigen::Vector3f) == 3 * sizeof(float), "DensePointCloud arrays are packed float3");
    hp_status st_local = HP_OK;
    hp_status& st = status ? *status : st_local;
    DensePointCloud cloud;
    if (depth_maps.empty()) return cloud;
    std::vector<hp_fuse_view> v(depth_maps.size());
    for (size_t i = 0; i < depth_maps.size(); ++i) {
        const DepthMap& dm = depth_maps[i];
        const size_t id = static_cast<size_t>(dm.image_id);
        if (id >= poses.size()) {
            st = HP_ERR_INVALID_ARG;
            return cloud;
        }
        std::memset(&v[i], 0, sizeof v[i]);
        v[i].cam = to_hp_camera(poses[id]);
        v[i].depth = reinterpret_cast<const float*>(dm.depth.data);
        v[i].normal = reinterpret_cast<const float*>(dm.normal.data);  // camera frame, as the stage writes it
        v[i].confidence = dm.confidence.empty() ? nullptr : reinterpret_cast<const float*>(dm.confidence.data);
        v[i].gray = id < images.size() && !images[id].gray.empty()
                        ? reinterpret_cast<const float*>(images[id].gray.data)
                        : nullptr;
        v[i].width = dm.width;
        v[i].height = dm.height;
    }
    hp_ctx* ctx = nullptr;
    if ((st = hp_ctx_create(gpu_id, &ctx)) != HP_OK) return cloud;
    hp_fuse_params fp;
    hp_fuse_params_default(&fp);
    fp.memory = HP_MEMORY_HOST;
    hp_point_cloud pc;
    std::memset(&pc, 0, sizeof pc);
    pc.memory = HP_MEMORY_HOST;
    st = hp_fuse_depth_maps(ctx, v.data(), static_cast<int>(v.size()), &fp, &pc);  // counts
    if (st == HP_OK && pc.count > 0) {
        cloud.positions.resize(static_cast<size_t>(pc.count));
        cloud.normals.resize(static_cast<size_t>(pc.count));
        cloud.colors.resize(static_cast<size_t>(pc.count));
        pc.positions = reinterpret_cast<float*>(cloud.positions.data());
        pc.normals = reinterpret_cast<float*>(cloud.normals.data());
        pc.colors = reinterpret_cast<float*>(cloud.colors.data());
        pc.capacity = pc.count;
        st = hp_fuse_depth_maps(ctx, v.data(), static_cast<int>(v.size()), &fp, &pc);
    }
    hp_ctx_destroy(ctx);
    if (st != HP_OK) cloud = DensePointCloud();
    return cloud;
}

}  // namespace hpmvs_stage
