// SfM front of the dense stage (include/hpmvs.h): source-view selection,
// depth ranges and seed projection from the sparse reconstruction, as
// runPatchMatchMVS derives them (src/dense_recon/patchmatch_mvs.cu:74-157,
// :1111-1177).  Host code: a few thousand points and tens of cameras.
//
// Arithmetic follows the reference's: FP64 vectors with left-to-right sums
// (P_cam = R P + t, centres -R^T t, unit vectors v / |v|), float casts where
// it casts.  The shared-point counts come from one pass over the tracks
// (every pair of cameras in a track) instead of the reference's per-pair scan
// of all points; the counts are the same.
#include <algorithm>
#include <cmath>
#include <cstring>
#include <vector>

#include "../../include/hpmvs.h"

namespace {

constexpr float kBaselineMinDeg = 5.0f;   // BASELINE_MIN_DEG, patchmatch_mvs.cu:19
constexpr float kBaselineMaxDeg = 30.0f;  // BASELINE_MAX_DEG, :20
constexpr double kPi = 3.14159265358979323846;

struct V3 {
    double x, y, z;
};

V3 sub(V3 a, V3 b) { return {a.x - b.x, a.y - b.y, a.z - b.z}; }
double dot(V3 a, V3 b) { return a.x * b.x + a.y * b.y + a.z * b.z; }
V3 unit(V3 a) {
    const double n = std::sqrt(dot(a, a));
    return n > 0.0 ? V3{a.x / n, a.y / n, a.z / n} : a;
}

// R P + t (row-major R).
V3 to_camera(const hp_camera& c, V3 p) {
    const double* R = c.R;
    return {R[0] * p.x + R[1] * p.y + R[2] * p.z + c.t[0], R[3] * p.x + R[4] * p.y + R[5] * p.z + c.t[1],
            R[6] * p.x + R[7] * p.y + R[8] * p.z + c.t[2]};
}

// Camera centre -R^T t.
V3 centre(const hp_camera& c) {
    const double* R = c.R;
    const double* t = c.t;
    return {-R[0] * t[0] + -R[3] * t[1] + -R[6] * t[2], -R[1] * t[0] + -R[4] * t[1] + -R[7] * t[2],
            -R[2] * t[0] + -R[5] * t[1] + -R[8] * t[2]};
}

V3 point(const hp_sparse_points* p, int i) {
    return {p->position[3 * i], p->position[3 * i + 1], p->position[3 * i + 2]};
}

bool valid_points(const hp_sparse_points* p, int num_cams) {
    if (!p || p->num_points < 0) return false;
    if (p->num_points == 0) return true;
    if (!p->position || !p->track_offset || !p->track_images || p->track_offset[0] != 0) return false;
    for (int i = 0; i < p->num_points; ++i)
        if (p->track_offset[i + 1] < p->track_offset[i]) return false;
    const int n = p->track_offset[p->num_points];
    for (int k = 0; k < n; ++k)
        if (p->track_images[k] < 0 || p->track_images[k] >= num_cams) return false;
    return true;
}

bool sees(const hp_sparse_points* p, int i, int cam) {
    for (int k = p->track_offset[i]; k < p->track_offset[i + 1]; ++k)
        if (p->track_images[k] == cam) return true;
    return false;
}

// Baseline angle (degrees) between the rays from two camera centres to the centroid (:54-63).
float baseline_angle(const hp_camera& a, const hp_camera& b, V3 centroid) {
    const V3 va = unit(sub(centroid, centre(a)));
    const V3 vb = unit(sub(centroid, centre(b)));
    const double c = std::min(1.0, std::max(-1.0, dot(va, vb)));
    return static_cast<float>(std::acos(c) * 180.0 / kPi);
}

// sin(angle) with the angle clamped to [5, 30] degrees; 0 outside [5, 90] (:66-72).
float baseline_score(float deg) {
    if (deg < kBaselineMinDeg || deg > kBaselineMaxDeg * 3.0f) return 0.0f;
    const float c = std::min(std::max(deg, kBaselineMinDeg), kBaselineMaxDeg);
    return std::sin(c * static_cast<float>(kPi) / 180.0f);
}

}  // namespace

extern "C" {

hp_status hp_select_sources(const hp_camera* cams, const int* registered, int num_cams,
                            const hp_sparse_points* points, int num_sources, hp_view_selection* out,
                            int* num_out) {
    if (!cams || !registered || num_cams < 1 || !out || !num_out || num_sources < 1 ||
        num_sources > HP_MAX_SOURCES || !valid_points(points, num_cams))
        return HP_ERR_INVALID_ARG;
    const int P = points->num_points;
    V3 centroid{0.0, 0.0, 0.0};
    for (int i = 0; i < P; ++i) {
        const V3 p = point(points, i);
        centroid.x += p.x;
        centroid.y += p.y;
        centroid.z += p.z;
    }
    if (P > 0) {
        centroid.x /= static_cast<double>(P);
        centroid.y /= static_cast<double>(P);
        centroid.z /= static_cast<double>(P);
    }
    // Shared points per camera pair, and per camera the points it sees.
    std::vector<int> shared(static_cast<size_t>(num_cams) * num_cams, 0);
    std::vector<std::vector<int>> seen(num_cams);
    std::vector<char> mark(num_cams, 0);
    std::vector<int> track;
    for (int i = 0; i < P; ++i) {
        track.clear();
        for (int k = points->track_offset[i]; k < points->track_offset[i + 1]; ++k) {
            const int c = points->track_images[k];
            if (!mark[c]) {  // a camera listed twice in a track counts once, as in the reference
                mark[c] = 1;
                track.push_back(c);
            }
        }
        for (int c : track) {
            mark[c] = 0;
            seen[c].push_back(i);
        }
        for (size_t a = 0; a < track.size(); ++a)
            for (size_t b = 0; b < track.size(); ++b)
                if (a != b) shared[static_cast<size_t>(track[a]) * num_cams + track[b]]++;
    }
    int n = 0;
    struct Cand {
        int id;
        float score, angle;
    };
    std::vector<Cand> cand;
    for (int ref = 0; ref < num_cams; ++ref) {
        if (!registered[ref]) continue;
        hp_view_selection& v = out[n++];
        std::memset(&v, 0, sizeof v);
        v.ref_image = ref;
        cand.clear();
        for (int src = 0; src < num_cams; ++src) {
            if (!registered[src] || src == ref) continue;
            const float angle = baseline_angle(cams[ref], cams[src], centroid);
            const float b = baseline_score(angle);
            if (b <= 0.0f) continue;
            const int sh = shared[static_cast<size_t>(ref) * num_cams + src];
            if (sh == 0) continue;
            cand.push_back({src, static_cast<float>(sh) * b, angle});
        }
        std::stable_sort(cand.begin(), cand.end(), [](const Cand& a, const Cand& b) { return a.score > b.score; });
        v.num_sources = std::min(num_sources, static_cast<int>(cand.size()));
        for (int s = 0; s < v.num_sources; ++s) {
            v.sources[s] = cand[s].id;
            v.scores[s] = cand[s].score;
            v.baseline_deg[s] = cand[s].angle;
        }
        // Depth range from the points this view sees (:125-147).
        std::vector<float> depths;
        depths.reserve(seen[ref].size());
        for (int i : seen[ref]) {
            const V3 pc = to_camera(cams[ref], point(points, i));
            if (pc.z > 0) depths.push_back(static_cast<float>(pc.z));
        }
        if (depths.size() >= 2) {
            std::sort(depths.begin(), depths.end());
            const size_t i5 = static_cast<size_t>(depths.size() * 0.05);
            const size_t i95 = std::min(static_cast<size_t>(depths.size() * 0.95), depths.size() - 1);
            v.depth_min = depths[i5] * 0.5f;
            v.depth_max = depths[i95] * 1.5f;
        } else {
            const float d = static_cast<float>(to_camera(cams[ref], centroid).z);
            v.depth_min = d * 0.3f;
            v.depth_max = d * 3.0f;
        }
    }
    *num_out = n;
    return HP_OK;
}

hp_status hp_project_seeds(const hp_camera* cam, int ref, float depth_min, float depth_max,
                           const hp_sparse_points* points, hp_seed* out, int capacity, int* num_seeds) {
    if (!cam || ref < 0 || !num_seeds || capacity < 0 || (capacity > 0 && !out) || !valid_points(points, 1 << 30))
        return HP_ERR_INVALID_ARG;
    const V3 c = centre(*cam);
    const double* K = cam->K;
    int n = 0;
    for (int i = 0; i < points->num_points; ++i) {
        if (!sees(points, i, ref)) continue;
        const V3 P = point(points, i);
        const V3 pc = to_camera(*cam, P);
        if (pc.z <= 0) continue;
        // K P_cam and the rounded pixel (std::round: halves away from zero).
        const double u = K[0] * pc.x + K[1] * pc.y + K[2] * pc.z;
        const double v = K[3] * pc.x + K[4] * pc.y + K[5] * pc.z;
        const double w = K[6] * pc.x + K[7] * pc.y + K[8] * pc.z;
        const double fx = std::round(u / w), fy = std::round(v / w);
        const float depth = static_cast<float>(pc.z);
        if (depth < depth_min || depth > depth_max) continue;
        // A pixel beyond +-2^30 cannot reach an image of at most 16384 px, even with its square.
        if (!(std::fabs(fx) < 1073741824.0 && std::fabs(fy) < 1073741824.0)) continue;
        // Normal: the unit vector from the point to the camera centre, rotated into the camera frame.
        const V3 to_cam = unit(sub(c, P));
        const double* R = cam->R;
        const V3 nc{R[0] * to_cam.x + R[1] * to_cam.y + R[2] * to_cam.z,
                    R[3] * to_cam.x + R[4] * to_cam.y + R[5] * to_cam.z,
                    R[6] * to_cam.x + R[7] * to_cam.y + R[8] * to_cam.z};
        if (n < capacity) {
            hp_seed& s = out[n];
            s.x = static_cast<int>(fx);
            s.y = static_cast<int>(fy);
            s.depth = depth;
            s.normal[0] = static_cast<float>(nc.x);
            s.normal[1] = static_cast<float>(nc.y);
            s.normal[2] = static_cast<float>(nc.z);
        }
        ++n;
    }
    *num_seeds = n;
    return HP_OK;
}

}  // extern "C"
