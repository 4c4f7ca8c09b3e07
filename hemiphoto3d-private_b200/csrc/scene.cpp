// Synthetic multi-view scenes with analytic ground truth (host C++, OpenMP).
//
// The reference renders a textured sphere with a CPU ray caster to exercise
// its pipeline (src/utils/synthetic_data.cpp:75, :222).  This generator renders
// the planes-and-spheres scenes the engine is measured on: every surface
// carries one albedo texture of uniform noise blurred by a Gaussian, mapped
// planar on planes and triplanar on spheres, so a surface point has the same
// value in every view.  Ray casting also yields exact per-pixel depth (camera
// z) and camera-frame normals.
#include "scene.h"

#include <algorithm>
#include <cmath>
#include <cstdint>
#include <cstring>
#include <vector>

namespace {

uint64_t splitmix64(uint64_t& s) {
    uint64_t z = (s += 0x9E3779B97F4A7C15ull);
    z = (z ^ (z >> 30)) * 0xBF58476D1CE4E5B9ull;
    z = (z ^ (z >> 27)) * 0x94D049BB133111EBull;
    return z ^ (z >> 31);
}

inline double dot3(const double* a, const double* b) { return a[0] * b[0] + a[1] * b[1] + a[2] * b[2]; }

struct Tex {
    const float* data;
    int n;
    double tpm;
    float at(long i, long j) const {
        i %= n;
        j %= n;
        if (i < 0) i += n;
        if (j < 0) j += n;
        return data[j * n + i];
    }
    // Bilinear, wrap addressing; (s, t) in metres.
    double sample(double s, double t) const {
        double x = s * tpm, y = t * tpm;
        double fx = std::floor(x), fy = std::floor(y);
        long i = static_cast<long>(fx), j = static_cast<long>(fy);
        double a = x - fx, b = y - fy;
        return (1 - a) * (1 - b) * at(i, j) + a * (1 - b) * at(i + 1, j) + (1 - a) * b * at(i, j + 1) +
               a * b * at(i + 1, j + 1);
    }
};

// First hit along origin + s*dir (s > 1e-9).  Returns object index or -1.
int intersect(const hps_object* objs, int n, const double* o, const double* d, double* s_hit) {
    int best = -1;
    double bs = 1e300;
    for (int k = 0; k < n; ++k) {
        const hps_object& ob = objs[k];
        if (ob.kind == HPS_SPHERE) {
            double oc[3] = {o[0] - ob.p[0], o[1] - ob.p[1], o[2] - ob.p[2]};
            double a = dot3(d, d), b = 2 * dot3(oc, d), c = dot3(oc, oc) - ob.radius * ob.radius;
            double disc = b * b - 4 * a * c;
            if (disc < 0) continue;
            double sq = std::sqrt(disc);
            double s = (-b - sq) / (2 * a);
            if (s <= 1e-9) s = (-b + sq) / (2 * a);
            if (s > 1e-9 && s < bs) { bs = s; best = k; }
        } else {
            double den = dot3(d, ob.n);
            if (std::fabs(den) < 1e-14) continue;
            double po[3] = {ob.p[0] - o[0], ob.p[1] - o[1], ob.p[2] - o[2]};
            double s = dot3(po, ob.n) / den;
            if (s <= 1e-9 || s >= bs) continue;
            if (ob.half_u > 0 || ob.half_v > 0) {
                double x[3] = {o[0] + s * d[0] - ob.p[0], o[1] + s * d[1] - ob.p[1], o[2] + s * d[2] - ob.p[2]};
                if (ob.half_u > 0 && std::fabs(dot3(x, ob.u)) > ob.half_u) continue;
                if (ob.half_v > 0 && std::fabs(dot3(x, ob.v)) > ob.half_v) continue;
            }
            bs = s;
            best = k;
        }
    }
    *s_hit = bs;
    return best;
}

double albedo(const hps_object& ob, const Tex& tex, const double* x) {
    if (ob.kind == HPS_SPHERE) {
        double q[3] = {x[0] - ob.p[0], x[1] - ob.p[1], x[2] - ob.p[2]};
        double w[3], ws = 0;
        for (int k = 0; k < 3; ++k) {
            double a = q[k] / ob.radius;
            w[k] = a * a * a * a;
            ws += w[k];
        }
        double v = 0;
        v += w[0] * tex.sample(q[1] + ob.tex_offset[0], q[2] + ob.tex_offset[1]);
        v += w[1] * tex.sample(q[2] + ob.tex_offset[1], q[0] + ob.tex_offset[0]);
        v += w[2] * tex.sample(q[0] + 0.37 + ob.tex_offset[0], q[1] + 0.61 + ob.tex_offset[1]);
        return v / ws;
    }
    double r[3] = {x[0] - ob.p[0], x[1] - ob.p[1], x[2] - ob.p[2]};
    return tex.sample(dot3(r, ob.u) + ob.tex_offset[0], dot3(r, ob.v) + ob.tex_offset[1]);
}

void inv3(const double* m, double* inv) {
    double det = m[0] * (m[4] * m[8] - m[5] * m[7]) - m[1] * (m[3] * m[8] - m[5] * m[6]) +
                 m[2] * (m[3] * m[7] - m[4] * m[6]);
    double id = 1.0 / det;
    inv[0] = (m[4] * m[8] - m[5] * m[7]) * id;
    inv[1] = (m[2] * m[7] - m[1] * m[8]) * id;
    inv[2] = (m[1] * m[5] - m[2] * m[4]) * id;
    inv[3] = (m[5] * m[6] - m[3] * m[8]) * id;
    inv[4] = (m[0] * m[8] - m[2] * m[6]) * id;
    inv[5] = (m[2] * m[3] - m[0] * m[5]) * id;
    inv[6] = (m[3] * m[7] - m[4] * m[6]) * id;
    inv[7] = (m[1] * m[6] - m[0] * m[7]) * id;
    inv[8] = (m[0] * m[4] - m[1] * m[3]) * id;
}

}  // namespace

extern "C" {

int hps_make_albedo(int n, double sigma, uint64_t seed, float contrast_std, float* out) {
    if (n <= 0 || !out || sigma < 0) return 1;
    uint64_t s = seed ^ 0xA1B2C3D4E5F60718ull;
    std::vector<double> a(static_cast<size_t>(n) * n), b(a.size());
    for (auto& v : a) v = static_cast<double>(splitmix64(s) >> 11) * (1.0 / 9007199254740992.0);
    if (sigma > 0) {
        int rad = static_cast<int>(std::ceil(4 * sigma));
        std::vector<double> w(2 * rad + 1);
        double ws = 0;
        for (int i = -rad; i <= rad; ++i) ws += (w[i + rad] = std::exp(-0.5 * i * i / (sigma * sigma)));
        for (auto& v : w) v /= ws;
#pragma omp parallel for schedule(static)
        for (int y = 0; y < n; ++y)
            for (int x = 0; x < n; ++x) {
                double acc = 0;
                for (int i = -rad; i <= rad; ++i) acc += w[i + rad] * a[static_cast<size_t>(y) * n + ((x + i) % n + n) % n];
                b[static_cast<size_t>(y) * n + x] = acc;
            }
#pragma omp parallel for schedule(static)
        for (int y = 0; y < n; ++y)
            for (int x = 0; x < n; ++x) {
                double acc = 0;
                for (int i = -rad; i <= rad; ++i) acc += w[i + rad] * b[static_cast<size_t>(((y + i) % n + n) % n) * n + x];
                a[static_cast<size_t>(y) * n + x] = acc;
            }
    }
    double mean = 0, var = 0;
    for (double v : a) mean += v;
    mean /= a.size();
    for (double v : a) var += (v - mean) * (v - mean);
    double sd = std::sqrt(var / a.size());
    double scale = sd > 0 ? contrast_std / sd : 1.0;
    for (size_t i = 0; i < a.size(); ++i)
        out[i] = static_cast<float>(std::min(0.98, std::max(0.02, 0.5 + (a[i] - mean) * scale)));
    return 0;
}

int hps_render(const hps_object* objs, int n_objs, const float* tex, int tex_n, double texels_per_meter,
               const double* K, const double* R, const double* t, int W, int H, int spp, float background,
               float* img, float* depth, float* normal) {
    if (!objs || n_objs < 0 || !tex || tex_n <= 0 || W <= 0 || H <= 0 || spp <= 0 || !img) return 1;
    Tex tx{tex, tex_n, texels_per_meter};
    double Ki[9];
    inv3(K, Ki);
    double C[3];  // camera centre = -R^T t
    for (int i = 0; i < 3; ++i) C[i] = -(R[i] * t[0] + R[3 + i] * t[1] + R[6 + i] * t[2]);
#pragma omp parallel for schedule(dynamic, 4)
    for (int y = 0; y < H; ++y) {
        for (int x = 0; x < W; ++x) {
            double acc = 0;
            for (int sy = 0; sy < spp; ++sy)
                for (int sx = 0; sx < spp; ++sx) {
                    double px = x + (sx + 0.5) / spp - 0.5, py = y + (sy + 0.5) / spp - 0.5;
                    double dc[3] = {Ki[0] * px + Ki[1] * py + Ki[2], Ki[3] * px + Ki[4] * py + Ki[5],
                                    Ki[6] * px + Ki[7] * py + Ki[8]};
                    double dw[3];
                    for (int i = 0; i < 3; ++i) dw[i] = R[i] * dc[0] + R[3 + i] * dc[1] + R[6 + i] * dc[2];
                    double s;
                    int k = intersect(objs, n_objs, C, dw, &s);
                    if (k < 0) { acc += background; continue; }
                    double X[3] = {C[0] + s * dw[0], C[1] + s * dw[1], C[2] + s * dw[2]};
                    acc += albedo(objs[k], tx, X);
                }
            size_t idx = static_cast<size_t>(y) * W + x;
            img[idx] = static_cast<float>(acc / (spp * spp));
            if (depth || normal) {
                double px = x, py = y;
                double dc[3] = {Ki[0] * px + Ki[1] * py + Ki[2], Ki[3] * px + Ki[4] * py + Ki[5],
                                Ki[6] * px + Ki[7] * py + Ki[8]};
                double dw[3];
                for (int i = 0; i < 3; ++i) dw[i] = R[i] * dc[0] + R[3 + i] * dc[1] + R[6 + i] * dc[2];
                double s;
                int k = intersect(objs, n_objs, C, dw, &s);
                double z = 0, nc[3] = {0, 0, 0};
                if (k >= 0) {
                    double X[3] = {C[0] + s * dw[0], C[1] + s * dw[1], C[2] + s * dw[2]};
                    z = R[6] * X[0] + R[7] * X[1] + R[8] * X[2] + t[2];
                    double nw[3];
                    if (objs[k].kind == HPS_SPHERE) {
                        for (int i = 0; i < 3; ++i) nw[i] = (X[i] - objs[k].p[i]) / objs[k].radius;
                    } else {
                        for (int i = 0; i < 3; ++i) nw[i] = objs[k].n[i];
                    }
                    for (int i = 0; i < 3; ++i) nc[i] = R[3 * i] * nw[0] + R[3 * i + 1] * nw[1] + R[3 * i + 2] * nw[2];
                    if (nc[0] * dc[0] + nc[1] * dc[1] + nc[2] * dc[2] > 0) {
                        for (double& v : nc) v = -v;
                    }
                }
                if (depth) depth[idx] = static_cast<float>(z);
                if (normal) {
                    normal[3 * idx] = static_cast<float>(nc[0]);
                    normal[3 * idx + 1] = static_cast<float>(nc[1]);
                    normal[3 * idx + 2] = static_cast<float>(nc[2]);
                }
            }
        }
    }
    return 0;
}

}  // extern "C"
