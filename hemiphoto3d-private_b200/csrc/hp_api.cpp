// Host side of the C ABI declared in include/hpmvs.h.
//
// A context owns one CUDA stream on one device, the uploaded images (FP32 and
// FP16 pitched planes plus linear-filter texture objects over block-linear
// arrays), and grow-only scratch for hypotheses.  A solve builds one ViewDesc
// per job, uploads them once, and issues every red-black half-pass as a single
// launch over the tiles of all jobs still iterating, with no host
// synchronisation between launches (the reference synchronises after each,
// src/utils/cuda_utils.cuh:18-22).
#include <cuda_fp16.h>
#include <cuda_runtime.h>

#include <algorithm>
#include <climits>
#include <cmath>
#include <cstdarg>
#include <cstdio>
#include <cstring>
#include <map>
#include <memory>
#include <string>
#include <vector>

#include "hp_host.h"

using namespace hpx;

namespace {

void mat3_mul(const double* a, const double* b, double* c) {
    for (int r = 0; r < 3; ++r)
        for (int k = 0; k < 3; ++k)
            c[3 * r + k] = a[3 * r] * b[k] + a[3 * r + 1] * b[3 + k] + a[3 * r + 2] * b[6 + k];
}

bool mat3_inv(const double* m, double* inv) {
    double det = m[0] * (m[4] * m[8] - m[5] * m[7]) - m[1] * (m[3] * m[8] - m[5] * m[6]) +
                 m[2] * (m[3] * m[7] - m[4] * m[6]);
    if (!(std::fabs(det) > 1e-300)) return false;
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
    return true;
}

}  // namespace

namespace hpx {

hp_status check_params(hp_ctx* ctx, const hp_params* p) {
    if (!p) return fail(ctx, HP_ERR_INVALID_ARG, "params is null");
    if (p->radius < 1 || p->radius > HP_MAX_RADIUS)
        return fail(ctx, HP_ERR_INVALID_ARG, "radius %d outside 1..%d", p->radius, HP_MAX_RADIUS);
    if (p->stride < 1 || p->stride > 2) return fail(ctx, HP_ERR_INVALID_ARG, "stride %d not 1 or 2", p->stride);
    if (p->top_k < 1 || p->top_k > HP_MAX_TOP_K)
        return fail(ctx, HP_ERR_INVALID_ARG, "top_k %d outside 1..%d", p->top_k, HP_MAX_TOP_K);
    if (p->precision != HP_PRECISION_F32 && p->precision != HP_PRECISION_F16ACC)
        return fail(ctx, HP_ERR_INVALID_ARG, "unknown precision %d", p->precision);
    if (p->refine_steps < 0 || p->refine_steps > 4)
        return fail(ctx, HP_ERR_INVALID_ARG, "refine_steps %d outside 0..4", p->refine_steps);
    if (!(p->iter_decay > 0.f && p->iter_decay <= 1.f) || !(p->step_decay > 0.f && p->step_decay <= 1.f))
        return fail(ctx, HP_ERR_INVALID_ARG, "decay factors must lie in (0, 1]");
    if (p->filter_min_consistent < 0 || p->filter_min_consistent > HP_MAX_SOURCES)
        return fail(ctx, HP_ERR_INVALID_ARG, "filter_min_consistent %d outside 0..%d", p->filter_min_consistent,
                    HP_MAX_SOURCES);
    if (p->filter_min_consistent > 0 &&
        (!(p->filter_depth_tol >= 0.f) || !std::isfinite(p->filter_depth_tol) || std::isnan(p->filter_normal_cos)))
        return fail(ctx, HP_ERR_INVALID_ARG, "filter tolerances invalid");
    if (p->tile_w != 0 && p->tile_w != hp::TILE_W)
        return fail(ctx, HP_ERR_UNSUPPORTED, "tile width %d: the kernels use %d", p->tile_w, hp::TILE_W);
    if (p->tile_h != 0 && p->tile_h != 8 && !(p->tile_h == 4 && p->precision == HP_PRECISION_F16ACC))
        return fail(ctx, HP_ERR_UNSUPPORTED, "tile height %d: 8, or 4 on the FP16-acc path", p->tile_h);
    if (p->staging != 0 && p->staging != 4 && p->staging != 8)
        return fail(ctx, HP_ERR_INVALID_ARG, "staging %d not 0, 4 or 8", p->staging);
    if (p->debug_checked_taps != 0 && p->debug_checked_taps != 1)
        return fail(ctx, HP_ERR_INVALID_ARG, "debug_checked_taps %d not 0 or 1", p->debug_checked_taps);
#ifndef HP_SELF_CHECK
    if (p->debug_checked_taps)
        return fail(ctx, HP_ERR_UNSUPPORTED, "debug_checked_taps needs the self-checking build (make check)");
#endif
    return HP_OK;
}

hp::SolveConsts consts_of(const hp_params* p) {
    hp::SolveConsts sc;
    sc.radius = p->radius;
    sc.stride = p->stride;
    sc.top_k = p->top_k;
    sc.refine_steps = p->refine_steps;
    sc.iter_decay = p->iter_decay;
    sc.step_decay = p->step_decay;
    // Default: every source through the software sampler (measured fastest).
    sc.soft_mask = p->precision == HP_PRECISION_F16ACC
                       ? (p->soft_sources < 0 ? 0xFFu : static_cast<unsigned>(p->soft_sources) & 0xFFu)
                       : 0u;
    if (p->precision == HP_PRECISION_F16ACC && p->debug_checked_taps) sc.soft_mask |= hp::SOFT_MASK_CHECKED;
    sc.tile_h = p->tile_h > 0 ? p->tile_h : hp::TILE_H;
    sc.staging = p->staging > 0 ? p->staging : 4;
    return sc;
}

// Validate a job and fill the image/camera part of its descriptor.
hp_status fill_desc(hp_ctx* ctx, const hp_job* j, int jobno, hp::ViewDesc* d, int tile_h) {
    std::memset(d, 0, sizeof *d);
    auto it = ctx->images.find(j->ref_image);
    if (it == ctx->images.end()) return fail(ctx, HP_ERR_NOT_FOUND, "job %d: unknown ref image %d", jobno, j->ref_image);
    const Image& ref = it->second;
    if (j->num_sources < 1 || j->num_sources > HP_MAX_SOURCES)
        return fail(ctx, HP_ERR_INVALID_ARG, "job %d: num_sources %d outside 1..%d", jobno, j->num_sources,
                    HP_MAX_SOURCES);
    if (!(j->depth_min > 0.f) || !(j->depth_max > j->depth_min) || !std::isfinite(j->depth_max))
        return fail(ctx, HP_ERR_INVALID_ARG, "job %d: depth range [%g, %g] invalid", jobno, j->depth_min,
                    j->depth_max);
    if (j->iterations < 0 || j->iterations > 1000)
        return fail(ctx, HP_ERR_INVALID_ARG, "job %d: iterations %d outside 0..1000", jobno, j->iterations);
    d->ref = ref.f32;
    d->ref16 = ref.f16;
    d->ref_pitch = static_cast<int>(ref.pitch32 / sizeof(float));
    d->ref16_pitch = static_cast<int>(ref.pitch16 / sizeof(__half));
    d->W = ref.W;
    d->H = ref.H;
    d->S = j->num_sources;
    for (int s = 0; s < j->num_sources; ++s) {
        auto si = ctx->images.find(j->src_images[s]);
        if (si == ctx->images.end())
            return fail(ctx, HP_ERR_NOT_FOUND, "job %d: unknown source image %d", jobno, j->src_images[s]);
        if (si->second.W != ref.W || si->second.H != ref.H)
            return fail(ctx, HP_ERR_INVALID_ARG, "job %d: source %d is %dx%d, reference is %dx%d", jobno, s,
                        si->second.W, si->second.H, ref.W, ref.H);
        d->src_tex[s] = si->second.tex32;
        d->src_tex16[s] = si->second.tex16;
        d->src_quad[s] = si->second.quads.base;
    }
    if (j->use_coeffs) {
        std::memcpy(d->kinv, j->kinv, sizeof d->kinv);
        for (int s = 0; s < j->num_sources; ++s) std::memcpy(d->ab[s], j->ab[s], sizeof d->ab[s]);
    } else {
        double kinv[9], ab[HP_MAX_SOURCES * 12];
        hp_status st = hp_setup_homographies(&j->ref_cam, j->src_cams, j->num_sources, kinv, ab);
        if (st != HP_OK) return fail(ctx, st, "job %d: singular reference intrinsics", jobno);
        for (int i = 0; i < 9; ++i) d->kinv[i] = static_cast<float>(kinv[i]);
        for (int s = 0; s < j->num_sources; ++s)
            for (int i = 0; i < 12; ++i) d->ab[s][i] = static_cast<float>(ab[12 * s + i]);
    }
    d->tile_h = tile_h;
    d->tiles_x = (ref.W + hp::TILE_W - 1) / hp::TILE_W;
    d->tiles_y = (ref.H + tile_h - 1) / tile_h;
    d->dmin = j->depth_min;
    d->dmax = j->depth_max;
    d->seed_lo = static_cast<uint32_t>(j->seed);
    d->seed_hi = static_cast<uint32_t>(j->seed >> 32);
    d->view_id = j->view_id;
    d->iterations = j->iterations;
    return HP_OK;
}

hp_status check_seeds(hp_ctx* ctx, const hp_job* j, int jobno) {
    if (j->num_seeds == 0) return HP_OK;
    if (j->num_seeds < 0 || j->num_seeds > (1 << 26) || !j->seeds || j->seed_radius < 0 || j->seed_radius > 4096)
        return fail(ctx, HP_ERR_INVALID_ARG, "job %d: seeds (%d, radius %d) invalid", jobno, j->num_seeds,
                    j->seed_radius);
    return HP_OK;
}

size_t seed_area_bytes(const hp_job* j, int W, int H) {
    if (j->num_seeds <= 0) return 0;
    auto a = [](size_t x) { return (x + 255) & ~size_t(255); };
    return a(static_cast<size_t>(j->num_seeds) * sizeof(hp_seed)) + a(static_cast<size_t>(W) * H * sizeof(int));
}

cudaError_t stage_seeds(const hp_job* j, void* area, hp::ViewDesc* d, cudaStream_t st) {
    d->seeds = nullptr;
    d->seed_map = nullptr;
    if (j->num_seeds <= 0) return cudaSuccess;
    const size_t list = ((static_cast<size_t>(j->num_seeds) * sizeof(hp_seed)) + 255) & ~size_t(255);
    hp_seed* seeds = static_cast<hp_seed*>(area);
    int* map = reinterpret_cast<int*>(static_cast<char*>(area) + list);
    // A pageable source: the copy has completed when the call returns.
    cudaError_t e = cudaMemcpyAsync(seeds, j->seeds, static_cast<size_t>(j->num_seeds) * sizeof(hp_seed),
                                    cudaMemcpyHostToDevice, st);
    if (e == cudaSuccess) e = hp::launch_seed_map(seeds, j->num_seeds, j->seed_radius, d->W, d->H, map, st);
    if (e == cudaSuccess) {
        d->seeds = seeds;
        d->seed_map = map;
    }
    return e;
}

bool filter_source_of(const hp_camera& ref, const hp_camera& src, hp::FilterSource* q) {
    double kinv[9];
    if (!mat3_inv(ref.K, kinv)) return false;
    double RrT[9], Rrel[9], M[9], A[9], trel[3];
    for (int r = 0; r < 3; ++r)
        for (int c = 0; c < 3; ++c) RrT[3 * r + c] = ref.R[3 * c + r];
    mat3_mul(src.R, RrT, Rrel);  // reference camera frame -> source camera frame
    for (int r = 0; r < 3; ++r)
        trel[r] = src.t[r] - (Rrel[3 * r] * ref.t[0] + Rrel[3 * r + 1] * ref.t[1] + Rrel[3 * r + 2] * ref.t[2]);
    mat3_mul(Rrel, kinv, M);  // pixel ray -> source camera frame
    mat3_mul(src.K, M, A);
    for (int i = 0; i < 9; ++i) {
        q->A[i] = static_cast<float>(A[i]);
        q->Rn[i] = static_cast<float>(Rrel[i]);
    }
    for (int r = 0; r < 3; ++r)
        q->b[r] = static_cast<float>(src.K[3 * r] * trel[0] + src.K[3 * r + 1] * trel[1] + src.K[3 * r + 2] * trel[2]);
    for (int c = 0; c < 3; ++c) q->m[c] = static_cast<float>(M[6 + c]);
    q->cz = static_cast<float>(trel[2]);
    q->view = -1;
    return true;
}

void filter_stages(const hp_job* jobs, int n, const hp_params* p, const std::vector<hp::ViewDesc>& descs,
                   std::vector<hp::FilterStage>* stages, std::vector<char>* has, std::vector<int>* order) {
    stages->assign(n, hp::FilterStage{});
    has->assign(n, 0);
    order->clear();
    if (!p || p->filter_min_consistent <= 0 || n < 2) return;
    std::map<int, int> solved;  // ref image -> the last job solving it
    for (int k = 0; k < n; ++k) solved[jobs[k].ref_image] = k;
    for (int k = 0; k < n; ++k) {
        if (jobs[k].iterations <= 0) continue;
        hp::FilterStage& f = (*stages)[k];
        std::memset(&f, 0, sizeof f);
        for (int i = 0; i < jobs[k].num_sources; ++i) {
            auto it = solved.find(jobs[k].src_images[i]);
            if (it == solved.end() || it->second == k) continue;
            const int j = it->second;
            if (descs[j].W != descs[k].W || descs[j].H != descs[k].H) continue;
            hp::FilterSource& q = f.src[f.n];
            if (!filter_source_of(jobs[k].ref_cam, jobs[k].src_cams[i], &q)) continue;
            q.view = j;
            ++f.n;
        }
        if (f.n < p->filter_min_consistent) continue;
        f.min_consistent = p->filter_min_consistent;
        f.depth_tol = p->filter_depth_tol;
        f.normal_cos = p->filter_normal_cos;
        f.prev = order->empty() ? -1 : order->back();
        f.tiles_done = nullptr;
        (*has)[k] = 1;
        order->push_back(k);
    }
}

}  // namespace hpx

namespace {

// Everything one solve needs on the device: descriptors, state, launch lists.
struct Prepared {
    std::vector<hp::ViewDesc> host;   // host copies (with device pointers)
    hp::ViewDesc* dev = nullptr;
    std::vector<int> list_offsets;    // per iteration: offset into lists buffer
    std::vector<int> list_counts;     // per iteration: number of active views
    std::vector<int> list_tiles;      // per iteration: total tiles
    int* lists = nullptr;
    int max_iter = 0;
    std::vector<int> filter_order;    // jobs with a filter stage, in the order they run
    int tile_h = hp::TILE_H;          // rows per tile of this solve's kernels
};

hp_status prepare(hp_ctx* ctx, const hp_job* jobs, int n, const hp_params* params, Prepared* P,
                  bool with_seeds = false, bool with_filter = false) {
    P->host.resize(n);
    P->tile_h = consts_of(params).tile_h;
    const hp_params* filter = with_filter ? params : nullptr;
    size_t state_bytes = 0;
    std::vector<size_t> offs(n);
    for (int k = 0; k < n; ++k) {
        hp_status st = fill_desc(ctx, &jobs[k], k, &P->host[k], P->tile_h);
        if (st != HP_OK) return st;
        offs[k] = state_bytes;
        size_t px = static_cast<size_t>(P->host[k].W) * P->host[k].H;
        state_bytes += ((px * sizeof(float4) + px * sizeof(float)) + 255) & ~size_t(255);
        P->max_iter = std::max(P->max_iter, jobs[k].iterations);
    }
    HP_CUDA(ctx->state.ensure(state_bytes));
    for (int k = 0; k < n; ++k) {
        char* base = static_cast<char*>(ctx->state.p) + offs[k];
        size_t px = static_cast<size_t>(P->host[k].W) * P->host[k].H;
        P->host[k].hyp = reinterpret_cast<float4*>(base);
        P->host[k].cost = reinterpret_cast<float*>(base + px * sizeof(float4));
    }
    if (with_seeds) {  // SfM seed lists and index maps, read by the initialisation stage
        size_t seed_bytes = 0;
        for (int k = 0; k < n; ++k) {
            hp_status st = check_seeds(ctx, &jobs[k], k);
            if (st != HP_OK) return st;
            seed_bytes += seed_area_bytes(&jobs[k], P->host[k].W, P->host[k].H);
        }
        if (seed_bytes) HP_CUDA(ctx->seedbuf.ensure(seed_bytes));
        size_t off = 0;
        for (int k = 0; k < n; ++k) {
            HP_CUDA(stage_seeds(&jobs[k], static_cast<char*>(ctx->seedbuf.p) + off, &P->host[k], ctx->stream));
            off += seed_area_bytes(&jobs[k], P->host[k].W, P->host[k].H);
        }
    }
    {  // geometric-consistency stages after the last half-pass (hp_params.filter_*)
        std::vector<hp::FilterStage> stages;
        std::vector<char> has;
        filter_stages(jobs, n, filter, P->host, &stages, &has, &P->filter_order);
        if (!P->filter_order.empty()) {
            HP_CUDA(ctx->filters.ensure(n * sizeof(hp::FilterStage)));
            hp::FilterStage* fd = static_cast<hp::FilterStage*>(ctx->filters.p);
            HP_CUDA(cudaMemcpyAsync(fd, stages.data(), n * sizeof(hp::FilterStage), cudaMemcpyHostToDevice,
                                    ctx->stream));
            for (int k = 0; k < n; ++k) P->host[k].filter = has[k] ? fd + k : nullptr;
        }
    }
    HP_CUDA(ctx->descs.ensure(n * sizeof(hp::ViewDesc)));
    P->dev = static_cast<hp::ViewDesc*>(ctx->descs.p);
    HP_CUDA(cudaMemcpyAsync(P->dev, P->host.data(), n * sizeof(hp::ViewDesc), cudaMemcpyHostToDevice,
                            ctx->stream));
    // Launch lists: entry 0 covers all views (init, initial cost); entry 1+it
    // the views still iterating at iteration it.
    std::vector<int> ints;
    const int n_lists = 1 + P->max_iter;
    for (int l = 0; l < n_lists; ++l) {
        std::vector<int> act;
        for (int k = 0; k < n; ++k)
            if (l == 0 || jobs[k].iterations > l - 1) act.push_back(k);
        P->list_offsets.push_back(static_cast<int>(ints.size()));
        P->list_counts.push_back(static_cast<int>(act.size()));
        for (int k : act) ints.push_back(k);
        int acc = 0;
        for (int k : act) {
            ints.push_back(acc);
            acc += P->host[k].tiles_x * P->host[k].tiles_y;
        }
        ints.push_back(acc);
        P->list_tiles.push_back(acc);
    }
    HP_CUDA(ctx->lists.ensure(ints.size() * sizeof(int)));
    P->lists = static_cast<int*>(ctx->lists.p);
    HP_CUDA(cudaMemcpyAsync(P->lists, ints.data(), ints.size() * sizeof(int), cudaMemcpyHostToDevice,
                            ctx->stream));
    // The staging vectors above are pageable: the copies complete before return.
    HP_CUDA(cudaStreamSynchronize(ctx->stream));
    flush_profile(ctx);
    return HP_OK;
}

hp::BatchList batch_of(const Prepared& P, int list) {
    hp::BatchList bl;
    bl.views = P.dev;
    bl.n_active = P.list_counts[list];
    bl.active = P.lists + P.list_offsets[list];
    bl.tile_prefix = bl.active + bl.n_active;
    bl.total_tiles = P.list_tiles[list];
    return bl;
}

// Copy a job's packed state out to the caller's maps.
hp_status export_maps(hp_ctx* ctx, const Prepared& P, int k, hp_maps* m, bool want_depth_normal, bool want_cost) {
    const hp::ViewDesc& v = P.host[k];
    const size_t px = static_cast<size_t>(v.W) * v.H;
    float* d = want_depth_normal ? m->depth : nullptr;
    float* nrm = want_depth_normal ? m->normal : nullptr;
    float* c = want_cost ? m->cost : nullptr;
    float* cf = want_cost ? m->confidence : nullptr;
    if (m->memory == HP_MEMORY_DEVICE) {
        HP_CUDA(counted(ctx, HP_KERNEL_OTHER,
                        [&] { return hp::launch_unpack(P.host.data(), k, d, nrm, c, cf, ctx->stream); }));
        return HP_OK;
    }
    HP_CUDA(ctx->staging.ensure(px * 6 * sizeof(float)));
    float* sd = static_cast<float*>(ctx->staging.p);
    float* sn = sd + px;
    float* sc = sn + 3 * px;
    float* scf = sc + px;
    HP_CUDA(counted(ctx, HP_KERNEL_OTHER, [&] {
        return hp::launch_unpack(P.host.data(), k, d ? sd : nullptr, nrm ? sn : nullptr, c ? sc : nullptr,
                                 cf ? scf : nullptr, ctx->stream);
    }));
    if (d) HP_CUDA(cudaMemcpyAsync(d, sd, px * sizeof(float), cudaMemcpyDeviceToHost, ctx->stream));
    if (nrm) HP_CUDA(cudaMemcpyAsync(nrm, sn, 3 * px * sizeof(float), cudaMemcpyDeviceToHost, ctx->stream));
    if (c) HP_CUDA(cudaMemcpyAsync(c, sc, px * sizeof(float), cudaMemcpyDeviceToHost, ctx->stream));
    if (cf) HP_CUDA(cudaMemcpyAsync(cf, scf, px * sizeof(float), cudaMemcpyDeviceToHost, ctx->stream));
    HP_CUDA(cudaStreamSynchronize(ctx->stream));
    flush_profile(ctx);
    return HP_OK;
}

// Load caller maps into a job's packed state.
hp_status import_maps(hp_ctx* ctx, const Prepared& P, int k, const hp_maps* m, bool with_cost) {
    const hp::ViewDesc& v = P.host[k];
    const size_t px = static_cast<size_t>(v.W) * v.H;
    if (!m->depth || !m->normal || (with_cost && !m->cost))
        return fail(ctx, HP_ERR_INVALID_ARG, "maps: depth/normal%s pointer is null", with_cost ? "/cost" : "");
    if (m->memory == HP_MEMORY_DEVICE) {
        HP_CUDA(counted(ctx, HP_KERNEL_OTHER, [&] {
            return hp::launch_pack(P.host.data(), k, m->depth, m->normal, with_cost ? m->cost : nullptr, ctx->stream);
        }));
        return HP_OK;
    }
    HP_CUDA(ctx->staging.ensure(px * 5 * sizeof(float)));
    float* sd = static_cast<float*>(ctx->staging.p);
    float* sn = sd + px;
    float* sc = sn + 3 * px;
    HP_CUDA(cudaMemcpyAsync(sd, m->depth, px * sizeof(float), cudaMemcpyHostToDevice, ctx->stream));
    HP_CUDA(cudaMemcpyAsync(sn, m->normal, 3 * px * sizeof(float), cudaMemcpyHostToDevice, ctx->stream));
    if (with_cost) HP_CUDA(cudaMemcpyAsync(sc, m->cost, px * sizeof(float), cudaMemcpyHostToDevice, ctx->stream));
    HP_CUDA(counted(ctx, HP_KERNEL_OTHER,
                    [&] { return hp::launch_pack(P.host.data(), k, sd, sn, with_cost ? sc : nullptr, ctx->stream); }));
    HP_CUDA(cudaStreamSynchronize(ctx->stream));
    flush_profile(ctx);
    return HP_OK;
}

hp_status launch_cost(hp_ctx* ctx, const hp::BatchList& bl, const hp_params* p) {
    hp::SolveConsts sc = consts_of(p);
    cudaError_t e = counted(ctx, HP_KERNEL_COST, [&] {
        return p->precision == HP_PRECISION_F16ACC ? hp::launch_cost_f16(bl, sc, ctx->stream)
                                                   : hp::launch_cost_f32(bl, sc, ctx->stream);
    });
    HP_CUDA(e);
    return HP_OK;
}

hp_status launch_pass(hp_ctx* ctx, const hp::BatchList& bl, const hp_params* p, int it, int color) {
    hp::SolveConsts sc = consts_of(p);
    cudaError_t e = counted(ctx, HP_KERNEL_PROPAGATE, [&] {
        return p->precision == HP_PRECISION_F16ACC ? hp::launch_propagate_f16(bl, sc, it, color, ctx->stream)
                                                   : hp::launch_propagate_f32(bl, sc, it, color, ctx->stream);
    });
    HP_CUDA(e);
    return HP_OK;
}

}  // namespace

namespace hpx {

size_t image_bytes(const Image& im) {
    const size_t px = static_cast<size_t>(im.W) * im.H;
    return im.pitch32 * im.H + im.pitch16 * im.H + px * (sizeof(float) + sizeof(__half)) + im.quads.physical;
}

void free_image(Image& im) {
    if (im.tex32) cudaDestroyTextureObject(im.tex32);
    if (im.tex16) cudaDestroyTextureObject(im.tex16);
    if (im.arr32) cudaFreeArray(im.arr32);
    if (im.arr16) cudaFreeArray(im.arr16);
    if (im.f32) cudaFree(im.f32);
    if (im.f16) cudaFree(im.f16);
    free_quads(&im.quads);
    im = Image();
}

cudaError_t make_linear_texture(cudaArray_t arr, cudaTextureObject_t* tex) {
    cudaResourceDesc rd;
    std::memset(&rd, 0, sizeof rd);
    rd.resType = cudaResourceTypeArray;
    rd.res.array.array = arr;
    cudaTextureDesc td;
    std::memset(&td, 0, sizeof td);
    td.addressMode[0] = cudaAddressModeClamp;
    td.addressMode[1] = cudaAddressModeClamp;
    td.filterMode = cudaFilterModeLinear;
    td.readMode = cudaReadModeElementType;
    td.normalizedCoords = 0;
    return cudaCreateTextureObject(tex, &rd, &td, nullptr);
}

}  // namespace hpx

extern "C" {

const char* hp_status_string(hp_status s) {
    switch (s) {
        case HP_OK: return "ok";
        case HP_ERR_INVALID_ARG: return "invalid argument";
        case HP_ERR_CUDA: return "CUDA error";
        case HP_ERR_OUT_OF_MEMORY: return "out of device memory";
        case HP_ERR_NOT_FOUND: return "not found";
        case HP_ERR_TIMEOUT: return "timed out";
        case HP_ERR_UNSUPPORTED: return "unsupported";
        case HP_ERR_IO: return "I/O error";
        case HP_ERR_BUSY: return "busy";
        case HP_ERR_CANCELLED: return "cancelled";
    }
    return "unknown status";
}

const char* hp_version(void) { return "0.1.0"; }

void hp_params_default(hp_params* p) {
    if (!p) return;
    p->radius = 5;
    p->stride = 1;
    p->top_k = 3;
    p->precision = HP_PRECISION_F32;
    p->refine_steps = 2;
    p->iter_decay = 0.6f;
    p->step_decay = 0.5f;
    p->tile_w = 0;
    p->tile_h = 0;
    p->soft_sources = -1;
    p->filter_min_consistent = 0;
    p->filter_depth_tol = 0.12f;
    p->filter_normal_cos = -1.0f;
    p->staging = 0;
    p->debug_checked_taps = 0;
}

hp_status hp_ctx_create(int device, hp_ctx** out) {
    if (!out) return HP_ERR_INVALID_ARG;
    *out = nullptr;
    int n = 0;
    if (cudaGetDeviceCount(&n) != cudaSuccess || n == 0) {
        cudaGetLastError();
        return HP_ERR_CUDA;
    }
    if (device < 0 || device >= n) return HP_ERR_INVALID_ARG;
    std::unique_ptr<hp_ctx> c(new hp_ctx);
    c->device = device;
    DeviceGuard g(device);
    if (cudaStreamCreateWithFlags(&c->stream, cudaStreamNonBlocking) != cudaSuccess) return HP_ERR_CUDA;
    *out = c.release();
    return HP_OK;
}

hp_status hp_ctx_destroy(hp_ctx* ctx) {
    if (!ctx) return HP_ERR_INVALID_ARG;
    {
        DeviceGuard g(ctx->device);
        cudaStreamSynchronize(ctx->stream);
        for (auto& kv : ctx->images) free_image(kv.second);
        for (auto& im : ctx->image_cache) free_image(im);
        ctx->upload.release();
        ctx->state.release();
        ctx->descs.release();
        ctx->lists.release();
        ctx->staging.release();
        ctx->seedbuf.release();
        ctx->filters.release();
        for (cudaEvent_t e : ctx->events) cudaEventDestroy(e);
        cudaStreamDestroy(ctx->stream);
    }
    delete ctx;
    return HP_OK;
}

const char* hp_ctx_last_error(const hp_ctx* ctx) { return ctx ? ctx->err.c_str() : "null context"; }

hp_status hp_ctx_synchronize(hp_ctx* ctx) {
    if (!ctx) return HP_ERR_INVALID_ARG;
    DeviceGuard g(ctx->device);
    HP_CUDA(cudaStreamSynchronize(ctx->stream));
    flush_profile(ctx);
    return HP_OK;
}

hp_status hp_ctx_mem_info(hp_ctx* ctx, size_t* free_bytes, size_t* total_bytes) {
    if (!ctx || !free_bytes || !total_bytes) return HP_ERR_INVALID_ARG;
    DeviceGuard g(ctx->device);
    HP_CUDA(cudaMemGetInfo(free_bytes, total_bytes));
    return HP_OK;
}

hp_status hp_ctx_stream(hp_ctx* ctx, void** stream) {
    if (!ctx || !stream) return HP_ERR_INVALID_ARG;
    *stream = static_cast<void*>(ctx->stream);
    return HP_OK;
}

hp_status hp_ctx_set_profiling(hp_ctx* ctx, int enable) {
    if (!ctx) return HP_ERR_INVALID_ARG;
    DeviceGuard g(ctx->device);
    HP_CUDA(cudaStreamSynchronize(ctx->stream));
    flush_profile(ctx);
    ctx->profiling = enable != 0;
    return HP_OK;
}

hp_status hp_ctx_profile(hp_ctx* ctx, hp_profile* out) {
    if (!ctx || !out) return HP_ERR_INVALID_ARG;
    DeviceGuard g(ctx->device);
    HP_CUDA(cudaStreamSynchronize(ctx->stream));
    flush_profile(ctx);
    *out = ctx->prof;
    return HP_OK;
}

hp_status hp_ctx_profile_reset(hp_ctx* ctx) {
    if (!ctx) return HP_ERR_INVALID_ARG;
    DeviceGuard g(ctx->device);
    HP_CUDA(cudaStreamSynchronize(ctx->stream));
    flush_profile(ctx);
    ctx->prof = hp_profile{};
    return HP_OK;
}

hp_status hp_image_upload(hp_ctx* ctx, const void* data, int memory, int width, int height, int dtype,
                          int* image_id) {
    if (!ctx) return HP_ERR_INVALID_ARG;
    if (!data || !image_id) return fail(ctx, HP_ERR_INVALID_ARG, "image_upload: null pointer");
    // 16384: the software sampler's fixed-point coordinate range (hp_kernels_f16.cu, SOFT_MAGIC).
    if (width < 2 || height < 2 || width > 16384 || height > 16384)
        return fail(ctx, HP_ERR_INVALID_ARG, "image_upload: size %dx%d outside 2..16384", width, height);
    if (dtype != HP_DTYPE_U8 && dtype != HP_DTYPE_F16 && dtype != HP_DTYPE_F32)
        return fail(ctx, HP_ERR_INVALID_ARG, "image_upload: unknown dtype %d", dtype);
    if (memory != HP_MEMORY_HOST && memory != HP_MEMORY_DEVICE)
        return fail(ctx, HP_ERR_INVALID_ARG, "image_upload: unknown memory kind %d", memory);
    DeviceGuard g(ctx->device);
    const size_t esz = dtype == HP_DTYPE_U8 ? 1 : (dtype == HP_DTYPE_F16 ? 2 : 4);
    const size_t bytes = static_cast<size_t>(width) * height * esz;
    Image im;
    im.W = width;
    im.H = height;
    auto cleanup = [&]() { free_image(im); };
    cudaError_t e;
#define HP_UP(call)                                                                                   \
    do {                                                                                              \
        e = (call);                                                                                   \
        if (e != cudaSuccess) {                                                                       \
            cleanup();                                                                                \
            return fail(ctx, e == cudaErrorMemoryAllocation ? HP_ERR_OUT_OF_MEMORY : HP_ERR_CUDA,      \
                        "image_upload: %s: %s", #call, cudaGetErrorString(e));                        \
        }                                                                                             \
    } while (0)
    const void* src = data;
    if (memory == HP_MEMORY_HOST) {
        HP_UP(ctx->upload.ensure(bytes));
        HP_UP(cudaMemcpyAsync(ctx->upload.p, data, bytes, cudaMemcpyHostToDevice, ctx->stream));
        src = ctx->upload.p;
    }
    // A released image of the same size lends its buffers (and texture objects) to this one.
    bool reused = false;
    for (size_t k = 0; k < ctx->image_cache.size(); ++k) {
        if (ctx->image_cache[k].W == width && ctx->image_cache[k].H == height) {
            im = ctx->image_cache[k];
            ctx->image_cache_bytes -= image_bytes(im);
            ctx->image_cache.erase(ctx->image_cache.begin() + static_cast<long>(k));
            reused = true;
            break;
        }
    }
    if (!reused) {
        HP_UP(cudaMallocPitch(reinterpret_cast<void**>(&im.f32), &im.pitch32, width * sizeof(float), height));
        HP_UP(cudaMallocPitch(reinterpret_cast<void**>(&im.f16), &im.pitch16, width * sizeof(__half), height));
    }
    HP_UP(counted(ctx, HP_KERNEL_OTHER, [&] {
        return hp::launch_to_f32(src, dtype, width, height, im.f32, static_cast<int>(im.pitch32 / sizeof(float)),
                                 im.f16, static_cast<int>(im.pitch16 / sizeof(__half)), ctx->stream);
    }));
    if (!reused) {
        cudaChannelFormatDesc d32 = cudaCreateChannelDesc<float>();
        cudaChannelFormatDesc d16 = cudaCreateChannelDescHalf();
        HP_UP(cudaMallocArray(&im.arr32, &d32, width, height));
        HP_UP(cudaMallocArray(&im.arr16, &d16, width, height));
    }
    HP_UP(cudaMemcpy2DToArrayAsync(im.arr32, 0, 0, im.f32, im.pitch32, width * sizeof(float), height,
                                   cudaMemcpyDeviceToDevice, ctx->stream));
    HP_UP(cudaMemcpy2DToArrayAsync(im.arr16, 0, 0, im.f16, im.pitch16, width * sizeof(__half), height,
                                   cudaMemcpyDeviceToDevice, ctx->stream));
    if (!reused) HP_UP(alloc_quads(ctx->device, width, height, &im.quads));
    HP_UP(counted(ctx, HP_KERNEL_OTHER, [&] {
        return hp::launch_quads(im.f16, static_cast<int>(im.pitch16 / sizeof(__half)), width, height, im.quads.base,
                                ctx->stream);
    }));
    if (!reused) {
        HP_UP(make_linear_texture(im.arr32, &im.tex32));
        HP_UP(make_linear_texture(im.arr16, &im.tex16));
    }
    HP_UP(cudaStreamSynchronize(ctx->stream));
#undef HP_UP
    int id = ctx->next_id++;
    ctx->images[id] = im;
    *image_id = id;
    return HP_OK;
}

hp_status hp_image_release(hp_ctx* ctx, int image_id) {
    if (!ctx) return HP_ERR_INVALID_ARG;
    auto it = ctx->images.find(image_id);
    if (it == ctx->images.end()) return fail(ctx, HP_ERR_NOT_FOUND, "image_release: unknown image %d", image_id);
    DeviceGuard g(ctx->device);
    cudaStreamSynchronize(ctx->stream);
    // Keep it for reuse when the cache has room (evicting the oldest entries), else free it.
    const size_t b = image_bytes(it->second);
    while (!ctx->image_cache.empty() && ctx->image_cache_bytes + b > ctx->image_cache_limit) {
        ctx->image_cache_bytes -= image_bytes(ctx->image_cache.front());
        free_image(ctx->image_cache.front());
        ctx->image_cache.erase(ctx->image_cache.begin());
    }
    if (b <= ctx->image_cache_limit) {
        ctx->image_cache.push_back(it->second);
        ctx->image_cache_bytes += b;
    } else {
        free_image(it->second);
    }
    ctx->images.erase(it);
    return HP_OK;
}

hp_status hp_ctx_set_image_cache(hp_ctx* ctx, uint64_t limit_bytes) {
    if (!ctx) return HP_ERR_INVALID_ARG;
    DeviceGuard g(ctx->device);
    ctx->image_cache_limit = static_cast<size_t>(limit_bytes);
    while (!ctx->image_cache.empty() && ctx->image_cache_bytes > ctx->image_cache_limit) {
        ctx->image_cache_bytes -= image_bytes(ctx->image_cache.front());
        free_image(ctx->image_cache.front());
        ctx->image_cache.erase(ctx->image_cache.begin());
    }
    return HP_OK;
}

hp_status hp_image_size(hp_ctx* ctx, int image_id, int* width, int* height) {
    if (!ctx || !width || !height) return HP_ERR_INVALID_ARG;
    auto it = ctx->images.find(image_id);
    if (it == ctx->images.end()) return fail(ctx, HP_ERR_NOT_FOUND, "image_size: unknown image %d", image_id);
    *width = it->second.W;
    *height = it->second.H;
    return HP_OK;
}

hp_status hp_setup_homographies(const hp_camera* ref, const hp_camera* srcs, int num_sources, double* kinv9,
                                double* ab) {
    if (!ref || !kinv9 || num_sources < 0 || num_sources > HP_MAX_SOURCES || (num_sources > 0 && (!srcs || !ab)))
        return HP_ERR_INVALID_ARG;
    if (!mat3_inv(ref->K, kinv9)) return HP_ERR_INVALID_ARG;
    double RrT[9];
    for (int r = 0; r < 3; ++r)
        for (int c = 0; c < 3; ++c) RrT[3 * r + c] = ref->R[3 * c + r];
    for (int s = 0; s < num_sources; ++s) {
        const hp_camera& cs = srcs[s];
        double Rrel[9], tmp[9], A[9], trel[3];
        mat3_mul(cs.R, RrT, Rrel);  // R_rel = R_s R_ref^T
        for (int r = 0; r < 3; ++r)
            trel[r] = cs.t[r] - (Rrel[3 * r] * ref->t[0] + Rrel[3 * r + 1] * ref->t[1] + Rrel[3 * r + 2] * ref->t[2]);
        mat3_mul(Rrel, kinv9, tmp);
        mat3_mul(cs.K, tmp, A);  // A = K_s R_rel K_ref^-1
        double* o = ab + 12 * s;
        std::memcpy(o, A, sizeof A);
        for (int r = 0; r < 3; ++r) o[9 + r] = cs.K[3 * r] * trel[0] + cs.K[3 * r + 1] * trel[1] + cs.K[3 * r + 2] * trel[2];
    }
    return HP_OK;
}

hp_status hp_solve(hp_ctx* ctx, const hp_job* jobs, int num_jobs, const hp_params* params, hp_maps* out) {
    if (!ctx) return HP_ERR_INVALID_ARG;
    if (!jobs || !out || num_jobs < 1) return fail(ctx, HP_ERR_INVALID_ARG, "solve: no jobs or outputs");
    hp_status st = check_params(ctx, params);
    if (st != HP_OK) return st;
    for (int k = 0; k < num_jobs; ++k) {
        if (!out[k].depth || !out[k].normal || !out[k].cost)
            return fail(ctx, HP_ERR_INVALID_ARG, "solve: output maps of job %d incomplete", k);
    }
    DeviceGuard g(ctx->device);
    Prepared P;
    if ((st = prepare(ctx, jobs, num_jobs, params, &P, true, true)) != HP_OK) return st;
    hp::BatchList all = batch_of(P, 0);
    HP_CUDA(counted(ctx, HP_KERNEL_INIT, [&] { return hp::launch_init(all, P.tile_h, ctx->stream); }));
    if ((st = launch_cost(ctx, all, params)) != HP_OK) return st;
    for (int it = 0; it < P.max_iter; ++it) {
        hp::BatchList bl = batch_of(P, 1 + it);
        if ((st = launch_pass(ctx, bl, params, it, 0)) != HP_OK) return st;
        if ((st = launch_pass(ctx, bl, params, it, 1)) != HP_OK) return st;
    }
    // Geometric-consistency stage, view by view in job order, in place on the
    // packed state (each launch sees the earlier views already filtered).
    for (int k : P.filter_order) {
        const int tiles = P.host[k].tiles_x * P.host[k].tiles_y;
        HP_CUDA(counted(ctx, HP_KERNEL_OTHER,
                        [&] { return hp::launch_filter_view(P.dev, k, tiles, P.tile_h, false, ctx->stream); }));
    }
    for (int k = 0; k < num_jobs; ++k)
        if ((st = export_maps(ctx, P, k, &out[k], true, true)) != HP_OK) return st;
    HP_CUDA(cudaStreamSynchronize(ctx->stream));
    flush_profile(ctx);
    return HP_OK;
}

hp_status hp_init_hypotheses(hp_ctx* ctx, const hp_job* job, const hp_params* params, hp_maps* out) {
    if (!ctx) return HP_ERR_INVALID_ARG;
    if (!job || !out || !out->depth || !out->normal) return fail(ctx, HP_ERR_INVALID_ARG, "init: null argument");
    hp_status st = check_params(ctx, params);
    if (st != HP_OK) return st;
    DeviceGuard g(ctx->device);
    Prepared P;
    if ((st = prepare(ctx, job, 1, params, &P, true)) != HP_OK) return st;
    HP_CUDA(counted(ctx, HP_KERNEL_INIT, [&] { return hp::launch_init(batch_of(P, 0), P.tile_h, ctx->stream); }));
    if ((st = export_maps(ctx, P, 0, out, true, false)) != HP_OK) return st;
    HP_CUDA(cudaStreamSynchronize(ctx->stream));
    flush_profile(ctx);
    return HP_OK;
}

hp_status hp_ncc_cost(hp_ctx* ctx, const hp_job* job, const hp_params* params, hp_maps* maps) {
    if (!ctx) return HP_ERR_INVALID_ARG;
    if (!job || !maps || !maps->cost) return fail(ctx, HP_ERR_INVALID_ARG, "ncc_cost: null argument");
    hp_status st = check_params(ctx, params);
    if (st != HP_OK) return st;
    DeviceGuard g(ctx->device);
    Prepared P;
    if ((st = prepare(ctx, job, 1, params, &P)) != HP_OK) return st;
    if ((st = import_maps(ctx, P, 0, maps, false)) != HP_OK) return st;
    if ((st = launch_cost(ctx, batch_of(P, 0), params)) != HP_OK) return st;
    if ((st = export_maps(ctx, P, 0, maps, false, true)) != HP_OK) return st;
    HP_CUDA(cudaStreamSynchronize(ctx->stream));
    flush_profile(ctx);
    return HP_OK;
}

hp_status hp_propagate_pass(hp_ctx* ctx, const hp_job* job, const hp_params* params, hp_maps* maps, int iteration,
                            int color) {
    if (!ctx) return HP_ERR_INVALID_ARG;
    if (!job || !maps) return fail(ctx, HP_ERR_INVALID_ARG, "propagate_pass: null argument");
    if (color != 0 && color != 1) return fail(ctx, HP_ERR_INVALID_ARG, "propagate_pass: color %d not 0/1", color);
    if (iteration < 0) return fail(ctx, HP_ERR_INVALID_ARG, "propagate_pass: negative iteration");
    hp_status st = check_params(ctx, params);
    if (st != HP_OK) return st;
    DeviceGuard g(ctx->device);
    Prepared P;
    if ((st = prepare(ctx, job, 1, params, &P)) != HP_OK) return st;
    if ((st = import_maps(ctx, P, 0, maps, true)) != HP_OK) return st;
    if ((st = launch_pass(ctx, batch_of(P, 0), params, iteration, color)) != HP_OK) return st;
    if ((st = export_maps(ctx, P, 0, maps, true, true)) != HP_OK) return st;
    HP_CUDA(cudaStreamSynchronize(ctx->stream));
    flush_profile(ctx);
    return HP_OK;
}

hp_status hp_geometric_filter(hp_ctx* ctx, const hp_camera* ref_cam, int width, int height, float* depth,
                              const float* normal, float* confidence, int num_sources, const hp_camera* src_cams,
                              const float* const* src_depths, const float* const* src_normals, int memory,
                              float depth_tol, float normal_tol_cos, int min_consistent) {
    if (!ctx) return HP_ERR_INVALID_ARG;
    if (!ref_cam || !depth || !normal || !confidence || (num_sources > 0 && (!src_cams || !src_depths || !src_normals)))
        return fail(ctx, HP_ERR_INVALID_ARG, "geometric_filter: null argument");
    if (num_sources < 0 || num_sources > HP_MAX_SOURCES)
        return fail(ctx, HP_ERR_INVALID_ARG, "geometric_filter: num_sources %d outside 0..%d", num_sources,
                    HP_MAX_SOURCES);
    if (width < 1 || height < 1) return fail(ctx, HP_ERR_INVALID_ARG, "geometric_filter: empty map");
    if (min_consistent < 0 || !(depth_tol >= 0.f) || std::isnan(normal_tol_cos))
        return fail(ctx, HP_ERR_INVALID_ARG, "geometric_filter: tolerances invalid");
    DeviceGuard g(ctx->device);
    hp::FilterMaps a;
    std::memset(&a, 0, sizeof a);
    for (int s = 0; s < num_sources; ++s)
        if (!filter_source_of(*ref_cam, src_cams[s], &a.f.src[s]))
            return fail(ctx, HP_ERR_INVALID_ARG, "geometric_filter: singular reference K");
    a.f.n = num_sources;
    a.f.min_consistent = min_consistent;
    a.f.depth_tol = depth_tol;
    a.f.normal_cos = normal_tol_cos;
    a.f.prev = -1;
    a.W = width;
    a.H = height;
    const size_t px = static_cast<size_t>(width) * height;
    if (memory == HP_MEMORY_DEVICE) {
        for (int s = 0; s < num_sources; ++s) {
            a.src_depth[s] = src_depths[s];
            a.src_normal[s] = src_normals[s];
        }
        HP_CUDA(counted(ctx, HP_KERNEL_OTHER,
                        [&] { return hp::launch_filter_maps(a, depth, normal, confidence, ctx->stream); }));
        HP_CUDA(cudaStreamSynchronize(ctx->stream));
        flush_profile(ctx);
        return HP_OK;
    }
    // Host maps: stage ref (depth, normal, conf) and every source map once.
    const size_t need = px * (5 + 4 * static_cast<size_t>(num_sources)) * sizeof(float);
    HP_CUDA(ctx->staging.ensure(need));
    float* sd = static_cast<float*>(ctx->staging.p);
    float* sn = sd + px;
    float* sc = sn + 3 * px;
    float* srcbase = sc + px;
    HP_CUDA(cudaMemcpyAsync(sd, depth, px * 4, cudaMemcpyHostToDevice, ctx->stream));
    HP_CUDA(cudaMemcpyAsync(sn, normal, 3 * px * 4, cudaMemcpyHostToDevice, ctx->stream));
    HP_CUDA(cudaMemcpyAsync(sc, confidence, px * 4, cudaMemcpyHostToDevice, ctx->stream));
    for (int s = 0; s < num_sources; ++s) {
        float* dd = srcbase + static_cast<size_t>(s) * 4 * px;
        HP_CUDA(cudaMemcpyAsync(dd, src_depths[s], px * 4, cudaMemcpyHostToDevice, ctx->stream));
        HP_CUDA(cudaMemcpyAsync(dd + px, src_normals[s], 3 * px * 4, cudaMemcpyHostToDevice, ctx->stream));
        a.src_depth[s] = dd;
        a.src_normal[s] = dd + px;
    }
    HP_CUDA(counted(ctx, HP_KERNEL_OTHER, [&] { return hp::launch_filter_maps(a, sd, sn, sc, ctx->stream); }));
    HP_CUDA(cudaMemcpyAsync(depth, sd, px * 4, cudaMemcpyDeviceToHost, ctx->stream));
    HP_CUDA(cudaMemcpyAsync(confidence, sc, px * 4, cudaMemcpyDeviceToHost, ctx->stream));
    HP_CUDA(cudaStreamSynchronize(ctx->stream));
    flush_profile(ctx);
    return HP_OK;
}

void hp_fuse_params_default(hp_fuse_params* p) {
    if (!p) return;
    p->memory = HP_MEMORY_HOST;
    p->min_views = 2;
    p->min_confidence = 0.0f;
    p->max_depth_rel = 0.01f;
    p->max_reproj_px = 2.0f;
    p->min_normal_cos = 0.98480775f;  // cos(10 deg)
}

hp_status hp_fuse_depth_maps(hp_ctx* ctx, const hp_fuse_view* views, int num_views, const hp_fuse_params* prm,
                             hp_point_cloud* out) {
    if (!ctx) return HP_ERR_INVALID_ARG;
    if (!views || !prm || !out) return fail(ctx, HP_ERR_INVALID_ARG, "fuse: null argument");
    if (num_views < 1) return fail(ctx, HP_ERR_INVALID_ARG, "fuse: no views");
    if (prm->memory != HP_MEMORY_HOST && prm->memory != HP_MEMORY_DEVICE)
        return fail(ctx, HP_ERR_INVALID_ARG, "fuse: map memory %d", prm->memory);
    if (out->memory != HP_MEMORY_HOST && out->memory != HP_MEMORY_DEVICE)
        return fail(ctx, HP_ERR_INVALID_ARG, "fuse: cloud memory %d", out->memory);
    if (prm->min_views < 1) return fail(ctx, HP_ERR_INVALID_ARG, "fuse: min_views %d < 1", prm->min_views);
    if (!(prm->max_depth_rel >= 0.f) || !(prm->max_reproj_px >= 0.f) ||
        !(prm->min_normal_cos >= -1.f && prm->min_normal_cos <= 1.f) || std::isnan(prm->min_confidence))
        return fail(ctx, HP_ERR_INVALID_ARG, "fuse: tolerance out of range");
    if (out->capacity < 0) return fail(ctx, HP_ERR_INVALID_ARG, "fuse: negative capacity");
    DeviceGuard g(ctx->device);
    // Device scratch freed on every return path (cudaFree waits for the device).
    struct Scratch {
        void* p = nullptr;
        ~Scratch() {
            if (p) cudaFree(p);
        }
    };
    const bool dev_in = prm->memory == HP_MEMORY_DEVICE;
    std::vector<hp::FuseView> fv(num_views);
    std::vector<int> nbs, vblock(num_views + 1);
    long long blocks = 0;
    size_t staged_floats = 0;
    for (int i = 0; i < num_views; ++i) {
        const hp_fuse_view& v = views[i];
        if (v.width < 1 || v.height < 1 || v.width > 65536 || v.height > 65536)
            return fail(ctx, HP_ERR_INVALID_ARG, "fuse: view %d size %dx%d", i, v.width, v.height);
        if (!v.depth || !v.normal) return fail(ctx, HP_ERR_INVALID_ARG, "fuse: view %d without depth or normal", i);
        double kinv[9];
        if (!mat3_inv(v.cam.K, kinv)) return fail(ctx, HP_ERR_INVALID_ARG, "fuse: view %d has a singular K", i);
        hp::FuseView& f = fv[i];
        std::memset(&f, 0, sizeof f);
        for (int k = 0; k < 9; ++k) {
            f.K[k] = static_cast<float>(v.cam.K[k]);
            f.kinv[k] = static_cast<float>(kinv[k]);
            f.R[k] = static_cast<float>(v.cam.R[k]);
        }
        for (int k = 0; k < 3; ++k) f.t[k] = static_cast<float>(v.cam.t[k]);
        f.W = v.width;
        f.H = v.height;
        f.nb_begin = static_cast<int>(nbs.size());
        if (v.neighbors) {
            if (v.num_neighbors < 0) return fail(ctx, HP_ERR_INVALID_ARG, "fuse: view %d neighbour count", i);
            for (int k = 0; k < v.num_neighbors; ++k) {
                const int j = v.neighbors[k];
                if (j < 0 || j >= num_views || j == i)
                    return fail(ctx, HP_ERR_INVALID_ARG, "fuse: view %d lists neighbour %d", i, j);
                nbs.push_back(j);
            }
        } else {
            for (int j = 0; j < num_views; ++j)
                if (j != i) nbs.push_back(j);
        }
        f.nb_count = static_cast<int>(nbs.size()) - f.nb_begin;
        vblock[i] = static_cast<int>(blocks);
        const size_t px = static_cast<size_t>(v.width) * v.height;
        blocks += static_cast<long long>((px + hp::FUSE_THREADS - 1) / hp::FUSE_THREADS);
        // The one-CTA scan splits the per-CTA counts into 1024 chunks with int
        // offsets; 2^30 CTAs (2.7e11 pixels) keeps those offsets in range.
        if (blocks > (1ll << 30)) return fail(ctx, HP_ERR_INVALID_ARG, "fuse: too many pixels");
        staged_floats += px * (4 + (v.confidence ? 1 : 0) + (v.gray ? 1 : 0));
    }
    vblock[num_views] = static_cast<int>(blocks);
    if (dev_in) {
        for (int i = 0; i < num_views; ++i) {
            fv[i].depth = views[i].depth;
            fv[i].normal = views[i].normal;
            fv[i].conf = views[i].confidence;
            fv[i].gray = views[i].gray;
        }
    } else {  // host maps go up once through the staging buffer
        HP_CUDA(ctx->staging.ensure(staged_floats * sizeof(float)));
        float* dst = static_cast<float*>(ctx->staging.p);
        auto stage = [&](const float* src, size_t n, const float** field) {
            *field = nullptr;
            if (!src) return cudaSuccess;
            const cudaError_t e = cudaMemcpyAsync(dst, src, n * sizeof(float), cudaMemcpyHostToDevice, ctx->stream);
            *field = dst;
            dst += n;
            return e;
        };
        for (int i = 0; i < num_views; ++i) {
            const size_t px = static_cast<size_t>(views[i].width) * views[i].height;
            HP_CUDA(stage(views[i].depth, px, &fv[i].depth));
            HP_CUDA(stage(views[i].normal, 3 * px, &fv[i].normal));
            HP_CUDA(stage(views[i].confidence, px, &fv[i].conf));
            HP_CUDA(stage(views[i].gray, px, &fv[i].gray));
        }
    }
    // Descriptor block: views | neighbours | first CTA per view | CTA counts | CTA offsets | total.
    auto up8 = [](size_t b) { return (b + 7) / 8 * 8; };
    const size_t o_nb = up8(sizeof(hp::FuseView) * num_views);
    const size_t o_vb = o_nb + up8(sizeof(int) * std::max<size_t>(nbs.size(), 1));
    const size_t o_cnt = o_vb + up8(sizeof(int) * (num_views + 1));
    const size_t o_off = o_cnt + up8(sizeof(int) * blocks);
    const size_t o_tot = o_off + sizeof(long long) * blocks;
    Scratch desc;
    HP_CUDA(cudaMalloc(&desc.p, o_tot + sizeof(long long)));
    char* base = static_cast<char*>(desc.p);
    HP_CUDA(cudaMemcpyAsync(base, fv.data(), sizeof(hp::FuseView) * num_views, cudaMemcpyHostToDevice, ctx->stream));
    if (!nbs.empty())
        HP_CUDA(cudaMemcpyAsync(base + o_nb, nbs.data(), sizeof(int) * nbs.size(), cudaMemcpyHostToDevice,
                                ctx->stream));
    HP_CUDA(cudaMemcpyAsync(base + o_vb, vblock.data(), sizeof(int) * (num_views + 1), cudaMemcpyHostToDevice,
                            ctx->stream));
    hp::FuseArgs a;
    a.views = reinterpret_cast<const hp::FuseView*>(base);
    a.neighbors = reinterpret_cast<const int*>(base + o_nb);
    a.view_block = reinterpret_cast<const int*>(base + o_vb);
    a.n_views = num_views;
    a.min_views = prm->min_views;
    a.min_conf = prm->min_confidence;
    a.max_depth_rel = prm->max_depth_rel;
    a.max_reproj_sq = prm->max_reproj_px * prm->max_reproj_px;
    a.min_normal_cos = prm->min_normal_cos;
    int* counts = reinterpret_cast<int*>(base + o_cnt);
    long long* offsets = reinterpret_cast<long long*>(base + o_off);
    long long* d_total = reinterpret_cast<long long*>(base + o_tot);
    const int nb = static_cast<int>(blocks);
    HP_CUDA(counted(ctx, HP_KERNEL_OTHER, [&] { return hp::launch_fuse_count(a, nb, counts, ctx->stream); }));
    HP_CUDA(counted(ctx, HP_KERNEL_OTHER,
                    [&] { return hp::launch_fuse_scan(counts, nb, offsets, d_total, ctx->stream); }));
    long long total = 0;
    HP_CUDA(cudaMemcpyAsync(&total, d_total, sizeof total, cudaMemcpyDeviceToHost, ctx->stream));
    HP_CUDA(cudaStreamSynchronize(ctx->stream));
    out->count = total;
    const long long nw = std::min<long long>(total, out->capacity);
    if (nw > 0 && (out->positions || out->normals || out->colors)) {
        if (out->memory == HP_MEMORY_DEVICE) {
            HP_CUDA(counted(ctx, HP_KERNEL_OTHER, [&] {
                return hp::launch_fuse_write(a, nb, offsets, out->positions, out->normals, out->colors, nw,
                                             ctx->stream);
            }));
        } else {  // written on the device, then copied out
            const size_t per = static_cast<size_t>(nw) * 3;
            Scratch tmp;
            HP_CUDA(cudaMalloc(&tmp.p, 3 * per * sizeof(float)));
            float* tp = static_cast<float*>(tmp.p);
            float* tn = tp + per;
            float* tc = tn + per;
            HP_CUDA(counted(ctx, HP_KERNEL_OTHER, [&] {
                return hp::launch_fuse_write(a, nb, offsets, out->positions ? tp : nullptr,
                                             out->normals ? tn : nullptr, out->colors ? tc : nullptr, nw,
                                             ctx->stream);
            }));
            if (out->positions)
                HP_CUDA(cudaMemcpyAsync(out->positions, tp, per * sizeof(float), cudaMemcpyDeviceToHost, ctx->stream));
            if (out->normals)
                HP_CUDA(cudaMemcpyAsync(out->normals, tn, per * sizeof(float), cudaMemcpyDeviceToHost, ctx->stream));
            if (out->colors)
                HP_CUDA(cudaMemcpyAsync(out->colors, tc, per * sizeof(float), cudaMemcpyDeviceToHost, ctx->stream));
            HP_CUDA(cudaStreamSynchronize(ctx->stream));
        }
    }
    HP_CUDA(cudaStreamSynchronize(ctx->stream));
    flush_profile(ctx);
    return HP_OK;
}

}  // extern "C"
