// Plans: a batched solve prepared once and replayed (include/hpmvs.h).
//
// A plan owns one device block holding, per view, its packed plane state,
// its per-tile completion flags and (for host-memory outputs) an unpacking
// area, plus the descriptors, the per-pass launch lists and the persistent
// ticket schedule.  Its launch sequence - either init, cost, one launch per
// red-black half-pass and one unpack per view, or a single persistent launch
// that runs all of them tile by tile - is captured once as a CUDA graph and
// replayed by every run.  The autotuner times each schedule candidate on the
// plan's own jobs and keeps the fastest; all candidates give bit-identical
// results.
#include <cuda_runtime.h>

#include <algorithm>
#include <cstring>
#include <memory>
#include <vector>

#include "hp_host.h"

using namespace hpx;

namespace hpx {

// Ticket order of the persistent schedule (see hp::Schedule): entries sorted
// by the stage's offset from its view's first stage in this launch, then by
// view.  A stage's dependencies (the same view's previous stage) therefore
// sit in an earlier entry, or in an earlier launch when the stage is the
// view's first here.
int build_schedule(int n, const int* tiles, const int* kb, const int* ke, std::vector<int>* ticket,
                   std::vector<int2>* info) {
    ticket->clear();
    info->clear();
    int span = 0;
    for (int v = 0; v < n; ++v) span = std::max(span, ke[v] - kb[v]);
    long long acc = 0;
    for (int j = 0; j < span; ++j)
        for (int v = 0; v < n; ++v) {
            if (kb[v] + j >= ke[v] || tiles[v] <= 0) continue;
            ticket->push_back(static_cast<int>(acc));
            info->push_back(make_int2(v, kb[v] + j));
            acc += tiles[v];
            if (acc > 0x7fffffffLL) return -1;
        }
    ticket->push_back(static_cast<int>(acc));
    return static_cast<int>(acc);
}

}  // namespace hpx

struct hp_plan {
    hp_ctx* ctx = nullptr;
    hp_params params{};
    hp_plan_options opt{};
    std::vector<hp::ViewDesc> host;  // descriptors as uploaded
    std::vector<hp_maps> out;
    std::vector<int> iters;
    int max_iter = 0;
    void* block = nullptr;
    size_t block_bytes = 0;
    hp::ViewDesc* d_views = nullptr;
    int* d_done = nullptr;
    size_t done_bytes = 0;
    int* d_lists = nullptr;
    std::vector<int> list_off, list_count, list_tiles;
    int* d_entry_ticket = nullptr;
    int2* d_entry_info = nullptr;
    int n_entries = 0, total = 0;
    unsigned* d_counter = nullptr;  // [0] counter, then status[3] at +4 bytes, main_done at +16
    int* d_status = nullptr;
    // Geometric-consistency stages: the filtered views in the order they run,
    // their per-view finished-tile counts, and the tickets of the solve proper.
    std::vector<int> filter_order;
    std::vector<char> filtered;
    int* d_filter_done = nullptr;
    int main_total = 0;
    // The jobs (and their seed lists), kept so the device side can be rebuilt
    // for another tile height; the tile height and staging depth in use.
    std::vector<hp_job> jobs;
    std::vector<std::vector<hp_seed>> seeds;
    int tile_h = hp::TILE_H;
    int depth = 4;  // FP16 staging depth
    int* h_status = nullptr;        // pinned copy of the status words
    std::vector<float*> staging;    // per view: host-output unpacking area, or nullptr
    cudaGraphExec_t exec = nullptr;
    int exec_schedule = -1, exec_cpsm = -1, exec_tile_h = -1, exec_staging = -1;
    int sms = 0, occ = 0;
    float tuned_ms = 0.f;
    double pix_iter = 0.0;
    cudaEvent_t ev0 = nullptr, ev1 = nullptr;
};

namespace {

size_t align256(size_t x) { return (x + 255) & ~size_t(255); }

int effective_schedule(const hp_plan* p) {
    return p->opt.schedule == HP_SCHEDULE_PER_PASS ? HP_SCHEDULE_PER_PASS : HP_SCHEDULE_PERSISTENT;
}

int effective_cpsm(const hp_plan* p) {
    int c = p->opt.ctas_per_sm;
    if (c <= 0 || c > p->occ) c = p->occ;
    return std::max(1, c);
}

int persistent_grid(const hp_plan* p) {
    return std::max(1, std::min(p->total, p->sms * effective_cpsm(p)));
}

hp::SolveConsts plan_consts(const hp_plan* p) {
    hp::SolveConsts sc = consts_of(&p->params);
    sc.tile_h = p->tile_h;
    sc.staging = p->depth;
    return sc;
}

hp::Schedule schedule_of(const hp_plan* p) {
    hp::Schedule s{};
    s.views = p->d_views;
    s.entry_ticket = p->d_entry_ticket;
    s.entry_info = p->d_entry_info;
    s.n_entries = p->n_entries;
    s.total = p->total;
    s.counter = p->d_counter;
    s.status = p->d_status;
    const int ms = p->opt.wait_limit_ms > 0 ? p->opt.wait_limit_ms : 2000;
    s.wait_limit_ns = static_cast<unsigned long long>(ms) * 1000000ull;
    s.stall_view = p->opt.debug_stall_view;
    s.stall_tile = p->opt.debug_stall_view >= 0 ? p->opt.debug_stall_tile : -1;
    s.sc = plan_consts(p);
    s.main_done = p->filter_order.empty() ? nullptr : p->d_counter + 4;
    s.main_total = p->filter_order.empty() ? p->total : p->main_total;
    return s;
}

hp::BatchList list_of(const hp_plan* p, int l) {
    hp::BatchList bl;
    bl.views = p->d_views;
    bl.n_active = p->list_count[l];
    bl.active = p->d_lists + p->list_off[l];
    bl.tile_prefix = bl.active + bl.n_active;
    bl.total_tiles = p->list_tiles[l];
    return bl;
}

// The device work of one run, on the context stream (captured or direct).
cudaError_t enqueue(hp_plan* p) {
    cudaStream_t st = p->ctx->stream;
    const bool f16 = p->params.precision == HP_PRECISION_F16ACC;
    cudaError_t e;
    if (effective_schedule(p) == HP_SCHEDULE_PERSISTENT) {
        if ((e = cudaMemsetAsync(p->d_done, 0xff, p->done_bytes, st)) != cudaSuccess) return e;
        if ((e = cudaMemsetAsync(p->d_counter, 0, 32, st)) != cudaSuccess) return e;
        if (!p->filter_order.empty() &&
            (e = cudaMemsetAsync(p->d_filter_done, 0, p->filter_order.size() * sizeof(int), st)) != cudaSuccess)
            return e;
        const hp::Schedule s = schedule_of(p);
        const int grid = persistent_grid(p);
        e = f16 ? hp::launch_persistent_f16(s, grid, st) : hp::launch_persistent_f32(s, grid, st);
        if (e != cudaSuccess) return e;
        return cudaMemcpyAsync(p->h_status, p->d_status, 3 * sizeof(int), cudaMemcpyDeviceToHost, st);
    }
    const hp::SolveConsts sc = plan_consts(p);
    const hp::BatchList all = list_of(p, 0);
    if ((e = hp::launch_init(all, p->tile_h, st)) != cudaSuccess) return e;
    if ((e = f16 ? hp::launch_cost_f16(all, sc, st) : hp::launch_cost_f32(all, sc, st)) != cudaSuccess) return e;
    for (int it = 0; it < p->max_iter; ++it) {
        const hp::BatchList bl = list_of(p, 1 + it);
        for (int color = 0; color < 2; ++color) {
            e = f16 ? hp::launch_propagate_f16(bl, sc, it, color, st) : hp::launch_propagate_f32(bl, sc, it, color, st);
            if (e != cudaSuccess) return e;
        }
    }
    // Filtered views: the geometric check, view by view, writes their maps too.
    for (int k : p->filter_order) {
        const hp::ViewDesc& v = p->host[k];
        if ((e = hp::launch_filter_view(p->d_views, k, v.tiles_x * v.tiles_y, p->tile_h, true, st)) != cudaSuccess)
            return e;
    }
    for (size_t k = 0; k < p->host.size(); ++k) {
        if (p->filtered[k]) continue;
        const hp::ViewDesc& v = p->host[k];
        if ((e = hp::launch_unpack(p->host.data(), static_cast<int>(k), v.out_depth, v.out_normal, v.out_cost,
                                   v.out_conf, st)) != cudaSuccess)
            return e;
    }
    return cudaSuccess;
}

int launches_per_run(const hp_plan* p) {
    if (effective_schedule(p) == HP_SCHEDULE_PERSISTENT) return 1;
    return 2 + 2 * p->max_iter + static_cast<int>(p->host.size());  // one filter or unpack per view
}

void count_launches(hp_plan* p) {
    hp_profile& pr = p->ctx->prof;
    if (effective_schedule(p) == HP_SCHEDULE_PERSISTENT) {
        pr.launches[HP_KERNEL_PERSISTENT] += 1;
    } else {
        pr.launches[HP_KERNEL_INIT] += 1;
        pr.launches[HP_KERNEL_COST] += 1;
        pr.launches[HP_KERNEL_PROPAGATE] += 2 * p->max_iter;
        pr.launches[HP_KERNEL_OTHER] += p->host.size();
    }
}

void drop_graph(hp_plan* p) {
    if (p->exec) cudaGraphExecDestroy(p->exec);
    p->exec = nullptr;
    p->exec_schedule = p->exec_cpsm = p->exec_tile_h = p->exec_staging = -1;
}

hp_status ensure_graph(hp_plan* p) {
    hp_ctx* ctx = p->ctx;
    const int sched = effective_schedule(p), cpsm = effective_cpsm(p);
    if (p->exec && p->exec_schedule == sched && p->exec_cpsm == cpsm && p->exec_tile_h == p->tile_h &&
        p->exec_staging == p->depth)
        return HP_OK;
    drop_graph(p);
    HP_CUDA(cudaStreamBeginCapture(ctx->stream, cudaStreamCaptureModeThreadLocal));
    cudaError_t e = enqueue(p);
    cudaGraph_t g = nullptr;
    cudaError_t e2 = cudaStreamEndCapture(ctx->stream, &g);
    if (e == cudaSuccess) e = e2;
    if (e == cudaSuccess) e = cudaGraphInstantiate(&p->exec, g, 0);
    if (g) cudaGraphDestroy(g);
    HP_CUDA(e);
    p->exec_schedule = sched;
    p->exec_cpsm = cpsm;
    p->exec_tile_h = p->tile_h;
    p->exec_staging = p->depth;
    return HP_OK;
}

// Enqueue one run (graph replay or direct launches), bracketed by the plan's events.
hp_status launch_run(hp_plan* p) {
    hp_ctx* ctx = p->ctx;
    if (p->opt.use_graph) {
        hp_status st = ensure_graph(p);
        if (st != HP_OK) return st;
    }
    HP_CUDA(cudaEventRecord(p->ev0, ctx->stream));
    if (p->opt.use_graph)
        HP_CUDA(cudaGraphLaunch(p->exec, ctx->stream));
    else
        HP_CUDA(enqueue(p));
    HP_CUDA(cudaEventRecord(p->ev1, ctx->stream));
    count_launches(p);
    return HP_OK;
}

// Wait for the run, copy host outputs, report the persistent status.
hp_status finish_run(hp_plan* p, float* ms) {
    hp_ctx* ctx = p->ctx;
    HP_CUDA(cudaEventSynchronize(p->ev1));
    float t = 0.f;
    HP_CUDA(cudaEventElapsedTime(&t, p->ev0, p->ev1));
    if (ms) *ms = t;
    if (ctx->profiling) {
        const int kind = effective_schedule(p) == HP_SCHEDULE_PERSISTENT ? HP_KERNEL_PERSISTENT : HP_KERNEL_PROPAGATE;
        ctx->prof.device_ms[kind] += t;
        ctx->prof.timed[kind] += 1;
    }
    if (effective_schedule(p) == HP_SCHEDULE_PERSISTENT && p->h_status[0] != hp::SCHED_OK)
        return fail(ctx, HP_ERR_TIMEOUT,
                    "plan: a persistent dependency wait ran out (status %d, ticket %d of %d); no result",
                    p->h_status[0], p->h_status[2], p->total);
    for (size_t k = 0; k < p->host.size(); ++k) {
        if (!p->staging[k]) continue;
        const hp::ViewDesc& v = p->host[k];
        const size_t px = static_cast<size_t>(v.W) * v.H;
        HP_CUDA(cudaMemcpyAsync(p->out[k].depth, v.out_depth, px * sizeof(float), cudaMemcpyDeviceToHost, ctx->stream));
        HP_CUDA(cudaMemcpyAsync(p->out[k].normal, v.out_normal, 3 * px * sizeof(float), cudaMemcpyDeviceToHost,
                                ctx->stream));
        HP_CUDA(cudaMemcpyAsync(p->out[k].cost, v.out_cost, px * sizeof(float), cudaMemcpyDeviceToHost, ctx->stream));
        if (p->out[k].confidence)
            HP_CUDA(cudaMemcpyAsync(p->out[k].confidence, v.out_conf, px * sizeof(float), cudaMemcpyDeviceToHost,
                                    ctx->stream));
    }
    HP_CUDA(cudaStreamSynchronize(ctx->stream));
    return HP_OK;
}

void free_plan(hp_plan* p) {
    drop_graph(p);
    if (p->ev0) cudaEventDestroy(p->ev0);
    if (p->ev1) cudaEventDestroy(p->ev1);
    if (p->h_status) cudaFreeHost(p->h_status);
    if (p->block) cudaFree(p->block);
    p->ev0 = p->ev1 = nullptr;
    p->h_status = nullptr;
    p->block = nullptr;
}

// Persistent-kernel occupancy of the plan's current kernel variant.
hp_status plan_occupancy(hp_plan* p) {
    hp_ctx* ctx = p->ctx;
    const hp::SolveConsts sc = plan_consts(p);
    HP_CUDA(p->params.precision == HP_PRECISION_F16ACC
                ? hp::persistent_occupancy_f16(sc, &p->occ)
                : hp::persistent_occupancy_f32(p->params.radius, p->params.stride, &p->occ));
    if (p->occ < 1) return fail(ctx, HP_ERR_UNSUPPORTED, "plan: persistent kernel does not fit on an SM");
    return HP_OK;
}

hp_status build_device(hp_plan* p, int tile_h);

// (Re)builds the plan's device side - descriptors, launch lists, ticket
// schedule, filter stages and the one device block - for tiles of tile_h rows.
hp_status build_device(hp_plan* p, int tile_h) {
    hp_ctx* ctx = p->ctx;
    const hp_job* jobs = p->jobs.data();
    const int num_jobs = static_cast<int>(p->jobs.size());
    const hp_params* params = &p->params;
    const hp_maps* out = p->out.data();
    hp_status st;
    free_plan(p);
    p->tile_h = tile_h;
    p->host.assign(num_jobs, hp::ViewDesc{});
    p->iters.clear();
    p->max_iter = 0;
    p->pix_iter = 0.0;
    p->list_off.clear();
    p->list_count.clear();
    p->list_tiles.clear();
    for (int k = 0; k < num_jobs; ++k) {
        if ((st = fill_desc(ctx, &jobs[k], k, &p->host[k], tile_h)) != HP_OK) return st;
        p->iters.push_back(jobs[k].iterations);
        p->max_iter = std::max(p->max_iter, jobs[k].iterations);
        p->pix_iter += static_cast<double>(p->host[k].W) * p->host[k].H * jobs[k].iterations;
    }
    // Per-pass launch lists (as hp_solve) and the persistent ticket schedule.
    std::vector<int> ints;
    for (int l = 0; l <= p->max_iter; ++l) {
        std::vector<int> act;
        for (int k = 0; k < num_jobs; ++k)
            if (l == 0 || jobs[k].iterations > l - 1) act.push_back(k);
        p->list_off.push_back(static_cast<int>(ints.size()));
        p->list_count.push_back(static_cast<int>(act.size()));
        for (int k : act) ints.push_back(k);
        int acc = 0;
        for (int k : act) {
            ints.push_back(acc);
            acc += p->host[k].tiles_x * p->host[k].tiles_y;
        }
        ints.push_back(acc);
        p->list_tiles.push_back(acc);
    }
    // Geometric-consistency stages (hp_params.filter_*).
    std::vector<hp::FilterStage> fstages;
    filter_stages(jobs, num_jobs, params, p->host, &fstages, &p->filtered, &p->filter_order);
    std::vector<int> tiles(num_jobs), kb(num_jobs, 0), ke(num_jobs);
    for (int k = 0; k < num_jobs; ++k) {
        tiles[k] = p->host[k].tiles_x * p->host[k].tiles_y;
        // init+cost, half-passes, then the unpack - or, for a filtered view,
        // the filter stage (which writes the maps) after every view's solve.
        ke[k] = 2 * jobs[k].iterations + (p->filtered[k] ? 1 : 2);
    }
    std::vector<int> eticket;
    std::vector<int2> einfo;
    p->total = build_schedule(num_jobs, tiles.data(), kb.data(), ke.data(), &eticket, &einfo);
    if (p->total < 0) return fail(ctx, HP_ERR_UNSUPPORTED, "plan_create: more than 2^31 tile tickets");
    p->main_total = p->total;
    if (!p->filter_order.empty()) {  // filter entries last, in view order
        eticket.pop_back();
        long long acc = p->total;
        for (int k : p->filter_order) {
            eticket.push_back(static_cast<int>(acc));
            einfo.push_back(make_int2(k, 2 * jobs[k].iterations + 1));
            acc += tiles[k];
            if (acc > 0x7fffffffLL) return fail(ctx, HP_ERR_UNSUPPORTED, "plan_create: more than 2^31 tile tickets");
        }
        eticket.push_back(static_cast<int>(acc));
        p->total = static_cast<int>(acc);
    }
    p->n_entries = static_cast<int>(einfo.size());
    // One device block: per view state, flags and staging; then descriptors, lists, schedule, counters.
    std::vector<size_t> off_state(num_jobs), off_done(num_jobs), off_stage(num_jobs);
    size_t bytes = 0;
    for (int k = 0; k < num_jobs; ++k) {
        const size_t px = static_cast<size_t>(p->host[k].W) * p->host[k].H;
        off_state[k] = bytes;
        bytes = align256(bytes + px * (sizeof(float4) + sizeof(float)));
    }
    const size_t off_flags = bytes;
    for (int k = 0; k < num_jobs; ++k) {
        off_done[k] = bytes;
        bytes += static_cast<size_t>(tiles[k]) * sizeof(int);
    }
    p->done_bytes = bytes - off_flags;
    bytes = align256(bytes);
    for (int k = 0; k < num_jobs; ++k) {
        off_stage[k] = bytes;
        if (out[k].memory == HP_MEMORY_HOST)
            bytes = align256(bytes + static_cast<size_t>(p->host[k].W) * p->host[k].H * 6 * sizeof(float));
    }
    const size_t off_filters = bytes;
    bytes = align256(bytes + num_jobs * sizeof(hp::FilterStage));
    const size_t off_fdone = bytes;
    bytes = align256(bytes + std::max<size_t>(1, p->filter_order.size()) * sizeof(int));
    std::vector<size_t> off_seed(num_jobs);  // SfM seed lists and index maps, built once here
    for (int k = 0; k < num_jobs; ++k) {
        off_seed[k] = bytes;
        bytes = align256(bytes + seed_area_bytes(&jobs[k], p->host[k].W, p->host[k].H));
    }
    const size_t off_desc = bytes;
    bytes = align256(bytes + num_jobs * sizeof(hp::ViewDesc));
    const size_t off_lists = bytes;
    bytes = align256(bytes + ints.size() * sizeof(int));
    const size_t off_et = bytes;
    bytes = align256(bytes + eticket.size() * sizeof(int));
    const size_t off_ei = bytes;
    bytes = align256(bytes + einfo.size() * sizeof(int2));
    const size_t off_ctr = bytes;
    bytes += 256;
    HP_CUDA(cudaMalloc(&p->block, bytes));
    p->block_bytes = bytes;
    char* base = static_cast<char*>(p->block);
    p->staging.assign(num_jobs, nullptr);
    for (int k = 0; k < num_jobs; ++k) {
        hp::ViewDesc& v = p->host[k];
        const size_t px = static_cast<size_t>(v.W) * v.H;
        v.hyp = reinterpret_cast<float4*>(base + off_state[k]);
        v.cost = reinterpret_cast<float*>(base + off_state[k] + px * sizeof(float4));
        v.done = reinterpret_cast<int*>(base + off_done[k]);
        if (out[k].memory == HP_MEMORY_DEVICE) {
            v.out_depth = out[k].depth;
            v.out_normal = out[k].normal;
            v.out_cost = out[k].cost;
            v.out_conf = out[k].confidence;
        } else {
            float* sd = reinterpret_cast<float*>(base + off_stage[k]);
            p->staging[k] = sd;
            v.out_depth = sd;
            v.out_normal = sd + px;
            v.out_cost = sd + 4 * px;
            v.out_conf = out[k].confidence ? sd + 5 * px : nullptr;
        }
    }
    p->d_filter_done = reinterpret_cast<int*>(base + off_fdone);
    hp::FilterStage* d_filters = reinterpret_cast<hp::FilterStage*>(base + off_filters);
    for (size_t i = 0; i < p->filter_order.size(); ++i) {
        const int k = p->filter_order[i];
        fstages[k].tiles_done = p->d_filter_done + i;
        p->host[k].filter = d_filters + k;
    }
    HP_CUDA(cudaMemcpy(d_filters, fstages.data(), num_jobs * sizeof(hp::FilterStage), cudaMemcpyHostToDevice));
    for (int k = 0; k < num_jobs; ++k)
        HP_CUDA(stage_seeds(&jobs[k], base + off_seed[k], &p->host[k], ctx->stream));
    HP_CUDA(cudaStreamSynchronize(ctx->stream));
    p->d_done = reinterpret_cast<int*>(base + off_flags);
    p->d_views = reinterpret_cast<hp::ViewDesc*>(base + off_desc);
    p->d_lists = reinterpret_cast<int*>(base + off_lists);
    p->d_entry_ticket = reinterpret_cast<int*>(base + off_et);
    p->d_entry_info = reinterpret_cast<int2*>(base + off_ei);
    p->d_counter = reinterpret_cast<unsigned*>(base + off_ctr);
    p->d_status = reinterpret_cast<int*>(base + off_ctr + 4);
    HP_CUDA(cudaMemcpy(p->d_views, p->host.data(), num_jobs * sizeof(hp::ViewDesc), cudaMemcpyHostToDevice));
    HP_CUDA(cudaMemcpy(p->d_lists, ints.data(), ints.size() * sizeof(int), cudaMemcpyHostToDevice));
    HP_CUDA(cudaMemcpy(p->d_entry_ticket, eticket.data(), eticket.size() * sizeof(int), cudaMemcpyHostToDevice));
    HP_CUDA(cudaMemcpy(p->d_entry_info, einfo.data(), einfo.size() * sizeof(int2), cudaMemcpyHostToDevice));
    HP_CUDA(cudaMallocHost(&p->h_status, 3 * sizeof(int)));
    p->h_status[0] = p->h_status[1] = p->h_status[2] = 0;
    HP_CUDA(cudaEventCreate(&p->ev0));
    HP_CUDA(cudaEventCreate(&p->ev1));
    return plan_occupancy(p);
}

}  // namespace

extern "C" {

void hp_plan_options_default(hp_plan_options* o) {
    if (!o) return;
    o->schedule = HP_SCHEDULE_AUTO;
    o->ctas_per_sm = 0;
    o->use_graph = 1;
    o->wait_limit_ms = 2000;
    o->debug_stall_view = -1;
    o->debug_stall_tile = -1;
}

hp_status hp_schedule_build(int num_views, const int* tiles, const int* stage_begin, const int* stage_end,
                            int capacity, int* entry_ticket, int* entry_view, int* entry_stage, int* num_entries) {
    if (num_views < 0 || !tiles || !stage_begin || !stage_end || !entry_ticket || !entry_view || !entry_stage ||
        !num_entries || capacity < 0)
        return HP_ERR_INVALID_ARG;
    for (int v = 0; v < num_views; ++v)
        if (tiles[v] < 0 || stage_begin[v] < 0 || stage_end[v] < stage_begin[v]) return HP_ERR_INVALID_ARG;
    std::vector<int> t;
    std::vector<int2> info;
    if (build_schedule(num_views, tiles, stage_begin, stage_end, &t, &info) < 0) return HP_ERR_UNSUPPORTED;
    *num_entries = static_cast<int>(info.size());
    if (static_cast<int>(info.size()) > capacity) return HP_ERR_INVALID_ARG;
    for (size_t e = 0; e < info.size(); ++e) {
        entry_ticket[e] = t[e];
        entry_view[e] = info[e].x;
        entry_stage[e] = info[e].y;
    }
    entry_ticket[info.size()] = t.back();
    return HP_OK;
}

hp_status hp_plan_create(hp_ctx* ctx, const hp_job* jobs, int num_jobs, const hp_params* params,
                         const hp_plan_options* options, const hp_maps* out, hp_plan** plan) {
    if (!ctx) return HP_ERR_INVALID_ARG;
    if (!plan) return fail(ctx, HP_ERR_INVALID_ARG, "plan_create: null plan pointer");
    *plan = nullptr;
    if (!jobs || !out || num_jobs < 1) return fail(ctx, HP_ERR_INVALID_ARG, "plan_create: no jobs or outputs");
    hp_status st = check_params(ctx, params);
    if (st != HP_OK) return st;
    std::unique_ptr<hp_plan> p(new hp_plan);
    struct Release {  // frees the device side of a plan that fails half-built
        hp_plan* p;
        ~Release() {
            if (p) free_plan(p);
        }
    } release{p.get()};
    p->ctx = ctx;
    p->params = *params;
    if (options)
        p->opt = *options;
    else
        hp_plan_options_default(&p->opt);
    if (p->opt.schedule < HP_SCHEDULE_AUTO || p->opt.schedule > HP_SCHEDULE_PERSISTENT)
        return fail(ctx, HP_ERR_INVALID_ARG, "plan_create: unknown schedule %d", p->opt.schedule);
    for (int k = 0; k < num_jobs; ++k) {
        const hp_maps& m = out[k];
        if (!m.depth || !m.normal || !m.cost)
            return fail(ctx, HP_ERR_INVALID_ARG, "plan_create: output maps of job %d incomplete", k);
        if (m.memory != HP_MEMORY_HOST && m.memory != HP_MEMORY_DEVICE)
            return fail(ctx, HP_ERR_INVALID_ARG, "plan_create: job %d: unknown memory kind %d", k, m.memory);
    }
    DeviceGuard g(ctx->device);
    p->out.assign(out, out + num_jobs);
    p->jobs.assign(jobs, jobs + num_jobs);
    p->seeds.resize(num_jobs);
    for (int k = 0; k < num_jobs; ++k) {
        if ((st = check_seeds(ctx, &jobs[k], k)) != HP_OK) return st;
        if (jobs[k].num_seeds > 0) {
            p->seeds[k].assign(jobs[k].seeds, jobs[k].seeds + jobs[k].num_seeds);
            p->jobs[k].seeds = p->seeds[k].data();
        }
    }
    const hp::SolveConsts sc0 = consts_of(params);
    p->depth = sc0.staging;
    HP_CUDA(cudaDeviceGetAttribute(&p->sms, cudaDevAttrMultiProcessorCount, ctx->device));
    if ((st = build_device(p.get(), sc0.tile_h)) != HP_OK) return st;
    release.p = nullptr;
    *plan = p.release();
    return HP_OK;
}

hp_status hp_plan_launch(hp_plan* p) {
    if (!p) return HP_ERR_INVALID_ARG;
    for (size_t k = 0; k < p->staging.size(); ++k)
        if (p->staging[k])
            return fail(p->ctx, HP_ERR_INVALID_ARG, "plan_launch: job %zu has host outputs; use hp_plan_run", k);
    DeviceGuard g(p->ctx->device);
    return launch_run(p);
}

hp_status hp_plan_wait(hp_plan* p) {
    if (!p) return HP_ERR_INVALID_ARG;
    DeviceGuard g(p->ctx->device);
    return finish_run(p, nullptr);
}

hp_status hp_plan_run(hp_plan* p) {
    if (!p) return HP_ERR_INVALID_ARG;
    DeviceGuard g(p->ctx->device);
    hp_status st = launch_run(p);
    if (st != HP_OK) return st;
    return finish_run(p, nullptr);
}

hp_status hp_plan_get_info(const hp_plan* p, hp_plan_info* info) {
    if (!p || !info) return HP_ERR_INVALID_ARG;
    std::memset(info, 0, sizeof *info);
    info->schedule = effective_schedule(p);
    info->ctas_per_sm = info->schedule == HP_SCHEDULE_PERSISTENT ? effective_cpsm(p) : 0;
    info->grid = info->schedule == HP_SCHEDULE_PERSISTENT ? persistent_grid(p) : 0;
    info->max_ctas_per_sm = p->occ;
    info->tickets = p->total;
    info->launches_per_run = launches_per_run(p);
    info->views = static_cast<int>(p->host.size());
    info->use_graph = p->opt.use_graph;
    info->state_bytes = p->block_bytes;
    info->pixel_iterations = p->pix_iter;
    info->tuned_ms = p->tuned_ms;
    info->tile_h = p->tile_h;
    info->staging = p->depth;
    return HP_OK;
}

hp_status hp_plan_tune(hp_plan* p, int repeats, hp_plan_info* best) {
    if (!p) return HP_ERR_INVALID_ARG;
    if (repeats < 1 || repeats > 100) return fail(p->ctx, HP_ERR_INVALID_ARG, "plan_tune: repeats %d", repeats);
    DeviceGuard g(p->ctx->device);
    const hp_plan_options keep = p->opt;
    // Median time of `repeats` runs of the current configuration.
    auto timed = [&](float* med) -> hp_status {
        std::vector<float> t;
        for (int r = 0; r < repeats; ++r) {
            float ms = 0.f;
            hp_status st = launch_run(p);
            if (st == HP_OK) st = finish_run(p, &ms);
            if (st != HP_OK) return st;
            t.push_back(ms);
        }
        std::sort(t.begin(), t.end());
        *med = t[t.size() / 2];
        return HP_OK;
    };
    hp_status st;
    // A failure while the device side is rebuilt for another tile height
    // (device memory, say) restores the plan's configuration before returning.
    const int keep_th = p->tile_h, keep_depth = p->depth;
    auto restore = [&](hp_status err) {
        p->opt = keep;
        p->depth = keep_depth;
        if (p->tile_h != keep_th || !p->block) {
            if (build_device(p, keep_th) != HP_OK) return err;  // the plan stays unusable: err says why
        }
        plan_occupancy(p);
        return err;
    };
    // Stage 1 (FP16-acc path, where the caller left them to the engine): tile
    // height x staging depth, each timed with the per-pass graph.
    const bool f16 = p->params.precision == HP_PRECISION_F16ACC;
    std::vector<int> th_opts = {p->tile_h}, d_opts = {p->depth};
    if (f16 && p->params.tile_h == 0) th_opts = {8, 4};
    if (f16 && p->params.staging == 0) d_opts = {4, 8};
    if (th_opts.size() * d_opts.size() > 1) {
        float best_ms = -1.f;
        int best_th = p->tile_h, best_d = p->depth;
        for (int th : th_opts) {
            if (th != p->tile_h && (st = build_device(p, th)) != HP_OK) return restore(st);
            for (int d : d_opts) {
                p->depth = d;
                p->opt.schedule = HP_SCHEDULE_PER_PASS;
                float ms = 0.f;
                if ((st = timed(&ms)) != HP_OK) return restore(st);
                if (best_ms < 0.f || ms < best_ms) {
                    best_ms = ms;
                    best_th = th;
                    best_d = d;
                }
            }
        }
        if (best_th != p->tile_h && (st = build_device(p, best_th)) != HP_OK) return restore(st);
        p->depth = best_d;
        if ((st = plan_occupancy(p)) != HP_OK) return restore(st);
    }
    // Stage 2: the schedule - the per-pass graph, or the persistent kernel at
    // each resident-CTA count up to its occupancy maximum.
    std::vector<std::pair<int, int>> cands = {{HP_SCHEDULE_PER_PASS, 0}};
    for (int c = 1; c <= p->occ; ++c) cands.emplace_back(HP_SCHEDULE_PERSISTENT, c);
    float best_ms = -1.f;
    std::pair<int, int> best_c = cands[0];
    for (const auto& c : cands) {
        p->opt.schedule = c.first;
        p->opt.ctas_per_sm = c.second;
        float ms = 0.f;
        if ((st = timed(&ms)) != HP_OK) {
            p->opt = keep;
            return st;
        }
        if (best_ms < 0.f || ms < best_ms) {
            best_ms = ms;
            best_c = c;
        }
    }
    p->opt.schedule = best_c.first;
    p->opt.ctas_per_sm = best_c.second;
    p->tuned_ms = best_ms;
    // Leave the maps holding a solve of the chosen candidate.
    st = hp_plan_run(p);
    if (st != HP_OK) return st;
    if (best) hp_plan_get_info(p, best);
    return HP_OK;
}

hp_status hp_plan_destroy(hp_plan* p) {
    if (!p) return HP_ERR_INVALID_ARG;
    {
        DeviceGuard g(p->ctx->device);
        cudaStreamSynchronize(p->ctx->stream);
        free_plan(p);
    }
    delete p;
    return HP_OK;
}

}  // extern "C"
