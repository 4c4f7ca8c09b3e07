// Tile-level stages shared by the FP32 and FP16 kernels (hypothesis
// initialisation, output unpacking) and the device side of the persistent
// schedule (ticket decoding, bounded dependency waits, completion flags).
#pragma once

#include "hp_check.cuh"
#include "hp_internal.h"
#include "hp_rng.cuh"

namespace hp {

// Initial hypotheses of one tile: depth uniform in [dmin, dmax]; normal from
// theta in [0, 2pi) and cos(phi) in (0, 1), flipped to face the camera,
// normalised (init_depth_normal_kernel, src/dense_recon/patchmatch_mvs.cu:164-216).
// Pixels the view's SfM seed map covers take their seed's plane instead.
// Every operation is explicitly rounded, so the result does not depend on the
// including translation unit's flags (no intermediate is ever subnormal:
// depths lie in [dmin, dmax] and normal components are at least ~1e-10).
__device__ __forceinline__ void tile_init(const ViewDesc* v, int tile_x, int tile_y) {
    const int ly = threadIdx.x >> 5, lane = threadIdx.x & 31;
    const int y = tile_y * v->tile_h + ly;
    if (y >= v->H) return;
    for (int j = 0; j < 2; ++j) {
        const int x = tile_x * TILE_W + j * 32 + lane;
        if (x >= v->W) continue;
        const uint32_t idx = static_cast<uint32_t>(y * v->W + x);
        if (v->seed_map) {  // SfM seed (runPatchMatchMVS, patchmatch_mvs.cu:1111-1177)
            const int k = v->seed_map[idx];
            if (k >= 0) {
                const hp_seed sd = v->seeds[k];
                v->hyp[idx] = make_float4(sd.depth, sd.normal[0], sd.normal[1], sd.normal[2]);
                continue;
            }
        }
        const uint4 r = philox4x32_10(make_uint4(idx, v->view_id, 0u, 0u), v->seed_lo, v->seed_hi);
        const float depth = __fmaf_rn(u01(r.x), __fsub_rn(v->dmax, v->dmin), v->dmin);
        const float3 ray = view_ray(v->kinv, x, y);
        float st, ct;
        sincos_2pi(u01(r.y), &st, &ct);
        const float cp = u01(r.z);
        const float sp = __fsqrt_rn(fmaxf(0.0f, __fmaf_rn(-cp, cp, 1.0f)));
        float3 n = make_float3(__fmul_rn(sp, ct), __fmul_rn(sp, st), cp);
        if (dot3_rn(n, ray) > 0.0f) n = make_float3(-n.x, -n.y, -n.z);
        n = normalize3_rn(n.x, n.y, n.z);
        v->hyp[idx] = make_float4(depth, n.x, n.y, n.z);
    }
}

// Final stage of a view in a persistent launch: its tile's packed state into
// the output maps (depth, camera-frame AoS normal, cost, and confidence
// 1 - cost / 2 when wanted).
__device__ __forceinline__ void tile_unpack(const ViewDesc* v, int tile_x, int tile_y) {
    const int ly = threadIdx.x >> 5, lane = threadIdx.x & 31;
    const int y = tile_y * v->tile_h + ly;
    if (y >= v->H) return;
    if (!HP_CHECK(v->out_depth && v->out_normal && v->out_cost, HP_CHECK_OUTPUT, v->W, v->H, tile_x, tile_y, 0, 0,
                  0.f, 0.f, 0.f, 0.f))
        return;
    for (int j = 0; j < 2; ++j) {
        const int x = tile_x * TILE_W + j * 32 + lane;
        if (x >= v->W) continue;
        const size_t i = static_cast<size_t>(y) * v->W + x;
        const float4 h = __ldcg(v->hyp + i);
        v->out_depth[i] = h.x;
        v->out_normal[3 * i] = h.y;
        v->out_normal[3 * i + 1] = h.z;
        v->out_normal[3 * i + 2] = h.w;
        const float c = __ldcg(v->cost + i);
        v->out_cost[i] = c;
        if (v->out_conf) v->out_conf[i] = __fsub_rn(1.0f, __fmul_rn(c, 0.5f));
    }
}

__device__ __forceinline__ int ld_acquire_gpu(const int* p) {
    int v;
    asm volatile("ld.acquire.gpu.global.s32 %0, [%1];" : "=r"(v) : "l"(p) : "memory");
    return v;
}

__device__ __forceinline__ void st_release_gpu(int* p, int v) {
    asm volatile("st.release.gpu.global.s32 [%0], %1;" ::"l"(p), "r"(v) : "memory");
}

__device__ __forceinline__ int ld_relaxed_gpu(const int* p) {
    int v;
    asm volatile("ld.relaxed.gpu.global.s32 %0, [%1];" : "=r"(v) : "l"(p) : "memory");
    return v;
}

__device__ __forceinline__ unsigned long long global_ns() {
    unsigned long long t;
    asm volatile("mov.u64 %0, %%globaltimer;" : "=l"(t));
    return t;
}

struct SchedTile {
    const ViewDesc* v;
    int view, stage;
    int tile, tx, ty;
    int ticket;
};

// Whether stage `stage` of view v is its geometric-consistency stage (which
// follows its last half-pass when the view has one).
__device__ __forceinline__ bool is_filter_stage(const ViewDesc* v, int stage) {
    return v->filter != nullptr && stage == 2 * v->iterations + 1;
}

__device__ __forceinline__ unsigned ld_acquire_gpu_u32(const unsigned* p) {
    unsigned v;
    asm volatile("ld.acquire.gpu.global.u32 %0, [%1];" : "=r"(v) : "l"(p) : "memory");
    return v;
}

__device__ __forceinline__ SchedTile decode_ticket(const Schedule& s, int t) {
    int lo = 0, hi = s.n_entries - 1;
    while (lo < hi) {  // last entry starting at or before t
        const int mid = (lo + hi + 1) >> 1;
        if (s.entry_ticket[mid] <= t) lo = mid; else hi = mid - 1;
    }
    const int2 info = s.entry_info[lo];
    SchedTile r;
    r.v = &s.views[info.x];
    r.view = info.x;
    r.stage = info.y;
    r.tile = t - s.entry_ticket[lo];
    r.tx = r.tile % r.v->tiles_x;
    r.ty = r.tile / r.v->tiles_x;
    r.ticket = t;
    return r;
}

// A wait of `ticket` ran out: record SCHED_TIMEOUT and the ticket (the first
// recorded wins) and raise the abort flag.
__device__ __forceinline__ void sched_abort(const Schedule& s, int ticket) {
    if (atomicCAS(s.status, SCHED_OK, SCHED_TIMEOUT) == SCHED_OK) atomicExch(s.status + 2, ticket);
    atomicExch(s.abort, 1);
}

// The abort flag is up.  When another launch raised it (a shared flag), this
// launch records SCHED_ABORTED: it stops with work left undone.
__device__ __forceinline__ bool sched_aborted(const Schedule& s) {
    if (!ld_relaxed_gpu(s.abort)) return false;
    atomicCAS(s.status, SCHED_OK, SCHED_ABORTED);
    return true;
}

// Bounded poll of thread 0 for `ticket`: spins while ready() is false.
// Bounded by the schedule's time limit and by a poll count (in case the
// global timer stands still); false when this or another CTA gave up.  The
// time limit counts only after kMinPolls sleeping polls, so a step of the
// global timer during a short wait cannot end it.
struct WaitBudget {
    unsigned long long start = 0;
    unsigned polls = 0;
};

template <class Ready>
__device__ __forceinline__ bool sched_poll(const Schedule& s, int ticket, WaitBudget& b, Ready ready) {
    constexpr unsigned kMinPolls = 4096, kMaxPolls = 1u << 26;
    while (!ready()) {
        if (sched_aborted(s)) return false;
        if (++b.polls > 16) {
            const unsigned long long now = global_ns();
            if (b.start == 0) b.start = now;
            if ((now - b.start > s.wait_limit_ns && b.polls > kMinPolls) || b.polls > kMaxPolls) {
                sched_abort(s, ticket);
                return false;
            }
            __nanosleep(256);
        }
    }
    return true;
}

// Thread 0 of a CTA: wait until the tile and its 4-neighbour tiles have
// finished stage - 1.  A filter stage also waits until every ticket of the
// solve proper has finished and the previous filtered view's stage has
// finished on all its tiles (both counts only grow, and every ticket they
// count precedes this one, so each is held by a running CTA).
__device__ __forceinline__ bool sched_wait(const Schedule& s, const SchedTile& t) {
    if (t.stage == 0) return true;
    const int need = t.stage - 1;
    const int* done = t.v->done;
    const int tx = t.v->tiles_x;
    int deps[5];
    int n = 0;
    deps[n++] = t.tile;
    if (t.tx > 0) deps[n++] = t.tile - 1;
    if (t.tx + 1 < tx) deps[n++] = t.tile + 1;
    if (t.ty > 0) deps[n++] = t.tile - tx;
    if (t.ty + 1 < t.v->tiles_y) deps[n++] = t.tile + tx;
    WaitBudget b;
    for (int i = 0; i < n; ++i) {
        const int* flag = done + deps[i];
        if (!sched_poll(s, t.ticket, b, [&] { return ld_acquire_gpu(flag) >= need; })) return false;
    }
    if (s.main_done && is_filter_stage(t.v, t.stage)) {
        const unsigned main_total = static_cast<unsigned>(s.main_total);
        if (!sched_poll(s, t.ticket, b, [&] { return ld_acquire_gpu_u32(s.main_done) >= main_total; }))
            return false;
        const int prev = t.v->filter->prev;
        if (prev >= 0) {
            const ViewDesc* pv = &s.views[prev];
            const int* cnt = pv->filter->tiles_done;
            const int want = pv->tiles_x * pv->tiles_y;
            if (!sched_poll(s, t.ticket, b, [&] { return ld_acquire_gpu(cnt) >= want; })) return false;
        }
    }
    return true;
}

// Thread 0, after the CTA's barrier at the end of a stage: publish it.
__device__ __forceinline__ void sched_publish(const Schedule& s, const SchedTile& t) {
    if (t.view == s.stall_view && t.tile == s.stall_tile) return;
    __threadfence();
    st_release_gpu(t.v->done + t.tile, t.stage);
    if (s.main_done) {
        if (t.ticket < s.main_total)
            atomicAdd(s.main_done, 1u);
        else if (is_filter_stage(t.v, t.stage))
            atomicAdd(t.v->filter->tiles_done, 1);
    }
}

// Thread 0: claims the CTA's next ticket and decodes it into *out; false when
// the schedule is exhausted or aborted (including a dependency wait of this
// ticket that ran out).
__device__ __forceinline__ bool sched_claim(const Schedule& s, SchedTile* out) {
    if (sched_aborted(s)) return false;
    const int t = static_cast<int>(atomicAdd(s.counter, 1u));
    if (t >= s.total) return false;
    const SchedTile d = decode_ticket(s, t);
    if (!sched_wait(s, d)) return false;
    *out = d;
    return true;
}

}  // namespace hp
