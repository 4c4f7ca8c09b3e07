// Server: continuous batching of depth-map solves (include/hpmvs.h).
//
// Policy (ServerCore, host only, also run by hp_server_simulate): requests
// wait in arrival order; before each step the head of the queue is admitted
// while a request slot is free and its state fits the byte budget.  The
// queue is strict FIFO - a request that does not fit holds back those behind
// it - so large requests are never starved by a stream of small ones.  A step
// runs, for each admitted request, its next passes_per_step stages (round
// robin), or, with the budget policy, as many as a per-step work budget
// covers for the oldest requests first (at least one each); a request
// whose last stage (the unpack into its maps) is in the step leaves the
// active set as the step is composed, so its slot and bytes serve the next
// step's admissions.  That reuse is safe before the step has executed: every
// allocation, free and launch is ordered on the server's one stream.
//
// Device side (worker thread): per step one pinned upload holding the step's
// view descriptors, its ticket schedule(s) and zeroed counters; one H2D copy;
// the persistent launch (or one launch per stage offset); the host-output
// copies and stream-ordered frees of finishing requests; an event.  Up to
// inflight_steps steps are enqueued ahead of the oldest unfinished one, and
// a request is reported complete once the event of its last step has fired.
//
// Failure containment: a step whose launch fails, or whose persistent kernel
// gives up on a dependency wait, leaves its members' state part-way through
// a stage.  Every admitted request is a member of every step, so the steps
// queued behind it would wait on that state in turn, and so would each
// request admitted later.  The launches of a server therefore share one
// abort flag: the launches behind a failed one stop at their first ticket
// claim.  The worker then retires the steps in flight, completes every
// admitted request with the failure, clears the flag and goes on with the
// queue, which is untouched.
#include <cuda_runtime.h>

#include <algorithm>
#include <chrono>
#include <cmath>
#include <condition_variable>
#include <cstdio>
#include <cstring>
#include <string>
#include <deque>
#include <memory>
#include <mutex>
#include <thread>
#include <vector>

#include "hp_host.h"

using namespace hpx;

namespace hpx {

int build_schedule(int n, const int* tiles, const int* kb, const int* ke, std::vector<int>* ticket,
                   std::vector<int2>* info);

struct CoreReq {
    int tiles = 0;
    int stages = 0;      // 2 * iterations + 2: init + cost, half-passes, unpack
    uint64_t bytes = 0;  // device state the request holds while admitted
    double work = 0.0;   // work of one stage, in pixel x source units (W * H * S)
    int stage = 0;       // next stage to run
    void* user = nullptr;
};

// One composed step: per member request its stage range [kb, ke).
struct StepPlan {
    std::vector<CoreReq*> reqs;
    std::vector<int> kb, ke;
    std::vector<CoreReq*> finishing;
};

struct ServerCore {
    std::deque<CoreReq*> queue;
    std::vector<CoreReq*> active;
    uint64_t held = 0;
    int max_active = 64;
    int passes = 4;            // stages per request per step (HP_SERVER_POLICY_BUDGET: at most)
    int policy = HP_SERVER_POLICY_ROUND_ROBIN;
    double step_work = 0.0;    // HP_SERVER_POLICY_BUDGET: work of a step, pixel x source x stage units

    // Head-of-queue admissions that fit `budget` bytes of request state.
    void admit(uint64_t budget, std::vector<CoreReq*>* admitted) {
        while (!queue.empty() && static_cast<int>(active.size()) < max_active) {
            CoreReq* r = queue.front();
            if (held + r->bytes > budget) break;
            queue.pop_front();
            active.push_back(r);
            held += r->bytes;
            admitted->push_back(r);
        }
    }

    // Undo the admission of `r` (its allocation failed).
    void drop(CoreReq* r) {
        active.erase(std::remove(active.begin(), active.end(), r), active.end());
        held -= r->bytes;
    }

    // Stage ranges of a step.  Round robin: every admitted request advances
    // `passes` stages.  Budget: requests in admission order (oldest first)
    // take as many of their next stages (up to `passes`) as the step's work
    // budget still covers, and every request at least one, so the oldest
    // finish first while none stalls.
    void compose(StepPlan* sp) {
        sp->reqs.clear();
        sp->kb.clear();
        sp->ke.clear();
        sp->finishing.clear();
        double left = step_work;
        for (CoreReq* r : active) {
            int n = passes;
            if (policy == HP_SERVER_POLICY_BUDGET) {
                const double c = std::max(r->work, 1.0);
                n = std::max(1, std::min(passes, static_cast<int>(std::min(left / c, 1e9))));
                left = std::max(0.0, left - n * c);
            }
            const int kb = r->stage, ke = std::min(r->stage + n, r->stages);
            sp->reqs.push_back(r);
            sp->kb.push_back(kb);
            sp->ke.push_back(ke);
            r->stage = ke;
            if (ke == r->stages) sp->finishing.push_back(r);
        }
        for (CoreReq* r : sp->finishing) held -= r->bytes;
        active.erase(std::remove_if(active.begin(), active.end(), [](CoreReq* r) { return r->stage == r->stages; }),
                     active.end());
    }
};

}  // namespace hpx

namespace {

using Clock = std::chrono::steady_clock;
constexpr int kRing = 4;

double ms_between(Clock::time_point a, Clock::time_point b) {
    return std::chrono::duration<double, std::milli>(b - a).count();
}

size_t align256(size_t x) { return (x + 255) & ~size_t(255); }

struct SrvReq {
    CoreReq core;
    uint64_t id = 0;
    hp::ViewDesc desc{};
    hp_maps out{};
    void* mem = nullptr;
    float* staging = nullptr;  // host outputs: depth, normal, cost, confidence on the device
    std::vector<hp_seed> seeds;  // the job's SfM seeds, copied at submission
    int seed_radius = 0;
    double pix_iter = 0.0;
    bool failed = false;
    Clock::time_point t_submit, t_admit;
};

struct StepRec {
    int ring = 0;
    int launches = 0;
    bool launch_failed = false;  // an upload or launch error: the members' state is part-way
    std::vector<SrvReq*> members;
    std::vector<SrvReq*> finishing;
    // Per launch the schedule's entry tickets and (member, stage) infos, kept
    // to name the tile of a wait that ran out.
    std::vector<std::vector<int>> tickets;
    std::vector<std::vector<int2>> infos;
    uint64_t step_no = 0;
};

// A ring slot: pinned upload area + device copy, status words read back.
struct RingSlot {
    char* host = nullptr;
    char* dev = nullptr;
    int* host_status = nullptr;  // 4 ints per launch: code, unused, ticket whose wait ran out, pad
    cudaEvent_t ev0 = nullptr, ev1 = nullptr;
};

}  // namespace

struct hp_server {
    hp_ctx* ctx = nullptr;
    hp_params params{};
    hp_server_options opt{};
    hp::SolveConsts sc{};
    cudaStream_t stream = nullptr;
    cudaMemPool_t pool = nullptr;
    int sms = 0, occ = 0, cpsm = 1;
    size_t total_mem = 0;
    size_t ring_bytes = 0;
    int max_launches = 1;
    RingSlot ring[kRing];
    int* d_abort = nullptr;  // abort flag shared by the server's launches

    std::mutex mu;
    std::condition_variable cv_work, cv_done;
    std::thread worker;
    bool stop = false;
    std::deque<SrvReq*> incoming;       // submitted, not yet taken by the worker
    std::deque<hp_completion> done;     // completed, not yet polled
    uint64_t next_id = 1;
    uint64_t outstanding = 0;           // submitted and not yet completed
    std::string err;
    std::string first_err;              // the worker's first error since creation
    hp_server_stats st{};
    std::vector<double> latencies;

    // Worker-only state.
    ServerCore core;
    std::deque<StepRec> inflight;
    uint64_t step_no = 0;
};

namespace {

// Worker-side error message (the caller-side ones of hp_submit do not count
// as the server's first error).  Call with s->mu held.
void note_err_locked(hp_server* s, std::string msg) {
    if (s->first_err.empty()) s->first_err = msg;
    s->err = std::move(msg);
}

void set_err(hp_server* s, const char* what, cudaError_t e) {
    std::lock_guard<std::mutex> lk(s->mu);
    note_err_locked(s, std::string(what) + ": " + cudaGetErrorName(e) + " (" + cudaGetErrorString(e) + ")");
}

// Bytes of request state the server may hold: the byte limit, or the part of
// mem_fraction * total that memory outside the server's pool leaves free.
// 0 with *err set when the device cannot be queried (a faulted context).
uint64_t admission_budget(hp_server* s, cudaError_t* err) {
    *err = cudaSuccess;
    if (s->opt.mem_limit) return s->opt.mem_limit;
    size_t fr = 0, tot = 0;
    if ((*err = cudaMemGetInfo(&fr, &tot)) != cudaSuccess) return 0;
    uint64_t pool_reserved = 0;
    cudaMemPoolGetAttribute(s->pool, cudaMemPoolAttrReservedMemCurrent, &pool_reserved);
    {
        std::lock_guard<std::mutex> lk(s->mu);
        s->st.device_free_bytes = fr;
        s->st.pool_reserved_bytes = pool_reserved;
    }
    const double used = static_cast<double>(tot - fr);
    const double other = std::max(0.0, used - static_cast<double>(pool_reserved));
    const double b = static_cast<double>(s->opt.mem_fraction) * static_cast<double>(tot) - other;
    return b > 0 ? static_cast<uint64_t>(b) : 0;
}

uint64_t request_bytes(const hp::ViewDesc& d, bool host_out, size_t seed_bytes) {
    const size_t px = static_cast<size_t>(d.W) * d.H;
    size_t b = align256(px * (sizeof(float4) + sizeof(float)));
    b = align256(b + static_cast<size_t>(d.tiles_x) * d.tiles_y * sizeof(int));
    if (host_out) b = align256(b + px * 6 * sizeof(float));
    return align256(b + seed_bytes);
}

void complete(hp_server* s, SrvReq* r, int status, Clock::time_point now) {
    hp_completion c{};
    c.request_id = r->id;
    c.status = status;
    c.latency_ms = ms_between(r->t_submit, now);
    c.queue_ms = r->t_admit.time_since_epoch().count() ? ms_between(r->t_submit, r->t_admit) : c.latency_ms;
    {
        std::lock_guard<std::mutex> lk(s->mu);
        if (status == HP_OK) {
            s->st.completed++;
            s->st.pixel_iterations += r->pix_iter;
            s->latencies.push_back(c.latency_ms);
        } else {
            s->st.failed++;
        }
        if (status != HP_ERR_CANCELLED) s->done.push_back(c);
        s->outstanding--;
    }
    s->cv_done.notify_all();
    delete r;
}

// Allocate and initialise the state of a newly admitted request.
cudaError_t materialise(hp_server* s, SrvReq* r) {
    cudaError_t e = cudaMallocFromPoolAsync(&r->mem, r->core.bytes, s->pool, s->stream);
    if (e != cudaSuccess) {
        r->mem = nullptr;
        return e;
    }
    hp::ViewDesc& v = r->desc;
    const size_t px = static_cast<size_t>(v.W) * v.H;
    char* base = static_cast<char*>(r->mem);
    v.hyp = reinterpret_cast<float4*>(base);
    v.cost = reinterpret_cast<float*>(base + px * sizeof(float4));
    size_t off = align256(px * (sizeof(float4) + sizeof(float)));
    v.done = reinterpret_cast<int*>(base + off);
    const size_t flags = static_cast<size_t>(v.tiles_x) * v.tiles_y * sizeof(int);
    off = align256(off + flags);
    if (r->out.memory == HP_MEMORY_DEVICE) {
        v.out_depth = r->out.depth;
        v.out_normal = r->out.normal;
        v.out_cost = r->out.cost;
        v.out_conf = r->out.confidence;
    } else {
        r->staging = reinterpret_cast<float*>(base + off);
        v.out_depth = r->staging;
        v.out_normal = r->staging + px;
        v.out_cost = r->staging + 4 * px;
        v.out_conf = r->out.confidence ? r->staging + 5 * px : nullptr;
        off = align256(off + px * 6 * sizeof(float));
    }
    if (!r->seeds.empty()) {  // SfM seed list and index map, read by the initialisation stage
        hp_job sj{};
        sj.seeds = r->seeds.data();
        sj.num_seeds = static_cast<int>(r->seeds.size());
        sj.seed_radius = r->seed_radius;
        cudaError_t e = stage_seeds(&sj, base + off, &v, s->stream);
        if (e != cudaSuccess) return e;
    }
    return cudaMemsetAsync(v.done, 0xff, flags, s->stream);  // -1: no stage finished
}

// Compose and enqueue one step.  Returns false when nothing was enqueued.
bool enqueue_step(hp_server* s) {
    uint64_t budget = 0;
    cudaError_t budget_err = cudaSuccess;
    std::vector<CoreReq*> admitted;
    if (!s->core.queue.empty()) {
        budget = admission_budget(s, &budget_err);
        s->core.admit(budget, &admitted);
    }
    const auto now = Clock::now();
    for (CoreReq* c : admitted) {
        SrvReq* r = static_cast<SrvReq*>(c->user);
        r->t_admit = now;
        cudaError_t e = materialise(s, r);
        if (e != cudaSuccess) {
            s->core.drop(c);
            cudaGetLastError();
            if (r->mem) cudaFreeAsync(r->mem, s->stream);  // allocated, then a later set-up step failed
            r->mem = nullptr;
            set_err(s, "server: state allocation", e);
            complete(s, r, e == cudaErrorMemoryAllocation ? HP_ERR_OUT_OF_MEMORY : HP_ERR_CUDA, Clock::now());
        }
    }
    // A head request that cannot fit even with nothing else admitted never will.
    if (s->core.active.empty() && !s->core.queue.empty()) {
        SrvReq* r = static_cast<SrvReq*>(s->core.queue.front()->user);
        s->core.queue.pop_front();
        {
            std::lock_guard<std::mutex> lk(s->mu);
            if (budget_err != cudaSuccess)
                note_err_locked(s, std::string("server: device memory query: ") + cudaGetErrorName(budget_err) +
                                       " (" + cudaGetErrorString(budget_err) + ")");
            else
                note_err_locked(s, "server: request state exceeds the admission budget");
        }
        complete(s, r, budget_err != cudaSuccess ? HP_ERR_CUDA : HP_ERR_OUT_OF_MEMORY, Clock::now());
        return false;
    }
    {
        std::lock_guard<std::mutex> lk(s->mu);
        s->st.admitted += admitted.size();
        s->st.queued = static_cast<int>(s->core.queue.size());
        if (!admitted.empty()) s->st.budget_bytes = budget;
        s->st.state_bytes = s->core.held;
        s->st.peak_state_bytes = std::max<uint64_t>(s->st.peak_state_bytes, s->core.held);
        s->st.active = static_cast<int>(s->core.active.size());
        s->st.peak_active = std::max(s->st.peak_active, s->st.active);
    }
    if (s->core.active.empty()) return false;

    StepPlan sp;
    s->core.compose(&sp);
    const int n = static_cast<int>(sp.reqs.size());
    StepRec rec;
    rec.ring = static_cast<int>(s->step_no % kRing);
    RingSlot& slot = s->ring[rec.ring];

    // Schedules: one persistent launch over every stage range, or one launch per stage offset.
    std::vector<std::vector<int>> tickets;
    std::vector<std::vector<int2>> infos;
    std::vector<int> totals;
    std::vector<int> tiles(n);
    for (int k = 0; k < n; ++k) tiles[k] = sp.reqs[k]->tiles;
    const int offsets = s->opt.split_launches ? s->opt.passes_per_step : 1;
    for (int j = 0; j < offsets; ++j) {
        std::vector<int> kb(n), ke(n);
        for (int k = 0; k < n; ++k) {
            if (s->opt.split_launches) {
                kb[k] = std::min(sp.kb[k] + j, sp.ke[k]);
                ke[k] = std::min(sp.kb[k] + j + 1, sp.ke[k]);
            } else {
                kb[k] = sp.kb[k];
                ke[k] = sp.ke[k];
            }
        }
        std::vector<int> t;
        std::vector<int2> info;
        const int total = build_schedule(n, tiles.data(), kb.data(), ke.data(), &t, &info);
        if (total <= 0) continue;
        tickets.push_back(std::move(t));
        infos.push_back(std::move(info));
        totals.push_back(total);
    }
    rec.launches = static_cast<int>(totals.size());

    // Pinned upload: descriptors | per launch {counter, status[2], pad} | per launch tickets, infos.
    size_t off = align256(n * sizeof(hp::ViewDesc));
    const size_t off_ctr = off;
    off = align256(off + 16 * static_cast<size_t>(rec.launches));
    std::vector<size_t> off_t(rec.launches), off_i(rec.launches);
    for (int l = 0; l < rec.launches; ++l) {
        off_t[l] = off;
        off = align256(off + tickets[l].size() * sizeof(int));
        off_i[l] = off;
        off = align256(off + infos[l].size() * sizeof(int2));
    }
    const size_t bytes = off;
    // A step that cannot run leaves its members part-way: raise the shared
    // abort flag in stream order, so the launches queued behind it stop at
    // their first claim instead of waiting out the limit on that state.
    auto fail_step = [&](const char* what, cudaError_t e) {
        cudaGetLastError();
        set_err(s, what, e);
        rec.launch_failed = true;
        for (CoreReq* c : sp.reqs) static_cast<SrvReq*>(c->user)->failed = true;
        cudaMemsetAsync(s->d_abort, 0xff, sizeof(int), s->stream);
        cudaGetLastError();
    };
    if (bytes > s->ring_bytes || rec.launches > s->max_launches) {
        // Cannot happen with the sizes fixed at creation (max_active views, passes_per_step offsets).
        fail_step("server: step exceeds its upload area", cudaErrorInvalidValue);
        rec.launches = 0;
    } else {
        hp::ViewDesc* hv = reinterpret_cast<hp::ViewDesc*>(slot.host);
        for (int k = 0; k < n; ++k) hv[k] = static_cast<SrvReq*>(sp.reqs[k]->user)->desc;
        std::memset(slot.host + off_ctr, 0, 16 * static_cast<size_t>(rec.launches));
        for (int l = 0; l < rec.launches; ++l) {
            std::memcpy(slot.host + off_t[l], tickets[l].data(), tickets[l].size() * sizeof(int));
            std::memcpy(slot.host + off_i[l], infos[l].data(), infos[l].size() * sizeof(int2));
        }
    }
    cudaError_t e = cudaEventRecord(slot.ev0, s->stream);
    if (e == cudaSuccess && rec.launches > 0)
        e = cudaMemcpyAsync(slot.dev, slot.host, bytes, cudaMemcpyHostToDevice, s->stream);
    if (e != cudaSuccess) {
        fail_step("server: step upload", e);
        rec.launches = 0;
    }
    const bool f16 = s->params.precision == HP_PRECISION_F16ACC;
    const int ms = s->opt.wait_limit_ms > 0 ? s->opt.wait_limit_ms : 2000;
    if (s->opt.debug_fail_step > 0 && s->step_no + 1 == static_cast<uint64_t>(s->opt.debug_fail_step) &&
        rec.launches > 0) {  // tests: this step's launch fails on the host, nothing runs
        fail_step("server: persistent launch (injected failure)", cudaErrorLaunchOutOfResources);
        rec.launches = 0;
    }
    for (int l = 0; l < rec.launches; ++l) {
        hp::Schedule sch{};
        sch.views = reinterpret_cast<const hp::ViewDesc*>(slot.dev);
        sch.entry_ticket = reinterpret_cast<const int*>(slot.dev + off_t[l]);
        sch.entry_info = reinterpret_cast<const int2*>(slot.dev + off_i[l]);
        sch.n_entries = static_cast<int>(infos[l].size());
        sch.total = totals[l];
        sch.counter = reinterpret_cast<unsigned*>(slot.dev + off_ctr + 16 * l);
        sch.status = reinterpret_cast<int*>(slot.dev + off_ctr + 16 * l + 4);
        sch.abort = s->d_abort;
        sch.wait_limit_ns = static_cast<unsigned long long>(ms) * 1000000ull;
        sch.stall_view = -1;
        sch.stall_tile = -1;
        if (s->opt.debug_stall_request)
            for (int k = 0; k < n; ++k)
                if (static_cast<SrvReq*>(sp.reqs[k]->user)->id == s->opt.debug_stall_request) {
                    sch.stall_view = k;
                    sch.stall_tile = s->opt.debug_stall_tile;
                }
        sch.sc = s->sc;
        const int grid = std::max(1, std::min(totals[l], s->sms * s->cpsm));
        e = f16 ? hp::launch_persistent_f16(sch, grid, s->stream) : hp::launch_persistent_f32(sch, grid, s->stream);
        if (e == cudaSuccess)
            e = cudaMemcpyAsync(slot.host_status + 4 * l, sch.status, 3 * sizeof(int), cudaMemcpyDeviceToHost,
                                s->stream);
        if (e != cudaSuccess) {
            fail_step("server: persistent launch", e);
            rec.launches = l;
            break;
        }
    }
    // Finishing requests: host outputs leave the device, then the state returns to the pool.
    for (CoreReq* c : sp.finishing) {
        SrvReq* r = static_cast<SrvReq*>(c->user);
        if (r->staging) {
            const size_t px = static_cast<size_t>(r->desc.W) * r->desc.H;
            cudaError_t ce = cudaMemcpyAsync(r->out.depth, r->staging, px * sizeof(float), cudaMemcpyDeviceToHost,
                                             s->stream);
            if (ce == cudaSuccess)
                ce = cudaMemcpyAsync(r->out.normal, r->staging + px, 3 * px * sizeof(float), cudaMemcpyDeviceToHost,
                                     s->stream);
            if (ce == cudaSuccess)
                ce = cudaMemcpyAsync(r->out.cost, r->staging + 4 * px, px * sizeof(float), cudaMemcpyDeviceToHost,
                                     s->stream);
            if (ce == cudaSuccess && r->out.confidence)
                ce = cudaMemcpyAsync(r->out.confidence, r->staging + 5 * px, px * sizeof(float),
                                     cudaMemcpyDeviceToHost, s->stream);
            if (ce != cudaSuccess) {
                cudaGetLastError();
                set_err(s, "server: result copy", ce);
                r->failed = true;
            }
        }
        cudaFreeAsync(r->mem, s->stream);
        r->mem = nullptr;
    }
    cudaEventRecord(slot.ev1, s->stream);
    for (CoreReq* c : sp.reqs) rec.members.push_back(static_cast<SrvReq*>(c->user));
    for (CoreReq* c : sp.finishing) rec.finishing.push_back(static_cast<SrvReq*>(c->user));
    rec.tickets = std::move(tickets);
    rec.infos = std::move(infos);
    rec.step_no = s->step_no;
    {
        std::lock_guard<std::mutex> lk(s->mu);
        s->st.steps++;
        s->st.launches += rec.launches;
        s->st.active = static_cast<int>(s->core.active.size());
        s->st.state_bytes = s->core.held;
    }
    s->step_no++;
    s->inflight.push_back(std::move(rec));
    return true;
}

// The member, stage and tile of `ticket` in launch l of a step, as text.
std::string describe_ticket(const StepRec& rec, int l, int ticket) {
    if (l < 0 || l >= static_cast<int>(rec.tickets.size())) return "an unknown tile";
    const std::vector<int>& t = rec.tickets[l];
    const std::vector<int2>& info = rec.infos[l];
    if (info.empty() || ticket < 0 || ticket >= t.back()) return "an unknown tile";
    const size_t e = static_cast<size_t>(std::upper_bound(t.begin(), t.begin() + info.size(), ticket) - t.begin()) - 1;
    const int m = info[e].x;
    if (m < 0 || m >= static_cast<int>(rec.members.size())) return "an unknown tile";
    const SrvReq* r = rec.members[m];
    char buf[192];
    std::snprintf(buf, sizeof(buf), "request %llu (%dx%d, %d sources), stage %d, tile %d of %dx%d",
                  static_cast<unsigned long long>(r->id), r->desc.W, r->desc.H, r->desc.S, info[e].y,
                  ticket - t[e], r->desc.tiles_x, r->desc.tiles_y);
    return buf;
}

// The members of a step with their stage ranges, as text.
std::string describe_members(const StepRec& rec) {
    std::vector<int> lo(rec.members.size(), 1 << 30), hi(rec.members.size(), -1);
    for (const std::vector<int2>& info : rec.infos)
        for (const int2& e : info)
            if (e.x >= 0 && e.x < static_cast<int>(rec.members.size())) {
                lo[e.x] = std::min(lo[e.x], e.y);
                hi[e.x] = std::max(hi[e.x], e.y);
            }
    std::string out;
    for (size_t k = 0; k < rec.members.size(); ++k) {
        const SrvReq* r = rec.members[k];
        char buf[128];
        std::snprintf(buf, sizeof(buf), "%s%llu (%dx%d, %d sources, stages %d-%d of %d)", k ? ", " : "",
                      static_cast<unsigned long long>(r->id), r->desc.W, r->desc.H, r->desc.S, lo[k], hi[k],
                      r->core.stages);
        out += buf;
    }
    return out;
}

// Wait for the oldest step and report its finishing requests.  HP_OK, or the
// status its members fail with: HP_ERR_CUDA for an upload, launch or device
// error, HP_ERR_TIMEOUT for a persistent launch that gave up (its own wait
// ran out, or it stopped on the shared abort flag raised before it).  `cause`
// (during a recovery): the failed step's status, which the requests of the
// steps retired behind it take.
hp_status retire_oldest(hp_server* s, hp_status cause = HP_OK) {
    StepRec rec = std::move(s->inflight.front());
    s->inflight.pop_front();
    RingSlot& slot = s->ring[rec.ring];
    cudaError_t e = cudaEventSynchronize(slot.ev1);
    const auto now = Clock::now();
    bool failed = rec.launch_failed;
    if (e != cudaSuccess) {
        const std::string msg = "server: step " + std::to_string(rec.step_no) + ": " + cudaGetErrorName(e) + " (" +
                                cudaGetErrorString(e) + "); members: " + describe_members(rec);
        std::lock_guard<std::mutex> lk(s->mu);
        note_err_locked(s, msg);
        failed = true;
    } else {
        for (int l = 0; l < rec.launches; ++l) {
            const int code = slot.host_status[4 * l];
            if (code == hp::SCHED_OK) continue;
            failed = true;
            if (code == hp::SCHED_TIMEOUT) {
                const std::string where = describe_ticket(rec, l, slot.host_status[4 * l + 2]);
                std::lock_guard<std::mutex> lk(s->mu);
                note_err_locked(s, "server: a persistent dependency wait ran out in step " +
                                       std::to_string(rec.step_no) + " at " + where);
            }
        }
        float t = 0.f;
        if (cudaEventElapsedTime(&t, slot.ev0, slot.ev1) == cudaSuccess) {
            std::lock_guard<std::mutex> lk(s->mu);
            s->st.device_ms += t;
        }
    }
    const hp_status code = !failed ? HP_OK : (e != cudaSuccess || rec.launch_failed ? HP_ERR_CUDA : HP_ERR_TIMEOUT);
    if (failed) {
        for (SrvReq* r : rec.members) r->failed = true;
        std::lock_guard<std::mutex> lk(s->mu);
        s->st.failed_steps++;
        if (s->err.empty()) note_err_locked(s, "server: a step stopped");
    }
    // In a step that ran, a finishing request fails alone only when its result copy failed.  During a
    // recovery (cause set) the requests of the steps behind the failed one fail with its status.
    const hp_status fail_as = cause != HP_OK ? cause : code;
    for (SrvReq* r : rec.finishing) complete(s, r, r->failed ? (failed ? fail_as : HP_ERR_CUDA) : HP_OK, now);
    return code;
}

// After a failed step: retire the steps still in flight (their launches stop
// at their first claim on the raised flag), complete every admitted request
// with the failure (each was a member of the failed step or of one queued
// behind it), release their state, and clear the abort flag.  The queue is
// kept; its requests are admitted into clean steps afterwards.
void recover(hp_server* s, hp_status code) {
    while (!s->inflight.empty()) retire_oldest(s, code);
    cudaError_t e = cudaStreamSynchronize(s->stream);
    const auto now = Clock::now();
    std::vector<CoreReq*> lost;
    lost.swap(s->core.active);
    for (CoreReq* c : lost) {
        SrvReq* r = static_cast<SrvReq*>(c->user);
        s->core.held -= c->bytes;
        if (r->mem) cudaFreeAsync(r->mem, s->stream);
        r->mem = nullptr;
        complete(s, r, e != cudaSuccess ? HP_ERR_CUDA : code, now);
    }
    cudaMemsetAsync(s->d_abort, 0, sizeof(int), s->stream);
    cudaStreamSynchronize(s->stream);
    std::lock_guard<std::mutex> lk(s->mu);
    s->st.active = 0;
    s->st.state_bytes = s->core.held;
}

void worker_main(hp_server* s) {
    cudaSetDevice(s->ctx->device);
    const int depth = s->opt.inflight_steps;
    for (;;) {
        bool stopping;
        {
            std::unique_lock<std::mutex> lk(s->mu);
            if (s->core.active.empty() && s->core.queue.empty() && s->inflight.empty())
                s->cv_work.wait(lk, [&] { return s->stop || !s->incoming.empty(); });
            while (!s->incoming.empty()) {
                s->core.queue.push_back(&s->incoming.front()->core);
                s->incoming.pop_front();
            }
            stopping = s->stop;
        }
        if (stopping) {
            // Queued requests are cancelled; admitted ones run to completion.
            while (!s->core.queue.empty()) {
                SrvReq* r = static_cast<SrvReq*>(s->core.queue.front()->user);
                s->core.queue.pop_front();
                complete(s, r, HP_ERR_CANCELLED, Clock::now());
            }
            if (s->core.active.empty() && s->inflight.empty()) break;
        }
        bool launched = false;
        if (static_cast<int>(s->inflight.size()) < depth) launched = enqueue_step(s);
        if (s->inflight.empty()) continue;
        if (static_cast<int>(s->inflight.size()) >= depth || !launched) {
            if (!launched && s->core.active.empty()) {
                // Nothing more to launch: wait for the oldest step, but take new arrivals meanwhile.
                RingSlot& slot = s->ring[s->inflight.front().ring];
                if (cudaEventQuery(slot.ev1) == cudaErrorNotReady) {
                    std::unique_lock<std::mutex> lk(s->mu);
                    s->cv_work.wait_for(lk, std::chrono::microseconds(200),
                                        [&] { return s->stop || !s->incoming.empty(); });
                    continue;
                }
            }
            const hp_status st = retire_oldest(s);
            if (st != HP_OK) recover(s, st);
        }
    }
}

void free_server(hp_server* s) {
    if (s->stream) cudaStreamSynchronize(s->stream);
    if (s->d_abort) cudaFree(s->d_abort);
    s->d_abort = nullptr;
    for (RingSlot& r : s->ring) {
        if (r.host) cudaFreeHost(r.host);
        if (r.dev) cudaFree(r.dev);
        if (r.ev0) cudaEventDestroy(r.ev0);
        if (r.ev1) cudaEventDestroy(r.ev1);
        r = RingSlot();
    }
    if (s->stream) {
        cudaStreamSynchronize(s->stream);
        cudaStreamDestroy(s->stream);
    }
    if (s->pool) cudaMemPoolDestroy(s->pool);
    s->stream = nullptr;
    s->pool = nullptr;
}

}  // namespace

extern "C" {

void hp_server_options_default(hp_server_options* o) {
    if (!o) return;
    std::memset(o, 0, sizeof *o);
    o->max_active = 64;
    o->mem_fraction = 0.8f;
    o->mem_limit = 0;
    o->passes_per_step = 32;
    o->policy = HP_SERVER_POLICY_BUDGET;
    o->step_budget_mpix = 1200.0;
    o->split_launches = 0;
    o->ctas_per_sm = 0;
    o->inflight_steps = 2;
    o->wait_limit_ms = 2000;
}

hp_status hp_server_create(hp_ctx* ctx, const hp_params* params, const hp_server_options* options,
                           hp_server** out) {
    if (!ctx) return HP_ERR_INVALID_ARG;
    if (!out) return fail(ctx, HP_ERR_INVALID_ARG, "server_create: null server pointer");
    *out = nullptr;
    hp_status stc = check_params(ctx, params);
    if (stc != HP_OK) return stc;
    hp_server_options o;
    hp_server_options_default(&o);
    if (options) {
        o = *options;
        if (o.max_active == 0) o.max_active = 64;
        if (o.mem_fraction == 0.f) o.mem_fraction = 0.8f;
        if (o.passes_per_step == 0) o.passes_per_step = 8;
        if (o.inflight_steps == 0) o.inflight_steps = 2;
        if (o.wait_limit_ms == 0) o.wait_limit_ms = 2000;
    }
    if (o.max_active < 1 || o.max_active > 4096)
        return fail(ctx, HP_ERR_INVALID_ARG, "server_create: max_active %d outside 1..4096", o.max_active);
    if (!(o.mem_fraction > 0.f && o.mem_fraction <= 1.f))
        return fail(ctx, HP_ERR_INVALID_ARG, "server_create: mem_fraction must lie in (0, 1]");
    if (o.passes_per_step < 1 || o.passes_per_step > 64)
        return fail(ctx, HP_ERR_INVALID_ARG, "server_create: passes_per_step %d outside 1..64", o.passes_per_step);
    if (o.policy != HP_SERVER_POLICY_ROUND_ROBIN && o.policy != HP_SERVER_POLICY_BUDGET)
        return fail(ctx, HP_ERR_INVALID_ARG, "server_create: unknown policy %d", o.policy);
    if (o.step_budget_mpix == 0.0) o.step_budget_mpix = 1200.0;
    if (!(o.step_budget_mpix > 0.0) || !std::isfinite(o.step_budget_mpix))
        return fail(ctx, HP_ERR_INVALID_ARG, "server_create: step_budget_mpix invalid");
    if (o.inflight_steps < 1 || o.inflight_steps > kRing)
        return fail(ctx, HP_ERR_INVALID_ARG, "server_create: inflight_steps %d outside 1..%d", o.inflight_steps,
                    kRing);
    if (o.debug_stall_request && o.debug_stall_tile < 0)
        return fail(ctx, HP_ERR_INVALID_ARG, "server_create: debug_stall_tile %d negative", o.debug_stall_tile);
    if (o.debug_fail_step < 0)
        return fail(ctx, HP_ERR_INVALID_ARG, "server_create: debug_fail_step %d negative", o.debug_fail_step);
    if (o.wait_limit_ms < 1 || o.ctas_per_sm < 0)
        return fail(ctx, HP_ERR_INVALID_ARG, "server_create: invalid wait limit or CTA count");
    std::unique_ptr<hp_server> s(new hp_server);
    s->ctx = ctx;
    s->params = *params;
    s->opt = o;
    s->sc = consts_of(params);
    s->core.max_active = o.max_active;
    s->core.passes = o.passes_per_step;
    s->core.policy = o.policy;
    s->core.step_work = o.step_budget_mpix * 1e6;
    DeviceGuard g(ctx->device);
    struct Release {
        hp_server* p;
        ~Release() {
            if (p) free_server(p);
        }
    } release{s.get()};
    HP_CUDA(cudaStreamCreateWithFlags(&s->stream, cudaStreamNonBlocking));
    cudaMemPoolProps pp{};
    pp.allocType = cudaMemAllocationTypePinned;
    pp.location.type = cudaMemLocationTypeDevice;
    pp.location.id = ctx->device;
    HP_CUDA(cudaMemPoolCreate(&s->pool, &pp));
    uint64_t keep = ~0ull;  // keep freed state cached for the next requests
    HP_CUDA(cudaMemPoolSetAttribute(s->pool, cudaMemPoolAttrReleaseThreshold, &keep));
    HP_CUDA(cudaDeviceGetAttribute(&s->sms, cudaDevAttrMultiProcessorCount, ctx->device));
    HP_CUDA(params->precision == HP_PRECISION_F16ACC ? hp::persistent_occupancy_f16(s->sc, &s->occ)
                                                     : hp::persistent_occupancy_f32(params->radius, params->stride, &s->occ));
    if (s->occ < 1) return fail(ctx, HP_ERR_UNSUPPORTED, "server_create: persistent kernel does not fit on an SM");
    s->cpsm = (o.ctas_per_sm > 0 && o.ctas_per_sm < s->occ) ? o.ctas_per_sm : s->occ;
    size_t fr = 0;
    HP_CUDA(cudaMemGetInfo(&fr, &s->total_mem));
    // Upload area of one step: max_active descriptors, and per launch its counters and a
    // schedule of at most max_active * passes_per_step entries.
    s->max_launches = o.split_launches ? o.passes_per_step : 1;
    const size_t entries = static_cast<size_t>(o.max_active) * o.passes_per_step;
    s->ring_bytes = align256(o.max_active * sizeof(hp::ViewDesc)) + align256(16 * s->max_launches) +
                    s->max_launches * (align256((entries + 1) * sizeof(int)) + align256(entries * sizeof(int2)));
    HP_CUDA(cudaMalloc(&s->d_abort, sizeof(int)));
    HP_CUDA(cudaMemset(s->d_abort, 0, sizeof(int)));
    for (RingSlot& r : s->ring) {
        HP_CUDA(cudaMallocHost(&r.host, s->ring_bytes + 4 * sizeof(int) * s->max_launches));
        r.host_status = reinterpret_cast<int*>(r.host + s->ring_bytes);
        HP_CUDA(cudaMalloc(&r.dev, s->ring_bytes));
        HP_CUDA(cudaEventCreate(&r.ev0));
        HP_CUDA(cudaEventCreateWithFlags(&r.ev1, cudaEventBlockingSync));
    }
    hp_server* raw = s.get();
    try {
        s->worker = std::thread(worker_main, raw);
    } catch (...) {
        return fail(ctx, HP_ERR_UNSUPPORTED, "server_create: cannot start the worker thread");
    }
    release.p = nullptr;
    *out = s.release();
    return HP_OK;
}

hp_status hp_submit(hp_server* s, const hp_job* job, const hp_maps* out, uint64_t* request_id) {
    if (!s) return HP_ERR_INVALID_ARG;
    auto bad = [&](hp_status code, const char* msg) {
        std::lock_guard<std::mutex> lk(s->mu);
        s->err = msg;
        return code;
    };
    if (!job || !out || !request_id) return bad(HP_ERR_INVALID_ARG, "submit: null argument");
    if (!out->depth || !out->normal || !out->cost) return bad(HP_ERR_INVALID_ARG, "submit: output maps incomplete");
    if (out->memory != HP_MEMORY_HOST && out->memory != HP_MEMORY_DEVICE)
        return bad(HP_ERR_INVALID_ARG, "submit: unknown memory kind");
    std::unique_ptr<SrvReq> r(new SrvReq);
    std::lock_guard<std::mutex> lk(s->mu);
    if (s->stop) {
        s->err = "submit: server is stopping";
        return HP_ERR_CANCELLED;
    }
    // The context's images are read under the server lock (fill_desc reports through the context).
    hp_status st = check_seeds(s->ctx, job, 0);
    if (st == HP_OK) st = fill_desc(s->ctx, job, 0, &r->desc, s->sc.tile_h);
    if (st != HP_OK) {
        s->err = std::string("submit: ") + s->ctx->err;
        return st;
    }
    if (job->num_seeds > 0) {
        r->seeds.assign(job->seeds, job->seeds + job->num_seeds);
        r->seed_radius = job->seed_radius;
    }
    r->out = *out;
    r->core.tiles = r->desc.tiles_x * r->desc.tiles_y;
    r->core.work = static_cast<double>(r->desc.W) * r->desc.H * r->desc.S;
    r->core.stages = 2 * job->iterations + 2;
    r->core.bytes = request_bytes(r->desc, out->memory == HP_MEMORY_HOST,
                                  seed_area_bytes(job, r->desc.W, r->desc.H));
    r->core.user = r.get();
    r->pix_iter = static_cast<double>(r->desc.W) * r->desc.H * job->iterations;
    const uint64_t cap = s->opt.mem_limit ? s->opt.mem_limit
                                          : static_cast<uint64_t>(static_cast<double>(s->opt.mem_fraction) *
                                                                  static_cast<double>(s->total_mem));
    if (r->core.bytes > cap) {
        s->err = "submit: request state exceeds the admission budget";
        return HP_ERR_OUT_OF_MEMORY;
    }
    r->id = s->next_id++;
    r->t_submit = Clock::now();
    *request_id = r->id;
    s->st.submitted++;
    s->outstanding++;
    s->incoming.push_back(r.release());
    s->cv_work.notify_one();
    return HP_OK;
}

hp_status hp_poll(hp_server* s, hp_completion* done, int capacity, int* num_done, int timeout_ms) {
    if (!s || !num_done || capacity < 0 || (capacity > 0 && !done)) return HP_ERR_INVALID_ARG;
    std::unique_lock<std::mutex> lk(s->mu);
    auto ready = [&] { return !s->done.empty(); };
    if (timeout_ms < 0)
        s->cv_done.wait(lk, [&] { return ready() || s->outstanding == 0; });
    else if (timeout_ms > 0)
        s->cv_done.wait_for(lk, std::chrono::milliseconds(timeout_ms), ready);
    int n = 0;
    while (n < capacity && !s->done.empty()) {
        done[n++] = s->done.front();
        s->done.pop_front();
    }
    *num_done = n;
    return HP_OK;
}

hp_status hp_server_drain(hp_server* s, int timeout_ms) {
    if (!s) return HP_ERR_INVALID_ARG;
    std::unique_lock<std::mutex> lk(s->mu);
    auto idle = [&] { return s->outstanding == 0; };
    if (timeout_ms < 0) {
        s->cv_done.wait(lk, idle);
        return HP_OK;
    }
    return s->cv_done.wait_for(lk, std::chrono::milliseconds(timeout_ms), idle) ? HP_OK : HP_ERR_TIMEOUT;
}

hp_status hp_server_stats_get(hp_server* s, hp_server_stats* out) {
    if (!s || !out) return HP_ERR_INVALID_ARG;
    std::lock_guard<std::mutex> lk(s->mu);
    *out = s->st;
    out->queued = static_cast<int>(s->incoming.size()) + s->st.queued;
    std::vector<double> l = s->latencies;
    if (!l.empty()) {
        std::sort(l.begin(), l.end());
        auto q = [&](double p) {  // nearest-rank percentile
            size_t i = static_cast<size_t>(std::ceil(p * l.size()));
            return l[std::min(l.size() - 1, i > 0 ? i - 1 : 0)];
        };
        out->p50_ms = q(0.50);
        out->p99_ms = q(0.99);
        double sum = 0;
        for (double x : l) sum += x;
        out->mean_ms = sum / l.size();
        out->max_ms = l.back();
    }
    return HP_OK;
}

hp_status hp_server_stats_reset(hp_server* s) {
    if (!s) return HP_ERR_INVALID_ARG;
    std::lock_guard<std::mutex> lk(s->mu);
    const int active = s->st.active, queued = s->st.queued;
    const uint64_t held = s->st.state_bytes;
    s->st = hp_server_stats{};
    s->st.active = s->st.peak_active = active;
    s->st.queued = queued;
    s->st.state_bytes = s->st.peak_state_bytes = held;
    s->latencies.clear();
    return HP_OK;
}

const char* hp_server_last_error(hp_server* s) {
    if (!s) return "null server";
    std::lock_guard<std::mutex> lk(s->mu);
    thread_local std::string copy;
    copy = s->err;
    return copy.c_str();
}

const char* hp_server_first_error(hp_server* s) {
    if (!s) return "null server";
    std::lock_guard<std::mutex> lk(s->mu);
    thread_local std::string copy;
    copy = s->first_err;
    return copy.c_str();
}

hp_status hp_server_destroy(hp_server* s) {
    if (!s) return HP_ERR_INVALID_ARG;
    {
        std::lock_guard<std::mutex> lk(s->mu);
        s->stop = true;
    }
    s->cv_work.notify_all();
    if (s->worker.joinable()) s->worker.join();
    {
        DeviceGuard g(s->ctx->device);
        free_server(s);
    }
    for (SrvReq* r : s->incoming) delete r;
    delete s;
    return HP_OK;
}

hp_status hp_server_simulate_policy(int n, const int* arrive_step, const uint64_t* state_bytes, const int* stages,
                                    const double* work, int max_active, uint64_t budget, int passes_per_step,
                                    int policy, double step_work, int* admit_step, int* finish_step, int* steps) {
    if (n < 0 || (n > 0 && (!arrive_step || !state_bytes || !stages || !admit_step || !finish_step)) || !steps ||
        max_active < 1 || passes_per_step < 1 ||
        (policy != HP_SERVER_POLICY_ROUND_ROBIN && policy != HP_SERVER_POLICY_BUDGET) ||
        (policy == HP_SERVER_POLICY_BUDGET && (n > 0 && !work)) || !(step_work >= 0.0))
        return HP_ERR_INVALID_ARG;
    std::vector<CoreReq> reqs(n);
    std::vector<int> order(n);
    for (int k = 0; k < n; ++k) {
        if (stages[k] < 2 || arrive_step[k] < 0) return HP_ERR_INVALID_ARG;
        if (state_bytes[k] > budget) return HP_ERR_OUT_OF_MEMORY;
        reqs[k].stages = stages[k];
        reqs[k].bytes = state_bytes[k];
        reqs[k].work = work ? work[k] : 0.0;
        reqs[k].tiles = 1;
        reqs[k].user = reinterpret_cast<void*>(static_cast<intptr_t>(k));
        order[k] = k;
        admit_step[k] = finish_step[k] = -1;
    }
    std::stable_sort(order.begin(), order.end(), [&](int a, int b) { return arrive_step[a] < arrive_step[b]; });
    ServerCore core;
    core.max_active = max_active;
    core.passes = passes_per_step;
    core.policy = policy;
    core.step_work = step_work;
    int next = 0, finished = 0, ran = 0;
    for (int tick = 0; finished < n; ++tick) {
        while (next < n && arrive_step[order[next]] <= tick) core.queue.push_back(&reqs[order[next++]]);
        std::vector<CoreReq*> admitted;
        core.admit(budget, &admitted);
        for (CoreReq* c : admitted) admit_step[reinterpret_cast<intptr_t>(c->user)] = tick;
        if (core.active.empty()) continue;
        StepPlan sp;
        core.compose(&sp);
        ++ran;
        for (CoreReq* c : sp.finishing) {
            finish_step[reinterpret_cast<intptr_t>(c->user)] = tick;
            ++finished;
        }
    }
    *steps = ran;
    return HP_OK;
}

hp_status hp_server_simulate(int n, const int* arrive_step, const uint64_t* state_bytes, const int* stages,
                             int max_active, uint64_t budget, int passes_per_step, int* admit_step,
                             int* finish_step, int* steps) {
    return hp_server_simulate_policy(n, arrive_step, state_bytes, stages, nullptr, max_active, budget,
                                     passes_per_step, HP_SERVER_POLICY_ROUND_ROBIN, 0.0, admit_step, finish_step,
                                     steps);
}

}  // extern "C"
