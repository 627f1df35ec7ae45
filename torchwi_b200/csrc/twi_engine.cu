// twi_engine.cu -- continuous batching of propagation requests.
//
// A request is a bound plan plus a kind: forward modelling, or a gradient
// (forward with checkpoints, residual against observed gathers, checkpointed
// adjoint).  Every tick advances each in-flight request by one time step;
// the steps of all requests that are in the same kernel mode form ONE
// multi-plan launch (twi_step.cu, step_kernel_multi).  Requests join and
// leave between ticks, so a short request admitted while a long one runs
// finishes after its own number of ticks, sharing the GPU with the long one.
//
// A request's static arguments (one template per kernel mode) and tensor
// maps are uploaded once, at admission, into fixed slots of the engine's
// workspace; a launch carries its jobs' per-step integers and CTA offsets in
// its kernel parameters, so ticks issue no copies.  Everything -- uploads,
// launches, residual and reduction kernels -- is enqueued on the stream
// passed to twi_engine_run, so reuse of a slot is ordered after the kernels
// that read it; its pinned host staging is reused only after the event of
// its last upload has completed.
#include <cuda.h>
#include <cuda_runtime.h>

#include <algorithm>
#include <cstring>
#include <deque>
#include <string>
#include <vector>

#include "twi_b200.h"
#include "twi_kernels.h"
#include "twi_plan_internal.h"

namespace twi {
void set_last_error(const std::string& msg);
}

namespace {

int efail(int code, const std::string& msg) {
    twi::set_last_error(msg);
    return code;
}

#define ENG_CUDA(expr)                                                                  \
    do {                                                                                \
        cudaError_t e_ = (expr);                                                        \
        if (e_ != cudaSuccess)                                                          \
            return efail(TWI_ERR_CUDA, std::string(#expr) + ": " + cudaGetErrorString(e_)); \
    } while (0)

}  // namespace

using namespace twi;

struct twi_engine {
    int order = 4;
    bool exact = true;
    LaunchShape shape{4, 4};
    LaunchShape shape_back{2, 4};   // fused backward steps of boundary-saving requests
    static constexpr int kModes = 6;   // templates indexed by StepMode
    int max_requests = 0;
    char* ws = nullptr;
    size_t off_tmaps = 0, off_tmpl = 0, total = 0;
    // pinned staging per request slot: its tensor maps and per-mode templates
    struct SlotStage {
        CUtensorMap tm[kMapsPerPlan];
        MultiJob tmpl[kModes];
    };
    SlotStage* staging = nullptr;
    std::vector<cudaEvent_t> slot_events;   // per slot: its last upload

    struct Request {
        twi_plan* plan = nullptr;
        int kind = 0;                   // 0 forward, 1 gradient
        const float* observed = nullptr;
        long long tag = 0;
        int slot = -1;                  // tensor-map / template slot
        std::vector<TwiStep> steps;     // forward steps, then gradient steps
        int nbc[kModes] = {}, ncta[kModes] = {};   // per kernel mode
        CUtensorMap tm[kMapsPerPlan];   // host copy of the plan's tensor maps
        size_t fwd_steps = 0, pos = 0;
        bool started = false;
    };
    std::vector<Request> active;
    std::vector<int> free_slots;
    std::deque<Request> waiting;        // submitted, not yet on the device
    std::deque<long long> completed;    // finished, not yet reported

    const MultiJob* tmpl_dev(int slot, int mode) const {
        return reinterpret_cast<const MultiJob*>(ws + off_tmpl) + kModes * slot + mode;
    }

    int admit(cudaStream_t st) {
        while (!waiting.empty() && !free_slots.empty()) {
            Request R = std::move(waiting.front());
            waiting.pop_front();
            R.slot = free_slots.back();
            free_slots.pop_back();
            // the previous upload of this slot's staging has been read
            ENG_CUDA(cudaEventSynchronize(slot_events[R.slot]));
            SlotStage& S = staging[R.slot];
            plan_tensor_maps(R.plan, S.tm);
            std::memcpy(R.tm, S.tm, sizeof(R.tm));
            bool seen[kModes] = {};
            for (const TwiStep& t : R.steps) {   // static arguments per kernel mode
                const int m = static_cast<int>(t.mode);
                if (seen[m]) continue;
                seen[m] = true;
                S.tmpl[m] = MultiJob{};
                S.tmpl[m].a = t.a;
                S.tmpl[m].plan = R.slot;
                R.ncta[m] = t.mode == kModeBackward
                                ? backward_ctas(order, shape_back.rows_per_warp, t.a, &R.nbc[m])
                                : step_ctas(order, shape, t.a, &R.nbc[m]);
                S.tmpl[m].nbc = R.nbc[m];
                S.tmpl[m].ncta = R.ncta[m];
                if (R.ncta[m] <= 0) return efail(TWI_ERR_INVALID, "request launch too large");
            }
            // enqueued on the engine's stream: ordered after every kernel that
            // read this slot for an earlier request
            ENG_CUDA(cudaMemcpyAsync(ws + off_tmaps + kMapsPerPlan * R.slot * sizeof(CUtensorMap), S.tm,
                                     sizeof(S.tm), cudaMemcpyHostToDevice, st));
            ENG_CUDA(cudaMemcpyAsync(const_cast<MultiJob*>(tmpl_dev(R.slot, 0)), S.tmpl,
                                     sizeof(S.tmpl), cudaMemcpyHostToDevice, st));
            ENG_CUDA(cudaEventRecord(slot_events[R.slot], st));
            active.push_back(std::move(R));
        }
        return TWI_OK;
    }

    // Extra work at phase boundaries of a request, enqueued before its next
    // step is launched (start of the gradient) or after its last one.
    int before_step(Request& R, cudaStream_t st) {
        if (R.kind == 1 && R.pos == R.fwd_steps && !R.started) {
            if (R.observed) {   // NULL observed gathers: zero data, residual = gathers
                float* frd = plan_gathers(R.plan);
                const long long n = plan_gathers_elems(R.plan);
                ENG_CUDA(launch_residual(frd, R.observed, n, st));
            }
            int s = plan_gradient_prologue(R.plan, st);
            if (s != TWI_OK) return s;
            R.started = true;
        }
        return TWI_OK;
    }

    int launch(EngineLaunch& L, StepMode m, long long nctas, cudaStream_t st) {
        const CUtensorMap* tm = reinterpret_cast<const CUtensorMap*>(ws + off_tmaps);
        ENG_CUDA(m == kModeBackward ? launch_backward_engine(order, exact, shape_back, L, nctas, tm, st)
                                    : launch_step_engine(order, exact, m, shape, L, nctas, tm, st));
        L.njobs = 0;
        return TWI_OK;
    }

    int tick(cudaStream_t st, std::vector<long long>& done) {
        for (Request& R : active) {
            int s = before_step(R, st);
            if (s != TWI_OK) return s;
        }
        EngineLaunch L;
        for (StepMode m : {kModeForward, kModeRecompute, kModeAdjoint, kModeBackward}) {
            L.njobs = 0;
            long long nctas = 0;
            // a mode with one job takes the single-plan kernel with the job's own
            // arguments and tensor maps, exactly as the plan alone launches it
            Request* only = nullptr;
            int count = 0;
            for (Request& R : active)
                if (R.pos < R.steps.size() && R.steps[R.pos].mode == m) only = &R, ++count;
            if (count == 1) {
                const StepArgs& a = only->steps[only->pos].a;
                cudaError_t e = m == kModeBackward
                    ? launch_backward(order, exact, shape_back, only->tm[3], only->tm[4], only->tm[5], a, st)
                    : launch_step(order, exact, m, shape, only->tm[0], only->tm[1], only->tm[2], a, st);
                if (e != cudaSuccess)
                    return efail(TWI_ERR_CUDA, std::string("engine launch: ") + cudaGetErrorString(e));
                continue;
            }
            for (Request& R : active) {
                if (R.pos >= R.steps.size() || R.steps[R.pos].mode != m) continue;
                if (L.njobs == kEngineMaxJobs) {   // full: launch and start another
                    int s = launch(L, m, nctas, st);
                    if (s != TWI_OK) return s;
                    nctas = 0;
                }
                L.cta_begin[L.njobs] = (int)nctas;
                L.tmpl[L.njobs] = tmpl_dev(R.slot, m);
                L.dyn[L.njobs] = dyn_of(R.steps[R.pos].a);
                ++L.njobs;
                nctas += R.ncta[m];
            }
            if (L.njobs) {
                int s = launch(L, m, nctas, st);
                if (s != TWI_OK) return s;
            }
        }
        std::vector<Request> still;
        for (Request& R : active) {
            ++R.pos;
            if (R.pos < R.steps.size()) {
                still.push_back(std::move(R));
                continue;
            }
            if (R.kind == 1) {
                int s = plan_gradient_epilogue(R.plan, st);
                if (s != TWI_OK) return s;
            }
            plan_mark_done(R.plan, R.kind);
            free_slots.push_back(R.slot);
            done.push_back(R.tag);
        }
        active.swap(still);
        return TWI_OK;
    }
};

extern "C" {

int twi_engine_create(int order, int exact, int rows_per_warp, int max_requests,
                      twi_engine** out) {
    if (!out) return efail(TWI_ERR_INVALID, "null argument");
    if (order != 2 && order != 4 && order != 8) return efail(TWI_ERR_INVALID, "order must be 2, 4 or 8");
    if (max_requests < 1 || max_requests > 4096)
        return efail(TWI_ERR_INVALID, "max_requests must be in [1, 4096]");
    if (rows_per_warp != 0 && rows_per_warp != 2 && rows_per_warp != 4 && rows_per_warp != 8)
        return efail(TWI_ERR_INVALID, "rows_per_warp must be 0, 2, 4 or 8");
    twi_engine* E = new twi_engine();
    E->order = order;
    E->exact = exact != 0;
    E->shape = LaunchShape{rows_per_warp == 8 || rows_per_warp == 2 ? rows_per_warp : 4, 4};
    E->shape_back = LaunchShape{backward_rows(rows_per_warp), 4};
    E->max_requests = max_requests;
    size_t off = 0;
    auto take = [&](size_t b) { size_t o = off; off = (off + b + 255) & ~size_t(255); return o; };
    E->off_tmaps = take((size_t)max_requests * kMapsPerPlan * sizeof(CUtensorMap));
    E->off_tmpl = take((size_t)max_requests * twi_engine::kModes * sizeof(MultiJob));
    E->total = off;
    for (int i = max_requests - 1; i >= 0; --i) E->free_slots.push_back(i);
    *out = E;
    return TWI_OK;
}

int twi_engine_workspace_size(const twi_engine* E, size_t* bytes) {
    if (!E || !bytes) return efail(TWI_ERR_INVALID, "null argument");
    *bytes = E->total;
    return TWI_OK;
}

int twi_engine_bind(twi_engine* E, void* workspace, size_t bytes) {
    if (!E || !workspace) return efail(TWI_ERR_INVALID, "null argument");
    if (bytes < E->total) return efail(TWI_ERR_NOMEM, "engine workspace too small");
    if (reinterpret_cast<uintptr_t>(workspace) % 256)
        return efail(TWI_ERR_INVALID, "workspace must be 256-byte aligned");
    if (!E->active.empty()) return efail(TWI_ERR_STATE, "engine has requests in flight");
    E->ws = static_cast<char*>(workspace);
    if (!E->staging) {
        void* p = nullptr;
        ENG_CUDA(cudaHostAlloc(&p, (size_t)E->max_requests * sizeof(twi_engine::SlotStage),
                               cudaHostAllocDefault));
        E->staging = static_cast<twi_engine::SlotStage*>(p);
        E->slot_events.assign(E->max_requests, nullptr);
        for (auto& ev : E->slot_events) ENG_CUDA(cudaEventCreateWithFlags(&ev, cudaEventDisableTiming));
    }
    return TWI_OK;
}

int twi_engine_submit(twi_engine* E, twi_plan* plan, int kind, const float* observed,
                      long long tag) {
    if (!E || !plan) return efail(TWI_ERR_INVALID, "null argument");
    if (kind != 0 && kind != 1) return efail(TWI_ERR_INVALID, "kind must be 0 (forward) or 1 (gradient)");
    int s = plan_check_compatible(plan, kind, E->order, E->exact, E->shape.rows_per_warp,
                                  E->shape_back.rows_per_warp);
    if (s != TWI_OK) return s;
    twi_engine::Request R;
    R.plan = plan;
    R.kind = kind;
    R.observed = observed;
    R.tag = tag;
    plan_steps(plan, kind, R.steps, &R.fwd_steps);
    E->waiting.push_back(std::move(R));
    return TWI_OK;
}

int twi_engine_run(twi_engine* E, int ticks, void* stream, long long* done_tags, int max_done,
                   int* ndone) {
    if (!E || !E->ws) return efail(TWI_ERR_STATE, "engine has no workspace");
    if (!ndone || (max_done > 0 && !done_tags)) return efail(TWI_ERR_INVALID, "null argument");
    cudaStream_t st = static_cast<cudaStream_t>(stream);
    int s = E->admit(st);
    // stop early once something finished so the caller can collect it
    for (int t = 0; t < ticks && s == TWI_OK && !E->active.empty() && E->completed.empty(); ++t) {
        std::vector<long long> done;
        s = E->tick(st, done);
        for (long long d : done) E->completed.push_back(d);
        if (s == TWI_OK && !done.empty()) s = E->admit(st);   // freed slots
    }
    if (s != TWI_OK) return s;
    int n = 0;
    while (n < max_done && !E->completed.empty()) {
        done_tags[n++] = E->completed.front();
        E->completed.pop_front();
    }
    *ndone = n;
    return TWI_OK;
}

int twi_engine_pending(const twi_engine* E, int* in_flight, int* waiting) {
    if (!E || !in_flight || !waiting) return efail(TWI_ERR_INVALID, "null argument");
    *in_flight = (int)E->active.size();
    *waiting = (int)E->waiting.size() + (int)E->completed.size();
    return TWI_OK;
}

int twi_engine_destroy(twi_engine* E) {
    if (!E) return TWI_OK;
    for (auto& ev : E->slot_events)
        if (ev) cudaEventSynchronize(ev), cudaEventDestroy(ev);
    if (E->staging) cudaFreeHost(E->staging);
    delete E;
    return TWI_OK;
}

}  // extern "C"
