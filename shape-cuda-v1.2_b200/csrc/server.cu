// Continuous-batching evaluation server of the SHAPE B200 engine.
//
// A workload is a model with its datasets, registered once from a
// configured engine. The server keeps device-resident INSTANCES of
// workloads (each an engine with its own device arenas, stream and captured
// evaluation graph). A request names a workload, its scale factors and its
// arrival time; the loop admits each arrived request, in arrival order, to an
// idle instance of its workload as soon as a slot is free, creating an
// instance when the HBM budget allows and evicting idle instances of other
// workloads (least recently used first) when it does not. Requests run on
// their instances' streams, so work of different requests overlaps on the
// device; completions are polled through events, and each request's latency
// is its completion time minus its arrival time.
#include <algorithm>
#include <chrono>
#include <deque>
#include <memory>
#include <thread>
#include <vector>

#include "engine_impl.h"

namespace shape {

struct Instance {
    std::unique_ptr<EngineImpl> eng;
    int id = 0;                          // stable number, in creation order
    int workload = -1;
    int busy = 0;
    int request = -1;
    double last_used = 0.0;
};

struct Workload {
    std::unique_ptr<EngineImpl> proto;   // host description (never finalized)
    int form = SHAPE_FORM_BATCHED_FP32;
    size_t footprint = 0;                // device bytes of one instance
    int frames = 0;                      // frame-evals per request
};

struct ServerImpl {
    int device = 0;
    size_t budget = 0, used = 0, peak_used = 0;
    int max_slots = 8;
    std::vector<Workload> wl;
    std::vector<std::unique_ptr<Instance>> inst;
    int created = 0, evicted = 0;

    int make_instance(int w, Instance **out)
    {
        auto I = std::make_unique<Instance>();
        I->eng = std::make_unique<EngineImpl>();
        EngineImpl &E = *I->eng;
        E.device = device;
        if (cudaStreamCreateWithFlags(&E.stream, cudaStreamNonBlocking) != cudaSuccess ||
            cudaEventCreate(&E.ev0) != cudaSuccess || cudaEventCreate(&E.ev1) != cudaSuccess)
            return report_error(SHAPE_E_CUDA, "server: stream/event creation failed");
        E.clone_host_state(*wl[w].proto);
        I->id = created;
        int rc = E.finalize();
        if (rc) return rc;
        shape_eval_summary s;
        rc = E.evaluate(wl[w].form, &s);       // captures the evaluation graph
        if (rc) return rc;
        wl[w].footprint = E.footprint();
        I->workload = w;
        used += wl[w].footprint;
        peak_used = std::max(peak_used, used);
        created++;
        *out = I.get();
        inst.push_back(std::move(I));
        return SHAPE_OK;
    }

    // Evicts idle instances of workloads other than w, least recently used
    // first, until need more bytes fit in the budget. False if they cannot.
    bool make_room(int w, size_t need)
    {
        while (used + need > budget) {
            Instance *victim = nullptr;
            for (auto &I : inst)
                if (!I->busy && I->workload != w && (!victim || I->last_used < victim->last_used))
                    victim = I.get();
            if (!victim) return false;
            used -= wl[victim->workload].footprint;
            for (size_t k = 0; k < inst.size(); k++)
                if (inst[k].get() == victim) { inst.erase(inst.begin() + k); break; }
            evicted++;
        }
        return true;
    }

    // An idle instance of workload w, creating one (and evicting idle
    // instances of other workloads, least recently used first) when the
    // budget needs it. *out = nullptr when nothing can be admitted now.
    int acquire(int w, double now, Instance **out)
    {
        *out = nullptr;
        for (auto &I : inst)
            if (I->workload == w && !I->busy) { *out = I.get(); return SHAPE_OK; }
        if (!make_room(w, wl[w].footprint)) return SHAPE_OK;   // wait for a running request
        (void)now;
        return make_instance(w, out);
    }
};

}  // namespace shape

using namespace shape;

struct shape_server {
    ServerImpl impl;
};

extern "C" int shape_server_create(int device, size_t hbm_budget_bytes, int max_slots, shape_server **out)
{
    if (!out || max_slots < 1 || hbm_budget_bytes == 0) return report_error(SHAPE_E_ARG, "server_create: bad argument");
    if (cudaSetDevice(device) != cudaSuccess) return report_error(SHAPE_E_CUDA, "server_create: bad device");
    shape_server *s = new shape_server();
    s->impl.device = device;
    s->impl.budget = hbm_budget_bytes;
    s->impl.max_slots = max_slots;
    *out = s;
    return SHAPE_OK;
}

extern "C" void shape_server_destroy(shape_server *s)
{
    if (!s) return;
    cudaSetDevice(s->impl.device);
    delete s;
}

// Copies the engine's host description and builds one instance right away,
// which measures the workload's device footprint and leaves a warm instance.
extern "C" int shape_server_add_workload(shape_server *s, shape_engine *engine, int form)
{
    if (!s || !engine) return report_error(SHAPE_E_ARG, "server_add_workload: null argument");
    if (form < 0 || form > 2) return report_error(SHAPE_E_ARG, "server_add_workload: unknown form");
    const EngineImpl &src = engine->impl;
    if (!src.have_model || (src.frames.empty() && src.points.empty()))
        return report_error(SHAPE_E_STATE, "server_add_workload: engine has no model or no data");
    ServerImpl &S = s->impl;
    cudaSetDevice(S.device);
    Workload W;
    W.proto = std::make_unique<EngineImpl>();
    W.proto->clone_host_state(src);
    W.form = form;
    W.frames = (int)(src.frames.size() + src.points.size());
    S.wl.push_back(std::move(W));
    const int w = (int)S.wl.size() - 1;
    Instance *I = nullptr;
    int rc = S.make_instance(w, &I);
    if (rc == SHAPE_OK && !S.make_room(w, 0)) {
        // larger than what the budget leaves free even after evictions
        S.used -= S.wl[w].footprint;
        S.inst.pop_back();
        S.created--;
        rc = report_error(SHAPE_E_NOMEM, "server_add_workload: one instance exceeds the HBM budget");
    }
    if (rc) {
        S.wl.pop_back();
        return rc;
    }
    return w;
}

extern "C" int shape_server_workload_bytes(shape_server *s, int w, size_t *bytes)
{
    if (!s || !bytes || w < 0 || w >= (int)s->impl.wl.size())
        return report_error(SHAPE_E_ARG, "server_workload_bytes: bad argument");
    *bytes = s->impl.wl[w].footprint;
    return SHAPE_OK;
}

extern "C" int shape_server_run(shape_server *s, const shape_request *req, int n, shape_request_result *res,
                                shape_server_stats *stats)
{
    if (!s || !req || n <= 0 || !res || !stats) return report_error(SHAPE_E_ARG, "server_run: bad argument");
    ServerImpl &S = s->impl;
    cudaSetDevice(S.device);
    for (int i = 0; i < n; i++)
        if (req[i].workload < 0 || req[i].workload >= (int)S.wl.size())
            return report_error(SHAPE_E_ARG, "server_run: unknown workload");
    std::vector<int> order(n);
    for (int i = 0; i < n; i++) order[i] = i;
    std::stable_sort(order.begin(), order.end(),
                     [&](int a, int b) { return req[a].arrival_s < req[b].arrival_s; });
    using clk = std::chrono::steady_clock;
    const auto t0 = clk::now();
    auto now_s = [&]() { return std::chrono::duration<double>(clk::now() - t0).count(); };
    std::deque<int> waiting;                 // arrived, not yet admitted
    std::vector<Instance *> running;
    int next = 0, done = 0, peak_conc = 0;
    const int created0 = S.created, evicted0 = S.evicted;
    S.peak_used = S.used;                    // peak over this run
    double conc_integral = 0.0, t_prev = 0.0;
    long long frames_done = 0;
    while (done < n) {
        const double t = now_s();
        conc_integral += (t - t_prev) * (double)running.size();
        t_prev = t;
        while (next < n && req[order[next]].arrival_s <= t) waiting.push_back(order[next++]);
        // completions
        bool progressed = false;
        for (size_t k = 0; k < running.size();) {
            Instance *I = running[k];
            int pr = I->eng->poll();
            if (pr < 0) return pr;
            if (pr == 1) {
                shape_eval_summary sm;
                int rc = I->eng->finish(&sm);
                if (rc) return rc;
                shape_request_result &R = res[I->request];
                R.chi2 = sm.chi2;
                R.objective = sm.objective;
                R.t_done = now_s();
                R.latency_s = R.t_done - req[I->request].arrival_s;
                R.device_ms = I->eng->last_ms;
                frames_done += S.wl[I->workload].frames;
                I->busy = 0;
                I->last_used = R.t_done;
                running.erase(running.begin() + k);
                done++;
                progressed = true;
            } else {
                k++;
            }
        }
        // admissions, in arrival order
        while (!waiting.empty() && (int)running.size() < S.max_slots) {
            const int r = waiting.front();
            Instance *I = nullptr;
            int rc = S.acquire(req[r].workload, t, &I);
            if (rc) return rc;
            if (!I) break;                     // memory frees up when a request finishes
            waiting.pop_front();
            EngineImpl &E = *I->eng;
            for (int j = 0; j < 3; j++) E.scale[j] = req[r].scale[j];
            res[r].t_start = now_s();
            res[r].instance = I->id;
            rc = E.launch(S.wl[req[r].workload].form);
            if (rc) return rc;
            I->busy = 1;
            I->request = r;
            running.push_back(I);
            peak_conc = std::max(peak_conc, (int)running.size());
            progressed = true;
        }
        if (!progressed) {
            if (running.empty() && waiting.empty() && next < n) {
                const double wait = req[order[next]].arrival_s - now_s();
                if (wait > 2e-4) std::this_thread::sleep_for(std::chrono::microseconds((long)(wait * 1e6) - 100));
            } else {
                std::this_thread::yield();
            }
        }
    }
    const double span = now_s();
    std::vector<double> lat(n);
    for (int i = 0; i < n; i++) lat[i] = res[i].latency_s;
    std::sort(lat.begin(), lat.end());
    auto pct = [&](double p) {
        double pos = p * (n - 1);
        int lo = (int)pos;
        int hi = std::min(lo + 1, n - 1);
        return lat[lo] + (pos - lo) * (lat[hi] - lat[lo]);
    };
    stats->span_s = span;
    stats->requests_per_s = n / span;
    stats->frame_evals_per_s = frames_done / span;
    stats->p50_latency_s = pct(0.50);
    stats->p99_latency_s = pct(0.99);
    stats->mean_concurrency = conc_integral / std::max(span, 1e-12);
    stats->peak_concurrency = peak_conc;
    stats->instances_created = S.created - created0;
    stats->instances_evicted = S.evicted - evicted0;
    stats->peak_hbm_bytes = (double)S.peak_used;
    return SHAPE_OK;
}
