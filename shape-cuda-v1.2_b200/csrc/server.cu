// Continuous-batching evaluation server of the SHAPE B200 engine.
//
// A workload is a model with its datasets, registered once from a
// configured engine. The server keeps device-resident INSTANCES of
// workloads (each an engine with its own device arenas, stream and captured
// evaluation graph). Requests (a workload and its scale factors) are
// submitted as they arrive and served by a scheduler thread:
//   - completions are polled through each running instance's event;
//   - admission walks the waiting requests oldest first and admits every
//     one it can right now: to an idle instance of its workload, or to a new
//     instance when the HBM budget allows (idle instances of other
//     workloads are evicted, least recently used first, to make room). A
//     request that cannot be admitted does not hold up the ones behind it,
//     except that once the oldest has waited longer than the starvation
//     bound, later requests may only use instances that already exist, so
//     the memory that frees up goes to it;
//   - up to max_slots requests run at once, each on its instance's stream,
//     so requests of unequal size overlap on the device.
// A request's latency is its completion time minus its arrival time (the
// time it was submitted, or its scheduled time in a replayed trace).
// shape_server_run replays a trace through the same scheduler: the calling
// thread submits each request at its arrival time and waits for the last.
#include <algorithm>
#include <chrono>
#include <condition_variable>
#include <deque>
#include <memory>
#include <mutex>
#include <thread>
#include <vector>

#include "engine_impl.h"

namespace shape {

struct Instance {
    std::unique_ptr<EngineImpl> eng;
    int id = 0;                          // stable number, in creation order
    int workload = -1;
    int busy = 0;
    long long request = -1;
    double last_used = 0.0;
};

struct Workload {
    std::unique_ptr<EngineImpl> proto;   // host description (never finalized)
    int form = SHAPE_FORM_BATCHED_FP32;
    size_t footprint = 0;                // device bytes of one instance
    int frames = 0;                      // frame-evals per request
};

// One submitted request.
struct Req {
    int workload = -1;
    double scale[3] = {1.0, 1.0, 1.0};
    double t_arrival = 0.0;              // server clock (seconds since create)
    int state = 0;                       // 0 waiting, 1 running, 2 done
    shape_request_result res{};
};

// Older waiting requests than this stop later ones from taking new memory.
constexpr double STARVE_S = 0.02;

struct ServerImpl {
    int device = 0;
    size_t budget = 0, used = 0, peak_used = 0;
    int max_slots = 8;
    std::vector<Workload> wl;
    std::vector<std::unique_ptr<Instance>> inst;
    int created = 0, evicted = 0;

    // scheduler state, guarded by mu
    std::mutex mu;
    std::condition_variable cv_work, cv_done;
    std::thread th;
    bool thread_on = false, stopping = false;
    std::deque<Req> reqs;                // index = ticket - ticket0
    long long ticket0 = 0;
    std::deque<long long> waiting;       // tickets, oldest first
    std::vector<Instance *> active;
    int err = SHAPE_OK;
    std::string errmsg;
    // statistics since the last reset
    double conc_integral = 0.0, t_prev = 0.0;
    int peak_conc = 0, created_mark = 0, evicted_mark = 0;
    long long frames_done = 0, stat_first = 0;
    double stat_t0 = 0.0;                // start of the statistics window

    std::chrono::steady_clock::time_point epoch = std::chrono::steady_clock::now();
    double now() const { return std::chrono::duration<double>(std::chrono::steady_clock::now() - epoch).count(); }

    ~ServerImpl() { stop(); }

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

    // Would evictions of idle instances of other workloads make room?
    bool room_possible(int w, size_t need) const
    {
        size_t freeable = 0;
        for (auto &I : inst)
            if (!I->busy && I->workload != w) freeable += wl[I->workload].footprint;
        return used - std::min(used, freeable) + need <= budget;
    }

    // An idle instance of workload w; with allow_new, one created when the
    // budget allows after evictions. *out = nullptr when none is available.
    int acquire(int w, bool allow_new, Instance **out)
    {
        *out = nullptr;
        for (auto &I : inst)
            if (I->workload == w && !I->busy) { *out = I.get(); return SHAPE_OK; }
        if (!allow_new || !room_possible(w, wl[w].footprint)) return SHAPE_OK;
        make_room(w, wl[w].footprint);
        return make_instance(w, out);
    }

    Req &req(long long t) { return reqs[(size_t)(t - ticket0)]; }

    // One scheduler pass (mu held): completions, then admissions.
    // *progressed tells whether anything changed.
    int step(bool *progressed)
    {
        const double t = now();
        conc_integral += (t - t_prev) * (double)active.size();
        t_prev = t;
        *progressed = false;
        for (size_t k = 0; k < active.size();) {
            Instance *I = active[k];
            int pr = I->eng->poll();
            if (pr < 0) return pr;
            if (pr == 0) { k++; continue; }
            shape_eval_summary sm;
            int rc = I->eng->finish(&sm);
            if (rc) return rc;
            Req &R = req(I->request);
            R.res.chi2 = sm.chi2;
            R.res.objective = sm.objective;
            R.res.t_done = now();
            R.res.latency_s = R.res.t_done - R.t_arrival;
            R.res.device_ms = I->eng->last_ms;
            R.state = 2;
            frames_done += wl[I->workload].frames;
            I->busy = 0;
            I->last_used = R.res.t_done;
            active.erase(active.begin() + k);
            *progressed = true;
        }
        if (*progressed) cv_done.notify_all();
        // admissions: oldest first, skipping requests that cannot start now
        bool allow_new = true;
        for (auto it = waiting.begin(); it != waiting.end() && (int)active.size() < max_slots;) {
            Req &R = req(*it);
            Instance *I = nullptr;
            int rc = acquire(R.workload, allow_new, &I);
            if (rc) return rc;
            if (!I) {
                // the oldest request has starved: keep new memory for it
                if (it == waiting.begin() && t - R.t_arrival > STARVE_S) allow_new = false;
                ++it;
                continue;
            }
            EngineImpl &E = *I->eng;
            for (int j = 0; j < 3; j++) E.scale[j] = R.scale[j];
            R.res.t_start = now();
            R.res.instance = I->id;
            rc = E.launch(wl[R.workload].form);
            if (rc) return rc;
            I->busy = 1;
            I->request = *it;
            R.state = 1;
            active.push_back(I);
            peak_conc = std::max(peak_conc, (int)active.size());
            it = waiting.erase(it);
            *progressed = true;
        }
        return SHAPE_OK;
    }

    void loop()
    {
        cudaSetDevice(device);
        std::unique_lock<std::mutex> lk(mu);
        for (;;) {
            if (stopping && waiting.empty() && active.empty()) break;
            bool progressed = false;
            int rc = step(&progressed);
            if (rc) {
                // a device or engine failure ends the server's work: every
                // request still open reports it
                err = rc;
                errmsg = shape_last_error();
                cv_done.notify_all();
                break;
            }
            if (active.empty() && waiting.empty()) {
                cv_work.wait(lk, [&] { return stopping || !waiting.empty(); });
            } else if (!progressed) {
                // requests in flight: poll again soon, letting submitters in
                lk.unlock();
                std::this_thread::yield();
                lk.lock();
            }
        }
        thread_on = false;
    }

    int start()
    {
        std::lock_guard<std::mutex> lk(mu);
        if (err) return report_error(err, "server: stopped after an error: " + errmsg);
        if (thread_on) return SHAPE_OK;
        if (th.joinable()) th.join();
        stopping = false;
        thread_on = true;
        th = std::thread([this] { loop(); });
        return SHAPE_OK;
    }

    void stop()
    {
        {
            std::lock_guard<std::mutex> lk(mu);
            stopping = true;
        }
        cv_work.notify_all();
        if (th.joinable()) th.join();
    }

    int submit(int w, const double sc[3], double t_arrival, long long *ticket)
    {
        std::lock_guard<std::mutex> lk(mu);
        if (err) return report_error(err, "server: stopped after an error: " + errmsg);
        if (!thread_on || stopping) return report_error(SHAPE_E_STATE, "server_submit: call shape_server_start first");
        if (w < 0 || w >= (int)wl.size()) return report_error(SHAPE_E_ARG, "server_submit: unknown workload");
        Req R;
        R.workload = w;
        for (int j = 0; j < 3; j++) R.scale[j] = sc ? sc[j] : 1.0;
        R.t_arrival = t_arrival < 0 ? now() : t_arrival;
        reqs.push_back(R);
        const long long t = ticket0 + (long long)reqs.size() - 1;
        waiting.push_back(t);
        *ticket = t;
        cv_work.notify_one();
        return SHAPE_OK;
    }

    // 1: done (*out filled), 0: not yet, < 0: error. Waits up to timeout_s
    // seconds (0: does not wait).
    int wait(long long t, double timeout_s, shape_request_result *out)
    {
        std::unique_lock<std::mutex> lk(mu);
        if (t < ticket0 || t >= ticket0 + (long long)reqs.size())
            return report_error(SHAPE_E_ARG, "server_poll: unknown ticket");
        auto ready = [&] { return req(t).state == 2 || err != SHAPE_OK; };
        if (!ready() && timeout_s > 0)
            cv_done.wait_for(lk, std::chrono::duration<double>(timeout_s), ready);
        if (req(t).state == 2) {
            if (out) *out = req(t).res;
            return 1;
        }
        if (err) return report_error(err, "server: stopped after an error: " + errmsg);
        return timeout_s > 0 ? report_error(SHAPE_E_TIMEOUT, "server_wait: request not done in time") : 0;
    }

    // statistics of tickets [first, last) over the window from t_from (mu held)
    void stats_of(long long first, long long last, double t_from, shape_server_stats *st)
    {
        std::vector<double> lat;
        double t_end = t_from;
        for (long long t = first; t < last; t++) {
            const Req &R = req(t);
            if (R.state != 2) continue;
            lat.push_back(R.res.latency_s);
            t_end = std::max(t_end, R.res.t_done);
        }
        std::sort(lat.begin(), lat.end());
        const int n = (int)lat.size();
        auto pct = [&](double p) {
            if (n == 0) return 0.0;
            double pos = p * (n - 1);
            int lo = (int)pos;
            int hi = std::min(lo + 1, n - 1);
            return lat[lo] + (pos - lo) * (lat[hi] - lat[lo]);
        };
        const double span = std::max(t_end - t_from, 1e-12);
        st->span_s = span;
        st->requests_per_s = n / span;
        st->frame_evals_per_s = frames_done / span;
        st->p50_latency_s = pct(0.50);
        st->p99_latency_s = pct(0.99);
        st->mean_concurrency = conc_integral / span;
        st->peak_concurrency = peak_conc;
        st->instances_created = created - created_mark;
        st->instances_evicted = evicted - evicted_mark;
        st->peak_hbm_bytes = (double)peak_used;
    }

    // starts a statistics window at time t (mu held)
    void reset_stats(double t)
    {
        conc_integral = 0.0;
        t_prev = t;
        peak_conc = (int)active.size();
        created_mark = created;
        evicted_mark = evicted;
        frames_done = 0;
        peak_used = used;
        stat_first = ticket0 + (long long)reqs.size();
        stat_t0 = t;
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
    s->impl.stop();
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
    std::lock_guard<std::mutex> lk(S.mu);
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

extern "C" int shape_server_start(shape_server *s)
{
    if (!s) return report_error(SHAPE_E_ARG, "server_start: null argument");
    int rc = s->impl.start();
    if (rc) return rc;
    std::lock_guard<std::mutex> lk(s->impl.mu);
    s->impl.reset_stats(s->impl.now());
    return SHAPE_OK;
}

extern "C" int shape_server_submit(shape_server *s, int workload, const double scale[3], long long *ticket)
{
    if (!s || !ticket) return report_error(SHAPE_E_ARG, "server_submit: null argument");
    return s->impl.submit(workload, scale, -1.0, ticket);
}

extern "C" int shape_server_poll(shape_server *s, long long ticket, shape_request_result *res)
{
    if (!s) return report_error(SHAPE_E_ARG, "server_poll: null argument");
    return s->impl.wait(ticket, 0.0, res);
}

extern "C" int shape_server_wait(shape_server *s, long long ticket, double timeout_s, shape_request_result *res)
{
    if (!s || !(timeout_s > 0)) return report_error(SHAPE_E_ARG, "server_wait: bad argument");
    return s->impl.wait(ticket, timeout_s, res);
}

extern "C" int shape_server_stats_get(shape_server *s, shape_server_stats *stats)
{
    if (!s || !stats) return report_error(SHAPE_E_ARG, "server_stats: null argument");
    ServerImpl &S = s->impl;
    std::lock_guard<std::mutex> lk(S.mu);
    const long long last = S.ticket0 + (long long)S.reqs.size();
    S.stats_of(std::max(S.stat_first, S.ticket0), last, S.stat_t0, stats);
    return SHAPE_OK;
}

extern "C" int shape_server_stop(shape_server *s)
{
    if (!s) return report_error(SHAPE_E_ARG, "server_stop: null argument");
    s->impl.stop();
    std::lock_guard<std::mutex> lk(s->impl.mu);
    if (s->impl.err) return report_error(s->impl.err, "server: stopped after an error: " + s->impl.errmsg);
    return SHAPE_OK;
}

extern "C" int shape_server_run(shape_server *s, const shape_request *req, int n, shape_request_result *res,
                                shape_server_stats *stats)
{
    if (!s || !req || n <= 0 || !res || !stats) return report_error(SHAPE_E_ARG, "server_run: bad argument");
    ServerImpl &S = s->impl;
    for (int i = 0; i < n; i++)
        if (req[i].workload < 0 || req[i].workload >= (int)S.wl.size())
            return report_error(SHAPE_E_ARG, "server_run: unknown workload");
    bool was_on;
    {
        std::lock_guard<std::mutex> lk(S.mu);
        if (!S.waiting.empty() || !S.active.empty())
            return report_error(SHAPE_E_STATE, "server_run: requests of an online session are still open");
        was_on = S.thread_on;
    }
    int rc = S.start();
    if (rc) return rc;
    std::vector<int> order(n);
    for (int i = 0; i < n; i++) order[i] = i;
    std::stable_sort(order.begin(), order.end(),
                     [&](int a, int b) { return req[a].arrival_s < req[b].arrival_s; });
    std::vector<long long> tk(n);
    double t0;
    long long first;
    {
        std::lock_guard<std::mutex> lk(S.mu);
        t0 = S.now();
        S.reset_stats(t0);
        first = S.stat_first;
    }
    // each request is submitted at its arrival time and stamped with it
    for (int k = 0; k < n; k++) {
        const int i = order[k];
        const double due = t0 + req[i].arrival_s;
        const double ahead = due - S.now();
        if (ahead > 2e-4) std::this_thread::sleep_for(std::chrono::duration<double>(ahead - 1e-4));
        while (S.now() < due) std::this_thread::yield();
        rc = S.submit(req[i].workload, req[i].scale, due, &tk[i]);
        if (rc) return rc;
    }
    for (int i = 0; i < n; i++) {
        shape_request_result r;
        rc = S.wait(tk[i], 3600.0, &r);
        if (rc < 0) return rc;
        r.t_start -= t0;
        r.t_done -= t0;
        res[i] = r;
    }
    {
        std::lock_guard<std::mutex> lk(S.mu);
        S.stats_of(first, first + n, t0, stats);
        // finished requests leave the ticket table
        while (!S.reqs.empty() && S.ticket0 < first + n && S.reqs.front().state == 2) {
            S.reqs.pop_front();
            S.ticket0++;
        }
    }
    if (!was_on) S.stop();
    return SHAPE_OK;
}
