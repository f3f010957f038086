"""Benchmark of SHAPE's model-evaluation hot path on B200.

    python bench.py [--gpus N] [--steps K] [--warmup W] [--impl ours|reference]
                    [--workload c2|c1|c3|c4] [--form batched_fp32|batched_fp64|plain_fp64]
                    [--mode eval|sweep] [--no-serve] [--no-cpu-baseline]

One step = one objective evaluation (realize_mod + calc_fits + chi2) of the
workload after a bestfit-style trial change of a model parameter. Default
workload: 64 delay-Doppler frames of uneven size (POS 101-301 px,
64-256 x 64-512 delay-Doppler) of an 8000-facet vertex model, batched FP32
form. Metric: frame-evals/s (one frame-eval = one delay-Doppler frame, or one
lightcurve point, through raster -> synthesis/photometry -> chi-square),
whole job over all ranks. The default run also replays the serving mix
(config 5) through the continuous-batching server (`serving` key).

Workloads: c1 one 100x100 frame of a 2300-facet ellipsoid; c2 the default;
c3 four lightcurves of 200 points (two raster passes per point, shadowing);
c4 16 frames of 511x511 POS / 256x256 delay-Doppler, 32768-facet model.
--mode sweep (c4): one bestfit sweep over vertex-deviation parameters, each
trial a graph replay; reports trials/s.

Multi-GPU (torchrun, one rank per GPU): frames are independent given the
model, so for c2 each rank evaluates its balanced block of a global dataset
of 64 frames per rank (weak scaling), and the per-rank chi-square totals are
summed with one all-reduce of a few doubles per step (the exchange a sharded
fit needs). Other workloads run as replicas.

--impl reference times the reference's own CPU code (oracle/_ref, built from
the reference sources) on the same workload with all host cores, one dataset
shard per thread as the reference's host multithreading does.
"""
import argparse
import json
import math
import os
import statistics
import subprocess
import sys
import threading
import time

REPO = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, REPO)
sys.path.insert(0, os.path.join(REPO, "shape-cuda-v1.2_b200", "python"))

import numpy as np  # noqa: E402

from shape_b200 import synth  # noqa: E402

L2_BYTES = 126 * 1024 * 1024

# vertex-deviation step and tolerances of the config-4 sweep (length_step,
# length_tol, length_abstol of the .par file; km and relative)
SWEEP_STEP, SWEEP_TOL, SWEEP_ABSTOL = 0.01, 1e-3, 1e-5


def workload(name, dd_syn, lc_syn, params):
    """(model, delay-Doppler datasets, lightcurve datasets, description)."""
    if name == "c1":
        m = synth.ellipsoid_model()
        return m, [synth.config1_dataset(dd_syn(m), params)], [], \
            "config 1: one 100x100 delay-Doppler frame, POS 151x151, 2300-facet ellipsoid vertex model"
    if name == "c3":
        m = synth.harmonic_model()
        return m, [], synth.config3_datasets(lc_syn(m), params), \
            ("config 3: 4 lightcurves x 200 points, POS 129-257 px, solar phase 5-60 deg, "
             "Kaasalainen (Lommel-Seeliger 0.7 + Lambert 0.3) law, shadowing; 8000-facet model")
    if name == "c4":
        m = synth.noisy_octa_model()
        return m, [synth.config4_dataset(dd_syn(m), params)], [], \
            "config 4: 16 frames, POS 511x511, 256x256 delay-Doppler, 32768-facet vertex model"
    m = synth.harmonic_model()
    return m, [synth.config2_dataset(dd_syn(m), params)], [], \
        ("config 2: 64 delay-Doppler frames, POS 101-301 px, 64-256 x 64-512 delay-Doppler, "
         "8000-facet vertex model (sphere + degree-8 harmonics, 5% RMS)")


def units(dds, lcs):
    return sum(d.nframes for d in dds) + sum(len(l.points) for l in lcs)


def algorithmic_bytes(model, dds, lcs, s):
    """Bytes per evaluation by the hot-path byte model: element size s (8 FP64,
    4 FP32); obs and 1/var at 8 B each in both forms.
      model:  nv*6s + nf*(12 + 3s)
      frame:  POS  P*(8+s)*2   (depth/facet word + cos(e), written and read once)
              dd   D*(2s+16)   (fit written and read, obs and 1/var read)
      point:  P*(32+4s)        (observer and sun views, mask, photometry)
    Returns (model, POS part, delay-Doppler part, the raster kernel's share)."""
    b_model = model.nv * 6 * s + model.nf * (12 + 3 * s)
    frames = [f for d in dds for f in d.frames]
    pts = [p for l in lcs for p in l.points]
    b_pos = sum((2 * f.pos_n + 1) ** 2 * (8 + s) * 2 for f in frames)
    b_pt = sum((2 * p.pos_n + 1) ** 2 * (32 + 4 * s) for p in pts)
    b_dd = sum(f.ndel * f.ndop * (2 * s + 16) for f in frames)
    # the fused raster reads the model, produces the POS words and cos(e) and
    # writes the fit images; for lightcurves it writes both views' maps (half
    # of the per-point figure; the photometry kernel reads them)
    raster = b_model + b_pos + sum(f.ndel * f.ndop * s for f in frames) + b_pt // 2
    return b_model, b_pos + b_pt, b_dd, raster


class ClockSampler:
    """nvidia-smi clocks / throttle reasons sampled every 100 ms."""
    Q = ("index,clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,"
         "clocks_event_reasons.hw_slowdown,clocks_event_reasons.hw_thermal_slowdown,"
         "clocks_event_reasons.sw_thermal_slowdown,clocks_event_reasons.sw_power_cap")

    def __init__(self, index):
        self.index = index
        self.proc = None
        self.lines = []

    def start(self):
        try:
            self.proc = subprocess.Popen(["nvidia-smi", "-i", str(self.index), "--query-gpu=" + self.Q,
                                          "--format=csv,noheader,nounits", "-lms", "100"],
                                         stdout=subprocess.PIPE, stderr=subprocess.DEVNULL, text=True)
            self.t = threading.Thread(target=self._read, daemon=True)
            self.t.start()
        except OSError:
            self.proc = None

    def _read(self):
        for line in self.proc.stdout:
            self.lines.append(line.strip())

    def stop(self):
        if self.proc:
            self.proc.terminate()
            try:
                self.proc.wait(timeout=5)
            except subprocess.TimeoutExpired:
                self.proc.kill()
        mhz, mx, reasons = [], None, set()
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        for ln in self.lines:
            p = [x.strip() for x in ln.split(",")]
            if len(p) < 9:
                continue
            try:
                mhz.append(float(p[1]))
                mx = float(p[2])
            except ValueError:
                continue
            for k, nm in enumerate(names):
                if p[5 + k].lower() == "active":
                    reasons.add(nm)
        return {"sm_mhz": statistics.median(mhz) if mhz else None, "sm_max_mhz": mx,
                "reasons": sorted(reasons), "samples": len(mhz)}


def dist_setup():
    ws = int(os.environ.get("WORLD_SIZE", "1"))
    if ws <= 1:
        return 0, 1, 0, None
    import torch.distributed as dist
    from datetime import timedelta
    os.environ.setdefault("MASTER_ADDR", "127.0.0.1")
    rank, lrank = int(os.environ["RANK"]), int(os.environ.get("LOCAL_RANK", "0"))
    import torch
    torch.cuda.set_device(lrank)
    dist.init_process_group("nccl", timeout=timedelta(seconds=120),
                            device_id=torch.device("cuda", lrank))
    return rank, ws, lrank, dist


def peak_hbm():
    try:
        peaks = json.load(open(os.path.join(REPO, "MEASURED_PEAKS.json")))
        return float(peaks["hbm_gbs"]), "measured"
    except Exception:
        return 6650.0, "fallback"


# ------------------------------------------------------------ reference arm

def ref_sessions(ref, model, params, dds, lcs, nthreads):
    """The workload split the way the reference's host multithreading splits
    it (one dataset per thread): frames of a delay-Doppler set in contiguous
    shards, lightcurve sets one per session."""
    sessions = []
    for ds in dds:
        shards = np.array_split(np.arange(ds.nframes), max(1, min(nthreads, ds.nframes)))
        for sh in shards:
            sub = synth.DeldopDataset(ds.set, [ds.frames[i] for i in sh],
                                      np.concatenate([ds.frame_obs(i) for i in sh]),
                                      np.concatenate([ds.oneovervar[ds.offsets[i]:ds.offsets[i + 1]]
                                                      for i in sh]), None)
            sub.offsets = np.concatenate([[0], np.cumsum([ds.frames[i].ndel * ds.frames[i].ndop
                                                          for i in sh])])
            sessions.append(ref.session(model, params, deldops=[sub]))
    for ls in lcs:
        sessions.append(ref.session(model, params, lghtcrvs=[ls]))
    return sessions


def ref_synthesizers(ref):
    def dd(model):
        def f(ds, p):
            S = ref.session(model, p, deldops=[ds])
            S.evaluate()
            out = [S.deldop_frame(0, k, fr)["fit"] for k, fr in enumerate(ds.frames)]
            S.close()
            return out
        return f

    def lc(model):
        def f(ds, p):
            S = ref.session(model, p, lghtcrvs=[ds])
            S.evaluate()
            y = S.lghtcrv(0, ds)["y"]
            S.close()
            return y
        return f
    return dd, lc


def run_reference(args, rank, ws):
    if rank != 0:
        return 0
    import ctypes as C
    from oracle.bindings import Reference
    ref = Reference()
    params = synth.eval_params()
    dd_syn, lc_syn = ref_synthesizers(ref)
    model, dds, lcs, desc = workload(args.workload, dd_syn, lc_syn, params)
    nu = units(dds, lcs)
    cores = os.cpu_count() or 1
    sessions = ref_sessions(ref, model, params, dds, lcs, cores)
    arr = (C.c_void_p * len(sessions))(*[s.h for s in sessions])
    for _ in range(args.warmup):
        ref.lib.ref_evaluate_mt(arr, len(sessions))
    times = []
    for _ in range(args.steps):
        t0 = time.perf_counter()
        ref.lib.ref_evaluate_mt(arr, len(sessions))
        times.append(time.perf_counter() - t0)
    ms = 1e3 * statistics.mean(times)
    value = nu / (ms / 1e3)
    threads = min(cores, len(sessions))
    line = {
        "impl": "reference", "metric": "frame-evals/sec", "value": value, "unit": "frame-evals/s",
        "n_gpus": ws, "steps": args.steps, "warmup": args.warmup, "ms_per_step": ms,
        "higher_is_better": True, "scaling": "weak", "vs_baseline": None, "dtype": "f64",
        "data": "synthetic",
        "config": {"workload": desc, "form": "reference CPU (calc_fits + chi2 per step)",
                   "threads": threads, "sessions": len(sessions), "frame_evals_per_step": nu},
        "cpu_baseline": {"value": value, "unit": "frame-evals/s", "cores": threads, "kind": "reference",
                         "sample": "%d full evaluations of the %d-unit workload" % (args.steps, nu)},
        "e2e": {"value": value, "unit": "frame-evals/s", "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0},
        "p50_ms": 1e3 * statistics.median(times), "p99_ms": 1e3 * float(np.percentile(times, 99)),
    }
    for s in sessions:
        s.close()
    print(json.dumps(line), flush=True)
    return 0


def cpu_baseline(model, dds, lcs, params, budget_s=15.0):
    """Reference CPU code (oracle/_ref) on the host cores, bounded sample:
    all cores with one dataset shard per thread, then a single thread."""
    try:
        from oracle.bindings import Reference
        ref = Reference()
    except Exception as exc:  # pragma: no cover
        return {"value": None, "unit": "frame-evals/s", "cores": 0, "kind": "reference",
                "sample": "unavailable: %s" % exc}
    import ctypes as C
    nu = units(dds, lcs)
    cores = os.cpu_count() or 1
    sessions = ref_sessions(ref, model, params, dds, lcs, cores)
    arr = (C.c_void_p * len(sessions))(*[s.h for s in sessions])
    ref.lib.ref_evaluate_mt(arr, len(sessions))
    reps, t_all = 0, 0.0
    while t_all < budget_s and reps < 50:
        t0 = time.perf_counter()
        ref.lib.ref_evaluate_mt(arr, len(sessions))
        t_all += time.perf_counter() - t0
        reps += 1
    S1 = ref.session(model, params, deldops=dds, lghtcrvs=lcs)
    S1.evaluate()
    r1, t1 = 0, 0.0
    while t1 < budget_s / 3 and r1 < 20:
        t0 = time.perf_counter()
        S1.evaluate()
        t1 += time.perf_counter() - t0
        r1 += 1
    S1.close()
    for s in sessions:
        s.close()
    threads = min(cores, len(sessions))
    return {"value": nu * reps / t_all, "unit": "frame-evals/s", "cores": threads, "kind": "reference",
            "sample": "%d evaluations of the %d-unit workload on %d threads (one dataset shard per thread)"
                      % (reps, nu, threads),
            "single_thread_value": nu * r1 / t1}


# ----------------------------------------------------------------- our arm

def serving_bench(lrank, nreq=4000, rate=2000.0, budget=64 << 30, slots=16):
    """The serving mix: a seeded Poisson stream of `rate` requests/s over the
    config-1..4 workloads (one workload per frame count), replayed through
    the continuous-batching server in the batched FP32 and FP64 forms. A first
    pass of the trace warms the instances; the second is reported. The
    offered rate saturates the GPU, so a second trace at 60% of the FP32
    form's served rate gives the latencies of an unsaturated server."""
    from shape_b200 import engine as eng
    params = synth.eval_params()
    cats, work = synth.serving_mix(lambda m: eng.engine_synthesizer(m, lrank)[0],
                                   lambda m: eng.engine_synthesizer(m, lrank)[1], params)
    trace = synth.serving_trace(cats, nreq, rate, seed=2026)
    cat_of = {}
    for c, ws_ in zip(("c1", "c2", "c3", "c4"), cats):
        for w in ws_:
            cat_of[w] = c
    out, chi = {}, {}
    sus_rate = None

    def stats(st):
        return {"frame_evals_per_s": st["frame_evals_per_s"], "requests_per_s": st["requests_per_s"],
                "p50_latency_ms": 1e3 * st["p50_latency_s"], "p99_latency_ms": 1e3 * st["p99_latency_s"],
                "mean_concurrency": st["mean_concurrency"], "peak_concurrency": st["peak_concurrency"],
                "instances_created_in_run": st["instances_created"],
                "instances_evicted_in_run": st["instances_evicted"],
                "peak_hbm_gb": st["peak_hbm_bytes"] / 1e9}

    # the step byte model of each workload (bytes per request, by form): the
    # served requests' bytes over the run's time give the serving mix's
    # achieved bandwidth beside the measured HBM peak
    peak, _ = peak_hbm()

    def req_bytes(s_elem):
        out_b = []
        for (_, m, dd_, lc_) in work:
            bm, bp, bd, _ = algorithmic_bytes(m, dd_, lc_, s_elem)
            out_b.append(bm + bp + bd)
        return out_b

    for name, form in (("fp32", eng.FORM_BATCHED_FP32), ("fp64", eng.FORM_BATCHED_FP64)):
        wbytes = req_bytes(4 if name == "fp32" else 8)
        srv = eng.Server(lrank, budget, slots)
        t0 = time.perf_counter()
        eng.register_workloads(srv, work, params, form, lrank)
        t_reg = time.perf_counter() - t0
        srv.run(trace)
        res, st = srv.run(trace)
        chi[name] = np.array([r["chi2"] for r in res])
        out[name] = {"offered": stats(st), "registration_s": t_reg}
        mean_b = float(np.mean([wbytes[w] for (w, _, _) in trace]))
        gbs = mean_b * st["requests_per_s"] / 1e9
        out[name]["offered"]["roofline"] = {"bound": "hbm", "achieved_gbs": gbs, "peak_gbs": peak,
                                            "frac": gbs / peak, "bytes_per_request": mean_b}
        if sus_rate is None:
            sus_rate = 0.6 * st["requests_per_s"]
        tr2 = synth.serving_trace(cats, int(sus_rate * 3.0), sus_rate, seed=2027)
        srv.run(tr2[: min(len(tr2), 200)])
        _, st2 = srv.run(tr2)
        out[name]["sustainable"] = stats(st2)
        srv.close()
    out["workloads"] = len(work)
    out["requests"] = nreq
    out["offered_rate_req_per_s"] = rate
    out["sustainable_rate_req_per_s"] = sus_rate
    out["max_slots"], out["hbm_budget_gb"] = slots, budget / 1e9
    rel = np.abs(chi["fp32"] - chi["fp64"]) / np.abs(chi["fp64"])
    out["max_dchi2_rel_fp32_vs_fp64"] = {c: float(max([rel[i] for i, (w, _, _) in enumerate(trace)
                                                       if cat_of[w] == c] or [0.0]))
                                         for c in ("c1", "c2", "c3", "c4")}
    return out


def sweep_bench(args, lrank):
    """Config 4: one bestfit sweep over the first args.params vertex-deviation
    parameters (each trial a graph replay), and the reference CPU code on the
    first few parameters of the same sweep."""
    from shape_b200 import engine as eng
    params = synth.eval_params()
    dd_syn = lambda m: eng.engine_synthesizer(m, lrank)[0]
    model, dds, lcs, desc = workload("c4", dd_syn, None, params)
    form = eng.FORMS[args.form]
    E = eng.make_engine(model, params, deldops=dds, device=lrank)
    E.evaluate(form)
    fit_params = [(eng.PAR_VERTEX_R, i, SWEEP_STEP, SWEEP_TOL, SWEEP_ABSTOL) for i in range(args.params)]
    clocks = ClockSampler(lrank)
    clocks.start()
    t0 = time.perf_counter()
    res, _ = E.bestfit(fit_params, form=form, term_prec=1e-4, term_maxiter=1)
    dt = time.perf_counter() - t0
    clk = clocks.stop()
    E.close()
    nfr = dds[0].nframes
    line = {
        "metric": "vertex-sweep trials/sec", "value": res["evaluations"] / dt, "unit": "trials/s",
        "n_gpus": 1, "higher_is_better": True, "dtype": "f32" if form == eng.FORM_BATCHED_FP32 else "f64",
        "data": "synthetic",
        "config": {"workload": desc + "; one bestfit sweep over %d vertex deviations" % args.params,
                   "form": args.form, "step_tol_abstol": [SWEEP_STEP, SWEEP_TOL, SWEEP_ABSTOL]},
        "trials": res["evaluations"], "seconds": dt, "ms_per_trial": 1e3 * dt / res["evaluations"],
        "frame_evals_per_s": res["evaluations"] * nfr / dt,
        "objective": [res["initial_objective"], res["final_objective"]],
        "clocks": clk,
    }
    if not args.no_cpu_baseline:
        line["cpu_baseline"] = sweep_cpu(model, dds, params, k=5)
    print(json.dumps(line), flush=True)
    return 0


def sweep_cpu(model, dds, params, k=5):
    """The same sweep on the reference CPU code for the first k parameters
    (host bestfit loop over the reference's realize_mod + calc_fits + chi2,
    all cores, one frame shard per thread)."""
    import ctypes as C
    from oracle.bindings import Reference
    from shape_b200 import engine as eng
    ref = Reference()
    sessions = ref_sessions(ref, model, params, dds, [], os.cpu_count() or 1)
    arr = (C.c_void_p * len(sessions))(*[s.h for s in sessions])
    dof = sum(f.dof for f in dds[0].frames)
    vals = np.array([model.r[i] for i in range(k)], dtype=np.float64)
    count = [0]

    def objective(v):
        for i in range(k):
            for s in sessions:
                ref.lib.ref_set_r(s.h, i, float(v[i]))
        chi2 = ref.lib.ref_evaluate_mt(arr, len(sessions))
        count[0] += 1
        return chi2 / dof, 0, 0
    fit_params = [(eng.PAR_VERTEX_R, i, SWEEP_STEP, SWEEP_TOL, SWEEP_ABSTOL) for i in range(k)]
    t0 = time.perf_counter()
    eng.bestfit_host(objective, vals, fit_params, term_prec=1e-4, term_maxiter=1)
    dt = time.perf_counter() - t0
    for s in sessions:
        s.close()
    return {"value": count[0] / dt, "unit": "trials/s", "cores": min(os.cpu_count() or 1, len(sessions)),
            "kind": "reference", "sample": "first %d parameters of the sweep: %d trials" % (k, count[0])}


def per_config(lrank, flush, budget_cpu_s=3.0):
    """Configs 1 and 3 (one evaluation per step) and config 4 (a short
    vertex sweep, each trial a graph replay) beside the config-2 headline:
    batched FP32 frame-evals/s (CUDA events, L2 flushed before each step),
    the raster kernel's roofline fraction, the FP32 form's worst
    delta-chi2/chi2 against the FP64 form over jittered trials, and the
    reference CPU code's rate on a bounded sample of the same workload."""
    import torch
    from shape_b200 import engine as eng
    peak, _ = peak_hbm()
    out = {}
    dd_syn = lambda m: eng.engine_synthesizer(m, lrank)[0]
    lc_syn = lambda m: eng.engine_synthesizer(m, lrank)[1]
    for name, steps in (("c1", 200), ("c3", 20), ("c4", 40)):
        params = synth.eval_params()
        model, dds, lcs, desc = workload(name, dd_syn, lc_syn, params)
        nu = units(dds, lcs)
        E = eng.make_engine(model, params, deldops=dds, lghtcrvs=lcs, device=lrank)
        rng = np.random.default_rng(17)
        worst = worst_frame = 0.0
        for k in range(4):
            sc = [1.0, 1.0, 1.0] if k == 0 else list(1.0 + 0.02 * rng.uniform(-1, 1, 3))
            for j in range(3):
                E.set_scale(j, sc[j])
            c64 = E.evaluate(eng.FORM_BATCHED_FP64)["chi2"]
            r64 = E.results() if dds else []
            c32 = E.evaluate(eng.FORM_BATCHED_FP32)["chi2"]
            r32 = E.results() if dds else []
            worst = max(worst, abs(c32 - c64) / abs(c64))
            for a, b in zip(r64, r32):
                if a["chi2"] != 0.0:
                    worst_frame = max(worst_frame, abs(b["chi2"] - a["chi2"]) / abs(a["chi2"]))
        for j in range(3):
            E.set_scale(j, 1.0)
        for k in range(3):
            E.evaluate(eng.FORM_BATCHED_FP32)
        dev = []
        for k in range(steps):
            flush.zero_()
            torch.cuda.synchronize()
            E.set_scale(0, 1.0 + 1e-3 * math.sin(0.7 * k))
            E.evaluate(eng.FORM_BATCHED_FP32)
            dev.append(E.last_ms())
        st = E.stage_times(eng.FORM_BATCHED_FP32)
        E.close()
        _, _, _, rs_bytes = algorithmic_bytes(model, dds, lcs, 4)
        rs_ms = st.get("raster_synth", float("nan"))
        ms = statistics.mean(dev)
        cpu = cpu_baseline(model, dds, lcs, params, budget_s=budget_cpu_s)
        out[name] = {"workload": desc, "frame_evals_per_s": nu / (ms / 1e3), "ms_per_step": ms,
                     "p50_ms": statistics.median(dev), "p99_ms": float(np.percentile(dev, 99)),
                     "raster_ms": rs_ms, "roofline_frac": rs_bytes / (rs_ms / 1e3) / 1e9 / peak,
                     "max_dchi2_rel_fp32_vs_fp64": worst,
                     "max_dchi2_rel_per_frame_fp32_vs_fp64": worst_frame if dds else None,
                     "cpu_reference_frame_evals_per_s": cpu["value"], "cpu_cores": cpu["cores"]}
    # config 4: the vertex-deviation sweep over its first parameters
    params = synth.eval_params()
    model, dds, lcs, desc = workload("c4", dd_syn, None, params)
    E = eng.make_engine(model, params, deldops=dds, device=lrank)
    E.evaluate(eng.FORM_BATCHED_FP32)
    npar = 100
    fit_params = [(eng.PAR_VERTEX_R, i, SWEEP_STEP, SWEEP_TOL, SWEEP_ABSTOL) for i in range(npar)]
    t0 = time.perf_counter()
    res, _ = E.bestfit(fit_params, form=eng.FORM_BATCHED_FP32, term_prec=1e-4, term_maxiter=1)
    dt = time.perf_counter() - t0
    E.close()
    cpu = sweep_cpu(model, dds, params, k=2)
    out["c4_sweep"] = {"workload": desc + "; one bestfit sweep over the first %d vertex deviations" % npar,
                       "trials_per_s": res["evaluations"] / dt, "trials": res["evaluations"],
                       "frame_evals_per_s": res["evaluations"] * dds[0].nframes / dt,
                       "cpu_reference_trials_per_s": cpu["value"], "cpu_sample": cpu["sample"],
                       "cpu_cores": cpu["cores"]}
    return out


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=600)
    ap.add_argument("--warmup", type=int, default=5)
    ap.add_argument("--impl", default="ours", choices=["ours", "reference"])
    ap.add_argument("--workload", default="c2", choices=["c1", "c2", "c3", "c4"])
    ap.add_argument("--form", default="batched_fp32", choices=["batched_fp32", "batched_fp64", "plain_fp64"])
    ap.add_argument("--mode", default="eval", choices=["eval", "sweep"])
    ap.add_argument("--params", type=int, default=2000, help="vertex parameters of the sweep mode")
    ap.add_argument("--no-cpu-baseline", action="store_true")
    ap.add_argument("--no-serve", action="store_true", help="skip the serving-mix measurement")
    ap.add_argument("--no-per-config", action="store_true", help="skip the configs 1, 3, 4 block")
    ap.add_argument("--raster-tuning", type=int, default=-1, choices=[-1, 0, 1],
                    help="-1: autotune the raster kernel; 0 / 1: the tile-per-CTA / warp kernel (profiling)")
    ap.add_argument("--no-plain", action="store_true", help="skip the plain FP64 comparison run (profiling)")
    args = ap.parse_args()
    args.warmup = max(args.warmup, 3)
    rank, ws, lrank, dist = dist_setup()
    if args.impl == "reference":
        rc = run_reference(args, rank, ws)
        if dist:
            dist.destroy_process_group()
        return rc

    import torch
    from shape_b200 import engine as eng
    torch.cuda.set_device(lrank)
    if args.mode == "sweep":
        return sweep_bench(args, lrank)
    params = synth.eval_params()
    dd_syn = lambda m: eng.engine_synthesizer(m, lrank)[0]
    lc_syn = lambda m: eng.engine_synthesizer(m, lrank)[1]
    model, dds, lcs, desc = workload(args.workload, dd_syn, lc_syn, params)
    if ws > 1 and args.workload == "c2":
        # weak scaling: a global dataset of 64 frames per rank with the
        # config-2 distributions, each rank evaluating its balanced block
        from shape_b200 import shard
        glob = synth.batched_dataset(64 * ws, (101, 301), (64, 256), (64, 512), dd_syn(model), params,
                                     seed=7)
        dds = [shard.shard_dataset(glob, rank, ws)[0]]
        desc += "; %d frames in all, frame blocks balanced by POS + delay-Doppler pixels" % (64 * ws)
    E = eng.make_engine(model, params, deldops=dds, lghtcrvs=lcs, device=lrank)
    E.set_raster_tuning(args.raster_tuning)
    form = eng.FORMS[args.form]
    nu = units(dds, lcs)
    flush = torch.empty(2 * L2_BYTES, dtype=torch.uint8, device="cuda")
    trial = lambda k: 1.0 + 1e-3 * math.sin(0.7 * k)

    # accuracy of the batched FP32 form against FP64 on the same trial model
    E.set_scale(0, trial(0))
    chi64 = E.evaluate(eng.FORM_BATCHED_FP64)["chi2"]
    r64 = E.results() if dds else []
    chi32 = E.evaluate(eng.FORM_BATCHED_FP32)["chi2"]
    r32 = E.results() if dds else []
    dchi = abs(chi32 - chi64) / abs(chi64)
    # the same error frame by frame (each frame's chi-square, FP32 against FP64)
    per_frame = [abs(b["chi2"] - a["chi2"]) / abs(a["chi2"]) for a, b in zip(r64, r32) if a["chi2"] != 0.0]
    dchi_frames = ({"frames": len(per_frame), "max": max(per_frame), "median": statistics.median(per_frame)}
                   if per_frame else None)

    ev_a = torch.cuda.Event(enable_timing=True)
    ev_b = torch.cuda.Event(enable_timing=True)

    def run(form_id, steps, warm, record):
        dev_ms, host_ms = [], []
        for k in range(warm):
            E.set_scale(0, trial(k))
            E.evaluate(form_id)
        if dist:
            dist.barrier()
        torch.cuda.synchronize()
        for k in range(steps):
            flush.zero_()
            torch.cuda.synchronize()
            t0 = time.perf_counter()
            E.set_scale(0, trial(k + warm))
            summ = E.evaluate(form_id)
            step_ms = E.last_ms()
            if dist and record:
                # the step's one exchange: the sum of the ranks' chi-square totals
                from shape_b200 import shard
                ev_a.record()
                shard.allreduce_summary(summ, dist, device="cuda")
                ev_b.record()
                ev_b.synchronize()
                step_ms += ev_a.elapsed_time(ev_b)
            host_ms.append(1e3 * (time.perf_counter() - t0))
            dev_ms.append(step_ms)
        if dist:
            dist.barrier()
        torch.cuda.synchronize()
        return dev_ms, host_ms

    # plain FP64 GPU path (the metric's comparison point), a few steps
    plain_dev = [float("nan")] if args.no_plain else run(eng.FORM_PLAIN_FP64, max(3, min(args.steps, 10)), 2, False)[0]
    clocks = ClockSampler(lrank)
    clocks.start()
    time.sleep(0.3)
    dev_ms, host_ms = run(form, args.steps, args.warmup, True)
    clk = clocks.stop()
    kpe = E.kernels_per_eval(form)
    stages = E.stage_times(form if form != eng.FORM_PLAIN_FP64 else eng.FORM_BATCHED_FP64)

    # the FP32 form with shape_engine_set_fp32_exact(0) (radar views keep
    # their FP32 coverage decisions), a short run beside the default
    fast = None
    if form == eng.FORM_BATCHED_FP32 and not lcs and not args.no_plain:
        E.set_fp32_exact(False)
        fx_ms, _ = run(form, max(20, min(args.steps, 100)), 3, False)
        E.set_scale(0, trial(0))           # both forms at the same scale factors
        c64 = E.evaluate(eng.FORM_BATCHED_FP64)["chi2"]
        c32f = E.evaluate(form)["chi2"]
        E.set_fp32_exact(True)
        fast = {"frame_evals_per_s": nu / (statistics.mean(fx_ms) / 1e3), "ms_per_step": statistics.mean(fx_ms),
                "dchi2_rel_fp32_vs_fp64": abs(c32f - c64) / abs(c64)}

    total_dev = sum(dev_ms)
    total_host = sum(host_ms)
    units_all = ws * nu
    if dist:
        t = torch.tensor([total_dev, total_host], dtype=torch.float64, device="cuda")
        dist.all_reduce(t, op=dist.ReduceOp.MAX)
        total_dev, total_host = t.tolist()
        t = torch.tensor([float(nu)], dtype=torch.float64, device="cuda")
        dist.all_reduce(t)
        units_all = int(t.item())
    ms_step = total_dev / args.steps
    value = units_all / (ms_step / 1e3)
    e2e = units_all / (total_host / args.steps / 1e3)
    plain_rate = nu / (statistics.mean(plain_dev) / 1e3)

    s_elem = 4 if form == eng.FORM_BATCHED_FP32 else 8
    b_model, b_pos, b_dd, rs_bytes = algorithmic_bytes(model, dds, lcs, s_elem)
    peak, peak_src = peak_hbm()
    # dominant kernel: the fused tile raster (+ delay-Doppler synthesis)
    rs_ms = stages.get("raster_synth", float("nan"))
    achieved = rs_bytes / (rs_ms / 1e3) / 1e9
    # DRAM traffic and issue-slot use of this kernel cannot be read inside
    # the run: they come from the ncu capture summarized in profiles/ (its
    # command and build named there), per launch of the same workload
    traffic, issue, prof_src = None, None, None
    traffic_path = os.path.join(REPO, "profiles", "raster_traffic.json")
    if os.path.exists(traffic_path):
        try:
            rec = json.load(open(traffic_path)).get(args.workload + "_" + args.form) or {}
            traffic, issue, prof_src = rec.get("dram_bytes"), rec.get("issue_active_pct"), rec.get("source")
        except Exception:
            traffic = None
    step_bytes = b_model + b_pos + b_dd
    line = {
        "metric": "frame-evals/sec", "value": value, "unit": "frame-evals/s", "n_gpus": ws,
        "steps": args.steps, "warmup": args.warmup, "ms_per_step": ms_step,
        "higher_is_better": True, "scaling": "weak", "vs_baseline": None,
        "dtype": "f32" if form == eng.FORM_BATCHED_FP32 else "f64", "data": "synthetic",
        "config": {"workload": desc, "form": args.form, "frame_evals_per_gpu": nu,
                   "frame_evals_total": units_all,
                   "model_facets": model.nf, "l2": "flushed (2x L2 buffer written) before every step",
                   "parallelism": "frame shards, one per GPU" if ws > 1 else "single GPU",
                   "dchi2_rel_fp32_vs_fp64": dchi,
                   "dchi2_rel_per_frame_fp32_vs_fp64": dchi_frames,
                   "plain_fp64_frame_evals_per_s": plain_rate,
                   "batched_over_plain_fp64": value / ws / plain_rate,
                   "fp32_fast_option": fast,
                   "p50_ms": statistics.median(dev_ms), "p99_ms": float(np.percentile(dev_ms, 99)),
                   "stage_ms": stages,
                   "step_algorithmic_bytes": step_bytes,
                   "step_achieved_gbs": step_bytes / (ms_step / 1e3) / 1e9},
        "roofline": {"bound": "hbm", "kernel": "k_raster (tile raster + delay-Doppler synthesis)",
                     "achieved": achieved, "peak": peak, "unit": "GB/s", "frac": achieved / peak,
                     "peak_source": peak_src, "traffic": traffic, "traffic_source": prof_src,
                     "issue_active_pct": issue,
                     "algorithmic_bytes_per_launch": rs_bytes},
        "e2e": {"value": e2e, "unit": "frame-evals/s", "h2d_bytes_per_step": 8 * (model.nv + 3),
                "d2h_bytes_per_step": 72,
                "what": "shape_engine_evaluate through the C ABI per bestfit trial: model parameters "
                        "host->device, chi-square summary device->host, host wall clock"},
        "gpu_launches": kpe * args.steps,
        "clocks": clk,
    }
    E.close()
    if rank == 0 and ws == 1 and not args.no_cpu_baseline:
        line["cpu_baseline"] = cpu_baseline(model, dds, lcs, params)
    if ws == 1 and not args.no_per_config and args.workload == "c2":
        line["per_config"] = per_config(lrank, flush)
    if ws == 1 and not args.no_serve and args.workload == "c2":
        line["serving"] = serving_bench(lrank)
    if dist:
        dist.destroy_process_group()
    if rank == 0:
        print(json.dumps(line), flush=True)
    return 0


def _json_stdout():
    """Keeps stdout for the JSON line: the reference's C code prints per-point
    lines to fd 1 (chi2_lghtcrv, src/shape/chi2.c:1147), so fd 1 is pointed
    at stderr and Python's stdout writes to a copy of the original fd 1."""
    real = os.dup(1)
    sys.stdout.flush()
    os.dup2(2, 1)
    sys.stdout = os.fdopen(real, "w", buffering=1)


if __name__ == "__main__":
    _json_stdout()
    sys.exit(main())
