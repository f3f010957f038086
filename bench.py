"""Benchmark of SHAPE's model-evaluation hot path on B200.

    python bench.py [--gpus N] [--steps K] [--warmup W] [--impl ours|reference]
                    [--workload c2|c1|c4] [--form batched_fp32|batched_fp64|plain_fp64]

One step = one objective evaluation (realize_mod + calc_fits + chi2) of the
workload after a bestfit-style trial change of a model parameter. Default
workload: 64 delay-Doppler frames of uneven size (POS 101-301 px,
64-256 x 64-512 delay-Doppler) of an 8000-facet vertex model, batched FP32
form. Metric: frame-evals/s (one frame-eval = one delay-Doppler frame through
raster -> synthesis -> chi-square), whole job over all ranks.

Multi-GPU (torchrun, one rank per GPU): frames are independent given the
model, so each rank evaluates its own 64-frame shard (weak scaling) and the
per-rank chi-square totals are summed with one all-reduce of a few doubles
per step (the exchange a sharded fit needs).

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


def workload(name, synthesize, params):
    if name == "c1":
        m = synth.ellipsoid_model()
        ds = synth.config1_dataset(synthesize(m), params)
        desc = "config 1: one 100x100 delay-Doppler frame, POS 151x151, 2300-facet ellipsoid vertex model"
    elif name == "c4":
        m = synth.noisy_octa_model()
        ds = synth.config4_dataset(synthesize(m), params)
        desc = "config 4: 16 frames, POS 511x511, 256x256 delay-Doppler, 32768-facet vertex model"
    else:
        m = synth.harmonic_model()
        ds = synth.config2_dataset(synthesize(m), params)
        desc = ("config 2: 64 delay-Doppler frames, POS 101-301 px, 64-256 x 64-512 delay-Doppler, "
                "8000-facet vertex model (sphere + degree-8 harmonics, 5% RMS)")
    return m, ds, desc


def algorithmic_bytes(model, ds, s):
    """Bytes per evaluation by the hot-path byte model: element size s (8 FP64,
    4 FP32); obs and 1/var at 8 B each in both forms.
      model:  nv*6s + nf*(12 + 3s)
      frame:  POS  P*(8+s)*2   (depth/facet word + cos(e), written and read once)
              dd   D*(2s+16)   (fit written and read, obs and 1/var read)"""
    b_model = model.nv * 6 * s + model.nf * (12 + 3 * s)
    b_pos = sum((2 * f.pos_n + 1) ** 2 * (8 + s) * 2 for f in ds.frames)
    b_dd = sum(f.ndel * f.ndop * (2 * s + 16) for f in ds.frames)
    return b_model, b_pos, b_dd


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
    backend = "nccl"
    import torch
    torch.cuda.set_device(lrank)
    dist.init_process_group(backend, timeout=timedelta(seconds=120),
                            device_id=torch.device("cuda", lrank))
    return rank, ws, lrank, dist


# ------------------------------------------------------------ reference arm

def run_reference(args, rank, ws):
    if rank != 0:
        return 0
    from oracle.bindings import Reference
    ref = Reference()
    params = synth.eval_params()

    def ref_synth(model):
        def f(ds, p):
            S = ref.session(model, p, deldops=[ds])
            S.evaluate()
            out = [S.deldop_frame(0, k, fr)["fit"] for k, fr in enumerate(ds.frames)]
            S.close()
            return out
        return f
    model, ds, desc = workload(args.workload, ref_synth, params)
    cores = os.cpu_count() or 1
    nthreads = min(cores, ds.nframes)
    # one dataset shard per thread (host multithreading: one set per thread)
    shards = np.array_split(np.arange(ds.nframes), nthreads)
    sessions = []
    for sh in shards:
        sub = synth.DeldopDataset(ds.set, [ds.frames[i] for i in sh],
                                  np.concatenate([ds.frame_obs(i) for i in sh]),
                                  np.concatenate([ds.oneovervar[ds.offsets[i]:ds.offsets[i + 1]] for i in sh]),
                                  None)
        sub.offsets = np.concatenate([[0], np.cumsum([ds.frames[i].ndel * ds.frames[i].ndop for i in sh])])
        sessions.append(ref.session(model, params, deldops=[sub]))
    import ctypes as C
    arr = (C.c_void_p * len(sessions))(*[s.h for s in sessions])
    for _ in range(args.warmup):
        ref.lib.ref_evaluate_mt(arr, len(sessions))
    times = []
    for _ in range(args.steps):
        t0 = time.perf_counter()
        ref.lib.ref_evaluate_mt(arr, len(sessions))
        times.append(time.perf_counter() - t0)
    ms = 1e3 * statistics.mean(times)
    value = ds.nframes / (ms / 1e3)
    line = {
        "impl": "reference", "metric": "frame-evals/sec", "value": value, "unit": "frame-evals/s",
        "n_gpus": ws, "steps": args.steps, "warmup": args.warmup, "ms_per_step": ms,
        "higher_is_better": True, "scaling": "weak", "vs_baseline": None, "dtype": "f64",
        "data": "synthetic",
        "config": {"workload": desc, "form": "reference CPU (calc_fits + chi2 per step)",
                   "threads": nthreads, "frames": ds.nframes},
        "cpu_baseline": {"value": value, "unit": "frame-evals/s", "cores": nthreads, "kind": "reference",
                         "sample": "%d full evaluations of the %d-frame workload" % (args.steps, ds.nframes)},
        "e2e": {"value": value, "unit": "frame-evals/s", "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0},
        "p50_ms": 1e3 * statistics.median(times), "p99_ms": 1e3 * float(np.percentile(times, 99)),
    }
    for s in sessions:
        s.close()
    print(json.dumps(line), flush=True)
    return 0


def cpu_baseline(model, ds, params, budget_s=15.0):
    """Reference CPU code (oracle/_ref) on the host cores, bounded sample:
    single-thread frames, then all cores with one frame shard per thread."""
    try:
        from oracle.bindings import Reference
        ref = Reference()
    except Exception as exc:  # pragma: no cover
        return {"value": None, "unit": "frame-evals/s", "cores": 0, "kind": "reference",
                "sample": "unavailable: %s" % exc}
    import ctypes as C
    cores = os.cpu_count() or 1
    nthreads = min(cores, ds.nframes)
    shards = np.array_split(np.arange(ds.nframes), nthreads)
    sessions = []
    for sh in shards:
        sub = synth.DeldopDataset(ds.set, [ds.frames[i] for i in sh],
                                  np.concatenate([ds.frame_obs(i) for i in sh]),
                                  np.concatenate([ds.oneovervar[ds.offsets[i]:ds.offsets[i + 1]] for i in sh]),
                                  None)
        sub.offsets = np.concatenate([[0], np.cumsum([ds.frames[i].ndel * ds.frames[i].ndop for i in sh])])
        sessions.append(ref.session(model, params, deldops=[sub]))
    arr = (C.c_void_p * len(sessions))(*[s.h for s in sessions])
    ref.lib.ref_evaluate_mt(arr, len(sessions))
    reps, t_all = 0, 0.0
    while t_all < budget_s and reps < 50:
        t0 = time.perf_counter()
        ref.lib.ref_evaluate_mt(arr, len(sessions))
        t_all += time.perf_counter() - t0
        reps += 1
    # single thread: one full-workload session, a few evaluations
    S1 = ref.session(model, params, deldops=[ds])
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
    return {"value": ds.nframes * reps / t_all, "unit": "frame-evals/s", "cores": nthreads,
            "kind": "reference",
            "sample": "%d evaluations of the %d-frame workload on %d threads (one frame shard per thread)"
                      % (reps, ds.nframes, nthreads),
            "single_thread_value": ds.nframes * r1 / t1}


# ----------------------------------------------------------------- our arm

def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=600)
    ap.add_argument("--warmup", type=int, default=5)
    ap.add_argument("--impl", default="ours", choices=["ours", "reference"])
    ap.add_argument("--workload", default="c2", choices=["c1", "c2", "c4"])
    ap.add_argument("--form", default="batched_fp32", choices=["batched_fp32", "batched_fp64", "plain_fp64"])
    ap.add_argument("--no-cpu-baseline", action="store_true")
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
    params = synth.eval_params()
    dd_synth = lambda m: eng.engine_synthesizer(m, lrank)[0]
    model, ds, desc = workload(args.workload, dd_synth, params)
    E = eng.make_engine(model, params, deldops=[ds], device=lrank)
    form = eng.FORMS[args.form]
    nfr = ds.nframes
    flush = torch.empty(2 * L2_BYTES, dtype=torch.uint8, device="cuda")
    trial = lambda k: 1.0 + 1e-3 * math.sin(0.7 * k)

    # accuracy of the batched FP32 form against FP64 on the same trial model
    E.set_scale(0, trial(0))
    chi64 = E.evaluate(eng.FORM_BATCHED_FP64)["chi2"]
    chi32 = E.evaluate(eng.FORM_BATCHED_FP32)["chi2"]
    dchi = abs(chi32 - chi64) / abs(chi64)

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
            E.evaluate(form_id)
            host_ms.append(1e3 * (time.perf_counter() - t0))
            dev_ms.append(E.last_ms())
            if dist and record:
                t = torch.tensor([dev_ms[-1]], dtype=torch.float64, device="cuda")
                dist.all_reduce(t)   # per-step exchange of the shard totals
        if dist:
            dist.barrier()
        torch.cuda.synchronize()
        return dev_ms, host_ms

    # plain FP64 GPU path (the metric's comparison point), a few steps
    plain_dev, _ = run(eng.FORM_PLAIN_FP64, max(3, min(args.steps, 10)), 2, False)
    clocks = ClockSampler(lrank)
    clocks.start()
    time.sleep(0.3)
    dev_ms, host_ms = run(form, args.steps, args.warmup, True)
    clk = clocks.stop()
    stages = E.stage_times(form if form != eng.FORM_PLAIN_FP64 else eng.FORM_BATCHED_FP64)

    total_dev = sum(dev_ms)
    total_host = sum(host_ms)
    if dist:
        t = torch.tensor([total_dev, total_host], dtype=torch.float64, device="cuda")
        dist.all_reduce(t, op=dist.ReduceOp.MAX)
        total_dev, total_host = t.tolist()
    ms_step = total_dev / args.steps
    value = ws * nfr / (ms_step / 1e3)
    e2e = ws * nfr / (total_host / args.steps / 1e3)
    plain_rate = nfr / (statistics.mean(plain_dev) / 1e3)

    s_elem = 4 if form == eng.FORM_BATCHED_FP32 else 8
    b_model, b_pos, b_dd = algorithmic_bytes(model, ds, s_elem)
    peaks_path = os.path.join(REPO, "MEASURED_PEAKS.json")
    try:
        peaks = json.load(open(peaks_path))
        peak, peak_src = float(peaks["hbm_gbs"]), "measured"
    except Exception:
        peak, peak_src = 6650.0, "fallback"
    # dominant kernel: the fused tile raster + delay-Doppler synthesis
    rs_ms = stages.get("raster_synth", float("nan"))
    d_elems = sum(f.ndel * f.ndop for f in ds.frames)
    rs_bytes = b_model + b_pos + d_elems * s_elem     # model read, POS word+cos(e), fit write
    achieved = rs_bytes / (rs_ms / 1e3) / 1e9
    traffic_path = os.path.join(REPO, "profiles", "raster_traffic.json")
    traffic = None
    if os.path.exists(traffic_path):
        try:
            traffic = json.load(open(traffic_path)).get(args.workload + "_" + args.form)
        except Exception:
            traffic = None
    step_bytes = b_model + b_pos + b_dd
    line = {
        "metric": "frame-evals/sec", "value": value, "unit": "frame-evals/s", "n_gpus": ws,
        "steps": args.steps, "warmup": args.warmup, "ms_per_step": ms_step,
        "higher_is_better": True, "scaling": "weak", "vs_baseline": None,
        "dtype": "f32" if form == eng.FORM_BATCHED_FP32 else "f64", "data": "synthetic",
        "config": {"workload": desc, "form": args.form, "frames_per_gpu": nfr,
                   "model_facets": model.nf, "l2": "flushed (2x L2 buffer written) before every step",
                   "parallelism": "frame shards, one per GPU" if ws > 1 else "single GPU",
                   "dchi2_rel_fp32_vs_fp64": dchi,
                   "plain_fp64_frame_evals_per_s": plain_rate,
                   "batched_over_plain_fp64": value / ws / plain_rate,
                   "p50_ms": statistics.median(dev_ms), "p99_ms": float(np.percentile(dev_ms, 99)),
                   "stage_ms": stages,
                   "step_algorithmic_bytes": step_bytes,
                   "step_achieved_gbs": step_bytes / (ms_step / 1e3) / 1e9},
        "roofline": {"bound": "hbm", "kernel": "k_raster (tile raster + delay-Doppler synthesis)",
                     "achieved": achieved, "peak": peak, "unit": "GB/s", "frac": achieved / peak,
                     "peak_source": peak_src, "traffic": traffic,
                     "algorithmic_bytes_per_launch": rs_bytes},
        "e2e": {"value": e2e, "unit": "frame-evals/s", "h2d_bytes_per_step": 8 * (model.nv + 3),
                "d2h_bytes_per_step": 72,
                "what": "shape_engine_evaluate through the C ABI per bestfit trial: model parameters "
                        "host->device, chi-square summary device->host, host wall clock"},
        "gpu_launches": 10 * args.steps if form != eng.FORM_PLAIN_FP64 else None,
        "clocks": clk,
    }
    if rank == 0 and ws == 1 and not args.no_cpu_baseline:
        line["cpu_baseline"] = cpu_baseline(model, ds, params)
    E.close()
    if dist:
        dist.destroy_process_group()
    if rank == 0:
        print(json.dumps(line), flush=True)
    return 0


if __name__ == "__main__":
    sys.exit(main())
