"""Benchmark: reconstructions/s of the shrink-wrap / HIO engine on B200.

Headline workload (default, N=1 per GPU): the single large reconstruction --
2048x2048 float32 modulus of 400 Gaussian blobs (sigma U(1.5,3) px,
amplitudes U(0.3,1)) in a centred disk of radius 300 px with Poisson noise
at 1e9 photons, seed 1; 128 shrink-wrap cycles x 20 HIO iterations, beta
0.9, sigma0 3.0, sigma change 0.01, cutoffs 0.04 / 0.20, targetError =
FLT_MIN so every cycle runs.  One step = one full reconstruction.

  python bench.py [--gpus N] [--steps K] [--warmup W] [--impl ours|reference]

Our arm times K reconstructions with CUDA events on the launch stream, the
modulus already resident in HBM (`value`), and K more through the drop-in C
ABI call imr_cuda_shrink_wrap with pinned host buffers, host<->device copies
inside the timed region (`e2e`).  The L2 (126 MB) is flushed by writing a
256 MB buffer before every timed reconstruction, outside the timed events.
The roofline entry times the two passes of a HIO iteration (the dominant
kernels) live with CUDA events.

At N=1 the same JSON line also carries the other workloads of the path,
each measured the same way and each with its accuracy against the FP64
restatement of the reference (aligned relative L2 modulo twin and
translation, next to the reference FP32 path's own distance to FP64 -- the
"equal error" yardstick):
  plain_256        256x256, 60 blobs, 64 x 20: GPU recon/s (device, e2e), the
                   reference's CPU shrinkWrap timed on a FULL reconstruction
  batched_uneven   512 reconstructions, W, H in {128..512}, 64 x 20: the
                   batched engine (one graph launch per cycle step, step
                   configuration chosen by its online tuner, cached in
                   $IMR_TUNE_CACHE or ~/.cache/imresh_b200/engine_tune.txt)
                   vs the plain path per request
  large_4096       4096x4096, 1500 blobs, 32 x 20: the FP32 path and the
                   split-precision tensor-core column passes (BF16 / FP16 hi+lo)
  served_stream    Poisson arrivals at 70 % of the measured capacity, sides
                   log-uniform 64..2048, stop at 1e-5 or 128 cycles: recon/s,
                   latency p50/p99, device bytes
The CPU baseline is the reference's own CPU shrinkWrap (compiled from its
sources over the project FFT, oracle/_ref), timed after all GPU work with
the host otherwise idle; the accuracy runs of the FP64 restatement come last.

Under torchrun each rank runs independent reconstructions on its own GPU
(replicas; the path has no exchange step), timing is the max over ranks.
"""
from __future__ import annotations

import argparse
import json
import os
import subprocess
import sys
import tempfile
import time

import numpy as np

ROOT = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, ROOT)

N_CYCLES, N_HIO = 128, 20
W = H = 2048
PARAMS = dict(beta=0.9, cut_auto=0.04, cut=0.2, sigma0=3.0, sigma_change=0.01)
METRIC = "recon/s"
WORKLOAD = "shrink-wrap 2048x2048 f32, 400 blobs + Poisson 1e9, 128 cycles x 20 HIO"
FLT_MIN = float(np.finfo(np.float32).tiny)


def main_config(world: int) -> dict:
    return {"workload": WORKLOAD, "width": W, "height": H, "cycles": N_CYCLES, "hio_per_cycle": N_HIO,
            "parallelism": f"replicas x{world}",
            "l2": "flushed (256 MB write) before every timed reconstruction"}


def _peaks():
    try:
        with open(os.path.join(ROOT, "MEASURED_PEAKS.json")) as f:
            d = json.load(f)
        return float(d["hbm_gbs"]), "measured"
    except Exception:
        return 6650.0, "fallback"


def cpu_model_name() -> str:
    try:
        with open("/proc/cpuinfo") as f:
            for line in f:
                if line.startswith("model name"):
                    return line.split(":", 1)[1].strip()
    except OSError:
        pass
    return "unknown"


def threads_used():
    return int(os.environ.get("OMP_NUM_THREADS", os.cpu_count() or 1))


class ClockSampler:
    """Samples nvidia-smi clocks and throttle reasons during the timed region."""

    Q = ("index,clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,"
         "clocks_event_reasons.hw_slowdown,clocks_event_reasons.hw_thermal_slowdown,"
         "clocks_event_reasons.sw_thermal_slowdown,clocks_event_reasons.sw_power_cap")

    def __init__(self, index: int):
        self.index = index
        self.proc = None
        self.path = None

    def start(self):
        fd, self.path = tempfile.mkstemp(suffix=".csv")
        os.close(fd)
        try:
            self.proc = subprocess.Popen(
                ["nvidia-smi", f"--id={self.index}", f"--query-gpu={self.Q}", "--format=csv,noheader,nounits",
                 "-lms", "200"], stdout=open(self.path, "w"), stderr=subprocess.DEVNULL)
        except Exception:
            self.proc = None

    def stop(self):
        if self.proc is None:
            return {"sm_mhz": None, "sm_max_mhz": None, "reasons": ["nvidia-smi unavailable"]}
        self.proc.terminate()
        try:
            self.proc.wait(timeout=5)
        except Exception:
            self.proc.kill()
        sm, smax, reasons = [], None, set()
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        for line in open(self.path):
            f = [x.strip() for x in line.split(",")]
            if len(f) < 9:
                continue
            try:
                sm.append(float(f[1]))
                smax = float(f[2])
            except ValueError:
                continue
            for name, v in zip(names, f[5:9]):
                if v.lower() == "active":
                    reasons.add(name)
        os.unlink(self.path)
        return {"sm_mhz": float(np.median(sm)) if sm else None, "sm_max_mhz": smax,
                "reasons": sorted(reasons), "samples": len(sm)}


def _lat_stats(lat_ms):
    lat = np.sort(np.asarray(lat_ms, dtype=np.float64))
    return float(np.percentile(lat, 50)), float(np.percentile(lat, 99))


def max_over_ranks(values, dist=None, device=None):
    """Element-wise max of a list of floats over all ranks (timings of the
    slowest replica); identity without a process group."""
    if dist is None or not dist.is_initialized() or dist.get_world_size() == 1:
        return [float(v) for v in values]
    import torch
    t = torch.tensor(values, dtype=torch.float64, device=device)
    dist.all_reduce(t, op=dist.ReduceOp.MAX)
    return [float(x) for x in t.tolist()]


def aggregate_throughput(steps: int, world: int, total_ms_max: float) -> float:
    """Whole-job reconstructions per second: every rank runs `steps`
    independent reconstructions; the job takes as long as the slowest rank."""
    return steps * world / (total_ms_max / 1e3)


def make_input():
    from imresh_b200 import data
    M, _ = data.make_modulus(data.cfg1_spec(), seed=1)
    return M


# ---------------------------------------------------------------- CPU side (oracle: baseline and checker)
def _sw(n_cycles, n_hio):
    import oracle
    return oracle.SwParams(n_cycles, FLT_MIN, PARAMS["beta"], PARAMS["cut_auto"], PARAMS["cut"],
                           PARAMS["sigma0"], PARAMS["sigma_change"], n_hio)


def cpu_reference_run(M, n_cycles: int, n_hio: int):
    """(wall seconds, output, kind) of the reference's CPU shrinkWrap (the
    restatement where oracle/_ref is not built)."""
    import oracle
    p = _sw(n_cycles, n_hio)
    t = time.perf_counter()
    if oracle.ref_lib() is not None:
        out = oracle.ref_shrinkwrap(M, p)
        kind = "reference"
    else:
        out = oracle.shrinkwrap(M, p).out
        kind = "port"
    return time.perf_counter() - t, out, kind


def cpu_model(M):
    """Per-iteration and per-cycle seconds of the CPU path, from two bounded
    samples (1 cycle x 1 HIO and 1 cycle x 3 HIO)."""
    t1, _, kind = cpu_reference_run(M, 1, 1)
    t3, _, _ = cpu_reference_run(M, 1, 3)
    it = max((t3 - t1) / 2.0, 1e-9)
    cyc = max(t1 - it, 0.0)
    return it, cyc, kind, t1 + t3


def _oracle_task(task):
    """Pool worker: one FP32 or FP64 run of the restated oracle."""
    kind, M, n_cycles, n_hio = task
    import oracle
    t = time.perf_counter()
    r = oracle.shrinkwrap(M, _sw(n_cycles, n_hio), fp64=(kind == "f64"))
    return r.out.astype(np.float64), np.asarray(r.errors, np.float64), time.perf_counter() - t


def accuracy(gpu_out, f64_out, f32_out, obj=None):
    """Aligned relative L2 (modulo twin and translation) of the GPU result and
    of the reference FP32 path's result to the FP64 run, on out / (W*H)."""
    from imresh_b200.metrics import aligned_rel_l2, rel_l2
    n = gpu_out.size
    g, d, r = gpu_out / n, f64_out / n, f32_out / n
    out = {"rel_l2_vs_fp64": aligned_rel_l2(g, d), "reference_fp32_rel_l2_vs_fp64": aligned_rel_l2(r, d),
           "unaligned_rel_l2_vs_fp64": rel_l2(g, d), "reference_fp32_unaligned_rel_l2_vs_fp64": rel_l2(r, d)}
    out["ratio_to_reference_error"] = out["rel_l2_vs_fp64"] / max(out["reference_fp32_rel_l2_vs_fp64"], 1e-30)
    if obj is not None:
        out["rel_l2_vs_object"] = aligned_rel_l2(g, obj)
        out["reference_fp32_rel_l2_vs_object"] = aligned_rel_l2(r, obj)
    return out


# ---------------------------------------------------------------- GPU workloads
def _timed_plan_runs(plan, d_m, d_o, steps, warmup, flush, stream):
    import torch
    for _ in range(warmup):
        plan.execute(d_m, d_o)
    torch.cuda.synchronize()
    ev = [(torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)) for _ in range(steps)]
    for i in range(steps):
        flush.fill_(float(i))
        ev[i][0].record(stream)
        plan.execute(d_m, d_o)
        ev[i][1].record(stream)
    torch.cuda.synchronize()
    return [a.elapsed_time(b) for a, b in ev]


def _timed_drop_in(imr, M, n_cycles, n_hio, steps, flush, stream):
    import torch
    Hh, Ww = M.shape
    host_in = torch.from_numpy(M.reshape(-1)).pin_memory()
    host_io = torch.empty_like(host_in).pin_memory()
    ms = []
    for i in range(steps):
        flush.fill_(float(i))
        torch.cuda.synchronize()
        host_io.copy_(host_in)
        t0 = time.perf_counter()
        rc = imr.lib().imr_cuda_shrink_wrap(host_io.data_ptr(), Ww, Hh, stream.cuda_stream, 0, 0, n_cycles,
                                            imr.FLT_MIN, PARAMS["beta"], PARAMS["cut_auto"], PARAMS["cut"],
                                            PARAMS["sigma0"], PARAMS["sigma_change"], n_hio)
        ms.append((time.perf_counter() - t0) * 1e3)
        if rc != 0:
            raise imr.ImrError(rc, "imr_cuda_shrink_wrap")
    return ms, host_io.numpy().reshape(Hh, Ww).copy()


def run_plain_256(args, flush, stream):
    """The 256x256 blob workload (60 blobs, sigma 2, r = 40, seed 0, no
    noise), 64 x 20, on the plain FP32 path; its working set stays in L2."""
    import torch
    import imresh_b200 as imr
    from imresh_b200 import data
    M, obj = data.make_modulus(data.cfg0_spec(), 0)
    prm = imr.Params(64, imr.FLT_MIN, PARAMS["beta"], PARAMS["cut_auto"], PARAMS["cut"], PARAMS["sigma0"],
                     PARAMS["sigma_change"], N_HIO)
    plan = imr.Plan(256, 256, prm)
    d_m = torch.from_numpy(M).cuda()
    d_o = torch.empty_like(d_m)
    steps = max(args.steps, 10)
    ms = _timed_plan_runs(plan, d_m, d_o, steps, max(args.warmup, 3), flush, stream)
    n, errs = plan.stats()
    plan.close()
    e2e, out = _timed_drop_in(imr, M, 64, N_HIO, steps, flush, stream)
    np.testing.assert_array_equal(out, d_o.cpu().numpy())
    r = {"workload": "shrink-wrap 256x256 f32, 60 blobs sigma 2 in r=40, seed 0, 64 cycles x 20 HIO",
         "recon_per_s": steps / (sum(ms) / 1e3), "ms_per_recon": float(np.mean(ms)),
         "e2e_recon_per_s": steps / (sum(e2e) / 1e3),
         "hio_iterations_per_s": steps * 64 * N_HIO / (sum(ms) / 1e3),
         "final_hio_error": float(errs[-1]) if len(errs) else None, "cycles_done": n,
         "l2": "flushed before every timed reconstruction; the 256x256 working set is L2-resident during it"}
    return r, {"M": M, "obj": obj, "out": out, "errors": errs}


def run_batched(n_jobs: int = 512, plain_sample: int = 64, schedule: int = 0, tune_cache: str | None = None,
                cycles_per_step: int = 1):
    """The uneven batch: n_jobs reconstructions, W and H each from
    {128,192,256,384,512}, 20-200 blobs, Poisson 1e7-1e9 photons, seed 2,
    64 cycles x 20 HIO.  Served by the batched engine (all jobs submitted at
    once, host buffers, copies included) vs the plain path (one plan per
    shape, one reconstruction at a time, host buffers) on a sample of the
    same jobs, whose results must be bit-identical.  Both wall-clock timed
    around synchronous calls."""
    import imresh_b200 as imr
    from imresh_b200 import data
    specs = data.cfg2_specs(n_jobs, seed=2)
    inputs = [data.make_modulus(sp, seed=2, index=i)[0] for i, sp in enumerate(specs)]
    prm = imr.Params(64, imr.FLT_MIN, 0.9, 0.04, 0.2, 3.0, 0.01, 20)
    # warm-up: one short job of every shape in the batch through the engine
    eng = imr.Engine()
    first = {}
    for i, M in enumerate(inputs):
        first.setdefault(M.shape, i)
    for i in first.values():
        eng.submit(inputs[i], imr.Params(1, imr.FLT_MIN, 0.9, 0.04, 0.2, 3.0, 0.01, 1), tag=i)
    eng.run()
    eng.poll(len(first))
    eng.close()
    eng = imr.Engine()
    eng.set_schedule(schedule)
    eng.set_cycles_per_step(cycles_per_step)
    if tune_cache is not None:
        eng.set_autotune(True, tune_cache)
    t0 = time.perf_counter()
    for i, M in enumerate(inputs):
        eng.submit(M, prm, tag=i)
    eng.run()
    dt = time.perf_counter() - t0
    res = eng.poll(n_jobs)
    info = eng.info()
    eng.close()
    assert len(res) == n_jobs and all(r["status"] == 0 for r in res)
    by_tag = {r["tag"]: r for r in res}
    p50, p99 = _lat_stats([r["latency_ms"] for r in res])
    # plain path on the first plain_sample jobs
    plans = {}
    for M in inputs[:plain_sample]:
        if M.shape not in plans:
            plans[M.shape] = imr.Plan(M.shape[1], M.shape[0], prm)
            plans[M.shape].execute_host(M)   # warm
    lat, identical = [], 0
    t1 = time.perf_counter()
    outs = []
    for M in inputs[:plain_sample]:
        a = time.perf_counter()
        outs.append(plans[M.shape].execute_host(M))
        lat.append((time.perf_counter() - a) * 1e3)
    dt_plain = time.perf_counter() - t1
    for i, o in enumerate(outs):
        identical += int(np.array_equal(o, by_tag[i]["out"]))
    for p in plans.values():
        p.close()
    px = sum(M.size for M in inputs)
    small = min(range(n_jobs), key=lambda i: inputs[i].size)
    return {
        "workload": f"{n_jobs} uneven reconstructions, W,H in {{128..512}}, 64 cycles x 20 HIO, "
                    "Poisson 1e7-1e9, seed 2",
        "engine_recon_per_s": n_jobs / dt, "engine_seconds": dt,
        "engine_hio_iterations_per_s": n_jobs * 64 * 20 / dt,
        "engine_gbs_algorithmic": px * 64 * 20 * 53 / dt / 1e9,
        "engine_latency_p50_ms": p50, "engine_latency_p99_ms": p99,
        "engine_device_bytes_peak": info["device_bytes_peak"], "engine_kernels": info["launches"],
        "engine_steps": info["steps"], "engine_host_launches": info["host_launches"],
        "engine_host_launches_per_step": info["host_launches"] / max(info["steps"], 1),
        "engine_kernels_per_step": info["kernels_per_step"],
        "engine_graph_builds": info["graph_builds"] + info["graph_updates"],
        "engine_device_seconds": info["device_ms"] / 1e3,
        "engine_schedule": "chained" if info["schedule"] else "grouped", "engine_grid_pct": info["grid_pct"],
        "engine_cycles_per_step": info["cycles_per_step"],
        "engine_tuner": {"explored_steps": info["tune_explored"], "cache_hits": info["tune_cache_hits"]}
                        if tune_cache is not None else None,
        "plain_recon_per_s": plain_sample / dt_plain, "plain_sample_jobs": plain_sample,
        "plain_latency_p50_ms": _lat_stats(lat)[0],
        "speedup_engine_vs_plain": (n_jobs / dt) / (plain_sample / dt_plain),
        "engine_equals_plain_bitwise": f"{identical}/{plain_sample}",
        "timing": "wall clock around synchronous calls; host buffers, copies included",
    }, {"M": inputs[small], "out": by_tag[small]["out"], "shape": list(inputs[small].shape)}


def run_large_4096(args, flush, stream):
    """4096x4096, 1500 blobs in r = 600, seed 3, 32 x 20: the FP32 path and
    the split-precision tensor-core column passes (BF16 hi+lo, FP16 hi+lo);
    each 2D transform alone against numpy's FP64 FFT."""
    import torch
    import imresh_b200 as imr
    from imresh_b200 import data
    from imresh_b200.metrics import rel_l2
    M, obj = data.make_modulus(data.cfg3_spec(), 3)
    prm = imr.Params(32, imr.FLT_MIN, PARAMS["beta"], PARAMS["cut_auto"], PARAMS["cut"], PARAMS["sigma0"],
                     PARAMS["sigma_change"], N_HIO)
    p1 = imr.Params(1, imr.FLT_MIN, PARAMS["beta"], PARAMS["cut_auto"], PARAMS["cut"], PARAMS["sigma0"],
                    PARAMS["sigma_change"], 1)
    d_m = torch.from_numpy(M).cuda()
    d_o = torch.empty_like(d_m)
    rng = np.random.default_rng(5)
    x = (rng.standard_normal((4096, 4096)) + 1j * rng.standard_normal((4096, 4096))).astype(np.complex64)
    want = np.fft.fft2(x.astype(np.complex128))
    peak, _ = _peaks()
    steps = 3
    res, keep = {"workload": "shrink-wrap 4096x4096 f32 data, 1500 blobs in r=600, seed 3, 32 cycles x 20 HIO"}, {}
    for name, prec in (("fp32", imr.PREC_FP32), ("bf16x3", imr.PREC_BF16X3), ("fp16x3", imr.PREC_FP16X3)):
        plan = imr.Plan(4096, 4096, prm)
        plan.set_precision(prec)
        ms = _timed_plan_runs(plan, d_m, d_o, steps, 1, flush, stream)
        n, errs = plan.stats()
        ms_row, ms_col = plan.profile(10)
        row_b, col_b = plan.pass_bytes()
        plan.close()
        q = imr.Plan(4096, 4096, p1)
        q.set_precision(prec)
        keep[name] = q.execute_host(M)
        q.close()
        d = torch.from_numpy(x.view(np.float32)).cuda()
        if prec == imr.PREC_FP32:
            imr.fft2d(d, 4096, 4096, -1)
        else:
            imr.fft2d_split(d, 4096, 4096, -1, prec)
        torch.cuda.synchronize()
        got = d.cpu().numpy().view(np.complex64)
        del d
        res[name] = {"recon_per_s": steps / (sum(ms) / 1e3), "ms_per_recon": float(np.mean(ms)),
                     "hio_iterations_per_s": steps * 32 * N_HIO / (sum(ms) / 1e3),
                     "final_hio_error": float(errs[-1]) if len(errs) else None,
                     "row_pass_gbs": row_b / (ms_row * 1e-3) / 1e9, "col_pass_gbs": col_b / (ms_col * 1e-3) / 1e9,
                     "col_pass_ms": ms_col, "col_pass_frac": col_b / (ms_col * 1e-3) / 1e9 / peak,
                     "fft2d_rel_l2_vs_numpy_fp64": rel_l2(got, want)}
    res["split_vs_fp32_recon_ratio"] = {k: res[k]["recon_per_s"] / res["fp32"]["recon_per_s"]
                                        for k in ("bf16x3", "fp16x3")}
    res["note"] = ("split precision: radix-16 column stages as DFT-16 products on the tensor cores (mma.sync "
                   "m16n8k16, hi+lo operands, three products, FP32 accumulation); rows, twiddles, the last "
                   "radix-8 stage, the modulus and the error sums stay FP32/FP64")
    return res, {"M": M, "obj": obj, "out1": keep}


def served_inputs(n_req: int, seed: int = 4, max_side: int = 2048):
    """The serving stream's requests: W, H log-uniform integers in [64,
    max_side] (any length: mixed radix or Bluestein), 0.5-3 blobs per 1000
    px^2, Poisson 1e6-1e9 photons."""
    from imresh_b200 import data
    specs = data.cfg4_specs(n_req, seed=seed)
    for sp in specs:
        sp.width = min(sp.width, max_side)
        sp.height = min(sp.height, max_side)
    return [data.make_modulus(sp, seed=seed, index=i)[0] for i, sp in enumerate(specs)]


def run_served(n_req: int, rate_hz: float, seed: int = 4, max_side: int = 2048, max_active_px: int = 0,
               schedule: int = 0, step_target_ms: float = 0.0, inputs=None):
    """Serving stream: n_req requests (served_inputs) with Poisson arrivals at
    rate_hz; each request stops at error 1e-5 or 128 cycles.  Requests are
    admitted by the engine between steps as device memory (and the
    admitted-work bound, when set) allows; latency = arrival -> result in
    host memory."""
    import imresh_b200 as imr
    if inputs is None:
        inputs = served_inputs(n_req, seed, max_side)
    inputs = inputs[:n_req]
    rng = np.random.default_rng([seed, 7])
    arrivals = np.cumsum(rng.exponential(1.0 / rate_hz, n_req))
    prm = imr.Params(128, 1e-5, 0.9, 0.04, 0.2, 3.0, 0.01, 20)
    eng = imr.Engine()
    eng.set_schedule(schedule)
    if max_active_px:
        eng.set_admission(max_active_px)
    if step_target_ms:
        eng.set_step_target(step_target_ms)
    done, nxt, lat, t0 = 0, 0, [], time.perf_counter()
    submit_t = {}
    peak_active, cycles = 0, []
    while done < n_req:
        now = time.perf_counter() - t0
        while nxt < n_req and arrivals[nxt] <= now:
            eng.submit(inputs[nxt], prm, tag=nxt)
            submit_t[nxt] = t0 + arrivals[nxt]
            nxt += 1
        info = eng.info()
        peak_active = max(peak_active, info["resident"])
        if info["active"] == 0 and info["pending"] == 0:
            time.sleep(max(0.0, min(0.01, arrivals[nxt] - now)) if nxt < n_req else 0)
            continue
        eng.step()
        for r in eng.poll():
            lat.append((time.perf_counter() - submit_t[r["tag"]]) * 1e3)
            cycles.append(r["cycles_done"])
            done += 1
    wall = time.perf_counter() - t0
    info = eng.info()
    eng.close()
    p50, p99 = _lat_stats(lat)
    px = sum(M.size for M in inputs)
    return {"workload": f"{n_req} requests, Poisson arrivals at {rate_hz:.2f} /s, sides log-uniform "
                        f"64..{max_side}, stop at 1e-5 or 128 cycles, seed {seed}",
            "recon_per_s": n_req / wall, "latency_p50_ms": p50, "latency_p99_ms": p99,
            "latency_max_ms": float(np.max(lat)), "offered_rate_hz": rate_hz,
            "peak_resident": peak_active, "device_bytes_peak": info["device_bytes_peak"],
            "mean_request_px": px / n_req,
            "max_active_px": max_active_px or None, "step_target_ms": step_target_ms or None,
            "schedule": "chained" if schedule else "grouped",
            "mean_cycles": float(np.mean(cycles)), "steps": info["steps"], "kernels": info["launches"],
            "host_launches": info["host_launches"], "graph_builds": info["graph_builds"],
            "graph_updates": info["graph_updates"], "device_seconds": info["device_ms"] / 1e3,
            "wall_seconds": wall}


def run_served_default(n_req: int, load: float = 0.7):
    """The served stream as the default bench runs it: the capacity first (the
    first 150 requests all at once), then n_req requests with Poisson arrivals
    at `load` x that capacity; both on the chained schedule with a 20 ms
    step-time admission target."""
    inputs = served_inputs(n_req)
    cap = run_served(min(150, n_req), 1e4, schedule=1, step_target_ms=20.0, inputs=inputs)
    rate = load * cap["recon_per_s"]
    r = run_served(n_req, rate, schedule=1, step_target_ms=20.0, inputs=inputs)
    r["capacity_recon_per_s"] = cap["recon_per_s"]
    r["capacity_sample"] = "first 150 requests of the stream, all submitted at once"
    r["load"] = load
    return r


# ---------------------------------------------------------------- reference arm
def run_reference(args, rank, world):
    """The reference's own CPU shrinkWrap on the headline workload.  A step is
    a bounded sample (1 cycle x 2 HIO at 2048^2, about a second); recon/s is
    extrapolated from a per-iteration / per-cycle model fitted on 1 x 1 and
    1 x 3 samples.  The model is checked once on the 256x256 workload, where
    a full reconstruction is timed."""
    if rank != 0:
        return
    from imresh_b200 import data
    M = make_input()
    it, cyc, kind, _ = cpu_model(M)              # warm-up + calibration (untimed)
    for _ in range(max(args.warmup - 2, 0)):
        cpu_reference_run(M, 1, 2)
    sample_s, per_recon = [], []
    for _ in range(args.steps):
        t, _, _ = cpu_reference_run(M, 1, 2)
        sample_s.append(t)
        # the sample ran 1 cycle x 2 HIO; scale to 128 cycles x 20 HIO
        per_recon.append(N_CYCLES * (t - 2 * it + N_HIO * it))
    s = float(np.mean(per_recon))
    v = 1.0 / s
    M0, _ = data.make_modulus(data.cfg0_spec(), 0)
    it0, cyc0, _, _ = cpu_model(M0)
    t0, _, _ = cpu_reference_run(M0, 64, N_HIO)
    out = {
        "impl": "reference", "metric": METRIC, "value": v, "unit": "recon/s", "n_gpus": 0,
        "steps": args.steps, "warmup": args.warmup, "ms_per_step": float(np.mean(sample_s)) * 1e3,
        "higher_is_better": True, "scaling": "weak", "vs_baseline": None, "dtype": "f32",
        "data": "synthetic (seeded Gaussian-blob objects, Poisson noise)",
        "config": main_config(1),
        "step": "a bounded sample: 1 cycle x 2 HIO at 2048^2 (ms_per_step is its wall time); value is "
                "extrapolated to 128 x 20 by the model below",
        "ms_per_recon_extrapolated": s * 1e3,
        "model": {"per_hio_iteration_s": it, "per_cycle_overhead_s": cyc,
                  "check_256x256_64x20": {"measured_s": t0, "predicted_s": 64 * (cyc0 + N_HIO * it0)}},
        "cpu_baseline": {"value": v, "unit": "recon/s", "cores": threads_used(), "cpu": cpu_model_name(),
                         "kind": kind,
                         "sample": "reference CPU shrinkWrap (project FFT shim, not FFTW; FFT single-threaded "
                                   "as in the reference), 1 cycle x 2 HIO per step at 2048^2, extrapolated "
                                   "to 128 x 20"},
        "e2e": {"value": v, "unit": "recon/s", "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0},
    }
    print(json.dumps(out), flush=True)


# ---------------------------------------------------------------- our arm
def run_ours(args, rank, world, local_rank):
    import torch
    import imresh_b200 as imr

    torch.cuda.set_device(local_rank)
    dev = torch.device("cuda", local_rank)
    stream = torch.cuda.current_stream()
    dist = None
    if world > 1:
        import torch.distributed as dist_mod
        dist = dist_mod

    M = make_input()
    prm = imr.Params(N_CYCLES, imr.FLT_MIN, PARAMS["beta"], PARAMS["cut_auto"], PARAMS["cut"],
                     PARAMS["sigma0"], PARAMS["sigma_change"], N_HIO)
    plan = imr.Plan(W, H, prm)
    d_m = torch.from_numpy(M).to(dev)
    d_o = torch.empty_like(d_m)
    flush = torch.empty(256 * 1024 * 1024 // 4, dtype=torch.float32, device=dev)

    def barrier():
        if dist is not None:
            dist.barrier()
        torch.cuda.synchronize()

    for _ in range(args.warmup):
        plan.execute(d_m, d_o)
    torch.cuda.synchronize()

    # ---- device-resident timing (value)
    clocks = ClockSampler(local_rank)
    clocks.start()
    ev = [(torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True))
          for _ in range(args.steps)]
    barrier()
    for i in range(args.steps):
        flush.fill_(float(i))
        ev[i][0].record(stream)
        plan.execute(d_m, d_o)
        ev[i][1].record(stream)
    barrier()
    ms = [a.elapsed_time(b) for a, b in ev]
    total_ms = float(sum(ms))

    # ---- roofline of the two passes of a HIO iteration (dominant kernels)
    ms_row, ms_col = plan.profile(20)
    row_b, col_b = plan.pass_bytes()

    # ---- end-to-end through the drop-in C ABI with pinned host buffers
    barrier()
    e2e_ms, _ = _timed_drop_in(imr, M, N_CYCLES, N_HIO, args.steps, flush, stream)
    barrier()
    clk = clocks.stop()
    check = float(torch.linalg.vector_norm(d_o).item())
    if not np.isfinite(check):
        raise RuntimeError("non-finite reconstruction")

    e2e_total = float(sum(e2e_ms))
    total_ms, e2e_total, ms_row, ms_col = max_over_ranks([total_ms, e2e_total, ms_row, ms_col], dist, dev)

    if rank != 0:
        return
    peak, peak_kind = _peaks()
    value = aggregate_throughput(args.steps, world, total_ms)
    e2e_value = aggregate_throughput(args.steps, world, e2e_total)
    row_gbs = row_b / (ms_row * 1e-3) / 1e9
    col_gbs = col_b / (ms_col * 1e-3) / 1e9
    dom = ("row", row_b, ms_row, row_gbs) if ms_row >= ms_col else ("col", col_b, ms_col, col_gbs)
    traffic = None
    try:   # DRAM bytes per launch of the dominant kernel, from the committed ncu capture
        with open(os.path.join(ROOT, "profiles", "traffic.json")) as f:
            tj = json.load(f)
        entry = tj.get("row_pass_2048" if dom[0] == "row" else "col_pass_2048")
        traffic = entry["dram_bytes_per_launch"] if entry else None
    except Exception:
        pass
    iter_gbs = (row_b + col_b) / ((ms_row + ms_col) * 1e-3) / 1e9
    launches = plan.launches() * args.steps
    plan.close()

    out = {
        "metric": METRIC, "value": value, "unit": "recon/s", "n_gpus": world,
        "steps": args.steps, "warmup": args.warmup, "ms_per_step": total_ms / args.steps,
        "higher_is_better": True, "scaling": "weak", "vs_baseline": None, "dtype": "f32",
        "data": "synthetic (seeded Gaussian-blob objects, Poisson noise)",
        "config": main_config(world),
        "hio_iterations_per_s": value * N_CYCLES * N_HIO,
        "e2e": {"value": e2e_value, "unit": "recon/s", "h2d_bytes_per_step": 4 * W * H,
                "d2h_bytes_per_step": 4 * W * H,
                "api": "imr_cuda_shrink_wrap (drop-in for cudaShrinkWrap), pinned host buffer"},
        "roofline": {"bound": "hbm", "achieved": dom[3], "peak": peak, "unit": "GB/s",
                     "frac": dom[3] / peak, "traffic": traffic,
                     "traffic_source": "profiles/traffic.json (ncu, cold cache, per launch)",
                     "kernel": f"{dom[0]} pass ({'k_row_hio_p<false,2048>' if dom[0] == 'row' else 'k_col_p16<2048,4>'})",
                     "peak_source": peak_kind,
                     "algorithmic_bytes_per_launch": dom[1], "ms_per_launch": dom[2],
                     "launch_timing": "pair time: CUDA events around 20 row/column pairs replayed "
                                      "from one captured graph (the reconstruction's own execution "
                                      "mode); split between the passes as a replay with an event "
                                      "after every pass measures",
                     "row_pass_gbs": row_gbs, "col_pass_gbs": col_gbs,
                     "hio_iteration_gbs": iter_gbs, "hio_iteration_frac": iter_gbs / peak},
        "clocks": clk,
        "gpu_launches": launches,
    }
    if world > 1 or args.only_main:
        print(json.dumps(out), flush=True)
        return

    # ---- the other workloads of the path (GPU), then the CPU legs
    wl = {}
    keep = {}
    wl["plain_256"], keep["plain_256"] = run_plain_256(args, flush, stream)
    tune_cache = os.environ.get("IMR_TUNE_CACHE") or os.path.join(os.path.expanduser("~"), ".cache",
                                                                      "imresh_b200", "engine_tune.txt")
    os.makedirs(os.path.dirname(tune_cache), exist_ok=True)
    wl["batched_uneven"], keep["batched"] = run_batched(tune_cache=tune_cache)
    wl["large_4096"], keep["large"] = run_large_4096(args, flush, stream)
    # four cycles of the headline workload on the GPU, for the FP64 comparison
    p4 = imr.Plan(W, H, imr.Params(4, imr.FLT_MIN, PARAMS["beta"], PARAMS["cut_auto"], PARAMS["cut"],
                                   PARAMS["sigma0"], PARAMS["sigma_change"], N_HIO))
    out4 = p4.execute_host(M)
    _, errs4 = p4.stats()
    p4.close()
    if args.serve_requests:
        wl["served_stream"] = run_served_default(args.serve_requests)

    if not args.no_cpu_baseline:
        # CPU legs, the host otherwise idle: the timed baselines first
        it, cyc, kind, spent = cpu_model(M)
        secs = N_CYCLES * (cyc + N_HIO * it)
        out["cpu_baseline"] = {
            "value": 1.0 / secs, "unit": "recon/s", "cores": threads_used(), "cpu": cpu_model_name(),
            "kind": kind,
            "sample": f"reference CPU shrinkWrap (project FFT shim, FFT single-threaded) at 2048^2: 1x1 and "
                      f"1x3 (cycles x HIO) samples, {spent:.1f} s, extrapolated to 128 x 20 "
                      f"({secs:.0f} s per reconstruction)"}
        k0 = keep["plain_256"]
        t0, ref0, kind0 = cpu_reference_run(k0["M"], 64, N_HIO)
        wl["plain_256"]["cpu_baseline"] = {"value": 1.0 / t0, "unit": "recon/s", "cores": threads_used(),
                                           "cpu": cpu_model_name(), "kind": kind0,
                                           "sample": "one full reconstruction (64 x 20), timed, not extrapolated"}
        wl["plain_256"]["speedup_vs_cpu_reference"] = wl["plain_256"]["recon_per_s"] * t0
        # the accuracy runs of the FP64 restatement (not timed), four at a time
        import multiprocessing as mp
        kb = keep["batched"]
        kl = keep["large"]
        tasks = {"256_f64": ("f64", k0["M"], 64, N_HIO),
                 "2048x4_f64": ("f64", M, 4, N_HIO), "2048x4_f32": ("f32", M, 4, N_HIO),
                 "batch_f64": ("f64", kb["M"], 64, N_HIO), "batch_f32": ("f32", kb["M"], 64, N_HIO),
                 "4096x1_f64": ("f64", kl["M"], 1, 1), "4096x1_f32": ("f32", kl["M"], 1, 1)}
        env_omp = os.environ.get("OMP_NUM_THREADS")
        os.environ["OMP_NUM_THREADS"] = str(max(1, (os.cpu_count() or 4) // 4))
        try:
            with mp.get_context("spawn").Pool(4) as pool:
                res = dict(zip(tasks, pool.map(_oracle_task, list(tasks.values()))))
        finally:
            if env_omp is None:
                os.environ.pop("OMP_NUM_THREADS", None)
            else:
                os.environ["OMP_NUM_THREADS"] = env_omp
        a0 = accuracy(k0["out"], res["256_f64"][0], ref0, k0["obj"])
        a0["scope"] = "full 64 x 20 reconstruction"
        a0["final_hio_error"] = {"gpu": wl["plain_256"]["final_hio_error"], "fp64": float(res["256_f64"][1][-1])}
        wl["plain_256"]["accuracy"] = a0
        a4 = accuracy(out4, res["2048x4_f64"][0], res["2048x4_f32"][0])
        a4["scope"] = "first 4 cycles x 20 HIO of the headline workload (the full run is out of reach of the CPU)"
        a4["per_cycle_hio_error"] = {"gpu": [float(x) for x in errs4],
                                     "fp32_reference": res["2048x4_f32"][1].tolist(),
                                     "fp64": res["2048x4_f64"][1].tolist()}
        out["accuracy"] = a4
        ab = accuracy(kb["out"], res["batch_f64"][0], res["batch_f32"][0])
        ab["scope"] = f"one job of the batch ({kb['shape'][1]}x{kb['shape'][0]}), full 64 x 20"
        wl["batched_uneven"]["accuracy"] = ab
        for name, o in kl["out1"].items():
            al = accuracy(o, res["4096x1_f64"][0], res["4096x1_f32"][0], kl["obj"])
            al["scope"] = "1 cycle x 1 HIO (before HIO's amplification; the full run is out of reach of the CPU)"
            wl["large_4096"][name]["accuracy"] = al
        bu = wl["batched_uneven"]
        wl["engine_vs_plain"] = {
            "recon_per_s_ratio": bu["speedup_engine_vs_plain"],
            "at_equal_error": f"engine results bit-identical to the plain FP32 path ({bu['engine_equals_plain_bitwise']} "
                              "sampled); aligned rel. L2 to FP64 of a batch job "
                              f"{bu['accuracy']['rel_l2_vs_fp64']:.3g} vs the reference FP32 path's "
                              f"{bu['accuracy']['reference_fp32_rel_l2_vs_fp64']:.3g}",
            "split_precision_vs_fp32": wl["large_4096"]["split_vs_fp32_recon_ratio"]}
        wl["equal_error"] = (
            "HIO amplifies rounding ~2x per iteration: past a few cycles any FP32 run, the reference's "
            "included, is as far from the FP64 run as unrelated images; 'equal error' = the GPU's aligned "
            "distance to FP64 next to the reference FP32 path's own (ratio_to_reference_error)")
    out["workloads"] = wl
    print(json.dumps(out), flush=True)


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=5)
    ap.add_argument("--warmup", type=int, default=3)
    ap.add_argument("--impl", choices=["ours", "reference"], default="ours")
    ap.add_argument("--no-cpu-baseline", action="store_true")
    ap.add_argument("--only-main", action="store_true", help="only the headline workload")
    ap.add_argument("--serve-requests", type=int, default=400, metavar="N",
                    help="requests of the served stream in the default run, at 70 %% of its measured "
                         "capacity (0: skip)")
    ap.add_argument("--rate", type=float, default=7.0, help="--serve: arrival rate, requests/s")
    ap.add_argument("--max-active-px", type=int, default=0,
                    help="served stream: bound on the pixels of the admitted requests (0: memory only)")
    ap.add_argument("--serve", type=int, default=0, metavar="N",
                    help="only run the serving stream with N requests and print its JSON")
    ap.add_argument("--schedule", type=int, default=0, help="--serve: 0 grouped, 1 chained step graphs")
    ap.add_argument("--step-target", type=float, default=0.0,
                    help="--serve: admission bound from the measured step time, ms (0: off)")
    ap.add_argument("--ncu-case", type=str, default="", metavar="N or WxH",
                    help="run one NxN (or WxH) reconstruction (1 cycle x 3 HIO) of the headline recipe scaled "
                         "to that size and exit: a small case for ncu")
    ap.add_argument("--ncu-prec", type=int, default=0,
                    help="column-pass precision of the ncu case (0 FP32, 1 BF16 hi+lo, 2 FP16 hi+lo)")
    args = ap.parse_args()
    if args.ncu_case:
        import torch
        import imresh_b200 as imr
        from imresh_b200 import data
        w, _, h = args.ncu_case.partition("x")
        w = int(w)
        h = int(h) if h else w
        # the headline's blob density, radius and Poisson noise, scaled to W x H
        M, _ = data.make_modulus(data.BlobSpec(w, h, max(1, 400 * w * h // 2048 ** 2), 300.0 * min(w, h) / 2048,
                                               (1.5, 3.0), (0.3, 1.0), 1e9), 0)
        plan = imr.Plan(w, h, imr.Params(1, imr.FLT_MIN, 0.9, 0.04, 0.2, 3.0, 0.01, 3))
        plan.set_precision(args.ncu_prec)
        d_m = torch.from_numpy(M).cuda()
        d_o = torch.empty_like(d_m)
        plan.execute(d_m, d_o)
        torch.cuda.synchronize()
        print(json.dumps({"ncu_case": [w, h], "precision": args.ncu_prec, "checksum": float(d_o.abs().sum())}))
        return
    if args.serve:
        import torch
        torch.cuda.set_device(0)
        print(json.dumps(run_served(args.serve, args.rate, max_active_px=args.max_active_px,
                                    schedule=args.schedule, step_target_ms=args.step_target)), flush=True)
        return
    rank = int(os.environ.get("RANK", 0))
    world = int(os.environ.get("WORLD_SIZE", 1))
    local_rank = int(os.environ.get("LOCAL_RANK", 0))
    if args.impl == "reference":
        run_reference(args, rank, world)
        return
    if world > 1:
        import datetime
        import torch
        import torch.distributed as dist
        torch.cuda.set_device(local_rank)
        dist.init_process_group("nccl", timeout=datetime.timedelta(seconds=120))
        try:
            run_ours(args, rank, world, local_rank)
        finally:
            dist.destroy_process_group()
    else:
        run_ours(args, rank, world, local_rank)


if __name__ == "__main__":
    main()
