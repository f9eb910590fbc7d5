#!/usr/bin/env python
"""Benchmark of the viscoelastic time step (one JSON line on rank 0).

A bench "step" is one whole forward solve of the single-shot workload:
2048 x 1024 grid, dx = 5 m, dt = 0.4 ms, 4000 time steps, FP32, seeded
8-layer VTI medium with 3 SLS mechanisms, 40-cell CPML, free surface,
12 Hz explosive Ricker and 512 receivers (synthetic inputs), on the
default kernel path (the split velocity/stress pair).

  value  Gpt/s = nx*nz*nt / time, inputs resident in HBM, max over ranks,
         summed over ranks (one independent shot per GPU: weak scaling)
  e2e    the same through vi_forward_host with pinned host buffers: medium
         and wavelet upload, the solve, and the trace download per step
  roofline  algorithmic bytes per time step (one velocity + one stress
         launch) / mean step time vs the measured HBM copy bandwidth
  accuracy  the timed solve against the same solve in FP64 (untimed)
  batched, batched_small  64-shot TTI gathers, batched vs one at a time
  gradient  the 16-shot 1024 x 512 FWI gradient, with FD and FP32 checks
  serving  the mixed request stream, continuous vs FIFO
  cpu_baseline  the CPU oracle (FP32 twin, all host threads) on a bounded
         sample of the same workload (rank 0, N = 1)

`--impl reference` times the reference's CPU path instead: the reference is
Julia (absent here) and its step does not execute, so the CPU restatement
in oracle/ stands in for it, on all host threads.
"""
from __future__ import annotations

import argparse
import json
import math
import os
import statistics
import subprocess
import sys
import tempfile
import time
from pathlib import Path

ROOT = Path(__file__).resolve().parent
sys.path.insert(0, str(ROOT))

METRIC = "Gpt/s & % HBM roofline per step; shots/s + p50/p99 latency, batched vs plain @1e-5"


def parse_args():
    p = argparse.ArgumentParser()
    p.add_argument("--gpus", type=int, default=1)
    p.add_argument("--steps", type=int, default=3)
    p.add_argument("--warmup", type=int, default=3)
    p.add_argument("--impl", default="ours", choices=["ours", "reference"])
    p.add_argument("--nx", type=int, default=2048)
    p.add_argument("--nz", type=int, default=1024)
    p.add_argument("--nt", type=int, default=4000)
    p.add_argument("--kind", default="vti", choices=["iso", "vti", "tti"])
    p.add_argument("--precision", default="f32", choices=["f32", "f64"])
    p.add_argument("--variant", type=int, default=0)
    p.add_argument("--no-e2e", action="store_true")
    p.add_argument("--no-accuracy", action="store_true")
    p.add_argument("--no-cpu", action="store_true")
    p.add_argument("--no-batch", action="store_true")
    p.add_argument("--batch-shots", type=int, default=64)
    p.add_argument("--batch-set", default="both", choices=["both", "c3", "small"],
                   help="which gathers the batch leg times")
    p.add_argument("--no-serve", action="store_true")
    p.add_argument("--no-grad", action="store_true")
    p.add_argument("--grad-nt", type=int, default=3000)
    p.add_argument("--grad-shots", type=int, default=16)
    p.add_argument("--serve-requests", type=int, default=40)
    p.add_argument("--serve-full", action="store_true",
                   help="the request stream as specified (every grid for both kinds, nt 1000..8000); "
                        "use with --serve-requests of a few hundred")
    p.add_argument("--serve-explore", action="store_true",
                   help="time several slice lengths and both scheduling policies")
    return p.parse_args()


def workload(a):
    from viscoelasticinversion_b200 import media

    return media.layered(nx=a.nx, nz=a.nz, nt=a.nt, kind=a.kind, seed=0)


def workload_name(a):
    return f"{a.kind}-layered-{a.nx}x{a.nz}-nt{a.nt}-{a.precision}-3sls-cpml40-freesurface"


class Clocks:
    """nvidia-smi sampling of this GPU's clocks during the timed region."""

    FIELDS = ("uuid,clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.hw_slowdown,"
              "clocks_event_reasons.hw_thermal_slowdown,clocks_event_reasons.sw_thermal_slowdown,"
              "clocks_event_reasons.sw_power_cap")

    def __init__(self, uuid: str):
        self.uuid = uuid
        self.f = tempfile.NamedTemporaryFile("w+", suffix=".csv", delete=False)
        try:
            self.p = subprocess.Popen(["nvidia-smi", f"--query-gpu={self.FIELDS}",
                                       "--format=csv,noheader,nounits", "-lms", "200"],
                                      stdout=self.f, stderr=subprocess.DEVNULL)
        except OSError:
            self.p = None

    def stop(self) -> dict:
        if self.p is None:
            return {"sm_mhz": None, "sm_max_mhz": None, "reasons": ["nvidia-smi unavailable"]}
        self.p.terminate()
        try:
            self.p.wait(timeout=5)
        except subprocess.TimeoutExpired:
            self.p.kill()
        self.f.seek(0)
        rows = [r.split(", ") for r in self.f.read().strip().splitlines()]
        os.unlink(self.f.name)
        mine = [r for r in rows if len(r) >= 8 and (not self.uuid or r[0].strip().endswith(self.uuid))]
        if not mine:
            mine = [r for r in rows if len(r) >= 8]
        sm = [float(r[1]) for r in mine if r[1].strip().replace(".", "").isdigit()]
        mx = [float(r[2]) for r in mine if r[2].strip().replace(".", "").isdigit()]
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        reasons = sorted({names[k] for r in mine for k in range(4) if "Active" == r[4 + k].strip()})
        return {"sm_mhz": statistics.median(sm) if sm else None,
                "sm_max_mhz": max(mx) if mx else None, "reasons": reasons, "samples": len(mine)}


def measured_peaks():
    p = ROOT / "MEASURED_PEAKS.json"
    if p.exists():
        d = json.loads(p.read_text())
        return d.get("hbm_gbs"), "measured"
    return 6650.0, "fallback"


KERNEL_NAMES = {"fused-tma": "k_fused_tma", "fused-tma-1stage": "k_fused_tma", "fused": "k_fused",
                "plain": "k_plain", "split": "k_split", "split-pipelined": "k_split_p",
                "split-ldg": "k_split", "stream": "k_stream", "wave": "k_wave"}
KERNEL_PAIRS = {"split": "k_split_vel_tma + k_split_stress",
                "split-ldg": "k_split_vel_ldg + k_split_stress",
                "split-pipelined": "k_split_vel_p + k_split_stress_p"}


def kernels_per_step(kernel: str, w) -> int:
    """Kernels of this library launched per time step by each path."""
    if kernel.startswith("split"):
        return 2
    if kernel == "wave":  # one persistent launch per solve, not per step
        return 0
    if kernel == "plain":  # velocity, strain, update (+ surface rate, mirror, sources, receivers)
        return 3 + (2 if w.free_surface else 0) + (2 if w.sources else 0) + (1 if w.receivers else 0)
    return 1


def ncu_traffic(name: str):
    """DRAM bytes per time step of the default kernel pair from the
    committed ncu summary of this workload (profiles/), or None."""
    f = ROOT / "profiles" / f"{name}.ncu.md"
    if not f.exists():
        return None
    for line in f.read_text().splitlines():
        if line.startswith("dram_bytes_per_launch:"):
            return float(line.split(":")[1].split()[0])
    return None


# Both CPU legs (cpu_baseline and --impl reference) time the same bounded
# sample: the first CPU_SAMPLE_STEPS steps of the workload (about 4 s of
# FP32 oracle work on 16 host threads for 2048 x 1024).
CPU_SAMPLE_STEPS = 200


def host_cpu():
    """The host's core count, CPU model and OpenMP thread setting."""
    model = ""
    try:
        for line in Path("/proc/cpuinfo").read_text().splitlines():
            if line.startswith("model name"):
                model = line.split(":", 1)[1].strip()
                break
    except OSError:
        pass
    return {"nproc": os.cpu_count(), "cpu_model": model,
            "OMP_NUM_THREADS": os.environ.get("OMP_NUM_THREADS", "unset (all cores)")}


def cpu_sample(w):
    """One timed FP32 oracle run of the bounded sample; (Gpt/s, steps, threads)."""
    import oracle

    oracle.build()
    n = min(CPU_SAMPLE_STEPS, w.nt)
    t0 = time.perf_counter()
    oracle.run(w, n, precision="f32")
    dt = time.perf_counter() - t0
    return w.nx * w.nz * n / dt / 1e9, n, oracle.num_threads()


def cpu_baseline(w):
    """Times the FP32 CPU oracle on the first steps of the workload."""
    cpu_sample(w)  # warm-up (pages, thread pool)
    value, n, threads = cpu_sample(w)
    return {"value": value, "unit": "Gpt/s", "cores": threads, "kind": "port", **host_cpu(),
            "sample": f"first {n} of {w.nt} time steps of the {w.nx}x{w.nz} {w.kind.upper()} "
                      f"workload, FP32 CPU oracle, {threads} OpenMP threads"}


def run_reference(a):
    rank = int(os.environ.get("RANK", "0"))
    if rank != 0:
        return
    w = workload(a)
    # each bench step: the same bounded sample of the solve as the
    # cpu_baseline leg of the GPU arm
    for _ in range(a.warmup):
        cpu_sample(w)
    rates = []
    for _ in range(a.steps):
        value, n, threads = cpu_sample(w)
        rates.append(value)
    value = len(rates) / sum(1.0 / r for r in rates)  # total points / total time
    ms = w.nx * w.nz * n / value / 1e6
    sample = (f"first {n} of {w.nt} time steps of the {w.nx}x{w.nz} {w.kind.upper()} workload per "
              f"step; FP32 CPU restatement of the reference step (the Julia reference does not run "
              f"here), {threads} OpenMP threads")
    print(json.dumps({
        "impl": "reference", "metric": METRIC, "value": value, "unit": "Gpt/s", "n_gpus": a.gpus,
        "steps": a.steps, "warmup": a.warmup, "ms_per_step": ms, "higher_is_better": True,
        "scaling": "weak", "vs_baseline": None, "dtype": "f32", "data": "synthetic",
        "config": {"workload": workload_name(a), "nx": w.nx, "nz": w.nz, "nt": w.nt, "nt_sampled": n,
                   "nsls": w.nsls, "medium": w.kind},
        "cpu_baseline": {"value": value, "unit": "Gpt/s", "cores": threads, "kind": "port",
                         "sample": sample, **host_cpu()},
        "e2e": {"value": value, "unit": "Gpt/s", "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0},
    }), flush=True)


SMALL_GRIDS = ((256, 256), (384, 256), (512, 256))


def measure_batch(a, dev, stream, max_over_ranks, barrier, world, small=False):
    """Shots/s of the batched TTI gather (64 shots, grids from {512²,
    1024x512, 1536x768, 2048x1024}, nt in [1500, 4000], the kernel form the
    tuner picks, one CUDA graph) against the plain path: the default split
    pair (vi_step kernel variant 5), one shot after the other, launched
    step by step, no graph.  small: the same with grids from {256²,
    384x256, 512x256}, where one shot does not fill the GPU.  Each rank
    runs its own gather."""
    import torch

    from viscoelasticinversion_b200 import StepPlan, media
    from viscoelasticinversion_b200.batch import ShotBatch

    rank = int(os.environ.get("RANK", "0"))
    if small:
        ws = media.shot_gather(a.batch_shots, seed=rank, kind="tti", grids=SMALL_GRIDS, pml=20)
    else:
        ws = media.shot_gather(a.batch_shots, seed=rank, kind="tti")
    b = ShotBatch(ws, "f32", device=dev.index)
    b.run()  # tunes the kernel form, captures the graph, runs once
    b.reset()
    form = b.status()
    variant = 5  # plain: the default single-shot split pair, whatever the tuner picked
    torch.cuda.synchronize()
    barrier()
    e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    e0.record(stream)
    b.run()
    e1.record(stream)
    torch.cuda.synchronize()
    batched_ms = max_over_ranks(e0.elapsed_time(e1))
    b.status()
    # plain: one shot at a time, one launch per step, no graph
    plans = [StepPlan.for_workload(w, "f32", device=dev.index) for w in ws]
    per_class = {}
    for w, p, med, st, wav, tr in zip(ws, plans, b.media, b.states, b.wavelets, b.traces):
        for t in st.values():
            t.zero_()
        p.reset()
        p.step(med, st, nsteps=min(w.nt, 20), sources=w.sources, wavelets=wav,
               receivers=w.receivers, traces=tr, variant=variant)  # warm-up
    torch.cuda.synchronize()
    barrier()
    t_plain = 0.0
    for w, p, med, st, wav, tr in zip(ws, plans, b.media, b.states, b.wavelets, b.traces):
        for t in st.values():
            t.zero_()
        p.reset()
        s0, s1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        s0.record(stream)
        p.step(med, st, nsteps=w.nt, sources=w.sources, wavelets=wav, receivers=w.receivers,
               traces=tr, variant=variant)
        s1.record(stream)
        torch.cuda.synchronize()
        ms = s0.elapsed_time(s1)
        t_plain += ms
        key = f"{w.nx}x{w.nz}"
        c = per_class.setdefault(key, {"shots": 0, "plain_ms": 0.0, "point_steps": 0})
        c["shots"] += 1
        c["plain_ms"] += ms
        c["point_steps"] += w.nx * w.nz * w.nt
    plain_ms = max_over_ranks(t_plain)
    for p in plans:
        p.close()
    pts = b.point_steps()
    n = len(ws)
    for c in per_class.values():
        c["plain_gpts"] = c["point_steps"] / (c["plain_ms"] / 1e3) / 1e9
    grids = "256x256..512x256-cpml20" if small else "512..2048x1024"
    out = {"workload": f"tti-gather-{n}shots-grids{grids}-nt1500..4000-f32",
           "shots": n * world, "kernel_form": form,
           "batched_ms": batched_ms, "plain_ms": plain_ms,
           "batched_shots_per_s": n * world / (batched_ms / 1e3),
           "plain_shots_per_s": n * world / (plain_ms / 1e3),
           "speedup": plain_ms / batched_ms,
           "batched_gpts": world * pts / (batched_ms / 1e3) / 1e9,
           "plain_gpts": world * pts / (plain_ms / 1e3) / 1e9,
           "plain_per_grid_class": per_class}
    b.close()
    return out


def measure_serving(a, dev, seed=0):
    """Request serving on the mixed request stream: Poisson arrivals at 50
    requests/s, 70 % forward / 30 % gradient, media from {iso, VTI, TTI}.
    Default (bounded sample, a.serve_requests requests): forward grids from
    {256², 1024x512, 2048x1024, 4096x2048} (4096x2048 as iso/VTI: its tilt
    field takes ~15 s to generate), gradient grids from {256², 1024x512},
    step counts a quarter of [1000, 8000].  a.serve_full: the stream as
    specified for both kinds (every grid, every medium, nt in [1000,
    8000]).  The same
    arrivals are served twice: by the server with time slices given to the
    request with the least remaining work (continuous batching) and FIFO one
    request at a time with no slicing (one lane).  Slices are 1024 steps;
    the continuous run has two lanes, i.e. up to two requests advancing on
    the device at once, each on its own stream.
    Latency = submit to results in host memory (ms)."""
    import dataclasses
    import threading

    import numpy as np

    from viscoelasticinversion_b200 import media
    from viscoelasticinversion_b200.serve import Server

    rng = np.random.default_rng(1234 + seed)
    grids = ((256, 256), (1024, 512), (2048, 1024), (4096, 2048))
    base = {}

    def workload(g, kind):
        if (g, kind) not in base:
            base[(g, kind)] = media.layered(nx=g[0], nz=g[1], nt=8000 if a.serve_full else 2000, kind=kind, seed=7,
                                            pml=20 if g[0] <= 256 else 40, nrec=64,
                                            nlayers=4)
        return base[(g, kind)]

    n = a.serve_requests
    reqs, t = [], 0.0
    for _ in range(n):
        t += rng.exponential(1 / 50.0)
        grad = rng.random() < 0.3
        kind = ("iso", "vti", "tti")[rng.integers(3)]
        g = grids[rng.integers(2)] if grad and not a.serve_full else grids[rng.integers(len(grids))]
        if g == (4096, 2048) and kind == "tti" and not a.serve_full:
            kind = "vti"  # the tilt field of a 4096x2048 TTI medium takes ~15 s to generate
        nt = int(rng.integers(1000, 8001)) if a.serve_full else int(rng.integers(250, 2001))
        w0 = workload(g, kind)
        w = dataclasses.replace(w0, nt=nt, wavelets=w0.wavelets[:, :nt])
        reqs.append((t, grad, w))

    def serve(slice_steps, max_active, policy, lanes):
        srv = Server(device=dev.index, slice_steps=slice_steps, max_active=max_active, policy=policy,
                     lanes=lanes)
        tickets = []

        def submitter():
            t0 = time.perf_counter()
            for at, grad, w in reqs:
                d = at - (time.perf_counter() - t0)
                if d > 0:
                    time.sleep(d)
                obs = np.zeros((2, len(w.receivers), w.nt), np.float32)
                tickets.append(srv.submit_gradient(w, obs, "f32") if grad else srv.submit_forward(w, "f32"))

        t0 = time.perf_counter()
        th = threading.Thread(target=submitter)
        th.start()
        th.join()
        for tk in tickets:
            srv.wait(tk)
        wall = time.perf_counter() - t0
        lat = np.array([srv.poll(tk)[1] for tk in tickets])
        srv.stop()
        return lat, wall

    # warm-up: one short request of every kind on every grid, so one-time
    # kernel loading and set-up fall outside the timed runs
    srv = Server(device=dev.index)
    warm = []
    for (g, kind), w0 in base.items():
        w = dataclasses.replace(w0, nt=8, wavelets=w0.wavelets[:, :8])
        warm.append(srv.submit_forward(w, "f32"))
        if g[0] <= 1024:
            warm.append(srv.submit_gradient(w, np.zeros((2, len(w.receivers), 8), np.float32), "f32"))
    for tk in warm:
        srv.wait(tk)
    srv.stop()
    pts = sum(w.nx * w.nz * w.nt * (3 if grad else 1) for _, grad, w in reqs)
    out = {"workload": (f"{n} requests, Poisson 50/s, 70% forward / 30% gradient, grids 256^2..4096x2048, "
                        "iso/VTI/TTI, nt 1000..8000, f32" if a.serve_full else
                        f"{n} requests, Poisson 50/s, 70% forward / 30% gradient, grids 256^2..4096x2048 "
                        "(gradients 256^2 and 1024x512), iso/VTI/TTI (4096x2048 forward: iso/VTI), "
                        "nt 250..2000 (a quarter of 1000..8000), f32"),
           "forward": sum(1 for _, g, _ in reqs if not g), "gradient": sum(1 for _, g, _ in reqs if g)}
    runs = [("sequential", (1 << 30, 1, "shortest-first", 1))] + [(n_, c) for n_, c in a.serve_policies]
    for name, (sl, ma, pol, ln) in runs:
        lat, wall = serve(sl, ma, pol, ln)
        out[name] = {"p50_ms": float(np.percentile(lat, 50)), "p99_ms": float(np.percentile(lat, 99)),
                     "mean_ms": float(lat.mean()), "requests_per_s": n / wall, "wall_s": wall}
    out["point_steps"] = pts
    return out


def measure_gradient_c4(a, dev):
    """The FWI-gradient workload as specified: 16 shots on the 1024 x 512,
    3000-step VTI model (sources every 1/17 of the width at the workload's
    source depth, 512 receivers), FP32 wavefields, FP64 accumulation of the
    summed gradient through vi_gradient (accumulate), start model smoothed
    100 m, observed data from the true model.  Timed: the 16 gradients.
    Untimed checks on shot 1: the same gradient with FP64 wavefields
    (FP64 observed data) and its central differences (h = 1e-3 of the cell
    value) of the FP64 forward misfit at 20 seeded cells drawn among the
    top decile of |g| in the interior, over the rho, c11, c13, c33, c55 and
    tau planes; and the relative L2 error of the FP32 gradient against the
    FP64 one, per plane."""
    import numpy as np
    import torch
    from scipy.ndimage import gaussian_filter

    from viscoelasticinversion_b200 import StepPlan, media
    from viscoelasticinversion_b200.gradient import misfit_gradient

    nshots = a.grad_shots
    true = media.layered(nx=1024, nz=512, nt=a.grad_nt, kind="vti", seed=3)
    start = {k: gaussian_filter(v, 100.0 / true.dx, mode="nearest") for k, v in true.medium.items()}
    sj = true.sources[0][1]
    xs = [int(round((n + 1) * true.nx / (nshots + 1))) for n in range(nshots)]
    shots = [[(i, sj, 0, 1.0)] for i in xs]

    def observed(plan, wav, srcs):
        med_t = plan.medium_to_device(true.medium)
        obs = torch.zeros(2, len(true.receivers), true.nt, dtype=plan.dtype, device=plan.device)
        st = plan.zeros_state()
        plan.reset()
        plan.step(med_t, st, nsteps=true.nt, sources=srcs, wavelets=wav, receivers=true.receivers, traces=obs)
        plan.status()
        return obs

    plan = StepPlan.for_workload(true, "f32", device=dev.index)
    wav = torch.as_tensor(true.wavelets, dtype=plan.dtype, device=plan.device).contiguous()
    obs = [observed(plan, wav, s) for s in shots]
    med = plan.medium_to_device(start)
    misfit_gradient(plan, med, shots[0], wav, true.receivers, obs[0])  # sizes the checkpoint workspace
    g = torch.zeros(8, plan.nz, plan.nx, dtype=torch.float64, device=plan.device)
    torch.cuda.synchronize()
    t0 = time.perf_counter()
    J = 0.0
    for n in range(nshots):
        Jn, _ = misfit_gradient(plan, med, shots[n], wav, true.receivers, obs[n], grad=g, accumulate=n > 0)
        J += Jn
    torch.cuda.synchronize()
    sec = time.perf_counter() - t0
    g1_32 = misfit_gradient(plan, med, shots[0], wav, true.receivers, obs[0])[1].clone()
    plan.close()
    # FP64 wavefields: gradient of shot 1 and central differences of its misfit
    p64 = StepPlan.for_workload(true, "f64", device=dev.index)
    wav64 = torch.as_tensor(true.wavelets, dtype=torch.float64, device=p64.device).contiguous()
    obs64 = observed(p64, wav64, shots[0])
    med64 = p64.medium_to_device(start)
    _, g64 = misfit_gradient(p64, med64, shots[0], wav64, true.receivers, obs64)
    g64 = g64.clone()
    tr = torch.zeros_like(obs64)

    def misfit64(m):
        st = p64.zeros_state()
        p64.reset()
        p64.step(m, st, nsteps=true.nt, sources=shots[0], wavelets=wav64, receivers=true.receivers, traces=tr)
        p64.status()
        return 0.5 * float(((tr - obs64) ** 2).sum().item())

    planes = {"rho": 0, "c11": 1, "c13": 2, "c33": 4, "c55": 6, "tau": 7}
    rng = np.random.default_rng(7)
    pml = true.pml + 8
    fd = []
    for n in range(20):
        name = list(planes)[n % len(planes)]
        gp = g64[planes[name], pml:-pml, pml:-pml].abs()
        thr = torch.quantile(gp.flatten()[:: max(1, gp.numel() // 1_000_000)], 0.9).item()
        cand = torch.nonzero(gp >= thr).cpu().numpy()
        j, i = cand[rng.integers(len(cand))] + pml
        base = med64[name][j, i].item()
        h = 1e-3 * abs(base)
        med64[name][j, i] = base + h
        jp = misfit64(med64)
        med64[name][j, i] = base - h
        jm = misfit64(med64)
        med64[name][j, i] = base
        d = (jp - jm) / (2 * h)
        adj = g64[planes[name], j, i].item()
        fd.append({"plane": name, "i": int(i), "j": int(j), "fd": d, "adjoint": adj,
                   "rel_err": abs(d - adj) / max(abs(d), 1e-300)})
    p64.close()
    err32 = {name: float(((g1_32[k] - g64[k]).norm() / g64[k].norm()).item()) for name, k in planes.items()}
    rel = [f["rel_err"] for f in fd]
    return {"workload": f"vti-1024x512-nt{true.nt}-f32-gradient-{nshots}shots (start model smoothed 100 m)",
            "shots": nshots, "seconds": sec, "shots_per_s": nshots / sec,
            "gpts": nshots * true.nx * true.nz * true.nt / sec / 1e9, "misfit": J,
            "grad_finite": bool(torch.isfinite(g).all().item()),
            "fd_check": {"reference": "central differences (h = 1e-3 of the cell) of the FP64 GPU forward misfit, "
                                      "shot 1, 20 seeded cells in the top decile of |g|",
                         "max_rel_err": max(rel), "median_rel_err": float(np.median(rel)), "cells": fd},
            "f32_vs_f64_rel_l2": err32}


def measure_accuracy(a, w, plan, med, st, traces, dev):
    """Relative L2 error of the timed solve (its traces and final fields,
    left by the last timed step) against the same solve in FP64 on the GPU,
    over the full step count.  The FP64 kernels are held to the FP64 oracle
    within 1e-10 on this workload over all its steps by
    tests/test_gpu_accuracy.py, so these errors are those against the oracle
    to within 1e-10."""
    import numpy as np
    import torch

    from viscoelasticinversion_b200 import StepPlan

    if a.precision == "f64":
        return None
    ref = StepPlan.for_workload(w, "f64", device=dev.index)
    med64 = ref.medium_to_device(w.medium)
    st64 = ref.zeros_state()
    wav64 = torch.as_tensor(w.wavelets, dtype=torch.float64, device=dev).contiguous()
    tr64 = torch.zeros(2, len(w.receivers), w.nt, dtype=torch.float64, device=dev)
    ref.reset()
    ref.step(med64, st64, nsteps=w.nt, sources=w.sources, wavelets=wav64, receivers=w.receivers,
             traces=tr64, variant=a.variant)
    ref.status()

    def rel(x, y):
        x = x.double()
        n = torch.linalg.vector_norm(y).item()
        return torch.linalg.vector_norm(x - y).item() / (n if n > 0 else 1.0)

    out = {"reference": "the same solve in FP64 on the GPU (FP64 kernels = FP64 oracle to 1e-10 over "
                        "all steps of this workload, tests/test_gpu_accuracy.py)",
           "nt": w.nt, "bar": 1e-5, "traces": rel(traces, tr64),
           "vx": rel(st["v"][0], st64["v"][0]), "vz": rel(st["v"][1], st64["v"][1]),
           "sxx": rel(st["s"][0], st64["s"][0]), "szz": rel(st["s"][1], st64["s"][1]),
           "sxz": rel(st["s"][2], st64["s"][2])}
    if w.nsls:
        m32, m64 = st["m"].reshape(3 * w.nsls, -1), st64["m"].reshape(3 * w.nsls, -1)
        out["m"] = rel(m32, m64)
        out["m_plane_max"] = max(rel(m32[q], m64[q]) for q in range(3 * w.nsls))
    out["max"] = max(v for k, v in out.items() if isinstance(v, float) and k != "bar")
    out["within_bar"] = out["max"] <= 1e-5
    ref.close()
    return out


def run_ours(a):
    import numpy as np
    import torch
    import torch.distributed as dist

    from viscoelasticinversion_b200 import StepPlan

    world = int(os.environ.get("WORLD_SIZE", "1"))
    rank = int(os.environ.get("RANK", "0"))
    local = int(os.environ.get("LOCAL_RANK", "0"))
    torch.cuda.set_device(local)
    dev = torch.device("cuda", local)
    if world > 1:
        import datetime

        dist.init_process_group("nccl", timeout=datetime.timedelta(seconds=300),
                                device_id=dev)

    def barrier():
        if world > 1:
            dist.barrier()

    def max_over_ranks(x: float) -> float:
        if world == 1:
            return x
        t = torch.tensor([x], device=dev, dtype=torch.float64)
        dist.all_reduce(t, op=dist.ReduceOp.MAX)
        return float(t.item())

    w = workload(a)
    esize = 8 if a.precision == "f64" else 4
    plan = StepPlan.for_workload(w, a.precision, device=local)
    med = plan.medium_to_device(w.medium)
    st = plan.zeros_state()
    wav = torch.as_tensor(w.wavelets, dtype=plan.dtype, device=dev).contiguous()
    traces = torch.zeros(2, len(w.receivers), w.nt, dtype=plan.dtype, device=dev)
    stream = torch.cuda.current_stream()
    kev = []

    def one_step(record=False):
        for t in st.values():
            t.zero_()
        plan.reset()
        if record:
            e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
            e0.record(stream)
        plan.step(med, st, nsteps=w.nt, sources=w.sources, wavelets=wav, receivers=w.receivers,
                  traces=traces, variant=a.variant)
        if record:
            e1.record(stream)
            kev.append((e0, e1))

    for _ in range(a.warmup):
        one_step()
    torch.cuda.synchronize()
    barrier()
    torch.cuda.synchronize()
    uuid = str(getattr(torch.cuda.get_device_properties(dev), "uuid", ""))
    clocks = Clocks(uuid)
    t0 = torch.cuda.Event(enable_timing=True)
    t1 = torch.cuda.Event(enable_timing=True)
    t0.record(stream)
    for _ in range(a.steps):
        one_step(record=True)
    t1.record(stream)
    torch.cuda.synchronize()
    barrier()
    torch.cuda.synchronize()
    clk = clocks.stop()
    ms = max_over_ranks(t0.elapsed_time(t1) / a.steps)
    kern_ms = sum(e0.elapsed_time(e1) for e0, e1 in kev) / a.steps
    pts = w.nx * w.nz * w.nt
    value = world * pts / (ms / 1e3) / 1e9
    # a "launch" of the roofline is one time step (the split path is a
    # two-kernel pair per step); gpu_launches counts kernels
    launches_per_step = w.nt
    mean_launch_s = kern_ms / 1e3 / launches_per_step
    # algorithmic bytes of one fused launch: state read+written once, medium
    # read once, CPML psi strips read+written once
    bpt = w.bytes_per_point(esize)
    wx = 2 * w.pml
    hz = w.pml * (1 if w.free_surface else 2)
    psi_bytes = 2 * esize * 4 * (wx * w.nz + w.nx * hz)
    launch_bytes = bpt * w.nx * w.nz + psi_bytes
    achieved = launch_bytes / mean_launch_s / 1e9
    peak, peak_kind = measured_peaks()
    kernel = plan.last_kernel()
    kname = KERNEL_NAMES.get(kernel, kernel)
    kernels = kernels_per_step(kernel, w) * w.nt or 1  # the time-blocked form: one launch per solve
    traffic = ncu_traffic(f"{kname}_{w.kind}_{w.nx}x{w.nz}")

    out = {
        "metric": METRIC, "value": value, "unit": "Gpt/s", "n_gpus": world, "steps": a.steps,
        "warmup": a.warmup, "ms_per_step": ms, "higher_is_better": True, "scaling": "weak",
        "vs_baseline": None, "dtype": a.precision, "data": "synthetic",
        "config": {"workload": workload_name(a), "nx": w.nx, "nz": w.nz, "nt": w.nt,
                   "nsls": w.nsls, "medium": w.kind, "bytes_per_point": bpt,
                   "l2": f"inputs larger than L2 ({launch_bytes / 1e6:.0f} MB per time step)",
                   "parallelism": f"shot-parallel x{world}", "kernel_variant": a.variant,
                   "kernel": kname},
        "gpu_launches": a.steps * kernels,
        "roofline": {"bound": "hbm", "achieved": achieved, "peak": peak, "unit": "GB/s",
                     "frac": achieved / peak, "peak_source": peak_kind,
                     "traffic": traffic, "bytes_per_launch": launch_bytes,
                     "mean_launch_us": mean_launch_s * 1e6,
                     "launch": f"one time step ({KERNEL_PAIRS.get(kernel, kname)})"},
        "clocks": clk,
    }

    if not a.no_accuracy:
        out["accuracy"] = measure_accuracy(a, w, plan, med, st, traces, dev)

    if not a.no_e2e:
        # end to end through vi_forward_host with pinned host buffers
        npdt = np.float64 if a.precision == "f64" else np.float32
        tdt = torch.float64 if a.precision == "f64" else torch.float32
        med_h = {k: torch.from_numpy(np.ascontiguousarray(v, dtype=npdt)).pin_memory()
                 for k, v in w.medium.items()}
        wav_h = torch.from_numpy(np.ascontiguousarray(w.wavelets, dtype=npdt)).pin_memory()
        tr_h = torch.empty(2, len(w.receivers), w.nt, dtype=tdt).pin_memory()
        h2d = sum(t.numel() * t.element_size() for t in med_h.values()) + wav_h.numel() * esize
        d2h = tr_h.numel() * esize
        for _ in range(max(1, a.warmup // 2)):
            plan.forward_host(med_h, w.sources, wav_h, w.receivers, w.nt, traces_out=tr_h)
        torch.cuda.synchronize()
        barrier()
        e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        e0.record(stream)
        for _ in range(a.steps):
            plan.forward_host(med_h, w.sources, wav_h, w.receivers, w.nt, traces_out=tr_h)
        e1.record(stream)
        torch.cuda.synchronize()
        barrier()
        ems = max_over_ranks(e0.elapsed_time(e1) / a.steps)
        out["e2e"] = {"value": world * pts / (ems / 1e3) / 1e9, "unit": "Gpt/s",
                      "h2d_bytes_per_step": h2d, "d2h_bytes_per_step": d2h, "ms_per_step": ems,
                      "api": "vi_forward_host"}
        out["gpu_launches"] += a.steps * kernels

    if not a.no_batch:
        if a.batch_set in ("both", "c3"):
            out["batched"] = measure_batch(a, dev, stream, max_over_ranks, barrier, world)
        if a.batch_set in ("both", "small"):
            out["batched_small"] = measure_batch(a, dev, stream, max_over_ranks, barrier, world, small=True)
    if not a.no_grad and rank == 0:
        out["gradient"] = measure_gradient_c4(a, dev)
    if not a.no_serve and rank == 0 and world == 1:
        # the server allocates its own device buffers: hand back torch's cache
        torch.cuda.empty_cache()
        a.serve_policies = [("continuous", (1024, 64, "shortest-first", 2))]
        if a.serve_explore:
            a.serve_policies += [("one-lane", (1024, 64, "shortest-first", 1)),
                                 ("four-lanes", (1024, 64, "shortest-first", 4)),
                                 ("eight-lanes", (1024, 64, "shortest-first", 8)),
                                 ("round-robin-256", (256, 64, "round-robin", 2)),
                                 ("shortest-first-4096", (4096, 64, "shortest-first", 2))]
        out["serving"] = measure_serving(a, dev)
    if rank == 0 and world == 1 and not a.no_cpu:
        out["cpu_baseline"] = cpu_baseline(w)
    if rank == 0:
        print(json.dumps(out), flush=True)
    plan.close()
    if world > 1:
        dist.destroy_process_group()


def main():
    a = parse_args()
    if a.impl == "reference":
        run_reference(a)
    else:
        run_ours(a)


if __name__ == "__main__":
    main()
