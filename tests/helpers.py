"""Shared helpers of the GPU tests: run a workload through the C ABI and
compare with the oracle."""
from __future__ import annotations

import numpy as np
import torch

from viscoelasticinversion_b200 import StepPlan


def rel_l2(a, b) -> float:
    a = np.asarray(a, dtype=np.float64)
    b = np.asarray(b, dtype=np.float64)
    nb = np.linalg.norm(b)
    return float(np.linalg.norm(a - b) / (nb if nb > 0 else 1.0))


def run_gpu(w, precision="f32", variant=2, chunks=None, nt=None, info=None):
    """Runs w from rest on cuda:0 through vi_step; returns (traces, state)
    as float64 numpy arrays.  `info`, if a dict, receives the kernel the
    plan ran."""
    nt = w.nt if nt is None else nt
    plan = StepPlan.for_workload(w, precision)
    med = plan.medium_to_device(w.medium)
    st = plan.zeros_state()
    wav = torch.as_tensor(w.wavelets[:, :nt], dtype=plan.dtype, device=plan.device).contiguous()
    traces = torch.zeros(2, len(w.receivers), nt, dtype=plan.dtype, device=plan.device)
    chunks = chunks or [nt]
    it = 0
    for n in chunks:
        plan.step(med, st, nsteps=n, it0=it, sources=w.sources, wavelets=wav,
                  receivers=w.receivers, traces=traces, variant=variant)
        it += n
    plan.status()
    if info is not None:
        info["kernel"] = plan.last_kernel()
    out = {k: v.double().cpu().numpy() for k, v in st.items()}
    out["m"] = out["m"].reshape(-1, w.nz, w.nx)
    plan.close()
    return traces.double().cpu().numpy(), out


def compare(tr, st, tr_ref, st_ref, nsls) -> dict:
    """Relative L2 errors of the traces and each final field."""
    err = {"traces": rel_l2(tr, tr_ref),
           "vx": rel_l2(st["v"][0], st_ref.v[0]), "vz": rel_l2(st["v"][1], st_ref.v[1]),
           "sxx": rel_l2(st["s"][0], st_ref.s[0]), "szz": rel_l2(st["s"][1], st_ref.s[1]),
           "sxz": rel_l2(st["s"][2], st_ref.s[2])}
    if nsls:
        err["m"] = rel_l2(st["m"][:3 * nsls], st_ref.m[:3 * nsls])
    return err
