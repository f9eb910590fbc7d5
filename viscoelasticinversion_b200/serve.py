"""Request server over the vi_serve C ABI.

Forward solves and misfit gradients are submitted from host code and run
by the library's worker lanes: admission against an HBM budget, time
slices of slice_steps steps given to the idle resident requests with the
least remaining work (requests join and leave between slices, short ones
preempt long ones), gradients run whole, and `lanes` requests advance on
the device at once, each on its own CUDA stream.  The reference solves one
problem per call (sciml_solver/ViscoelasticProblem.jl:273-309); this is
its time step served to many callers.
"""
from __future__ import annotations

import ctypes as C
from dataclasses import dataclass, field

import numpy as np

from ._abi import (ViMedium, ViReceiver, ViRequest, ViServeConfig, ViSource, VI_F64,
                   VI_REQ_DONE, VI_REQ_FAILED, VI_REQ_FORWARD, VI_REQ_GRADIENT, check, lib)
from .solver import MEDIUM_NAMES, config_from_workload

STATES = {0: "queued", 1: "running", 2: "done", 3: "failed"}


@dataclass
class Ticket:
    """A submitted request: its id and the host buffers it reads and writes
    (kept alive here until the server is done with them)."""
    id: int
    kind: str
    traces: np.ndarray
    grad: np.ndarray | None = None
    misfit: np.ndarray | None = None
    _keep: list = field(default_factory=list, repr=False)


class Server:
    def __init__(self, device: int = 0, hbm_budget_bytes: int = 0, slice_steps: int = 1024,
                 max_active: int = 64, policy: str = "shortest-first", lanes: int = 2):
        """lanes: requests advancing on the device at once (each resident
        request has its own CUDA stream; 1 = one at a time)."""
        pol = {"shortest-first": 0, "round-robin": 1}[policy]
        cfg = ViServeConfig(device=device, slice_steps=slice_steps, max_active=max_active,
                            policy=pol, hbm_budget_bytes=hbm_budget_bytes, lanes=lanes)
        self._h = C.c_void_p()
        check(lib().vi_serve_start(C.byref(cfg), C.byref(self._h)))

    def _request(self, w, precision, kind, obs=None):
        cfg = config_from_workload(w, precision)
        npdt = np.float64 if cfg.precision == VI_F64 else np.float32
        keep = []
        r = ViRequest()
        r.kind, r.nt, r.cfg = kind, int(w.nt), cfg
        med = ViMedium()
        for k in MEDIUM_NAMES:
            if k in w.medium:
                a = np.ascontiguousarray(w.medium[k], dtype=npdt)
                keep.append(a)
                setattr(med, k, a.ctypes.data)
        r.medium_host = med
        src = (ViSource * max(len(w.sources), 1))()
        for q, (i, j, k, amp) in enumerate(w.sources):
            src[q].i, src[q].j, src[q].kind, src[q].amp = int(i), int(j), int(k), float(amp)
        rec = (ViReceiver * max(len(w.receivers), 1))()
        for q, (i, j) in enumerate(w.receivers):
            rec[q].i, rec[q].j = int(i), int(j)
        wav = np.ascontiguousarray(w.wavelets, dtype=npdt)
        traces = np.zeros((2, len(w.receivers), w.nt), npdt)
        keep += [src, rec, wav]
        r.nsrc, r.src_host = len(w.sources), C.cast(src, C.POINTER(ViSource))
        r.wavelet_nt, r.wavelet_host = wav.shape[1], wav.ctypes.data
        r.nrec, r.rec_host = len(w.receivers), C.cast(rec, C.POINTER(ViReceiver))
        r.traces_host = traces.ctypes.data
        grad = misfit = None
        if kind == VI_REQ_GRADIENT:
            o = np.ascontiguousarray(obs, dtype=npdt)
            if o.shape != traces.shape:
                raise ValueError("obs must be [2, nrec, nt]")
            grad = np.zeros((8, w.nz, w.nx))
            misfit = np.zeros(1)
            keep.append(o)
            r.obs_host, r.grad_host, r.misfit_host = o.ctypes.data, grad.ctypes.data, misfit.ctypes.data
        return r, traces, grad, misfit, keep

    def submit_forward(self, w, precision: str = "f32") -> Ticket:
        r, traces, _, _, keep = self._request(w, precision, VI_REQ_FORWARD)
        t = C.c_uint64()
        check(lib().vi_serve_submit(self._h, C.byref(r), C.byref(t)))
        return Ticket(t.value, "forward", traces, _keep=keep + [r])

    def submit_gradient(self, w, obs, precision: str = "f64") -> Ticket:
        r, traces, grad, misfit, keep = self._request(w, precision, VI_REQ_GRADIENT, obs)
        t = C.c_uint64()
        check(lib().vi_serve_submit(self._h, C.byref(r), C.byref(t)))
        return Ticket(t.value, "gradient", traces, grad, misfit, _keep=keep + [r])

    def poll(self, ticket: Ticket):
        """(state name, latency in ms so far or submit-to-done)."""
        st, lat = C.c_int32(), C.c_double()
        check(lib().vi_serve_poll(self._h, ticket.id, C.byref(st), C.byref(lat)))
        return STATES[st.value], lat.value

    def wait(self, ticket: Ticket, timeout_s: float = -1.0) -> str:
        st = C.c_int32()
        check(lib().vi_serve_wait(self._h, ticket.id, float(timeout_s), C.byref(st)))
        return STATES[st.value]

    def stop(self):
        if self._h:
            check(lib().vi_serve_stop(self._h))
            self._h = C.c_void_p()

    def __del__(self):
        try:
            self.stop()
        except Exception:
            pass
