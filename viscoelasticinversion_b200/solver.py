"""Host side of the time step: a plan object over the C ABI.

torch provides device memory and streams only; every computation runs in
libvisco_b200.so.  Arrays follow the reference's layout turned row-major:
a Julia column-major [Nx, Nz] plane is a C-order [nz, nx] tensor here, the
stacked Fields s[Nx,Nz,3] / v[Nx,Nz,2] / M[Nx,Nz,N,3] (visco-kernels.jl:102-106)
are [3, nz, nx] / [2, nz, nx] / [3, N, nz, nx].
"""
from __future__ import annotations

import ctypes as C
from dataclasses import dataclass

import numpy as np
import torch

from . import _abi
from ._abi import (ViConfig, ViFields, ViMedium, ViReceiver, ViShot, ViSource, check, lib,
                   MEDIUM_KINDS, PRECISIONS, VI_F32, VI_F64)

MEDIUM_NAMES = ("rho", "c11", "c13", "c15", "c33", "c35", "c55", "tau")
# vi_config.free_surface: 1 = stress imaging (CPML.jl:366-393), 2 = H-AFDA
# one-sided derivatives (free-surface-kernels.jl, Stencil.jl:52-105)
FREE_SURFACE_IMAGING, FREE_SURFACE_HAFDA = 1, 2


@dataclass
class CPMLSpec:
    """CPMLConfig(;thickness, d0, alpha_max, kappa_max, power, left, right,
    top, bottom, vmax, dx, reflection_coef) — sciml_solver/CPML.jl:28-63."""

    thickness: int = 10
    d0: float | None = None
    alpha_max: float = 0.0
    kappa_max: float = 1.0
    power: float = 2.0
    left: bool = True
    right: bool = True
    top: bool = False
    bottom: bool = True
    vmax: float | None = None
    reflection_coef: float = 1e-5


def make_config(nx, nz, dx, dz, dt, kind="iso", precision="f32", taus=(), free_surface=True,
                cpml: CPMLSpec | None = None, vmax: float | None = None) -> ViConfig:
    c = ViConfig()
    c.nx, c.nz, c.dx, c.dz, c.dt = int(nx), int(nz), float(dx), float(dz), float(dt)
    c.medium = MEDIUM_KINDS[kind]
    c.precision = PRECISIONS[precision]
    c.nsls = len(taus)
    for n, t in enumerate(taus):
        c.tau_sls[n] = float(t)
    # False / 0: none; True / 1: stress imaging; 2 (FREE_SURFACE_HAFDA): H-AFDA
    c.free_surface = FREE_SURFACE_HAFDA if free_surface == FREE_SURFACE_HAFDA else int(bool(free_surface))
    if cpml is not None and cpml.thickness > 0:
        c.pml_thickness = cpml.thickness
        c.pml_left, c.pml_right = int(cpml.left), int(cpml.right)
        c.pml_top, c.pml_bottom = int(cpml.top), int(cpml.bottom)
        c.pml_d0 = float(cpml.d0) if cpml.d0 is not None else 0.0
        c.pml_vmax = float(cpml.vmax if cpml.vmax is not None else (vmax or 0.0))
        c.pml_reflection = cpml.reflection_coef
        c.pml_power = cpml.power
        c.pml_alpha_max = cpml.alpha_max
        c.pml_kappa_max = cpml.kappa_max
    else:
        c.pml_vmax = float(vmax or 0.0)
        c.pml_reflection = 1e-5
        c.pml_power = 2.0
        c.pml_kappa_max = 1.0
    return c


def config_from_workload(w, precision="f32") -> ViConfig:
    cp = CPMLSpec(thickness=w.pml, alpha_max=w.pml_alpha_max, top=not w.free_surface,
                  vmax=w.pml_vmax)
    c = make_config(w.nx, w.nz, w.dx, w.dz, w.dt, w.kind, precision, w.taus, w.free_surface, cp)
    return c


def _ptr(t) -> int | None:
    return None if t is None else t.data_ptr()


def _stream_handle(stream) -> int | None:
    if stream is None:
        return torch.cuda.current_stream().cuda_stream
    return getattr(stream, "cuda_stream", stream)


# tune() choices per grid class: (nx, nz, medium, nsls, precision, free surface)
_TUNED: dict = {}


class StepPlan:
    """Owns one vi_plan: CPML profiles and ψ memory, the fused path's second
    state copy and the staged source/receiver lists."""

    def __init__(self, cfg: ViConfig, device=None):
        self.cfg = cfg
        self.device = torch.device("cuda", torch.cuda.current_device() if device is None else device)
        self.dtype = torch.float64 if cfg.precision == VI_F64 else torch.float32
        self._h = C.c_void_p()
        with torch.cuda.device(self.device):
            check(lib().vi_plan_create(C.byref(cfg), C.byref(self._h)))

    @classmethod
    def for_workload(cls, w, precision="f32", device=None):
        return cls(config_from_workload(w, precision), device)

    # ---- helpers ---------------------------------------------------------
    @property
    def nx(self):
        return self.cfg.nx

    @property
    def nz(self):
        return self.cfg.nz

    @property
    def nsls(self):
        return self.cfg.nsls

    def close(self):
        if self._h:
            lib().vi_plan_destroy(self._h)
            self._h = C.c_void_p()

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    def workspace_bytes(self) -> int:
        b = C.c_int64()
        check(lib().vi_plan_workspace_bytes(self._h, C.byref(b)))
        return b.value

    def reset(self, stream=None):
        check(lib().vi_plan_reset(self._h, _stream_handle(stream)))

    def status(self, stream=None):
        """Synchronizes and raises if a bounded in-kernel wait gave up."""
        check(lib().vi_plan_status(self._h, _stream_handle(stream)))

    def last_kernel(self) -> str:
        k = C.c_int32()
        check(lib().vi_plan_last_kernel(self._h, C.byref(k)))
        return {0: "none", 1: "plain", 2: "fused", 3: "fused-tma", 4: "fused-tma-1stage",
                5: "split", 6: "split-pipelined", 7: "stream", 8: "split-ldg", 9: "wave"}[k.value]

    def zeros_state(self) -> dict:
        """Zeroed device state {vx, vz, sxx, szz, sxz, m}."""
        kw = dict(device=self.device, dtype=self.dtype)
        v = torch.zeros(2, self.nz, self.nx, **kw)
        s = torch.zeros(3, self.nz, self.nx, **kw)
        m = torch.zeros(3, max(self.nsls, 1), self.nz, self.nx, **kw)
        return {"v": v, "s": s, "m": m}

    def medium_to_device(self, medium: dict) -> dict:
        return {k: torch.as_tensor(np.ascontiguousarray(v), dtype=self.dtype).to(self.device)
                for k, v in medium.items()}

    @staticmethod
    def _medium_struct(med: dict) -> ViMedium:
        m = ViMedium()
        for k in MEDIUM_NAMES:
            t = med.get(k)
            if t is not None:
                if not t.is_contiguous():
                    raise ValueError(f"medium plane {k} must be contiguous")
                setattr(m, k, t.data_ptr())
        return m

    @staticmethod
    def fields_struct(vx, vz, sxx, szz, sxz, m=None) -> ViFields:
        f = ViFields()
        for name, t in (("vx", vx), ("vz", vz), ("sxx", sxx), ("szz", szz), ("sxz", sxz)):
            if not t.is_contiguous():
                raise ValueError(f"field {name} must be contiguous")
            setattr(f, name, t.data_ptr())
        if m is not None:
            f.m = m.data_ptr()
            f.m_plane_stride = m.shape[-1] * m.shape[-2]
        return f

    def _shot(self, sources, wavelets, receivers, traces):
        keep = []
        shot = ViShot()
        if sources:
            src = (ViSource * len(sources))()
            for q, s in enumerate(sources):
                i, j, kind, amp = s
                src[q].i, src[q].j, src[q].kind, src[q].amp = int(i), int(j), int(kind), float(amp)
            if wavelets is None or wavelets.dim() != 2 or wavelets.shape[0] != len(sources):
                raise ValueError("wavelets must be a [nsrc, nt] device tensor")
            shot.nsrc = len(sources)
            shot.src_host = src
            shot.wavelet_dev = wavelets.data_ptr()
            shot.wavelet_nt = wavelets.shape[1]
            keep.append(src)
        if receivers:
            rec = (ViReceiver * len(receivers))()
            for r, (i, j) in enumerate(receivers):
                rec[r].i, rec[r].j = int(i), int(j)
            shot.nrec = len(receivers)
            shot.rec_host = rec
            if traces is not None:
                if traces.shape[:2] != (2, len(receivers)):
                    raise ValueError("traces must be [2, nrec, nt]")
                shot.traces_dev = traces.data_ptr()
                shot.traces_nt = traces.shape[2]
            keep.append(rec)
        return shot, keep

    # ---- stepping ----------------------------------------------------------
    # (depth, lag) of the time-blocked step tried by tune()
    WAVE_CANDIDATES = ((2, 4), (4, 4), (4, 8), (8, 8), (16, 8))

    def tune(self, medium: dict, nsteps: int = 32, reps: int = 2, candidates=None) -> dict:
        """Autotuner of the step's kernel form for this grid class: times
        the split pair (kernel variant 5) and the time-blocked step (variant
        9) at each (depth, lag) on a scratch state of this plan with the
        caller's medium, keeps the fastest, and makes it the choice of
        step(..., variant="auto") for every plan of the same class (grid,
        medium kind, N_sls, precision, free surface).  Returns
        {"variant", "depth", "lag", "us_per_step": {form: us}}."""
        key = self._tune_key()
        st = self.zeros_state()
        table = {}
        forms = [(5, 0, 0)]
        if self.cfg.medium != _abi.VI_MEDIUM_TTI and self.cfg.precision != _abi.VI_F32C and \
                self.cfg.free_surface != FREE_SURFACE_HAFDA and self.nx % 4 == 0:
            forms += [(9, k, d) for k, d in (candidates or self.WAVE_CANDIDATES)]
        best = None
        for variant, k, d in forms:
            if variant == 9:
                self.set_wave(k, d)
            self.step(medium, st, nsteps=nsteps, variant=variant)  # warm-up
            ms = []
            for _ in range(reps):
                e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
                e0.record()
                self.step(medium, st, nsteps=nsteps, variant=variant)
                e1.record()
                e1.synchronize()
                ms.append(e0.elapsed_time(e1))
            us = min(ms) * 1e3 / nsteps
            name = "split" if variant == 5 else f"wave k={k} d={d}"
            table[name] = us
            if best is None or us < best[0]:
                best = (us, variant, k, d)
        del st
        self.reset()
        _, variant, k, d = best
        self.set_wave(k, d)
        choice = {"variant": variant, "depth": k, "lag": d, "us_per_step": table}
        _TUNED[key] = choice
        return choice

    def _tune_key(self):
        c = self.cfg
        return (c.nx, c.nz, c.medium, c.nsls, c.precision, c.free_surface)

    def set_wave(self, depth: int = 0, lag: int = 0):
        """Time blocking of kernel variant 9: sweeps of `depth` steps with
        `lag` bands between consecutive passes (0 = the built-in defaults)."""
        check(lib().vi_plan_set_wave(self._h, int(depth), int(lag)))

    def step(self, medium: dict, state: dict, nsteps: int = 1, it0: int = 0, sources=None,
             wavelets=None, receivers=None, traces=None, variant=0, stream=None):
        """Advances state {v, s, m} by nsteps in place (asynchronous on stream).
        variant="auto": the form tune() chose for this grid class (tuned
        on first use)."""
        if variant == "auto":
            choice = _TUNED.get(self._tune_key())
            if choice is None:
                choice = self.tune(medium)
            self.set_wave(choice["depth"], choice["lag"])
            variant = choice["variant"]
        v, s, m = state["v"], state["s"], state.get("m")
        f = self.fields_struct(v[0], v[1], s[0], s[1], s[2], m if self.nsls else None)
        med = self._medium_struct(medium)
        shot, keep = self._shot(sources, wavelets, receivers, traces)
        check(lib().vi_step(self._h, C.byref(med), C.byref(f),
                            C.byref(shot) if (sources or receivers) else None, int(it0),
                            int(nsteps), int(variant), _stream_handle(stream)))
        del keep

    def forward_host(self, medium_host: dict, sources, wavelets_host: np.ndarray, receivers,
                     nt: int, return_fields: bool = False, traces_out=None):
        """Whole solve through vi_forward_host with host (numpy or pinned
        torch) buffers.  Returns traces [2, nrec, nt] (and final fields);
        traces_out, if given, is the host buffer the traces land in."""
        npdt = np.float64 if self.cfg.precision == VI_F64 else np.float32
        keep = []
        med = ViMedium()
        for k in MEDIUM_NAMES:
            a = medium_host.get(k)
            if a is None:
                continue
            if isinstance(a, torch.Tensor):
                setattr(med, k, a.data_ptr())
            else:
                a = np.ascontiguousarray(a, dtype=npdt)
                keep.append(a)
                setattr(med, k, a.ctypes.data)
        src = (ViSource * max(len(sources), 1))()
        for q, (i, j, kind, amp) in enumerate(sources):
            src[q].i, src[q].j, src[q].kind, src[q].amp = i, j, kind, amp
        rec = (ViReceiver * max(len(receivers), 1))()
        for r, (i, j) in enumerate(receivers):
            rec[r].i, rec[r].j = i, j
        if isinstance(wavelets_host, torch.Tensor):
            wptr = wavelets_host.data_ptr()
        else:
            wv = np.ascontiguousarray(wavelets_host[:, :nt], dtype=npdt)
            keep.append(wv)
            wptr = wv.ctypes.data
        if traces_out is None:
            traces = np.zeros((2, len(receivers), nt), npdt)
            tptr = traces.ctypes.data
        else:
            if tuple(traces_out.shape) != (2, len(receivers), nt):
                raise ValueError("traces_out must be [2, nrec, nt]")
            traces = traces_out
            tptr = traces_out.data_ptr() if isinstance(traces_out, torch.Tensor) else traces_out.ctypes.data
        fin = None
        fptr = None
        if return_fields:
            fin = {"v": np.zeros((2, self.nz, self.nx), npdt),
                   "s": np.zeros((3, self.nz, self.nx), npdt),
                   "m": np.zeros((3 * max(self.nsls, 1), self.nz, self.nx), npdt)}
            ff = ViFields()
            ff.vx, ff.vz = fin["v"][0].ctypes.data, fin["v"][1].ctypes.data
            ff.sxx, ff.szz, ff.sxz = (fin["s"][k].ctypes.data for k in range(3))
            ff.m = fin["m"].ctypes.data
            ff.m_plane_stride = self.nx * self.nz
            fptr = C.byref(ff)
        with torch.cuda.device(self.device):
            check(lib().vi_forward_host(self._h, C.byref(med), len(sources), src, wptr,
                                        len(receivers), rec, int(nt), tptr, fptr))
        return (traces, fin) if return_fields else traces


def diff(u: torch.Tensor, op: str, h: float = 1.0, stream=None) -> torch.Tensor:
    """Array form of the staggered operators ddxp/ddxm/ddzp/ddzm
    (diff-funcs.jl:3-32) over the update region of one [nz, nx] plane."""
    ops = {"ddxp": 0, "ddxm": 1, "ddzp": 2, "ddzm": 3}
    if not u.is_cuda or not u.is_contiguous() or u.dim() != 2:
        raise ValueError("u must be a contiguous 2D CUDA tensor")
    prec = VI_F64 if u.dtype == torch.float64 else VI_F32
    if u.dtype not in (torch.float32, torch.float64):
        raise ValueError("u must be float32 or float64")
    du = torch.zeros_like(u)
    check(lib().vi_diff(prec, ops[op], u.data_ptr(), du.data_ptr(), u.shape[1], u.shape[0],
                        float(h), _stream_handle(stream)))
    return du


__all__ = ["StepPlan", "CPMLSpec", "make_config", "config_from_workload", "diff", "_abi"]
