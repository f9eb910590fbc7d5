"""CPU oracle of the viscoelastic staggered-grid step — TEST INFRASTRUCTURE.

Only tests/, __graft_entry__.smoke() and bench.py's CPU-baseline /
reference leg may import this package, and only as the checker or the
timed CPU baseline.  The product (viscoelasticinversion_b200) never does.

liboracle.so is built from visco_oracle.c by the Makefile beside it
(`make -C oracle`); build() does that on demand.
"""
from __future__ import annotations

import ctypes as C
import os
import subprocess
from pathlib import Path

import numpy as np

from viscoelasticinversion_b200._abi import (ViConfig, ViMedium, ViReceiver, ViSource,
                                             MEDIUM_KINDS, VI_F32, VI_F64)

HERE = Path(__file__).resolve().parent
LIB = HERE / "liboracle.so"


class OrState(C.Structure):
    _fields_ = [(n, C.c_void_p) for n in ("vx", "vz", "sxx", "szz", "sxz", "m", "psi")]


_lib = None


def build() -> Path:
    srcs = [HERE / "visco_oracle.c", HERE / "oracle_step.inc", HERE / "oracle_adjoint.c",
            HERE / "visco_oracle.h", HERE / "Makefile"]
    if not LIB.exists() or LIB.stat().st_mtime < max(s.stat().st_mtime for s in srcs):
        subprocess.run(["make", "-s", "-C", str(HERE)], check=True)
    return LIB


def lib():
    global _lib
    if _lib is None:
        build()
        h = C.CDLL(str(LIB))
        for sfx, real in (("f64", C.c_double), ("f32", C.c_float)):
            fn = getattr(h, f"or_run_{sfx}")
            fn.restype = C.c_int
            fn.argtypes = [C.POINTER(ViConfig), C.POINTER(ViMedium), C.POINTER(OrState),
                           C.c_int, C.c_int, C.c_int, C.POINTER(ViSource), C.POINTER(real),
                           C.c_int, C.c_int, C.POINTER(ViReceiver), C.POINTER(real), C.c_int]
        h.or_cpml_profile.restype = C.c_int
        h.or_cpml_profile.argtypes = [C.POINTER(ViConfig), C.c_int, C.c_int] + [
            C.POINTER(C.c_double)] * 5
        h.or_ricker.restype = C.c_double
        h.or_ricker.argtypes = [C.c_double, C.c_double]
        h.or_stencil8.restype = None
        h.or_stencil8.argtypes = [C.POINTER(C.c_double)]
        h.or_num_threads.restype = C.c_int
        h.or_adjoint_step_f64.restype = C.c_int
        h.or_adjoint_step_f64.argtypes = [C.POINTER(ViConfig), C.POINTER(ViMedium), C.POINTER(OrState)]
        h.or_gradient_f64.restype = C.c_int
        h.or_gradient_f64.argtypes = [C.POINTER(ViConfig), C.POINTER(ViMedium), C.c_int, C.POINTER(ViSource),
                                      C.POINTER(C.c_double), C.c_int, C.c_int, C.POINTER(ViReceiver),
                                      C.POINTER(C.c_double), C.c_int, C.POINTER(C.c_double),
                                      C.POINTER(C.c_double)]
        h.or_afda_weights.restype = None
        h.or_afda_weights.argtypes = [C.POINTER(C.c_double)]
        _lib = h
    return _lib


def make_config(w, precision: str = "f64") -> ViConfig:
    """ViConfig of a Workload (viscoelasticinversion_b200.media.Workload)."""
    c = ViConfig()
    c.nx, c.nz, c.dx, c.dz, c.dt = w.nx, w.nz, w.dx, w.dz, w.dt
    c.medium = MEDIUM_KINDS[w.kind]
    c.precision = VI_F64 if precision == "f64" else VI_F32
    c.nsls = w.nsls
    for n, t in enumerate(w.taus):
        c.tau_sls[n] = float(t)
    c.free_surface = 2 if w.free_surface == 2 else int(bool(w.free_surface))
    c.pml_thickness = w.pml
    c.pml_left = c.pml_right = c.pml_bottom = 1
    c.pml_top = 0 if w.free_surface else 1
    c.pml_d0 = 0.0
    c.pml_vmax = w.pml_vmax
    c.pml_reflection = 1e-5
    c.pml_power = 2.0
    c.pml_alpha_max = w.pml_alpha_max
    c.pml_kappa_max = 1.0
    return c


class OracleState:
    """Full-plane oracle state (numpy)."""

    def __init__(self, nx, nz, nsls, dtype):
        self.v = np.zeros((2, nz, nx), dtype)
        self.s = np.zeros((3, nz, nx), dtype)
        self.m = np.zeros((3 * max(nsls, 1), nz, nx), dtype)
        self.psi = np.zeros((8, nz, nx), dtype)

    def struct(self) -> OrState:
        st = OrState()
        st.vx = self.v[0].ctypes.data
        st.vz = self.v[1].ctypes.data
        st.sxx = self.s[0].ctypes.data
        st.szz = self.s[1].ctypes.data
        st.sxz = self.s[2].ctypes.data
        st.m = self.m.ctypes.data
        st.psi = self.psi.ctypes.data
        return st

    def fields(self) -> dict:
        return {"vx": self.v[0], "vz": self.v[1], "sxx": self.s[0], "szz": self.s[1],
                "sxz": self.s[2], "m": self.m}


def run(w, nsteps: int | None = None, precision: str = "f64", state: OracleState | None = None,
        it0: int = 0, cfg: ViConfig | None = None):
    """Runs the oracle on workload w.  Returns (traces [2, nrec, nt], state)."""
    dt = np.float64 if precision == "f64" else np.float32
    nsteps = w.nt if nsteps is None else nsteps
    cfg = cfg or make_config(w, precision)
    med_arrays = {k: np.ascontiguousarray(v, dtype=dt) for k, v in w.medium.items()}
    med = ViMedium()
    for k, a in med_arrays.items():
        setattr(med, k, a.ctypes.data)
    if state is None:
        state = OracleState(w.nx, w.nz, w.nsls, dt)
    st = state.struct()
    nsrc = len(w.sources)
    src = (ViSource * max(nsrc, 1))()
    for q, (i, j, kind, amp) in enumerate(w.sources):
        src[q].i, src[q].j, src[q].kind, src[q].amp = i, j, kind, amp
    wav = np.ascontiguousarray(w.wavelets, dtype=dt)
    nrec = len(w.receivers)
    rec = (ViReceiver * max(nrec, 1))()
    for r, (i, j) in enumerate(w.receivers):
        rec[r].i, rec[r].j = i, j
    tnt = it0 + nsteps
    traces = np.zeros((2, nrec, tnt), dt)
    real = C.c_double if precision == "f64" else C.c_float
    fn = lib().or_run_f64 if precision == "f64" else lib().or_run_f32
    rc = fn(C.byref(cfg), C.byref(med), C.byref(st), it0, nsteps, nsrc, src,
            wav.ctypes.data_as(C.POINTER(real)), wav.shape[1], nrec, rec,
            traces.ctypes.data_as(C.POINTER(real)), tnt)
    if rc != 0:
        raise RuntimeError(f"oracle failed with status {rc}")
    return traces, state


def _medium_struct(w, dt=np.float64):
    arrays = {k: np.ascontiguousarray(v, dtype=dt) for k, v in w.medium.items()}
    med = ViMedium()
    for k, a in arrays.items():
        setattr(med, k, a.ctypes.data)
    return med, arrays


def adjoint_step(w, state: OracleState) -> OracleState:
    """Applies the transpose of one FP64 step (no sources) to the adjoint
    state in place (the dot-product partner of run(w, 1) without sources)."""
    cfg = make_config(w, "f64")
    med, keep = _medium_struct(w)
    st = state.struct()
    rc = lib().or_adjoint_step_f64(C.byref(cfg), C.byref(med), C.byref(st))
    if rc != 0:
        raise RuntimeError(f"oracle adjoint failed with status {rc}")
    del keep
    return state


def gradient(w, obs: np.ndarray, nt: int | None = None):
    """(J, grad [8, nz, nx]) of the misfit 1/2 sum (d - obs)^2 of an
    nt-step FP64 run from rest, by the oracle's discrete adjoint (every
    forward state kept in memory: small grids only)."""
    nt = w.nt if nt is None else nt
    cfg = make_config(w, "f64")
    med, keep = _medium_struct(w)
    nsrc = len(w.sources)
    src = (ViSource * max(nsrc, 1))()
    for q, (i, j, kind, amp) in enumerate(w.sources):
        src[q].i, src[q].j, src[q].kind, src[q].amp = i, j, kind, amp
    wav = np.ascontiguousarray(w.wavelets, dtype=np.float64)
    nrec = len(w.receivers)
    rec = (ViReceiver * max(nrec, 1))()
    for r, (i, j) in enumerate(w.receivers):
        rec[r].i, rec[r].j = i, j
    obs = np.ascontiguousarray(obs[:, :, :nt], dtype=np.float64)
    grad = np.zeros((8, w.nz, w.nx))
    J = C.c_double()
    P = C.POINTER(C.c_double)
    rc = lib().or_gradient_f64(C.byref(cfg), C.byref(med), nsrc, src, wav.ctypes.data_as(P), wav.shape[1], nrec,
                               rec, obs.ctypes.data_as(P), nt, grad.ctypes.data_as(P), C.byref(J))
    if rc != 0:
        raise RuntimeError(f"oracle gradient failed with status {rc}")
    del keep
    return J.value, grad


def cpml_profile(cfg: ViConfig, axis: int, half: int):
    n = cfg.nx if axis == 0 else cfg.nz
    out = [np.zeros(n) for _ in range(5)]
    ptrs = [o.ctypes.data_as(C.POINTER(C.c_double)) for o in out]
    lib().or_cpml_profile(C.byref(cfg), axis, half, *ptrs)
    return dict(zip(("d", "alpha", "kappa", "a", "b"), out))


def ricker(f: float, t: float) -> float:
    return lib().or_ricker(f, t)


def stencil8() -> np.ndarray:
    out = np.zeros(4)
    lib().or_stencil8(out.ctypes.data_as(C.POINTER(C.c_double)))
    return out


def afda_weights() -> np.ndarray:
    """The oracle's H-AFDA one-sided weights w[op, q, m] (unit spacing)."""
    out = np.zeros((4, 4, 5))
    lib().or_afda_weights(out.ctypes.data_as(C.POINTER(C.c_double)))
    return out


def num_threads() -> int:
    return lib().or_num_threads()


def set_threads(n: int) -> None:
    os.environ["OMP_NUM_THREADS"] = str(n)
