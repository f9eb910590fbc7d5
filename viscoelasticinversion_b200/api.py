"""Reference-facing names of the time-step path.

Mirrors the Julia API the reference defines for this path so that code
written against it ports line for line (Julia `f!` becomes `f_`):

  Fields(s, M, v), Parameters(λs, μs, τs, τns) ..... src/visco-kernels.jl:102-113
  leapfrog_step!(fields, parameters, dt) ......... src/visco-kernels.jl:87-100
  ddxp / ddxm / ddzp / ddzm ...................... src/diff-funcs.jl:3-32 (array form)
  Solver(vx, vz, sxx, szz, sxz), Model(ε, δ, γ) .. src/custom_solver/Model.jl:4-16
  PointSource, Ricker(fM, t0), get_value(s, t) ... src/custom_solver/PointSource.jl:1-14
  _ricker, RickerSource(freq, tc, nx, nz) ........ src/sciml_solver/Source.jl:3-33
  CPMLConfig(; ...), FreeSurfaceBC ............... src/sciml_solver/CPML.jl:28-63,366-370

Every array operation goes through libvisco_b200.so on the GPU; these are
host-side containers and argument plumbing only.
"""
from __future__ import annotations

import math
from dataclasses import dataclass

import numpy as np
import torch

from . import solver as _solver
from .media import ricker as _ricker_np
from .solver import CPMLSpec, StepPlan, make_config

# ----------------------------------------------------------------- sources


class PointSource:
    """abstract type PointSource (PointSource.jl:1)."""


@dataclass
class Ricker(PointSource):
    """Ricker(fM, t0): peak frequency fM, time shift t0 (PointSource.jl:3-6)."""

    fM: float
    t0: float


def get_value(s: PointSource, t):
    """get_value(::Ricker, t) = (1 - 2(π fM (t-t0))²) exp(-(π fM (t-t0))²)
    (PointSource.jl:8-14); other PointSource types raise like the
    reference's fallback method."""
    if isinstance(s, Ricker):
        return _ricker_np(s.fM, np.asarray(t, dtype=np.float64) - s.t0)
    raise NotImplementedError(f"get_value for `{type(s).__name__} <: PointSource` not implemented")


def _ricker(f, t):
    """Source.jl:3-5."""
    return float(_ricker_np(f, t)) if np.isscalar(t) else _ricker_np(f, t)


class RickerSource:
    """RickerSource(freq, tc, nx, nz; rtol): a single-point source at grid
    point (nx, nz) with weight 1 and an active window (t1, t2) around tc
    where |w| first reaches ~0 (Source.jl:7-33).  The window is found by a
    bracketed root search on |w| starting from tc ∓ 1/freq, as the
    reference does with Roots.find_zero."""

    def __init__(self, freq: float, tc: float, nx: int, nz: int, rtol: float = 1e-6):
        self.freq, self.tc = float(freq), float(tc)
        self.grid = [(int(nx), int(nz))]
        self.coefs = [1.0]
        self.tspan = (self._edge(-1, rtol), self._edge(+1, rtol))

    def _edge(self, sign: int, rtol: float) -> float:
        # |w(tc + sign*x)| -> 0 as x grows; march out from 1/freq until it
        # drops below rtol, then bisect
        f = self.freq
        lo, hi = 1.0 / f, 1.0 / f
        while abs(_ricker(f, hi)) > rtol:
            hi *= 1.25
        for _ in range(200):
            mid = 0.5 * (lo + hi)
            if abs(_ricker(f, mid)) > rtol:
                lo = mid
            else:
                hi = mid
        return self.tc + sign * hi

    def value(self, t: float) -> float:
        t1, t2 = self.tspan
        return _ricker(self.freq, t - self.tc) if t1 < t < t2 else 0.0

    def __call__(self, du: torch.Tensor, t: float):
        """du[gx, gz] += c * w(t) inside the active window (Source.jl:42-58);
        du is a [nz, nx] tensor and (gx, gz) are 1-based like the reference."""
        val = self.value(t)
        if val != 0.0:
            for (gx, gz), c in zip(self.grid, self.coefs):
                du[gz - 1, gx - 1] += c * val
        return None


# ---------------------------------------------------------------- boundary


def CPMLConfig(thickness=10, d0=None, alpha_max=0.0, kappa_max=1.0, power=2.0, left=True,
               right=True, top=False, bottom=True, vmax=None, dx=None, reflection_coef=1e-5):
    """CPMLConfig(; ...) (CPML.jl:40-63): needs d0 or (vmax and dx)."""
    if d0 is None:
        if vmax is None or dx is None:
            raise ValueError("Must provide either d0 or (vmax and dx) for automatic damping calculation")
        d0 = -(power + 1) * vmax * math.log(reflection_coef) / (2 * thickness * dx)
    return CPMLSpec(thickness=thickness, d0=d0, alpha_max=alpha_max, kappa_max=kappa_max,
                    power=power, left=left, right=right, top=top, bottom=bottom, vmax=vmax,
                    reflection_coef=reflection_coef)


@dataclass
class FreeSurfaceBC:
    """Stress-imaging free surface (CPML.jl:366-370).  The reference mirrors
    `depth` = 1 row; an 8th-order stencil reaches 4 rows above the surface,
    so the step images 4 and this is the only depth it accepts."""

    depth: int = 4

    def __post_init__(self):
        if self.depth != 4:
            raise ValueError("the 8th-order step images exactly 4 rows (depth = 4)")


# ------------------------------------------------------------------ fields


class Fields:
    """Fields(s, M, v) (visco-kernels.jl:102-106): s [3, nz, nx],
    M [3, N, nz, nx], v [2, nz, nx] CUDA tensors (the row-major form of the
    reference's s[Nx,Nz,3], M[Nx,Nz,N,3], v[Nx,Nz,2])."""

    def __init__(self, s: torch.Tensor, M: torch.Tensor, v: torch.Tensor):
        for name, t, d in (("s", s, 3), ("M", M, 4), ("v", v, 3)):
            if not (isinstance(t, torch.Tensor) and t.is_cuda and t.is_contiguous() and t.dim() == d):
                raise ValueError(f"Fields.{name} must be a contiguous {d}-D CUDA tensor")
        self.s, self.M, self.v = s, M, v


class Parameters:
    """Parameters(λs, μs, τs, τns) (visco-kernels.jl:108-113) plus what the
    full step needs that the reference's stress-only kernel did not: ρs for
    the velocity update, the spacing (the reference's global D carries 1/h),
    the CPML and the free surface."""

    def __init__(self, λs, μs, τs, τns, ρs=None, dx=1.0, dz=None, cpml: CPMLSpec | None = None,
                 free_surface: bool = False):
        self.λs, self.μs, self.τs = λs, μs, τs
        self.τns = [float(t) for t in (τns.tolist() if hasattr(τns, "tolist") else τns)]
        self.ρs = ρs
        self.dx = float(dx)
        self.dz = float(dx if dz is None else dz)
        self.cpml = cpml
        self.free_surface = bool(free_surface)
        self._plans: dict = {}

    def __iter__(self):  # λs, μs, τs, τns = parameters  (visco-kernels.jl:92)
        return iter((self.λs, self.μs, self.τs, self.τns))

    def plan(self, nx, nz, dt, dtype) -> StepPlan:
        key = (nx, nz, float(dt), dtype)
        if key not in self._plans:
            cfg = make_config(nx, nz, self.dx, self.dz, dt, "iso",
                              "f64" if dtype == torch.float64 else "f32", self.τns,
                              self.free_surface, self.cpml)
            self._plans[key] = StepPlan(cfg, device=self.λs.device.index)
        return self._plans[key]

    def medium(self) -> dict:
        if self.ρs is None:
            raise ValueError("Parameters needs ρs: the full step updates velocities, which need buoyancy")
        med = {"rho": self.ρs, "c13": self.λs, "c55": self.μs}
        if self.τns:
            med["tau"] = self.τs
        return {k: v.contiguous() for k, v in med.items()}


def leapfrog_step_(fields: Fields, parameters: Parameters, dt: float):
    """leapfrog_step!(fields, parameters, dt) (visco-kernels.jl:87-100): one
    full staggered step (velocity, then SLS stress + memory variables, CPML
    and free surface) on the fields in place, blocking until it is done like
    the reference's `synchronize(device)`."""
    nz, nx = fields.v.shape[1:]
    plan = parameters.plan(nx, nz, dt, fields.v.dtype)
    if fields.M.shape[1] != max(len(parameters.τns), 1):
        raise ValueError("M must hold one plane per mechanism and component")
    plan.step(parameters.medium(), {"v": fields.v, "s": fields.s, "m": fields.M}, nsteps=1)
    torch.cuda.synchronize(fields.v.device)


leapfrog_step = leapfrog_step_

# ---------------------------------------------------------- custom solver


@dataclass
class Solver:
    """Solver(vx, vz, sxx, szz, sxz) (custom_solver/Model.jl:4-10): separate
    [nz, nx] CUDA planes."""

    vx: torch.Tensor
    vz: torch.Tensor
    sxx: torch.Tensor
    szz: torch.Tensor
    sxz: torch.Tensor


@dataclass
class Model:
    """Model(ε, δ, γ) Thomsen parameters (custom_solver/Model.jl:12-16)."""

    ε: object
    δ: object
    γ: object


def solver_step_(solver: Solver, medium: dict, plan: StepPlan, nsteps: int = 1, it0: int = 0,
                 M: torch.Tensor | None = None, **shot):
    """Advances a Solver's planes in place (the time loop the custom solver
    sketches around timestep_strain_interior!/timestep_velocity_interior!,
    custom_solver/Model.jl:75-140)."""
    f = StepPlan.fields_struct(solver.vx, solver.vz, solver.sxx, solver.szz, solver.sxz,
                               M if plan.nsls else None)
    import ctypes as C
    from ._abi import check, lib
    med = plan._medium_struct(medium)
    srcs, rec = shot.get("sources"), shot.get("receivers")
    sh, keep = plan._shot(srcs, shot.get("wavelets"), rec, shot.get("traces"))
    check(lib().vi_step(plan._h, C.byref(med), C.byref(f), C.byref(sh) if (srcs or rec) else None,
                        int(it0), int(nsteps), 0, _solver._stream_handle(None)))
    del keep


# --------------------------------------------------------- derivatives


def ddxp(u: torch.Tensor, h: float = 1.0) -> torch.Tensor:
    """ddxp: derivative at i+1/2 from u[i-3..i+4] (diff-funcs.jl:3-8)."""
    return _solver.diff(u, "ddxp", h)


def ddxm(u: torch.Tensor, h: float = 1.0) -> torch.Tensor:
    """ddxm: derivative at i-1/2 from u[i-4..i+3] (diff-funcs.jl:10-16)."""
    return _solver.diff(u, "ddxm", h)


def ddzp(u: torch.Tensor, h: float = 1.0) -> torch.Tensor:
    """ddzp: derivative at j+1/2 (diff-funcs.jl:18-24)."""
    return _solver.diff(u, "ddzp", h)


def ddzm(u: torch.Tensor, h: float = 1.0) -> torch.Tensor:
    """ddzm: derivative at j-1/2 (diff-funcs.jl:26-32)."""
    return _solver.diff(u, "ddzm", h)


def staggered_stencil(order: int = 8):
    """Weights of the staggered first derivative of the given even order on
    the half-integer points, by the rational Vandermonde solve of
    Stencil.jl:_stencil (:9-14) — D[ℓ] multiplies (u[i+ℓ] - u[i-ℓ+1])."""
    from fractions import Fraction

    half = order // 2
    pts = [Fraction(2 * k - 1, 2) for k in range(-half + 1, half + 1)]
    n = len(pts)
    A = [[p**r / math.factorial(r) for p in pts] for r in range(n)]
    b = [Fraction(int(r == 1)) for r in range(n)]
    # Gaussian elimination in exact arithmetic
    M = [row[:] + [b[r]] for r, row in enumerate(A)]
    for c in range(n):
        piv = next(r for r in range(c, n) if M[r][c] != 0)
        M[c], M[piv] = M[piv], M[c]
        for r in range(n):
            if r != c and M[r][c] != 0:
                f = M[r][c] / M[c][c]
                M[r] = [x - f * y for x, y in zip(M[r], M[c])]
    w = [M[r][n] / M[r][r] for r in range(n)]
    return w[half:]  # weights of +1/2, +3/2, ... (antisymmetric)
