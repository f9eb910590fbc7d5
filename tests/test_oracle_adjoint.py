"""The oracle's discrete adjoint (oracle/oracle_adjoint.c), on the CPU.

Dot-product test: for the one-step state map A (fixed medium, no sources)
and random states x, y, <A x, y> = <x, A^T y> to 1e-12.  Each pair of plane
groups (velocities, stresses, memory variables, CPML psi) is tested on its
own, so a wrong block cannot hide below the rounding of a larger one.
Gradient: the oracle's misfit gradient against central differences of its
own misfit along the gradient (every stiffness plane, ISO/VTI/TTI, with and
without the free surface, force sources)."""
import dataclasses

import numpy as np
import pytest

import oracle
from viscoelasticinversion_b200 import media

GROUPS = {"v": ("v",), "s": ("s",), "m": ("m",), "psi": ("psi",)}


def _case(kind, fs=True, nsls=3):
    if kind == "iso":
        w = media.homogeneous_iso(nx=48, nz=40, nt=60, pml=8, nrec=6, src=(24, 14), free_surface=fs)
        if nsls != 3:
            w = dataclasses.replace(w, taus=w.taus[:nsls])
    else:
        w = media.layered(nx=48, nz=40, nt=60, kind=kind, seed=3, pml=8, nrec=6, nlayers=3, nsls=nsls,
                          free_surface=fs)
    return w


def _state(w, rng, groups):
    st = oracle.OracleState(w.nx, w.nz, w.nsls, np.float64)
    for gname in groups:
        arr = getattr(st, gname)
        if gname == "m" and w.nsls == 0:
            continue
        arr[...] = rng.standard_normal(arr.shape)
    return st


def _dot(a, b, groups):
    return sum(float(np.sum(getattr(a, g) * getattr(b, g))) for g in groups)


def _norm(a, groups):
    return np.sqrt(sum(float(np.sum(getattr(a, g) ** 2)) for g in groups))


@pytest.mark.parametrize("kind,fs,nsls", [("iso", True, 3), ("vti", True, 3), ("tti", True, 3),
                                          ("tti", False, 3), ("vti", False, 0)])
def test_adjoint_dot_product(kind, fs, nsls):
    w = _case(kind, fs, nsls)
    bare = dataclasses.replace(w, sources=[], receivers=[], wavelets=np.zeros((0, w.nt)))
    rng = np.random.default_rng(5)
    names = [g for g in GROUPS if not (g == "m" and w.nsls == 0)]
    for P in names:
        for Q in names:
            x = _state(w, rng, (P,))
            y = _state(w, rng, (Q,))
            Ax = oracle.OracleState(w.nx, w.nz, w.nsls, np.float64)
            for g in ("v", "s", "m", "psi"):
                getattr(Ax, g)[...] = getattr(x, g)
            oracle.run(bare, 1, precision="f64", state=Ax)
            ATy = oracle.OracleState(w.nx, w.nz, w.nsls, np.float64)
            for g in ("v", "s", "m", "psi"):
                getattr(ATy, g)[...] = getattr(y, g)
            oracle.adjoint_step(bare, ATy)
            lhs, rhs = _dot(Ax, y, (Q,)), _dot(x, ATy, (P,))
            scale = _norm(Ax, (Q,)) * _norm(y, (Q,)) + _norm(x, (P,)) * _norm(ATy, (P,))
            assert abs(lhs - rhs) <= 1e-12 * scale, (kind, fs, P, Q, lhs, rhs, scale)


def _perturbed(w, seed=11):
    rng = np.random.default_rng(seed)
    med = {k: v * (1.0 + 0.03 * rng.standard_normal(v.shape)) for k, v in w.medium.items()}
    return dataclasses.replace(w, medium=med)


@pytest.mark.parametrize("kind,fs,force", [("iso", True, False), ("vti", True, False), ("tti", True, False),
                                           ("tti", False, True)])
def test_oracle_gradient_matches_its_finite_differences(kind, fs, force):
    w = _case(kind, fs)
    if force:
        wav = w.wavelets[0]
        w = dataclasses.replace(w, sources=[(24, 14, 1, 1.0), (20, 18, 2, 0.6)],
                                wavelets=np.stack([wav, np.roll(wav, 3)]))
    obs, _ = oracle.run(_perturbed(w), precision="f64")
    J, g = oracle.gradient(w, obs)
    planes = {"iso": ("rho", "c13", "c55", "tau"), "vti": ("rho", "c11", "c13", "c33", "c55", "tau"),
              "tti": ("rho", "c11", "c13", "c15", "c33", "c35", "c55", "tau")}[kind]
    order = ("rho", "c11", "c13", "c15", "c33", "c35", "c55", "tau")
    for k in planes:
        gk = g[order.index(k)]
        d = 1e-4 * np.abs(w.medium[k]).max() * gk / np.abs(gk).max()

        def J_of(h):
            med = dict(w.medium)
            med[k] = w.medium[k] + h * d
            tr, _ = oracle.run(dataclasses.replace(w, medium=med), precision="f64")
            return 0.5 * float(np.sum((tr - obs) ** 2))

        c = [(J_of(h) - J_of(-h)) / (2 * h) for h in (1.0, 0.5)]
        fd = (4 * c[1] - c[0]) / 3
        an = float(np.sum(gk * d))
        assert abs(fd - an) <= 1e-6 * abs(an), (kind, k, fd, an)
