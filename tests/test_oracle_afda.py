"""The oracle's H-AFDA free surface (vi_config.free_surface = 2) on the CPU:
its one-sided weights against an exact rational solve of the same
Vandermonde conditions (the construction of Stencil.jl:_stencil and
FreeSurfaceStencil, Stencil.jl:9-14,52-105), a long run that stays stable,
and agreement with the stress-imaging surface on a homogeneous half-space
(two discretisations of the same traction-free condition)."""
import dataclasses
import math
from fractions import Fraction as F

import numpy as np

import oracle
from viscoelasticinversion_b200 import media
from tests.helpers import rel_l2

N = 5  # samples per one-sided approximation


def _exact(points, x0):
    """Weights w with sum_k w_k (x_k - x0)^l / l! = [l == 1], in rationals."""
    n = len(points)
    A = [[(x - x0) ** l / math.factorial(l) for x in points] + [F(int(l == 1))] for l in range(n)]
    for c in range(n):
        p = next(r for r in range(c, n) if A[r][c] != 0)
        A[c], A[p] = A[p], A[c]
        for r in range(n):
            if r != c and A[r][c] != 0:
                f = A[r][c] / A[c][c]
                A[r] = [a - f * b for a, b in zip(A[r], A[c])]
    return [A[k][n] / A[k][k] for k in range(n)]


def test_afda_weights_exact():
    w = oracle.afda_weights()
    half = [F(2 * m + 1, 2) for m in range(N)]
    ref = np.zeros((4, 4, N))
    for q in range(4):
        ref[0, q] = [float(v) for v in _exact([F(0)] + half, F(q))[1:]]  # sxz(0) = 0
        if q < 3:
            ref[1, q] = [float(v) for v in _exact([F(m) for m in range(N + 1)], F(2 * q + 1, 2))[1:]]  # szz(0) = 0
            ref[3, q] = [float(v) for v in _exact([F(m) for m in range(N)], F(2 * q + 1, 2))]
        if q >= 1:
            ref[2, q] = [float(v) for v in _exact(half, F(q))]
    assert np.allclose(w, ref, rtol=1e-13, atol=1e-13), np.abs(w - ref).max()
    # each approximation differentiates z and z^2 exactly (away from the
    # zero boundary value those need f(0) = 0: z and z^2 both have it)
    for q in range(4):
        z = np.array([m + 0.5 for m in range(N)])
        assert abs(w[0, q] @ z - 1.0) < 1e-12 and abs(w[0, q] @ z**2 - 2 * q) < 1e-12


def test_afda_long_run_is_stable():
    """With the 5-sample one-sided approximations the wavefield decays once
    the source is over, as with the imaging surface (8-sample ones, sized
    like the interior stencil, give the semi-discrete 1D half-space
    operator eigenvalues with positive real part)."""
    w = media.layered(nx=96, nz=64, nt=6000, kind="tti", seed=3, pml=12, nrec=8, free_surface=2)
    st = None
    norms = []
    for k in range(6):
        _, st = oracle.run(w, 1000, precision="f64", state=st, it0=1000 * k)
        norms.append(np.linalg.norm(st.v))
    assert np.all(np.isfinite(norms))
    assert norms[-1] < 1e-3 * max(norms), norms


def test_afda_close_to_imaging():
    w = media.homogeneous_iso(nx=128, nz=128, nt=500, pml=16, nrec=24, src=(64, 40))
    tr1, _ = oracle.run(w, precision="f64")
    tr2, _ = oracle.run(dataclasses.replace(w, free_surface=2), precision="f64")
    assert np.abs(tr1).max() > 0
    assert rel_l2(tr2, tr1) < 0.05, rel_l2(tr2, tr1)
