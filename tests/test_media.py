"""Host-side set-up: Thomsen stiffness, Bond rotation, constant-Q fit,
seeded workloads (Models.jl:65-107, custom_solver/Model.jl:12-16)."""
import math

import numpy as np
import pytest

from viscoelasticinversion_b200 import media


def test_thomsen_isotropic_limit_and_delta():
    vp, vs, rho = 3000.0, 1700.0, 2200.0
    C11, C13, C33, C55 = media.thomsen_vti(vp, vs, rho, 0.0, 0.0)
    assert C11 == pytest.approx(rho * vp**2) and C33 == pytest.approx(C11)
    assert C13 == pytest.approx(rho * (vp**2 - 2 * vs**2))
    C11, C13, C33, C55 = media.thomsen_vti(vp, vs, rho, 0.2, 0.1)
    assert (C11 - C33) / (2 * C33) == pytest.approx(0.2)
    delta = ((C13 + C55) ** 2 - (C33 - C55) ** 2) / (2 * C33 * (C33 - C55))
    assert delta == pytest.approx(0.1)


def test_bond_rotation_matches_tensor_rotation():
    rng = np.random.default_rng(1)
    vp = rng.uniform(2000, 4000, 16)
    C11, C13, C33, C55 = media.thomsen_vti(vp, vp / 1.8, 2300.0, rng.uniform(0, .25, 16),
                                           rng.uniform(-.05, .15, 16))
    th = rng.uniform(-0.6, 0.6, 16)
    a = media.bond_rotate(C11, C13, C33, C55, th)
    b = media.bond_rotate_tensor(C11, C13, C33, C55, th)
    for x, y in zip(a, b):
        assert np.allclose(x, y, rtol=1e-12, atol=1e-3)
    # zero tilt is the identity; ±90° swaps C11 and C33
    z = media.bond_rotate(C11, C13, C33, C55, np.zeros(16))
    assert np.allclose(z[0], C11) and np.allclose(z[3], C33) and np.allclose(z[2], 0, atol=1e-6)
    r = media.bond_rotate(C11, C13, C33, C55, np.full(16, math.pi / 2))
    assert np.allclose(r[0], C33) and np.allclose(r[3], C11)


def test_q_fit_is_nearly_constant():
    qf = media.q_fit(5.0, 50.0, 3)
    mean_err, max_err = qf.q_error(50.0)
    assert mean_err < 0.05 and max_err < 0.15
    assert np.all(np.diff(qf.taus) > 0)
    # Q(ω) = N/(τ K(ω)) inverts τ = N/(K̄ Q0) on average
    om = np.linspace(2 * np.pi * 5, 2 * np.pi * 50, 100)
    assert np.mean(media.get_Q(om, qf.tau_for(50.0), qf.taus) ** -1) == pytest.approx(1 / 50.0, rel=0.05)


def test_layered_workload_recipe():
    w = media.layered(nx=256, nz=128, nt=10, kind="vti", seed=3)
    assert set(w.planes()) == {"rho", "c11", "c13", "c33", "c55", "tau"}
    assert w.bytes_per_point(4) == 136
    assert media.cfl_number(w) < 1.0
    vp = np.sqrt(w.medium["c33"] / w.medium["rho"])
    assert 1800 * 0.85 < vp.min() and vp.max() < 4500 * 1.15
    w2 = media.layered(nx=256, nz=128, nt=10, kind="vti", seed=3)
    assert all(np.array_equal(w.medium[k], w2.medium[k]) for k in w.medium)
    t = media.layered(nx=256, nz=128, nt=10, kind="tti", seed=3)
    assert t.bytes_per_point(4) == 144
    assert np.abs(t.meta["theta"]).max() <= math.radians(30) + 1e-12
    iso = media.homogeneous_iso()
    assert iso.bytes_per_point(4) == 128 and iso.bytes_per_point(8) == 256
