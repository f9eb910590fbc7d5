"""Pins the oracle to the facts the reference's own tests hold for this path.

Reference tests (read as text; Julia is not available to run them):
  tests/test_source.jl:8-31 ........ Ricker peak 1 at t = 0, symmetry, decay
  tests/test_source.jl:66-140 ...... single-point, exact, additive injection
  tests/test_cpml.jl:7-26 .......... CPMLConfig defaults and automatic d0
  tests/test_cpml.jl:42-61 ......... d_x = 0 in the interior, > 0 in both strips
  tests/test_viscoelastic_problem.jl:70-104,106-122
                                     dvz[src] = w/ρ (source added before the
                                     buoyancy scaling); zero when inactive
  src/common/Stencil.jl:9-14 ....... staggered weights from the rational solve
"""
import math

import numpy as np
import pytest

from viscoelasticinversion_b200 import api, media
from viscoelasticinversion_b200.solver import make_config, CPMLSpec


def test_stencil_weights_from_rational_solve(oracle_lib):
    from fractions import Fraction as F

    w = api.staggered_stencil(8)
    assert w == [F(1225, 1024), F(-245, 3072), F(49, 5120), F(-5, 7168)]
    assert np.allclose(oracle_lib.stencil8(), [float(x) for x in w], rtol=0, atol=0)
    # 4th order: 9/8, -1/24
    assert api.staggered_stencil(4) == [F(9, 8), F(-1, 24)]


def test_ricker_known_answers(oracle_lib):
    # test_source.jl:8-31
    assert oracle_lib.ricker(25.0, 0.0) == pytest.approx(1.0)
    assert oracle_lib.ricker(25.0, 0.01) == pytest.approx(oracle_lib.ricker(25.0, -0.01))
    assert abs(oracle_lib.ricker(25.0, 0.1)) < 0.01
    assert oracle_lib.ricker(50.0, 0.0) == pytest.approx(1.0)
    # host restatements agree with the oracle
    for f, t in [(25.0, 0.013), (12.0, -0.04), (15.0, 0.0)]:
        assert media.ricker(f, t) == pytest.approx(oracle_lib.ricker(f, t), rel=1e-15, abs=1e-15)
        assert api._ricker(f, t) == pytest.approx(oracle_lib.ricker(f, t), rel=1e-15, abs=1e-15)
    assert api.get_value(api.Ricker(25.0, 0.1), 0.1) == pytest.approx(1.0)
    with pytest.raises(NotImplementedError):
        api.get_value(api.PointSource(), 0.0)


def test_ricker_source_window_and_injection():
    # test_source.jl:33-51, 66-140 (CPU container: the injection is a
    # host-side helper writing one value into an array)
    import torch

    s = api.RickerSource(25.0, 0.1, 10, 15)
    assert s.grid == [(10, 15)] and s.coefs == [1.0]
    assert s.tspan[0] < 0.1 < s.tspan[1]
    assert abs((s.tspan[1] - s.tspan[0]) - 2.0 / 25.0) < 0.1
    du = torch.zeros(12, 8)
    s2 = api.RickerSource(25.0, 0.1, 8, 12)
    s2(du, s2.tspan[0] - 0.01)
    s2(du, s2.tspan[1] + 0.01)
    assert torch.count_nonzero(du) == 0
    s2(du, 0.1)
    nz = torch.nonzero(du)
    assert nz.shape[0] == 1 and tuple(nz[0].tolist()) == (11, 7)
    assert du[11, 7].item() == pytest.approx(1.0)
    s2(du, 0.1)
    assert du[11, 7].item() == pytest.approx(2.0)
    low, high = api.RickerSource(1.0, 0.1, 4, 6), api.RickerSource(100.0, 0.1, 4, 6)
    assert low.tspan[1] - low.tspan[0] > 2.0
    assert high.tspan[1] - high.tspan[0] < 0.1


def test_cpml_config_defaults():
    # test_cpml.jl:7-26
    c = api.CPMLConfig(thickness=10, d0=100.0)
    assert (c.thickness, c.d0, c.left, c.right, c.top, c.bottom) == (10, 100.0, True, True, False, True)
    auto = api.CPMLConfig(thickness=10, vmax=3000.0, dx=10.0, reflection_coef=1e-5)
    assert auto.d0 > 0 and auto.thickness == 10
    assert auto.d0 == pytest.approx(-3 * 3000 * math.log(1e-5) / (2 * 10 * 10.0))
    with pytest.raises(ValueError):
        api.CPMLConfig(thickness=10)


def test_cpml_profile_zero_inside_positive_in_strips(oracle_lib):
    # test_cpml.jl:42-61: thickness 5, Nx = Nz = 32, d0 = 100, alpha = pi, kappa 1.5
    cfg = make_config(32, 32, 10.0, 10.0, 0.001, cpml=CPMLSpec(thickness=5, d0=100.0, alpha_max=math.pi,
                                                                kappa_max=1.5))
    p = oracle_lib.cpml_profile(cfg, 0, 0)
    d = p["d"]
    assert np.all(d[5:32 - 5] == 0)          # Julia d_x[6:Nx-5]
    assert np.all(d[:5] > 0) and np.all(d[32 - 5:] > 0)
    # values equal the reference formula at the integer nodes (CPML.jl:121-140)
    L = 5
    for i in range(1, L + 1):
        pl = (L - i + 0.5) / L
        assert d[i - 1] == pytest.approx(100.0 * pl**2, rel=1e-14)
        assert p["alpha"][i - 1] == pytest.approx(math.pi * (1 - pl), rel=1e-14)
        assert p["kappa"][i - 1] == pytest.approx(1 + 0.5 * pl, rel=1e-14)
        pr = (i - 0.5) / L
        assert d[32 - L + i - 1] == pytest.approx(100.0 * pr**2, rel=1e-14)
        # b = exp(-(d/k + a) dt), a = d/(k(d + k a))(b - 1)   (CPML.jl:171-179)
        k, al, dd = 1 + 0.5 * pl, math.pi * (1 - pl), 100.0 * pl**2
        b = math.exp(-(dd / k + al) * 0.001)
        assert p["b"][i - 1] == pytest.approx(b, rel=1e-14)
        assert p["a"][i - 1] == pytest.approx(dd / (k * (dd + k * al)) * (b - 1), rel=1e-13)
    assert np.all(p["b"][5:27] == 0) and np.all(p["a"][5:27] == 0) and np.all(p["kappa"][5:27] == 1)
    # top strip off by default, bottom on
    pz = oracle_lib.cpml_profile(cfg, 1, 0)["d"]
    assert np.all(pz[:27] == 0) and np.all(pz[27:] > 0)
    # half nodes: the interface half node (i = L-1 + 1/2) is undamped
    ph = oracle_lib.cpml_profile(cfg, 0, 1)["d"]
    assert ph[L - 1] == 0 and ph[L - 2] > 0 and ph[31] > 0 and ph[32 - L - 1] == 0


def _one_cell_workload(kind_src, nx=32, nz=32, rho=2000.0):
    w = media.homogeneous_iso(nx=nx, nz=nz, dx=10.0, dt=1e-3, nt=1, rho=rho, nsls=0, pml=0,
                              free_surface=False, nrec=4)
    w.sources = [(nx // 2, nz // 2, kind_src, 1.0)]
    w.wavelets = np.ones((1, 1))
    return w


def test_force_source_scaled_by_buoyancy(oracle_lib):
    # test_viscoelastic_problem.jl:70-104: dvz[src] = w/ρ, everything else 0.
    # One step from rest with w = 1: vz[src] = dt * b * w, b = 2/(ρ_j + ρ_j+1) = 1/ρ.
    w = _one_cell_workload(2)
    _, st = oracle_lib.run(w, 1)
    vz = st.v[1]
    assert vz[16, 16] == pytest.approx(1e-3 / 2000.0, rel=1e-14)
    vz2 = vz.copy()
    vz2[16, 16] = 0
    assert np.all(vz2 == 0) and np.all(st.v[0] == 0)


def test_zero_response_when_source_inactive(oracle_lib):
    # test_viscoelastic_problem.jl:106-122
    w = _one_cell_workload(0)
    w.wavelets = np.zeros((1, 1))
    _, st = oracle_lib.run(w, 1)
    assert np.all(st.v == 0) and np.all(st.s == 0)


def test_explosive_source_adds_to_normal_stresses(oracle_lib):
    w = _one_cell_workload(0)
    _, st = oracle_lib.run(w, 1)
    assert st.s[0, 16, 16] == pytest.approx(1e-3) and st.s[1, 16, 16] == pytest.approx(1e-3)
    s = st.s.copy()
    s[0:2, 16, 16] = 0
    assert np.all(s == 0)
