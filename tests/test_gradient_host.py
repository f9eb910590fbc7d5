"""Host logic on the CPU (no GPU): gradient.shot_misfit, the autograd
function, maps each medium plane to its gradient plane and scales by the
cotangent (vi_gradient replaced by a stand-in with a known gradient; the
real one is checked against the oracle in test_gpu_gradient.py); the
device parameterisation wrapper checks its arguments before any device
work."""
import pytest
import torch

from viscoelasticinversion_b200 import gradient as G


def _fake_misfit_gradient(plan, medium, sources, wavelets, receivers, obs, checkpoint_every=0):
    # J = sum_k (index_k + 1) * sum(plane_k): dJ/dplane_k = index_k + 1
    nz, nx = next(iter(medium.values())).shape
    g = torch.zeros(8, nz, nx, dtype=torch.float64)
    J = 0.0
    for k, t in medium.items():
        i = G.GRADIENT_PLANES.index(k)
        g[i] = i + 1.0
        J += (i + 1.0) * float(t.detach().sum())
    return J, g


def test_shot_misfit_backward_through_torch(monkeypatch):
    monkeypatch.setattr(G, "misfit_gradient", _fake_misfit_gradient)
    rho = torch.rand(3, 4, dtype=torch.float64) + 1.0
    vp = torch.full((3, 4), 2.0, dtype=torch.float64, requires_grad=True)
    vs = torch.full((3, 4), 1.0, dtype=torch.float64, requires_grad=True)
    med = {"rho": rho, "c13": rho * (vp**2 - 2 * vs**2), "c55": rho * vs**2,
           "tau": torch.zeros(3, 4, dtype=torch.float64)}
    J = G.shot_misfit(None, med, [], None, [], None)
    assert J.dtype == torch.float64 and J.dim() == 0
    (2.0 * J).backward()
    k13, k55 = G.GRADIENT_PLANES.index("c13") + 1.0, G.GRADIENT_PLANES.index("c55") + 1.0
    assert torch.allclose(vp.grad, 2.0 * k13 * rho * 2 * vp.detach())
    assert torch.allclose(vs.grad, 2.0 * (k13 * rho * (-4) * vs.detach() + k55 * rho * 2 * vs.detach()))


def test_shot_misfit_rejects_unknown_planes():
    with pytest.raises(ValueError, match="medium keys"):
        G.shot_misfit(None, {"lambda": torch.zeros(2, 2)}, [], None, [], None)


def test_device_parameterisation_checks_arguments_before_device_work():
    from viscoelasticinversion_b200.param import medium_from_velocity_device

    z = torch.zeros(3, 4, dtype=torch.float64)
    with pytest.raises(ValueError, match="kind"):
        medium_from_velocity_device("ortho", z, z, z)
    with pytest.raises(ValueError, match="tau_scale"):
        medium_from_velocity_device("iso", z, z, z, Q=z)
