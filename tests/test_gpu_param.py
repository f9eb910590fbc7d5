"""vi_medium_from_velocity (param.medium_from_velocity_device) against the
host forms media.medium_from_velocity and media.bond_rotate on seeded
planes: per plane, the largest difference relative to the plane's largest
magnitude is at most 1e-13 in FP64 and 1e-6 in FP32 (one rounding)."""
import numpy as np
import pytest
import torch

from viscoelasticinversion_b200 import media
from viscoelasticinversion_b200.param import medium_from_velocity_device

pytestmark = pytest.mark.gpu

TOL = {"f64": 1e-13, "f32": 1e-6}


@pytest.mark.parametrize("kind", ["iso", "vti", "tti"])
@pytest.mark.parametrize("precision", ["f32", "f64"])
def test_device_parameterisation_matches_host(kind, precision):
    rng = np.random.default_rng(5)
    shape = (37, 52)
    vp = rng.uniform(1800.0, 4500.0, shape)
    vs = vp / rng.uniform(1.6, 2.2, shape)
    rho = rng.uniform(1800.0, 2700.0, shape)
    eps, dlt = rng.uniform(0.0, 0.25, shape), rng.uniform(-0.05, 0.15, shape)
    theta, Q = rng.uniform(-0.6, 0.6, shape), rng.uniform(30.0, 200.0, shape)
    qf = media.q_fit(2.0, 30.0, 3)
    aniso = kind != "iso"
    host = media.medium_from_velocity("vti" if aniso else "iso", vp, vs, rho,
                                      eps if aniso else None, dlt if aniso else None, Q, qf)
    if kind == "tti":
        n = media.bond_rotate(host["c11"], host["c13"], host["c33"], host["c55"], theta)
        host.update(zip(("c11", "c13", "c15", "c33", "c35", "c55"), n))
    d = lambda a: torch.as_tensor(a, dtype=torch.float64, device="cuda").contiguous()
    out = medium_from_velocity_device(kind, d(vp), d(vs), d(rho), d(eps) if aniso else None,
                                      d(dlt) if aniso else None, d(theta) if kind == "tti" else None,
                                      d(Q), tau_scale=len(qf.taus) / qf.Kbar, precision=precision)
    torch.cuda.synchronize()
    assert set(out) == set(host)
    for k, ref in host.items():
        got = out[k].double().cpu().numpy()
        err = np.abs(got - ref).max() / np.abs(ref).max()
        assert err <= TOL[precision], (k, err)
