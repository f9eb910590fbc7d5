"""Reference-facing API on the GPU: staggered derivatives (diff-funcs.jl),
leapfrog_step! with Fields/Parameters (visco-kernels.jl:87-113), and the
custom Solver planes (custom_solver/Model.jl:4-10)."""
import numpy as np
import pytest
import torch

from viscoelasticinversion_b200 import api, media
from viscoelasticinversion_b200.solver import CPMLSpec
from tests.helpers import rel_l2

pytestmark = pytest.mark.gpu

D = [1225 / 1024, -245 / 3072, 49 / 5120, -5 / 7168]


def np_diff(u, op, h):
    nz, nx = u.shape
    out = np.zeros_like(u)
    for j in range(4, nz - 4):
        for i in range(4, nx - 4):
            v = 0.0
            for k in range(4):
                l = k + 1
                if op == "ddxp":
                    v += D[k] * (u[j, i + l] - u[j, i - l + 1])
                elif op == "ddxm":
                    v += D[k] * (u[j, i + l - 1] - u[j, i - l])
                elif op == "ddzp":
                    v += D[k] * (u[j + l, i] - u[j - l + 1, i])
                else:
                    v += D[k] * (u[j + l - 1, i] - u[j - l, i])
            out[j, i] = v / h
    return out


@pytest.mark.parametrize("op", ["ddxp", "ddxm", "ddzp", "ddzm"])
def test_staggered_derivatives(op):
    rng = np.random.default_rng(0)
    u = rng.standard_normal((23, 31))
    fn = getattr(api, op)
    got = fn(torch.tensor(u, device="cuda"), 2.5).cpu().numpy()
    assert np.allclose(got, np_diff(u, op, 2.5), rtol=1e-13, atol=1e-13)
    got32 = fn(torch.tensor(u, device="cuda", dtype=torch.float32), 2.5).cpu().numpy()
    assert rel_l2(got32, np_diff(u, op, 2.5)) < 1e-6
    # exact on a linear function away from the edges
    x = np.arange(31) * 2.5
    lin = np.tile(3.0 * x, (23, 1)) if "x" in op else np.tile(3.0 * np.arange(23)[:, None] * 2.5, (1, 31))
    d = fn(torch.tensor(lin, device="cuda"), 2.5).cpu().numpy()
    assert np.allclose(d[4:-4, 4:-4], 3.0, rtol=1e-12)


def test_leapfrog_step_matches_oracle(oracle_lib):
    w = media.homogeneous_iso(nx=128, nz=96, nt=80, pml=12, nrec=8)
    tr_ref, st_ref = oracle_lib.run(w, precision="f64")
    dev = "cuda"
    nz, nx, N = w.nz, w.nx, w.nsls
    fields = api.Fields(torch.zeros(3, nz, nx, dtype=torch.float64, device=dev),
                        torch.zeros(3, N, nz, nx, dtype=torch.float64, device=dev),
                        torch.zeros(2, nz, nx, dtype=torch.float64, device=dev))
    t = lambda k: torch.tensor(w.medium[k], device=dev)
    cp = CPMLSpec(thickness=w.pml, alpha_max=w.pml_alpha_max, vmax=w.pml_vmax)
    params = api.Parameters(t("c13"), t("c55"), t("tau"), w.taus, ρs=t("rho"), dx=w.dx,
                            cpml=cp, free_surface=True)
    (si, sj, _, amp), = w.sources
    for it in range(w.nt):
        api.leapfrog_step_(fields, params, w.dt)
        # explosive source the way a caller drives the reference's step
        fields.s[0, sj, si] += w.dt * amp * w.wavelets[0, it]
        fields.s[1, sj, si] += w.dt * amp * w.wavelets[0, it]
    # the oracle adds the source inside the step; same arithmetic, same order
    assert rel_l2(fields.v.cpu().numpy(), st_ref.v) < 1e-10
    assert rel_l2(fields.s.cpu().numpy(), st_ref.s) < 1e-10
    assert rel_l2(fields.M.reshape(-1, nz, nx).cpu().numpy(), st_ref.m) < 1e-10


def test_parameters_need_density():
    z = torch.zeros(32, 32, device="cuda")
    p = api.Parameters(z, z, z, [0.01])
    with pytest.raises(ValueError):
        p.medium()
