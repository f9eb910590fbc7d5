"""Misfit gradient (vi_gradient): the discrete adjoint on the GPU against
central finite differences of the FP64 oracle's misfit — directional
derivatives of every medium plane (along the gradient and along a bump
between source and receivers), and single-cell derivatives at 20 seeded
cells — plus checkpoint-interval
independence, FP32 vs FP64, and the (vp, vs, rho, 1/Q) and Thomsen
(epsilon, delta) chain rules.

The reference has no gradient to compare with (no Enzyme call exists); the
oracle's finite differences stand in for it."""
import dataclasses

import numpy as np
import pytest
import torch

from viscoelasticinversion_b200 import StepPlan, media
from viscoelasticinversion_b200.gradient import (GRADIENT_PLANES, misfit_gradient, shot_misfit,
                                                 thomsen_gradient, velocity_gradient)
from tests.helpers import rel_l2

pytestmark = pytest.mark.gpu

# Directional FD vs adjoint, FP64.  Directions: the gradient itself (no
# cancellation) and a positive bump between the source and the receivers.
# The oracle's misfit carries roundoff of ~1e-13 relative to the wavefield,
# so directions along which J barely changes cannot be checked by FD.
FD_REL_TOL = 1e-6
BUMP_REL_TOL = 1e-4
CELL_TOL = 1e-4      # single-cell FD vs adjoint, relative to the cell's gradient


def _field(w, seed, corr=6.0):
    rng = np.random.default_rng(seed)
    jj, ii = np.mgrid[0:w.nz, 0:w.nx]
    f = np.zeros((w.nz, w.nx))
    for _ in range(6):
        ci, cj = rng.uniform(0, w.nx), rng.uniform(0, w.nz)
        f += rng.normal() * np.exp(-((ii - ci) ** 2 + (jj - cj) ** 2) / (2 * corr**2))
    return f / np.abs(f).max()


def _with(w, **planes):
    med = dict(w.medium)
    med.update(planes)
    return dataclasses.replace(w, medium=med)


def _truth(w, seed=11):
    """True model: the start model with smooth perturbations of every plane."""
    return _with(w, **{k: v * (1.0 + 0.04 * _field(w, seed + n)) for n, (k, v) in enumerate(w.medium.items())})


def _oracle_J(oracle_lib, w, obs):
    tr, _ = oracle_lib.run(w, precision="f64")
    return 0.5 * float(np.sum((tr - obs) ** 2))


def _gpu_gradient(w, obs, precision="f64", K=0):
    plan = StepPlan.for_workload(w, precision)
    med = plan.medium_to_device(w.medium)
    wav = torch.as_tensor(w.wavelets, dtype=plan.dtype, device=plan.device).contiguous()
    obs_d = torch.as_tensor(obs, dtype=plan.dtype, device=plan.device).contiguous()
    J, g = misfit_gradient(plan, med, w.sources, wav, w.receivers, obs_d, checkpoint_every=K)
    out = g.cpu().numpy()
    plan.close()
    return J, out


def _iso(fs=True, force=False, nt=240):
    w = media.homogeneous_iso(nx=96, nz=80, nt=nt, pml=12, nrec=16, src=(40, 30), free_surface=fs)
    if force:
        wav = w.wavelets[0]
        w = dataclasses.replace(w, sources=[(40, 30, 1, 1.0), (57, 36, 2, 0.7)],
                                wavelets=np.stack([wav, np.roll(wav, 7)]))
    return w


def _vti(nt=300):
    # 25 Hz Ricker (t0 = 48 ms): the pulse has passed the receivers by 120 ms
    return media.layered(nx=128, nz=96, nt=nt, kind="vti", pml=12, nrec=16, nlayers=4, seed=2,
                         f0=25.0)


def _tti(nt=300, fs=True):
    # the C3-style tilted medium at test size: every stiffness plane of the
    # rotated law (C15 and C35 included) is non-zero
    return media.layered(nx=128, nz=96, nt=nt, kind="tti", pml=12, nrec=16, nlayers=4, seed=6,
                         f0=25.0, free_surface=fs)


def _bump(w, rel=0.25):
    """Positive Gaussian bump between the source and the receiver line."""
    (si, sj), (ri, rj) = w.sources[0][:2], w.receivers[len(w.receivers) // 2]
    ci, cj = 0.5 * (si + ri) + 6, 0.5 * (sj + rj) + 3
    jj, ii = np.mgrid[0:w.nz, 0:w.nx]
    return np.exp(-((ii - ci) ** 2 + (jj - cj) ** 2) / (2 * (rel * 0.5 * abs(sj - rj) + 3) ** 2))


def _richardson(J_of_h):
    """Central difference at h = 1 and 1/2, Richardson-extrapolated (error
    O(h^4)): directions concentrated at the source and receivers make the
    plain central difference's O(h^2) term visible at 1e-6."""
    c = [(J_of_h(h) - J_of_h(-h)) / (2 * h) for h in (1.0, 0.5)]
    return (4 * c[1] - c[0]) / 3


def _fd(oracle_lib, w, obs, k, d):
    return _richardson(lambda h: _oracle_J(oracle_lib, _with(w, **{k: w.medium[k] + h * d}), obs))


def _directional(oracle_lib, w, obs, g, planes, scale=1e-4):
    for k in planes:
        gk = g[GRADIENT_PLANES.index(k)]
        for name, dirn, tol in (("gradient", gk, FD_REL_TOL), ("bump", _bump(w), BUMP_REL_TOL)):
            d = scale * np.abs(w.medium[k]).max() * dirn / np.abs(dirn).max()
            fd = _fd(oracle_lib, w, obs, k, d)
            an = float(np.sum(gk * d))
            assert abs(fd - an) <= tol * abs(an), (k, name, fd, an)


@pytest.mark.parametrize("case", ["iso", "iso-force-nosurface", "vti", "tti", "tti-nosurface"])
def test_gradient_matches_oracle_finite_differences(oracle_lib, case):
    if case == "vti":
        w = _vti()
    elif case.startswith("tti"):
        w = _tti(fs=case == "tti")
    else:
        w = _iso(fs=case == "iso", force="force" in case)
    obs, _ = oracle_lib.run(_truth(w), precision="f64")
    J, g = _gpu_gradient(w, obs)
    J0 = _oracle_J(oracle_lib, w, obs)
    assert abs(J - J0) <= 1e-10 * J0, (J, J0)
    planes = {"iso": ["rho", "c13", "c55", "tau"], "vti": ["rho", "c11", "c13", "c33", "c55", "tau"],
              "tti": list(GRADIENT_PLANES)}[w.kind]
    _directional(oracle_lib, w, obs, g, planes)
    for k in GRADIENT_PLANES:
        if k not in planes:
            assert not np.any(g[GRADIENT_PLANES.index(k)]), k


@pytest.mark.parametrize("kind", ["iso", "tti"])
def test_gradient_single_cells(oracle_lib, kind):
    w = _iso() if kind == "iso" else _tti()
    obs, _ = oracle_lib.run(_truth(w), precision="f64")
    _, g = _gpu_gradient(w, obs)
    rng = np.random.default_rng(20)
    lo = w.pml + 4
    names = ("c55", "c13") if kind == "iso" else ("c15", "c35", "c55", "c13", "c11", "c33")
    for n in range(20):
        k = names[n % len(names)]
        gi = g[GRADIENT_PLANES.index(k)]
        i, j = int(rng.integers(lo, w.nx - lo)), int(rng.integers(5, w.nz - lo))
        h = 1e-4 * w.medium[k][j, i]
        pert = np.zeros_like(w.medium[k])
        pert[j, i] = h
        fd = (_oracle_J(oracle_lib, _with(w, **{k: w.medium[k] + pert}), obs)
              - _oracle_J(oracle_lib, _with(w, **{k: w.medium[k] - pert}), obs)) / (2 * h)
        assert abs(fd - gi[j, i]) <= CELL_TOL * abs(gi[j, i]) + 1e-7 * np.abs(gi).max(), (k, i, j, fd, gi[j, i])


@pytest.mark.parametrize("kind", ["vti", "tti"])
def test_checkpoint_interval_and_precision(oracle_lib, kind):
    w = _vti(nt=200) if kind == "vti" else _tti(nt=200)
    obs, _ = oracle_lib.run(_truth(w), precision="f64")
    J0, g0 = _gpu_gradient(w, obs, K=0)  # every state kept in HBM: no recompute
    for K in (1, 7, 15, w.nt):
        J, g = _gpu_gradient(w, obs, K=K)
        assert J == J0 and np.array_equal(g, g0), K
    J32, g32 = _gpu_gradient(w, obs, precision="f32")
    assert abs(J32 - J0) <= 1e-4 * J0
    planes = ("rho", "c11", "c13", "c33", "c55", "tau") + (("c15", "c35") if kind == "tti" else ())
    for k in planes:
        i = GRADIENT_PLANES.index(k)
        assert rel_l2(g32[i], g0[i]) <= 1e-3, (k, rel_l2(g32[i], g0[i]))


@pytest.mark.parametrize("kind", ["iso", "vti"])
def test_velocity_chain_rule(oracle_lib, kind):
    w = _iso() if kind == "iso" else _vti()
    qf = media.q_fit(*w.meta["band"], w.nsls)
    if kind == "iso":
        shape = (w.nz, w.nx)
        fields = {"vp": np.full(shape, 3000.0), "vs": np.full(shape, 1732.0),
                  "rho": np.full(shape, 2200.0), "Q": np.full(shape, w.meta["Q"])}
    else:
        fields = dict(w.meta["fields"])
    eps, dlt = fields.get("eps"), fields.get("delta")

    def build(f):
        return _with(w, **media.medium_from_velocity(kind, f["vp"], f["vs"], f["rho"], eps, dlt,
                                                     f["Q"], qf))

    w = build(fields)
    obs, _ = oracle_lib.run(_truth(w), precision="f64")
    _, g = _gpu_gradient(w, obs)
    dev = lambda a: torch.as_tensor(np.ascontiguousarray(a), dtype=torch.float64, device="cuda")
    gv = velocity_gradient(kind, dev(g), dev(fields["vp"]), dev(fields["vs"]), dev(fields["rho"]),
                           None if eps is None else dev(eps), None if dlt is None else dev(dlt),
                           tau_scale=w.nsls / qf.Kbar).cpu().numpy()
    for n, name in enumerate(("vp", "vs", "rho", "qinv")):
        # along the gradient: J changes well above the oracle's roundoff
        base = 1.0 / fields["Q"] if name == "qinv" else fields[name]
        d = 1e-4 * np.abs(base).max() * gv[n] / np.abs(gv[n]).max()

        def J_of(h):
            f = dict(fields)
            if name == "qinv":
                f["Q"] = 1.0 / (base + h * d)
            else:
                f[name] = base + h * d
            return _oracle_J(oracle_lib, build(f), obs)

        fd = _richardson(J_of)
        an = float(np.sum(gv[n] * d))
        assert abs(fd - an) <= FD_REL_TOL * abs(an), (name, fd, an)


def test_thomsen_chain_rule(oracle_lib):
    """dJ/d(epsilon, delta) of a VTI medium at fixed vp, vs, rho and Q
    (vi_gradient_thomsen): against the chain rule restated in numpy, and
    against central differences of the oracle's misfit along the gradient."""
    w = _vti()
    qf = media.q_fit(*w.meta["band"], w.nsls)
    fields = dict(w.meta["fields"])

    def build(f):
        return _with(w, **media.medium_from_velocity("vti", f["vp"], f["vs"], f["rho"], f["eps"],
                                                     f["delta"], f["Q"], qf))

    w = build(fields)
    obs, _ = oracle_lib.run(_truth(w), precision="f64")
    _, g = _gpu_gradient(w, obs)
    dev = lambda a: torch.as_tensor(np.ascontiguousarray(a), dtype=torch.float64, device="cuda")
    vp, vs, rho, dlt = fields["vp"], fields["vs"], fields["rho"], fields["delta"]
    gt = thomsen_gradient(dev(g), dev(vp), dev(vs), dev(rho), dev(dlt)).cpu().numpy()
    C33, C55 = rho * vp**2, rho * vs**2
    A, B = C33 - C55, C33 * (1 + 2 * dlt) - C55
    ref = np.stack([g[GRADIENT_PLANES.index("c11")] * 2 * C33,
                    g[GRADIENT_PLANES.index("c13")] * A * C33 / np.sqrt(A * B)])
    assert rel_l2(gt, ref) <= 1e-13
    for n, name in enumerate(("eps", "delta")):
        base = fields[name]
        d = 1e-4 * np.abs(base).max() * gt[n] / np.abs(gt[n]).max()

        def J_of(h):
            f = dict(fields)
            f[name] = base + h * d
            return _oracle_J(oracle_lib, build(f), obs)

        fd = _richardson(J_of)
        an = float(np.sum(gt[n] * d))
        assert abs(fd - an) <= FD_REL_TOL * abs(an), (name, fd, an)


def test_autograd_function(oracle_lib):
    """shot_misfit as a torch autograd function: J and the plane gradients
    equal misfit_gradient's, and J backpropagates through torch ops from vp
    (ISO: lambda = rho (vp^2 - 2 vs^2), mu = rho vs^2) to the dJ/dvp of
    vi_gradient_velocity."""
    w = _iso(nt=160)
    obs_np, _ = oracle_lib.run(_truth(w), precision="f64")
    plan = StepPlan.for_workload(w, "f64")
    wav = torch.as_tensor(w.wavelets, dtype=plan.dtype, device=plan.device).contiguous()
    obs = torch.as_tensor(obs_np, dtype=plan.dtype, device=plan.device).contiguous()
    med = {k: v.clone().requires_grad_(True) for k, v in plan.medium_to_device(w.medium).items()}
    J = shot_misfit(plan, med, w.sources, wav, w.receivers, obs)
    J.backward()
    J0, g0 = misfit_gradient(plan, {k: v.detach() for k, v in med.items()}, w.sources, wav,
                             w.receivers, obs)
    assert J0 > 0 and abs(float(J.detach()) - J0) <= 1e-13 * J0
    for k, v in med.items():
        ref = g0[GRADIENT_PLANES.index(k)]
        assert rel_l2(v.grad.cpu().numpy(), ref.cpu().numpy()) <= 1e-13, k
    shape = (w.nz, w.nx)
    rho, tau = med["rho"].detach(), med["tau"].detach()
    vs = torch.full(shape, 1732.0, dtype=torch.float64, device=plan.device)
    vp = torch.full(shape, 3000.0, dtype=torch.float64, device=plan.device, requires_grad=True)
    J2 = shot_misfit(plan, {"rho": rho, "c13": rho * (vp**2 - 2 * vs**2), "c55": rho * vs**2,
                            "tau": tau}, w.sources, wav, w.receivers, obs)
    J2.backward()
    gv = velocity_gradient("iso", g0, vp.detach(), vs, rho)
    assert rel_l2(vp.grad.cpu().numpy(), gv[0].cpu().numpy()) <= 1e-12
    plan.close()


def test_tti_parameter_chain_rule(oracle_lib):
    """dJ/d(vp, vs, rho, 1/Q, epsilon, delta, theta) of a TTI medium
    (vi_gradient_tti): against central differences of the host map (Thomsen
    law tilted by media.bond_rotate) contracted with the stiffness gradient,
    and for epsilon and theta against central differences of the oracle's
    misfit along the gradient."""
    from viscoelasticinversion_b200.gradient import TTI_PARAMETERS, tti_gradient

    w = _tti()
    qf = media.q_fit(*w.meta["band"], w.nsls)
    fields = dict(w.meta["fields"])
    fields["theta"] = w.meta["theta"]

    def planes(f):
        vti = media.medium_from_velocity("vti", f["vp"], f["vs"], f["rho"], f["eps"], f["delta"], f["Q"], qf)
        n11, n13, n15, n33, n35, n55 = media.bond_rotate(vti["c11"], vti["c13"], vti["c33"], vti["c55"],
                                                         f["theta"])
        return {"rho": vti["rho"], "c11": n11, "c13": n13, "c15": n15, "c33": n33, "c35": n35, "c55": n55,
                "tau": vti["tau"]}

    w = _with(w, **planes(fields))
    obs, _ = oracle_lib.run(_truth(w), precision="f64")
    _, g = _gpu_gradient(w, obs)
    dev = lambda a: torch.as_tensor(np.ascontiguousarray(a), dtype=torch.float64, device="cuda")
    gt = tti_gradient(dev(g), dev(fields["vp"]), dev(fields["vs"]), dev(fields["rho"]), dev(fields["eps"]),
                      dev(fields["delta"]), dev(fields["theta"]), tau_scale=w.nsls / qf.Kbar).cpu().numpy()
    # the host map's derivative, parameter by parameter, contracted with g
    for n, name in enumerate(TTI_PARAMETERS):
        base = 1.0 / fields["Q"] if name == "qinv" else fields[name]
        h = 1e-6 * max(np.abs(base).max(), 1e-3)

        def pl(sign):
            f = dict(fields)
            if name == "qinv":
                f["Q"] = 1.0 / (base + sign * h)
            else:
                f[name] = base + sign * h
            return planes(f)

        pp, pm = pl(1.0), pl(-1.0)
        ref = sum(g[GRADIENT_PLANES.index(k)] * (pp[k] - pm[k]) / (2 * h) for k in GRADIENT_PLANES)
        assert rel_l2(gt[n], ref) <= 1e-6, (name, rel_l2(gt[n], ref))
    for name in ("eps", "theta"):
        n = TTI_PARAMETERS.index(name)
        d = 1e-4 * gt[n] / np.abs(gt[n]).max()

        def J_of(hh):
            f = dict(fields)
            f[name] = fields[name] + hh * d
            return _oracle_J(oracle_lib, _with(w, **planes(f)), obs)

        fd = _richardson(J_of)
        an = float(np.sum(gt[n] * d))
        assert abs(fd - an) <= FD_REL_TOL * abs(an), (name, fd, an)


@pytest.mark.parametrize("kind,fs,force", [("iso", True, False), ("iso", False, True), ("vti", True, False),
                                           ("tti", True, False), ("tti", False, True)])
def test_gradient_equals_oracle_adjoint(oracle_lib, kind, fs, force):
    """The GPU adjoint against the oracle's own discrete adjoint
    (oracle/oracle_adjoint.c, itself dot-product tested): misfit and every
    gradient plane to 1e-10 relative in FP64, a far tighter pin than finite
    differences."""
    if kind == "iso":
        w = media.homogeneous_iso(nx=64, nz=48, nt=120, pml=8, nrec=8, src=(30, 16), free_surface=fs)
    else:
        w = media.layered(nx=64, nz=48, nt=120, kind=kind, seed=4, pml=8, nrec=8, nlayers=3, f0=30.0,
                          free_surface=fs)
    if force:
        wav = w.wavelets[0]
        w = dataclasses.replace(w, sources=[(30, 16, 1, 1.0), (25, 20, 2, 0.5)],
                                wavelets=np.stack([wav, np.roll(wav, 4)]))
    obs, _ = oracle_lib.run(_truth(w), precision="f64")
    J0, g0 = oracle_lib.gradient(w, obs)
    J, g = _gpu_gradient(w, obs)
    assert abs(J - J0) <= 1e-12 * J0, (J, J0)
    for n, k in enumerate(GRADIENT_PLANES):
        ref = g0[n]
        if not np.any(ref):
            assert not np.any(g[n]), k
            continue
        assert rel_l2(g[n], ref) <= 1e-10, (k, rel_l2(g[n], ref))


def test_kept_states_reused_across_calls(oracle_lib):
    """One plan, gradients with every state kept (K = 0), then checkpointed
    (K = 7), a forward solve through vi_forward_host (which reuses the
    workspace), then kept again: all bitwise equal; the kept states' zero
    cells are set up again whenever the workspace was used otherwise."""
    w = _vti(nt=120)
    obs, _ = oracle_lib.run(_truth(w), precision="f64")
    plan = StepPlan.for_workload(w, "f64")
    med = plan.medium_to_device(w.medium)
    wav = torch.as_tensor(w.wavelets, dtype=plan.dtype, device=plan.device).contiguous()
    obs_d = torch.as_tensor(obs, dtype=plan.dtype, device=plan.device).contiguous()
    runs = []
    for K in (0, 0, 7, "host", 0):
        if K == "host":
            plan.forward_host(w.medium, w.sources, w.wavelets, w.receivers, w.nt)
            continue
        J, g = misfit_gradient(plan, med, w.sources, wav, w.receivers, obs_d, checkpoint_every=K)
        runs.append((J, g.cpu().numpy()))
    plan.close()
    for J, g in runs[1:]:
        assert J == runs[0][0] and np.array_equal(g, runs[0][1])
