"""Shot sharding and the gradient all-reduce across ranks, on CPU with the
gloo backend (world size 2): the same host logic that runs over NCCL on
GPUs, for shot_gradient and for the FWI driver (fwi.FWIProblem, its
per-shot work replaced by an analytic stand-in).  Also the failure path: a
rank that dies before the all-reduce makes the survivor's collective end
with an error instead of hanging."""
import datetime
import os
import socket

import numpy as np
import pytest
import torch
import torch.distributed as dist
import torch.multiprocessing as mp

from viscoelasticinversion_b200 import fwi, media
from viscoelasticinversion_b200.gradient import GRADIENT_PLANES, reduce_gradient, shard, shot_gradient

SHAPE = (6, 10)
NSHOTS = 7


def _free_port():
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        return s.getsockname()[1]


def _fake_gradient(i):
    """Deterministic per-shot (misfit, gradient) standing in for vi_gradient."""
    g = torch.arange(8 * SHAPE[0] * SHAPE[1], dtype=torch.float64).reshape(8, *SHAPE)
    return 0.5 * (i + 1) ** 2, torch.sin(g * (i + 1)) * (i + 1)


class _AnalyticFWI(fwi.FWIProblem):
    """FWIProblem with the GPU work replaced: shot i has the misfit
    J_i(θ) = (i + 1)/2 · |θ - (i + 1)/10|², as dJ/dplane = dJ/dθ / base."""

    def _target(self, i):
        return 0.1 * (i + 1)

    def _shots_value_and_grad(self, theta, shots):
        th = np.asarray(theta).reshape(len(self.planes), self.base.nz, self.base.nx)
        g = np.zeros((8, self.base.nz, self.base.nx))
        J = 0.0
        for i in shots:
            J += 0.5 * (i + 1) * float(np.sum((th - self._target(i)) ** 2))
            for n, k in enumerate(self.planes):
                g[GRADIENT_PLANES.index(k)] += (i + 1) * (th[n] - self._target(i)) / self.base.medium[k]
        return J, g

    def _shots_batch_loss(self, thetas, shots):
        return np.array([self._shots_value_and_grad(t, shots)[0] for t in thetas])


def _fwi_problem():
    w = media.homogeneous_iso(nx=12, nz=10, nt=4, pml=2, nrec=2, nsls=0)
    return _AnalyticFWI(w, [w] * NSHOTS, [np.zeros((2, 2, 4))] * NSHOTS, planes=("c13", "c55"))


def _fwi_run(prob):
    theta0 = np.linspace(-0.2, 0.3, prob.n_params)
    J, g = prob.value_and_grad(theta0)
    losses = prob.batch_loss([theta0, theta0 * 0.5])
    opt = fwi.EnergyNaturalGradientOptimizer(line_search_points=7, line_search_bounds=(1e-4, 1.0))
    st = fwi.OptimizationState(theta0)
    fwi.optimize(st, opt, prob.loss, prob.grad, None, 3, batch_loss_fn=prob.batch_loss)
    return {"J": J, "g": g, "losses": losses, "theta": st.theta, "hist": st.loss_history,
            "mine": prob.mine}


def _worker(rank, world, port, out_dir, mode):
    dist.init_process_group("gloo", init_method=f"tcp://127.0.0.1:{port}", rank=rank,
                            world_size=world, timeout=datetime.timedelta(seconds=8))
    try:
        if mode == "sum":
            J, g = shot_gradient(_fake_gradient, NSHOTS, SHAPE)
            torch.save({"J": J, "g": g, "mine": shard(NSHOTS, rank, world)},
                       os.path.join(out_dir, f"r{rank}.pt"))
        elif mode == "fwi":
            torch.save(_fwi_run(_fwi_problem()), os.path.join(out_dir, f"r{rank}.pt"))
        elif mode == "dies":
            if rank == 1:
                raise SystemExit(3)  # leaves between steps, before the collective
            err = None
            try:
                reduce_gradient(torch.ones(8, *SHAPE, dtype=torch.float64), 1.0)
            except Exception as e:  # the short process-group timeout ends the wait
                err = type(e).__name__
            torch.save({"err": err}, os.path.join(out_dir, f"r{rank}.pt"))
    finally:
        if mode != "dies" or rank == 0:
            try:
                dist.destroy_process_group()
            except Exception:
                pass


def test_shards_cover_every_shot_once():
    for world in (1, 2, 3, 8):
        got = sorted(i for r in range(world) for i in shard(NSHOTS, r, world))
        assert got == list(range(NSHOTS))


def test_gradient_sum_over_two_ranks(tmp_path):
    mp.spawn(_worker, args=(2, _free_port(), str(tmp_path), "sum"), nprocs=2, join=True)
    J_ref, g_ref = 0.0, torch.zeros(8, *SHAPE, dtype=torch.float64)
    for i in range(NSHOTS):
        Ji, gi = _fake_gradient(i)
        J_ref += Ji
        g_ref += gi
    r = [torch.load(tmp_path / f"r{k}.pt") for k in range(2)]
    assert sorted(r[0]["mine"] + r[1]["mine"]) == list(range(NSHOTS))
    for k in range(2):  # every rank ends with the full sum
        assert abs(r[k]["J"] - J_ref) <= 1e-12 * J_ref
        torch.testing.assert_close(r[k]["g"], g_ref, rtol=1e-12, atol=1e-12)
    assert torch.equal(r[0]["g"], r[1]["g"])


def test_fwi_driver_over_two_ranks(tmp_path):
    """Each rank evaluates its share of the shots; after the all-reduce both
    hold the single-process loss, gradient and line-search losses and take
    the same three optimizer steps."""
    mp.spawn(_worker, args=(2, _free_port(), str(tmp_path), "fwi"), nprocs=2, join=True)
    ref = _fwi_run(_fwi_problem())
    r = [torch.load(tmp_path / f"r{k}.pt", weights_only=False) for k in range(2)]
    assert sorted(r[0]["mine"] + r[1]["mine"]) == list(range(NSHOTS)) and r[0]["mine"] != r[1]["mine"]
    assert ref["hist"][-1] < ref["J"]
    for k in range(2):
        assert abs(r[k]["J"] - ref["J"]) <= 1e-12 * ref["J"]
        np.testing.assert_allclose(r[k]["g"], ref["g"], rtol=1e-12, atol=1e-14)
        np.testing.assert_allclose(r[k]["losses"], ref["losses"], rtol=1e-12)
        np.testing.assert_allclose(r[k]["theta"], ref["theta"], rtol=1e-12, atol=1e-14)
        np.testing.assert_allclose(r[k]["hist"], ref["hist"], rtol=1e-12)
    assert np.array_equal(r[0]["theta"], r[1]["theta"])


def test_rank_failure_surfaces_as_error(tmp_path):
    ctx = mp.start_processes(_worker, args=(2, _free_port(), str(tmp_path), "dies"), nprocs=2,
                             join=False, start_method="spawn")
    for p in ctx.processes:
        p.join(60)
    assert all(not p.is_alive() for p in ctx.processes)
    assert ctx.processes[1].exitcode == 3
    r0 = torch.load(tmp_path / "r0.pt")
    assert r0["err"] is not None
