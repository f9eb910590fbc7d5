"""Shot sharding and the gradient all-reduce across ranks, on CPU with the
gloo backend (world size 2): the same host logic that runs over NCCL on
GPUs.  Also the failure path: a rank that dies before the all-reduce makes
the survivor's collective end with an error instead of hanging."""
import datetime
import os
import socket

import pytest
import torch
import torch.distributed as dist
import torch.multiprocessing as mp

from viscoelasticinversion_b200.gradient import reduce_gradient, shard, shot_gradient

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


def _worker(rank, world, port, out_dir, mode):
    dist.init_process_group("gloo", init_method=f"tcp://127.0.0.1:{port}", rank=rank,
                            world_size=world, timeout=datetime.timedelta(seconds=8))
    try:
        if mode == "sum":
            J, g = shot_gradient(_fake_gradient, NSHOTS, SHAPE)
            torch.save({"J": J, "g": g, "mine": shard(NSHOTS, rank, world)},
                       os.path.join(out_dir, f"r{rank}.pt"))
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


def test_rank_failure_surfaces_as_error(tmp_path):
    ctx = mp.start_processes(_worker, args=(2, _free_port(), str(tmp_path), "dies"), nprocs=2,
                             join=False, start_method="spawn")
    for p in ctx.processes:
        p.join(60)
    assert all(not p.is_alive() for p in ctx.processes)
    assert ctx.processes[1].exitcode == 3
    r0 = torch.load(tmp_path / "r0.pt")
    assert r0["err"] is not None
