"""The request server (vi_serve): every request's results equal the direct
call on the same inputs, alone or in a mix of grids, media and step counts
served in slices by several lanes at once; gradients through the server
equal vi_gradient; requests overlap on the device; HBM-budget admission;
failure reporting."""
import numpy as np
import pytest
import torch

from viscoelasticinversion_b200 import StepPlan, ViError, media
from viscoelasticinversion_b200.gradient import misfit_gradient
from viscoelasticinversion_b200.serve import Server
from tests.helpers import rel_l2

pytestmark = pytest.mark.gpu


def _mix():
    return [
        media.homogeneous_iso(nx=96, nz=80, nt=150, pml=12, nrec=16, src=(40, 30)),
        media.layered(nx=160, nz=96, nt=230, kind="vti", seed=1, pml=12, nrec=16),
        media.layered(nx=128, nz=96, nt=170, kind="tti", seed=2, pml=12, nrec=16),
        media.homogeneous_iso(nx=37, nz=29, nt=90, pml=6, nrec=7, src=(18, 14)),
        media.layered(nx=136, nz=72, nt=201, kind="vti", seed=5, pml=10, nrec=12, nsls=1),
    ]


def _direct(w, precision):
    plan = StepPlan.for_workload(w, precision)
    tr = plan.forward_host(w.medium, w.sources, w.wavelets, w.receivers, w.nt)
    plan.close()
    return tr


@pytest.mark.parametrize("precision", ["f32", "f64"])
def test_forward_requests_equal_direct_calls(precision):
    ws = _mix()
    srv = Server(slice_steps=64)
    tickets = [srv.submit_forward(w, precision) for w in ws]
    for t in tickets:
        assert srv.wait(t, 120.0) == "done"
    for w, t in zip(ws, tickets):
        state, lat = srv.poll(t)
        assert state == "done" and lat > 0
        assert np.array_equal(t.traces, _direct(w, precision)), w.name
        assert np.abs(t.traces).max() > 0
    srv.stop()


def test_same_alone_and_in_the_mix():
    ws = _mix()
    srv = Server(slice_steps=50)
    alone = srv.submit_forward(ws[1])
    assert srv.wait(alone, 120.0) == "done"
    mixed = [srv.submit_forward(w) for w in ws]
    for t in mixed:
        srv.wait(t, 120.0)
    assert np.array_equal(alone.traces, mixed[1].traces)
    srv.stop()


def test_gradient_request_equals_vi_gradient(oracle_lib):
    w = media.homogeneous_iso(nx=96, nz=80, nt=160, pml=12, nrec=16, src=(40, 30))
    truth = dict(w.medium)
    truth["c55"] = truth["c55"] * 1.03
    import dataclasses
    obs, _ = oracle_lib.run(dataclasses.replace(w, medium=truth), precision="f64")
    srv = Server(slice_steps=64)
    fwd = srv.submit_forward(w, "f64")
    gt = srv.submit_gradient(w, obs, "f64")
    assert srv.wait(gt, 120.0) == "done" and srv.wait(fwd, 120.0) == "done"
    srv.stop()
    plan = StepPlan.for_workload(w, "f64")
    med = plan.medium_to_device(w.medium)
    wav = torch.as_tensor(w.wavelets, dtype=plan.dtype, device=plan.device).contiguous()
    obs_d = torch.as_tensor(obs, dtype=plan.dtype, device=plan.device).contiguous()
    J, g = misfit_gradient(plan, med, w.sources, wav, w.receivers, obs_d)
    plan.close()
    assert gt.misfit[0] == J
    assert np.array_equal(gt.grad, g.cpu().numpy())
    # the gradient's forward run (plain kernels) reproduces the forward solve
    assert rel_l2(gt.traces, fwd.traces) <= 1e-12


@pytest.mark.parametrize("lanes", [1, 3])
def test_mix_equal_direct_calls_for_any_lane_count(lanes):
    ws = _mix()
    srv = Server(slice_steps=40, lanes=lanes, policy="round-robin")
    tickets = [srv.submit_forward(w) for w in ws]
    for t in tickets:
        assert srv.wait(t, 120.0) == "done"
    srv.stop()
    for w, t in zip(ws, tickets):
        assert np.array_equal(t.traces, _direct(w, "f32")), w.name


def test_short_request_finishes_while_a_gradient_runs():
    """With two lanes a small forward solve submitted while a long gradient
    is on the device completes before the gradient does (its work overlaps
    the gradient's instead of waiting for it)."""
    big = media.homogeneous_iso(nx=1024, nz=512, nt=1200, pml=20, nrec=32, src=(512, 100))
    obs = np.zeros((2, len(big.receivers), big.nt), np.float32)
    small = media.homogeneous_iso(nx=96, nz=80, nt=60, pml=12, nrec=8, src=(40, 30))
    srv = Server(lanes=2)
    g = srv.submit_gradient(big, obs, "f32")
    import time
    t0 = time.perf_counter()
    while srv.poll(g)[0] != "running" and time.perf_counter() - t0 < 30:
        time.sleep(0.002)
    time.sleep(0.02)
    f = srv.submit_forward(small)
    assert srv.wait(f, 60.0) == "done"
    assert srv.poll(g)[0] == "running"
    assert srv.wait(g, 120.0) == "done"
    srv.stop()
    assert np.array_equal(f.traces, _direct(small, "f32"))


def test_gradient_is_sliced_on_one_lane():
    """Gradient requests advance in slices like forward ones: on a single
    lane a small forward solve submitted while a long gradient runs still
    completes first, and the sliced gradient equals the direct call."""
    big = media.homogeneous_iso(nx=512, nz=256, nt=1200, pml=20, nrec=16, src=(256, 60))
    obs = np.zeros((2, len(big.receivers), big.nt), np.float32)
    small = media.homogeneous_iso(nx=96, nz=80, nt=60, pml=12, nrec=8, src=(40, 30))
    srv = Server(lanes=1, slice_steps=256)
    g = srv.submit_gradient(big, obs, "f32")
    import time
    t0 = time.perf_counter()
    while srv.poll(g)[0] != "running" and time.perf_counter() - t0 < 30:
        time.sleep(0.002)
    f = srv.submit_forward(small)
    assert srv.wait(f, 60.0) == "done"
    assert srv.poll(g)[0] == "running"
    assert srv.wait(g, 120.0) == "done"
    srv.stop()
    plan = StepPlan.for_workload(big, "f32")
    med = plan.medium_to_device(big.medium)
    wav = torch.as_tensor(big.wavelets, dtype=plan.dtype, device=plan.device).contiguous()
    obs_d = torch.as_tensor(obs, dtype=plan.dtype, device=plan.device).contiguous()
    J, gd = misfit_gradient(plan, med, big.sources, wav, big.receivers, obs_d)
    plan.close()
    assert g.misfit[0] == J and np.array_equal(g.grad, gd.cpu().numpy())


def test_budget_admission():
    w = media.homogeneous_iso(nx=96, nz=80, nt=120, pml=12, nrec=8, src=(40, 30))
    small = Server(hbm_budget_bytes=1 << 20)
    with pytest.raises(ViError) as e:
        small.submit_forward(w)
    assert e.value.code == 3  # VI_ERR_BUDGET
    small.stop()
    # room for about one request at a time: all complete, one after another
    one = Server(hbm_budget_bytes=25 << 20, slice_steps=30)
    ts = [one.submit_forward(w) for _ in range(3)]
    for t in ts:
        assert one.wait(t, 120.0) == "done"
    ref = _direct(w, "f32")
    for t in ts:
        assert np.array_equal(t.traces, ref)
    one.stop()


def test_failed_request_reports_error():
    import dataclasses

    w = media.layered(nx=128, nz=64, nt=40, kind="tti", seed=1, pml=8, nrec=4)
    bad = dataclasses.replace(w, free_surface=2)  # the adjoint covers the imaging surface only
    srv = Server()
    t = srv.submit_gradient(bad, np.zeros((2, len(w.receivers), w.nt)), "f64")
    with pytest.raises(ViError, match="H-AFDA"):
        srv.wait(t, 60.0)
    with pytest.raises(ViError):
        srv.poll(t)
    ok = srv.submit_forward(w)  # the server keeps serving
    assert srv.wait(ok, 60.0) == "done"
    srv.stop()
