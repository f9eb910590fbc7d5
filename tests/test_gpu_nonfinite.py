"""Non-finite detection: a NaN planted in the medium on the host makes the
stresses non-finite within a step, and every path reports VI_ERR_NONFINITE
through the plan's (or the batch's) error word instead of returning VI_OK.
The split pair folds the check into its stress pass; the other step paths
check the stresses once at the end of each call.  Nothing faults: the NaN
is ordinary data to the kernels."""
import numpy as np
import pytest
import torch

from viscoelasticinversion_b200 import StepPlan, ViError, media
from viscoelasticinversion_b200._abi import VI_ERR_NONFINITE
from viscoelasticinversion_b200.batch import ShotBatch

pytestmark = pytest.mark.gpu


def _poisoned(kind, nan_at=None):
    w = media.layered(nx=128, nz=96, nt=40, kind=kind, seed=4, pml=12, nrec=8)
    if nan_at is not None:
        rho = w.medium["rho"].copy()
        rho[nan_at] = np.nan
        w.medium = dict(w.medium, rho=rho)
    return w


def _run(w, precision, variant):
    plan = StepPlan.for_workload(w, precision)
    med = plan.medium_to_device(w.medium)
    st = plan.zeros_state()
    wav = torch.as_tensor(w.wavelets, dtype=plan.dtype, device=plan.device).contiguous()
    tr = torch.zeros(2, len(w.receivers), w.nt, dtype=plan.dtype, device=plan.device)
    try:
        plan.step(med, st, nsteps=w.nt, sources=w.sources, wavelets=wav, receivers=w.receivers,
                  traces=tr, variant=variant)
        plan.status()
    finally:
        plan.close()


@pytest.mark.parametrize("kind", ["vti", "tti"])
@pytest.mark.parametrize("precision", ["f32", "f64"])
@pytest.mark.parametrize("variant", [0, 1, 3])
def test_nan_medium_reported(kind, precision, variant):
    _run(_poisoned(kind), precision, variant)  # clean medium: no error
    with pytest.raises(ViError) as e:
        _run(_poisoned(kind, nan_at=(60, 70)), precision, variant)
    assert e.value.code == VI_ERR_NONFINITE


def test_nan_reported_by_forward_host_and_cleared():
    w = _poisoned("vti", nan_at=(50, 64))
    plan = StepPlan.for_workload(w, "f32")
    with pytest.raises(ViError) as e:
        plan.forward_host(w.medium, w.sources, w.wavelets, w.receivers, w.nt)
    assert e.value.code == VI_ERR_NONFINITE
    # the error word is cleared by the report: a clean run on the same plan succeeds
    clean = _poisoned("vti")
    tr = plan.forward_host(clean.medium, clean.sources, clean.wavelets, clean.receivers, clean.nt)
    assert np.isfinite(tr).all() and np.abs(tr).max() > 0
    plan.close()


def test_nan_reported_by_batch():
    ws = [_poisoned("tti"), _poisoned("tti", nan_at=(40, 30))]
    b = ShotBatch(ws, "f32")
    b.run()
    with pytest.raises(ViError) as e:
        b.status()
    assert e.value.code == VI_ERR_NONFINITE
    b.close()
