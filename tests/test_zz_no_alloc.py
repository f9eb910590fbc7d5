"""vi_step_noalloc (static device scratch, no allocation) against vi_step's
plain path: two calls in a row, each compared with the allocating entry
point's output.  Collected last on purpose."""
import ctypes as C

import numpy as np
import pytest
import torch

from viscoelasticinversion_b200 import StepPlan, media
from viscoelasticinversion_b200._abi import ViError, check, lib
from viscoelasticinversion_b200.solver import _stream_handle
from tests.helpers import rel_l2

pytestmark = pytest.mark.gpu


def _noalloc(plan, med, st, it0, n, w, wav, traces):
    f = plan.fields_struct(st["v"][0], st["v"][1], st["s"][0], st["s"][1], st["s"][2],
                           st["m"] if plan.nsls else None)
    m = plan._medium_struct(med)
    shot, keep = plan._shot(w.sources, wav, w.receivers, traces)
    check(lib().vi_step_noalloc(plan._h, C.byref(m), C.byref(f), C.byref(shot), int(it0), int(n),
                                _stream_handle(None)))
    del keep


@pytest.mark.parametrize("kind,precision", [("iso", "f32"), ("tti", "f32"), ("vti", "f64")])
def test_noalloc_matches_plain_step_two_calls(kind, precision):
    if kind == "iso":
        w = media.homogeneous_iso(nx=96, nz=80, nt=120, pml=12, nrec=16)
    else:
        w = media.layered(nx=128, nz=96, nt=120, kind=kind, pml=12, nrec=16, nlayers=4)
    plan = StepPlan.for_workload(w, precision)
    med = plan.medium_to_device(w.medium)
    wav = torch.as_tensor(w.wavelets, dtype=plan.dtype, device=plan.device).contiguous()
    tol = 1e-12 if precision == "f64" else 1e-6
    ref_st, new_st = plan.zeros_state(), plan.zeros_state()
    ref_tr = torch.zeros(2, len(w.receivers), w.nt, dtype=plan.dtype, device=plan.device)
    new_tr = torch.zeros_like(ref_tr)
    # reference: the allocating plain path, in the same two chunks
    plan.reset()
    it = 0
    ref_chunks = []
    for n in (70, 50):
        plan.step(med, ref_st, nsteps=n, it0=it, sources=w.sources, wavelets=wav,
                  receivers=w.receivers, traces=ref_tr, variant=1)
        plan.status()
        ref_chunks.append(({k: v.clone() for k, v in ref_st.items()}, ref_tr.clone()))
        it += n
    plan.reset()
    it = 0
    for k, n in enumerate((70, 50)):  # two calls in a row
        _noalloc(plan, med, new_st, it, n, w, wav, new_tr)
        plan.status()
        st_ref, tr_ref = ref_chunks[k]
        assert rel_l2(new_tr.double().cpu().numpy(), tr_ref.double().cpu().numpy()) <= tol
        for name in ("v", "s", "m"):
            assert rel_l2(new_st[name].double().cpu().numpy(),
                          st_ref[name].double().cpu().numpy()) <= tol, (k, name)
        it += n
    assert np.abs(new_tr.double().cpu().numpy()).max() > 0
    plan.close()


def test_noalloc_rejects_oversize_grid():
    # 6 FP64 planes of 1024 x 1024 exceed the 24 MiB static array
    w = media.homogeneous_iso(nx=1024, nz=1024, nt=4, pml=12, nrec=4)
    plan = StepPlan.for_workload(w, "f64")
    med = plan.medium_to_device(w.medium)
    st = plan.zeros_state()
    wav = torch.as_tensor(w.wavelets, dtype=plan.dtype, device=plan.device).contiguous()
    tr = torch.zeros(2, len(w.receivers), w.nt, dtype=plan.dtype, device=plan.device)
    with pytest.raises(ViError, match="static scratch"):
        _noalloc(plan, med, st, 0, 2, w, wav, tr)
    plan.close()
