"""vi_step_noalloc (static device scratch, no allocation) against vi_step's
plain path: two calls in a row, each compared bit for bit with the
allocating entry point's output, with no device memory taken by either
call.  Collected last on purpose: callers that cannot allocate (a process
sharing the GPU with a serving loop, a fully reserved memory pool) depend
on this path, and every other test has run before it."""
import ctypes as C

import pytest
import torch

from viscoelasticinversion_b200 import StepPlan, media
from viscoelasticinversion_b200._abi import ViError, check, lib
from viscoelasticinversion_b200.solver import _stream_handle

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
    """Two vi_step_noalloc calls in a row on a fresh plan that has never run
    vi_step, each bitwise equal to vi_step's plain path (the same kernels)
    after the same steps, with the plan's device bytes and the device's
    free memory unchanged across both calls."""
    if kind == "iso":
        w = media.homogeneous_iso(nx=96, nz=80, nt=120, pml=12, nrec=16)
    else:
        w = media.layered(nx=128, nz=96, nt=120, kind=kind, pml=12, nrec=16, nlayers=4)
    chunks = (70, 50)
    # reference: the allocating plain path on its own plan, in the same chunks
    ref = StepPlan.for_workload(w, precision)
    med = ref.medium_to_device(w.medium)
    wav = torch.as_tensor(w.wavelets, dtype=ref.dtype, device=ref.device).contiguous()
    ref_st = ref.zeros_state()
    ref_tr = torch.zeros(2, len(w.receivers), w.nt, dtype=ref.dtype, device=ref.device)
    ref.reset()
    it, ref_chunks = 0, []
    for n in chunks:
        ref.step(med, ref_st, nsteps=n, it0=it, sources=w.sources, wavelets=wav,
                 receivers=w.receivers, traces=ref_tr, variant=1)
        ref.status()
        ref_chunks.append(({k: v.clone() for k, v in ref_st.items()}, ref_tr.clone()))
        it += n
    # one throw-away call on the reference plan loads the module that holds
    # the static array and the plain kernels (lazy loading maps them on first
    # use), so the measured calls below start from a loaded library
    warm_st = ref.zeros_state()
    _noalloc(ref, med, warm_st, 0, 2, w, wav, torch.zeros_like(ref_tr))
    ref.status()
    # the plan under test has never run vi_step: nothing was grown on it
    plan = StepPlan.for_workload(w, precision)
    new_st = plan.zeros_state()
    new_tr = torch.zeros_like(ref_tr)
    first = ({k: torch.empty_like(v) for k, v in new_st.items()}, torch.empty_like(new_tr))
    torch.cuda.synchronize()
    bytes0 = plan.workspace_bytes()
    free0 = torch.cuda.mem_get_info()[0]
    plan.reset()
    it = 0
    for k, n in enumerate(chunks):  # two calls in a row
        _noalloc(plan, med, new_st, it, n, w, wav, new_tr)
        plan.status()
        if k == 0:  # copy into buffers allocated before the measurement
            for name, t in new_st.items():
                first[0][name].copy_(t)
            first[1].copy_(new_tr)
        it += n
    torch.cuda.synchronize()
    assert plan.workspace_bytes() == bytes0
    assert torch.cuda.mem_get_info()[0] == free0
    for (st_got, tr_got), (st_ref, tr_ref) in zip((first, (new_st, new_tr)), ref_chunks):
        assert torch.equal(tr_got, tr_ref)
        for name in ("v", "s", "m"):
            assert torch.equal(st_got[name], st_ref[name]), name
    assert new_tr.abs().max().item() > 0
    plan.close()
    ref.close()


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
