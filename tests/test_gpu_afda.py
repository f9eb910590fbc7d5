"""The H-AFDA free surface (vi_config.free_surface = 2) on the GPU against
the FP64 oracle: the split pair (default, and both velocity-pass forms)
and the plain path, every medium, FP32 and FP64; the batched split form
bit for bit equal to the unbatched runs; the paths without it refuse it.
Reference: free-surface-kernels.jl:16-213, Stencil.jl:52-105."""
import dataclasses

import numpy as np
import pytest
import torch

from viscoelasticinversion_b200 import ViError, media
from viscoelasticinversion_b200._abi import VI_ERR_ARG
from viscoelasticinversion_b200.batch import ShotBatch
from viscoelasticinversion_b200.gradient import misfit_gradient
from viscoelasticinversion_b200 import StepPlan
from tests.helpers import compare, run_gpu

pytestmark = pytest.mark.gpu

TOL = {"f32": 1e-5, "f64": 1e-10}
_cache = {}


def _workload(kind):
    if kind == "iso":
        w = media.homogeneous_iso(nx=160, nz=96, nt=400, pml=16, nrec=24, src=(80, 20))
    else:
        w = media.layered(nx=192, nz=112, nt=400, kind=kind, seed=9, pml=16, nrec=24)
    return dataclasses.replace(w, free_surface=2)


def _oracle(oracle_lib, kind):
    if kind not in _cache:
        w = _workload(kind)
        _cache[kind] = (w,) + oracle_lib.run(w, precision="f64")
    return _cache[kind]


@pytest.mark.parametrize("kind", ["iso", "vti", "tti"])
@pytest.mark.parametrize("precision", ["f32", "f64"])
@pytest.mark.parametrize("variant", [0, 1, 5, 8])
def test_afda_parity_with_oracle(oracle_lib, kind, precision, variant):
    w, tr_ref, st_ref = _oracle(oracle_lib, kind)
    info = {}
    tr, st = run_gpu(w, precision, variant, info=info)
    assert info["kernel"] == {0: "split", 1: "plain", 5: "split", 8: "split-ldg"}[variant]
    err = compare(tr, st, tr_ref, st_ref, w.nsls)
    assert max(err.values()) <= TOL[precision], (kind, precision, variant, err)
    # nothing is written above the surface
    assert not np.any(st["s"][:, :4]) and not np.any(st["v"][:, :4])


def test_afda_default_on_unaligned_grid_runs_plain(oracle_lib):
    w = dataclasses.replace(media.homogeneous_iso(nx=98, nz=70, nt=200, pml=12, nrec=8, src=(49, 20)),
                            free_surface=2)
    tr_ref, st_ref = oracle_lib.run(w, precision="f64")
    info = {}
    tr, st = run_gpu(w, "f64", 0, info=info)
    assert info["kernel"] == "plain"
    assert max(compare(tr, st, tr_ref, st_ref, w.nsls).values()) <= 1e-10


@pytest.mark.parametrize("variant", [2, 3, 4, 6, 7])
def test_afda_refused_by_other_paths(variant):
    w = _workload("vti")
    with pytest.raises(ViError) as e:
        run_gpu(w, "f32", variant, nt=2)
    assert e.value.code == VI_ERR_ARG


def test_afda_gradient_refused():
    w = _workload("iso")
    plan = StepPlan.for_workload(w, "f64")
    med = plan.medium_to_device(w.medium)
    wav = torch.as_tensor(w.wavelets, dtype=plan.dtype, device=plan.device)
    obs = torch.zeros(2, len(w.receivers), w.nt, dtype=plan.dtype, device=plan.device)
    with pytest.raises(ViError) as e:
        misfit_gradient(plan, med, w.sources, wav, w.receivers, obs)
    assert e.value.code == VI_ERR_ARG
    plan.close()


def test_afda_batch_equals_unbatched(oracle_lib):
    grids = ((256, 128), (192, 96), (128, 128))
    ws = [dataclasses.replace(w, free_surface=2)
          for w in media.shot_gather(4, seed=2, kind="tti", nt_range=(90, 200), grids=grids, pml=12, nrec=16)]
    b = ShotBatch(ws, "f32")
    b.run()
    form = b.status()
    assert form in ("streams", "per-shot", "split")
    variant = {"streams": 0, "per-shot": 0, "split": 5}[form]
    for i, w in enumerate(ws):
        tr, st = b.result(i)
        tr1, st1 = run_gpu(w, "f32", variant)
        assert np.array_equal(tr, tr1), i
        if i == 0:
            tr_ref, st_ref = oracle_lib.run(w, precision="f64")
            assert max(compare(tr, st, tr_ref, st_ref, w.nsls).values()) <= 1e-5
    b.close()
