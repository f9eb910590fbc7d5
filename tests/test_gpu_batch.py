"""Batched shots (vi_batch): every shot of a batch of uneven grids and
step counts equals its own unbatched run, with and without the CUDA graph,
and agrees with the FP64 oracle."""
import numpy as np
import pytest

from viscoelasticinversion_b200 import media
from viscoelasticinversion_b200.batch import ShotBatch
from tests.helpers import compare, rel_l2, run_gpu

pytestmark = pytest.mark.gpu


def small_gather(kind, seed=0, n=6):
    grids = ((256, 128), (192, 96), (128, 128), (320, 160))
    return media.shot_gather(n, seed=seed, kind=kind, nt_range=(90, 220), grids=grids, pml=12,
                             nrec=24)


@pytest.mark.parametrize("kind", ["tti", "vti", "iso"])
def test_batch_equals_unbatched_and_oracle(oracle_lib, kind):
    ws = small_gather(kind)
    b = ShotBatch(ws, "f32")
    b.run()
    form = b.status()
    variant = {"streams": 0, "per-shot": 0, "split": 5, "two-stage": 3, "one-stage": 4}[form]
    for i, w in enumerate(ws):
        tr, st = b.result(i)
        tr1, st1 = run_gpu(w, "f32", variant)
        # same kernel arithmetic: bit-identical to the unbatched run
        assert np.array_equal(tr, tr1), (i, rel_l2(tr, tr1))
        for k in ("v", "s"):
            assert np.array_equal(st[k], st1[k]), (i, k)
        if i < 2:
            tr_ref, st_ref = oracle_lib.run(w, precision="f64")
            err = compare(tr, st, tr_ref, st_ref, w.nsls)
            assert max(err.values()) < 1e-5, (i, err)
    b.close()


def test_graph_and_direct_launches_agree_and_runs_repeat():
    ws = small_gather("tti", seed=3, n=5)
    b = ShotBatch(ws, "f32")
    b.run(graph=True)
    first = [b.result(i)[0] for i in range(len(ws))]
    b.reset()
    b.run(graph=True)  # cached graph, from rest again
    second = [b.result(i)[0] for i in range(len(ws))]
    b.reset()
    b.run(graph=False)
    third = [b.result(i)[0] for i in range(len(ws))]
    for a, c, d in zip(first, second, third):
        assert np.array_equal(a, c) and np.array_equal(a, d)
    b.close()


def test_retune_keeps_results():
    ws = small_gather("vti", seed=5, n=4)
    b = ShotBatch(ws, "f32")
    b.run()
    r1 = [b.result(i)[0] for i in range(len(ws))]
    b.reset()
    b.run(retune=True)
    r2 = [b.result(i)[0] for i in range(len(ws))]
    for x, y in zip(r1, r2):
        assert rel_l2(x, y) < 1e-5
    b.close()


@pytest.mark.parametrize("kind", ["vti", "tti"])
def test_compensated_batch_matches_unbatched_and_oracle(oracle_lib, kind):
    """Compensated FP32 (VI_F32C) shots run on the split form (or one by one)
    and agree with their own unbatched runs to rounding (TTI bit for bit;
    ISO/VTI within 1e-6: the merged and single-shot stress kernels round the
    last bit of a few cells differently) and with the FP64 oracle."""
    ws = small_gather(kind, seed=1, n=4)
    b = ShotBatch(ws, "f32c")
    b.run()
    form = b.status()
    assert form in ("streams", "per-shot", "split")
    variant = {"streams": 0, "per-shot": 0, "split": 5}[form]
    for i, w in enumerate(ws):
        tr, st = b.result(i)
        tr1, st1 = run_gpu(w, "f32c", variant)
        assert rel_l2(tr, tr1) <= 1e-6, (i, rel_l2(tr, tr1))
        if kind == "tti":
            assert np.array_equal(tr, tr1), i
        if i == 0:
            tr_ref, st_ref = oracle_lib.run(w, precision="f64")
            err = compare(tr, st, tr_ref, st_ref, w.nsls)
            assert max(err.values()) < 1e-5, err
    b.close()
