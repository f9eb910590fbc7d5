"""The streaming step kernel (kernel_variant 7, FP32 ISO/VTI) against the
FP64 oracle (relative L2 <= 1e-5 on the traces and every final field) and
against the split pair."""
import numpy as np
import pytest

from viscoelasticinversion_b200 import ViError, media
from tests.helpers import compare, rel_l2, run_gpu

pytestmark = pytest.mark.gpu

TOL = 1e-5


def _check(oracle_lib, w, **kw):
    tr_ref, st_ref = oracle_lib.run(w, precision="f64")
    assert np.abs(tr_ref).max() > 0
    info = {}
    tr, st = run_gpu(w, "f32", 7, info=info, **kw)
    assert info["kernel"] == "stream"
    err = compare(tr, st, tr_ref, st_ref, w.nsls)
    assert max(err.values()) <= TOL, err
    return tr, st


@pytest.mark.parametrize("case", ["iso256", "vti256x128", "vti200x100-nsls0", "iso184x96-nsls1",
                                  "vti136x72-nsls5"])
def test_stream_matches_oracle(oracle_lib, case):
    w = {
        "iso256": lambda: media.homogeneous_iso(nt=400),
        "vti256x128": lambda: media.layered(nx=256, nz=128, nt=500, kind="vti", seed=1, pml=20, nrec=64),
        # nx - 8 not a multiple of 128, nz - 8 not a multiple of 4
        "vti200x100-nsls0": lambda: media.layered(nx=200, nz=101, nt=300, kind="vti", seed=3, pml=12,
                                                  nrec=16, nsls=0),
        "iso184x96-nsls1": lambda: media.layered(nx=184, nz=96, nt=300, kind="iso", seed=4, pml=12,
                                                 nrec=16, nsls=1),
        "vti136x72-nsls5": lambda: media.layered(nx=136, nz=72, nt=250, kind="vti", seed=5, pml=10,
                                                 nrec=12, nsls=5),
    }[case]()
    _check(oracle_lib, w)


def test_stream_no_free_surface_force_sources(oracle_lib):
    w = media.layered(nx=160, nz=120, nt=300, kind="vti", seed=7, pml=12, nrec=16, free_surface=False)
    # force sources next to strip edges (column 131 is in the halo of the first strip)
    w.sources = [(131, 60, 1, 1.0), (132, 59, 2, -0.5), (40, 30, 0, 2.0), (80, 60, 2, 0.25)]
    w.wavelets = np.stack([w.wavelets[0]] * 4)
    _check(oracle_lib, w)


def test_stream_full_size_first_steps(oracle_lib):
    # 2048 x 1024: ~14 chunks per CTA, several pieces per strip
    w = media.layered(nt=160)
    _check(oracle_lib, w)


def test_stream_chunked_equals_one_call_and_split():
    w = media.layered(nx=256, nz=128, nt=301, kind="vti", seed=1, pml=20, nrec=64)
    tr1, st1 = run_gpu(w, "f32", 7)
    tr2, st2 = run_gpu(w, "f32", 7, chunks=[1, 100, 77, 123])
    assert np.array_equal(tr1, tr2)
    for k in ("v", "s", "m"):
        assert np.array_equal(st1[k], st2[k]), k
    tr5, _ = run_gpu(w, "f32", 5)
    assert rel_l2(tr1, tr5) < 1e-6


def test_stream_refuses_ineligible():
    w = media.layered(nx=128, nz=64, nt=10, kind="tti", seed=1, pml=8, nrec=4)
    with pytest.raises(ViError):
        run_gpu(w, "f32", 7)
    w = media.layered(nx=128, nz=64, nt=10, kind="vti", seed=1, pml=8, nrec=4)
    with pytest.raises(ViError):
        run_gpu(w, "f64", 7)
