"""The time-blocked split step (kernel variant 9) against the one-launch-per-
pass split pair (variant 5): the same tile code in another order, so the
traces and every final field must be bitwise equal; and against the FP64
oracle at the parity tolerances (1e-5 FP32, 1e-10 FP64)."""
import numpy as np
import pytest
import torch

from viscoelasticinversion_b200 import StepPlan, ViError, media
from tests.helpers import compare

pytestmark = pytest.mark.gpu


def _run(w, precision, variant, wave=None, chunks=None):
    plan = StepPlan.for_workload(w, precision)
    if wave is not None:
        plan.set_wave(*wave)
    med = plan.medium_to_device(w.medium)
    st = plan.zeros_state()
    wav = torch.as_tensor(w.wavelets, dtype=plan.dtype, device=plan.device).contiguous()
    tr = torch.zeros(2, len(w.receivers), w.nt, dtype=plan.dtype, device=plan.device)
    it = 0
    for n in chunks or [w.nt]:
        plan.step(med, st, nsteps=n, it0=it, sources=w.sources, wavelets=wav,
                  receivers=w.receivers, traces=tr, variant=variant)
        it += n
    plan.status()
    kernel = plan.last_kernel()
    out = {k: v.cpu().numpy() for k, v in st.items()}
    plan.close()
    return tr.cpu().numpy(), out, kernel


def _bitwise(a, b):
    tr_a, st_a, _ = a
    tr_b, st_b, _ = b
    assert np.array_equal(tr_a, tr_b)
    for k in st_a:
        assert np.array_equal(st_a[k], st_b[k]), k


CASES = {
    # partial last band (nz - 8 not a multiple of 8), one stress tile row in it
    "vti196x100": lambda: media.layered(nx=196, nz=100, nt=120, kind="vti", seed=3, pml=12, nrec=16),
    # more velocity tiles per band than stress tiles (ntx_v = 5, 2 ntx_s = 4)
    "iso264x60": lambda: media.layered(nx=264, nz=60, nt=90, kind="iso", seed=4, pml=10, nrec=9,
                                       free_surface=False),
    "vti256x128": lambda: media.layered(nx=256, nz=128, nt=200, kind="vti", seed=1, pml=20, nrec=64),
}


@pytest.mark.parametrize("name", sorted(CASES))
@pytest.mark.parametrize("precision", ["f32", "f64"])
@pytest.mark.parametrize("wave", [(0, 0), (1, 2), (3, 2), (8, 5), (64, 64)])
def test_wave_bitwise_equals_split(name, precision, wave):
    w = CASES[name]()
    ref = _run(w, precision, 5)
    got = _run(w, precision, 9, wave=wave)
    assert got[2] == "wave"
    _bitwise(got, ref)


@pytest.mark.parametrize("nsls", [0, 1, 5])
def test_wave_instantiations_and_chunks(nsls):
    """Every N_sls instantiation, calls of uneven length continuing one
    another (sweeps cut at call boundaries)."""
    w = media.layered(nx=192, nz=84, nt=77, kind="vti", seed=11, pml=12, nrec=16, nsls=nsls)
    ref = _run(w, "f32", 5)
    got = _run(w, "f32", 9, wave=(5, 3), chunks=[1, 30, 0, 46])
    _bitwise(got, ref)


def test_wave_parity_with_oracle(oracle_lib):
    w = media.layered(nx=256, nz=128, nt=600, kind="vti", seed=1, pml=20, nrec=64)
    tr_ref, st_ref = oracle_lib.run(w, precision="f64")
    for precision, tol in (("f32", 1e-5), ("f64", 1e-10)):
        tr, st, kernel = _run(w, precision, 9)
        assert kernel == "wave"
        st = {k: v.astype(np.float64) for k, v in st.items()}
        st["m"] = st["m"].reshape(-1, w.nz, w.nx)
        err = compare(tr.astype(np.float64), st, tr_ref, st_ref, w.nsls)
        bad = {k: v for k, v in err.items() if not v <= tol}
        assert not bad, f"{precision}: {err}"


def test_wave_refuses_what_it_does_not_cover():
    tti = media.layered(nx=128, nz=64, nt=4, kind="tti", seed=2, pml=8, nrec=4)
    with pytest.raises(ViError):
        _run(tti, "f32", 9)
    odd = media.homogeneous_iso(nx=37, nz=29, nt=4, pml=6, nrec=3, src=(18, 14))
    with pytest.raises(ViError):
        _run(odd, "f32", 9)
    w = media.layered(nx=128, nz=64, nt=4, kind="vti", seed=2, pml=8, nrec=4)
    plan = StepPlan.for_workload(w, "f32")
    with pytest.raises(ViError):
        plan.set_wave(4, 1)  # lags below 2 are refused (2 keeps every dependency at an earlier tau)
    plan.close()


def test_autotuner_choice_is_cached_and_exact():
    """tune() times the split pair and the time-blocked forms for the grid
    class; variant="auto" then runs the choice, bitwise equal to the split
    pair whichever form won."""
    from viscoelasticinversion_b200 import solver

    w = media.layered(nx=256, nz=128, nt=60, kind="vti", seed=5, pml=16, nrec=8)
    plan = StepPlan.for_workload(w, "f32")
    med = plan.medium_to_device(w.medium)
    choice = plan.tune(med, nsteps=8, reps=1)
    assert choice["variant"] in (5, 9)
    assert "split" in choice["us_per_step"] and len(choice["us_per_step"]) == 1 + len(plan.WAVE_CANDIDATES)
    assert solver._TUNED[plan._tune_key()] is choice
    plan.close()
    ref = _run(w, "f32", 5)
    got = _run(w, "f32", "auto")
    _bitwise(got, ref)
