"""The committed golden step fixtures (tests/golden/step_*.npz, written by
tests/golden/make_golden.py from the FP64 oracle).

CPU: the workload builder still yields the fixture's medium and the oracle
still yields its traces and final planes (1e-13 relative L2: the oracle is
deterministic, but another host's compiler may round differently); the
oracle's FP32 twin meets the FP32 bar below.
GPU: the default CUDA step, through the C ABI, against the fixture:
  FP32 ... 1e-5 relative L2 (traces, every final plane, memory-variable norms)
  FP64 ... 1e-10
"""
import numpy as np
import pytest

from tests.golden.make_golden import CASES, medium_sum, path, workload
from tests.helpers import rel_l2

TOL = {"f32": 1e-5, "f64": 1e-10}


def _fixture(name):
    d = np.load(path(name))
    return {k: d[k] for k in d.files}


def _errors(traces, v, s, m_planes, g) -> dict:
    err = {"traces": rel_l2(traces, g["traces"]),
           "vx": rel_l2(v[0], g["v"][0]), "vz": rel_l2(v[1], g["v"][1]),
           "sxx": rel_l2(s[0], g["s"][0]), "szz": rel_l2(s[1], g["s"][1]),
           "sxz": rel_l2(s[2], g["s"][2])}
    norms = np.array([np.linalg.norm(m_planes[q]) for q in range(len(g["m_norm"]))])
    err["m_norm"] = float(np.max(np.abs(norms - g["m_norm"]) / g["m_norm"]))
    return err


@pytest.mark.parametrize("name", list(CASES))
def test_fixture_medium_and_oracle(oracle_lib, name):
    g = _fixture(name)
    w = workload(name)
    assert np.allclose(medium_sum(w), g["medium_sum"], rtol=1e-14, atol=0), \
        "the workload builder no longer yields the fixture's medium"
    assert np.abs(g["traces"]).max() > 0 and np.all(g["m_norm"] > 0)
    traces, st = oracle_lib.run(w, precision="f64")
    err = _errors(traces, st.v, st.s, st.m, g)
    assert max(err.values()) <= 1e-13, err


@pytest.mark.parametrize("name", list(CASES))
def test_fp32_oracle_matches_fixture(oracle_lib, name):
    """The oracle's FP32 twin — the timed CPU baseline and reference arm —
    meets the FP32 bar against the FP64 fixture, as the GPU path does."""
    g = _fixture(name)
    traces, st = oracle_lib.run(workload(name), precision="f32")
    err = _errors(traces, st.v, st.s, st.m.astype(np.float64), g)
    assert max(err.values()) <= TOL["f32"], err


@pytest.mark.gpu
@pytest.mark.parametrize("name", list(CASES))
@pytest.mark.parametrize("precision", ["f32", "f64"])
def test_default_step_matches_fixture(name, precision):
    from tests.helpers import run_gpu

    g = _fixture(name)
    w = workload(name)
    info = {}
    traces, st = run_gpu(w, precision, variant=0, info=info)
    assert info["kernel"] == "split"
    err = _errors(traces, st["v"], st["s"], st["m"], g)
    print(name, precision, err)
    assert max(err.values()) <= TOL[precision], err
