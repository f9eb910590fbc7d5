"""Writes the golden step fixtures of tests/golden/ from the FP64 oracle.

Each case is a small seeded layered workload (96 x 32 cells, wider than
every TMA box of the split step; 3 SLS, 6-cell CPML, free surface, one
explosive 25 Hz Ricker, 8 receivers, 160 steps) run from rest by the
oracle.  A fixture (step_<case>.npz) holds:

  traces      [2, nrec, nt]  vx and vz at the receivers (float64)
  v, s        [2|3, nz, nx]  final velocity and stress planes (float64)
  m_norm      [3 * nsls]     L2 norm of every final memory-variable plane
  medium_sum  [nplanes]      sum of every medium plane, in workload order

medium_sum tells a change of the workload builder (numpy / scipy random
streams) apart from a change of the step.  The fixtures are test data of
the oracle; tests/test_golden_fixtures.py checks the oracle against them on
the CPU and the CUDA step against them on the GPU.

Usage: python -m tests.golden.make_golden
"""
from __future__ import annotations

from pathlib import Path

import numpy as np

HERE = Path(__file__).resolve().parent

CASES = {
    "iso96x32": {"kind": "iso", "seed": 21},
    "vti96x32": {"kind": "vti", "seed": 22},
    "tti96x32": {"kind": "tti", "seed": 23},
}


def workload(name: str):
    from viscoelasticinversion_b200 import media

    c = CASES[name]
    return media.layered(nx=96, nz=32, nt=160, kind=c["kind"], seed=c["seed"], nlayers=4,
                         pml=6, f0=25.0, nrec=8, corr=15.0)


def path(name: str) -> Path:
    return HERE / f"step_{name}.npz"


def medium_sum(w) -> np.ndarray:
    return np.array([float(np.sum(w.medium[k])) for k in w.planes()])


def make(name: str) -> Path:
    import oracle

    oracle.build()
    w = workload(name)
    traces, st = oracle.run(w, precision="f64")
    nm = 3 * w.nsls
    m_norm = np.array([np.linalg.norm(st.m[q]) for q in range(nm)])
    np.savez_compressed(path(name), traces=traces, v=st.v, s=st.s, m_norm=m_norm,
                        medium_sum=medium_sum(w))
    return path(name)


if __name__ == "__main__":
    for n in CASES:
        print(make(n))
