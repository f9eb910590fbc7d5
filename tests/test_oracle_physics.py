"""Sanity of the oracle's physics (no reference test pins the step, so these
checks stand in): symmetry, absorption, the free-surface condition,
precision agreement, and chunked stepping."""
import numpy as np
import pytest

from viscoelasticinversion_b200 import media


def small_iso(nt=300, **kw):
    args = dict(nx=96, nz=96, dx=5.0, dt=0.5e-3, nt=nt, nsls=3, pml=16, nrec=20)
    args.update(kw)
    return media.homogeneous_iso(**args)


def test_symmetry_of_centred_explosive_source(oracle_lib):
    # homogeneous, no free surface, grid centred on the source column:
    # vz(i0 - k, j) = vz(i0 + k, j) while the front is inside the strips
    w = small_iso(nt=100, nx=97, free_surface=False)
    _, st = oracle_lib.run(w)
    i0 = w.sources[0][0]
    vz = st.v[1]
    left = vz[:, i0 - 30:i0]
    right = vz[:, i0 + 1:i0 + 31][:, ::-1]
    assert np.allclose(left, right, rtol=0, atol=1e-9 * np.abs(vz).max())
    # vx at i+1/2 is antisymmetric about the source node: vx(i0-1-k) = -vx(i0+k)
    vx = st.v[0]
    assert np.allclose(vx[:, i0 - 30:i0][:, ::-1], -vx[:, i0:i0 + 30], atol=1e-9 * np.abs(vx).max())


def test_cpml_absorbs_energy(oracle_lib):
    w = small_iso(nt=1200, free_surface=False, Q=1e6, nsls=0)
    energy = []
    st = None
    it = 0
    for chunk in range(6):
        _, st = oracle_lib.run(w, 200, state=st, it0=it)
        it += 200
        energy.append(float(np.sum(st.v**2)))
    # the pulse leaves through the CPML: kinetic energy falls by orders of magnitude
    assert energy[-1] < 1e-3 * max(energy)


def test_free_surface_condition_and_images(oracle_lib):
    w = small_iso(nt=200)
    _, st = oracle_lib.run(w)
    js = 4
    assert np.all(st.s[1, js] == 0)
    for k in range(1, 5):
        assert np.array_equal(st.s[1, js - k], -st.s[1, js + k])
    for k in range(4):
        assert np.array_equal(st.s[2, js - 1 - k], -st.s[2, js + k])
    assert np.all(st.m[3:6, js] == 0)          # Mzz = 0 on the surface
    assert np.all(st.v[:, :js] == 0)           # velocities above the surface stay zero


def test_chunked_run_equals_single_run(oracle_lib):
    w = small_iso(nt=120)
    tr1, st1 = oracle_lib.run(w)
    st = None
    tr = np.zeros_like(tr1)
    for it in range(0, 120, 40):
        t, st = oracle_lib.run(w, 40, state=st, it0=it)
        tr[:, :, it:it + 40] = t[:, :, it:it + 40]
    assert np.array_equal(tr, tr1)
    assert np.array_equal(st.v, st1.v) and np.array_equal(st.m, st1.m) and np.array_equal(st.psi, st1.psi)


@pytest.mark.parametrize("kind", ["iso", "vti", "tti"])
def test_f32_twin_tracks_f64(oracle_lib, kind):
    w = media.layered(nx=128, nz=96, nt=400, kind=kind, seed=5, pml=16, nrec=32)
    tr64, st64 = oracle_lib.run(w, precision="f64")
    tr32, st32 = oracle_lib.run(w, precision="f32")
    rel = np.linalg.norm(tr32 - tr64) / np.linalg.norm(tr64)
    assert rel < 1e-5, rel
    assert np.isfinite(tr64).all() and np.abs(tr64).max() > 0
