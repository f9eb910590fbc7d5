"""SEG-Y model ingest (segy.py), on the CPU: IBM hexadecimal float
known answers, write/read round trips in both sample formats, a file laid
out by hand (ASCII text header, one extended textual header, IEEE
samples), error paths, and a workload built from vp / vs / rho model files
that the oracle steps."""
import numpy as np
import pytest

from viscoelasticinversion_b200 import media, segy

# IBM float words and their values: -118.625 is the textbook example
# (sign 1, exponent 0x42, fraction 0x76A000); the others are exact powers.
IBM_KNOWN = [(0xC276A000, -118.625), (0x42640000, 100.0), (0x41100000, 1.0),
             (0x40800000, 0.5), (0xC1100000, -1.0), (0x00000000, 0.0)]


def test_ibm_known_answers_both_ways():
    words = np.array([w for w, _ in IBM_KNOWN], dtype=np.uint32)
    vals = np.array([v for _, v in IBM_KNOWN])
    assert np.array_equal(segy.ibm_to_ieee(words), vals.astype(np.float32))
    assert np.array_equal(segy.ieee_to_ibm(vals), words)


def test_ibm_round_trip_precision():
    rng = np.random.default_rng(3)
    x = (rng.standard_normal(4000) * 10.0 ** rng.uniform(-20, 20, 4000)).astype(np.float32)
    back = segy.ibm_to_ieee(segy.ieee_to_ibm(x))
    # 24-bit hexadecimal fraction: at least 21 significant bits, rounded
    assert np.all(np.abs(back.astype(np.float64) - x) <= 2.0**-21 * np.abs(x.astype(np.float64)))
    # values that need no rounding come back exactly
    exact = np.array([3.0, -0.15625, 1500.0, 2.0**-10], dtype=np.float32)
    assert np.array_equal(segy.ibm_to_ieee(segy.ieee_to_ibm(exact)), exact)


@pytest.mark.parametrize("fmt", [1, 5])
def test_write_read_round_trip(tmp_path, fmt):
    rng = np.random.default_rng(fmt)
    data = rng.uniform(1500.0, 4500.0, (37, 11)).astype(np.float32)
    p = tmp_path / f"model_{fmt}.segy"
    segy.segy_write(p, data, dt_us=1250, fmt=fmt, text="C 1 test model\nC 2 second line",
                    traceheaders={"SourceX": np.arange(11) * 10, "RecSourceScalar": -100})
    assert p.stat().st_size == 3200 + 400 + 11 * (240 + 37 * 4)
    b = segy.segy_read(p)
    assert b.fileheader["ns"] == 37 and b.fileheader["dt"] == 1250
    assert b.fileheader["DataSampleFormat"] == fmt and b.fileheader["SegyFormatRevisionNumber"] == 0x0100
    assert b.data.shape == (37, 11) and b.data.dtype == np.float32
    tol = 0 if fmt == 5 else 2.0**-21
    assert np.all(np.abs(b.data - data) <= tol * np.abs(data))
    assert list(b.traceheaders["TraceNumber"]) == list(range(1, 12))
    assert list(b.traceheaders["SourceX"]) == list(np.arange(11) * 10)
    assert np.all(b.traceheaders["RecSourceScalar"] == -100) and np.all(b.traceheaders["ns"] == 37)
    assert b.text_header.startswith("C 1 test model") and b.text_header[80:].startswith("C 2 second")


def test_hand_built_ascii_file_with_extended_header(tmp_path):
    ns, ntr = 5, 3
    text = ("C 1 ASCII HEADER".ljust(80) * 40).encode("ascii")
    bfh = np.zeros(400, dtype=np.uint8)
    for off, val in ((16, 2000), (20, ns), (24, 5), (300, 0x0100), (304, 1)):
        bfh[off:off + 2] = np.frombuffer(np.array(val, ">i2").tobytes(), np.uint8)
    ext = ("(( EXTENDED ))".ljust(3200)).encode("cp037")
    traces = b""
    vals = np.arange(ns * ntr, dtype=np.float32).reshape(ntr, ns) + 0.5
    for t in range(ntr):
        h = np.zeros(240, dtype=np.uint8)
        h[12:16] = np.frombuffer(np.array(t + 7, ">i4").tobytes(), np.uint8)  # TraceNumber
        traces += h.tobytes() + vals[t].astype(">f4").tobytes()
    p = tmp_path / "hand.sgy"
    p.write_bytes(text + bfh.tobytes() + ext + traces)
    b = segy.segy_read(p)
    assert b.text_header.startswith("C 1 ASCII HEADER")
    assert len(b.extended_text) == 1 and b.extended_text[0].startswith("(( EXTENDED ))")
    assert np.array_equal(b.data, vals.T)
    assert list(b.traceheaders["TraceNumber"]) == [7, 8, 9]


def test_read_errors(tmp_path):
    p = tmp_path / "short.segy"
    p.write_bytes(b"\0" * 1000)
    with pytest.raises(ValueError, match="shorter"):
        segy.segy_read(p)
    q = tmp_path / "m.segy"
    segy.segy_write(q, np.ones((4, 2)), dt_us=1000, fmt=5)
    raw = bytearray(q.read_bytes())
    raw[3224:3226] = np.array(4, ">i2").tobytes()  # format 4 (fixed point with gain): unsupported
    q.write_bytes(bytes(raw))
    with pytest.raises(ValueError, match="format code 4"):
        segy.segy_read(q)
    raw[3224:3226] = np.array(5, ">i2").tobytes()
    q.write_bytes(bytes(raw[:-3]))  # truncated last trace
    with pytest.raises(ValueError, match="whole number"):
        segy.segy_read(q)


def test_workload_from_segy_models(tmp_path, oracle_lib):
    # a layered elastic model on a 1.25 m grid (the Marmousi files' spacing)
    nz, nx = 120, 203
    z = np.arange(nz)[:, None] * np.ones((1, nx))
    vp = 1500.0 + 18.0 * z + 40.0 * np.sin(np.arange(nx) / 9.0)[None, :]
    vs = vp / 1.9
    rho = 1800.0 + 2.0 * z
    paths = []
    for name, plane in (("vp", vp), ("vs", vs), ("rho", rho)):
        paths.append(tmp_path / f"MODEL_{name}.segy")
        segy.segy_write(paths[-1], plane, dt_us=1250, fmt=1)
    vp_r, vs_r, rho_r = (segy.read_model(p) for p in paths)
    assert vp_r.shape == (nz, nx) and np.allclose(vp_r, vp, rtol=2.0**-21)
    w = segy.workload_from_models(vp_r, vs_r, rho_r, dx=1.25, nt=60, stride=2,
                                  window=(0, 110, 3, 203), Q=80.0, pml=10, nrec=8, f0=60.0)
    assert (w.nz, w.nx) == (55, 100) and w.nx % 4 == 0 and w.dx == 2.5
    assert media.cfl_number(w) == pytest.approx(0.45, rel=1e-9)
    ref = media.medium_from_velocity("iso", vp_r[0:110:2, 3:203:2][:, :100],
                                     vs_r[0:110:2, 3:203:2][:, :100], rho_r[0:110:2, 3:203:2][:, :100],
                                     Q=np.full((55, 100), 80.0), qfit=media.q_fit(2.0, 30.0, 3))
    for k in ("rho", "c13", "c55", "tau"):
        assert np.allclose(w.medium[k], ref[k], rtol=1e-12, atol=0), k
    tr, st = oracle_lib.run(w, precision="f64")
    assert np.all(np.isfinite(tr)) and np.abs(tr).max() > 0
    with pytest.raises(ValueError, match="vp > vs"):
        segy.workload_from_models(vp_r, vp_r, rho_r, dx=1.25, nt=10)
