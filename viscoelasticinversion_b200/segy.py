"""SEG-Y model ingest: the reference reads its models with SegyIO.jl's
`segy_read` (src/common/read_model.jl:4-6, the Marmousi elastic P-wave
model; SegyIO is a third-party Julia package, absent here).  This module
reads and writes the SEG-Y rev 1 layout itself, from the published
standard:

* a 3200-byte textual header (EBCDIC or ASCII), a 400-byte binary header
  (big-endian; sample interval in µs at byte 3217, samples per trace at
  3221, sample format code at 3225, revision at 3501, extended textual
  headers at 3505), the extended textual headers (3200 bytes each);
* then per trace a 240-byte header (big-endian) and its samples.  Sample
  formats: 1 = 4-byte IBM hexadecimal float, 2 = int32, 3 = int16,
  5 = IEEE float32, 8 = int8.

`segy_read` returns a SeisBlock like SegyIO's: `data` [ns, ntraces] float32
(one column per trace; for a model file ns is depth and traces run along
x, i.e. the [nz, nx] planes this package uses), `fileheader` and
`traceheaders`.  `workload_from_models` turns vp / vs / rho planes read
this way into a media.Workload.
"""
from __future__ import annotations

import math
from dataclasses import dataclass, field
from pathlib import Path

import numpy as np

TEXT_BYTES = 3200
BIN_BYTES = 400
TRACE_HEADER_BYTES = 240

# binary file header fields: name -> (byte offset within the 400-byte block, numpy type)
_BFH = {
    "Job": (0, ">i4"), "Line": (4, ">i4"), "Reel": (8, ">i4"),
    "DataTracePerEnsemble": (12, ">i2"), "AuxiliaryTracePerEnsemble": (14, ">i2"),
    "dt": (16, ">i2"), "dtOrig": (18, ">i2"), "ns": (20, ">i2"), "nsOrig": (22, ">i2"),
    "DataSampleFormat": (24, ">i2"), "EnsembleFold": (26, ">i2"), "TraceSorting": (28, ">i2"),
    "MeasurementSystem": (54, ">i2"),
    "SegyFormatRevisionNumber": (300, ">i2"), "FixedLengthTraceFlag": (302, ">i2"),
    "NumberOfExtTextualHeaders": (304, ">i2"),
}

# trace header fields kept: name -> (byte offset within the 240-byte header, numpy type)
_TH = {
    "TraceNumWithinLine": (0, ">i4"), "TraceNumWithinFile": (4, ">i4"),
    "FieldRecord": (8, ">i4"), "TraceNumber": (12, ">i4"), "EnergySourcePoint": (16, ">i4"),
    "CDP": (20, ">i4"), "CDPTrace": (24, ">i4"), "TraceIDCode": (28, ">i2"),
    "Offset": (36, ">i4"), "RecGroupElevation": (40, ">i4"), "SourceSurfaceElevation": (44, ">i4"),
    "ElevationScalar": (68, ">i2"), "RecSourceScalar": (70, ">i2"),
    "SourceX": (72, ">i4"), "SourceY": (76, ">i4"), "GroupX": (80, ">i4"), "GroupY": (84, ">i4"),
    "CoordUnits": (88, ">i2"), "ns": (114, ">i2"), "dt": (116, ">i2"),
    "CDPX": (180, ">i4"), "CDPY": (184, ">i4"), "Inline3D": (188, ">i4"), "Crossline3D": (192, ">i4"),
}
_TH_DTYPE = np.dtype({"names": list(_TH), "formats": [t for _, t in _TH.values()],
                      "offsets": [o for o, _ in _TH.values()], "itemsize": TRACE_HEADER_BYTES})

_SAMPLE = {1: (4, ">u4"), 2: (4, ">i4"), 3: (2, ">i2"), 5: (4, ">f4"), 8: (1, "i1")}

# Σ|D_k| of the 8th-order staggered weights (1225/1024, -245/3072, 49/5120, -5/7168)
_SUM_D = 1225 / 1024 + 245 / 3072 + 49 / 5120 + 5 / 7168


# ------------------------------------------------------------ IBM floats
def ibm_to_ieee(words) -> np.ndarray:
    """4-byte IBM hexadecimal floats (as uint32 words) to float32:
    (-1)^s · 0.f · 16^(e - 64), 7-bit exponent e, 24-bit fraction f."""
    u = np.asarray(words, dtype=np.uint32)
    sign = np.where(u >> np.uint32(31), -1.0, 1.0)
    expo = ((u >> np.uint32(24)) & np.uint32(0x7F)).astype(np.int64)
    frac = (u & np.uint32(0xFFFFFF)).astype(np.float64)
    return (sign * np.ldexp(frac, 4 * (expo - 64) - 24)).astype(np.float32)


def ieee_to_ibm(values) -> np.ndarray:
    """float values to 4-byte IBM hexadecimal floats (uint32 words), the
    fraction rounded to nearest; magnitudes beyond 16^63 saturate, those
    below 16^-65 flush to zero."""
    x = np.asarray(values, dtype=np.float64)
    out = np.zeros(x.shape, dtype=np.uint32)
    nz = (x != 0) & np.isfinite(x)
    a = np.abs(x[nz])
    m, e2 = np.frexp(a)                        # a = m 2^e2, m in [0.5, 1)
    E = -((-e2) // 4)                          # ceil(e2 / 4): a = f 16^E, f in [1/16, 1)
    frac = np.rint(np.ldexp(m, e2 - 4 * E + 24)).astype(np.int64)
    carry = frac >= (1 << 24)                  # rounding reached 1.0: renormalise
    frac = np.where(carry, frac >> 4, frac)
    E = E + carry
    expo = E + 64
    small, big = expo < 0, expo > 127
    frac = np.where(small, 0, np.where(big, 0xFFFFFF, frac))
    expo = np.clip(expo, 0, 127)
    word = (expo.astype(np.uint64) << 24) | frac.astype(np.uint64)
    word = np.where(small, 0, word)
    word = word | np.where(x[nz] < 0, np.uint64(1) << 31, np.uint64(0))
    out[nz] = word.astype(np.uint32)
    return out


# ------------------------------------------------------------ read / write
@dataclass
class SeisBlock:
    """SegyIO's SeisBlock: file header, trace headers, data [ns, ntraces]."""
    fileheader: dict
    traceheaders: np.ndarray
    data: np.ndarray
    text_header: str = ""
    extended_text: list = field(default_factory=list)


def _decode_text(raw: bytes) -> str:
    # EBCDIC (cp037) unless the block already reads as printable ASCII
    if raw[:1] in (b"C", b" ") and all(32 <= b < 127 or b in (10, 13, 0) for b in raw[:80]):
        return raw.decode("ascii", errors="replace")
    return raw.decode("cp037", errors="replace")


def segy_read(path) -> SeisBlock:
    """Reads a SEG-Y rev 0/1 file with fixed-length traces (the
    binary header's sample count for every trace), as SegyIO.segy_read."""
    raw = Path(path).read_bytes()
    if len(raw) < TEXT_BYTES + BIN_BYTES:
        raise ValueError(f"{path}: shorter than the SEG-Y file headers")
    text = _decode_text(raw[:TEXT_BYTES])
    b = raw[TEXT_BYTES:TEXT_BYTES + BIN_BYTES]
    bfh = {k: int(np.frombuffer(b, dtype=t, count=1, offset=o)[0]) for k, (o, t) in _BFH.items()}
    fmt, ns = bfh["DataSampleFormat"], bfh["ns"]
    if fmt not in _SAMPLE:
        raise ValueError(f"{path}: sample format code {fmt} is not supported")
    if ns <= 0:
        raise ValueError(f"{path}: {ns} samples per trace")
    next_ = max(bfh["NumberOfExtTextualHeaders"], 0) if bfh["SegyFormatRevisionNumber"] else 0
    pos = TEXT_BYTES + BIN_BYTES
    ext = [_decode_text(raw[pos + k * TEXT_BYTES:pos + (k + 1) * TEXT_BYTES]) for k in range(next_)]
    pos += next_ * TEXT_BYTES
    size, stype = _SAMPLE[fmt]
    rec = TRACE_HEADER_BYTES + ns * size
    body = len(raw) - pos
    if body % rec:
        raise ValueError(f"{path}: {body} trace bytes are not a whole number of {rec}-byte traces")
    ntr = body // rec
    tr = np.frombuffer(raw, dtype=np.uint8, count=ntr * rec, offset=pos).reshape(ntr, rec)
    th = np.frombuffer(np.ascontiguousarray(tr[:, :TRACE_HEADER_BYTES]).tobytes(), dtype=_TH_DTYPE)
    samples = np.frombuffer(np.ascontiguousarray(tr[:, TRACE_HEADER_BYTES:]).tobytes(), dtype=stype)
    samples = samples.reshape(ntr, ns)
    data = ibm_to_ieee(samples) if fmt == 1 else samples.astype(np.float32)
    return SeisBlock(fileheader=bfh, traceheaders=th.copy(), data=np.ascontiguousarray(data.T),
                     text_header=text, extended_text=ext)


def segy_write(path, data, dt_us: int, fmt: int = 1, text: str = "", traceheaders=None):
    """Writes data [ns, ntraces] as a SEG-Y rev 1 file (EBCDIC text header,
    fixed-length traces, sample format 1 IBM float or 5 IEEE float32).
    traceheaders: optional dict of _TH field name -> per-trace values."""
    data = np.asarray(data, dtype=np.float64)
    if data.ndim != 2:
        raise ValueError("data must be [ns, ntraces]")
    if fmt not in (1, 5):
        raise ValueError("fmt must be 1 (IBM) or 5 (IEEE)")
    ns, ntr = data.shape
    if not 0 < ns < 32768:
        raise ValueError("ns must fit the 16-bit header field")
    lines = (text.splitlines() or ["C 1 SEG-Y written by viscoelasticinversion_b200"])[:40]
    th_text = "".join(l[:80].ljust(80) for l in lines).ljust(TEXT_BYTES)
    b = np.zeros(BIN_BYTES, dtype=np.uint8)
    for k, v in (("dt", dt_us), ("dtOrig", dt_us), ("ns", ns), ("nsOrig", ns),
                 ("DataSampleFormat", fmt), ("DataTracePerEnsemble", ntr),
                 ("SegyFormatRevisionNumber", 0x0100), ("FixedLengthTraceFlag", 1),
                 ("MeasurementSystem", 1)):
        o, t = _BFH[k]
        b[o:o + np.dtype(t).itemsize] = np.frombuffer(np.array(v, dtype=t).tobytes(), np.uint8)
    th = np.zeros(ntr, dtype=_TH_DTYPE)
    th["TraceNumWithinLine"] = th["TraceNumWithinFile"] = th["TraceNumber"] = np.arange(1, ntr + 1)
    th["ns"], th["dt"] = ns, dt_us
    for k, v in (traceheaders or {}).items():
        th[k] = v
    samples = ieee_to_ibm(data.T) if fmt == 1 else data.T.astype(">f4")
    samples = samples.astype(">u4") if fmt == 1 else samples
    with open(path, "wb") as f:
        f.write(th_text.encode("cp037"))
        f.write(b.tobytes())
        for i in range(ntr):
            f.write(th[i:i + 1].tobytes())
            f.write(samples[i].tobytes())


# ------------------------------------------------------------ models to workloads
def read_model(path, dtype=np.float64) -> np.ndarray:
    """One model plane [nz, nx] from a SEG-Y model file (depth samples down
    each trace, one trace per x position), as read_model.jl:4-6 reads the
    Marmousi P-wave velocity."""
    return np.asarray(segy_read(path).data, dtype=dtype)


def workload_from_models(vp, vs, rho, dx: float, nt: int, dt: float | None = None,
                         stride: int = 1, window=None, Q=None, nsls: int = 3,
                         band=(2.0, 30.0), pml: int = 20, f0: float = 10.0, nrec: int = 128,
                         free_surface: bool = True, src=None, cfl: float = 0.45):
    """An ISO media.Workload from vp, vs, rho planes [nz, nx] (e.g. the
    three Marmousi elastic SEG-Y models): optional window (z0, z1, x0, x1)
    and decimation by `stride` (dx is the model's spacing before it), nx cut
    to a multiple of 4, dt from the CFL number when not given, Q (scalar or
    plane) by an nsls-mechanism fit over `band`, an explosive Ricker of f0
    Hz at src (default: 20 m below the surface at mid-x) and nrec receivers
    10 m below the surface."""
    from . import media

    shape = np.shape(vp)
    Qplane = np.full(shape, 100.0 if Q is None else float(Q)) if Q is None or np.isscalar(Q) else Q
    planes = [np.asarray(a, dtype=np.float64) for a in (vp, vs, rho, Qplane)]
    if any(a.shape != shape for a in planes):
        raise ValueError("vp, vs, rho (and a Q plane) must have one shape")
    if window is not None:
        z0, z1, x0, x1 = window
        planes = [a[z0:z1, x0:x1] for a in planes]
    planes = [a[::stride, ::stride] for a in planes]
    nz, nx = planes[0].shape
    nx -= nx % 4
    vp, vs, rho, Qp = [np.ascontiguousarray(a[:, :nx]) for a in planes]
    if nx < 8 or nz < 8:
        raise ValueError("the model window is too small")
    if np.any(vp <= 0) or np.any(rho <= 0) or np.any(vs < 0) or np.any(vs >= vp):
        raise ValueError("models need vp > vs >= 0 and rho > 0")
    h = dx * stride
    qf = media.q_fit(*band, nsls) if nsls else None
    med = media.medium_from_velocity("iso", vp, vs, rho, Q=Qp, qfit=qf)
    tmax = float(med["tau"].max()) if nsls else 0.0
    vmax = float(vp.max() * math.sqrt(1.0 + tmax))
    if dt is None:
        # CFL of the 8th-order staggered step: vmax dt sqrt(2) / h · Σ|D_k| = cfl
        dt = cfl * h / (vmax * math.sqrt(2.0) * _SUM_D)
    js = media.VI_HALF
    si, sj = src if src is not None else (nx // 2, js + max(1, int(round(20.0 / h))))
    w = media.Workload(
        name=f"models-{nx}x{nz}", nx=nx, nz=nz, dx=h, dz=h, dt=dt, nt=nt, kind="iso",
        medium=med, taus=qf.taus if nsls else np.zeros(0), free_surface=free_surface, pml=pml,
        pml_vmax=float(vp.max()), pml_alpha_max=math.pi * f0, sources=[(si, sj, 0, 1.0)],
        wavelets=media.ricker_table(f0, 1.2 / f0, dt, nt)[None, :],
        receivers=media._receiver_line(nx, pml, js + max(1, int(round(10.0 / h))), nrec),
        vmax=vmax, meta={"f0": f0, "band": band, "Q": Qp})
    return w
