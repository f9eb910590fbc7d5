"""The ticket order of the time-blocked step (kernel variant 9), restated on
the host: the decode of csrc/wave.cu (prefix table wave_before, binary
search for tau, q = qlo + offset) gives every unit exactly once, and every
unit a CTA can wait on has an earlier ticket — the property that lets the
kernel run without co-resident CTAs.  CPU only."""
import pytest


def _before(tau, twok, d, nb):
    return sum(min(max(tau - d * q, 0), nb) for q in range(twok))


def _decode(w, t):
    r, u = divmod(t, w["slots"])
    full = w["nfull"] * w["per_full"]
    sweep = r // w["per_full"] if r < full else w["nfull"]
    rr = r - sweep * w["per_full"]
    ks = w["k"] if sweep < w["nfull"] else w["nsteps"] - w["nfull"] * w["k"]
    twok = 2 * ks
    if ks <= 0 or rr >= twok * w["nb"]:
        return None
    lo, hi = 0, w["nb"] + w["d"] * (twok - 1)
    while lo < hi:
        mid = (lo + hi + 1) // 2
        if _before(mid, twok, w["d"], w["nb"]) <= rr:
            lo = mid
        else:
            hi = mid - 1
    tau = lo
    qlo = (tau - w["nb"] + 1 + w["d"] - 1) // w["d"] if tau - w["nb"] + 1 > 0 else 0
    q = qlo + (rr - _before(tau, twok, w["d"], w["nb"]))
    b = tau - w["d"] * q
    assert 0 <= b < w["nb"] and 0 <= q < twok
    s, p = w["it0"] + sweep * w["k"] + q // 2, q & 1
    return (s, p, b, u) if u < _units(w, p, b) else None


def _units(w, p, b):
    return w["ntx_v"] if p == 0 else w["ntx_s"] * min(2, w["ntz_s"] - 2 * b)


@pytest.mark.parametrize("nb,ntx_v,ntx_s,ntz_s,k,d,nsteps", [
    (5, 3, 2, 9, 2, 2, 7),        # partial last band, full and partial sweeps
    (16, 4, 2, 32, 4, 4, 10),
    (7, 5, 3, 13, 3, 2, 5),       # fewer stress tiles than slots
    (1, 2, 1, 1, 4, 4, 3),        # one band, one stress row
    (3, 2, 1, 6, 4, 3, 1),        # one step
    (4, 3, 2, 8, 16, 5, 40),
    (40, 8, 4, 79, 8, 8, 17),
])
def test_every_unit_once_and_every_dependency_earlier(nb, ntx_v, ntx_s, ntz_s, k, d, nsteps):
    it0 = 3
    k = min(k, nsteps)
    w = dict(nb=nb, ntx_v=ntx_v, ntx_s=ntx_s, ntz_s=ntz_s, slots=max(ntx_v, 2 * ntx_s), k=k, d=d,
             it0=it0, nsteps=nsteps, nfull=nsteps // k, per_full=2 * k * nb)
    total = (w["nfull"] * w["per_full"] + 2 * (nsteps - w["nfull"] * k) * nb) * w["slots"]
    seen = {}
    for t in range(total):
        x = _decode(w, t)
        if x is not None:
            assert x not in seen
            seen[x] = t
    first, last = {}, {}
    for (s, p, b, u), t in seen.items():
        first[(s, p, b)] = min(first.get((s, p, b), t), t)
        last[(s, p, b)] = max(last.get((s, p, b), t), t)
    for s in range(it0, it0 + nsteps):
        for b in range(nb):
            for p in (0, 1):
                assert sum(1 for u in range(_units(w, p, b)) if (s, p, b, u) in seen) == _units(w, p, b)
    # velocity (s, b) waits on stress (s - 1) of bands b-1..b+1; stress (s, b)
    # on velocity (s) of the same bands: all their units come earlier
    for (s, p, b), t0 in first.items():
        so = s - 1 if p == 0 else s
        if so < it0:
            continue
        for bb in range(max(b - 1, 0), min(b + 1, nb - 1) + 1):
            assert last[(so, 1 - p, bb)] < t0
