"""Host-side set-up: wavelets, the constant-Q fit, media and the seeded
workload recipes.

Reference items restated here (haralddd/ViscoelasticInversion, Julia):
  _ricker(f, t) ................................ src/sciml_solver/Source.jl:3-5
  Ricker(fM, t0), get_value(s, t) .............. src/custom_solver/PointSource.jl:3-14
  K, dK_dω, get_τ, get_Q ....................... src/sciml_solver/Models.jl:65-68
  find_optimal_τns, QModel ..................... src/sciml_solver/Models.jl:70-102
  IsotropicModel / VTIModel / TTIModel fields .. src/sciml_solver/Models.jl:3-43
  Model(ε, δ, γ) (Thomsen) ..................... src/custom_solver/Model.jl:12-16

All of this runs once per model on the host; the time step consumes its
outputs (planes of ρ, C and τ, and the τ_n of the mechanisms).
"""
from __future__ import annotations

import functools
import math
from dataclasses import dataclass, field

import numpy as np

from ._abi import VI_HALF

# ---------------------------------------------------------------- wavelets


def ricker(f: float, t):
    """(1 - 2(π f t)²) exp(-(π f t)²) — Source.jl:3-5."""
    x = np.pi * f * np.asarray(t, dtype=np.float64)
    return (1.0 - 2.0 * x * x) * np.exp(-x * x)


def ricker_table(f: float, t0: float, dt: float, nt: int) -> np.ndarray:
    """Per-step wavelet samples w[n] = ricker(f, n*dt - t0) (float64)."""
    return ricker(f, np.arange(nt) * dt - t0)


# ------------------------------------------------------------ constant Q


def K(omega, taus):
    """K(ω) = Σ ω τ_n / (1 + τ_n² ω²) — Models.jl:65."""
    omega = np.asarray(omega, dtype=np.float64)[..., None]
    taus = np.asarray(taus, dtype=np.float64)
    return np.sum(omega * taus / (1.0 + taus**2 * omega**2), axis=-1)


def dK_domega(omega, taus):
    """dK/dω — Models.jl:66."""
    omega = np.asarray(omega, dtype=np.float64)[..., None]
    taus = np.asarray(taus, dtype=np.float64)
    return np.sum(taus * (1.0 - taus**2 * omega**2) / (1.0 + taus**2 * omega**2) ** 2, axis=-1)


def get_tau(Q0, Kbar, N):
    """τ = N / (K̄ Q0) — Models.jl:67."""
    return N / (Kbar * np.asarray(Q0, dtype=np.float64))


def get_Q(omega, tau, taus):
    """Q(ω) = N / (τ K(ω)) — Models.jl:68."""
    return len(taus) / (tau * K(omega, taus))


def find_optimal_taus(omega1: float, omega2: float, N: int) -> np.ndarray:
    """Relaxation times of N mechanisms for a nearly constant Q over
    [ω1, ω2] (Models.jl:70-87).

    The reference minimises ∫(dK/dω)² with Nelder–Mead from τ_n = 1/ω on a
    linear grid.  That objective also falls by shrinking K everywhere
    (τ_n → 0 or ∞), so here the flatness is measured relative to the mean:
    J = mean_ω (K(ω)/K̄ - 1)², over log τ_n, from the same starting point.
    """
    from scipy.optimize import minimize

    omegas = np.linspace(omega1, omega2, 200)
    x0 = np.log(1.0 / np.linspace(omega1, omega2, N))

    def J(logt):
        k = K(omegas, np.exp(logt))
        return float(np.mean((k / k.mean() - 1.0) ** 2))

    res = minimize(J, x0, method="Nelder-Mead",
                   options={"maxiter": 20000, "xatol": 1e-10, "fatol": 1e-14})
    return np.sort(np.exp(res.x))


@dataclass
class QFit:
    taus: np.ndarray   # τ_n of the mechanisms
    Kbar: float        # mean of K over the band (Models.jl:91-92)
    f1: float
    f2: float

    def tau_for(self, Q):
        return get_tau(Q, self.Kbar, len(self.taus))

    def q_error(self, Q0: float):
        """Mean and max relative Q error over the band (tests/test_Q_model.jl:3-19)."""
        omegas = np.linspace(2 * np.pi * self.f1, 2 * np.pi * self.f2, 100)
        Qs = get_Q(omegas, self.tau_for(Q0), self.taus)
        err = np.abs(Qs - Q0) / Q0
        return float(err.mean()), float(err.max())


@functools.lru_cache(maxsize=64)
def q_fit(f1: float, f2: float, N: int) -> QFit:
    """QModel(f1, f2, Nx, Nz, Q0, N) without the grids (Models.jl:90-102)."""
    w1, w2 = 2 * np.pi * f1, 2 * np.pi * f2
    taus = find_optimal_taus(w1, w2, N)
    Kbar = float(np.mean(K(np.linspace(w1, w2, 100), taus)))
    return QFit(taus=taus, Kbar=Kbar, f1=f1, f2=f2)


# ---------------------------------------------------------------- stiffness


def thomsen_vti(vp, vs, rho, eps, delta):
    """VTI stiffness (C11, C13, C33, C55) from Thomsen parameters
    (custom_solver/Model.jl:12-16 carries ε, δ, γ; γ only enters SH motion
    and has no effect on 2D P-SV)."""
    C33 = rho * vp**2
    C55 = rho * vs**2
    C11 = C33 * (1.0 + 2.0 * eps)
    C13 = np.sqrt(np.maximum((C33 - C55) * (C33 * (1.0 + 2.0 * delta) - C55), 0.0)) - C55
    return C11, C13, C33, C55


def medium_from_velocity(kind, vp, vs, rho, eps=None, delta=None, Q=None, qfit=None) -> dict:
    """Medium planes of vi_medium from (vp, vs, rho[, eps, delta], Q) fields:
    ISO Lame (lambda in c13, mu in c55), VTI Thomsen (Models.jl:27-52), and
    tau = N / (Kbar Q) of the Q fit (Models.jl:67) when qfit is given."""
    vp, vs, rho = (np.asarray(a, dtype=np.float64) for a in (vp, vs, rho))
    med = {"rho": rho.copy()}
    if kind == "iso":
        med["c13"] = rho * (vp**2 - 2 * vs**2)
        med["c55"] = rho * vs**2
    elif kind == "vti":
        z = np.zeros_like(vp)
        C11, C13, C33, C55 = thomsen_vti(vp, vs, rho, z if eps is None else eps,
                                         z if delta is None else delta)
        med.update(c11=C11, c13=C13, c33=C33, c55=C55)
    else:
        raise ValueError("medium_from_velocity: iso or vti")
    if qfit is not None and len(qfit.taus):
        med["tau"] = qfit.tau_for(np.broadcast_to(np.asarray(Q, dtype=np.float64), vp.shape)).copy()
    return med


def bond_rotate(C11, C13, C33, C55, theta):
    """Tilts a VTI medium by θ (radians, symmetry axis rotated from z
    towards x) and returns the 2D P-SV Voigt stiffness
    (C11, C13, C15, C33, C35, C55) of the TTI medium."""
    c = np.cos(theta)
    s = np.sin(theta)
    c2, s2, cs = c * c, s * s, c * s
    # C'_ijkl = R_ip R_jq R_kr R_ls C_pqrs in the x-z plane
    A = C13 + 2.0 * C55
    n11 = c2 * c2 * C11 + 2 * c2 * s2 * A + s2 * s2 * C33
    n33 = s2 * s2 * C11 + 2 * c2 * s2 * A + c2 * c2 * C33
    n13 = c2 * s2 * (C11 + C33 - 4.0 * C55) + (c2 * c2 + s2 * s2) * C13
    n55 = c2 * s2 * (C11 + C33 - 2.0 * C13) + (c2 - s2) ** 2 * C55
    n15 = -cs * (c2 * C11 - s2 * C33 - (c2 - s2) * A)
    n35 = -cs * (s2 * C11 - c2 * C33 + (c2 - s2) * A)
    return n11, n13, n15, n33, n35, n55


def bond_rotate_tensor(C11, C13, C33, C55, theta):
    """The same rotation by explicit 4th-order tensor algebra (used to
    check bond_rotate)."""
    Ct = np.zeros(np.shape(C11) + (2, 2, 2, 2))
    vo = {(0, 0): C11, (1, 1): C33}
    Ct[..., 0, 0, 0, 0] = C11
    Ct[..., 1, 1, 1, 1] = C33
    for (i, j, k, l) in [(0, 0, 1, 1), (1, 1, 0, 0)]:
        Ct[..., i, j, k, l] = C13
    for (i, j, k, l) in [(0, 1, 0, 1), (0, 1, 1, 0), (1, 0, 0, 1), (1, 0, 1, 0)]:
        Ct[..., i, j, k, l] = C55
    del vo
    c, s = np.cos(theta), np.sin(theta)
    R = np.zeros(np.shape(theta) + (2, 2))
    R[..., 0, 0] = c
    R[..., 0, 1] = s
    R[..., 1, 0] = -s
    R[..., 1, 1] = c
    Cr = np.einsum("...ip,...jq,...kr,...ls,...pqrs->...ijkl", R, R, R, R, Ct)
    return (Cr[..., 0, 0, 0, 0], Cr[..., 0, 0, 1, 1], Cr[..., 0, 0, 0, 1],
            Cr[..., 1, 1, 1, 1], Cr[..., 1, 1, 0, 1], Cr[..., 0, 1, 0, 1])


# ---------------------------------------------------------------- workloads


@dataclass
class Workload:
    """A complete single-shot problem: grid, medium planes (float64,
    shape [nz, nx], x fastest), mechanisms, boundary set-up, sources and
    receivers."""

    name: str
    nx: int
    nz: int
    dx: float
    dz: float
    dt: float
    nt: int
    kind: str                    # "iso" | "vti" | "tti"
    medium: dict                 # name -> float64 array [nz, nx]
    taus: np.ndarray             # τ_n (empty for elastic)
    free_surface: int  # 0/False none, 1/True stress imaging, 2 H-AFDA
    pml: int
    pml_vmax: float
    pml_alpha_max: float
    sources: list                # [(i, j, kind, amp)]
    wavelets: np.ndarray         # [nsrc, nt] float64
    receivers: list              # [(i, j)]
    vmax: float                  # max phase velocity (CFL)
    meta: dict = field(default_factory=dict)

    @property
    def nsls(self) -> int:
        return len(self.taus)

    def planes(self) -> list[str]:
        base = {"iso": ["rho", "c13", "c55"], "vti": ["rho", "c11", "c13", "c33", "c55"],
                "tti": ["rho", "c11", "c13", "c15", "c33", "c35", "c55"]}[self.kind]
        return base + (["tau"] if self.nsls else [])

    def state_planes(self) -> int:
        return 5 + 3 * self.nsls

    def medium_planes(self) -> int:
        return len(self.planes())

    def bytes_per_point(self, esize: int) -> int:
        """Algorithmic HBM bytes per grid point per step: the state is read
        and written once, the medium read once."""
        return esize * (2 * self.state_planes() + self.medium_planes())


def _gaussian_field(rng, shape, corr_cells: float, sigma: float) -> np.ndarray:
    from scipy.ndimage import gaussian_filter

    f = gaussian_filter(rng.standard_normal(shape), corr_cells, mode="wrap")
    f *= sigma / max(f.std(), 1e-30)
    return f


def _receiver_line(nx: int, pml: int, j: int, n: int) -> list:
    lo, hi = max(VI_HALF, pml), nx - max(VI_HALF, pml) - 1
    xs = np.unique(np.round(np.linspace(lo, hi, n)).astype(int))
    return [(int(i), int(j)) for i in xs]


def homogeneous_iso(nx=256, nz=256, dx=5.0, dt=0.5e-3, nt=1000, vp=3000.0, vs=1732.0,
                    rho=2200.0, Q=50.0, nsls=3, band=(5.0, 50.0), pml=20, f0=15.0,
                    nrec=100, free_surface=True, src=None) -> Workload:
    """2D isotropic viscoelastic medium on a homogeneous grid: the plain
    forward model the reference runs on the CPU (FP64): 256², dx = dz = 5 m,
    dt = 0.5 ms, 1000 steps, Q = 50 by 3 SLS over 5–50 Hz, 20-cell CPML,
    free surface, 15 Hz explosive Ricker at the centre, 100 receivers 10 m
    below the surface."""
    shape = (nz, nx)
    lam = rho * (vp**2 - 2 * vs**2)
    mu = rho * vs**2
    med = {"rho": np.full(shape, rho), "c13": np.full(shape, lam), "c55": np.full(shape, mu)}
    taus = np.zeros(0)
    if nsls:
        qf = q_fit(*band, nsls)
        taus = qf.taus
        med["tau"] = np.full(shape, qf.tau_for(Q))
    t_unrelaxed = 1.0 + (med["tau"].max() if nsls else 0.0)
    vmax = vp * math.sqrt(t_unrelaxed)
    js = VI_HALF  # surface row, or the first row of the update region
    si, sj = src if src is not None else (nx // 2, nz // 2)
    return Workload(
        name=f"iso-homogeneous-{nx}x{nz}", nx=nx, nz=nz, dx=dx, dz=dx, dt=dt, nt=nt, kind="iso",
        medium=med, taus=taus, free_surface=free_surface, pml=pml, pml_vmax=vp,
        pml_alpha_max=math.pi * f0, sources=[(si, sj, 0, 1.0)],
        wavelets=ricker_table(f0, 1.2 / f0, dt, nt)[None, :],
        receivers=_receiver_line(nx, pml, js + int(round(10.0 / dx)), nrec), vmax=vmax,
        meta={"f0": f0, "Q": Q, "band": band})


def layered(nx=2048, nz=1024, dx=5.0, dt=0.4e-3, nt=4000, kind="vti", seed=0, nlayers=8,
            nsls=3, band=(2.0, 30.0), pml=40, f0=12.0, nrec=512, free_surface=True,
            pert=0.03, corr=50.0, tilt_max_deg=30.0) -> Workload:
    """Seeded layered medium: nlayers layers, vp uniform in [1800, 4500]
    increasing with depth, vs = vp/1.8, ρ = 310 vp^0.25 (Gardner), each
    overlaid with a 3 % Gaussian random field of 50 m correlation length
    (multiplicative); per layer ε ∈ U[0, 0.25], δ ∈ U[-0.05, 0.15],
    γ ∈ U[0, 0.2], Q ∈ U[30, 200].  kind = "vti" (the 2048 x 1024 FP32
    single-shot workload) or "tti" (adds a smooth tilt field θ in ±30°) or
    "iso" (ε = δ = 0).  Source: explosive Ricker 20 m below the surface;
    receivers 10 m below it."""
    rng = np.random.default_rng(seed)
    shape = (nz, nx)
    z = np.arange(nz) * dx
    depth = nz * dx
    interfaces = np.sort(rng.uniform(0.05 * depth, 0.95 * depth, nlayers - 1))
    layer = np.searchsorted(interfaces, z)                   # [nz]
    vp_l = np.sort(rng.uniform(1800.0, 4500.0, nlayers))
    eps_l = rng.uniform(0.0, 0.25, nlayers)
    del_l = rng.uniform(-0.05, 0.15, nlayers)
    gam_l = rng.uniform(0.0, 0.2, nlayers)
    q_l = rng.uniform(30.0, 200.0, nlayers)
    corr_cells = corr / dx
    fvp = _gaussian_field(rng, shape, corr_cells, pert)
    frho = _gaussian_field(rng, shape, corr_cells, pert)
    vp = vp_l[layer][:, None] * (1.0 + fvp)
    vs = vp / 1.8
    rho = 310.0 * vp**0.25 * (1.0 + frho)
    if kind == "iso":
        eps = np.zeros(shape)
        dlt = np.zeros(shape)
    else:
        eps = np.broadcast_to(eps_l[layer][:, None], shape).copy()
        dlt = np.broadcast_to(del_l[layer][:, None], shape).copy()
    gamma = np.broadcast_to(gam_l[layer][:, None], shape).copy()
    C11, C13, C33, C55 = thomsen_vti(vp, vs, rho, eps, dlt)
    med = {"rho": rho}
    theta = None
    if kind == "tti":
        th = _gaussian_field(rng, shape, 200.0 / dx, 1.0)
        th = th / max(np.abs(th).max(), 1e-30) * math.radians(tilt_max_deg)
        theta = th
        n11, n13, n15, n33, n35, n55 = bond_rotate(C11, C13, C33, C55, th)
        med.update(c11=n11, c13=n13, c15=n15, c33=n33, c35=n35, c55=n55)
    elif kind == "vti":
        med.update(c11=C11, c13=C13, c33=C33, c55=C55)
    else:
        med.update(c13=C13, c55=C55)
    taus = np.zeros(0)
    tmax = 0.0
    if nsls:
        qf = q_fit(*band, nsls)
        taus = qf.taus
        Q = np.broadcast_to(q_l[layer][:, None], shape)
        med["tau"] = qf.tau_for(Q)
        tmax = float(med["tau"].max())
    # fastest phase velocity: horizontal P in VTI, sqrt(max(C11, C33)/rho) bound for TTI
    cmax = np.maximum(med.get("c11", C11), med.get("c33", C33))
    vmax = float(np.sqrt(cmax / rho).max() * math.sqrt(1.0 + tmax))
    js = VI_HALF  # surface row, or the first row of the update region
    src_j = js + int(round(20.0 / dx))
    return Workload(
        name=f"{kind}-layered-{nx}x{nz}-seed{seed}", nx=nx, nz=nz, dx=dx, dz=dx, dt=dt, nt=nt,
        kind=kind, medium=med, taus=taus, free_surface=free_surface, pml=pml,
        pml_vmax=float(np.sqrt(cmax / rho).max()), pml_alpha_max=math.pi * f0,
        sources=[(nx // 2, src_j, 0, 1.0)], wavelets=ricker_table(f0, 1.2 / f0, dt, nt)[None, :],
        receivers=_receiver_line(nx, pml, js + int(round(10.0 / dx)), nrec), vmax=vmax,
        meta={"f0": f0, "band": band, "eps": eps_l, "delta": del_l, "gamma": gam_l, "Q": q_l,
              "theta": theta, "gamma_field": gamma, "seed": seed,
              "fields": {"vp": vp, "vs": vs, "rho": rho, "eps": eps, "delta": dlt,
                         "Q": np.broadcast_to(q_l[layer][:, None], shape).copy()}})


GATHER_GRIDS = ((512, 512), (1024, 512), (1536, 768), (2048, 1024))


def shot_gather(nshots: int = 64, seed: int = 0, kind: str = "tti", nt_range=(1500, 4000),
                grids=GATHER_GRIDS, **kw) -> list:
    """The batched workload: nshots shots, grid sizes drawn from
    {512², 1024x512, 1536x768, 2048x1024}, nt uniform in [1500, 4000], each
    a seeded layered medium (the 2048 x 1024 recipe) with a smooth tilt
    field θ in ±30° for TTI.  Shot s uses medium seed 1000*seed + s."""
    rng = np.random.default_rng(seed)
    out = []
    for s in range(nshots):
        nx, nz = grids[int(rng.integers(len(grids)))]
        nt = int(rng.integers(nt_range[0], nt_range[1] + 1))
        w = layered(nx=nx, nz=nz, nt=nt, kind=kind, seed=1000 * seed + s, **kw)
        w.name = f"{kind}-gather{seed}-shot{s}-{nx}x{nz}-nt{nt}"
        out.append(w)
    return out


def cfl_number(w: Workload) -> float:
    """vmax dt sqrt(1/dx² + 1/dz²) Σ|D_k|; must be ≤ 1."""
    s = 1225 / 1024 + 245 / 3072 + 49 / 5120 + 5 / 7168
    return w.vmax * w.dt * math.sqrt(1 / w.dx**2 + 1 / w.dz**2) * s
