"""Full-waveform inversion on the GPU gradient: the Energy Natural Gradient
optimizer of sciml_solver/EnergyNaturalGradient.jl, with its names, over
loss and gradient functions that run the B200 step.

The reference optimizer works on a parameter vector θ with callables
loss_fn(θ), grad_fn(θ) and sensitivity_fn(θ) (EnergyNaturalGradient.jl:
239-276) and is never wired to the wave solver.  Here:

* the optimizer (`EnergyNaturalGradientOptimizer`, `OptimizationState`,
  `step`, `optimize`, `line_search_log`, the Gram matrices and the natural
  gradient solve) follows the reference step by step, on the host (numpy);
* its Gram matrices are p x p, so they exist only for small p.  With
  sensitivity_fn = None the metric is the identity — the natural gradient
  is grad / (1 + regularization) — the one form that scales to gridded
  media (p = planes x nx x nz);
* the sensitivity helpers (`compute_sensitivities_forwardmode`,
  `make_jvp_function`) take central differences of a forward solve where
  the reference takes ForwardDiff derivatives;
* `FWIProblem` supplies loss_fn and grad_fn for seismic shots: the summed
  misfit J = 1/2 sum (d - obs)^2 and dJ/dθ by vi_gradient (the discrete
  adjoint in libvisco_b200.so), and `batch_loss` evaluates every trial
  model of a line search, for every shot, as one vi_batch run.
"""
from __future__ import annotations

import dataclasses
import math
from dataclasses import dataclass, field

import numpy as np
import torch

from . import media as _media
from .batch import ShotBatch
from .gradient import GRADIENT_PLANES, misfit_gradient, shard
from .solver import StepPlan


# ---------------------------------------------------------------- inner products
def energy_inner_product(u1, u2, energy_ip=None) -> float:
    """L2 inner product (energy_ip None) or density-weighted L2 (energy_ip an
    array ρ of u's shape) — EnergyNaturalGradient.jl:37-47."""
    u1 = np.asarray(u1, dtype=np.float64)
    u2 = np.asarray(u2, dtype=np.float64)
    if energy_ip is None:
        return float(np.dot(u1.ravel(), u2.ravel()))
    return float(np.sum(np.asarray(energy_ip, dtype=np.float64) * u1 * u2))


def compute_gram_exact(sensitivities, energy_ip=None) -> np.ndarray:
    """G[i, j] = <∂θi u, ∂θj u>, symmetric — EnergyNaturalGradient.jl:63-78."""
    p = len(sensitivities)
    G = np.zeros((p, p))
    for j in range(p):
        for i in range(j, p):
            G[i, j] = G[j, i] = energy_inner_product(sensitivities[i], sensitivities[j], energy_ip)
    return G


def compute_gram_stochastic(jvp_fn, p: int, n_probes: int, energy_ip=None, rng=None) -> np.ndarray:
    """Rademacher-probe estimate: mean over probes z of z zᵀ <Jz, Jz> —
    EnergyNaturalGradient.jl:92-112."""
    rng = np.random.default_rng() if rng is None else rng
    G = np.zeros((p, p))
    for _ in range(n_probes):
        z = rng.choice(np.array([-1.0, 1.0]), size=p)
        Jz = jvp_fn(z)
        G += np.outer(z, z) * energy_inner_product(Jz, Jz, energy_ip)
    return G / n_probes


def compute_natural_gradient(G, grad, regularization: float = 1e-8) -> np.ndarray:
    """Solves (G + regularization I) ψ = grad — EnergyNaturalGradient.jl:128-137."""
    G = np.asarray(G, dtype=np.float64)
    return np.linalg.solve(G + regularization * np.eye(G.shape[0]), np.asarray(grad, dtype=np.float64))


# ---------------------------------------------------------------- line search
def line_search_log(loss_fn, theta, direction, n_points: int = 10, bounds=(1e-6, 1.0),
                    batch_loss_fn=None):
    """Best η on a log10-spaced grid of n_points over bounds, trial θ - η d;
    the first of equal losses wins — EnergyNaturalGradient.jl:155-177.
    batch_loss_fn, if given, takes the list of trial θ and returns their
    losses in one call (the GPU evaluates them together)."""
    lo, hi = bounds
    etas = 10.0 ** np.linspace(math.log10(lo), math.log10(hi), n_points)
    theta = np.asarray(theta, dtype=np.float64)
    direction = np.asarray(direction, dtype=np.float64)
    trials = [theta - eta * direction for eta in etas]
    losses = (list(batch_loss_fn(trials)) if batch_loss_fn is not None
              else [loss_fn(t) for t in trials])
    best_eta, best_loss = float(etas[0]), math.inf
    for eta, loss in zip(etas, losses):
        if loss < best_loss:
            best_loss, best_eta = float(loss), float(eta)
    return best_eta, best_loss


# ---------------------------------------------------------------- optimizer
@dataclass
class EnergyNaturalGradientOptimizer:
    """EnergyNaturalGradient.jl:195-202 (same fields and defaults)."""
    n_probes: int = 50
    regularization: float = 1e-8
    line_search_points: int = 10
    line_search_bounds: tuple = (1e-6, 1.0)
    energy_ip: object = None
    stochastic_threshold: int = 1000


@dataclass
class OptimizationState:
    """θ, iteration count and histories — EnergyNaturalGradient.jl:209-223."""
    theta: np.ndarray
    iteration: int = 0
    loss_history: list = field(default_factory=list)
    eta_history: list = field(default_factory=list)

    def __post_init__(self):
        self.theta = np.array(self.theta, dtype=np.float64).ravel()


def step(state: OptimizationState, opt: EnergyNaturalGradientOptimizer, loss_fn, grad_fn,
         sensitivity_fn=None, batch_loss_fn=None, rng=None):
    """One optimizer step — EnergyNaturalGradient.jl:239-276: gradient,
    Gram matrix (exact when p <= stochastic_threshold and n_probes == 0, else
    the probe estimate; identity when sensitivity_fn is None), natural
    gradient, log-grid line search, update.  Returns (loss, η)."""
    theta = state.theta
    p = theta.size
    grad = np.asarray(grad_fn(theta), dtype=np.float64).ravel()
    if sensitivity_fn is None:
        nat = grad / (1.0 + opt.regularization)
    else:
        if p <= opt.stochastic_threshold and opt.n_probes == 0:
            G = compute_gram_exact(sensitivity_fn(theta), opt.energy_ip)
        else:
            G = compute_gram_stochastic(sensitivity_fn(theta), p, opt.n_probes, opt.energy_ip, rng)
        nat = compute_natural_gradient(G, grad, opt.regularization)
    eta, loss = line_search_log(loss_fn, theta, nat, opt.line_search_points,
                                opt.line_search_bounds, batch_loss_fn)
    state.theta = theta - eta * nat
    state.iteration += 1
    state.loss_history.append(loss)
    state.eta_history.append(eta)
    return loss, eta


def optimize(state: OptimizationState, opt: EnergyNaturalGradientOptimizer, loss_fn, grad_fn,
             sensitivity_fn, n_iterations: int, callback=None, verbose: bool = False,
             batch_loss_fn=None, rng=None) -> OptimizationState:
    """Up to n_iterations steps; stops when the loss changes by less than
    1e-10 relative — EnergyNaturalGradient.jl:294-321."""
    for k in range(1, n_iterations + 1):
        loss, eta = step(state, opt, loss_fn, grad_fn, sensitivity_fn, batch_loss_fn, rng)
        if verbose and (k % 10 == 0 or k == 1):
            print(f"iteration {k}: loss = {loss:.6g}, eta = {eta:.3g}")
        if callback is not None:
            callback(state, k, loss, eta)
        if len(state.loss_history) > 1:
            a, b = state.loss_history[-1], state.loss_history[-2]
            if abs(a - b) / (abs(b) + 1e-12) < 1e-10:
                break
    return state


# ---------------------------------------------------------------- sensitivities
def compute_sensitivities_forwardmode(forward_solve, theta, step: float = 1e-6,
                                      forward_batch=None) -> list:
    """Wavefield sensitivities [∂θ1 u, ∂θ2 u, ...] for compute_gram_exact —
    EnergyNaturalGradient.jl:337-356, which takes ForwardDiff derivatives
    along each unit vector.  Here central differences of forward_solve
    (θ -> u) with a step of `step` relative to max(1, |θi|); forward_batch,
    if given, takes the list of 2p perturbed θ and returns their u in one
    call (the GPU runs them as one batch)."""
    theta = np.asarray(theta, dtype=np.float64).ravel()
    hs = step * np.maximum(1.0, np.abs(theta))
    trials = []
    for i, h in enumerate(hs):
        e = np.zeros_like(theta)
        e[i] = h
        trials += [theta + e, theta - e]
    us = list(forward_batch(trials)) if forward_batch is not None else [forward_solve(t) for t in trials]
    return [(np.asarray(us[2 * i], dtype=np.float64) - np.asarray(us[2 * i + 1], dtype=np.float64))
            / (2.0 * h) for i, h in enumerate(hs)]


def make_jvp_function(forward_solve, theta, step: float = 1e-6):
    """v -> J v, the wavefield's directional derivative along v at θ, for
    compute_gram_stochastic — EnergyNaturalGradient.jl:367-375 (ForwardDiff
    there; a central difference of step `step` / max(|v|) here)."""
    theta = np.asarray(theta, dtype=np.float64).ravel()

    def jvp(v):
        v = np.asarray(v, dtype=np.float64).ravel()
        h = step / max(float(np.abs(v).max()), 1e-300)
        up = np.asarray(forward_solve(theta + h * v), dtype=np.float64)
        um = np.asarray(forward_solve(theta - h * v), dtype=np.float64)
        return (up - um) / (2.0 * h)

    return jvp


# ---------------------------------------------------------------- seismic problem
class FWIProblem:
    """Loss and gradient of seismic shots for the optimizer.

    θ holds, for each medium plane named in `planes` (keys of
    GRADIENT_PLANES), the relative perturbation of that plane from `base`
    (plane = base_plane · (1 + θ)), flattened plane after plane; the other
    planes stay as in `base`.  `shots` are workloads on base's grid (their
    own sources, wavelets, receivers, nt) and `obs` their observed traces
    ([2, nrec, nt] each).  loss(θ) = Σ_shots J, grad(θ) = dloss/dθ by
    vi_gradient; batch_loss evaluates many θ for all shots as one vi_batch.

    Under torch.distributed each rank evaluates its round-robin share of the
    shots and one FP64 all-reduce sums the misfit with the gradient (or the
    line search's losses), so every rank holds the same sums and takes the
    same optimizer step; only the ranks' share of `obs` is read."""

    def __init__(self, base: _media.Workload, shots, obs, planes=("c13", "c55"),
                 precision: str = "f64", checkpoint_every: int = 0, group=None):
        unknown = [k for k in planes if k not in GRADIENT_PLANES or k not in base.medium]
        if unknown:
            raise ValueError(f"planes not in the medium: {unknown}")
        if len(shots) != len(obs):
            raise ValueError("one observed gather per shot")
        for w in shots:
            if (w.nx, w.nz, w.kind, w.nsls) != (base.nx, base.nz, base.kind, base.nsls):
                raise ValueError("every shot must share base's grid, medium kind and nsls")
        self.base, self.shots, self.planes = base, list(shots), tuple(planes)
        self.obs = [np.asarray(o, dtype=np.float64) for o in obs]
        self.precision, self.checkpoint_every = precision, int(checkpoint_every)
        self.np = base.nx * base.nz
        self.n_params = len(self.planes) * self.np
        self.group = group
        rank, world = 0, 1
        if torch.distributed.is_available() and torch.distributed.is_initialized():
            rank, world = torch.distributed.get_rank(group), torch.distributed.get_world_size(group)
        self.mine = shard(len(self.shots), rank, world)
        self._plan = None

    @property
    def plan(self) -> StepPlan:
        if self._plan is None:
            self._plan = StepPlan.for_workload(self.base, self.precision)
        return self._plan

    def medium(self, theta) -> dict:
        theta = np.asarray(theta, dtype=np.float64).reshape(len(self.planes), self.base.nz, self.base.nx)
        med = dict(self.base.medium)
        for n, k in enumerate(self.planes):
            med[k] = self.base.medium[k] * (1.0 + theta[n])
        return med

    # per-shot work on this rank's GPU
    def _shots_value_and_grad(self, theta, shots):
        """(Σ J, Σ dJ/dplane [8, nz, nx] float64 numpy) over the given shots."""
        plan, dev = self.plan, self.plan.device
        med = plan.medium_to_device(self.medium(theta))
        g = torch.zeros(8, self.base.nz, self.base.nx, dtype=torch.float64, device=dev)
        J = 0.0
        for i in shots:
            w = self.shots[i]
            wav = torch.as_tensor(w.wavelets[:, :w.nt], dtype=plan.dtype, device=dev).contiguous()
            obs = torch.as_tensor(self.obs[i], dtype=plan.dtype, device=dev).contiguous()
            Jw, g = misfit_gradient(plan, med, w.sources, wav, w.receivers, obs, nt=w.nt,
                                    checkpoint_every=self.checkpoint_every, grad=g, accumulate=True)
            J += Jw
        return J, g.cpu().numpy()

    def _shots_batch_loss(self, thetas, shots) -> np.ndarray:
        """Σ_shots J for every θ over the given shots, as one batched run."""
        if not shots:
            return np.zeros(len(thetas))
        ws = [dataclasses.replace(self.shots[i], medium=self.medium(t)) for t in thetas for i in shots]
        b = ShotBatch(ws, self.precision)
        try:
            b.run()
            b.status()
            out = np.zeros(len(thetas))
            for n in range(len(thetas)):
                for k, i in enumerate(shots):
                    d = b.traces[n * len(shots) + k].double()
                    o = torch.as_tensor(self.obs[i], device=d.device)
                    out[n] += 0.5 * float(torch.sum((d - o) ** 2))
            return out
        finally:
            b.close()

    # sums over every shot (all ranks)
    def _allreduce(self, flat: np.ndarray) -> np.ndarray:
        if not (torch.distributed.is_available() and torch.distributed.is_initialized()):
            return flat
        t = torch.as_tensor(flat, dtype=torch.float64)
        if torch.distributed.get_backend(self.group) == "nccl":
            t = t.to(self.plan.device)
        torch.distributed.all_reduce(t, op=torch.distributed.ReduceOp.SUM, group=self.group)
        return t.cpu().numpy()

    def value_and_grad(self, theta):
        J, g = self._shots_value_and_grad(theta, self.mine)
        # plane = base · (1 + θ): dJ/dθ = dJ/dplane · base
        gp = np.stack([g[GRADIENT_PLANES.index(k)] * self.base.medium[k] for k in self.planes])
        tot = self._allreduce(np.concatenate([gp.ravel(), [J]]))
        return float(tot[-1]), tot[:-1]

    def loss(self, theta) -> float:
        return self.value_and_grad(theta)[0]

    def grad(self, theta) -> np.ndarray:
        return self.value_and_grad(theta)[1]

    def batch_loss(self, thetas) -> list:
        """Σ_shots J for every θ: this rank's shots as one batched run, then
        one all-reduce of the losses."""
        return list(self._allreduce(self._shots_batch_loss(thetas, self.mine)))

    def close(self):
        if self._plan is not None:
            self._plan.close()
            self._plan = None
