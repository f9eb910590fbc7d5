"""Misfit gradient of the time step over the vi_gradient C ABI.

The reference has no receivers, misfit or adjoint; its optimizer
(sciml_solver/EnergyNaturalGradient.jl:239-321, `step!` / `optimize!`)
takes a `grad_fn` and a `loss_fn` and is never wired to the wave solver
(examples/energy_natural_gradient_example.jl:252-315).  `misfit_gradient`
is that grad_fn for the leapfrog step: J = 1/2 sum (d - obs)^2 over the vx
and vz traces and dJ/d(medium planes), by the discrete adjoint of the step
in libvisco_b200.so; `shot_misfit` wraps it as a torch autograd function.
`shot_gradient` sums over shots, sharded by shot over
the ranks of a process group with one FP64 all-reduce of the gradient
planes and the misfit.
"""
from __future__ import annotations

import ctypes as C

import numpy as np
import torch

from ._abi import MEDIUM_KINDS, check, lib
from .solver import MEDIUM_NAMES, StepPlan, _stream_handle

GRADIENT_PLANES = MEDIUM_NAMES  # rho, c11, c13, c15, c33, c35, c55, tau
VELOCITY_PLANES = ("vp", "vs", "rho", "qinv")


def misfit_gradient(plan: StepPlan, medium: dict, sources, wavelets, receivers, obs: torch.Tensor,
                    nt: int | None = None, checkpoint_every: int = 0, grad: torch.Tensor | None = None,
                    accumulate: bool = False, traces: torch.Tensor | None = None, stream=None):
    """Misfit J and its gradient for one shot run from rest.

    medium: device planes in the plan's precision; obs: device [2, nrec, nt]
    observed traces in the plan's precision.  Returns (J, grad) with grad a
    float64 [8, nz, nx] tensor of dJ/d(rho, c11, c13, c15, c33, c35, c55,
    tau); for ISO media plane c13 holds dJ/dlambda and c55 dJ/dmu.
    accumulate=True adds into the given grad (shots summed)."""
    nt = obs.shape[2] if nt is None else int(nt)
    if tuple(obs.shape) != (2, len(receivers), nt) or not obs.is_contiguous():
        raise ValueError("obs must be a contiguous [2, nrec, nt] device tensor")
    if obs.dtype != plan.dtype:
        raise ValueError(f"obs must be {plan.dtype}")
    if grad is None:
        grad = torch.zeros(8, plan.nz, plan.nx, dtype=torch.float64, device=plan.device)
        accumulate = False
    elif tuple(grad.shape) != (8, plan.nz, plan.nx) or grad.dtype != torch.float64:
        raise ValueError("grad must be float64 [8, nz, nx]")
    med = plan._medium_struct(medium)
    shot, keep = plan._shot(sources, wavelets, receivers, traces)
    J = C.c_double()
    with torch.cuda.device(plan.device):
        check(lib().vi_gradient(plan._h, C.byref(med), C.byref(shot), nt, obs.data_ptr(),
                                int(checkpoint_every), int(bool(accumulate)), grad.data_ptr(),
                                C.byref(J), _stream_handle(stream)))
    del keep
    return J.value, grad


class ShotMisfit(torch.autograd.Function):
    """The misfit J(medium) of one shot as a torch autograd function, the
    counterpart of a ChainRulesCore.rrule on the Julia side: forward runs
    vi_gradient, which yields J and dJ/d(medium planes) in one forward and
    adjoint pass, and keeps the gradient; backward scales it by the incoming
    cotangent.  Use through `shot_misfit`."""

    @staticmethod
    def forward(ctx, plan, sources, wavelets, receivers, obs, checkpoint_every, names, *planes):
        J, g = misfit_gradient(plan, dict(zip(names, planes)), sources, wavelets, receivers, obs,
                               checkpoint_every=checkpoint_every)
        ctx.names = names
        ctx.dtypes = [t.dtype for t in planes]
        ctx.save_for_backward(g)
        return torch.tensor(J, dtype=torch.float64, device=g.device)

    @staticmethod
    def backward(ctx, gJ):
        (g,) = ctx.saved_tensors
        grads = [(gJ * g[GRADIENT_PLANES.index(n)]).to(dt) for n, dt in zip(ctx.names, ctx.dtypes)]
        return (None,) * 7 + tuple(grads)


def shot_misfit(plan: StepPlan, medium: dict, sources, wavelets, receivers, obs: torch.Tensor,
                checkpoint_every: int = 0) -> torch.Tensor:
    """J of one shot (0-d float64 tensor) differentiable with respect to
    every medium plane given (device tensors in the plan's precision, keys
    of GRADIENT_PLANES), so that J.backward() reaches parameters the planes
    were computed from in torch (velocities, Thomsen parameters, 1/Q)."""
    names = tuple(k for k in GRADIENT_PLANES if k in medium)
    if set(names) != set(medium):
        raise ValueError(f"medium keys must be among {GRADIENT_PLANES}")
    return ShotMisfit.apply(plan, sources, wavelets, receivers, obs, int(checkpoint_every), names,
                            *[medium[n].contiguous() for n in names])


def velocity_gradient(kind: str, grad: torch.Tensor, vp: torch.Tensor, vs: torch.Tensor,
                      rho: torch.Tensor, eps: torch.Tensor | None = None,
                      delta: torch.Tensor | None = None, tau_scale: float = 1.0,
                      stream=None) -> torch.Tensor:
    """[4, nz, nx] float64: dJ/d(vp, vs, rho at fixed velocities, 1/Q) from
    the stiffness gradient (ISO: Lame from vp, vs, rho; VTI: Thomsen,
    Models.jl:27-52).  tau_scale = d tau / d(1/Q) = N / Kbar of the Q fit."""
    np_ = grad.shape[1] * grad.shape[2]
    out = torch.empty(4, grad.shape[1], grad.shape[2], dtype=torch.float64, device=grad.device)

    def p(t):
        if t is None:
            return None
        if t.dtype != torch.float64 or not t.is_contiguous() or t.numel() != np_:
            raise ValueError("velocity planes must be contiguous float64 [nz, nx]")
        return t.data_ptr()

    with torch.cuda.device(grad.device):
        check(lib().vi_gradient_velocity(MEDIUM_KINDS[kind], np_, grad.data_ptr(), p(vp), p(vs),
                                         p(rho), p(eps), p(delta), float(tau_scale),
                                         out.data_ptr(), _stream_handle(stream)))
    return out


def thomsen_gradient(grad: torch.Tensor, vp: torch.Tensor, vs: torch.Tensor, rho: torch.Tensor,
                     delta: torch.Tensor | None = None, stream=None) -> torch.Tensor:
    """[2, nz, nx] float64: dJ/d(epsilon, delta) of a VTI medium at fixed
    vp, vs, rho, from the stiffness gradient (C11 = C33 (1 + 2 epsilon),
    C13 from delta: media.thomsen_vti).  gamma, the third Thomsen parameter
    of custom_solver/Model.jl:12-16, enters only SH motion: its gradient is
    zero in 2D P-SV."""
    np_ = grad.shape[1] * grad.shape[2]
    out = torch.empty(2, grad.shape[1], grad.shape[2], dtype=torch.float64, device=grad.device)

    def p(t):
        if t is None:
            return None
        if t.dtype != torch.float64 or not t.is_contiguous() or t.numel() != np_:
            raise ValueError("velocity planes must be contiguous float64 [nz, nx]")
        return t.data_ptr()

    with torch.cuda.device(grad.device):
        check(lib().vi_gradient_thomsen(np_, grad.data_ptr(), p(vp), p(vs), p(rho), p(delta),
                                        out.data_ptr(), _stream_handle(stream)))
    return out


TTI_PARAMETERS = ("vp", "vs", "rho", "qinv", "eps", "delta", "theta")


def tti_gradient(grad: torch.Tensor, vp: torch.Tensor, vs: torch.Tensor, rho: torch.Tensor,
                 eps: torch.Tensor | None = None, delta: torch.Tensor | None = None,
                 theta: torch.Tensor | None = None, tau_scale: float = 0.0, stream=None) -> torch.Tensor:
    """[7, nz, nx] float64: dJ/d(vp, vs, rho, 1/Q, epsilon, delta, theta) of
    a TTI medium (TTI_PARAMETERS order) from the stiffness gradient of
    vi_gradient, through Thomsen's law tilted by theta (the map of
    medium_from_velocity / media.bond_rotate)."""
    np_ = grad.shape[1] * grad.shape[2]
    out = torch.empty(7, grad.shape[1], grad.shape[2], dtype=torch.float64, device=grad.device)

    def p(t):
        if t is None:
            return None
        if t.dtype != torch.float64 or not t.is_contiguous() or t.numel() != np_:
            raise ValueError("parameter planes must be contiguous float64 [nz, nx]")
        return t.data_ptr()

    with torch.cuda.device(grad.device):
        check(lib().vi_gradient_tti(np_, grad.data_ptr(), p(vp), p(vs), p(rho), p(eps), p(delta), p(theta),
                                    float(tau_scale), out.data_ptr(), _stream_handle(stream)))
    return out


def shard(nshots: int, rank: int, world: int) -> list[int]:
    """Shots of this rank: round robin, so uneven shot costs spread."""
    return list(range(rank, nshots, world))


def reduce_gradient(grad: torch.Tensor, misfit: float, group=None):
    """Sums the gradient planes (FP64) and the misfit over the process group
    (NCCL on GPUs, gloo on CPUs) in one all-reduce.  Every rank calls it
    once per gradient evaluation, in the same order."""
    import torch.distributed as dist

    if not dist.is_available() or not dist.is_initialized():
        return grad, misfit
    flat = torch.cat([grad.reshape(-1), torch.tensor([misfit], dtype=torch.float64,
                                                      device=grad.device)])
    dist.all_reduce(flat, op=dist.ReduceOp.SUM, group=group)
    return flat[:-1].view_as(grad), float(flat[-1].item())


def shot_gradient(gradient_fn, nshots: int, shape, device="cpu", group=None):
    """(J, grad): the sum over shots of gradient_fn(i) -> (J_i, grad_i
    [8, nz, nx] float64), each rank evaluating its shard and one all-reduce
    combining them; every rank returns the full sum."""
    import torch.distributed as dist

    rank, world = 0, 1
    if dist.is_available() and dist.is_initialized():
        rank, world = dist.get_rank(group), dist.get_world_size(group)
    total = torch.zeros(8, *shape, dtype=torch.float64, device=device)
    J = 0.0
    for i in shard(nshots, rank, world):
        Ji, gi = gradient_fn(i)
        total += gi
        J += Ji
    total, J = reduce_gradient(total, J, group)
    return J, total
