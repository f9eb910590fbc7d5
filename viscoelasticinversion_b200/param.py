"""Medium planes from velocity-domain parameters on the device
(vi_medium_from_velocity): the GPU form of media.medium_from_velocity and
media.bond_rotate, which the reference runs on the host before every solve
(sciml_solver/Models.jl:27-67, custom_solver/Model.jl:12-16)."""
from __future__ import annotations

import ctypes as C

import torch

from ._abi import MEDIUM_KINDS, VI_F32, VI_F64, ViMedium, check, lib
from .solver import _stream_handle

PLANES = {"iso": ("rho", "c13", "c55"), "vti": ("rho", "c11", "c13", "c33", "c55"),
          "tti": ("rho", "c11", "c13", "c15", "c33", "c35", "c55")}


def medium_from_velocity_device(kind: str, vp: torch.Tensor, vs: torch.Tensor, rho: torch.Tensor,
                                eps: torch.Tensor | None = None, delta: torch.Tensor | None = None,
                                theta: torch.Tensor | None = None, Q: torch.Tensor | None = None,
                                tau_scale: float | None = None, precision: str = "f32",
                                stream=None) -> dict:
    """Medium planes (device tensors of the plan's precision, keyed as
    vi_medium) from contiguous FP64 device planes [nz, nx]: ISO Lamé, VTI
    Thomsen (eps, delta), TTI the VTI stiffness tilted by theta (radians);
    with Q also tau = tau_scale / Q (tau_scale = N / Kbar of the Q fit)."""
    if kind not in PLANES:
        raise ValueError(f"kind must be one of {tuple(PLANES)}")
    if Q is not None and tau_scale is None:
        raise ValueError("Q needs tau_scale (N / Kbar of the Q fit)")
    shape, dev = vp.shape, vp.device
    np_ = vp.numel()

    def p(t):
        if t is None:
            return None
        if t.dtype != torch.float64 or not t.is_contiguous() or t.shape != shape or t.device != dev:
            raise ValueError("parameter planes must be contiguous float64 [nz, nx] on one device")
        return t.data_ptr()

    dtype = torch.float64 if precision == "f64" else torch.float32
    names = PLANES[kind] + (("tau",) if Q is not None else ())
    out = {k: torch.empty(shape, dtype=dtype, device=dev) for k in names}
    m = ViMedium()
    for k, t in out.items():
        setattr(m, k, t.data_ptr())
    with torch.cuda.device(dev):
        check(lib().vi_medium_from_velocity(MEDIUM_KINDS[kind], VI_F64 if precision == "f64" else VI_F32,
                                            np_, p(vp), p(vs), p(rho), p(eps), p(delta), p(theta),
                                            p(Q), float(tau_scale or 0.0), C.byref(m),
                                            _stream_handle(stream)))
    return out
