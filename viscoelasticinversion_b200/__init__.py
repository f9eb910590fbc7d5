"""B200-native 2D viscoelastic / anisotropic staggered-grid time step.

libvisco_b200.so (hand-written sm_100a CUDA behind a C ABI, see
include/visco_b200.h) does all the work; this package is the host side:
ctypes bindings (_abi), the plan wrapper (solver), the reference-facing
names (api) and the host-side set-up of media, wavelets and Q (media).
"""
from ._abi import VI_HALF, VI_MAX_SLS, ViError, CFLError, BudgetError, lib  # noqa: F401
from .solver import StepPlan, CPMLSpec, make_config, config_from_workload, diff  # noqa: F401
from . import media  # noqa: F401

__version__ = "0.1.0"
