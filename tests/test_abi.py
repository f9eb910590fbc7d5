"""The C-ABI library loads here (no GPU needed) and exports every entry point
include/*.h declares; the ctypes mirror matches the header."""
import ctypes as C
import re
from pathlib import Path

import pytest

from viscoelasticinversion_b200 import _abi

ROOT = Path(__file__).resolve().parents[1]


def declared_functions() -> set[str]:
    names = set()
    for h in (ROOT / "include").glob("*.h"):
        text = re.sub(r"/\*.*?\*/", "", h.read_text(), flags=re.S)
        names |= set(re.findall(r"\b(vi_[a-z0-9_]+)\s*\(", text))
    return names


def test_library_exports_every_declared_symbol():
    lib = _abi.lib()
    declared = declared_functions()
    assert declared, "no declarations found"
    missing = [n for n in sorted(declared) if not hasattr(lib, n)]
    assert not missing, f"not exported: {missing}"
    assert declared == set(_abi.exported_names()), "ctypes signatures differ from the header"


def test_version_and_error_without_gpu():
    lib = _abi.lib()
    assert lib.vi_version() == 1
    # an argument error needs no device
    rc = lib.vi_plan_create(None, C.byref(C.c_void_p()))
    assert rc == _abi.VI_ERR_ARG
    assert b"NULL" in lib.vi_last_error()


def test_struct_layouts_match_header():
    # sizes follow the C layout of include/visco_b200.h on LP64
    assert C.sizeof(_abi.ViSource) == 24
    assert C.sizeof(_abi.ViReceiver) == 8
    assert C.sizeof(_abi.ViMedium) == 64
    assert C.sizeof(_abi.ViFields) == 56
    assert C.sizeof(_abi.ViConfig) == 160
    assert _abi.ViConfig.tau_sls.offset == 48
    assert _abi.ViConfig.pml_d0.offset == 112


@pytest.mark.parametrize("bad", [
    dict(nx=8), dict(dt=0.0), dict(nsls=6), dict(medium=7), dict(precision=3),
])
def test_config_validation_errors(bad):
    from viscoelasticinversion_b200.solver import make_config

    cfg = make_config(64, 64, 5.0, 5.0, 1e-4)
    for k, v in bad.items():
        setattr(cfg, k, v)
    h = C.c_void_p()
    rc = _abi.lib().vi_plan_create(C.byref(cfg), C.byref(h))
    assert rc == _abi.VI_ERR_ARG and not h.value


def test_cfl_violation_is_reported_before_any_device_work():
    from viscoelasticinversion_b200.solver import make_config

    cfg = make_config(64, 64, 5.0, 5.0, 2e-3, vmax=3000.0)
    h = C.c_void_p()
    assert _abi.lib().vi_plan_create(C.byref(cfg), C.byref(h)) == _abi.VI_ERR_CFL
    with pytest.raises(_abi.CFLError):
        _abi.check(_abi.VI_ERR_CFL)


def test_missing_library_fails_loudly(monkeypatch, tmp_path):
    """No fallback: without the built library every call path raises."""
    monkeypatch.setattr(_abi, "LIB_PATH", tmp_path / "libvisco_b200.so")
    monkeypatch.setattr(_abi, "_lib", None)
    with pytest.raises(RuntimeError, match="no CPU fallback"):
        _abi.lib()
    with pytest.raises(RuntimeError, match="not built"):
        _abi.check(_abi.VI_ERR_ARG)


def test_medium_from_velocity_argument_checks():
    """Argument errors are found before any device work (no GPU needed)."""
    lib = _abi.lib()
    dummy = C.c_void_p(16)  # never dereferenced: the checks fail first
    out = _abi.ViMedium()
    out.rho = out.c55 = 16  # c13 missing
    rc = lib.vi_medium_from_velocity(_abi.VI_MEDIUM_ISO, _abi.VI_F32, 10, dummy, dummy, dummy, None,
                                     None, None, None, 0.0, C.byref(out), None)
    assert rc == _abi.VI_ERR_ARG and b"NULL" in lib.vi_last_error()
    out.c13 = 16
    rc = lib.vi_medium_from_velocity(_abi.VI_MEDIUM_ISO, 7, 10, dummy, dummy, dummy, None, None,
                                     None, None, 0.0, C.byref(out), None)
    assert rc == _abi.VI_ERR_ARG and b"precision" in lib.vi_last_error()
    rc = lib.vi_medium_from_velocity(_abi.VI_MEDIUM_VTI, _abi.VI_F32, 10, dummy, dummy, dummy, None,
                                     None, None, None, 0.0, C.byref(out), None)
    assert rc == _abi.VI_ERR_ARG  # VTI needs c11 and c33
