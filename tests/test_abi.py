"""The C ABI library loads, exports every symbol include/wayland_b200.h declares, and its
host-only entry points behave (no GPU needed)."""
import ctypes as C
import subprocess

import pytest

from wayland_b200 import _abi


def test_exports_every_declared_symbol(native_lib):
    declared = _abi.header_symbols()
    assert len(declared) >= 25
    for name in declared:
        assert hasattr(native_lib, name), name
    assert set(declared) == set(_abi.SIGNATURES)


def test_dynamic_symbols_are_only_the_abi():
    out = subprocess.run(["nm", "-D", "--defined-only", _abi.LIB_PATH], capture_output=True,
                         text=True, check=True).stdout
    exported = {l.split()[-1] for l in out.splitlines() if " T " in l}
    wl = {s for s in exported if s.startswith("wl_")}
    assert wl == set(_abi.header_symbols())


def test_version_and_defaults(native_lib):
    assert b"sm_100a" in native_lib.wl_version()
    p = _abi.RenderParams()
    native_lib.wl_render_params_default(C.byref(p), 64, 32, 4)
    assert (p.width, p.height, p.spp) == (64, 32, 4)
    # the reference's constants: PathTracing.cu:19-29, 68, 130, 235
    assert p.max_depth == 25 and p.rr_depth == 5 and abs(p.rr_prob - 0.9) < 1e-7
    assert abs(p.eps - 1e-3) < 1e-9 and p.strategy == _abi.STRATEGY_MIS and p.rng == _abi.RNG_TEA_LCG


def test_null_arguments_are_rejected(native_lib):
    assert native_lib.wl_context_create(0, None) == 1  # WL_ERR_INVALID_ARG
    assert b"null" in native_lib.wl_last_error_string()
    assert native_lib.wl_render(None, None, None, None, None) == 1
    assert native_lib.wl_cast_rays(None, None, None, 0, 0) == 1
    assert native_lib.wl_film_download(None, None, None) == 1


def test_struct_sizes():
    assert C.sizeof(_abi.Disney) == 64
    assert C.sizeof(_abi.AreaLight) == 24
    assert C.sizeof(_abi.Camera) == 48
    assert C.sizeof(_abi.RenderParams) == 80
    assert _abi.RAY_DTYPE.itemsize == 32 and _abi.HIT_DTYPE.itemsize == 16
