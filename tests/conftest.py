"""Test configuration. `-m gpu` tests need a CUDA device and the built native library; every
other test runs on the CPU (oracle, golden vectors, host-compiled BVH logic, ABI symbols)."""
import os
import subprocess
import sys

import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
sys.path.insert(0, ROOT)
sys.path.insert(0, os.path.join(ROOT, "oracle"))
BUILD = os.path.join(ROOT, "tests", "_build")


def pytest_configure(config):
    config.addinivalue_line("markers", "gpu: needs a CUDA GPU (B200) and the native library")


def _has_gpu():
    try:
        import torch
        return torch.cuda.is_available()
    except Exception:
        return False


def pytest_collection_modifyitems(config, items):
    if _has_gpu():
        return
    skip = pytest.mark.skip(reason="no CUDA device")
    for it in items:
        if "gpu" in it.keywords:
            it.add_marker(skip)


@pytest.fixture(scope="session")
def oracle():
    import pyoracle
    return pyoracle.Oracle()


@pytest.fixture(scope="session")
def native_lib():
    """The product library (built in-tree if it is missing)."""
    from wayland_b200 import _abi, build
    if not os.path.exists(_abi.LIB_PATH):
        build.build()
    return _abi.load()


@pytest.fixture(scope="session")
def host_bvh():
    """Test harness: wl_bvh.cuh compiled for the CPU (tests/native/bvh_host.cpp)."""
    import ctypes as C
    os.makedirs(BUILD, exist_ok=True)
    out = os.path.join(BUILD, "libbvh_host.so")
    src = os.path.join(ROOT, "tests", "native", "bvh_host.cpp")
    deps = [src] + [os.path.join(ROOT, "wayland_b200", "csrc", f) for f in ("wl_bvh.cuh", "wl_math.cuh")]
    if not os.path.exists(out) or any(os.path.getmtime(d) > os.path.getmtime(out) for d in deps):
        subprocess.check_call(["g++", "-O2", "-std=c++17", "-ffp-contract=off", "-fPIC", "-shared", "-w",
                               "-I", os.path.join(ROOT, "wayland_b200", "csrc"),
                               "-I", "/usr/local/cuda/include", src, "-o", out])
    lib = C.CDLL(out)
    lib.hb_build.restype = C.c_void_p
    lib.hb_build.argtypes = [C.c_void_p, C.c_void_p, C.c_uint32]
    lib.hb_destroy.argtypes = [C.c_void_p]
    lib.hb_cast.argtypes = [C.c_void_p, C.c_void_p, C.c_uint32, C.c_uint32, C.c_void_p, C.c_void_p]
    lib.hb_cast_batched.argtypes = [C.c_void_p, C.c_void_p, C.c_uint32, C.c_uint32, C.c_uint32,
                                    C.c_uint32, C.c_uint32, C.c_void_p, C.c_void_p]
    lib.hb_info.restype = C.c_uint32
    lib.hb_info.argtypes = [C.c_void_p, C.c_void_p]
    lib.hb_export.argtypes = [C.c_void_p] * 5
    return lib


@pytest.fixture(scope="session")
def ctx(native_lib):
    import wayland_b200 as wl
    c = wl.Context(0)
    yield c
    c.close()
