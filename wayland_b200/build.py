"""Build the native library in-tree: wayland_b200/lib/libwayland_b200.so (sm_100a).

Each translation unit gets the arithmetic flags its kernels are specified with:
  pt_fast.cu    --use_fast_math (the reference's own device compile mode)
  pt_strict.cu  -fmad=false -prec-div=true -prec-sqrt=true -ftz=false (bit-exact with the oracle)
  others        IEEE defaults; hit arithmetic uses explicitly rounded intrinsics.
"""
import os
import subprocess
import sys
from concurrent.futures import ThreadPoolExecutor

PKG = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(PKG)
CSRC = os.path.join(PKG, "csrc")
OBJ = os.path.join(PKG, "_build")
LIB = os.path.join(PKG, "lib", "libwayland_b200.so")
NVCC = os.environ.get("NVCC", "/usr/local/cuda/bin/nvcc")
ARCH = ["-gencode", "arch=compute_100a,code=sm_100a"]
COMMON = ["-O3", "-std=c++17", "-lineinfo", "-Xcompiler", "-fPIC", "-Xcompiler", "-fvisibility=hidden",
          "-I", CSRC, "-I", os.path.join(ROOT, "include"), "--expt-relaxed-constexpr"]
UNITS = {
    "api.cu": [],
    "bvh_build.cu": [],
    "traverse.cu": [],
    "pt_fast.cu": ["--use_fast_math"],
    "pt_strict.cu": ["-fmad=false", "-prec-div=true", "-prec-sqrt=true", "-ftz=false"],
    "noalloc.cu": [],
    "ao.cu": ["-fmad=false", "-prec-div=true", "-prec-sqrt=true", "-ftz=false"],
    "nrc.cu": [],
    "nrc_tc.cu": [],
}


def _deps():
    return [os.path.join(CSRC, f) for f in os.listdir(CSRC) if f.endswith((".cuh", ".h"))] + \
        [os.path.join(ROOT, "include", "wayland_b200.h")]


def _stale(target, sources):
    if not os.path.exists(target):
        return True
    t = os.path.getmtime(target)
    return any(os.path.getmtime(s) > t for s in sources)


def compile_unit(name, flags, verbose=False, extra=()):
    src = os.path.join(CSRC, name)
    obj = os.path.join(OBJ, name + ".o")
    if not _stale(obj, [src, *_deps(), __file__]):
        return obj
    cmd = [NVCC, *ARCH, *COMMON, *flags, *extra, "-c", src, "-o", obj]
    if verbose:
        print(" ".join(cmd), flush=True)
    r = subprocess.run(cmd, capture_output=True, text=True)
    if r.returncode != 0:
        raise RuntimeError(f"nvcc failed for {name}:\n{r.stdout}\n{r.stderr}")
    if r.stderr.strip() and verbose:
        print(r.stderr)
    return obj


def build(verbose=False, ptxas_info=False):
    os.makedirs(OBJ, exist_ok=True)
    os.makedirs(os.path.dirname(LIB), exist_ok=True)
    extra = ["-Xptxas", "-v"] if ptxas_info else []
    with ThreadPoolExecutor(max_workers=len(UNITS)) as ex:
        objs = list(ex.map(lambda kv: compile_unit(kv[0], kv[1], verbose, extra), UNITS.items()))
    if _stale(LIB, objs):
        cmd = [NVCC, *ARCH, "-shared", "-o", LIB, *objs]
        r = subprocess.run(cmd, capture_output=True, text=True)
        if r.returncode != 0:
            raise RuntimeError(f"link failed:\n{r.stdout}\n{r.stderr}")
    return LIB


if __name__ == "__main__":
    print(build(verbose="-v" in sys.argv, ptxas_info="--ptxas" in sys.argv))
