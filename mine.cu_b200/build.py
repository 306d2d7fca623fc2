"""Build the native parts of the package, in-tree, for sm_100a.

  minecu/libminecu_b200.so  C-ABI library (include/minecu_b200.h): CUDA
                            kernels + host runtime, no torch dependency.
                            mc_fast.cu is compiled with --use_fast_math (the
                            reference's numerics), mc_ieee.cu with -fmad=false
                            (IEEE numerics), mc_runtime.cu with defaults.
  minecu/libminecu_b200_checked.so
                            the same library with every index bounds-checked
                            (-DMC_CHECK_BOUNDS=1): a debug build for tests.
  minecu/_C*.so             torch extension (minecu._C) binding tensors to the
                            C-ABI; linked against libminecu_b200.so.

Run `python mine.cu_b200/build.py`; it only rebuilds what changed.
"""
from __future__ import annotations

import glob
import os
import shutil
import subprocess
import sys
import sysconfig

PKG_ROOT = os.path.dirname(os.path.abspath(__file__))
REPO = os.path.dirname(PKG_ROOT)
CSRC = os.path.join(PKG_ROOT, "csrc")
OUT = os.path.join(PKG_ROOT, "minecu")
BUILD = os.path.join(PKG_ROOT, "_build")
INCLUDE = os.path.join(REPO, "include")
LIB = os.path.join(OUT, "libminecu_b200.so")
CHECKED_LIB = os.path.join(OUT, "libminecu_b200_checked.so")

ARCH = ["-gencode", "arch=compute_100a,code=sm_100a"]
NVCC_COMMON = ["-std=c++17", "-O3", "-lineinfo", "-Xcompiler", "-fPIC", "-I", INCLUDE, "-I", CSRC] + ARCH

UNITS = {
    "mc_fast": ["--use_fast_math"],
    "mc_ieee": ["-fmad=false", "-prec-div=true", "-prec-sqrt=true", "-ftz=false"],
    "mc_runtime": [],
    "mc_noalloc": [],
    "mc_server": [],
}


def _nvcc() -> str:
    cand = [os.environ.get("NVCC"), shutil.which("nvcc"), "/usr/local/cuda/bin/nvcc"]
    for c in cand:
        if c and os.path.exists(c):
            return c
    raise RuntimeError("nvcc not found")


def _headers():
    return glob.glob(os.path.join(CSRC, "*.h")) + glob.glob(os.path.join(CSRC, "*.cuh")) + \
        glob.glob(os.path.join(INCLUDE, "*.h"))


def _stale(target: str, deps) -> bool:
    if not os.path.exists(target):
        return True
    t = os.path.getmtime(target)
    return any(os.path.getmtime(d) > t for d in deps)


def _run(cmd, verbose):
    if verbose:
        print(" ".join(cmd), flush=True)
    subprocess.run(cmd, check=True)


def build_lib(verbose: bool = False, checked: bool = False) -> str:
    bdir = os.path.join(BUILD, "checked") if checked else BUILD
    lib = CHECKED_LIB if checked else LIB
    os.makedirs(bdir, exist_ok=True)
    nvcc = _nvcc()
    hdrs = _headers()
    objs = []
    extra = ["-DMC_CHECK_BOUNDS=1"] if checked else []
    for unit, flags in UNITS.items():
        src = os.path.join(CSRC, unit + ".cu")
        obj = os.path.join(bdir, unit + ".o")
        objs.append(obj)
        if _stale(obj, [src] + hdrs):
            _run([nvcc] + NVCC_COMMON + flags + extra + ["-c", src, "-o", obj], verbose)
    if _stale(lib, objs):
        # -Bsymbolic: the library's own calls bind to its own functions, so the
        # normal and the checked build can be loaded into one process
        _run([nvcc] + ARCH + ["-shared", "-Xlinker", "-soname=" + os.path.basename(lib), "-Xlinker", "-Bsymbolic",
                              "-o", lib] + objs + ["-lcudart_static", "-lrt", "-ldl", "-lpthread"], verbose)
    return lib


def build_torch_ext(verbose: bool = False) -> str:
    src = os.path.join(CSRC, "mc_torch.cpp")
    suffix = sysconfig.get_config_var("EXT_SUFFIX") or ".so"
    target = os.path.join(OUT, "_C" + suffix)
    if not _stale(target, [src, LIB, os.path.join(INCLUDE, "minecu_b200.h")]):
        return target
    import ctypes

    from torch.utils.cpp_extension import load  # noqa: imported lazily (slow)

    # load() imports the result from the build directory, where $ORIGIN does
    # not hold the library; make it resolvable by soname first
    ctypes.CDLL(LIB, mode=ctypes.RTLD_GLOBAL)

    bdir = os.path.join(BUILD, "torch_ext")
    os.makedirs(bdir, exist_ok=True)
    load(
        name="_C",
        sources=[src],
        extra_include_paths=[INCLUDE, CSRC],
        extra_cflags=["-O3", "-std=c++17"],
        extra_ldflags=[f"-L{OUT}", "-lminecu_b200", "-Wl,-rpath,$ORIGIN"],
        build_directory=bdir,
        with_cuda=True,
        is_python_module=False,
        verbose=verbose,
    )
    built = os.path.join(bdir, "_C.so")
    shutil.copy(built, target + ".tmp")  # a fresh mtime: the next build sees it up to date
    os.replace(target + ".tmp", target)
    return target


def build(verbose: bool = False) -> None:
    build_lib(verbose)
    build_torch_ext(verbose)
    build_lib(verbose, checked=True)


if __name__ == "__main__":
    build(verbose="-v" in sys.argv)
    print("built", LIB)
