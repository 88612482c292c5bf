"""Builds the native library and the bsim_cuda-compatible driver, in-tree.

    python -m bitstreamzoo_b200.build [-v] [--force]

Outputs (git-ignored, shipped with the source tree):
    bitstreamzoo_b200/lib/libbsz.so   C ABI of include/bsz.h
    bitstreamzoo_b200/lib/bsim_cuda   drop-in for the reference binary

Every CUDA translation unit is compiled for sm_100a only
(-gencode arch=compute_100a,code=sm_100a).  Fused segment kernels are
generated at run time and compiled by NVRTC for the same target.
"""

from __future__ import annotations

import argparse
import concurrent.futures as cf
import os
import shutil
import subprocess
import sys

PKG = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(PKG)
CSRC = os.path.join(PKG, "csrc")
LIB = os.path.join(PKG, "lib")
OBJ = os.path.join(PKG, "lib", "obj")
CUDA_HOME = os.environ.get("CUDA_HOME", "/usr/local/cuda")
NVCC = os.path.join(CUDA_HOME, "bin", "nvcc") if os.path.exists(os.path.join(CUDA_HOME, "bin", "nvcc")) else "nvcc"

ARCH = ["-gencode", "arch=compute_100a,code=sm_100a"]
COMMON = ["-std=c++17", "-O3", "-lineinfo", "-Xcompiler", "-fPIC,-Wall,-Wno-unused-function",
          "-I", CSRC, "-I", os.path.join(ROOT, "include")]

LIB_SOURCES = ["frontend.cpp", "device.cu", "kernels.cu", "engine.cpp", "fused.cpp", "io.cpp",
               "capi.cpp", "noalloc.cu", "mlp.cu", "s2p.cu", "vm.cu", "vmprog.cpp"]
MAIN_SOURCES = ["bsim_main.cpp"]
HEADERS = ["frontend.h", "device.h", "engine.h", "fused.h", "io.h", "mlp.h", "s2p.h", "vm.h"]


def _newer(target: str, deps: list[str]) -> bool:
    if not os.path.exists(target):
        return True
    t = os.path.getmtime(target)
    return any(os.path.getmtime(d) > t for d in deps)


def _compile(src: str, force: bool, verbose: bool) -> str:
    path = os.path.join(CSRC, src)
    obj = os.path.join(OBJ, src + ".o")
    deps = [path] + [os.path.join(CSRC, h) for h in HEADERS] + [os.path.join(ROOT, "include", "bsz.h")]
    if force or _newer(obj, deps):
        cmd = [NVCC, *COMMON, *ARCH, "-c", path, "-o", obj]
        if src.endswith(".cpp"):
            cmd = [NVCC, *COMMON, "-x", "cu", *ARCH, "-c", path, "-o", obj]
        if verbose:
            print(" ".join(cmd))
        subprocess.run(cmd, check=True)
    return obj


def build(force: bool = False, verbose: bool = False) -> dict:
    os.makedirs(OBJ, exist_ok=True)
    with cf.ThreadPoolExecutor(max_workers=min(8, os.cpu_count() or 2)) as ex:
        objs = list(ex.map(lambda s: _compile(s, force, verbose), LIB_SOURCES))
        mains = list(ex.map(lambda s: _compile(s, force, verbose), MAIN_SOURCES))
    so = os.path.join(LIB, "libbsz.so")
    # no -lcuda: driver entry points are resolved at run time (fused.cpp);
    # the CUDA runtime and NVRTC are linked statically (the toolkit version
    # this was built with), so whatever libcudart / libnvrtc another library
    # in the process loads (PyTorch ships an older NVRTC, whose ptxas rejects
    # the 256-bit loads and stores of the generated kernels) does not matter.
    link_libs = ["-L", os.path.join(CUDA_HOME, "lib64"), "-lnvrtc_static", "-lnvrtc-builtins_static",
                 "-lnvptxcompiler_static", "-cudart", "static", "-lpthread", "-ldl", "-lrt"]
    if force or _newer(so, objs):
        # -Bsymbolic + --exclude-libs: the library's calls into its static
        # NVRTC bind to its own copy and none of those symbols is exported
        cmd = [NVCC, *ARCH, "-shared", "-o", so, *objs, *link_libs,
               "-Xlinker", "-Bsymbolic", "-Xlinker", "--exclude-libs,ALL",
               "-Xlinker", "-rpath", "-Xlinker", os.path.join(CUDA_HOME, "lib64")]
        if verbose:
            print(" ".join(cmd))
        subprocess.run(cmd, check=True)
    exe = os.path.join(LIB, "bsim_cuda")
    if force or _newer(exe, mains + [so]):
        cmd = [NVCC, *ARCH, "-o", exe, *mains, "-L", LIB, "-lbsz", *link_libs,
               "-Xlinker", "-rpath", "-Xlinker", "$ORIGIN",
               "-Xlinker", "-rpath", "-Xlinker", os.path.join(CUDA_HOME, "lib64")]
        if verbose:
            print(" ".join(cmd))
        subprocess.run(cmd, check=True)
    return {"lib": so, "exe": exe}


def main(argv=None):
    ap = argparse.ArgumentParser()
    ap.add_argument("-v", "--verbose", action="store_true")
    ap.add_argument("--force", action="store_true")
    ap.add_argument("--clean", action="store_true")
    a = ap.parse_args(argv)
    if a.clean and os.path.isdir(LIB):
        shutil.rmtree(LIB)
    out = build(force=a.force, verbose=a.verbose)
    print(out)


if __name__ == "__main__":
    sys.exit(main())
