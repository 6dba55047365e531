"""In-tree build of the native libraries (no JIT cache, so the .so files travel with the repo).

* ``_lib/libriv2_b200.so``  -- sm_100a kernels + C-ABI host encoder (nvcc, -gencode
  arch=compute_100a,code=sm_100a).
* ``_lib/libriv_synth.so``  -- host-only synthetic clip generator.
* ``_lib/libm_fixups.bin``  -- glibc logf/exp2f fix-up tables (generated by running glibc).
"""
from __future__ import annotations

import os
import shutil
import subprocess

from ._native import LIB_DIR, PKG_DIR

CSRC = os.path.join(PKG_DIR, "csrc")
REPO = os.path.dirname(PKG_DIR)
NVCC = shutil.which("nvcc") or "/usr/local/cuda/bin/nvcc"
ARCH = ["-gencode", "arch=compute_100a,code=sm_100a"]
CUDA_SOURCES = ["riv_kernels.cu", "riv_nn.cu", "riv_host.cpp", "riv_entropy.cpp"]
HOST_FLAGS = "-fPIC,-fwrapv,-ffp-contract=off,-fno-fast-math,-O2"


def _stale(target: str, deps: list[str]) -> bool:
    if not os.path.exists(target):
        return True
    t = os.path.getmtime(target)
    return any(os.path.getmtime(d) > t for d in deps)


def _run(cmd: list[str]) -> None:
    r = subprocess.run(cmd, capture_output=True, text=True)
    if r.returncode != 0:
        raise RuntimeError(f"build step failed: {' '.join(cmd)}\n{r.stdout}\n{r.stderr}")


def build_cuda(force: bool = False) -> str:
    os.makedirs(LIB_DIR, exist_ok=True)
    out = os.path.join(LIB_DIR, "libriv2_b200.so")
    deps = [os.path.join(CSRC, f) for f in os.listdir(CSRC)] + [os.path.join(REPO, "include", h) for h in ("riv_gpu.h", "riv_nn.h")]
    if not force and not _stale(out, deps):
        return out
    objs = []
    bdir = os.path.join(LIB_DIR, "_obj")
    os.makedirs(bdir, exist_ok=True)
    for src in CUDA_SOURCES:
        obj = os.path.join(bdir, src + ".o")
        cmd = [NVCC, *ARCH, "-lineinfo", "-O3", "-std=c++17", "-Xcompiler", HOST_FLAGS, "-fmad=false",
               "-I", os.path.join(REPO, "include"), "-c", os.path.join(CSRC, src), "-o", obj]
        if src.endswith(".cpp"):
            cmd[1:1] = ["-x", "cu"] if src == "riv_host.cpp" else []
        _run(cmd)
        objs.append(obj)
    _run([NVCC, *ARCH, "-shared", "-o", out, *objs, "-lcudart", "-ldl", "-lpthread"])
    return out


def build_synth(force: bool = False) -> str:
    os.makedirs(LIB_DIR, exist_ok=True)
    out = os.path.join(LIB_DIR, "libriv_synth.so")
    src = os.path.join(CSRC, "synth.cpp")
    if force or _stale(out, [src, os.path.join(CSRC, "riv_synth.h")]):
        _run(["g++", "-O2", "-fPIC", "-std=c++17", "-fopenmp", "-shared", "-I", CSRC, "-o", out, src])
    return out


def build_libm_fixups(force: bool = False) -> str:
    os.makedirs(LIB_DIR, exist_ok=True)
    out = os.path.join(LIB_DIR, "libm_fixups.bin")
    src = os.path.join(CSRC, "gen_libm_fixups.cpp")
    if force or _stale(out, [src]):
        exe = os.path.join(LIB_DIR, "_obj", "gen_libm_fixups")
        os.makedirs(os.path.dirname(exe), exist_ok=True)
        _run(["g++", "-O2", "-std=c++17", "-fopenmp", "-ffp-contract=off", "-o", exe, src, "-lm"])
        _run([exe, out])
    return out


def build_all(force: bool = False) -> None:
    build_synth(force)
    build_libm_fixups(force)
    build_cuda(force)
