"""Locating and loading the in-tree native libraries.

The CUDA library (``_lib/libriv2_b200.so``) and the host-only synthetic-clip generator
(``_lib/libriv_synth.so``) are built in-tree by ``riv2_b200.build.build_all()``.  There is
no fallback: if a library is missing, loading raises.
"""
from __future__ import annotations

import ctypes as C
import os

PKG_DIR = os.path.dirname(os.path.abspath(__file__))
LIB_DIR = os.path.join(PKG_DIR, "_lib")
CUDA_LIB = os.path.join(LIB_DIR, "libriv2_b200.so")
SYNTH_LIB = os.path.join(LIB_DIR, "libriv_synth.so")

_cache: dict[str, C.CDLL] = {}


def _load(path: str) -> C.CDLL:
    if path not in _cache:
        if not os.path.exists(path):
            raise RuntimeError(f"native library {path} is missing; run riv2_b200.build.build_all() first")
        _cache[path] = C.CDLL(path)
    return _cache[path]


def load_cuda() -> C.CDLL:
    return _load(CUDA_LIB)


def load_synth() -> C.CDLL:
    return _load(SYNTH_LIB)
