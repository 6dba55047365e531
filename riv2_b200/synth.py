"""Seeded synthetic RGB24 clips (ctypes binding of csrc/synth.cpp).

Stands in for the public sequences the reference benchmarks on; see synth.cpp for the
scene model.  Presets: ``cif`` (352x288, 8 rects), ``720p``, ``1080p`` (16 rects, sides
64-384, v +-16, lattice 16, pan +-4) and ``4k`` (24 rects, v +-48, sigma 4).
"""
from __future__ import annotations

import ctypes as C

import numpy as np

from ._native import load_synth


class SynthParams(C.Structure):
    _fields_ = [
        ("width", C.c_uint32), ("height", C.c_uint32), ("n_rects", C.c_uint32), ("side_min", C.c_uint32),
        ("side_max", C.c_uint32), ("lattice", C.c_uint32), ("vmax", C.c_double), ("pan_max", C.c_double),
        ("sigma", C.c_double), ("seed", C.c_uint32), ("clip", C.c_uint32),
    ]


def _lib():
    L = load_synth()
    if not getattr(L, "_riv_typed", False):
        L.riv_synth_preset.argtypes = [C.POINTER(SynthParams), C.c_char_p, C.c_uint32, C.c_uint32]
        L.riv_synth_new.restype = C.c_void_p
        L.riv_synth_new.argtypes = [C.POINTER(SynthParams)]
        L.riv_synth_frame.argtypes = [C.c_void_p, C.c_uint32, C.POINTER(C.c_uint8)]
        L.riv_synth_free.argtypes = [C.c_void_p]
        L._riv_typed = True
    return L


class SynthClip:
    """A deterministic synthetic clip; ``frame(t)`` returns an (H, W, 3) uint8 array."""

    def __init__(self, preset: str = "cif", seed: int = 1, clip: int = 0, width: int | None = None,
                 height: int | None = None):
        L = _lib()
        self.params = SynthParams()
        L.riv_synth_preset(C.byref(self.params), preset.encode(), seed, clip)
        if width:
            self.params.width = width
        if height:
            self.params.height = height
        self.h = L.riv_synth_new(C.byref(self.params))
        if not self.h:
            raise ValueError("invalid synth parameters")
        self.width, self.height = self.params.width, self.params.height

    def frame(self, t: int, out: np.ndarray | None = None) -> np.ndarray:
        if out is None:
            out = np.empty((self.height, self.width, 3), np.uint8)
        assert out.flags["C_CONTIGUOUS"] and out.nbytes == self.width * self.height * 3
        _lib().riv_synth_frame(self.h, t, out.ctypes.data_as(C.POINTER(C.c_uint8)))
        return out

    def frames(self, n: int) -> np.ndarray:
        arr = np.empty((n, self.height, self.width, 3), np.uint8)
        for t in range(n):
            self.frame(t, arr[t])
        return arr

    def __del__(self):
        try:
            if self.h:
                _lib().riv_synth_free(self.h)
                self.h = None
        except Exception:
            pass
