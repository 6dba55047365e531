"""Multi-clip encoding over the C ABI (riv_batch_* in include/riv_gpu.h).

The reference encodes one stream per ``Encoder``; a ``Batch`` holds many independent clips
(each its own ``EncoderConfig`` and writer, any mix of sizes) and encodes them one step at a
time, one frame per clip per step, with one GPU launch per stage over every clip of the
step.  Every clip's stream is byte-identical to a single-clip ``Encoder`` run on the same
frames::

    b = Batch.new([cfg_a, cfg_b], [VecWriter(), VecWriter()])
    b.encode_step([rgb_a, None])        # None: that clip has no frame in this step
    b.encode_step([rgb_a2, rgb_b])
    b.finish()
    streams = [w.into_inner() for w in b.writers]
"""
from __future__ import annotations

import ctypes as C
from typing import Optional, Sequence

import numpy as np

from . import encoder as E

U8P = C.POINTER(C.c_uint8)
STAGES = ["convert", "sad_table", "search", "predict", "aq_mean", "residual", "deblock", "scan", "pack", "step"]


class RivBatchTune(C.Structure):
    _fields_ = [("search_rows_pct", C.c_int32), ("res_mbs", C.c_int32), ("db_tw", C.c_int32),
                ("sad_table", C.c_int32)]


def _lib() -> C.CDLL:
    L = E.lib()
    if getattr(L, "_riv_batch_typed", False):
        return L
    P = C.c_void_p
    L.riv_batch_new.argtypes = [C.POINTER(E.RivConfig), C.POINTER(E.RivWriterVtable), C.c_uint32, C.POINTER(P)]
    L.riv_batch_encode.argtypes = [P, C.POINTER(C.c_void_p), C.POINTER(C.c_uint64)]
    L.riv_batch_encode_device.argtypes = [P, C.POINTER(C.c_void_p), C.POINTER(C.c_uint64)]
    L.riv_batch_finish.argtypes = [P]
    L.riv_batch_free.argtypes = [P]
    L.riv_batch_last_error.restype = C.c_char_p
    L.riv_batch_last_error.argtypes = [P]
    L.riv_batch_set_tune.argtypes = [P, C.POINTER(RivBatchTune)]
    L.riv_batch_get_tune.argtypes = [P, C.POINTER(RivBatchTune), C.POINTER(C.c_int)]
    L.riv_batch_counters.argtypes = [P, C.POINTER(C.c_uint64), C.POINTER(C.c_double)]
    L.riv_batch_last_recon.argtypes = [P, C.c_uint32, U8P, U8P, U8P]
    L.riv_batch_clip_counters.argtypes = [P, C.c_uint32, C.POINTER(C.c_uint64), C.POINTER(C.c_double)]
    L.riv_batch_host_times.argtypes = [P, C.POINTER(C.c_double)]
    L._riv_batch_typed = True
    return L


class Batch:
    """Many clips encoded together; ``configs[i]`` / ``writers[i]`` describe clip i."""

    def __init__(self, configs, writers, h, bridges):
        self.configs = list(configs)
        self.writers = list(writers)
        self._h = h
        self._bridges = bridges

    @staticmethod
    def new(configs: Sequence[E.EncoderConfig], writers: Sequence[E.VideoWriter]) -> "Batch":
        if len(configs) != len(writers) or not configs:
            raise E.InvalidConfig("one writer per clip, at least one clip")
        L = _lib()
        n = len(configs)
        cfgs = (E.RivConfig * n)()
        vts = (E.RivWriterVtable * n)()
        bridges = []
        for i, (c, w) in enumerate(zip(configs, writers)):
            c.validate()
            cfgs[i] = c.to_c()
            if isinstance(w, E.VecWriter):
                vts[i] = w.vtable()
            else:
                br = E._PyWriterBridge(w)
                bridges.append(br)
                vts[i] = br.vtable()
        h = C.c_void_p()
        st = L.riv_batch_new(cfgs, vts, n, C.byref(h))
        if st != 0:
            raise E._ERRORS.get(st, E.EncodeError)(f"riv_batch_new failed (status {st})")
        return Batch(configs, writers, h, bridges)

    def _check(self, st: int) -> None:
        if st != 0:
            msg = _lib().riv_batch_last_error(self._h).decode(errors="replace")
            raise E._ERRORS.get(st, E.EncodeError)(msg)

    def encode_step(self, frames: Sequence[Optional[np.ndarray]], timestamps: Optional[Sequence[int]] = None) -> None:
        """One step: ``frames[i]`` = clip i's display-size RGB24 frame (host array) or None."""
        n = len(self.configs)
        if len(frames) != n:
            raise E.FrameError(f"one entry per clip: expected {n}, got {len(frames)}")
        ptrs = (C.c_void_p * n)()
        ts = (C.c_uint64 * n)()
        keep = []
        for i, f in enumerate(frames):
            if f is None:
                continue
            c = self.configs[i]
            a = np.ascontiguousarray(f, dtype=np.uint8).reshape(-1)
            if a.size != c.display_width * c.display_height * 3:
                raise E.FrameError(f"clip {i}: expected {c.display_width * c.display_height * 3} bytes, got {a.size}")
            keep.append(a)
            ptrs[i] = a.ctypes.data
            ts[i] = int(timestamps[i]) if timestamps is not None else 0
        self._check(_lib().riv_batch_encode(self._h, ptrs, ts))

    def encode_step_device(self, ptrs: Sequence[int], timestamps: Sequence[int]) -> None:
        """One step with frames already in device memory (0 = clip has no frame)."""
        n = len(self.configs)
        p = (C.c_void_p * n)(*[x if x else None for x in ptrs])
        ts = (C.c_uint64 * n)(*[int(t) for t in timestamps])
        self._check(_lib().riv_batch_encode_device(self._h, p, ts))

    def finish(self) -> None:
        self._check(_lib().riv_batch_finish(self._h))

    def set_tune(self, search_rows_pct: int, res_mbs: int, db_tw: int, sad_table: int = 1) -> None:
        t = RivBatchTune(search_rows_pct, res_mbs, db_tw, sad_table)
        self._check(_lib().riv_batch_set_tune(self._h, C.byref(t)))

    def tune(self) -> dict:
        t = RivBatchTune()
        s = C.c_int()
        self._check(_lib().riv_batch_get_tune(self._h, C.byref(t), C.byref(s)))
        return {"search_rows_pct": t.search_rows_pct, "res_mbs": t.res_mbs, "db_tw": t.db_tw,
                "sad_table": t.sad_table, "state": {0: "tuning", 1: "autotuned", 2: "fixed"}[s.value]}

    def counters(self) -> dict:
        c = (C.c_uint64 * 7)()
        us = (C.c_double * 10)()
        self._check(_lib().riv_batch_counters(self._h, c, us))
        return {"steps": c[0], "frames": c[1], "mbs": c[2], "launches": c[3], "timed_steps": c[4], "h2d_bytes": c[5],
                "d2h_bytes": c[6], "stage_us": dict(zip(STAGES, list(us)))}

    def host_times(self) -> dict:
        """Cumulative host milliseconds of the batch's own thread."""
        ms = (C.c_double * 5)()
        self._check(_lib().riv_batch_host_times(self._h, ms))
        return dict(zip(["making_room", "launch", "copies_back", "advance", "finish"], list(ms)))

    def clip_counters(self, i: int) -> dict:
        n = C.c_uint64()
        hm = (C.c_double * 6)()
        self._check(_lib().riv_batch_clip_counters(self._h, i, C.byref(n), hm))
        return {"frames_written": n.value, "host_ms": list(hm)}

    def last_recon(self, i: int):
        c = self.configs[i]
        sw, sh = c.storage_width, c.storage_height
        y = np.empty((sh, sw), np.uint8)
        u = np.empty((sh // 2, sw // 2), np.uint8)
        v = np.empty((sh // 2, sw // 2), np.uint8)
        self._check(_lib().riv_batch_last_recon(self._h, i, E._u8(y), E._u8(u), E._u8(v)))
        return y, u, v

    def close(self) -> None:
        if self._h:
            _lib().riv_batch_free(self._h)
            self._h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass
