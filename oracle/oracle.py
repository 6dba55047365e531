"""ctypes binding of the CPU oracle (test infrastructure only).

The oracle is a single-threaded C++ restatement of the reference riv2 encoder path
(reitero_encode + reitero_residual + reitero_dct + reitero_video_common) and of its
decoder (reitero_decode); see riv_oracle.cpp for the file:line citations.  Only the
test suite, ``__graft_entry__.smoke()`` and the CPU-baseline leg of ``bench.py`` may
use it, and only as the checker -- the product never routes through it.
"""
from __future__ import annotations

import ctypes as C
import os
import subprocess

import numpy as np

_HERE = os.path.dirname(os.path.abspath(__file__))
_LIB_PATH = os.path.join(_HERE, "liboracle.so")


class OracleConfig(C.Structure):
    """Mirror of ``oracle_config`` (riv_oracle.h) == reitero_encode::EncoderConfig."""

    _fields_ = [
        ("display_width", C.c_uint32), ("display_height", C.c_uint32),
        ("storage_width", C.c_uint32), ("storage_height", C.c_uint32),
        ("fps", C.c_uint32), ("keyframe_mode", C.c_uint32), ("keyframe_interval", C.c_uint64),
        ("intra_quality", C.c_uint8), ("inter_quality", C.c_uint8), ("search_range", C.c_uint8),
        ("mv_deflate_level", C.c_uint8), ("skip_threshold", C.c_uint8), ("_pad", C.c_uint8 * 3),
        ("me_zero_mv_threshold", C.c_int64), ("me_predictor_threshold", C.c_int64),
        ("rdo_lambda_mult", C.c_double), ("inter_dead_zone", C.c_float), ("_pad2", C.c_uint32),
    ]


def build() -> str:
    """Compile liboracle.so with the committed Makefile (idempotent)."""
    subprocess.run(["make", "-s", "-C", _HERE], check=True)
    return _LIB_PATH


def use_native_build() -> str:
    """Switch this process to the -O3 -march=native build of the same source (compiled here,
    for this host's CPU), for the timed CPU baseline.  Returns the CPU model it targets."""
    import hashlib
    global _LIB_PATH, _lib
    model = cpu_model()
    out = "_ref/liboracle_native_%s.so" % hashlib.sha1(model.encode()).hexdigest()[:10]
    subprocess.run(["make", "-s", "-C", _HERE, "native", "NATIVE_OUT=" + out], check=True)
    _LIB_PATH = os.path.join(_HERE, out)
    _lib = None
    return model


def cpu_model() -> str:
    try:
        with open("/proc/cpuinfo") as f:
            for line in f:
                if line.startswith("model name"):
                    return line.split(":", 1)[1].strip()
    except OSError:
        pass
    return "unknown"


_lib = None


def lib():
    global _lib
    if _lib is None:
        if not os.path.exists(_LIB_PATH):
            build()
        L = C.CDLL(_LIB_PATH)
        P, U8, I8, I16, I64, F32 = (C.c_void_p, C.POINTER(C.c_uint8), C.POINTER(C.c_int8),
                                     C.POINTER(C.c_int16), C.POINTER(C.c_int64), C.POINTER(C.c_float))
        L.oracle_config_default.argtypes = [C.POINTER(OracleConfig), C.c_uint32, C.c_uint32, C.c_uint32]
        L.oracle_enc_new.restype = P
        L.oracle_enc_new.argtypes = [C.POINTER(OracleConfig), C.POINTER(C.c_int)]
        L.oracle_enc_frame_rgb.argtypes = [P, U8, C.c_uint32, C.c_uint32, C.c_uint64]
        L.oracle_enc_frame_yuv.argtypes = [P, U8, U8, U8, C.c_uint64]
        L.oracle_enc_finish.argtypes = [P]
        L.oracle_enc_bytes.restype = C.c_size_t
        L.oracle_enc_bytes.argtypes = [P, C.POINTER(U8)]
        L.oracle_enc_free.argtypes = [P]
        L.oracle_enc_last_type.argtypes = [P]
        for n in ("recon", "recon_pre", "curr", "pred"):
            getattr(L, f"oracle_enc_last_{n}").argtypes = [P, U8, U8, U8]
        L.oracle_enc_last_mvs.argtypes = [P, I8, I8, I64]
        L.oracle_enc_last_side.argtypes = [P, U8]
        L.oracle_enc_last_qsteps.argtypes = [P, F32]
        L.oracle_enc_last_coeffs.argtypes = [P, I16]
        L.oracle_enc_last_bias.argtypes = [P, I8]
        L.oracle_enc_last_stats.argtypes = [P, C.POINTER(C.c_double), C.c_size_t]
        L.oracle_enc_last_stats.restype = C.c_size_t
        L.oracle_enc_last_record.restype = C.c_size_t
        L.oracle_enc_last_record.argtypes = [P, C.POINTER(U8)]
        L.oracle_dec_new.restype = P
        L.oracle_dec_new.argtypes = [U8, C.c_size_t, C.POINTER(C.c_int)]
        L.oracle_dec_next.argtypes = [P, U8, U8, U8]
        L.oracle_dec_dims.argtypes = [P, C.POINTER(C.c_uint32)]
        L.oracle_dec_free.argtypes = [P]
        L.oracle_rgb_to_yuv420.argtypes = [U8, C.c_uint32, C.c_uint32, C.c_uint32, C.c_uint32, U8, U8, U8]
        L.oracle_deblock.argtypes = [U8, U8, U8, C.c_uint32, C.c_uint32, C.c_int, C.c_int, U8]
        L.oracle_deblock_level.argtypes = [C.c_uint8]
        L.oracle_quant_step.restype = C.c_float
        L.oracle_quant_step.argtypes = [C.c_uint8]
        for n in ("oracle_build_predicted", "oracle_reference_build_predicted"):
            getattr(L, n).argtypes = [U8, U8, U8, C.c_uint32, C.c_uint32, I8, U8, U8, U8]
        L.oracle_motion_search.argtypes = [U8, U8, C.c_uint32, C.c_uint32, C.c_uint8, I8, C.c_int64, C.c_int64,
                                           C.c_double, I8, I64]
        for n in ("oracle_sad_int", "oracle_sad_halfpel"):
            getattr(L, n).restype = C.c_int64
            getattr(L, n).argtypes = [U8, U8, C.c_uint32, C.c_uint32, C.c_int, C.c_int, C.c_int, C.c_int,
                                      C.c_int64, C.c_int]
        L.oracle_aq_steps.argtypes = [U8, C.c_uint32, C.c_uint32, C.c_float, F32]
        L.oracle_residual_inter.argtypes = [U8, U8, C.c_uint32, C.c_uint32, U8, F32, C.c_float, I16, U8, U8]
        L.oracle_rdo_lambda.restype = C.c_double
        L.oracle_rdo_lambda.argtypes = [C.c_uint8, C.c_double]
        for n in ("oracle_fdct16_quant", "oracle_fdct8_quant"):
            getattr(L, n).argtypes = [I16, C.c_float, C.c_float, I16]
        for n in ("oracle_idct16_aq", "oracle_idct8_aq"):
            getattr(L, n).argtypes = [I16, C.c_float, I16]
        L.oracle_yuv_to_rgb.argtypes = [C.c_void_p, C.c_void_p, C.c_void_p, C.c_uint32, C.c_uint32, C.c_uint32,
                                         C.c_uint32, C.c_void_p]
        L.oracle_dct_encode.restype = C.c_size_t
        L.oracle_dct_encode.argtypes = [C.c_void_p, C.c_int, C.c_int, C.c_void_p, C.c_size_t]
        L.oracle_dct_decode.argtypes = [C.c_void_p, C.c_size_t, C.c_void_p, C.c_int, C.c_int, C.c_void_p]
        L.oracle_delta_bias.argtypes = [C.c_void_p, C.c_void_p, C.c_uint32, C.c_void_p, C.c_void_p]
        L.oracle_mv_encode.restype = C.c_size_t
        L.oracle_mv_encode.argtypes = [C.c_void_p, C.c_void_p, C.c_int, C.c_void_p, C.c_size_t, C.c_void_p]
        L.oracle_mv_decode.argtypes = [C.c_void_p, C.c_void_p, C.c_void_p, C.c_int, C.c_void_p]
        L.oracle_rans_roundtrip.restype = C.c_size_t
        L.oracle_rans_roundtrip.argtypes = [U8, U8, C.c_size_t, U8, U8, C.c_size_t]
        _lib = L
    return _lib


def _p(a: np.ndarray, ct):
    assert a.flags["C_CONTIGUOUS"]
    return a.ctypes.data_as(C.POINTER(ct))


def u8(a):
    return _p(a, C.c_uint8)


def i8(a):
    return _p(a, C.c_int8)


def i16(a):
    return _p(a, C.c_int16)


def default_config(w: int, h: int, fps: int = 30) -> OracleConfig:
    c = OracleConfig()
    lib().oracle_config_default(C.byref(c), w, h, fps)
    return c


class Frames:
    """YUV 4:2:0 planes of one frame."""

    def __init__(self, w: int, h: int):
        self.w, self.h = w, h
        self.y = np.zeros((h, w), np.uint8)
        self.u = np.zeros((h // 2, w // 2), np.uint8)
        self.v = np.zeros((h // 2, w // 2), np.uint8)

    def ptrs(self):
        return u8(self.y), u8(self.u), u8(self.v)

    def equal(self, o) -> bool:
        return (np.array_equal(self.y, o.y) and np.array_equal(self.u, o.u) and np.array_equal(self.v, o.v))


# oracle_enc_last_stats's layout (riv_oracle.h): (field, width)
STATS_FIELDS = (
    ("frame_type", 1), ("total_bytes", 1), ("mv_bytes", 1), ("mv_raw_bytes", 1), ("residual_bytes", 1),
    ("blocks_total", 1), ("blocks_skipped", 1), ("mv_zero_delta_blocks", 1), ("mv_mode_counts", 7),
    ("mv_new_zero_pre_bias", 1), ("mv_new_zero_post_bias", 1), ("mv_new_zero_axes_x", 1), ("mv_new_zero_axes_y", 1),
    ("mv_new_base_counts", 5), ("mv_new_best_ref_counts", 5), ("mv_new_best_ref_l1_saved_sum", 1),
    ("mv_new_blocks", 1), ("mv_new_delta_count", 1), ("mv_new_delta_mag_sum", 1), ("mv_new_delta_mag_sq_sum", 1),
    ("mv_class_histogram", 11), ("mv_bias_dx", 1), ("mv_bias_dy", 1), ("mv_candidate_unique_total", 1),
    ("mv_candidate_unique_samples", 1), ("mv_candidate_unique_min", 1), ("mv_candidate_unique_max", 1),
    ("mv_match_source_counts", 6), ("mv_match_nonzero_blocks", 1), ("mv_match_any_spatial", 1),
    ("mv_match_any_temporal", 1), ("resi_raw", 1), ("resi_rans", 1), ("rdo_lambda", 1), ("rdo_blocks_evaluated", 1),
    ("rdo_blocks_selected_skip", 1), ("rdo_forced_fractional", 1), ("rdo_forced_threshold", 1),
    ("rdo_forced_disabled", 1), ("rdo_avg_skip_cost", 1), ("rdo_avg_coded_cost", 1),
)
STATS_N = sum(w for _, w in STATS_FIELDS)


class OracleEncoder:
    """Oracle encoder: Encoder::new / encode_frame / finish over an in-memory writer."""

    def __init__(self, cfg: OracleConfig):
        st = C.c_int(0)
        self.cfg = cfg
        self.h = lib().oracle_enc_new(C.byref(cfg), C.byref(st))
        if not self.h:
            raise ValueError(f"oracle config rejected (status {st.value})")
        self.sw, self.sh = cfg.storage_width, cfg.storage_height
        self.mbs = (self.sw // 16) * (self.sh // 16)

    def encode_rgb(self, rgb: np.ndarray, ts: int) -> int:
        rgb = np.ascontiguousarray(rgb, dtype=np.uint8)
        return lib().oracle_enc_frame_rgb(self.h, u8(rgb), self.cfg.display_width, self.cfg.display_height, ts)

    def encode_yuv(self, f: Frames, ts: int) -> int:
        return lib().oracle_enc_frame_yuv(self.h, *f.ptrs(), ts)

    def finish(self) -> bytes:
        lib().oracle_enc_finish(self.h)
        return self.bytes()

    def bytes(self) -> bytes:
        p = C.POINTER(C.c_uint8)()
        n = lib().oracle_enc_bytes(self.h, C.byref(p))
        return C.string_at(p, n)

    def last_record(self) -> bytes:
        p = C.POINTER(C.c_uint8)()
        n = lib().oracle_enc_last_record(self.h, C.byref(p))
        return C.string_at(p, n)

    def last(self, what: str) -> Frames:
        f = Frames(self.sw, self.sh)
        getattr(lib(), f"oracle_enc_last_{what}")(self.h, *f.ptrs())
        return f

    def last_type(self) -> int:
        return lib().oracle_enc_last_type(self.h)

    def last_mvs(self):
        raw = np.zeros((self.mbs, 4), np.int8)
        coded = np.zeros((self.mbs, 4), np.int8)
        sad = np.zeros(self.mbs, np.int64)
        lib().oracle_enc_last_mvs(self.h, i8(raw), i8(coded), _p(sad, C.c_int64))
        return raw, coded, sad

    def last_side(self) -> np.ndarray:
        s = np.zeros((self.mbs, 8), np.uint8)
        lib().oracle_enc_last_side(self.h, u8(s))
        return s

    def last_qsteps(self) -> np.ndarray:
        q = np.zeros(self.mbs, np.float32)
        lib().oracle_enc_last_qsteps(self.h, _p(q, C.c_float))
        return q

    def last_coeffs(self) -> np.ndarray:
        c = np.zeros((self.mbs, 384), np.int16)
        lib().oracle_enc_last_coeffs(self.h, i16(c))
        return c

    def last_bias(self):
        b = np.zeros(2, np.int8)
        lib().oracle_enc_last_bias(self.h, i8(b))
        return int(b[0]), int(b[1])

    def last_stats(self) -> dict:
        """EncodeFrameStats of the last frame (enc/encoder.rs:58-124), arrays as tuples,
        Options as None."""
        v = np.zeros(STATS_N, np.float64)
        got = lib().oracle_enc_last_stats(self.h, v.ctypes.data_as(C.POINTER(C.c_double)), STATS_N)
        assert got == STATS_N, got
        out, k = {}, 0
        for name, width in STATS_FIELDS:
            vals = v[k:k + width]
            out[name] = tuple(vals.tolist()) if width > 1 else float(vals[0])
            k += width
        for name in ("resi_raw", "resi_rans"):
            if out[name] < 0:
                out[name] = None
        return out

    def close(self):
        if self.h:
            lib().oracle_enc_free(self.h)
            self.h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass


class OracleDecoder:
    def __init__(self, stream: bytes):
        self._buf = np.frombuffer(stream, np.uint8).copy()
        st = C.c_int(0)
        self.h = lib().oracle_dec_new(u8(self._buf), len(stream), C.byref(st))
        if not self.h:
            raise ValueError("bad .riv header")
        d = (C.c_uint32 * 6)()
        lib().oracle_dec_dims(self.h, d)
        self.dw, self.dh, self.sw, self.sh, self.fps, self.frame_count = list(d)

    def next(self):
        f = Frames(self.sw, self.sh)
        t = lib().oracle_dec_next(self.h, *f.ptrs())
        return t, f

    def close(self):
        if self.h:
            lib().oracle_dec_free(self.h)
            self.h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass


def yuv_to_rgb(f: Frames, dw: int, dh: int) -> np.ndarray:
    """Decoder output: the frame's YUV 4:2:0 planes to display-size (dh, dw, 3) RGB24."""
    out = np.zeros((dh, dw, 3), np.uint8)
    y, u, v = (np.ascontiguousarray(p, dtype=np.uint8) for p in (f.y, f.u, f.v))
    lib().oracle_yuv_to_rgb(y.ctypes.data, u.ctypes.data, v.ctypes.data, f.w, f.h, dw, dh, out.ctypes.data)
    return out


def dct_encode(blocks: np.ndarray, intra: bool) -> bytes:
    """The oracle's DCT-coefficient coder of one frame on dense (n, 384) int16 blocks.
    Raises ValueError where the reference encoder panics (a magnitude class above 13)."""
    b = np.ascontiguousarray(blocks, dtype=np.int16)
    n = b.shape[0]
    size = lib().oracle_dct_encode(b.ctypes.data, n, int(intra), None, 0)
    if size == C.c_size_t(-1).value:
        raise ValueError("magnitude class above 13: the reference encoder panics")
    out = np.zeros(max(size, 1), np.uint8)
    lib().oracle_dct_encode(b.ctypes.data, n, int(intra), out.ctypes.data, size)
    return out[:size].tobytes()


def dct_decode(data: bytes, coded: np.ndarray, intra: bool):
    """The oracle's coefficient decoder of one frame: (dense (n, 384) int16 blocks, ok), ok
    False where the stream is malformed (the reference decoder panics there)."""
    c = np.ascontiguousarray(coded, dtype=np.uint8)
    out = np.zeros((c.size, 384), np.int16)
    buf = np.frombuffer(data, np.uint8) if len(data) else np.zeros(1, np.uint8)
    st = lib().oracle_dct_decode(buf.ctypes.data, len(data), c.ctypes.data, c.size, int(intra), out.ctypes.data)
    return out, st == 0


def delta_bias(dx: np.ndarray, dy: np.ndarray):
    """The oracle's compute_delta_bias_for_new over NEW-block raw deltas: (bias x, bias y)."""
    x = np.ascontiguousarray(dx, dtype=np.int8)
    y = np.ascontiguousarray(dy, dtype=np.int8)
    bx, by = C.c_int8(0), C.c_int8(0)
    lib().oracle_delta_bias(x.ctypes.data, y.ctypes.data, x.size, C.byref(bx), C.byref(by))
    return bx.value, by.value


def mv_encode(blocks: np.ndarray, dims) -> list:
    """The oracle's MV coder over a sequence of frames, one coder throughout: blocks is
    (total blocks, 7) uint8 (mode, NEW base, dx, dy, subpel x, subpel y, skip), dims the
    (bw, bh) of each frame.  Returns each frame's bytes; raises ValueError where the reference
    encoder panics (a NEW block with a raw -1/2 subpel)."""
    b = np.ascontiguousarray(blocks, dtype=np.uint8)
    d = np.ascontiguousarray(np.asarray(dims, dtype=np.uint32).reshape(-1))
    nf = d.size // 2
    fl = np.zeros(max(nf, 1), np.uint32)
    if b.ndim != 2 or b.shape[1] != 7 or b.shape[0] != int(sum(int(d[2 * f]) * int(d[2 * f + 1]) for f in range(nf))):
        raise ValueError("blocks must be (sum of bw * bh over the frames, 7)")
    total = lib().oracle_mv_encode(b.ctypes.data, d.ctypes.data, nf, None, 0, fl.ctypes.data)
    if total == C.c_size_t(-1).value:
        raise ValueError("raw -0.5 subpixel: the reference encoder panics")
    out = np.zeros(max(total, 1), np.uint8)
    lib().oracle_mv_encode(b.ctypes.data, d.ctypes.data, nf, out.ctypes.data, total, fl.ctypes.data)
    frames, pos = [], 0
    for f in range(nf):
        frames.append(out[pos:pos + int(fl[f])].tobytes())
        pos += int(fl[f])
    return frames


def mv_decode(frames: list, dims):
    """Inverse of mv_encode with a fresh coder: ((total blocks, 7) uint8, ok)."""
    d = np.ascontiguousarray(np.asarray(dims, dtype=np.uint32).reshape(-1))
    nf = d.size // 2
    fl = np.array([len(f) for f in frames] or [0], np.uint32)
    data = np.frombuffer(b"".join(frames) or b"\0", np.uint8)
    n = int(sum(int(d[2 * f]) * int(d[2 * f + 1]) for f in range(nf)))
    out = np.zeros((max(n, 1), 7), np.uint8)
    st = lib().oracle_mv_decode(data.ctypes.data, fl.ctypes.data, d.ctypes.data, nf, out.ctypes.data)
    return out[:n], st == 0


def rgb_to_yuv(rgb: np.ndarray, dw: int, dh: int, sw: int, sh: int) -> Frames:
    f = Frames(sw, sh)
    rgb = np.ascontiguousarray(rgb, dtype=np.uint8)
    lib().oracle_rgb_to_yuv420(u8(rgb), dw, dh, sw, sh, *f.ptrs())
    return f


def deblock(f: Frames, level: int, intra: bool, mask=None) -> Frames:
    o = Frames(f.w, f.h)
    o.y[:], o.u[:], o.v[:] = f.y, f.u, f.v
    m = None if mask is None else u8(np.ascontiguousarray(mask, dtype=np.uint8))
    lib().oracle_deblock(*o.ptrs(), f.w, f.h, level, int(intra), m)
    return o


def build_predicted(prev: Frames, mvs4: np.ndarray, reference: bool = False) -> Frames:
    o = Frames(prev.w, prev.h)
    m = np.ascontiguousarray(mvs4, dtype=np.int8)
    fn = lib().oracle_reference_build_predicted if reference else lib().oracle_build_predicted
    fn(*prev.ptrs(), prev.w, prev.h, i8(m), *o.ptrs())
    return o


def aq_steps(pred_y: np.ndarray, w: int, h: int, base: float) -> np.ndarray:
    """compute_aq_quant_steps (res/residual.rs:116-167) on a luma prediction plane."""
    out = np.zeros((w // 16) * (h // 16), np.float32)
    lib().oracle_aq_steps(u8(np.ascontiguousarray(pred_y, dtype=np.uint8)), w, h, base, _p(out, C.c_float))
    return out


def residual_inter(cur: np.ndarray, pred: np.ndarray, w: int, h: int, skip: np.ndarray, qs: np.ndarray, dz: float):
    """encode_inter's residual, transforms, quantisation and reconstruction (res/residual.rs:520-752)
    for given AQ steps: returns (coefficients n x 384, optimized skip n, reconstruction planes)."""
    n = (w // 16) * (h // 16)
    co = np.zeros((n, 384), np.int16)
    os_ = np.zeros(n, np.uint8)
    rec = np.zeros(w * h * 3 // 2, np.uint8)
    lib().oracle_residual_inter(u8(np.ascontiguousarray(cur, np.uint8)), u8(np.ascontiguousarray(pred, np.uint8)),
                                w, h, u8(np.ascontiguousarray(skip, np.uint8)),
                                _p(np.ascontiguousarray(qs, np.float32), C.c_float), dz, i16(co), u8(os_), u8(rec))
    return co, os_, rec
