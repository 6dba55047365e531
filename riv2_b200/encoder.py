"""Python mirror of reitero_encode's public API over the C ABI (include/riv_gpu.h).

Same names, argument meaning and error behaviour as the reference crate
(reitero_video/reitero_encode/src/{config,encoder,writer,error}.rs):

    cfg = EncoderConfig.new(1920, 1080, 50).with_intra_quality(85).with_inter_quality(80)
    enc = Encoder.new(cfg, VecWriter())
    enc.encode_frame(Frame(rgb_bytes, 1920, 1080, timestamp_ms))
    enc.finish()
    data = enc.writer.into_inner()

The encoder runs on the GPU; there is no CPU fallback -- constructing an Encoder without
the CUDA library or without a device raises.
"""
from __future__ import annotations

import ctypes as C
import dataclasses
from typing import Optional

import numpy as np

from ._native import load_cuda

# ---------------------------------------------------------------------------------------
# Errors (enc/error.rs:4-20)
# ---------------------------------------------------------------------------------------


class EncodeError(Exception):
    status = 3


class IoError(EncodeError):
    status = 1


class InvalidConfig(EncodeError):
    status = 2


class EncodingFailed(EncodeError):
    status = 3


class UnsupportedCodec(EncodeError):
    status = 4


class FrameError(EncodeError):
    status = 5


class CudaError(EncodeError):
    status = 6


class DeviceTimeout(EncodeError):
    status = 7


_ERRORS = {1: IoError, 2: InvalidConfig, 3: EncodingFailed, 4: UnsupportedCodec, 5: FrameError, 6: CudaError,
           7: DeviceTimeout}

# ---------------------------------------------------------------------------------------
# C structures
# ---------------------------------------------------------------------------------------


class RivConfig(C.Structure):
    _fields_ = [
        ("display_width", C.c_uint32), ("display_height", C.c_uint32),
        ("storage_width", C.c_uint32), ("storage_height", C.c_uint32),
        ("fps", C.c_uint32), ("keyframe_mode", C.c_uint32), ("keyframe_interval", C.c_uint64),
        ("intra_quality", C.c_uint8), ("inter_quality", C.c_uint8), ("search_range", C.c_uint8),
        ("mv_deflate_level", C.c_uint8), ("skip_threshold", C.c_uint8), ("_pad", C.c_uint8 * 3),
        ("me_zero_mv_threshold", C.c_int64), ("me_predictor_threshold", C.c_int64),
        ("rdo_lambda_mult", C.c_double), ("inter_dead_zone", C.c_float),
        ("device", C.c_int32), ("pipeline_depth", C.c_uint32), ("entropy_threads", C.c_uint32),
        ("encode_form", C.c_uint32), ("proposal_margin", C.c_uint32),
    ]


WRITE_FN = C.CFUNCTYPE(C.c_int, C.c_void_p, C.POINTER(C.c_uint8), C.c_size_t)
POS_FN = C.CFUNCTYPE(C.c_uint64, C.c_void_p)
SEEK_FN = C.CFUNCTYPE(C.c_int, C.c_void_p, C.c_uint64)
FLUSH_FN = C.CFUNCTYPE(C.c_int, C.c_void_p)


class RivWriterVtable(C.Structure):
    _fields_ = [("write", WRITE_FN), ("position", POS_FN), ("seek", SEEK_FN), ("flush", FLUSH_FN),
                ("user", C.c_void_p)]


class RivFrameStats(C.Structure):
    _fields_ = [
        ("frame_index", C.c_uint64), ("timestamp_ms", C.c_uint64), ("frame_type", C.c_uint32),
        ("total_bytes", C.c_uint32), ("mv_bytes", C.c_uint32), ("mv_raw_bytes", C.c_uint32),
        ("residual_bytes", C.c_uint32), ("storage_width", C.c_uint32), ("storage_height", C.c_uint32),
        ("blocks_total", C.c_uint32), ("blocks_skipped", C.c_uint32), ("mv_zero_delta_blocks", C.c_uint32),
        ("mv_mode_counts", C.c_uint32 * 7), ("mv_new_zero_pre_bias", C.c_uint32), ("mv_new_zero_post_bias", C.c_uint32),
        ("mv_new_zero_axes_x", C.c_uint32), ("mv_new_zero_axes_y", C.c_uint32), ("mv_new_base_counts", C.c_uint32 * 5),
        ("mv_new_best_ref_counts", C.c_uint32 * 5), ("mv_new_best_ref_l1_saved_sum", C.c_uint64),
        ("mv_new_blocks", C.c_uint32), ("mv_new_delta_count", C.c_uint32), ("mv_new_delta_mag_sum", C.c_double),
        ("mv_new_delta_mag_sq_sum", C.c_double), ("mv_class_histogram", C.c_uint64 * 11),
        ("mv_bias_dx", C.c_int32), ("mv_bias_dy", C.c_int32), ("mv_candidate_unique_total", C.c_uint32),
        ("mv_candidate_unique_samples", C.c_uint32), ("mv_candidate_unique_min", C.c_uint32),
        ("mv_candidate_unique_max", C.c_uint32), ("mv_match_source_counts", C.c_uint32 * 6),
        ("mv_match_nonzero_blocks", C.c_uint32), ("mv_match_any_spatial", C.c_uint32),
        ("mv_match_any_temporal", C.c_uint32), ("resi_raw", C.c_int64), ("resi_rans", C.c_int64),
        ("rdo_lambda", C.c_double), ("rdo_blocks_evaluated", C.c_uint32), ("rdo_blocks_selected_skip", C.c_uint32),
        ("rdo_forced_fractional", C.c_uint32), ("rdo_forced_threshold", C.c_uint32),
        ("rdo_forced_disabled", C.c_uint32), ("rdo_avg_skip_cost", C.c_double), ("rdo_avg_coded_cost", C.c_double),
    ]


# Every symbol include/riv_gpu.h declares (checked by the CPU test suite).
EXPORTED_SYMBOLS = (
    "riv_config_default", "riv_encoder_new", "riv_encode_frame", "riv_encode_frame_device", "riv_encode_frame_yuv",
    "riv_finish", "riv_encoder_free", "riv_last_error", "riv_frame_count", "riv_last_recon", "riv_last_kernel_times",
    "riv_memwriter_new", "riv_memwriter_vtable", "riv_memwriter_size", "riv_memwriter_data", "riv_memwriter_free",
    "riv_stage_rgb_to_yuv", "riv_stage_deblock", "riv_stage_libm", "riv_libm_fixup_counts", "riv_dct_tables",
    "riv_debug_frame_state", "riv_counters", "riv_host_times", "riv_stage_deblock_noalloc",
    "riv_decoder_new", "riv_decoder_info", "riv_decode_frame_yuv", "riv_decode_frame_rgb", "riv_decoder_current_frame",
    "riv_decoder_last_error", "riv_decoder_free", "riv_test_dct_encode", "riv_test_dct_decode", "riv_test_mv_encode",
    "riv_test_mv_decode", "riv_test_delta_bias", "riv_test_worker_queue", "riv_test_libm_range",
    "riv_stage_predict", "riv_stage_residual", "riv_test_wait_expiry", "riv_encoder_set_proposal",
    "riv_learned_counters", "riv_test_mv_encode_threads",
    "riv_batch_new", "riv_batch_encode", "riv_batch_encode_device", "riv_batch_finish", "riv_batch_free",
    "riv_batch_last_error", "riv_batch_set_tune", "riv_batch_get_tune", "riv_batch_counters", "riv_batch_last_recon",
    "riv_batch_clip_counters", "riv_batch_host_times",
)


def lib() -> C.CDLL:
    L = load_cuda()
    if getattr(L, "_riv_typed", False):
        return L
    P, U8P = C.c_void_p, C.POINTER(C.c_uint8)
    L.riv_config_default.argtypes = [C.POINTER(RivConfig), C.c_uint32, C.c_uint32, C.c_uint32]
    L.riv_encoder_new.argtypes = [C.POINTER(RivConfig), C.POINTER(RivWriterVtable), C.POINTER(P)]
    L.riv_encode_frame.argtypes = [P, U8P, C.c_uint32, C.c_uint32, C.c_uint64, C.POINTER(RivFrameStats)]
    L.riv_encode_frame_device.argtypes = [P, P, C.c_uint64, C.POINTER(RivFrameStats)]
    L.riv_encode_frame_yuv.argtypes = [P, U8P, U8P, U8P, C.c_uint64, C.POINTER(RivFrameStats)]
    L.riv_finish.argtypes = [P]
    L.riv_test_dct_encode.argtypes = [P, C.c_uint32, C.c_int, C.c_uint32, P, C.c_size_t, C.POINTER(C.c_size_t)]
    L.riv_test_dct_decode.argtypes = [P, C.c_size_t, P, C.c_uint32, C.c_int, P]
    L.riv_test_mv_encode.argtypes = [P, P, C.c_uint32, P, C.c_size_t, C.POINTER(C.c_size_t), P]
    L.riv_test_mv_decode.argtypes = [P, P, P, C.c_uint32, P]
    L.riv_test_mv_encode_threads.argtypes = [P, P, C.c_uint32, C.c_uint32, P, C.c_size_t, C.POINTER(C.c_size_t), P]
    L.riv_test_delta_bias.argtypes = [P, P, C.c_uint32, P, P]
    L.riv_test_worker_queue.argtypes = [C.c_uint32, C.c_uint32, C.c_uint32, C.c_int, C.c_int, C.c_int, C.c_int, P,
                                        C.c_size_t, C.POINTER(C.c_size_t)]
    L.riv_encoder_free.argtypes = [P]
    L.riv_last_error.restype = C.c_char_p
    L.riv_last_error.argtypes = [P]
    L.riv_frame_count.restype = C.c_uint64
    L.riv_frame_count.argtypes = [P]
    L.riv_last_recon.argtypes = [P, U8P, U8P, U8P]
    L.riv_last_kernel_times.argtypes = [P, C.POINTER(C.c_float)]
    L.riv_memwriter_new.restype = P
    L.riv_memwriter_vtable.argtypes = [P, C.POINTER(RivWriterVtable)]
    L.riv_memwriter_size.restype = C.c_size_t
    L.riv_memwriter_size.argtypes = [P]
    L.riv_memwriter_data.restype = P
    L.riv_memwriter_data.argtypes = [P]
    L.riv_memwriter_free.argtypes = [P]
    L.riv_stage_rgb_to_yuv.argtypes = [U8P, C.c_uint32, C.c_uint32, C.c_uint32, C.c_uint32, U8P]
    L.riv_stage_deblock.argtypes = [U8P, C.c_uint32, C.c_uint32, C.c_int, C.c_int, U8P]
    L.riv_stage_deblock_noalloc.argtypes = [U8P, C.c_uint32, C.c_uint32, C.c_int, C.c_int, U8P, C.c_char_p,
                                            C.c_size_t]
    L.riv_stage_libm.argtypes = [C.c_int, C.POINTER(C.c_float), C.POINTER(C.c_float), C.c_size_t]
    L.riv_libm_fixup_counts.argtypes = [C.POINTER(C.c_uint32), C.POINTER(C.c_uint32)]
    L.riv_stage_predict.argtypes = [U8P, P, C.c_uint32, C.c_uint32, C.c_uint8, U8P, C.POINTER(C.c_float)]
    L.riv_stage_residual.argtypes = [U8P, U8P, C.POINTER(C.c_float), U8P, P, C.c_float, C.c_uint32, C.c_uint32, P,
                                     U8P, U8P, U8P]
    L.riv_encoder_set_proposal.argtypes = [P, C.POINTER(C.c_float), C.c_size_t]
    L.riv_learned_counters.argtypes = [P, C.POINTER(C.c_uint64), C.POINTER(C.c_uint64), C.POINTER(C.c_uint64)]
    L.riv_test_wait_expiry.argtypes = [C.c_int, C.c_int64, C.POINTER(C.c_uint32)]
    L.riv_test_libm_range.argtypes = [C.c_int, C.c_uint32, C.c_uint32, C.POINTER(C.c_uint64), C.POINTER(C.c_uint32)]
    L.riv_dct_tables.argtypes = [C.POINTER(C.c_int32), C.POINTER(C.c_int32)]
    L.riv_debug_frame_state.argtypes = [P, C.c_int, P, C.c_size_t]
    L.riv_counters.argtypes = [P, C.POINTER(C.c_double), C.POINTER(C.c_uint64), C.POINTER(C.c_uint64)]
    L.riv_host_times.argtypes = [P, C.POINTER(C.c_double)]
    L.riv_decoder_new.argtypes = [U8P, C.c_size_t, C.c_int, C.POINTER(P)]
    L.riv_decoder_info.argtypes = [P, C.POINTER(C.c_uint32), C.POINTER(C.c_uint64)]
    L.riv_decode_frame_yuv.argtypes = [P, U8P, U8P, U8P, C.POINTER(C.c_uint32), C.POINTER(C.c_uint64)]
    L.riv_decode_frame_rgb.argtypes = [P, U8P, C.POINTER(C.c_uint32), C.POINTER(C.c_uint64)]
    L.riv_decoder_current_frame.restype = C.c_uint64
    L.riv_decoder_current_frame.argtypes = [P]
    L.riv_decoder_last_error.restype = C.c_char_p
    L.riv_decoder_last_error.argtypes = [P]
    L.riv_decoder_free.argtypes = [P]
    L._riv_typed = True
    return L


def _u8(a: np.ndarray):
    return a.ctypes.data_as(C.POINTER(C.c_uint8))


# ---------------------------------------------------------------------------------------
# Config (enc/config.rs)
# ---------------------------------------------------------------------------------------


@dataclasses.dataclass(frozen=True)
class KeyframeInterval:
    """KeyframeInterval::{AllIntra, Automatic, Fixed(n)} (enc/config.rs:5-19)."""

    mode: int
    interval: int = 0

    @staticmethod
    def all_intra() -> "KeyframeInterval":
        return KeyframeInterval(0)

    @staticmethod
    def automatic() -> "KeyframeInterval":
        return KeyframeInterval(1)

    @staticmethod
    def fixed(n: int) -> "KeyframeInterval":
        return KeyframeInterval(2, n)


@dataclasses.dataclass
class EncoderConfig:
    display_width: int
    display_height: int
    storage_width: int
    storage_height: int
    fps: int
    keyframe_interval: KeyframeInterval = dataclasses.field(default_factory=lambda: KeyframeInterval.fixed(30))
    intra_quality: int = 90
    inter_quality: int = 35
    search_range: int = 12
    mv_deflate_level: int = 6
    skip_threshold: int = 3
    me_zero_mv_threshold: int = 0
    me_predictor_threshold: int = 0
    rdo_lambda_mult: float = 0.49
    inter_dead_zone: float = 0.75
    # device / runtime tuning (never changes the bitstream)
    device: int = 0
    pipeline_depth: int = 0
    entropy_threads: int = 0
    encode_form: int = 0      # 0 plain (reference-identical), 1 learned proposal, 2 parallel without the network
    proposal_margin: int = 256

    @staticmethod
    def new(width: int, height: int, fps: int) -> "EncoderConfig":
        """EncoderConfig::new: storage dims rounded up to multiples of 16 (enc/config.rs:56-77)."""
        return EncoderConfig(width, height, (width + 15) // 16 * 16, (height + 15) // 16 * 16, fps)

    def _with(self, **kw) -> "EncoderConfig":
        return dataclasses.replace(self, **kw)

    def with_rdo_lambda_mult(self, v: float): return self._with(rdo_lambda_mult=v)
    def with_inter_dead_zone(self, v: float): return self._with(inter_dead_zone=v)
    def with_intra_quality(self, v: int): return self._with(intra_quality=v)
    def with_inter_quality(self, v: int): return self._with(inter_quality=v)
    def with_keyframe_interval(self, v: KeyframeInterval): return self._with(keyframe_interval=v)
    def with_search_range(self, v: int): return self._with(search_range=v)
    def with_mv_deflate_level(self, v: int): return self._with(mv_deflate_level=v)
    def with_skip_threshold(self, v: int): return self._with(skip_threshold=v)
    def with_me_zero_mv_threshold(self, v: int): return self._with(me_zero_mv_threshold=v)
    def with_me_predictor_threshold(self, v: int): return self._with(me_predictor_threshold=v)
    def with_pipeline_depth(self, v: int): return self._with(pipeline_depth=v)
    def with_encode_form(self, v: int): return self._with(encode_form=v)
    def with_proposal_margin(self, v: int): return self._with(proposal_margin=v)
    def with_device(self, v: int): return self._with(device=v)
    def with_entropy_threads(self, v: int): return self._with(entropy_threads=v)

    def validate(self) -> None:
        """EncoderConfig::validate (enc/config.rs:129-164)."""
        if self.display_width == 0 or self.display_height == 0:
            raise InvalidConfig("Width and height must be greater than 0")
        if self.storage_width < self.display_width or self.storage_height < self.display_height:
            raise InvalidConfig("Storage dimensions must be >= display dimensions")
        if self.fps == 0:
            raise InvalidConfig("FPS must be greater than 0")
        if self.search_range > 127:
            raise InvalidConfig("search_range must be <= 127 for current MV encoding")
        if self.mv_deflate_level > 10:
            raise InvalidConfig("mv_deflate_level must be in 0..=10")
        if self.keyframe_interval.mode == 2 and self.keyframe_interval.interval == 0:
            raise InvalidConfig("Keyframe interval must be greater than 0")
        if self.encode_form not in (0, 1, 2):
            raise InvalidConfig("encode_form must be 0 (plain), 1 (learned) or 2 (parallel)")
        if self.encode_form and self.search_range > 63:
            raise InvalidConfig("the learned and parallel forms need search_range <= 63")

    def to_c(self) -> RivConfig:
        c = RivConfig()
        for f in ("display_width", "display_height", "storage_width", "storage_height", "fps", "intra_quality",
                  "inter_quality", "search_range", "mv_deflate_level", "skip_threshold", "me_zero_mv_threshold",
                  "me_predictor_threshold", "rdo_lambda_mult", "inter_dead_zone", "device", "pipeline_depth",
                  "entropy_threads", "encode_form", "proposal_margin"):
            setattr(c, f, getattr(self, f))
        c.keyframe_mode = self.keyframe_interval.mode
        c.keyframe_interval = self.keyframe_interval.interval
        return c


@dataclasses.dataclass
class Frame:
    """Raw RGB24 input frame (enc/encoder.rs:18-34): width*height*3 bytes, row-major."""

    data: object
    width: int
    height: int
    timestamp: int


# ---------------------------------------------------------------------------------------
# Writers (enc/writer.rs)
# ---------------------------------------------------------------------------------------


class VideoWriter:
    """Trait VideoWriter: write / position / seek / flush (enc/writer.rs:5-18)."""

    def write(self, data: bytes) -> None: raise NotImplementedError
    def position(self) -> int: raise NotImplementedError
    def seek(self, pos: int) -> None: raise NotImplementedError
    def flush(self) -> None: raise NotImplementedError


class VecWriter(VideoWriter):
    """In-memory writer (enc/writer.rs:20-69), backed by the C library's buffer."""

    def __init__(self):
        self._h = lib().riv_memwriter_new()

    def vtable(self) -> RivWriterVtable:
        vt = RivWriterVtable()
        lib().riv_memwriter_vtable(self._h, C.byref(vt))
        return vt

    def into_inner(self) -> bytes:
        n = lib().riv_memwriter_size(self._h)
        return C.string_at(lib().riv_memwriter_data(self._h), n)

    def __del__(self):
        try:
            if self._h:
                lib().riv_memwriter_free(self._h)
                self._h = None
        except Exception:
            pass


class _PyWriterBridge:
    """Adapts a Python VideoWriter to the C vtable."""

    def __init__(self, w: VideoWriter):
        self.w = w
        self.error: Optional[BaseException] = None

        def _write(_u, ptr, n):
            try:
                self.w.write(C.string_at(ptr, n))
                return 0
            except BaseException as e:  # noqa: BLE001 - reported as Io
                self.error = e
                return 1

        def _pos(_u):
            return int(self.w.position())

        def _seek(_u, p):
            try:
                self.w.seek(int(p))
                return 0
            except BaseException as e:  # noqa: BLE001
                self.error = e
                return 1

        def _flush(_u):
            try:
                self.w.flush()
                return 0
            except BaseException as e:  # noqa: BLE001
                self.error = e
                return 1

        self._cbs = (WRITE_FN(_write), POS_FN(_pos), SEEK_FN(_seek), FLUSH_FN(_flush))

    def vtable(self) -> RivWriterVtable:
        vt = RivWriterVtable()
        vt.write, vt.position, vt.seek, vt.flush = self._cbs
        vt.user = None
        return vt


# ---------------------------------------------------------------------------------------
# Encoder (enc/encoder.rs)
# ---------------------------------------------------------------------------------------


@dataclasses.dataclass
class EncodeFrameStats:
    """EncodeFrameStats (enc/encoder.rs:58-124): every field of the reference except
    ``rle_stats``, whose sizes are ``resi_raw`` / ``resi_rans`` (None when absent)."""
    frame_index: int
    timestamp_ms: int
    frame_type: int
    total_bytes: int
    mv_bytes: int
    mv_raw_bytes: int
    residual_bytes: int
    storage_width: int
    storage_height: int
    blocks_total: int
    blocks_skipped: int
    mv_zero_delta_blocks: int
    mv_mode_counts: tuple
    mv_new_zero_pre_bias: int
    mv_new_zero_post_bias: int
    mv_new_zero_axes_x: int
    mv_new_zero_axes_y: int
    mv_new_base_counts: tuple
    mv_new_best_ref_counts: tuple
    mv_new_best_ref_l1_saved_sum: int
    mv_new_blocks: int
    mv_new_delta_count: int
    mv_new_delta_mag_sum: float
    mv_new_delta_mag_sq_sum: float
    mv_class_histogram: tuple
    mv_bias_dx: int
    mv_bias_dy: int
    mv_candidate_unique_total: int
    mv_candidate_unique_samples: int
    mv_candidate_unique_min: int
    mv_candidate_unique_max: int
    mv_match_source_counts: tuple
    mv_match_nonzero_blocks: int
    mv_match_any_spatial: int
    mv_match_any_temporal: int
    resi_raw: Optional[int]
    resi_rans: Optional[int]
    rdo_lambda: float
    rdo_blocks_evaluated: int
    rdo_blocks_selected_skip: int
    rdo_forced_fractional: int
    rdo_forced_threshold: int
    rdo_forced_disabled: int
    rdo_avg_skip_cost: float
    rdo_avg_coded_cost: float

    @staticmethod
    def from_c(s: RivFrameStats) -> "EncodeFrameStats":
        kw = {}
        for f in dataclasses.fields(EncodeFrameStats):
            v = getattr(s, f.name)
            if isinstance(v, C.Array):
                v = tuple(v)
            if f.name in ("resi_raw", "resi_rans") and v < 0:
                v = None
            kw[f.name] = v
        return EncodeFrameStats(**kw)


class Encoder:
    """Stateful GPU encoder: ``Encoder.new(config, writer)``, ``encode_frame``, ``finish``."""

    def __init__(self, config: EncoderConfig, writer: VideoWriter, _h, _bridge):
        self.config = config
        self.writer = writer
        self._h = _h
        self._bridge = _bridge

    @staticmethod
    def new(config: EncoderConfig, writer: VideoWriter) -> "Encoder":
        config.validate()
        L = lib()
        bridge = None
        if isinstance(writer, VecWriter):
            vt = writer.vtable()
        else:
            bridge = _PyWriterBridge(writer)
            vt = bridge.vtable()
        h = C.c_void_p()
        cfg = config.to_c()
        st = L.riv_encoder_new(C.byref(cfg), C.byref(vt), C.byref(h))
        if st != 0:
            raise _ERRORS.get(st, EncodeError)(f"riv_encoder_new failed (status {st})")
        return Encoder(config, writer, h, bridge)

    def _check(self, st: int) -> None:
        if st != 0:
            msg = lib().riv_last_error(self._h).decode(errors="replace")
            if self._bridge is not None and self._bridge.error is not None:
                msg += f" ({self._bridge.error!r})"
            raise _ERRORS.get(st, EncodeError)(msg)

    def encode_frame(self, frame: Frame) -> None:
        self._encode(frame, None)

    def encode_frame_with_stats(self, frame: Frame) -> EncodeFrameStats:
        s = RivFrameStats()
        self._encode(frame, s)
        return EncodeFrameStats.from_c(s)

    def _encode(self, frame: Frame, stats: Optional[RivFrameStats]) -> None:
        data = frame.data
        if isinstance(data, (bytes, bytearray, memoryview)):
            arr = np.frombuffer(data, np.uint8)
        else:
            arr = np.ascontiguousarray(data, dtype=np.uint8).reshape(-1)
        if frame.width != self.config.display_width or frame.height != self.config.display_height:
            raise FrameError(f"Frame dimensions ({frame.width}, {frame.height}) do not match config "
                             f"({self.config.display_width}, {self.config.display_height})")
        if arr.size != frame.width * frame.height * 3:
            raise FrameError(f"Display RGB24 size mismatch: expected {frame.width * frame.height * 3}, got {arr.size}")
        st = lib().riv_encode_frame(self._h, _u8(arr), frame.width, frame.height, frame.timestamp,
                                    C.byref(stats) if stats is not None else None)
        self._check(st)

    def encode_frame_device(self, ptr: int, timestamp: int, drain: bool = False) -> Optional[EncodeFrameStats]:
        """Encode a display-size RGB24 frame already resident in device memory.  With
        ``drain`` the call returns only after this frame's record was written."""
        s = RivFrameStats() if drain else None
        self._check(lib().riv_encode_frame_device(self._h, C.c_void_p(ptr), timestamp,
                                                  C.byref(s) if s is not None else None))
        return EncodeFrameStats.from_c(s) if s is not None else None

    def set_proposal(self, params: np.ndarray) -> None:
        """Load the proposal network's parameters (learned form), e.g. from
        riv2_b200.proposal.load_params()."""
        p = np.ascontiguousarray(params, dtype=np.float32)
        self._check(lib().riv_encoder_set_proposal(self._h, p.ctypes.data_as(C.POINTER(C.c_float)), p.size))

    def learned_counters(self) -> dict:
        """Learned / parallel forms: MBs searched, hexagon fallbacks, skip shortcuts."""
        a, b, c = C.c_uint64(), C.c_uint64(), C.c_uint64()
        self._check(lib().riv_learned_counters(self._h, C.byref(a), C.byref(b), C.byref(c)))
        return {"mbs": a.value, "fallbacks": b.value, "shortcuts": c.value}

    def encode_frame_yuv(self, y: np.ndarray, u: np.ndarray, v: np.ndarray, timestamp: int) -> None:
        y, u, v = (np.ascontiguousarray(p, dtype=np.uint8) for p in (y, u, v))
        self._check(lib().riv_encode_frame_yuv(self._h, _u8(y), _u8(u), _u8(v), timestamp, None))

    def finish(self) -> None:
        self._check(lib().riv_finish(self._h))

    def frame_count(self) -> int:
        return int(lib().riv_frame_count(self._h))

    def last_recon(self):
        sw, sh = self.config.storage_width, self.config.storage_height
        y = np.empty((sh, sw), np.uint8)
        u = np.empty((sh // 2, sw // 2), np.uint8)
        v = np.empty((sh // 2, sw // 2), np.uint8)
        self._check(lib().riv_last_recon(self._h, _u8(y), _u8(u), _u8(v)))
        return y, u, v

    def last_kernel_times_us(self) -> np.ndarray:
        t = np.zeros(9, np.float32)
        self._check(lib().riv_last_kernel_times(self._h, t.ctypes.data_as(C.POINTER(C.c_float))))
        return t

    def counters(self) -> dict:
        """Cumulative GPU stage times (us, P-frames), I/O bytes and kernel launches."""
        us = (C.c_double * 9)()
        io = (C.c_uint64 * 2)()
        n = (C.c_uint64 * 4)()
        self._check(lib().riv_counters(self._h, us, io, n))
        hm = (C.c_double * 6)()
        self._check(lib().riv_host_times(self._h, hm))
        return {"stage_us_sum": list(us), "h2d_bytes": io[0], "d2h_bytes": io[1], "pframes": n[0], "launches": n[1],
                "deferred_pframes": n[2], "timed_pframes": n[3],
                "host_ms": list(hm)}

    def debug_state(self, what: int) -> np.ndarray:
        """Device state of the most recent frame (see riv_debug_frame_state)."""
        sw, sh = self.config.storage_width, self.config.storage_height
        nmb = (sw // 16) * (sh // 16)
        spec = {0: (nmb * 20, np.uint8), 1: (nmb, np.float32), 2: (sw * sh * 3 // 2, np.uint8),
                3: (sw * sh * 3 // 2, np.uint8), 4: (nmb * 384, np.int16), 5: (nmb, np.uint8),
                6: (nmb * 32, np.int64)}[what]
        out = np.empty(spec[0], spec[1])
        self._check(lib().riv_debug_frame_state(self._h, what, C.c_void_p(out.ctypes.data), out.nbytes))
        return out

    def close(self) -> None:
        if self._h:
            lib().riv_encoder_free(self._h)
            self._h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass


# ---------------------------------------------------------------------------------------
# Stage entry points (one kernel each) used by the parity tests
# ---------------------------------------------------------------------------------------


def stage_rgb_to_yuv(rgb: np.ndarray, dw: int, dh: int, sw: int, sh: int) -> np.ndarray:
    rgb = np.ascontiguousarray(rgb, dtype=np.uint8)
    out = np.empty(sw * sh * 3 // 2, np.uint8)
    st = lib().riv_stage_rgb_to_yuv(_u8(rgb), dw, dh, sw, sh, _u8(out))
    if st:
        raise _ERRORS.get(st, EncodeError)("riv_stage_rgb_to_yuv failed")
    return out


def stage_deblock(yuv: np.ndarray, w: int, h: int, level: int, intra: bool, mask=None) -> np.ndarray:
    out = np.ascontiguousarray(yuv, dtype=np.uint8).copy()
    m = None if mask is None else _u8(np.ascontiguousarray(mask, dtype=np.uint8))
    st = lib().riv_stage_deblock(_u8(out), w, h, level, int(intra), m)
    if st:
        raise _ERRORS.get(st, EncodeError)("riv_stage_deblock failed")
    return out


def stage_libm(which: int, x: np.ndarray) -> np.ndarray:
    x = np.ascontiguousarray(x, dtype=np.float32)
    out = np.empty_like(x)
    st = lib().riv_stage_libm(which, x.ctypes.data_as(C.POINTER(C.c_float)),
                              out.ctypes.data_as(C.POINTER(C.c_float)), x.size)
    if st:
        raise _ERRORS.get(st, EncodeError)("riv_stage_libm failed")
    return out


def stage_predict(ref_yuv: np.ndarray, mv4: np.ndarray, w: int, h: int, quality: int):
    """build_predicted + compute_aq_quant_steps on the GPU: (prediction planes, AQ steps)."""
    ref = np.ascontiguousarray(ref_yuv, dtype=np.uint8)
    mv = np.ascontiguousarray(mv4, dtype=np.int8)
    pred = np.empty(w * h * 3 // 2, np.uint8)
    qs = np.empty((w // 16) * (h // 16), np.float32)
    st = lib().riv_stage_predict(_u8(ref), mv.ctypes.data, w, h, quality, _u8(pred),
                                 qs.ctypes.data_as(C.POINTER(C.c_float)))
    if st:
        raise _ERRORS.get(st, EncodeError)("riv_stage_predict failed")
    return pred, qs


def stage_residual(cur_yuv, pred_yuv, qs, rdo_skip, w: int, h: int, dead_zone: float, coded4=None):
    """encode_inter's residual path on the GPU: (coefficients n x 384, optimized skip,
    pre-deblock reconstruction planes, deblock mask)."""
    n = (w // 16) * (h // 16)
    cur = np.ascontiguousarray(cur_yuv, dtype=np.uint8)
    pred = np.ascontiguousarray(pred_yuv, dtype=np.uint8)
    q = np.ascontiguousarray(qs, dtype=np.float32)
    sk = np.ascontiguousarray(rdo_skip, dtype=np.uint8)
    cd = None if coded4 is None else np.ascontiguousarray(coded4, dtype=np.int8)
    co = np.empty((n, 384), np.int16)
    os_ = np.empty(n, np.uint8)
    rec = np.empty(w * h * 3 // 2, np.uint8)
    fm = np.empty(n, np.uint8)
    st = lib().riv_stage_residual(_u8(cur), _u8(pred), q.ctypes.data_as(C.POINTER(C.c_float)), _u8(sk),
                                  None if cd is None else cd.ctypes.data, dead_zone, w, h, co.ctypes.data, _u8(os_),
                                  _u8(rec), _u8(fm))
    if st:
        raise _ERRORS.get(st, EncodeError)("riv_stage_residual failed")
    return co, os_, rec, fm


def dct_encode_host(blocks: np.ndarray, intra: bool, threads: int = 0) -> bytes:
    """The encoder's host DCT-coefficient coder on dense (n, 384) int16 blocks (test hook,
    no GPU needed); threads > 0 runs its parallel form on this thread and a pool of that many
    threads (frames of 16K to 2M coded coefficients), as the encoder does for the newest
    frame of a drain.  Raises EncodingFailed where the reference encoder panics."""
    b = np.ascontiguousarray(blocks, dtype=np.int16)
    n = C.c_size_t(0)
    st = lib().riv_test_dct_encode(b.ctypes.data, b.shape[0], int(intra), threads, None, 0, C.byref(n))
    if st != 0:
        raise EncodingFailed(f"riv_test_dct_encode failed (status {st})")
    out = np.zeros(max(n.value, 1), np.uint8)
    lib().riv_test_dct_encode(b.ctypes.data, b.shape[0], int(intra), threads, out.ctypes.data, n.value, C.byref(n))
    return out[:n.value].tobytes()


def dct_decode_host(data: bytes, coded: np.ndarray, intra: bool):
    """The decoder's host DCT-coefficient decoder on one frame's stream (test hook, no GPU
    needed): (dense (n, 384) int16 blocks, ok), ok False where the stream is malformed."""
    c = np.ascontiguousarray(coded, dtype=np.uint8)
    out = np.zeros((c.size, 384), np.int16)
    buf = np.frombuffer(data, np.uint8) if len(data) else np.zeros(1, np.uint8)
    st = lib().riv_test_dct_decode(buf.ctypes.data, len(data), c.ctypes.data, c.size, int(intra), out.ctypes.data)
    return out, st == 0


def delta_bias_host(dx: np.ndarray, dy: np.ndarray):
    """The encoder's NEW-delta bias over raw deltas (test hook, no GPU needed): (bias x, bias y)."""
    x = np.ascontiguousarray(dx, dtype=np.int8)
    y = np.ascontiguousarray(dy, dtype=np.int8)
    bx, by = C.c_int8(0), C.c_int8(0)
    if lib().riv_test_delta_bias(x.ctypes.data, y.ctypes.data, x.size, C.byref(bx), C.byref(by)) != 0:
        raise EncodingFailed("riv_test_delta_bias failed")
    return bx.value, by.value


def mv_encode_host(blocks: np.ndarray, dims, threads: int = 0) -> list:
    """The encoder's host MV coder over a sequence of frames, one coder throughout (test hook,
    no GPU needed): blocks is (total blocks, 7) uint8 (mode, NEW base, dx, dy, subpel x,
    subpel y, skip), dims the (bw, bh) of each frame.  threads > 0: the parallel form the
    encoder runs (this thread and a pool of that many).  Returns each frame's bytes; raises
    EncodingFailed where the reference encoder panics (a NEW block with a raw -1/2 subpel)."""
    b = np.ascontiguousarray(blocks, dtype=np.uint8)
    d = np.ascontiguousarray(np.asarray(dims, dtype=np.uint32).reshape(-1))
    nf = d.size // 2
    fl = np.zeros(max(nf, 1), np.uint32)
    if b.ndim != 2 or b.shape[1] != 7 or b.shape[0] != int(sum(int(d[2 * f]) * int(d[2 * f + 1]) for f in range(nf))):
        raise ValueError("blocks must be (sum of bw * bh over the frames, 7)")
    n = C.c_size_t(0)
    st = lib().riv_test_mv_encode_threads(b.ctypes.data, d.ctypes.data, nf, threads, None, 0, C.byref(n),
                                          fl.ctypes.data)
    if st != 0:
        raise _ERRORS.get(st, EncodeError)(f"riv_test_mv_encode failed (status {st})")
    out = np.zeros(max(n.value, 1), np.uint8)
    lib().riv_test_mv_encode_threads(b.ctypes.data, d.ctypes.data, nf, threads, out.ctypes.data, n.value, C.byref(n),
                                     fl.ctypes.data)
    frames, pos = [], 0
    for f in range(nf):
        frames.append(out[pos:pos + int(fl[f])].tobytes())
        pos += int(fl[f])
    return frames


def mv_decode_host(frames: list, dims):
    """The decoder's host MV decoder over a sequence of frames with a fresh coder (test hook):
    ((total blocks, 7) uint8, ok), ok False on malformed data."""
    d = np.ascontiguousarray(np.asarray(dims, dtype=np.uint32).reshape(-1))
    nf = d.size // 2
    fl = np.array([len(f) for f in frames] or [0], np.uint32)
    data = np.frombuffer(b"".join(frames) or b"\0", np.uint8)
    n = int(sum(int(d[2 * f]) * int(d[2 * f + 1]) for f in range(nf)))
    out = np.zeros((max(n, 1), 7), np.uint8)
    st = lib().riv_test_mv_decode(data.ctypes.data, fl.ctypes.data, d.ctypes.data, nf, out.ctypes.data)
    return out[:n], st == 0


def worker_queue(bw: int, bh: int, w: int, defer: bool, deblock: bool, tables: bool, compact: bool) -> np.ndarray:
    """The fused search launch's worker tasks in hand-out order, (n, 3) int32 rows of (kind,
    row, index): kind 0 residual pair, 1 deblock tile, 2 SAD-table MB, 3 scan, 4 pack row."""
    n = C.c_size_t(0)
    args = (bw, bh, w, int(defer), int(deblock), int(tables), int(compact))
    if lib().riv_test_worker_queue(*args, None, 0, C.byref(n)) != 0:
        raise EncodingFailed("riv_test_worker_queue: task count disagrees with the queue total")
    out = np.zeros((max(n.value, 1), 3), np.int32)
    lib().riv_test_worker_queue(*args, out.ctypes.data, out.size, C.byref(n))
    return out[:n.value]


def libm_fixup_counts():
    a, b = C.c_uint32(), C.c_uint32()
    st = lib().riv_libm_fixup_counts(C.byref(a), C.byref(b))
    if st:
        raise EncodeError("libm fix-up table missing")
    return a.value, b.value


def dct_tables():
    t16 = np.zeros(256, np.int32)
    t8 = np.zeros(64, np.int32)
    lib().riv_dct_tables(t16.ctypes.data_as(C.POINTER(C.c_int32)), t8.ctypes.data_as(C.POINTER(C.c_int32)))
    return t16.reshape(16, 16), t8.reshape(8, 8)
