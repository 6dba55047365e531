"""Python mirror of reitero_decode's Decoder over the C ABI (include/riv_gpu.h).

Same names as the reference crate (reitero_video/reitero_decode/src/decoder.rs):

    dec = Decoder.new(stream_bytes)
    while dec.has_more_frames():
        f = dec.decode_frame()      # DecodedFrame: y, u, v planes (storage size), timestamp, ...

The frames are the YUV 4:2:0 reconstruction at storage size; the reference's final RGB24
conversion and crop are not part of this path.  Reconstruction runs on the GPU; there is no
CPU fallback.
"""
from __future__ import annotations

import ctypes as C
import dataclasses

import numpy as np

from .encoder import lib


class DecodeError(Exception):
    status = 3


class IoError(DecodeError):
    status = 1


class InvalidHeader(DecodeError):
    status = 2


class DecodingFailed(DecodeError):
    status = 3


class InvalidFrame(DecodeError):
    status = 4


class EndOfStream(DecodeError):
    status = 5


class CudaError(DecodeError):
    status = 6


_ERRORS = {1: IoError, 2: InvalidHeader, 3: DecodingFailed, 4: InvalidFrame, 5: EndOfStream, 6: CudaError}


@dataclasses.dataclass
class VideoHeader:
    display_width: int
    display_height: int
    storage_width: int
    storage_height: int
    fps: int
    frame_count: int


@dataclasses.dataclass
class DecodedFrame:
    """decoder.rs:34-50, with the storage-size YUV planes instead of cropped RGB24."""
    y: np.ndarray
    u: np.ndarray
    v: np.ndarray
    timestamp: int
    frame_index: int
    frame_type: int  # 1 intra, 2 inter


@dataclasses.dataclass
class DecodedRgbFrame:
    """decoder.rs:34-50: the frame as display-size RGB24 (dec/decoder.rs:445-456)."""
    rgb: np.ndarray  # (display_height, display_width, 3) uint8
    timestamp: int
    frame_index: int
    frame_type: int  # 1 intra, 2 inter


class Decoder:
    def __init__(self, handle, data):
        self._h = handle
        self._data = data
        d = (C.c_uint32 * 5)()
        n = C.c_uint64()
        lib().riv_decoder_info(self._h, d, C.byref(n))
        self._header = VideoHeader(d[0], d[1], d[2], d[3], d[4], n.value)

    @staticmethod
    def new(stream: bytes, device: int = 0) -> "Decoder":
        """Decoder::new (decoder.rs:112-171)."""
        buf = np.frombuffer(bytes(stream), np.uint8)
        h = C.c_void_p()
        st = lib().riv_decoder_new(buf.ctypes.data_as(C.POINTER(C.c_uint8)), len(buf), device, C.byref(h))
        if st:
            raise _ERRORS.get(st, DecodeError)("riv_decoder_new failed")
        return Decoder(h, buf)

    def header(self) -> VideoHeader:
        return self._header

    def current_frame(self) -> int:
        return int(lib().riv_decoder_current_frame(self._h))

    def has_more_frames(self) -> bool:
        return self.current_frame() < self._header.frame_count

    def decode_frame(self, copy_out: bool = True) -> DecodedFrame | None:
        """Decoder::decode_frame (decoder.rs:174-460) up to the YUV reconstruction.  With
        copy_out=False the frame is decoded on the GPU but not copied back (None)."""
        hd = self._header
        w, h = hd.storage_width, hd.storage_height
        y = np.empty((h, w), np.uint8) if copy_out else None
        u = np.empty((h // 2, w // 2), np.uint8) if copy_out else None
        v = np.empty((h // 2, w // 2), np.uint8) if copy_out else None
        ptr = (lambda a: a.ctypes.data_as(C.POINTER(C.c_uint8)) if a is not None else None)
        t = C.c_uint32()
        ts = C.c_uint64()
        idx = self.current_frame()
        st = lib().riv_decode_frame_yuv(self._h, ptr(y), ptr(u), ptr(v), C.byref(t), C.byref(ts))
        if st:
            msg = lib().riv_decoder_last_error(self._h)
            raise _ERRORS.get(st, DecodeError)(msg.decode() if msg else "decode failed")
        return DecodedFrame(y, u, v, ts.value, idx, t.value) if copy_out else None

    def decode_frame_rgb(self) -> DecodedRgbFrame:
        """Decoder::decode_frame (decoder.rs:174-460) with its RGB output: the reconstruction
        converted to RGB24 on the GPU (BT.709 limited range, this library's definition; the
        reference uses the `yuv` crate, so byte parity with it is not established) and
        cropped to the display size."""
        hd = self._header
        rgb = np.empty((hd.display_height, hd.display_width, 3), np.uint8)
        t = C.c_uint32()
        ts = C.c_uint64()
        idx = self.current_frame()
        st = lib().riv_decode_frame_rgb(self._h, rgb.ctypes.data_as(C.POINTER(C.c_uint8)), C.byref(t), C.byref(ts))
        if st:
            msg = lib().riv_decoder_last_error(self._h)
            raise _ERRORS.get(st, DecodeError)(msg.decode() if msg else "decode failed")
        return DecodedRgbFrame(rgb, ts.value, idx, t.value)

    def close(self) -> None:
        if self._h:
            lib().riv_decoder_free(self._h)
            self._h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass
