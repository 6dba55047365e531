"""riv2_b200 -- B200 (sm_100a) implementation of the riv2 (.riv) P-frame encoder hot path.

Public API mirrors reitero_encode: EncoderConfig / KeyframeInterval / Frame / VecWriter /
Encoder (new, encode_frame, encode_frame_with_stats, finish) and the EncodeError family.
"""
from .batch import Batch  # noqa: F401
from .encoder import (  # noqa: F401
    CudaError,
    DeviceTimeout,
    EncodeError,
    EncodeFrameStats,
    Encoder,
    EncoderConfig,
    EncodingFailed,
    Frame,
    FrameError,
    InvalidConfig,
    IoError,
    KeyframeInterval,
    UnsupportedCodec,
    VecWriter,
    VideoWriter,
)
