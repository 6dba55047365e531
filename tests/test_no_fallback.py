"""Without a usable CUDA device the encoder and decoder fail loudly: there is no CPU fallback
of the hot path.  Runs where no GPU is visible (on a machine with one, the device path is
what the -m gpu tests exercise, and these checks skip)."""
import numpy as np
import pytest


def _device_present() -> bool:
    import ctypes
    try:
        rt = ctypes.CDLL("libcudart.so")
    except OSError:
        try:
            import glob
            import os
            import torch  # noqa: F401  (the wheel bundles the runtime)
            cands = glob.glob(os.path.join(os.path.dirname(torch.__file__), "..", "nvidia", "cuda_runtime", "lib",
                                           "libcudart.so*"))
            if not cands:
                return False
            rt = ctypes.CDLL(cands[0])
        except Exception:
            return False
    n = ctypes.c_int(0)
    return rt.cudaGetDeviceCount(ctypes.byref(n)) == 0 and n.value > 0


def test_encoder_without_device_raises_cuda_error():
    if _device_present():
        pytest.skip("a CUDA device is visible")
    from riv2_b200 import encoder as E
    cfg = E.EncoderConfig.new(64, 48, 30)
    w = E.VecWriter()
    with pytest.raises(E.CudaError):
        E.Encoder.new(cfg, w)
    assert w.into_inner() == b""  # nothing written: no header from a half-built encoder


def test_decoder_without_device_raises():
    if _device_present():
        pytest.skip("a CUDA device is visible")
    from oracle import oracle as O
    from riv2_b200 import decoder as D
    cfg = O.default_config(32, 32, 30)
    enc = O.OracleEncoder(cfg)
    enc.encode_rgb(np.zeros((32, 32, 3), np.uint8), 0)
    stream = enc.finish()
    with pytest.raises(D.CudaError):
        D.Decoder.new(stream)


def test_batch_without_device_raises_cuda_error():
    if _device_present():
        pytest.skip("a CUDA device is visible")
    from riv2_b200 import encoder as E
    from riv2_b200.batch import Batch
    cfgs = [E.EncoderConfig.new(64, 48, 30), E.EncoderConfig.new(352, 288, 30)]
    ws = [E.VecWriter(), E.VecWriter()]
    with pytest.raises(E.CudaError):
        Batch.new(cfgs, ws)
    assert all(w.into_inner() == b"" for w in ws)


def test_batch_rejects_bad_clip_sets():
    # checked before any device call
    from riv2_b200 import encoder as E
    from riv2_b200.batch import Batch
    with pytest.raises(E.InvalidConfig):
        Batch.new([], [])
    learned = E.EncoderConfig.new(64, 48, 30).with_encode_form(1)
    with pytest.raises(E.InvalidConfig):
        Batch.new([E.EncoderConfig.new(64, 48, 30), learned], [E.VecWriter(), E.VecWriter()])
    other_dev = E.EncoderConfig.new(64, 48, 30).with_device(1)
    with pytest.raises(E.InvalidConfig):
        Batch.new([E.EncoderConfig.new(64, 48, 30), other_dev], [E.VecWriter(), E.VecWriter()])
