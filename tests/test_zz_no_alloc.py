"""The no-allocation deblock entry point (riv_stage_deblock_noalloc) against the existing
riv_stage_deblock.  It serves callers that cannot allocate device memory per call (their
memory belongs to their own pool allocator, or cudaFree's device-wide synchronisation would
stall a latency-critical thread).  Checked: identical planes over two calls in a row (the
fixed device scratch carries nothing from one call to the next), and the size limit
rejected with a message.  Collected last, so a run that stops at its first failure has
already run every other test."""
import ctypes as C

import numpy as np
import pytest

MAX_BYTES = 4 << 20


def _lib():
    from riv2_b200 import encoder as E
    return E.lib()


def _u8(a):
    return a.ctypes.data_as(C.POINTER(C.c_uint8))


def _noalloc(yuv, w, h, level, intra, mask):
    out = yuv.copy()
    err = C.create_string_buffer(256)
    m = None if mask is None else _u8(mask)
    st = _lib().riv_stage_deblock_noalloc(_u8(out), w, h, level, int(intra), m, err, len(err))
    return st, out, err.value.decode()


def _existing(yuv, w, h, level, intra, mask):
    out = yuv.copy()
    m = None if mask is None else _u8(mask)
    st = _lib().riv_stage_deblock(_u8(out), w, h, level, int(intra), m)
    return st, out


def _planes(w, h, seed):
    rng = np.random.default_rng(seed)
    n = w * h * 3 // 2
    # blocky content with small steps at the MB edges, so the filter changes many samples
    base = rng.integers(60, 200, size=n, dtype=np.int32)
    noise = rng.integers(-3, 4, size=n, dtype=np.int32)
    y = np.repeat(np.repeat(rng.integers(90, 110, size=(h // 16, w // 16)), 16, 0), 16, 1).reshape(-1)
    base[: w * h] = y + noise[: w * h]
    return np.clip(base, 0, 255).astype(np.uint8)


def test_noalloc_rejects_oversize_and_bad_dims():
    # no device call happens before these checks
    w, h = 3840, 2160
    st, _, msg = _noalloc(np.zeros(w * h * 3 // 2, np.uint8), w, h, 20, False, None)
    assert st == 5 and "RIV_DEBLOCK_NOALLOC_MAX_BYTES" in msg and str(MAX_BYTES) in msg
    st, _, msg = _noalloc(np.zeros(100 * 70 * 3 // 2, np.uint8), 100, 70, 20, False, None)
    assert st == 5 and "multiples of 16" in msg


@pytest.mark.gpu
@pytest.mark.parametrize("w,h,with_mask", [(352, 288, True), (1920, 1088, False), (1920, 1088, True)])
def test_noalloc_matches_existing_entry_point_twice(w, h, with_mask):
    rng = np.random.default_rng(w + h)
    for call in range(2):  # two calls in a row, different content each time
        yuv = _planes(w, h, seed=call * 7 + w)
        mask = (rng.integers(0, 2, size=(w // 16) * (h // 16)).astype(np.uint8) if with_mask else None)
        level, intra = (30 + 9 * call), bool(call)
        st0, ref = _existing(yuv, w, h, level, intra, mask)
        st1, out, msg = _noalloc(yuv, w, h, level, intra, mask)
        assert st0 == 0 and st1 == 0, msg
        assert not np.array_equal(ref, yuv), "the filter should change this content"
        assert np.array_equal(out, ref), f"call {call}: {(out != ref).sum()} samples differ"


@pytest.mark.gpu
def test_noalloc_at_the_size_limit_edge():
    # 2048x1360 with a mask fills the scratch to within 5.5 KB of its end (4,188,800 of
    # 4,194,304 bytes): the planes and the mask both sit at the scratch's far end
    w, h = 2048, 1360
    need = w * h * 3 // 2 + (w // 16) * (h // 16)
    assert MAX_BYTES - 8192 < need <= MAX_BYTES
    rng = np.random.default_rng(5)
    for call in range(2):
        yuv = _planes(w, h, seed=11 + call)
        mask = rng.integers(0, 2, size=(w // 16) * (h // 16)).astype(np.uint8)
        mask[-64:] = 1  # the last MB rows (the mask's last bytes) are filtered
        st0, ref = _existing(yuv, w, h, 36, False, mask)
        st1, out, msg = _noalloc(yuv, w, h, 36, False, mask)
        assert st0 == 0 and st1 == 0, msg
        assert not np.array_equal(ref, yuv)
        assert np.array_equal(out, ref), f"call {call}: {(out != ref).sum()} samples differ"
    # one 16-pixel row more no longer fits
    st, _, msg = _noalloc(np.zeros(w * (h + 16) * 3 // 2, np.uint8), w, h + 16, 36, False, mask)
    assert st == 5 and "RIV_DEBLOCK_NOALLOC_MAX_BYTES" in msg
