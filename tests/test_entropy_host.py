"""The encoder's host DCT-coefficient coder (riv_entropy.cpp, behind riv_test_dct_encode)
against the oracle's restatement of res/rans.rs:195-330, byte for byte, on CPU: P-frame
and intra (DC prediction) blocks, frames shorter than one rANS batch and frames of several
batches, coded inline, with the full batches on a thread pool, and by the parallel coder
(block ranges, models evolved per thread, batches in parallel) as the pipelined encoder
does."""
import numpy as np
import pytest

from oracle import oracle as O


def _blocks(n, seed, density=0.25, big=False):
    rng = np.random.default_rng(seed)
    b = np.zeros((n, 384), np.int16)
    for plane, (lo, hi, d) in enumerate(((0, 256, density), (256, 320, density / 2), (320, 384, density / 2))):
        width = hi - lo
        # significance fades with the coefficient index, like quantised DCT blocks
        p = d * np.exp(-np.arange(width) / (width / 6.0))
        mask = rng.random((n, width)) < p
        mag = rng.geometric(0.4, (n, width)).astype(np.int32)
        if big:
            mag[rng.random((n, width)) < 0.01] = rng.integers(100, 4000, 1)[0]
        sign = np.where(rng.random((n, width)) < 0.5, -1, 1)
        b[:, lo:hi] = np.where(mask, sign * mag, 0).astype(np.int16)
    b[::7, 0] = rng.integers(-900, 900, b[::7, 0].shape)  # some large DC values
    return b


@pytest.mark.parametrize("intra", [False, True])
@pytest.mark.parametrize("threads", [0, 3])
@pytest.mark.parametrize("n,seed", [(1, 1), (37, 2), (3000, 3)])
def test_dct_coder_matches_oracle(n, seed, threads, intra):
    from riv2_b200.encoder import dct_encode_host
    b = _blocks(n, seed, big=seed == 3)
    assert dct_encode_host(b, intra, threads) == O.dct_encode(b, intra)


def test_dct_coder_spans_several_batches_and_all_zero_blocks():
    from riv2_b200.encoder import dct_encode_host
    b = _blocks(6000, 9, density=0.6)
    b[100:200] = 0                      # all-zero blocks are coded too (EOB class 0)
    ref = O.dct_encode(b, False)
    # a binary symbol carries at most 8 bits here (probabilities >= 1/256), so more than
    # 50,000 bytes means more than 3 rANS batches of 16386 symbols
    assert len(ref) > 50_000
    assert dct_encode_host(b, False, 0) == ref
    assert dct_encode_host(b, False, 4) == ref


@pytest.mark.parametrize("intra", [False, True])
@pytest.mark.parametrize("threads", [1, 2, 6])
def test_parallel_dct_coder_matches_oracle(threads, intra):
    """Frames of 16K to 2M coded coefficients are split over threads + 1 parts: the symbols
    of block ranges are listed in parallel, grouped by model, each model's probabilities
    evolved on one thread, and the rANS batches coded in parallel.  Same bytes, including
    the intra DC prediction across range boundaries and all-zero blocks."""
    from riv2_b200.encoder import dct_encode_host
    b = _blocks(2500, 11 + threads, density=0.4, big=True)
    b[300:340] = 0
    assert dct_encode_host(b, intra, threads) == O.dct_encode(b, intra)


@pytest.mark.parametrize("threads", [0, 3])
def test_magnitude_classes_13_and_14(threads):
    """A magnitude of class 13 (|v| - 1 in [4096, 8191]) is coded with 13 continue bits and
    no stop bit, as the reference's encode_magnitude does (reitero_residual/src/rans.rs:72-98);
    from class 14 the reference indexes past its 13 models and panics, and the frame fails."""
    from riv2_b200.encoder import dct_encode_host, EncodingFailed
    b = _blocks(400, 21, density=0.5)
    b[5, 3] = 5000
    b[200, 260] = -8000
    assert dct_encode_host(b, False, threads) == O.dct_encode(b, False)
    b[300, 40] = 9000
    with pytest.raises(ValueError):
        O.dct_encode(b, False)
    with pytest.raises(EncodingFailed):
        dct_encode_host(b, False, threads)


@pytest.mark.parametrize("intra", [False, True])
def test_dct_decoder_round_trip_and_oracle(intra):
    """The decoder's host coefficient decoder (riv_entropy.cpp, behind riv_test_dct_decode)
    inverts the coder, leaves the blocks outside the coded mask zero, and agrees with the
    oracle's restatement of the reference decoder (res/rans.rs:340-459)."""
    from riv2_b200.encoder import dct_encode_host, dct_decode_host
    rng = np.random.default_rng(5)
    n = 900
    coded = (rng.random(n) < 0.7).astype(np.uint8)
    b = _blocks(int(coded.sum()), 31, density=0.4, big=not intra)
    data = dct_encode_host(b, intra, 0)
    got, ok = dct_decode_host(data, coded, intra)
    assert ok
    assert np.array_equal(got[coded == 1], b) and not got[coded == 0].any()
    ref, ref_ok = O.dct_decode(data, coded, intra)
    assert ref_ok and np.array_equal(got, ref)


def test_dct_decoder_class_13_and_malformed_streams_match_oracle():
    """A class-13 magnitude is written with 13 continue bits but read back, as by the
    reference decoder, as class 12: the rest of the frame decodes to the same wrong values on
    both sides.  A truncated stream is malformed for both."""
    from riv2_b200.encoder import dct_encode_host, dct_decode_host
    b = _blocks(300, 41, density=0.3)
    b[10, 5] = 5000
    coded = np.ones(300, np.uint8)
    data = dct_encode_host(b, False, 0)
    got, ok = dct_decode_host(data, coded, False)
    ref, ref_ok = O.dct_decode(data, coded, False)
    assert ok == ref_ok
    if ok:
        assert np.array_equal(got, ref)
    assert not np.array_equal(got, b)
    short, short_ok = dct_decode_host(data[: len(data) // 3], coded, False)
    _, short_ref_ok = O.dct_decode(data[: len(data) // 3], coded, False)
    assert not short_ok and not short_ref_ok
