"""The encoder's host MV coder and the decoder's MV decoder (riv_entropy.cpp, behind
riv_test_mv_encode / riv_test_mv_decode) on CPU, against the oracle's restatement of
res/mv_rans/encoder.rs and decoder.rs: the reference's own round-trip cases
(res/mv_rans/tests.rs) restated, byte equality with the oracle's coder, frames that carry
contexts and the candidate history across a sequence, and the raw -1/2 panic."""
import numpy as np
import pytest

from oracle import oracle as O

ZERO, NEAREST, NEAR, TOPRIGHT, TOPLEFT, NEW, TEMPORAL = range(7)


def from_interleaved(triples):
    """(ddx, ddy, flags) per block as in res/mv_rans/tests.rs:3-31: Zero mode when both deltas
    and the subpel flags are 0, else New with base 0; subpel x = flags & 3, subpel y =
    (flags >> 2) & 3 (1 +1/2, 2 -1/2, else 0); skip = flags & 0x40."""
    out = np.zeros((len(triples), 7), np.uint8)
    for i, (dx, dy, fl) in enumerate(triples):
        sx = {1: 1, 2: 2}.get(fl & 3, 0)
        sy = {1: 1, 2: 2}.get((fl >> 2) & 3, 0)
        zero = dx == 0 and dy == 0 and (fl & 0x0F) == 0
        out[i] = (ZERO if zero else NEW, 0, dx & 0xFF, dy & 0xFF, sx, sy, 1 if fl & 0x40 else 0)
    return out


def check(frames_blocks, dims):
    from riv2_b200.encoder import mv_decode_host, mv_encode_host
    blocks = np.concatenate(frames_blocks)
    got = mv_encode_host(blocks, dims)
    assert got == O.mv_encode(blocks, dims)
    back, ok = mv_decode_host(got, dims)
    assert ok and np.array_equal(back, blocks)
    ref_back, ref_ok = O.mv_decode(got, dims)
    assert ref_ok and np.array_equal(ref_back, blocks)
    return got


def test_reference_single_frame():  # res/mv_rans/tests.rs:32-56
    check([from_interleaved([(5, -3, 0x05), (-2, 1, 0x40), (0, 0, 0x00)])], [(3, 1)])


def test_reference_multiple_frames():  # res/mv_rans/tests.rs:70-115
    f1 = from_interleaved([(1, 2, 0x05), (-1, 0, 0x00)])
    f2 = from_interleaved([(0, 0, 0x40), (5, -5, 0x05), (-10, 10, 0x00)])
    check([f1, f2], [(2, 1), (3, 1)])


def test_reference_all_halfpel_codes():  # res/mv_rans/tests.rs:117-141
    check([from_interleaved([(0, 0, qx | (qy << 2)) for qx in range(2) for qy in range(2)])], [(4, 1)])


def test_reference_edge_cases():  # res/mv_rans/tests.rs:143-171
    check([from_interleaved([(-128, 127, 0x00), (127, -128, 0x40), (0, 0, 0x45), (127, -128, 0x00)])], [(4, 1)])


def test_reference_large_frame():  # res/mv_rans/tests.rs:173-210
    i = np.arange(40 * 30)
    triples = [(int(a), int(b), int(f)) for a, b, f in
               zip(i % 17 - 8, i % 13 - 6, (i % 2) | (((i // 3) % 2) << 2) | ((i % 10 == 0) << 6))]
    check([from_interleaved(triples)], [(40, 30)])


def test_reference_500_frames():  # res/mv_rans/tests.rs:212-320: contexts and candidates carry
    i = np.arange(40 * 30)
    frames = []
    for f in range(500):
        dx = (f % 30 + i % 17 - 8).astype(np.int64)
        dy = np.full_like(i, f % 13 - 6)
        qx, qy = (f + i) % 2, (f * 2 + i) % 2
        skip = (i % 10 == 0) | ((np.abs(dx) < 2) & (np.abs(dy) < 2))
        fl = qx | (qy << 2) | (skip.astype(np.int64) << 6)
        frames.append(from_interleaved(list(zip(dx.tolist(), dy.tolist(), fl.tolist()))))
    check(frames, [(40, 30)] * 500)


def test_all_modes_with_candidate_history():
    """Every mode and NEW base, mixed over 40 frames of 24 x 16 blocks: after 100 NEW blocks
    the coder keeps up to 16 candidates, so hits, misses and the hit contexts all occur."""
    rng = np.random.default_rng(7)
    frames = []
    for f in range(40):
        n = 24 * 16
        b = np.zeros((n, 7), np.uint8)
        b[:, 0] = rng.choice(7, n, p=[0.2, 0.15, 0.1, 0.05, 0.05, 0.4, 0.05])
        new = b[:, 0] == NEW
        b[new, 1] = rng.integers(0, 5, new.sum())
        common = rng.random(n) < 0.6  # a few recurring deltas feed the candidate list
        dx = np.where(common, rng.choice([-3, 0, 2, 5], n), rng.integers(-128, 128, n))
        dy = np.where(common, rng.choice([-1, 0, 4], n), rng.integers(-128, 128, n))
        b[new, 2] = (dx[new] & 0xFF).astype(np.uint8)
        b[new, 3] = (dy[new] & 0xFF).astype(np.uint8)
        b[new, 4] = rng.integers(0, 2, new.sum())
        b[new, 5] = rng.integers(0, 2, new.sum())
        b[:, 6] = rng.random(n) < 0.3
        frames.append(b)
    check(frames, [(24, 16)] * 40)


def test_raw_minus_half_is_the_reference_panic():  # res/mv_rans/tests.rs:58-68
    from riv2_b200.encoder import EncodingFailed, mv_encode_host
    b = from_interleaved([(0, 0, 0x08)])
    with pytest.raises(ValueError):
        O.mv_encode(b, [(1, 1)])
    with pytest.raises(EncodingFailed):
        mv_encode_host(b, [(1, 1)])
    # a non-NEW block's subpel fields are not coded: no panic
    z = b.copy()
    z[0, 0] = NEAREST
    assert mv_encode_host(z, [(1, 1)]) == O.mv_encode(z, [(1, 1)])


def test_truncated_mv_stream_is_malformed_for_both():
    from riv2_b200.encoder import mv_decode_host, mv_encode_host
    i = np.arange(40 * 30)
    b = from_interleaved([(int(a), int(c), 0x05) for a, c in zip(i % 17 - 8, i % 13 - 6)])
    got = mv_encode_host(b, [(40, 30)])
    short = [got[0][: len(got[0]) // 4]]
    assert not mv_decode_host(short, [(40, 30)])[1]
    assert not O.mv_decode(short, [(40, 30)])[1]


@pytest.mark.parametrize("case", ["empty", "random", "clustered", "extremes"])
def test_delta_bias_matches_oracle(case):
    """The encoder's NEW-delta bias (compute_delta_bias_for_new, enc/encoder.rs:984-1048) is
    computed from per-axis histograms; the oracle restates the reference's loop over the
    deltas.  Same bias on both axes, including the -128 wrap of i8::abs and the clamp."""
    from riv2_b200.encoder import delta_bias_host
    rng = np.random.default_rng(11)
    if case == "empty":
        dx = dy = np.zeros(0, np.int8)
    elif case == "random":
        dx, dy = rng.integers(-128, 128, 5000), rng.integers(-128, 128, 5000)
    elif case == "clustered":
        dx = np.clip(np.round(rng.normal(7, 3, 8160)), -128, 127)
        dy = np.clip(np.round(rng.normal(-19, 5, 8160)), -128, 127)
    else:
        dx = rng.choice([-128, -127, -105, 104, 127, 0], 3000)
        dy = rng.choice([-128, 127, -24, 24, 1], 3000)
    dx, dy = np.asarray(dx, np.int8), np.asarray(dy, np.int8)
    assert delta_bias_host(dx, dy) == O.delta_bias(dx, dy)


def _random_sequence(nf, bw, bh, seed):
    """Frames of every mode, NEW blocks drawn from a small set of MVs so that the candidate
    history fills (hits, candidate indices) and carries across frames."""
    rng = np.random.default_rng(seed)
    frames = []
    pool = [(int(a), int(b), int(c), int(d)) for a, b, c, d in zip(rng.integers(-20, 21, 24), rng.integers(-20, 21, 24),
                                                                 rng.integers(0, 2, 24), rng.integers(0, 2, 24))]
    for _ in range(nf):
        n = bw * bh
        f = np.zeros((n, 7), np.uint8)
        f[:, 0] = rng.choice([ZERO, NEAREST, NEAR, TOPRIGHT, TOPLEFT, NEW, TEMPORAL], n,
                             p=[0.2, 0.3, 0.1, 0.05, 0.05, 0.25, 0.05])
        new = f[:, 0] == NEW
        f[new, 1] = rng.integers(0, 5, new.sum())
        pick = rng.integers(0, len(pool), new.sum())
        for j, (i, k) in enumerate(zip(np.nonzero(new)[0], pick)):
            dx, dy, sx, sy = pool[k] if rng.random() < 0.7 else (int(rng.integers(-100, 101)), int(rng.integers(-100, 101)),
                                                                int(rng.integers(0, 2)), int(rng.integers(0, 2)))
            f[i, 2:6] = (dx & 0xFF, dy & 0xFF, sx, sy)
        f[:, 6] = rng.random(n) < 0.3
        frames.append(f)
    return frames


@pytest.mark.parametrize("threads", [1, 2, 3, 7])
def test_parallel_mv_coder_is_byte_identical(threads):
    """The encoder's parallel MV coder (symbol lists per MB range, each model over its own
    symbols, rANS batches in parallel) writes the sequential coder's bytes, and the oracle's,
    frame after frame (contexts and candidate history carried), for frames of one rANS batch
    and of several."""
    from riv2_b200.encoder import mv_encode_host
    for bw, bh, nf in ((120, 68, 4), (16, 9, 6), (240, 135, 2)):
        frames = _random_sequence(nf, bw, bh, seed=bw + threads)
        blocks = np.concatenate(frames)
        dims = [(bw, bh)] * nf
        seq = mv_encode_host(blocks, dims)
        par = mv_encode_host(blocks, dims, threads=threads)
        assert par == seq, (bw, bh)
        assert seq == O.mv_encode(blocks, dims)
