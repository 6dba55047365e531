"""Stage parity on adversarial inputs: prediction + AQ steps and the residual path.

The whole-encode tests reach these kernels only through the synthetic clips' smooth content
at q 75-95.  Here each stage gets inputs the generator rarely or never produces, and its
output is compared with the oracle's bit for bit:

* prediction (build_predicted, com/fast_motion.rs:103-352): MVs at +-search range at all
  four frame borders, with half-pel in either axis, over white-noise and full-range step
  planes;
* AQ steps (compute_aq_quant_steps, res/residual.rs:116-167) at q 1, 80 and 100;
* residual (res/residual.rs:520-752): white noise, full-range steps, steps small enough to
  saturate the i16 quantiser output, steps large enough to zero every MB, dead zones 0.75
  and 0.
"""
import zlib

import numpy as np
import pytest

from oracle import oracle as O

pytestmark = pytest.mark.gpu


def _planes(kind, w, h, rng):
    n = w * h * 3 // 2
    if kind == "noise":
        return rng.integers(0, 256, n, dtype=np.uint8)
    if kind == "steps":  # 0 / 255 blocks of random sizes, full-range edges everywhere
        out = np.empty(n, np.uint8)
        for off, pw, ph in ((0, w, h), (w * h, w // 2, h // 2), (w * h * 5 // 4, w // 2, h // 2)):
            cell = int(rng.integers(3, 12))
            yy, xx = np.mgrid[0:ph, 0:pw]
            out[off:off + pw * ph] = np.where(((yy // cell) + (xx // (cell + 1))) % 2 == 0, 0, 255).reshape(-1)
        return out
    if kind == "flat":
        return np.full(n, int(rng.integers(0, 256)), np.uint8)
    raise ValueError(kind)


def _frames(flat, w, h):
    f = O.Frames(w, h)
    f.y[:] = flat[: w * h].reshape(h, w)
    f.u[:] = flat[w * h: w * h * 5 // 4].reshape(h // 2, w // 2)
    f.v[:] = flat[w * h * 5 // 4:].reshape(h // 2, w // 2)
    return f


def _flat(f):
    return np.concatenate([f.y.reshape(-1), f.u.reshape(-1), f.v.reshape(-1)])


def _border_mvs(w, h, sr, rng):
    """Canonical MVs (dx, dy, sx, sy; sx, sy in {0, 1}) within [-sr-1, sr] + half-pel; MBs on
    the borders point as far out of the frame as the range allows."""
    bw, bh = w // 16, h // 16
    n = bw * bh
    mv = np.zeros((n, 4), np.int8)
    mv[:, 0] = rng.integers(-sr - 1, sr + 1, n)
    mv[:, 1] = rng.integers(-sr - 1, sr + 1, n)
    mv[:, 2] = rng.integers(0, 2, n)
    mv[:, 3] = rng.integers(0, 2, n)
    by, bx = np.divmod(np.arange(n), bw)
    mv[bx == 0, 0] = -sr - 1
    mv[bx == bw - 1, 0] = sr
    mv[by == 0, 1] = -sr - 1
    mv[by == bh - 1, 1] = sr
    # a quarter of the border MBs exactly at the integer limit, with no half-pel
    edge = (bx == 0) | (bx == bw - 1) | (by == 0) | (by == bh - 1)
    pick = edge & (rng.random(n) < 0.25)
    mv[pick, 2:] = 0
    mv[pick & (bx == 0), 0] = -sr
    mv[pick & (by == 0), 1] = -sr
    return mv


@pytest.mark.parametrize("kind", ["noise", "steps"])
@pytest.mark.parametrize("sr", [12, 31])
@pytest.mark.parametrize("q", [1, 80, 100])
def test_predict_and_aq_steps_at_the_borders(kind, sr, q):
    from riv2_b200 import encoder as E
    w, h = 352, 288
    rng = np.random.default_rng(sr * 1000 + q)
    ref = _planes(kind, w, h, rng)
    mv = _border_mvs(w, h, sr, rng)
    pred, qs = E.stage_predict(ref, mv, w, h, q)
    want = _flat(O.build_predicted(_frames(ref, w, h), mv))
    assert np.array_equal(pred, want), f"{(pred != want).sum()} predicted samples differ"
    wq = O.aq_steps(pred[: w * h].reshape(h, w), w, h, float(np.float32(O.lib().oracle_quant_step(q))))
    assert np.array_equal(qs.view(np.uint32), wq.view(np.uint32))


CASES = [
    # cur, pred, quality for the steps, step scale, dead zone
    ("noise", "noise", 80, 1.0, 0.75),
    ("steps", "flat", 100, 1.0, 0.75),
    ("steps", "noise", 1, 1.0, 0.75),
    ("noise", "flat", 100, 0.002, 0.75),  # tiny steps: quantised values saturate at +-32767
    ("steps", "flat", 100, 0.002, 0.0),   # no dead zone, saturation
    ("noise", "noise", 1, 400.0, 0.75),   # huge steps: every MB quantises to zero (optimized skip)
    ("noise", "steps", 95, 1.0, 0.0),
]


@pytest.mark.parametrize("cur_kind,pred_kind,q,scale,dz", CASES)
def test_residual_matches_oracle(cur_kind, pred_kind, q, scale, dz):
    from riv2_b200 import encoder as E
    w, h = 352, 288
    n = (w // 16) * (h // 16)
    rng = np.random.default_rng(zlib.crc32(repr((cur_kind, pred_kind, q, scale, dz)).encode()))
    cur = _planes(cur_kind, w, h, rng)
    pred = _planes(pred_kind, w, h, rng)
    base = float(np.float32(O.lib().oracle_quant_step(q)))
    qs = (O.aq_steps(pred[: w * h].reshape(h, w), w, h, base) * np.float32(scale)).astype(np.float32)
    skip = (rng.random(n) < 0.2).astype(np.uint8)
    coded = np.zeros((n, 4), np.int8)
    coded[:, 0] = rng.integers(-2, 3, n)
    co, osk, rec, fm = E.stage_residual(cur, pred, qs, skip, w, h, dz, coded)
    wco, wosk, wrec = O.residual_inter(cur, pred, w, h, skip, qs, dz)
    assert np.array_equal(osk, wosk), f"{(osk != wosk).sum()} optimized-skip flags differ"
    assert np.array_equal(co, wco), f"{(co != wco).any(axis=1).sum()} MBs' coefficients differ"
    assert np.array_equal(rec, wrec), f"{(rec != wrec).sum()} reconstructed samples differ"
    # the deblock mask of enc/encoder.rs:831-841: coded, or a non-zero MV
    assert np.array_equal(fm, ((1 - osk) | (coded != 0).any(axis=1)).astype(np.uint8))
    if scale <= 0.002:
        assert (np.abs(co.astype(np.int32)) >= 32767).any(), "expected saturated coefficients"
    if scale >= 400:
        assert osk.all()
