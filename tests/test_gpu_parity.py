"""GPU parity tests: the CUDA path through the C ABI against the CPU oracle.

Bit-exact for everything (integer, byte and index work; the f32/f64 arithmetic of the
reference is reproduced op for op).  Streams are compared byte for byte, reconstructions
pixel for pixel, and the oracle's decoder must decode every GPU stream to the GPU's
reconstruction.
"""
import numpy as np
import pytest

from oracle import oracle as O

pytestmark = pytest.mark.gpu


def _cfgs(w, h, iq=85, pq=80, **kw):
    from riv2_b200 import encoder as E
    gc = E.EncoderConfig.new(w, h, 30).with_intra_quality(iq).with_inter_quality(pq)
    gc = gc.with_keyframe_interval(E.KeyframeInterval.fixed(kw.pop("keyint", 1000)))
    oc = O.default_config(w, h, 30)
    oc.intra_quality, oc.inter_quality = iq, pq
    oc.keyframe_mode, oc.keyframe_interval = gc.keyframe_interval.mode, gc.keyframe_interval.interval
    for k, v in kw.items():
        gc = gc._with(**{k: v})
        setattr(oc, k, v)
    return gc, oc


def _encode_both(frames, gc, oc, check_every_frame=True):
    from riv2_b200 import encoder as E
    w = E.VecWriter()
    enc = E.Encoder.new(gc, w)
    oenc = O.OracleEncoder(oc)
    orecons = []
    for t, f in enumerate(frames):
        assert oenc.encode_rgb(f, t * 20) == 0
        enc.encode_frame(E.Frame(f, gc.display_width, gc.display_height, t * 20))
        orecons.append(oenc.last("recon"))
        if check_every_frame and gc.pipeline_depth == 0:
            y, u, v = enc.last_recon()
            r = orecons[-1]
            if not (np.array_equal(y, r.y) and np.array_equal(u, r.u) and np.array_equal(v, r.v)):
                _explain(enc, oenc, t)
    enc.finish()
    ostream = oenc.finish()
    gstream = w.into_inner()
    enc.close()
    return gstream, ostream, orecons


def _explain(enc, oenc, t):
    """Locate the first diverging stage of frame t."""
    nmb = oenc.mbs
    mbo = enc.debug_state(0).reshape(nmb, 20)
    raw_o, coded_o, sad_o = oenc.last_mvs()
    side_o = oenc.last_side()
    msgs = []
    if oenc.last_type() == 2:
        raw_g = mbo[:, 0:4].view(np.int8)
        coded_g = mbo[:, 4:8].view(np.int8)
        bad = np.nonzero((raw_g != raw_o).any(1))[0]
        if bad.size:
            i = bad[0]
            msgs.append(f"raw MV differs at {bad.size} MBs, first {i}: gpu {raw_g[i]} oracle {raw_o[i]}")
        bad = np.nonzero((coded_g != coded_o).any(1))[0]
        if bad.size:
            msgs.append(f"coded MV differs at {bad.size} MBs, first {bad[0]}")
        sad_g = mbo[:, 16:20].copy().view(np.int32).reshape(-1)
        bad = np.nonzero(sad_g != sad_o)[0]
        if bad.size:
            msgs.append(f"best SAD differs at {bad.size} MBs, first {bad[0]}: {sad_g[bad[0]]} vs {sad_o[bad[0]]}")
        for col, name in ((10, "mode"), (11, "base"), (13, "rdo_skip")):
            o_col = {10: 0, 11: 1, 13: 5}[col]
            bad = np.nonzero(mbo[:, col] != side_o[:, o_col])[0]
            if bad.size:
                msgs.append(f"{name} differs at {bad.size} MBs, first {bad[0]}")
        qs_g = enc.debug_state(1)
        qs_o = oenc.last_qsteps()
        bad = np.nonzero(qs_g.view(np.uint32) != qs_o.view(np.uint32))[0]
        if bad.size:
            msgs.append(f"AQ step differs at {bad.size} MBs, first {bad[0]}: {qs_g[bad[0]]!r} vs {qs_o[bad[0]]!r}")
        pred_g = enc.debug_state(2)
        p = oenc.last("pred")
        pred_o = np.concatenate([p.y.reshape(-1), p.u.reshape(-1), p.v.reshape(-1)])
        if not np.array_equal(pred_g, pred_o):
            msgs.append(f"prediction differs at {(pred_g != pred_o).sum()} samples")
    cur_g = enc.debug_state(3)
    c = oenc.last("curr")
    if not np.array_equal(cur_g, np.concatenate([c.y.reshape(-1), c.u.reshape(-1), c.v.reshape(-1)])):
        msgs.append("converted input differs")
    co_g = enc.debug_state(4).reshape(nmb, 384)
    co_o = oenc.last_coeffs()
    bad = np.nonzero((co_g != co_o).any(1))[0]
    if bad.size:
        msgs.append(f"coefficients differ at {bad.size} MBs, first {bad[0]}")
    pytest.fail(f"frame {t}: reconstruction differs; " + "; ".join(msgs or ["deblock only"]))


def _check(gstream, ostream, orecons):
    assert len(gstream) == len(ostream), (len(gstream), len(ostream))
    if gstream != ostream:
        i = next(k for k in range(len(gstream)) if gstream[k] != ostream[k])
        pytest.fail(f"streams differ first at byte {i} of {len(gstream)}")
    dec = O.OracleDecoder(gstream)
    for r in orecons:
        typ, f = dec.next()
        assert typ > 0 and f.equal(r)


def _clip(preset, n, seed=5, **kw):
    from riv2_b200.synth import SynthClip
    c = SynthClip(preset, seed=seed, **kw)
    return [c.frame(t) for t in range(n)]


# ---------------------------------------------------------------------------------------
# Stage parity
# ---------------------------------------------------------------------------------------

@pytest.mark.parametrize("dw,dh", [(352, 288), (100, 70), (1920, 1080)])
def test_rgb_to_yuv_matches_oracle(dw, dh):
    from riv2_b200 import encoder as E
    rng = np.random.default_rng(dw)
    rgb = rng.integers(0, 256, (dh, dw, 3)).astype(np.uint8)
    sw, sh = (dw + 15) // 16 * 16, (dh + 15) // 16 * 16
    g = E.stage_rgb_to_yuv(rgb, dw, dh, sw, sh)
    o = O.rgb_to_yuv(rgb, dw, dh, sw, sh)
    assert np.array_equal(g, np.concatenate([o.y.reshape(-1), o.u.reshape(-1), o.v.reshape(-1)]))


def _kat_frame(w, h, left, right):
    f = O.Frames(w, h)
    f.y[:, : w // 2] = left
    f.y[:, w // 2:] = right
    f.u[:] = 128
    f.v[:] = 128
    return f


@pytest.mark.parametrize("case", ["wide", "large", "texture", "masked", "either", "zero"])
def test_deblock_kats_on_gpu(case):
    from riv2_b200 import encoder as E
    f = _kat_frame(32, 32, 40 if case == "large" else 100, 200 if case == "large" else 106)
    if case == "texture":
        f.y[:, 13] = 160
    level = {"texture": 8, "zero": 0}.get(case, 20)
    mask = {"masked": [0, 0, 0, 0], "either": [0, 1, 0, 1]}.get(case)
    flat = np.concatenate([f.y.reshape(-1), f.u.reshape(-1), f.v.reshape(-1)])
    g = E.stage_deblock(flat, 32, 32, level, False, mask)
    o = O.deblock(f, level, False, mask)
    assert np.array_equal(g, np.concatenate([o.y.reshape(-1), o.u.reshape(-1), o.v.reshape(-1)]))
    y = g[:1024].reshape(32, 32)[0]
    if case in ("large",):
        assert y[15] == 40 and y[16] == 200
    if case in ("texture", "masked", "zero"):
        assert y[15] == 100 and y[16] == 106
    if case in ("wide", "either"):
        assert y[15] > 100 and y[16] < 106


@pytest.mark.parametrize("w,h,intra", [(352, 288, True), (352, 288, False), (1920, 1088, False)])
def test_deblock_random_matches_oracle(w, h, intra):
    from riv2_b200 import encoder as E
    rng = np.random.default_rng(w + intra)
    f = O.Frames(w, h)
    base = rng.integers(60, 200, (h // 16, w // 16))
    f.y[:] = np.clip(np.kron(base, np.ones((16, 16))) + rng.integers(-3, 4, (h, w)), 0, 255)
    f.u[:] = np.clip(np.kron(base, np.ones((8, 8))) + rng.integers(-2, 3, (h // 2, w // 2)), 0, 255)
    f.v[:] = rng.integers(0, 256, (h // 2, w // 2))
    mask = None if intra else rng.integers(0, 2, (h // 16) * (w // 16)).astype(np.uint8)
    flat = np.concatenate([f.y.reshape(-1), f.u.reshape(-1), f.v.reshape(-1)])
    for level in (3, 17, 25, 44, 63):
        g = E.stage_deblock(flat, w, h, level, intra, mask)
        o = O.deblock(f, level, intra, mask)
        assert np.array_equal(g, np.concatenate([o.y.reshape(-1), o.u.reshape(-1), o.v.reshape(-1)])), level


def test_libm_samples_match_glibc():
    """Device logf/exp2f (correctly rounded + glibc fix-ups) on a sample, incl. fix-up keys."""
    from riv2_b200 import encoder as E
    rng = np.random.default_rng(0)
    x = rng.uniform(4.0, 16256.25, 20000).astype(np.float32)
    import ctypes
    libm = ctypes.CDLL("libm.so.6")
    libm.logf.restype = ctypes.c_float
    libm.logf.argtypes = [ctypes.c_float]
    libm.exp2f.restype = ctypes.c_float
    libm.exp2f.argtypes = [ctypes.c_float]
    # every 8th logf fix-up input of the AQ's variance range [4, 16256.25] and the inputs either
    # side of it (bitmap bit set, and clear next to a set one)
    import os
    from riv2_b200.build import LIB_DIR
    raw = np.fromfile(os.path.join(LIB_DIR, "libm_fixups.bin"), np.uint8)
    nlog = int(raw[8:12].view(np.uint32)[0])
    keys = raw[16:16 + 8 * nlog].view(np.uint32)[0::2]
    keys = keys[(keys >= np.float32(4.0).view(np.uint32)) & (keys <= np.float32(16256.25).view(np.uint32))][::8]
    assert keys.size > 1000
    near = np.concatenate([keys, keys - 1, keys + 1]).view(np.float32)
    xs = np.concatenate([x, near])
    g = E.stage_libm(0, xs)
    want = np.array([libm.logf(float(v)) for v in xs], np.float32)
    assert np.array_equal(g.view(np.uint32), want.view(np.uint32))
    e = rng.uniform(-1.2, 1.2, 20000).astype(np.float32)
    g = E.stage_libm(1, e)
    want = np.array([libm.exp2f(float(v)) for v in e], np.float32)
    assert np.array_equal(g.view(np.uint32), want.view(np.uint32))


# ---------------------------------------------------------------------------------------
# Whole-encoder parity
# ---------------------------------------------------------------------------------------

def test_encode_cif_matches_oracle():
    frames = _clip("cif", 8)
    gc, oc = _cfgs(352, 288)
    _check(*_encode_both(frames, gc, oc))


@pytest.mark.parametrize("variant", ["q95", "sr31", "thresholds", "keyint3", "odd_dims", "tiny", "skip0"])
def test_encode_variants_match_oracle(variant):
    kw = {}
    w, h, preset, n = 352, 288, "cif", 6
    iq, pq = 85, 80
    if variant == "q95":
        iq, pq = 95, 90
    elif variant == "sr31":
        kw["search_range"] = 31
    elif variant == "thresholds":
        kw["me_zero_mv_threshold"] = 400
        kw["me_predictor_threshold"] = 900
    elif variant == "keyint3":
        kw["keyint"] = 3
    elif variant == "odd_dims":
        w, h = 100, 70
    elif variant == "tiny":
        w, h, n = 16, 16, 4
    elif variant == "skip0":
        kw["skip_threshold"] = 0
    frames = _clip(preset, n, seed=9, width=w, height=h)
    gc, oc = _cfgs(w, h, iq, pq, **kw)
    _check(*_encode_both(frames, gc, oc))


def test_encode_pipelined_is_identical():
    frames = _clip("cif", 10, seed=3)
    gc, oc = _cfgs(352, 288)
    g0, o0, r0 = _encode_both(frames, gc, oc)
    gc4 = gc.with_pipeline_depth(4)
    g4, _, _ = _encode_both(frames, gc4, oc, check_every_frame=False)
    assert g0 == o0 == g4


@pytest.mark.parametrize("w,h", [(352, 288), (100, 70), (16, 16)])
def test_deferred_reconstruction_flush_paths(w, h):
    """From pipeline depth 2 a P-frame is reconstructed inside the next P-frame's search
    launch; before a key frame, for a per-frame-stats call, for last_recon and at finish it
    is reconstructed with separate kernels instead.  A mix of all of them gives the oracle's
    stream, last_recon returns the oracle's reconstruction of the frame just submitted, and
    both kinds of reconstruction occur."""
    from riv2_b200 import encoder as E
    frames = _clip("cif", 14, seed=5, width=w, height=h)
    gc, oc = _cfgs(w, h, keyint=5)
    gc = gc.with_pipeline_depth(16)
    wr = E.VecWriter()
    enc = E.Encoder.new(gc, wr)
    oenc = O.OracleEncoder(oc)
    for t, f in enumerate(frames):
        assert oenc.encode_rgb(f, t * 20) == 0
        fr = E.Frame(f, w, h, t * 20)
        if t % 6 == 3:
            assert enc.encode_frame_with_stats(fr).frame_index == t
        else:
            enc.encode_frame(fr)
        if t in (7, 8, 12):
            y, u, v = enc.last_recon()
            r = oenc.last("recon")
            assert np.array_equal(y, r.y) and np.array_equal(u, r.u) and np.array_equal(v, r.v), t
    enc.finish()
    c = enc.counters()
    assert wr.into_inner() == oenc.finish()
    enc.close()
    assert 0 < c["deferred_pframes"] < c["pframes"]


@pytest.mark.parametrize("q", [(85, 80), (95, 90)])
def test_encode_1080p_matches_oracle(q):
    frames = _clip("1080p", 3, seed=2)
    gc, oc = _cfgs(1920, 1080, *q)
    _check(*_encode_both(frames, gc, oc))


# ---------------------------------------------------------------------------------------
# Whole-encode parity on content and qualities the synthetic clips do not reach
# ---------------------------------------------------------------------------------------

def _noise_clip(n, w, h, seed):
    rng = np.random.default_rng(seed)
    return [rng.integers(0, 256, (h, w, 3), dtype=np.uint8) for _ in range(n)]


def _step_clip(n, w, h, seed):
    """Full-range 0/255 blocks that move by a few pixels per frame (MVs up to the range)."""
    rng = np.random.default_rng(seed)
    yy, xx = np.mgrid[0:h + 64, 0:w + 64]
    base = np.where(((yy // 13) + (xx // 11)) % 2 == 0, 0, 255).astype(np.uint8)
    out = []
    for t in range(n):
        dy, dx = int(rng.integers(0, 32)), int(rng.integers(0, 32))
        f = base[dy:dy + h, dx:dx + w]
        out.append(np.stack([f, 255 - f, f], axis=-1).copy())
    return out


@pytest.mark.parametrize("case", ["q1", "q100", "noise_q100", "noise_q1", "steps_q100", "steps_sr31"])
def test_encode_extreme_content_and_quality_matches_oracle(case):
    w, h, kw = 352, 288, {}
    if case in ("q1", "q100"):
        frames = _clip("cif", 6, seed=21)
    elif case.startswith("noise"):
        frames = _noise_clip(4, w, h, seed=22)
    else:
        frames = _step_clip(5, w, h, seed=23)
    q = 1 if case.endswith("q1") else 100
    if case == "steps_sr31":
        q, kw = 90, {"search_range": 31}
    gc, oc = _cfgs(w, h, q, q, **kw)
    _check(*_encode_both(frames, gc, oc))
