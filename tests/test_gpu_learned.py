"""The learned-proposal and parallel encode forms (GPU).

Their streams differ from the reference encoder's by design (the search is seeded
differently), so the check is validity: the oracle's restatement of reitero_decode
(dec/decoder.rs:195-460) must decode every frame of every stream to exactly the encoder's
reconstruction, and the mode decisions made for all MBs at once must be those the decoder's
MV reconstruction expects.  Also checked: the forms' counters, loud failure without a network,
and that the learned form's quality stays near the plain form's on a short clip.
"""
import numpy as np
import pytest

from oracle import oracle as O

pytestmark = pytest.mark.gpu


def _cfg(w, h, form, depth=0, q=(85, 80), sr=12):
    from riv2_b200 import encoder as E
    return (E.EncoderConfig.new(w, h, 30).with_intra_quality(q[0]).with_inter_quality(q[1])
            .with_keyframe_interval(E.KeyframeInterval.fixed(1000)).with_pipeline_depth(depth)
            .with_search_range(sr).with_encode_form(form))


def _encode(frames, cfg, params=None, recons=True):
    from riv2_b200 import encoder as E
    w = E.VecWriter()
    enc = E.Encoder.new(cfg, w)
    if params is not None:
        enc.set_proposal(params)
    out = []
    for t, f in enumerate(frames):
        enc.encode_frame(E.Frame(f, cfg.display_width, cfg.display_height, t * 33))
        if recons:
            out.append(enc.last_recon())
    enc.finish()
    counters = enc.learned_counters()
    enc.close()
    return w.into_inner(), out, counters


def _decodes_to(stream, recons):
    dec = O.OracleDecoder(stream)
    for t, (y, u, v) in enumerate(recons):
        typ, f = dec.next()
        assert typ == (1 if t == 0 else 2), t
        assert np.array_equal(f.y, y) and np.array_equal(f.u, u) and np.array_equal(f.v, v), f"frame {t}"


def _params(seed=0):
    from riv2_b200 import proposal as P
    return P.init_params(seed)


@pytest.mark.parametrize("form", [1, 2])
@pytest.mark.parametrize("preset,w,h,n", [("cif", 352, 288, 10), ("720p", 1280, 720, 6)])
def test_stream_decodes_to_the_encoder_reconstruction(form, preset, w, h, n):
    from riv2_b200.synth import SynthClip
    clip = SynthClip(preset, seed=41)
    frames = [clip.frame(t) for t in range(n)]
    stream, recons, c = _encode(frames, _cfg(w, h, form), _params() if form == 1 else None)
    _decodes_to(stream, recons)
    nmb = (w // 16) * ((h + 15) // 16)
    assert c["mbs"] == nmb * (n - 1)
    if form == 2:
        assert c["fallbacks"] == 0 and c["shortcuts"] == 0  # no network: nothing to fall back from
    else:
        assert 0 <= c["fallbacks"] <= c["mbs"]


@pytest.mark.parametrize("form", [1, 2])
def test_1080p_stream_with_the_trained_network_decodes(form):
    """The bench's size and network: every kernel of the form at 8160 MBs (convolution tiles
    that cross MB boundaries, four-position search steps at the frame's borders)."""
    import os
    from riv2_b200 import proposal as P
    from riv2_b200.synth import SynthClip
    clip = SynthClip("1080p", seed=2026)
    frames = [clip.frame(t) for t in range(4)]
    weights = os.path.join(os.path.dirname(os.path.dirname(os.path.abspath(__file__))), "riv2_b200", "weights",
                           "proposal.bin")
    params = P.load_params(weights) if form == 1 else None
    stream, recons, c = _encode(frames, _cfg(1920, 1080, form), params)
    _decodes_to(stream, recons)
    assert c["mbs"] == 8160 * 3
    if form == 1:
        assert c["fallbacks"] < c["mbs"] // 2  # the trained network's proposals are mostly taken


@pytest.mark.parametrize("form", [1, 2])
def test_pipelined_stream_equals_synchronous(form):
    from riv2_b200.synth import SynthClip
    clip = SynthClip("cif", seed=43)
    frames = [clip.frame(t) for t in range(12)]
    p = _params(1) if form == 1 else None
    s0, r0, _ = _encode(frames, _cfg(352, 288, form, depth=0), p)
    s4, _, _ = _encode(frames, _cfg(352, 288, form, depth=4), p, recons=False)
    assert s0 == s4
    _decodes_to(s0, r0)


@pytest.mark.parametrize("case", ["noise", "sr31", "odd_dims", "q1", "q100"])
def test_extreme_inputs_stay_valid(case):
    from riv2_b200.synth import SynthClip
    w, h, sr, q = 352, 288, 12, (85, 80)
    if case == "noise":
        rng = np.random.default_rng(3)
        frames = [rng.integers(0, 256, (h, w, 3), dtype=np.uint8) for _ in range(4)]
    else:
        if case == "odd_dims":
            w, h = 100, 70
        frames = [SynthClip("cif", seed=5, width=w, height=h).frame(t) for t in range(6)]
        sr = 31 if case == "sr31" else 12
        q = {"q1": (1, 1), "q100": (100, 100)}.get(case, q)
    stream, recons, _ = _encode(frames, _cfg(w, h, 1, q=q, sr=sr), _params(2))
    _decodes_to(stream, recons)


def test_learned_form_without_a_network_fails_loudly():
    from riv2_b200 import encoder as E
    from riv2_b200.synth import SynthClip
    clip = SynthClip("cif", seed=1)
    enc = E.Encoder.new(_cfg(352, 288, 1), E.VecWriter())
    enc.encode_frame(E.Frame(clip.frame(0), 352, 288, 0))  # key frame: no search
    with pytest.raises(E.EncodingFailed):
        enc.encode_frame(E.Frame(clip.frame(1), 352, 288, 33))
    enc.close()
    with pytest.raises(E.InvalidConfig):
        E.Encoder.new(_cfg(352, 288, 1, sr=64), E.VecWriter())
