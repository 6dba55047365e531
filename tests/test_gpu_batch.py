"""Multi-clip encoding (riv_batch) against single-clip encodes (GPU, marked gpu).

Every clip of a batch must write the stream a single-clip encoder writes for it alone, byte
for byte, and end with the same reconstruction.  The single-clip GPU encoder is itself
byte-identical to the oracle (tests/test_gpu_parity.py, tests/test_gpu_fullsize.py); one clip
here is also compared with the oracle directly.

The mixes cover what one step can hold: clips of different sizes (including a storage size
padded from an odd display size), different qualities, a search range above the SAD-table
limit (another search variant in the same step), key frames in some clips while others code
P-frames, and clips that start late or end early (steps where they have no frame).
"""
import numpy as np
import pytest

from oracle import oracle as O

pytestmark = pytest.mark.gpu


def _cfg(w, h, iq=85, pq=80, keyint=1 << 40, sr=12, depth=4):
    from riv2_b200 import encoder as E
    return (E.EncoderConfig.new(w, h, 30).with_intra_quality(iq).with_inter_quality(pq).with_search_range(sr)
            .with_keyframe_interval(E.KeyframeInterval.fixed(keyint)).with_pipeline_depth(depth))


def _single(cfg, frames, ts):
    from riv2_b200 import encoder as E
    w = E.VecWriter()
    enc = E.Encoder.new(cfg, w)
    for f, t in zip(frames, ts):
        enc.encode_frame(E.Frame(f, cfg.display_width, cfg.display_height, t))
    last = enc.last_recon()
    enc.finish()
    data = w.into_inner()
    enc.close()
    return data, last


def _run_batch(cfgs, clips, spans, tune=None):
    """spans[i] = (first step, frame count) of clip i."""
    from riv2_b200 import encoder as E
    from riv2_b200.batch import Batch
    writers = [E.VecWriter() for _ in cfgs]
    b = Batch.new(cfgs, writers)
    if tune is not None:
        b.set_tune(*tune)
    steps = max(s + n for s, n in spans)
    recons = [None] * len(cfgs)
    for k in range(steps):
        fr, ts = [], []
        for i, (s, n) in enumerate(spans):
            t = k - s
            fr.append(clips[i].frame(t) if 0 <= t < n else None)
            ts.append(t * 33 if 0 <= t < n else 0)
        b.encode_step(fr, ts)
        for i, (s, n) in enumerate(spans):
            if k - s == n - 1:
                recons[i] = b.last_recon(i)
    b.finish()
    info = {"tune": b.tune(), "counters": b.counters()}
    b.close()
    return [w.into_inner() for w in writers], recons, info


def _check_against_single(cfgs, clips, spans, streams, recons):
    for i, (cfg, (s, n)) in enumerate(zip(cfgs, spans)):
        frames = [clips[i].frame(t) for t in range(n)]
        ref, last = _single(cfg, frames, [t * 33 for t in range(n)])
        assert streams[i] == ref, f"clip {i} ({cfg.display_width}x{cfg.display_height}): stream differs from the single-clip encode"
        for p, q in zip(recons[i], last):
            assert np.array_equal(p, q), f"clip {i}: reconstruction differs"


def test_batch_mixed_sizes_qualities_and_spans_match_single_clip():
    from riv2_b200.synth import SynthClip
    cfgs = [_cfg(352, 288), _cfg(352, 288, 95, 90), _cfg(640, 360, keyint=4), _cfg(1280, 720),
            _cfg(100, 70), _cfg(352, 288, sr=20)]
    clips = [SynthClip("cif", seed=31), SynthClip("cif", seed=32), SynthClip("720p", seed=33, width=640, height=360),
             SynthClip("720p", seed=34), SynthClip("cif", seed=35, width=100, height=70), SynthClip("cif", seed=36)]
    spans = [(0, 9), (0, 7), (1, 8), (0, 6), (3, 5), (2, 6)]
    streams, recons, info = _run_batch(cfgs, clips, spans)
    _check_against_single(cfgs, clips, spans, streams, recons)
    assert info["counters"]["frames"] == sum(n for _, n in spans)


def test_batch_clip_matches_oracle():
    from riv2_b200.synth import SynthClip
    cfgs = [_cfg(352, 288), _cfg(640, 360)]
    clips = [SynthClip("cif", seed=41), SynthClip("720p", seed=42, width=640, height=360)]
    spans = [(0, 6), (0, 6)]
    streams, _, _ = _run_batch(cfgs, clips, spans)
    oc = O.default_config(352, 288, 30)
    oc.intra_quality, oc.inter_quality = 85, 80
    oc.keyframe_mode, oc.keyframe_interval = 2, 1 << 40
    oe = O.OracleEncoder(oc)
    for t in range(6):
        assert oe.encode_rgb(clips[0].frame(t), t * 33) == 0
    assert streams[0] == oe.finish()


@pytest.mark.parametrize("tune", [(100, 2, 64, 1), (50, 8, 256, 0), (1, 4, 128, 1), (75, 4, 128, 0)])
def test_batch_tile_shapes_do_not_change_the_streams(tune):
    from riv2_b200.synth import SynthClip
    cfgs = [_cfg(352, 288), _cfg(1280, 720), _cfg(640, 360)]
    clips = [SynthClip("cif", seed=51), SynthClip("720p", seed=52), SynthClip("720p", seed=53, width=640, height=360)]
    spans = [(0, 5), (0, 5), (0, 5)]
    streams, recons, info = _run_batch(cfgs, clips, spans, tune=tune)
    assert info["tune"]["state"] == "fixed"
    _check_against_single(cfgs, clips, spans, streams, recons)


def test_batch_autotuner_settles_and_keeps_streams():
    from riv2_b200.synth import SynthClip
    cfgs = [_cfg(352, 288), _cfg(352, 288), _cfg(640, 360)]
    clips = [SynthClip("cif", seed=61), SynthClip("cif", seed=62), SynthClip("720p", seed=63, width=640, height=360)]
    spans = [(0, 18), (0, 18), (0, 18)]
    streams, recons, info = _run_batch(cfgs, clips, spans)
    assert info["tune"]["state"] == "autotuned", info
    assert info["tune"]["sad_table"] in (0, 1)
    assert info["tune"]["res_mbs"] in (2, 4, 8) and info["tune"]["db_tw"] in (64, 128, 256)
    _check_against_single(cfgs, clips, spans, streams, recons)
