"""Parity at the workloads' full sizes (GPU, marked gpu).

* CIF 352x288, 60 frames, q 85/80: the GPU stream equals the oracle's byte for byte.
* 1080p, 120 frames, q 85/80 and 95/90, frames in flight: byte-identical to the oracle, and
  the oracle decoder reproduces the GPU's last reconstruction.
* 720p, 30 frames, and CIF at search range 15, 20 frames, both 16 frames in flight:
  byte-identical to the oracle.
* 4K 3840x2160 high-motion stress, 60 frames, q 95/90 and 75/70: byte-identical to the
  oracle encoder over all 60 frames, and the oracle decoder decodes the GPU stream to the
  GPU's reconstruction of every frame.
"""
import numpy as np
import pytest

from oracle import oracle as O

pytestmark = pytest.mark.gpu


def _configs(w, h, fps, iq, pq, depth):
    from riv2_b200 import encoder as E
    gc = (E.EncoderConfig.new(w, h, fps).with_intra_quality(iq).with_inter_quality(pq)
          .with_keyframe_interval(E.KeyframeInterval.fixed(1 << 40)).with_pipeline_depth(depth))
    oc = O.default_config(w, h, fps)
    oc.intra_quality, oc.inter_quality = iq, pq
    oc.keyframe_mode, oc.keyframe_interval = 2, 1 << 40
    return gc, oc


def _gpu_stream(clip, n, gc, recons=False):
    from riv2_b200 import encoder as E
    w = E.VecWriter()
    enc = E.Encoder.new(gc, w)
    out = []
    for t in range(n):
        enc.encode_frame(E.Frame(clip.frame(t), gc.display_width, gc.display_height, t * 1000 // gc.fps))
        if recons:
            out.append(enc.last_recon())
    last = enc.last_recon() if not recons else out[-1]
    enc.finish()
    data = w.into_inner()
    enc.close()
    return data, out, last


def _oracle_stream(clip, n, oc, fps):
    enc = O.OracleEncoder(oc)
    for t in range(n):
        assert enc.encode_rgb(clip.frame(t), t * 1000 // fps) == 0
    return enc.finish()


def _same_frame(dec_frame, yuv):
    y, u, v = yuv
    return np.array_equal(dec_frame.y, y) and np.array_equal(dec_frame.u, u) and np.array_equal(dec_frame.v, v)


def test_cif_60_frames_byte_identical():
    from riv2_b200.synth import SynthClip
    clip = SynthClip("cif", seed=11)
    gc, oc = _configs(352, 288, 30, 85, 80, depth=4)
    g, _, _ = _gpu_stream(clip, 60, gc)
    assert g == _oracle_stream(clip, 60, oc, 30)


@pytest.mark.parametrize("q", [(85, 80), (95, 90)])
def test_1080p_120_frames_byte_identical(q):
    from riv2_b200.synth import SynthClip
    clip = SynthClip("1080p", seed=2026)
    gc, oc = _configs(1920, 1080, 50, *q, depth=16)
    g, _, last = _gpu_stream(clip, 120, gc)
    o = _oracle_stream(clip, 120, oc, 50)
    assert len(g) == len(o)
    assert g == o
    dec = O.OracleDecoder(g)
    assert dec.frame_count == 120
    for _ in range(119):
        typ, f = dec.next()
        assert typ > 0
    typ, f = dec.next()
    assert typ == 2 and _same_frame(f, last)


def test_720p_pipelined_byte_identical():
    """720p (80 x 45 MBs: other worker-queue counts and deblock tiling) at depth 16, where each
    P-frame is reconstructed inside the next frame's search launch."""
    from riv2_b200.synth import SynthClip
    clip = SynthClip("720p", seed=31)
    gc, oc = _configs(1280, 720, 30, 85, 80, depth=16)
    g, _, _ = _gpu_stream(clip, 30, gc)
    assert g == _oracle_stream(clip, 30, oc, 30)


def test_cif_search_range_15_pipelined_byte_identical():
    """Search range 15 (the largest SAD-table window and reference band) at depth 16."""
    from riv2_b200.synth import SynthClip
    clip = SynthClip("cif", seed=17)
    gc, oc = _configs(352, 288, 30, 85, 80, depth=16)
    gc = gc._with(search_range=15)
    oc.search_range = 15
    g, _, _ = _gpu_stream(clip, 20, gc)
    assert g == _oracle_stream(clip, 20, oc, 30)


@pytest.mark.parametrize("q", [(95, 90), (75, 70)])
def test_4k_stress_decodes_to_encoder_recon(q):
    from riv2_b200.synth import SynthClip
    clip = SynthClip("4k", seed=7)
    gc, oc = _configs(3840, 2160, 30, *q, depth=0)
    g, recons, _ = _gpu_stream(clip, 60, gc, recons=True)
    dec = O.OracleDecoder(g)
    assert (dec.sw, dec.sh, dec.frame_count) == (3840, 2160, 60)
    for t in range(60):
        typ, f = dec.next()
        assert typ == (1 if t == 0 else 2) and _same_frame(f, recons[t]), t
    # every frame's record is byte-identical to the oracle encoder's
    o = _oracle_stream(clip, 60, oc, 30)
    assert len(g) == len(o)
    assert g == o
