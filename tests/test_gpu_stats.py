"""EncodeFrameStats of the GPU encoder against the oracle's (GPU, marked gpu).

``encode_frame_with_stats`` returns every field of the reference's EncodeFrameStats
(enc/encoder.rs:58-124) except ``rle_stats`` (its two sizes are ``resi_raw`` / ``resi_rans``).
Each frame's stats must equal the oracle's restatement of the reference's bookkeeping: counts
exactly, and the f64 sums (delta magnitudes, RDO costs) exactly too, since both sum the same
values in raster order without contraction.
"""
import numpy as np
import pytest

from oracle import oracle as O

pytestmark = pytest.mark.gpu


def _pair(w, h, iq, pq, keyint, skip_threshold):
    from riv2_b200 import encoder as E
    gc = (E.EncoderConfig.new(w, h, 30).with_intra_quality(iq).with_inter_quality(pq)
          .with_keyframe_interval(E.KeyframeInterval.fixed(keyint)).with_skip_threshold(skip_threshold)
          .with_pipeline_depth(4))
    oc = O.default_config(w, h, 30)
    oc.intra_quality, oc.inter_quality = iq, pq
    oc.keyframe_mode, oc.keyframe_interval = 2, keyint
    oc.skip_threshold = skip_threshold
    return gc, oc


@pytest.mark.parametrize("iq,pq,keyint,skip_threshold", [(85, 80, 1 << 40, 3), (95, 90, 4, 3), (85, 80, 1 << 40, 0)])
def test_frame_stats_match_oracle(iq, pq, keyint, skip_threshold):
    from riv2_b200 import encoder as E
    from riv2_b200.synth import SynthClip
    w, h, n = 352, 288, 8
    clip = SynthClip("cif", seed=71 + pq)
    gc, oc = _pair(w, h, iq, pq, keyint, skip_threshold)
    enc = E.Encoder.new(gc, E.VecWriter())
    oe = O.OracleEncoder(oc)
    for t in range(n):
        f = clip.frame(t)
        g = enc.encode_frame_with_stats(E.Frame(f, w, h, t * 33))
        assert oe.encode_rgb(f, t * 33) == 0
        o = oe.last_stats()
        assert g.frame_index == t and g.timestamp_ms == t * 33
        assert (g.storage_width, g.storage_height) == (w, h)
        for name, want in o.items():
            got = getattr(g, name)
            if isinstance(want, tuple):
                assert tuple(float(x) for x in got) == want, f"frame {t}: {name} {got} != {want}"
            elif want is None:
                assert got is None, f"frame {t}: {name} {got} is not None"
            else:
                assert float(got) == want, f"frame {t}: {name} {got} != {want}"
    enc.finish()
    assert enc.writer.into_inner() == oe.finish()
    enc.close()
