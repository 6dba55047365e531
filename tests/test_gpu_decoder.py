"""The GPU decoder (riv_decoder_*, riv2_b200.decoder) against the oracle's decoder: every frame
of streams written by the GPU encoder and by the oracle encoder decodes to the same planes,
which also equal the encoder's own reconstruction.  Header validation runs on the CPU."""
import numpy as np
import pytest

from oracle import oracle as O


def _stream(preset, n, w, h, fps=30, iq=85, pq=80, keyint=1000, **kw):
    from riv2_b200 import encoder as E
    from riv2_b200.synth import SynthClip
    clip = SynthClip(preset, seed=4, width=w, height=h)
    cfg = (E.EncoderConfig.new(w, h, fps).with_intra_quality(iq).with_inter_quality(pq)
           .with_keyframe_interval(E.KeyframeInterval.fixed(keyint)))
    for k, v in kw.items():
        cfg = cfg._with(**{k: v})
    wr = E.VecWriter()
    enc = E.Encoder.new(cfg, wr)
    recons = []
    for t in range(n):
        enc.encode_frame(E.Frame(clip.frame(t), w, h, t * 1000 // fps))
        recons.append(enc.last_recon())
    enc.finish()
    data = wr.into_inner()
    enc.close()
    return data, recons


def _decode_all_and_compare(data, recons=None):
    from riv2_b200.decoder import Decoder, EndOfStream
    dec = Decoder.new(data)
    odec = O.OracleDecoder(data)
    hd = dec.header()
    assert (hd.storage_width, hd.storage_height, hd.frame_count) == (odec.sw, odec.sh, odec.frame_count)
    for t in range(hd.frame_count):
        f = dec.decode_frame()
        typ, o = odec.next()
        assert f.frame_type == typ and f.frame_index == t
        assert np.array_equal(f.y, o.y) and np.array_equal(f.u, o.u) and np.array_equal(f.v, o.v), t
        if recons is not None:
            y, u, v = recons[t]
            assert np.array_equal(f.y, y) and np.array_equal(f.u, u) and np.array_equal(f.v, v), t
    assert not dec.has_more_frames()
    with pytest.raises(EndOfStream):
        dec.decode_frame()
    dec.close()


def test_decoder_rejects_bad_headers():
    from riv2_b200.decoder import Decoder, InvalidHeader
    with pytest.raises(InvalidHeader):
        Decoder.new(b"RIFF" + bytes(40))
    with pytest.raises(InvalidHeader):
        Decoder.new(b"RIV\x00" + bytes(8))
    bad_dims = bytearray(b"RIV\x00" + (5).to_bytes(4, "little") + bytes(28))
    bad_dims[16:20] = (100).to_bytes(4, "little")  # storage width not a multiple of 16
    bad_dims[20:24] = (64).to_bytes(4, "little")
    with pytest.raises(InvalidHeader):
        Decoder.new(bytes(bad_dims))


@pytest.mark.gpu
def test_decode_gpu_stream_cif():
    data, recons = _stream("cif", 10, 352, 288)
    _decode_all_and_compare(data, recons)


@pytest.mark.gpu
@pytest.mark.parametrize("variant", ["q95", "keyint3", "skip0", "odd_dims", "sr31", "thresholds"])
def test_decode_gpu_stream_variants(variant):
    kw = {}
    w, h, iq, pq, keyint = 352, 288, 85, 80, 1000
    if variant == "q95":
        iq, pq = 95, 90
    elif variant == "keyint3":
        keyint = 3
    elif variant == "skip0":
        kw["skip_threshold"] = 0
    elif variant == "odd_dims":
        w, h = 100, 70
    elif variant == "sr31":
        kw["search_range"] = 31
    elif variant == "thresholds":
        kw["me_zero_mv_threshold"] = 400
        kw["me_predictor_threshold"] = 900
    data, recons = _stream("cif", 7, w, h, iq=iq, pq=pq, keyint=keyint, **kw)
    _decode_all_and_compare(data, recons)


@pytest.mark.gpu
def test_decode_oracle_stream():
    from riv2_b200.synth import SynthClip
    clip = SynthClip("cif", seed=8)
    oc = O.default_config(352, 288, 30)
    oc.intra_quality, oc.inter_quality = 80, 70
    oc.keyframe_mode, oc.keyframe_interval = 2, 4
    enc = O.OracleEncoder(oc)
    for t in range(9):
        assert enc.encode_rgb(clip.frame(t), t * 33) == 0
    _decode_all_and_compare(enc.finish())


@pytest.mark.gpu
def test_decode_1080p_120_frames():
    data, recons = _stream("1080p", 120, 1920, 1080, fps=50)
    _decode_all_and_compare(data, recons)


@pytest.mark.gpu
def test_decode_truncated_stream_reports_io():
    from riv2_b200.decoder import Decoder, IoError
    data, _ = _stream("cif", 3, 352, 288)
    dec = Decoder.new(data[: len(data) - 50])
    dec.decode_frame()
    dec.decode_frame()
    with pytest.raises(IoError):
        dec.decode_frame()
    dec.close()


def test_oracle_rgb_output_inverts_the_input_conversion():
    """The decoder's RGB output definition (BT.709 limited range, each chroma sample on its 2x2
    quad) inverts the input conversion: on colours constant over each 2x2 quad, RGB -> YUV ->
    RGB is within the limited-range quantisation (at most 3 levels per channel)."""
    rng = np.random.default_rng(1)
    quads = rng.integers(0, 256, (18, 22, 3), dtype=np.uint8)
    rgb = np.repeat(np.repeat(quads, 2, axis=0), 2, axis=1)  # 36 x 44, constant per quad
    f = O.rgb_to_yuv(rgb, 44, 36, 48, 48)
    back = O.yuv_to_rgb(f, 44, 36)
    assert back.shape == (36, 44, 3)
    assert np.abs(back.astype(int) - rgb.astype(int)).max() <= 3


@pytest.mark.gpu
@pytest.mark.parametrize("w,h", [(352, 288), (100, 70)])
def test_decode_rgb_output_matches_oracle(w, h):
    from riv2_b200.decoder import Decoder
    data, _ = _stream("cif", 5, w, h, keyint=3)
    dec = Decoder.new(data)
    odec = O.OracleDecoder(data)
    for t in range(5):
        f = dec.decode_frame_rgb()
        typ, o = odec.next()
        assert f.frame_index == t and f.frame_type == typ and f.rgb.shape == (h, w, 3)
        assert np.array_equal(f.rgb, O.yuv_to_rgb(o, w, h)), t
    dec.close()
