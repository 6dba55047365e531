"""Failure paths on the GPU, made to happen without faulting, trapping or hanging a GPU.

* Bounded device waits give up: a test hook runs the search launch's wait helpers on flags
  nothing sets with a short spin limit; the call returns RIV_ERR_DEVICE_TIMEOUT (the status
  the encoder reports when a wavefront wait expires) and the context stays usable: an
  encode in the same process afterwards is byte-identical to the oracle's.
* The writer refuses one record (the reference's `writer.write(..)?`, enc/encoder.rs:249):
  the call that sees it raises Io, that record is lost, every later record is written and
  finish patches the header with the number written (enc/encoder.rs:950-961).
* A coefficient of magnitude class 14, which the reference's coefficient coder indexes past
  its models for (res/rans.rs:72-98: a panic), makes the encoder fail with EncodingFailed,
  as the oracle does.
"""
import numpy as np
import pytest

from oracle import oracle as O

pytestmark = pytest.mark.gpu


def _cif_configs(depth, iq=85, pq=80):
    from riv2_b200 import encoder as E
    gc = (E.EncoderConfig.new(352, 288, 30).with_intra_quality(iq).with_inter_quality(pq)
          .with_keyframe_interval(E.KeyframeInterval.fixed(1000)).with_pipeline_depth(depth))
    oc = O.default_config(352, 288, 30)
    oc.intra_quality, oc.inter_quality = iq, pq
    oc.keyframe_mode, oc.keyframe_interval = 2, 1000
    return gc, oc


@pytest.mark.parametrize("which", [0, 1, 2, 3], ids=["record", "counter", "handoff", "mbarrier"])
def test_bounded_wait_expires_and_the_context_stays_usable(which):
    import ctypes as C

    from riv2_b200 import encoder as E
    from riv2_b200.synth import SynthClip
    word = C.c_uint32(0)
    st = E.lib().riv_test_wait_expiry(which, 2000, C.byref(word))
    assert st == 7 and word.value & 1  # RIV_ERR_DEVICE_TIMEOUT, ST_WAIT_TIMEOUT
    clip = SynthClip("cif", seed=5)
    gc, oc = _cif_configs(depth=2)
    w = E.VecWriter()
    enc = E.Encoder.new(gc, w)
    oenc = O.OracleEncoder(oc)
    for t in range(3):
        f = clip.frame(t)
        enc.encode_frame(E.Frame(f, 352, 288, t * 33))
        assert oenc.encode_rgb(f, t * 33) == 0
    enc.finish()
    assert w.into_inner() == oenc.finish()
    enc.close()


def _refusing_writer(refuse):
    """An in-memory VideoWriter whose write number `refuse` (1 = the header) fails."""
    from riv2_b200 import encoder as E

    class RefusingWriter(E.VideoWriter):
        def __init__(self):
            self.buf, self.pos, self.calls = bytearray(), 0, 0

        def write(self, data):
            self.calls += 1
            if self.calls == refuse:
                raise OSError("refused by the test writer")
            self.buf[self.pos:self.pos + len(data)] = data
            self.pos += len(data)

        def position(self):
            return self.pos

        def seek(self, p):
            self.pos = p

        def flush(self):
            pass

    return RefusingWriter()


@pytest.mark.parametrize("depth", [0, 4])
def test_refused_record_is_dropped_and_later_frames_are_written(depth):
    from riv2_b200 import encoder as E
    from riv2_b200.synth import SynthClip
    n, dropped = 8, 3  # frame 3's record: write call 1 is the header, call 2 frame 0, ...
    clip = SynthClip("cif", seed=9)
    gc, oc = _cif_configs(depth)
    oenc = O.OracleEncoder(oc)
    records = []
    for t in range(n):
        assert oenc.encode_rgb(clip.frame(t), t * 33) == 0
        records.append(oenc.last_record())
    header = oenc.finish()[:36]
    wr = _refusing_writer(refuse=dropped + 2)
    enc = E.Encoder.new(gc, wr)
    errors = 0
    for t in range(n):
        try:
            enc.encode_frame(E.Frame(clip.frame(t), 352, 288, t * 33))
        except E.IoError:
            errors += 1
    try:
        enc.finish()
    except E.IoError:
        errors += 1
    enc.close()
    assert errors == 1
    want = bytearray(header)
    want[28:36] = (n - 1).to_bytes(8, "little")  # frame_count patched to the records written
    for t in range(n):
        if t != dropped:
            want += records[t]
    assert bytes(wr.buf) == bytes(want)


def _class14_frames():
    """Key frame: a 0/255 checkerboard with a flat 5x5-MB hole; P-frame: the hole's centre MB
    turned to 255.  Its prediction is flat (variance floor 4) while the frame's mean ln
    variance is near ln 16256, so at q 100 its AQ step is about 0.49 and its DC coefficient
    about 8400: magnitude class 14."""
    w, h = 352, 288
    yy, xx = np.mgrid[0:h, 0:w]
    y0 = np.where((yy + xx) % 2 == 0, 0, 255).astype(np.uint8)
    y0[5 * 16:10 * 16, 7 * 16:12 * 16] = 0
    y1 = y0.copy()
    y1[7 * 16:8 * 16, 9 * 16:10 * 16] = 255
    c = np.full((h // 2, w // 2), 128, np.uint8)
    return [(y0, c, c), (y1, c, c)]


@pytest.mark.parametrize("depth", [0, 4])
def test_magnitude_class_14_fails_like_the_reference(depth):
    from riv2_b200 import encoder as E
    gc, oc = _cif_configs(depth, iq=100, pq=100)
    oenc = O.OracleEncoder(oc)
    f = O.Frames(352, 288)
    st = []
    for t, (y, u, v) in enumerate(_class14_frames()):
        f.y[:], f.u[:], f.v[:] = y, u, v
        st.append(oenc.encode_yuv(f, t * 33))
    assert st == [0, 3]  # the oracle fails on the P-frame (EncodingFailed)
    enc = E.Encoder.new(gc, E.VecWriter())
    with pytest.raises(E.EncodingFailed):
        for t, (y, u, v) in enumerate(_class14_frames()):
            enc.encode_frame_yuv(y, u, v, t * 33)
        enc.finish()
    # the encoder stays failed
    with pytest.raises(E.EncodingFailed):
        enc.finish()
    enc.close()
