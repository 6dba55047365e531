"""CPU tests: the oracle pinned against the reference's own constants and known-answer
tests, its encoder/decoder self-consistency, and the host side of the C ABI."""
import json
import os
import re

import numpy as np
import pytest

from oracle import oracle as O

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
GOLD = json.load(open(os.path.join(ROOT, "tests", "golden", "reference_constants.json")))
CSRC = os.path.join(ROOT, "riv2_b200", "csrc")


# ---------------------------------------------------------------------------------------
# Reference constants (tests/golden, extracted from the reference sources)
# ---------------------------------------------------------------------------------------

def test_dct_tables_equal_reference():
    from riv2_b200.encoder import dct_tables
    t16, t8 = dct_tables()
    assert t16.reshape(-1).tolist() == GOLD["fdct16"]
    assert t8.reshape(-1).tolist() == GOLD["fdct8"]
    # IDCT_ROWS_16[i][x] is the transpose of FDCT_TRANSPOSE_16 (both used by the device)
    assert t16.T.reshape(-1).tolist() == GOLD["idct16"]


AAN_ORDER = ["F2F_0541", "F2F_1848", "F2F_0765", "F2F_1176", "F2F_0299", "F2F_2053", "F2F_3073", "F2F_1501",
             "F2F_0900", "F2F_2563", "F2F_1962", "F2F_0390"]


@pytest.mark.parametrize("path,pattern", [
    ("riv2_b200/csrc/riv_kernels.cu", r"aan_1d\(const int32_t s\[8\].*?\n}\n"),
    ("oracle/riv_oracle.cpp", r"static const int32_t K0541.*?;"),
])
def test_aan_constants_equal_reference(path, pattern):
    src = open(os.path.join(ROOT, path)).read()
    seg = re.search(pattern, src, re.S).group(0)
    nums = [int(x) for x in re.findall(r"(?<![\w.])-?\d{3,5}(?![\w.])", seg)]
    want = [GOLD["aan"][k] for k in AAN_ORDER]
    for v in want:
        assert v in nums, (path, v)


@pytest.mark.parametrize("path", ["riv2_b200/csrc/riv_host.cpp", "oracle/riv_oracle.cpp"])
def test_jpeg_tables_equal_reference(path):
    src = open(os.path.join(ROOT, path)).read()
    for name, key in (("JPEG_LUMA", "jpeg_luma"), ("JPEG_CHROMA", "jpeg_chroma")):
        seg = re.search(name + r"\[64\] = \{(.*?)\};", src, re.S).group(1)
        assert [float(x) for x in re.findall(r"\d+", seg)] == GOLD[key]


def test_scalar_constants_equal_reference():
    src = open(os.path.join(ROOT, "oracle", "riv_oracle.cpp")).read()
    hexs = re.search(r"HEX\[6\]\[2\] = \{(.*?)\};", src).group(1)
    assert [int(x) for x in re.findall(r"-?\d+", hexs)] == GOLD["hex_offsets"]
    card = re.search(r"CARD\[4\]\[2\] = \{(.*?)\};", src).group(1)
    assert [int(x) for x in re.findall(r"-?\d+", card)] == GOLD["cardinal_offsets"]
    assert f"BATCH = {GOLD['rans_batch']}" in src
    assert f"BATCH = {GOLD['rans_batch']}" in open(os.path.join(CSRC, "riv_entropy.cpp")).read()
    assert GOLD["quant_step_best_worst"] == [1.0, 112.0]
    assert abs(O.lib().oracle_quant_step(1) - 112.0) < 1e-6 and abs(O.lib().oracle_quant_step(100) - 1.0) < 1e-6


# ---------------------------------------------------------------------------------------
# Deblock known-answer tests (com/deblock.rs:205-290), restated
# ---------------------------------------------------------------------------------------

def flat_frame(w, h, left, right):
    f = O.Frames(w, h)
    f.y[:, : w // 2] = left
    f.y[:, w // 2:] = right
    f.u[:] = 128
    f.v[:] = 128
    return f


def test_deblock_small_step_is_smoothed_wide():
    y = O.deblock(flat_frame(32, 32, 100, 106), 20, False).y[0]
    assert y[15] > 100 and y[16] < 106
    assert 100 <= y[14] <= y[15] and y[16] <= y[17] <= 106
    assert y[8] == 100 and y[24] == 106


def test_deblock_large_step_is_preserved():
    y = O.deblock(flat_frame(32, 32, 40, 200), 20, False).y[0]
    assert y[15] == 40 and y[16] == 200


def test_deblock_rough_interior_blocks_filtering():
    f = flat_frame(32, 32, 100, 106)
    f.y[:, 13] = 160
    y = O.deblock(f, 8, False).y[0]
    assert y[15] == 100 and y[16] == 106


def test_deblock_masked_static_blocks_untouched():
    y = O.deblock(flat_frame(32, 32, 100, 106), 20, False, mask=[0, 0, 0, 0]).y[0]
    assert y[15] == 100 and y[16] == 106


def test_deblock_edge_filtered_if_either_side_coded():
    y = O.deblock(flat_frame(32, 32, 100, 106), 20, False, mask=[0, 1, 0, 1]).y[0]
    assert y[15] > 100 and y[16] < 106


def test_deblock_zero_level_is_noop():
    f = flat_frame(32, 32, 100, 106)
    assert O.deblock(f, 0, False).equal(f)


# ---------------------------------------------------------------------------------------
# Transforms, SAD paths, prediction, rANS
# ---------------------------------------------------------------------------------------

def test_dct_roundtrip_tolerance():
    """dct16/dct8 encode + decode stay close to the input (dct/tests/roundtrip.rs)."""
    rng = np.random.default_rng(7)
    L = O.lib()
    for _ in range(20):
        blk = rng.integers(-255, 256, 256).astype(np.int16)
        q = np.zeros(256, np.int16)
        r = np.zeros(256, np.int16)
        L.oracle_fdct16_quant(O.i16(blk), 1.0, 0.5, O.i16(q))
        L.oracle_idct16_aq(O.i16(q), 1.0, O.i16(r))
        assert np.abs(r.astype(int) - blk).max() <= 2
        b8 = rng.integers(-255, 256, 64).astype(np.int16)
        q8 = np.zeros(64, np.int16)
        r8 = np.zeros(64, np.int16)
        L.oracle_fdct8_quant(O.i16(b8), 8.0, 0.5, O.i16(q8))
        L.oracle_idct8_aq(O.i16(q8), 8.0, O.i16(r8))
        assert np.abs(r8.astype(int) - b8).max() <= 25  # fast_dct8.rs:367-393 tolerance


def gradient_luma(w, h):
    """enc/motion/tests.rs:9-28: gradient RGB frame reduced to (77R+150G+29B)>>8."""
    y, x = np.mgrid[0:h, 0:w]
    r = (x * 3) % 256
    g = (y * 5) % 256
    b = ((x + y) * 7) % 256
    return np.ascontiguousarray(((r * 77 + g * 150 + b * 29) >> 8).astype(np.uint8))


def test_sad_scalar_equals_simd_paths():
    """The reference's scalar and SIMD SAD kernels agree; so must their restatements."""
    w = h = 64
    rng = np.random.default_rng(1)
    prev = gradient_luma(w, h)
    curr = np.ascontiguousarray(np.roll(prev, (1, 2), (0, 1)) ^ rng.integers(0, 4, (h, w)).astype(np.uint8))
    L = O.lib()
    big = 2 ** 62
    for x0 in (0, 16, 32, 48):
        for y0 in (0, 16, 48):
            for dx in (-12, -3, 0, 5, 12):
                for dy in (-12, 0, 7):
                    a = L.oracle_sad_int(O.u8(prev), O.u8(curr), w, h, x0, y0, dx, dy, big, 0)
                    b = L.oracle_sad_int(O.u8(prev), O.u8(curr), w, h, x0, y0, dx, dy, big, 1)
                    assert a == b
                    ah = L.oracle_sad_halfpel(O.u8(prev), O.u8(curr), w, h, x0, y0, 2 * dx + 1, 2 * dy - 1, big, 0)
                    bh = L.oracle_sad_halfpel(O.u8(prev), O.u8(curr), w, h, x0, y0, 2 * dx + 1, 2 * dy - 1, big, 1)
                    assert ah == bh


def test_halfpel_sad_detects_shift_and_limit():
    """enc/motion/tests.rs:30-102."""
    w = h = 32
    luma = gradient_luma(w, h)
    L = O.lib()
    big = 2 ** 62
    assert L.oracle_sad_halfpel(O.u8(luma), O.u8(luma), w, h, 8, 8, 0, 0, big, 1) == 0
    assert L.oracle_sad_halfpel(O.u8(luma), O.u8(luma), w, h, 8, 8, 1, 0, big, 1) > 0
    full = L.oracle_sad_halfpel(O.u8(luma), O.u8(np.ascontiguousarray(255 - luma)), w, h, 8, 5, 1, 1, big, 1)
    lim = max(full // 4, 1)
    part = L.oracle_sad_halfpel(O.u8(luma), O.u8(np.ascontiguousarray(255 - luma)), w, h, 8, 5, 1, 1, lim, 1)
    assert lim <= part <= full


@pytest.mark.parametrize("w,h", [(640, 368), (1280, 720)])
def test_build_predicted_fast_equals_scalar(w, h):
    """tests/fast_pred.rs:35-56 (luma), extended to chroma."""
    prev = O.Frames(w, h)
    idx = np.arange(w * h)
    prev.y[:] = ((idx * 31 + 7) % 256).reshape(h, w)
    ci = np.arange((w // 2) * (h // 2))
    prev.u[:] = ((ci * 17 + 3) % 256).reshape(h // 2, w // 2)
    prev.v[:] = ((ci * 13 + 11) % 256).reshape(h // 2, w // 2)
    nmb = (w // 16) * (h // 16)
    for dxh, dyh in [(0, 0), (1, 0), (0, 1), (1, 1), (2, 2), (3, 1), (-1, 0), (-2, 0), (-3, 1)]:
        mv = np.array([int(dxh / 2), int(dyh / 2), int(np.fmod(dxh, 2)), int(np.fmod(dyh, 2))], np.int8)
        mvs = np.ascontiguousarray(np.tile(mv, (nmb, 1)))
        a = O.build_predicted(prev, mvs)
        b = O.build_predicted(prev, mvs, reference=True)
        assert np.array_equal(a.y, b.y), (dxh, dyh)
        assert np.array_equal(a.u, b.u) and np.array_equal(a.v, b.v), (dxh, dyh)


def test_rans_roundtrip():
    rng = np.random.default_rng(3)
    for n in (1, 2, 3, 1000, 16386, 16387, 40000):
        bits = (rng.random(n) < 0.2).astype(np.uint8)
        byp = (rng.random(n) < 0.3).astype(np.uint8)
        out = np.zeros(n, np.uint8)
        O.lib().oracle_rans_roundtrip(O.u8(bits), O.u8(byp), n, O.u8(out), None, 0)
        assert np.array_equal(bits, out), n


# ---------------------------------------------------------------------------------------
# Encoder / decoder self-consistency ("reitero_decode reproduces the encoder recon")
# ---------------------------------------------------------------------------------------

def encode_clip(cfg, frames):
    enc = O.OracleEncoder(cfg)
    recons = []
    for t, f in enumerate(frames):
        assert enc.encode_rgb(f, t * 33) == 0
        recons.append(enc.last("recon"))
    return enc.finish(), recons


def check_decodes(stream, recons):
    dec = O.OracleDecoder(stream)
    assert dec.frame_count == len(recons)
    for r in recons:
        typ, f = dec.next()
        assert typ in (1, 2)
        assert f.equal(r)
    assert dec.next()[0] < 0


@pytest.mark.parametrize("variant", ["default", "intra_every_3", "all_intra", "sr31_thresholds", "odd_dims", "q95"])
def test_oracle_encoder_decoder_consistent(variant):
    from riv2_b200.synth import SynthClip
    w, h = (100, 70) if variant == "odd_dims" else (352, 288)
    clip = SynthClip("cif", seed=11, width=w, height=h)
    frames = [clip.frame(t) for t in range(5)]
    cfg = O.default_config(w, h, 30)
    cfg.intra_quality, cfg.inter_quality = 85, 80
    cfg.keyframe_mode, cfg.keyframe_interval = 2, 1000
    if variant == "intra_every_3":
        cfg.keyframe_interval = 3
    elif variant == "all_intra":
        cfg.keyframe_mode = 0
    elif variant == "sr31_thresholds":
        cfg.search_range = 31
        cfg.me_zero_mv_threshold = 300
        cfg.me_predictor_threshold = 800
    elif variant == "q95":
        cfg.intra_quality, cfg.inter_quality = 95, 90
    stream, recons = encode_clip(cfg, frames)
    assert stream[:4] == b"RIV\0"
    check_decodes(stream, recons)


def test_oracle_rejects_bad_config():
    cfg = O.default_config(0, 10, 30)
    with pytest.raises(ValueError):
        O.OracleEncoder(cfg)
    cfg = O.default_config(64, 64, 30)
    cfg.keyframe_interval = 0
    with pytest.raises(ValueError):
        O.OracleEncoder(cfg)


# ---------------------------------------------------------------------------------------
# Host side of the C ABI (no device calls)
# ---------------------------------------------------------------------------------------

def test_cabi_exports_every_declared_symbol():
    from riv2_b200 import encoder as E
    from riv2_b200 import proposal as P
    for name, listed in (("riv_gpu.h", E.EXPORTED_SYMBOLS), ("riv_nn.h", P.EXPORTED_SYMBOLS)):
        header = open(os.path.join(ROOT, "include", name)).read()
        declared = set(re.findall(r"\b(riv_\w+)\s*\(", header))
        assert declared == set(listed), name
        L = E.lib()
        for s in declared:
            assert getattr(L, s) is not None


def test_cabi_config_default_and_validation():
    import ctypes as C

    from riv2_b200 import encoder as E
    c = E.RivConfig()
    E.lib().riv_config_default(C.byref(c), 1920, 1080, 50)
    assert (c.storage_width, c.storage_height) == (1920, 1088)
    assert (c.intra_quality, c.inter_quality, c.search_range, c.skip_threshold) == (90, 35, 12, 3)
    assert abs(c.rdo_lambda_mult - 0.49) < 1e-12 and abs(c.inter_dead_zone - 0.75) < 1e-7
    assert (c.keyframe_mode, c.keyframe_interval) == (2, 30)
    w = E.VecWriter()
    h = C.c_void_p()
    bad = E.RivConfig()
    E.lib().riv_config_default(C.byref(bad), 64, 64, 0)  # fps 0 -> InvalidConfig before any device call
    vt = w.vtable()
    assert E.lib().riv_encoder_new(C.byref(bad), C.byref(vt), C.byref(h)) == 2
    with pytest.raises(E.InvalidConfig):
        E.EncoderConfig.new(64, 64, 30).with_search_range(200).validate()
    with pytest.raises(E.InvalidConfig):
        E.EncoderConfig.new(64, 64, 30).with_keyframe_interval(E.KeyframeInterval.fixed(0)).validate()


def test_libm_fixup_tables_load_on_host():
    """The glibc fix-up tables load without a device (the coefficient coder itself is pinned
    against the oracle in test_entropy_host.py, the MV coder by the GPU parity tests)."""
    from riv2_b200.encoder import libm_fixup_counts
    nlog, nexp = libm_fixup_counts()
    assert 1000 < nlog < 200000 and 1000 < nexp < 500000


def test_fdct_int32_accumulation_is_exact_for_reference_bases():
    """The device forward DCTs accumulate in int32 where the reference uses i64 and clamps to
    i32; that is exact only while every partial sum of both passes stays below 2^31 for
    residuals in [-255, 255].  Checked from the reference's own bases."""
    import numpy as np
    d = json.load(open(os.path.join(ROOT, "tests", "golden", "reference_constants.json")))
    for name, n in (("fdct16", 16), ("fdct8", 8)):
        T = np.array(d[name], dtype=np.int64).reshape(n, n)
        col = np.abs(T).sum(axis=0).max()          # largest sum over i of |T[i][j]|
        row_pass = 255 * col + (1 << 17)
        rows = row_pass >> 18
        col_pass = rows * col + (1 << 17)
        assert row_pass < 2 ** 31 and col_pass < 2 ** 31, (name, row_pass, col_pass)
