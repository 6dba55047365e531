"""Extract the reference's normative constants into tests/golden/reference_constants.json.

Run once where the reference sources are available (``python tests/golden/make_golden.py
/path/to/riv2``); the JSON is committed, so the tests never read the reference at run time.
The reference is Rust and cannot be built here, so its tables are read as text from:

* reitero_video/reitero_dct/src/dct16.rs      FDCT_TRANSPOSE_16, IDCT_ROWS_16
* reitero_video/reitero_dct/src/dct8.rs       FDCT_TRANSPOSE_8
* reitero_video/reitero_dct/src/fast_dct8.rs  F2F_* AAN constants
* reitero_video/reitero_residual/src/residual.rs  JPEG_LUMA_8X8, JPEG_CHROMA_8X8, AQ constants
* reitero_video/reitero_encode/src/motion/scalar.rs  HEX_OFFSETS, CARDINAL_OFFSETS
* reitero_video/reitero_video_common/src/rans.rs  BATCH, RANS_L
* reitero_video/reitero_video_common/src/deblock.rs  LEVEL_SCALE
"""
import json
import os
import re
import sys


def _ints(text):
    return [int(x) for x in re.findall(r"-?\d+", text)]


def _block(src, name):
    i = src.index(name)
    j = src.index("= [", i) + 2
    depth, k = 0, j
    while True:
        if src[k] == "[":
            depth += 1
        elif src[k] == "]":
            depth -= 1
            if depth == 0:
                return src[j:k + 1]
        k += 1


def main(root):
    rd = lambda *p: open(os.path.join(root, *p)).read()  # noqa: E731
    d16 = rd("reitero_video", "reitero_dct", "src", "dct16.rs")
    d8 = rd("reitero_video", "reitero_dct", "src", "dct8.rs")
    f8 = rd("reitero_video", "reitero_dct", "src", "fast_dct8.rs")
    res = rd("reitero_video", "reitero_residual", "src", "residual.rs")
    sc = rd("reitero_video", "reitero_encode", "src", "motion", "scalar.rs")
    rans = rd("reitero_video", "reitero_video_common", "src", "rans.rs")
    dbl = rd("reitero_video", "reitero_video_common", "src", "deblock.rs")
    strip = lambda t: re.sub(r"i32x8::new|i32x8", "", t)  # noqa: E731
    out = {
        "fdct16": _ints(strip(_block(d16, "const FDCT_TRANSPOSE_16"))),
        "idct16": _ints(strip(_block(d16, "const IDCT_ROWS_16"))),
        "fdct8": _ints(strip(_block(d8, "const FDCT_TRANSPOSE_8"))),
        "aan": {m.group(1): int(m.group(2)) for m in re.finditer(r"const (F2F_\w+): i32 = (-?\d+);", f8)},
        "jpeg_luma": [float(x) for x in re.findall(r"\d+\.\d+", _block(res, "const JPEG_LUMA_8X8"))],
        "jpeg_chroma": [float(x) for x in re.findall(r"\d+\.\d+", _block(res, "const JPEG_CHROMA_8X8"))],
        "aq_strength": float(re.search(r"AQ_STRENGTH_DEFAULT: f32 = ([\d.]+)", res).group(1)),
        "aq_min_variance": float(re.search(r"AQ_MIN_VARIANCE: f32 = ([\d.]+)", res).group(1)),
        "quant_step_best_worst": [float(re.search(r"BEST_QUALITY_QUANT_STEP: f32 = ([\d.]+)", res).group(1)),
                                  float(re.search(r"WORST_QUALITY_QUANT_STEP: f32 = ([\d.]+)", res).group(1))],
        "hex_offsets": _ints(re.search(r"HEX_OFFSETS: &\[\(i32, i32\)\] = (&\[.*?\]);", sc).group(1)),
        "cardinal_offsets": _ints(re.search(r"CARDINAL_OFFSETS: &\[\(i32, i32\)\] = (&\[.*?\]);", sc).group(1)),
        "rans_batch": int(re.search(r"const BATCH: usize = (\d+);", rans).group(1)),
        "deblock_level_scale": float(re.search(r"LEVEL_SCALE: f32 = ([\d.]+)", dbl).group(1)),
    }
    assert len(out["fdct16"]) == 256 and len(out["idct16"]) == 256 and len(out["fdct8"]) == 64
    assert len(out["jpeg_luma"]) == 64 and len(out["jpeg_chroma"]) == 64 and len(out["aan"]) == 12
    path = os.path.join(os.path.dirname(os.path.abspath(__file__)), "reference_constants.json")
    with open(path, "w") as f:
        json.dump(out, f, indent=1)
    print("wrote", path)


if __name__ == "__main__":
    if len(sys.argv) != 2:
        sys.exit("usage: make_golden.py <path of the riv2 reference checkout>")
    main(sys.argv[1])
