"""Held-out evaluation of the learned encode form against the plain form.

For each held-out seeded clip: encode it with the plain form (the reference-identical path),
the learned form (the trained proposal network) and, for comparison, the parallel form (the
same parallel search without the network) and the learned form with an untrained network.
Every stream is decoded on the GPU (riv_decoder_*, bit-exact with the reference decoder's
restatement) and compared with the encoder's input planes:

* PSNR-Y: mean over frames of 10 log10(255^2 / MSE) of the luma plane (display area);
* bitrate: the stream's size; Delta-bitrate = size / plain size - 1;
* fallback rate: share of P-frame MBs whose proposals lost to the predictors by more than the
  margin and were searched by the hexagon search instead.

    python -m riv2_b200.eval_proposal --weights riv2_b200/weights/proposal.bin \\
        --preset 1080p --seeds 16 --frames 120 --out eval.json

Held-out seeds are 2026 + k (training clips use seeds from 1,000,000).
"""
from __future__ import annotations

import argparse
import json
import time

import numpy as np

EVAL_SEED_BASE = 2026


def _psnr(a: np.ndarray, b: np.ndarray) -> float:
    d = a.astype(np.float64) - b.astype(np.float64)
    mse = float(np.mean(d * d))
    return 99.0 if mse == 0 else 10.0 * np.log10(255.0 * 255.0 / mse)


def encode_clip(frames_y, rgb_frames, w, h, form, params=None, quality=(85, 80), sr=12, margin=256, depth=16):
    """Encode one clip; returns (stream bytes, learned counters, per-frame PSNR-Y)."""
    from . import decoder as D
    from . import encoder as E
    cfg = (E.EncoderConfig.new(w, h, 30).with_intra_quality(quality[0]).with_inter_quality(quality[1])
           .with_search_range(sr).with_keyframe_interval(E.KeyframeInterval.fixed(1 << 40))
           .with_pipeline_depth(depth).with_encode_form(form).with_proposal_margin(margin))
    wr = E.VecWriter()
    enc = E.Encoder.new(cfg, wr)
    if form == 1:
        enc.set_proposal(params)
    for t, f in enumerate(rgb_frames):
        enc.encode_frame(E.Frame(f, w, h, t * 33))
    enc.finish()
    counters = enc.learned_counters()
    enc.close()
    stream = wr.into_inner()
    dec = D.Decoder.new(stream)
    psnr = []
    for t in range(len(rgb_frames)):
        y = dec.decode_frame().y
        psnr.append(_psnr(y[:h, :w], frames_y[t][:h, :w]))
    dec.close()
    return stream, counters, psnr


def evaluate(weights: str, preset: str = "1080p", seeds: int = 16, frames: int = 120, quality=(85, 80), margin=256,
             seed_base: int = EVAL_SEED_BASE, forms=("plain", "learned", "parallel", "untrained"), verbose=True):
    from . import encoder as E
    from . import proposal as P
    from .synth import SynthClip
    params = P.load_params(weights) if weights else None
    untrained = P.init_params(0)
    rows = []
    t0 = time.time()
    for k in range(seeds):
        clip = SynthClip(preset, seed=seed_base + k)
        w, h = clip.width, clip.height
        sw, sh = (w + 15) // 16 * 16, (h + 15) // 16 * 16
        rgb = [clip.frame(t) for t in range(frames)]
        ys = [E.stage_rgb_to_yuv(f, w, h, sw, sh)[: sw * sh].reshape(sh, sw) for f in rgb]
        row = {"seed": seed_base + k}
        for form in forms:
            fid = {"plain": 0, "learned": 1, "parallel": 2, "untrained": 1}[form]
            p = untrained if form == "untrained" else params
            if fid == 1 and p is None:
                continue
            stream, c, ps = encode_clip(ys, rgb, w, h, fid, p, quality, margin=margin)
            row[form] = {"bytes": len(stream), "psnr_y": float(np.mean(ps)), "mbs": c["mbs"],
                         "fallbacks": c["fallbacks"], "shortcuts": c["shortcuts"]}
        rows.append(row)
        if verbose:
            msg = "  ".join(f"{f}: {row[f]['bytes']} B {row[f]['psnr_y']:.3f} dB" for f in forms if f in row)
            print(f"seed {row['seed']}: {msg}  ({time.time() - t0:.0f} s)", flush=True)
    summary = {}
    for form in forms:
        if form == "plain" or form not in rows[0]:
            continue
        db = [r[form]["psnr_y"] - r["plain"]["psnr_y"] for r in rows]
        br = [r[form]["bytes"] / r["plain"]["bytes"] - 1.0 for r in rows]
        mbs = sum(r[form]["mbs"] for r in rows)
        summary[form] = {"delta_psnr_db_mean": float(np.mean(db)), "delta_psnr_db_min": float(np.min(db)),
                         "delta_bitrate_mean": float(np.mean(br)), "delta_bitrate_max": float(np.max(br)),
                         "fallback_rate": (sum(r[form]["fallbacks"] for r in rows) / mbs) if mbs else None,
                         "shortcut_rate": (sum(r[form]["shortcuts"] for r in rows) / mbs) if mbs else None}
    return {"preset": preset, "seeds": seeds, "frames": frames, "quality": list(quality), "margin": margin,
            "rows": rows, "summary": summary}


def main():
    ap = argparse.ArgumentParser(description=__doc__, formatter_class=argparse.RawDescriptionHelpFormatter)
    ap.add_argument("--weights", required=True)
    ap.add_argument("--preset", default="1080p")
    ap.add_argument("--seeds", type=int, default=16)
    ap.add_argument("--frames", type=int, default=120)
    ap.add_argument("--quality", default="85,80")
    ap.add_argument("--margin", type=int, default=256)
    ap.add_argument("--out", default=None)
    a = ap.parse_args()
    q = tuple(int(v) for v in a.quality.split(","))
    res = evaluate(a.weights, a.preset, a.seeds, a.frames, q, a.margin)
    print(json.dumps(res["summary"], indent=1))
    if a.out:
        with open(a.out, "w") as f:
            json.dump(res, f, indent=1)


if __name__ == "__main__":
    main()
