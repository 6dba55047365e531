"""Training of the motion-proposal network on records logged by the plain GPU encoder.

Records: for every P-frame of seeded synthetic clips, every MB's network input, computed on
the GPU by the same kernel and from the same planes the learned encoder uses (the correlation
volume of the current input block against the previous frame's input planes, the predictor
prior map and values from the coded MVs of the frame two back: the encoder runs the network of
frame t while frame t-1 is still being reconstructed), and the plain encoder's choice for it
(its search MV in half-pel units and its RDO skip decision).  The plain encoder is the
reference-identical path, so the network learns to propose what the reference's search would
pick.

Training: AdamW (lr 1e-3, batch 4096 MBs) with this library's forward, backward and optimizer
kernels (riv2_b200.proposal); the parameters are written with proposal.save_params.

    python -m riv2_b200.train_proposal --clips 256 --frames 11 --steps 3000 \\
        --out riv2_b200/weights/proposal.bin

Clip seeds start at 1_000_000 so that they never coincide with the evaluation clips' seeds.
"""
from __future__ import annotations

import argparse
import json
import time

import numpy as np

TRAIN_SEED_BASE = 1_000_000


def log_records(clips: int, frames: int, preset: str = "720p", keep: float = 1.0, quality=(85, 80), sr: int = 12,
                seed_base: int = TRAIN_SEED_BASE, device: int = 0, verbose: bool = True):
    """Encode `clips` seeded clips of `frames` frames with the plain encoder and return device
    tensors (feat n x 24 x 24 x 2 bf16, x1 n x 320 bf16, tmv n x 2 i16, tskip n u8) for a
    random `keep` fraction of the P-frame MBs."""
    import torch

    from . import encoder as E
    from . import proposal as P
    from .synth import SynthClip
    dev = torch.device("cuda", device)
    rng = np.random.default_rng(seed_base)
    feats, x1s, tmvs, tskips = [], [], [], []
    t0 = time.time()
    for ci in range(clips):
        clip = SynthClip(preset, seed=seed_base + ci)
        w, h = clip.width, clip.height
        cfg = (E.EncoderConfig.new(w, h, 30).with_intra_quality(quality[0]).with_inter_quality(quality[1])
               .with_search_range(sr).with_keyframe_interval(E.KeyframeInterval.fixed(1 << 40)).with_pipeline_depth(0))
        enc = E.Encoder.new(cfg, E.VecWriter())
        sw, sh = cfg.storage_width, cfg.storage_height
        nmb = (sw // 16) * (sh // 16)
        prev_in, coded1, coded2 = None, None, None  # input luma of t-1; coded MVs of t-1 and t-2
        for t in range(frames):
            enc.encode_frame(E.Frame(clip.frame(t), w, h, t * 33))
            cur = np.ascontiguousarray(enc.debug_state(3)[: sw * sh])
            coded_t = None
            if t >= 1:
                mbo = enc.debug_state(0).reshape(nmb, 20)
                raw = mbo[:, 0:4].view(np.int8).astype(np.int16)
                keep_idx = np.nonzero(rng.random(nmb) < keep)[0].astype(np.int64)
                if keep_idx.size:
                    cur_d = torch.from_numpy(cur).to(dev)
                    ref_d = torch.from_numpy(prev_in).to(dev)
                    pc_d = None if coded2 is None else torch.from_numpy(coded2).to(dev)
                    f = torch.empty((nmb, 24, 24, 2), dtype=torch.bfloat16, device=dev)
                    x = torch.zeros((nmb, 320), dtype=torch.bfloat16, device=dev)
                    rc = P.lib().riv_nn_features(cur_d.data_ptr(), ref_d.data_ptr(), sw, sh,
                                                 None if pc_d is None else pc_d.data_ptr(), 0, nmb, f.data_ptr(),
                                                 x.data_ptr(), None)
                    if rc:
                        raise RuntimeError(f"riv_nn_features failed ({rc})")
                    ki = torch.from_numpy(keep_idx).to(dev)
                    feats.append(f.index_select(0, ki))
                    x1s.append(x.index_select(0, ki))
                    tm = np.stack([2 * raw[:, 0] + raw[:, 2], 2 * raw[:, 1] + raw[:, 3]], axis=1).astype(np.int16)
                    tmvs.append(torch.from_numpy(tm[keep_idx]).to(dev))
                    tskips.append(torch.from_numpy(mbo[keep_idx, 13].copy()).to(dev))  # rdo_skip byte
                coded_t = np.ascontiguousarray(mbo[:, 4:8].view(np.int8))
            coded1, coded2 = coded_t, coded1
            prev_in = cur
        enc.close()
        if verbose and (ci + 1) % 16 == 0:
            print(f"  logged {ci + 1}/{clips} clips ({time.time() - t0:.1f} s)", flush=True)
    return (torch.cat(feats), torch.cat(x1s), torch.cat(tmvs), torch.cat(tskips))


def train(data, steps: int, batch: int = 4096, lr: float = 1e-3, seed: int = 0, params=None, log_every: int = 100,
          verbose: bool = True):
    """AdamW over `steps` batches drawn without replacement per epoch; returns (net, losses)."""
    import torch

    from . import proposal as P
    feat, x1, tmv, tskip = data
    n = feat.shape[0]
    net = P.ProposalNet(params, seed=seed, device=feat.device.index or 0)
    g = torch.Generator(device="cpu").manual_seed(seed)
    perm = torch.randperm(n, generator=g).to(feat.device)
    pos = 0
    losses = []
    fb = net.buf("train_feat", (batch, 24, 24, 2), torch.bfloat16)
    xb = net.buf("train_x1", (batch, 320), torch.bfloat16)
    mb = net.buf("train_tmv", (batch, 2), torch.int16)
    sb = net.buf("train_skip", (batch,), torch.uint8)
    t0 = time.time()
    for step in range(steps):
        if pos + batch > n:
            perm = torch.randperm(n, generator=g).to(feat.device)
            pos = 0
        idx = perm[pos:pos + batch]
        pos += batch
        torch.index_select(feat, 0, idx, out=fb)
        torch.index_select(x1, 0, idx, out=xb)
        torch.index_select(tmv, 0, idx, out=mb)
        torch.index_select(tskip, 0, idx, out=sb)
        loss = net.train_step(fb, xb, mb, sb, lr=lr)
        if step % log_every == 0 or step == steps - 1:
            v = loss.item() / batch
            losses.append((step, v))
            if verbose:
                print(f"  step {step:5d}  loss {v:.4f}  ({time.time() - t0:.1f} s)", flush=True)
    net.check()
    return net, losses


def main():
    ap = argparse.ArgumentParser(description=__doc__, formatter_class=argparse.RawDescriptionHelpFormatter)
    ap.add_argument("--clips", type=int, default=256)
    ap.add_argument("--frames", type=int, default=11)
    ap.add_argument("--preset", default="720p")
    ap.add_argument("--keep", type=float, default=1.0)
    ap.add_argument("--steps", type=int, default=3000)
    ap.add_argument("--batch", type=int, default=4096)
    ap.add_argument("--lr", type=float, default=1e-3)
    ap.add_argument("--out", required=True)
    ap.add_argument("--log", default=None, help="JSON file for the loss curve and data sizes")
    a = ap.parse_args()
    from . import proposal as P
    t0 = time.time()
    data = log_records(a.clips, a.frames, a.preset, a.keep)
    t1 = time.time()
    print(f"records: {data[0].shape[0]} MBs from {a.clips} clips in {t1 - t0:.1f} s", flush=True)
    net, losses = train(data, a.steps, a.batch, a.lr)
    t2 = time.time()
    P.save_params(a.out, net.params_numpy())
    print(f"trained {a.steps} steps in {t2 - t1:.1f} s; wrote {a.out}", flush=True)
    if a.log:
        with open(a.log, "w") as f:
            json.dump({"records": int(data[0].shape[0]), "clips": a.clips, "frames": a.frames, "preset": a.preset,
                       "steps": a.steps, "batch": a.batch, "lr": a.lr, "log_s": t1 - t0, "train_s": t2 - t1,
                       "loss": losses}, f, indent=1)


if __name__ == "__main__":
    main()
