#!/usr/bin/env python3
"""Benchmark: 1080p P-frame encode throughput of the B200 riv2 encoder, learned-proposal form
against the plain form.

Workload: a seeded synthetic 1920x1080 RGB24 clip (16 rectangles, sides 64-384 px,
velocities +-16 px/frame at 0.5 px steps, pan +-4, noise sigma 2), quality 85/80, one
key frame at frame 0, encoder defaults otherwise (search range 12, skip threshold 3,
lambda multiplier 0.49, dead zone 0.75).  A step is one P-frame.

* ``value``: frames/s of the whole encode in the learned-proposal form (proposal network on
  the tensor cores, parallel proposal-seeded search, parallel mode decision; the network
  weights riv2_b200/weights/proposal.bin, trained by riv2_b200.train_proposal) with the RGB
  frames already resident in HBM.  ``plain`` holds the same for the plain form (the
  reference-identical path), and ``learned_vs_plain`` the fps ratio and the quality deltas
  of the two streams of the timed frames (PSNR-Y and size, both streams decoded on the GPU).
* ``e2e``: the same through ``riv_encode_frame`` with pinned host RGB buffers; the
  host->device copy of each frame and the device->host copy of its side info and
  coefficients are inside the timed region.
* ``roofline``: the plain form's dominant kernel (the search/mode wavefront), achieved
  bytes/s over its algorithmic bytes against the measured HBM copy bandwidth; the learned
  form's GPU stages are in ``learned_stage_us_per_pframe``.
* ``cpu_baseline``: the CPU oracle (single-threaded restatement of the reference encoder,
  library-default raster-serial search) on a bounded sample of the same clip.

``--impl reference`` times that CPU implementation alone (the reference itself is Rust
and cannot be built in this image): one stream on one thread (the encoder is serial within a
stream), plus, as ``cpu_all_cores``, every host thread (up to --cpu-workers) encoding an
independent stream of the clip at once.  Multi-GPU: one process per GPU, each encoding its
own clip (replicas, no collective), value = total frames / max time over ranks.
"""
from __future__ import annotations

import argparse
import json
import os
import statistics
import sys
import threading
import time

import numpy as np

ROOT = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, ROOT)

W_DISP, H_DISP, FPS = 1920, 1080, 50
MBS_PER_FRAME = (1920 // 16) * (1088 // 16)
# the headline metric this line reports: learned-proposal fps, with the plain form beside it
METRIC = "1080p encode fps: learned-proposal vs plain GPU at \u22640.1 dB PSNR, \u22642% bitrate"
WEIGHTS = os.path.join(ROOT, "riv2_b200", "weights", "proposal.bin")


def parse():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=100)
    ap.add_argument("--warmup", type=int, default=5)
    ap.add_argument("--impl", default="ours", choices=["ours", "reference"])
    ap.add_argument("--quality", default="85/80")
    ap.add_argument("--pipeline-depth", type=int, default=16)
    ap.add_argument("--seed", type=int, default=2026)
    ap.add_argument("--cpu-sample-frames", type=int, default=12)
    ap.add_argument("--cpu-workers", type=int, default=96, help="cap on the reference arm's host threads")
    ap.add_argument("--no-cpu-baseline", action="store_true")
    ap.add_argument("--weights", default=WEIGHTS)
    ap.add_argument("--no-secondary", action="store_true", help="skip the secondary measurement points")
    ap.add_argument("--batch-steps", type=int, default=12, help="timed steps of the multi-clip point (0: skip it)")
    ap.add_argument("--workload", default="single", choices=["single", "batch"],
                    help="batch: only the 64-clip multi-clip workload over its whole length, one JSON line")
    ap.add_argument("--margin", type=int, default=256, help="learned form: proposal fallback SAD margin")
    return ap.parse_args()


# ---------------------------------------------------------------------------------------
# distributed plumbing (replicas)
# ---------------------------------------------------------------------------------------

def dist_env():
    ws = int(os.environ.get("WORLD_SIZE", "1"))
    rank = int(os.environ.get("RANK", "0"))
    local = int(os.environ.get("LOCAL_RANK", "0"))
    return ws, rank, local


def init_dist(ws, backend):
    if ws <= 1:
        return None
    import datetime

    import torch.distributed as dist
    os.environ.setdefault("MASTER_ADDR", "127.0.0.1")
    dist.init_process_group(backend, timeout=datetime.timedelta(seconds=120))
    return dist


def max_over_ranks(x: float, dist, device=None) -> float:
    if dist is None:
        return x
    import torch
    t = torch.tensor([x], dtype=torch.float64, device=device)
    dist.all_reduce(t, op=dist.ReduceOp.MAX)
    return float(t.item())


def barrier(dist, device=None):
    if dist is not None:
        import torch
        t = torch.zeros(1, device=device)
        dist.all_reduce(t)


# ---------------------------------------------------------------------------------------
# clocks during the timed region
# ---------------------------------------------------------------------------------------

class ClockSampler:
    """Samples the SM clock and the clock-event reasons of the benchmarked GPU every
    ``period`` seconds while the timed region runs (NVML reads only; nothing is set).
    The GPU is found by its PCI bus id, so the sample is of the device CUDA uses even
    when CUDA_VISIBLE_DEVICES renumbers devices."""

    REASONS = (("hw_slowdown", 0x8), ("hw_thermal_slowdown", 0x40), ("sw_thermal_slowdown", 0x20),
               ("sw_power_cap", 0x4))

    def __init__(self, cuda_index: int, period: float = 0.02):
        self.idx, self.period = cuda_index, period
        self.samples, self.max_mhz = [], None
        self.stop_ev, self.t, self.nvml, self.h = threading.Event(), None, None, None

    def start(self):
        try:
            import pynvml
            import torch
            pynvml.nvmlInit()
            self.nvml = pynvml
            pr = torch.cuda.get_device_properties(self.idx)
            bus = "%08X:%02X:%02X.0" % (pr.pci_domain_id, pr.pci_bus_id, pr.pci_device_id)
            try:
                self.h = pynvml.nvmlDeviceGetHandleByPciBusId(bus)
            except Exception:
                self.h = pynvml.nvmlDeviceGetHandleByIndex(self.idx)
            self.max_mhz = float(pynvml.nvmlDeviceGetMaxClockInfo(self.h, pynvml.NVML_CLOCK_SM))
        except Exception:
            self.nvml = None
            return
        self.t = threading.Thread(target=self._run, daemon=True)
        self.t.start()

    def _run(self):
        while not self.stop_ev.is_set():
            try:
                mhz = self.nvml.nvmlDeviceGetClockInfo(self.h, self.nvml.NVML_CLOCK_SM)
                rs = self.nvml.nvmlDeviceGetCurrentClocksEventReasons(self.h)
                self.samples.append((float(mhz), int(rs)))
            except Exception:
                pass
            self.stop_ev.wait(self.period)

    def stop(self):
        self.stop_ev.set()
        if self.t:
            self.t.join(timeout=2)
        if self.nvml is not None:
            try:
                self.nvml.nvmlShutdown()
            except Exception:
                pass
        sm = [m for m, _ in self.samples]
        reasons = sorted({n for _, r in self.samples for n, bit in self.REASONS if r & bit})
        return {"sm_mhz": statistics.median(sm) if sm else None, "sm_max_mhz": self.max_mhz, "reasons": reasons,
                "samples": len(sm), "source": "nvml %d ms" % int(self.period * 1000)}


# ---------------------------------------------------------------------------------------
# workload
# ---------------------------------------------------------------------------------------

def make_frames(n: int, seed: int, clip: int) -> np.ndarray:
    from riv2_b200.synth import SynthClip
    return SynthClip("1080p", seed=seed, clip=clip).frames(n)


def entropy_threads() -> int:
    """Host threads per entropy pool of one encoder: the encoder's default (half the host) for
    one rank; with several ranks on the node each takes its share, so that N replicas do not
    oversubscribe the host N times."""
    local = int(os.environ.get("LOCAL_WORLD_SIZE", "1"))
    if local <= 1:
        return 0
    return max(2, min(16, (os.cpu_count() or 2) // (2 * local)))


def config(iq: int, pq: int, depth: int, device: int, form: int = 0, margin: int = 256):
    from riv2_b200 import encoder as E
    return (E.EncoderConfig.new(W_DISP, H_DISP, FPS).with_intra_quality(iq).with_inter_quality(pq)
            .with_keyframe_interval(E.KeyframeInterval.fixed(1 << 40)).with_pipeline_depth(depth).with_device(device)
            .with_encode_form(form).with_proposal_margin(margin).with_entropy_threads(entropy_threads()))


def psnr_y_of_stream(stream: bytes, src_y, dev_index: int):
    """Mean PSNR-Y (display area) of a stream decoded on the GPU against the source luma."""
    from riv2_b200.decoder import Decoder
    dec = Decoder.new(stream, dev_index)
    vals = []
    for ys in src_y:
        y = dec.decode_frame().y[:H_DISP, :W_DISP].astype(np.float64)
        mse = float(np.mean((y - ys[:H_DISP, :W_DISP]) ** 2))
        vals.append(99.0 if mse == 0 else 10.0 * np.log10(255.0 ** 2 / mse))
    dec.close()
    return float(np.mean(vals))


def run_ours(args, frames_host, dev_index, dist, form=0, params=None):
    import torch

    from riv2_b200 import encoder as E
    iq, pq = (int(x) for x in args.quality.split("/"))
    K, Wm = args.steps, args.warmup
    n = K + Wm + 1
    torch.cuda.set_device(dev_index)
    dev = torch.device("cuda", dev_index)
    frames_dev = torch.from_numpy(frames_host).to(dev)  # (n, H, W, 3), resident in HBM
    pinned = torch.from_numpy(frames_host).pin_memory()
    stride = W_DISP * H_DISP * 3

    def session(device_inputs: bool):
        w = E.VecWriter()
        enc = E.Encoder.new(config(iq, pq, args.pipeline_depth, dev_index, form, args.margin), w)
        if form == 1:
            enc.set_proposal(params)
        base = frames_dev.data_ptr() if device_inputs else pinned.data_ptr()

        def put(t, drain=False):
            if device_inputs:
                enc.encode_frame_device(base + t * stride, t * 20, drain=drain)
            else:
                arr = np.ctypeslib.as_array((np.ctypeslib.ctypes.c_uint8 * stride).from_address(base + t * stride))
                f = E.Frame(arr, W_DISP, H_DISP, t * 20)
                enc.encode_frame_with_stats(f) if drain else enc.encode_frame(f)

        for t in range(Wm):
            put(t)
        put(Wm, drain=True)  # the timed region starts with an empty pipeline
        c0 = enc.counters()
        torch.cuda.synchronize()
        barrier(dist, dev)
        torch.cuda.synchronize()
        ev0, ev1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        clocks = ClockSampler(dev_index)
        clocks.start()
        ev0.record()
        for t in range(Wm + 1, n):
            put(t)
        enc.finish()  # drains the pipeline: every timed frame's record is written
        ev1.record()
        torch.cuda.synchronize()
        clk = clocks.stop()
        barrier(dist, dev)
        ms = ev0.elapsed_time(ev1)
        c1 = enc.counters()
        lc = enc.learned_counters()
        data = w.into_inner()
        enc.close()
        return ms, c0, c1, clk, data, lc

    ms_v, c0v, c1v, clk_v, data_v, lc = session(True)
    dec = decode_rate(data_v, dev_index) if form == 0 else None
    ms_e, c0e, c1e, clk_e, data_e, _ = session(False)
    del frames_dev
    return {"ms_value": ms_v, "ms_e2e": ms_e, "c0": c0v, "c1": c1v, "c0e": c0e, "c1e": c1e, "clocks": clk_v,
            "clocks_e2e": clk_e, "stream_bytes": len(data_v), "streams_equal": data_v == data_e, "decode": dec,
            "stream": data_v, "learned_counters": lc}


def decode_rate(stream: bytes, dev_index: int):
    """GPU decoder (riv_decode_frame_yuv) over the stream just encoded: host entropy decoding
    and MV reconstruction, GPU reconstruction, no copy-out; whole-call wall time with CUDA
    events around it."""
    import torch

    from riv2_b200.decoder import Decoder
    dec = Decoder.new(stream, dev_index)
    n = dec.header().frame_count
    dec.decode_frame(copy_out=False)  # the key frame, untimed
    torch.cuda.synchronize()
    ev0, ev1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    ev0.record()
    for _ in range(n - 1):
        dec.decode_frame(copy_out=False)
    ev1.record()
    torch.cuda.synchronize()
    ms = ev0.elapsed_time(ev1)
    dec.close()
    return {"value": (n - 1) / (ms / 1000.0), "unit": "frames/s", "frames": n - 1,
            "what": "P-frames of the bench stream through the GPU decoder (YUV reconstruction, no copy-out)"}


def quick_fps(frames_dev, w, h, iq, pq, depth, form, params, steps, warmup, sr=12, margin=256):
    """Frames/s of a secondary configuration: device-resident RGB frames, `warmup` untimed
    frames, then `steps` frames timed with CUDA events up to the last record's write."""
    import torch

    from riv2_b200 import encoder as E
    cfg = (E.EncoderConfig.new(w, h, FPS).with_intra_quality(iq).with_inter_quality(pq).with_search_range(sr)
           .with_keyframe_interval(E.KeyframeInterval.fixed(1 << 40)).with_pipeline_depth(depth)
           .with_encode_form(form).with_proposal_margin(margin))
    enc = E.Encoder.new(cfg, E.VecWriter())
    if form == 1:
        enc.set_proposal(params)
    stride = w * h * 3
    base = frames_dev.data_ptr()
    for t in range(warmup):
        enc.encode_frame_device(base + t * stride, t * 20)
    enc.encode_frame_device(base + warmup * stride, warmup * 20, drain=True)
    torch.cuda.synchronize()
    ev0, ev1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    ev0.record()
    for t in range(warmup + 1, warmup + 1 + steps):
        enc.encode_frame_device(base + t * stride, t * 20)
    enc.finish()
    ev1.record()
    torch.cuda.synchronize()
    enc.close()
    return steps / (ev0.elapsed_time(ev1) / 1000.0)


BATCH_SIZES = (("cif", 352, 288), ("720p", 640, 360), ("720p", 1280, 720), ("1080p", 1920, 1080))


def batch_clips(seed: int):
    """The multi-clip workload: 16 clips at each of 352x288, 640x360, 1280x720 and 1920x1080
    with 30-90 frames each (uniform per clip, seeded), generator presets of their size class."""
    rng = np.random.default_rng(seed)
    out = []
    for k, (preset, w, h) in enumerate(BATCH_SIZES):
        for i in range(16):
            out.append({"preset": preset, "w": w, "h": h, "frames": int(rng.integers(30, 91)),
                        "seed": seed * 100 + 16 * k + i})
    return out


def batch_point(dev_index: int, seed: int, steps: int, warmup: int, full: bool = False, check: int = 4):
    """Aggregate throughput of the multi-clip encoder on the 64-clip mixed-resolution workload:
    RGB frames resident in device memory, one frame per clip per step, `warmup` untimed steps,
    then the timed steps up to the last record's write (riv_batch_finish inside the timed
    region).  `full`: every clip's whole length (up to 90 steps); otherwise `steps` steps (every
    clip has at least 30 frames, so all 64 clips are in every step).  `check` clips (the first of
    each size class) are encoded again alone by the single-clip encoder and their streams
    compared byte for byte."""
    import torch

    from riv2_b200 import encoder as E
    from riv2_b200.batch import Batch
    from riv2_b200.synth import SynthClip
    dev = torch.device("cuda", dev_index)
    clips = batch_clips(seed)
    nsteps = max(c["frames"] for c in clips) if full else warmup + steps
    t0 = time.perf_counter()
    dframes = []
    for c in clips:
        n = min(c["frames"], nsteps)
        sc = SynthClip(c["preset"], seed=c["seed"], width=c["w"], height=c["h"])
        dframes.append(torch.from_numpy(sc.frames(n)).to(dev))
    gen_s = time.perf_counter() - t0
    cfgs = [(E.EncoderConfig.new(c["w"], c["h"], 30).with_intra_quality(85).with_inter_quality(80)
             .with_keyframe_interval(E.KeyframeInterval.fixed(1 << 40)).with_pipeline_depth(4).with_device(dev_index))
            for c in clips]
    writers = [E.VecWriter() for _ in clips]
    b = Batch.new(cfgs, writers)
    strides = [c["w"] * c["h"] * 3 for c in clips]

    def step(k):
        ptrs = [f.data_ptr() + k * s if k < f.shape[0] else 0 for f, s in zip(dframes, strides)]
        b.encode_step_device(ptrs, [k * 33] * len(clips))

    for k in range(warmup):
        step(k)
    torch.cuda.synchronize()
    c0 = b.counters()
    clk = ClockSampler(dev_index)
    clk.start()
    ev0, ev1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    w0 = time.perf_counter()
    ev0.record()
    for k in range(warmup, nsteps):
        step(k)
    b.finish()
    ev1.record()
    torch.cuda.synchronize()
    wall = time.perf_counter() - w0
    clocks = clk.stop()
    ms = ev0.elapsed_time(ev1)
    c1 = b.counters()
    tune = b.tune()
    host = {k: round(v, 1) for k, v in b.host_times().items()}
    clip_host = np.sum([b.clip_counters(i)["host_ms"] for i in range(len(clips))], axis=0)
    host_clips = dict(zip(["submit", "retire", "mv_coding", "dct_coding_sum", "write", "blocked"],
                          [round(float(x), 1) for x in clip_host]))
    mbs = c1["mbs"] - c0["mbs"]
    frames = c1["frames"] - c0["frames"]
    b.close()
    streams = [w.into_inner() for w in writers]
    checked = []
    for k in range(min(check, len(BATCH_SIZES))):
        i = 16 * k
        n = min(clips[i]["frames"], nsteps)
        enc = E.Encoder.new(cfgs[i], E.VecWriter())
        for t in range(n):
            enc.encode_frame_device(dframes[i].data_ptr() + t * strides[i], t * 33)
        enc.finish()
        checked.append(enc.writer.into_inner() == streams[i])
        enc.close()
    del dframes
    torch.cuda.empty_cache()
    return {"macroblocks_per_s": mbs / (ms / 1000.0), "frames_per_s": frames / (ms / 1000.0),
            "per_clip_fps": (nsteps - warmup) / (ms / 1000.0), "ms": ms, "wall_s": wall, "steps": nsteps - warmup,
            "warmup": warmup, "clips": len(clips), "frames": frames, "mbs": mbs, "tune": tune,
            "gpu_stage_us_per_step": {k: round(v, 1) for k, v in c1["stage_us"].items()},
            "launches_per_step": (c1["launches"] - c0["launches"]) / max(1, nsteps - warmup),
            "host_ms_total": host, "clips_host_ms_total": host_clips,
            "streams_identical_to_single_clip": f"{sum(checked)}/{len(checked)}", "clocks": clocks,
            "frame_generation_s": round(gen_s, 1),
            "what": "64 clips (16 each at 352x288, 640x360, 1280x720, 1920x1080; 30-90 frames), q 85/80, one "
                    "frame per clip per step, RGB resident in device memory" + (", whole clips" if full else "")}


def secondary_points(frames_host, dev_index, params, steps, warmup, depth):
    """The other measurement points of the 1080p workload (quality 95/90, search range 31,
    pipeline depth 0 = the reference's one record per call), the CIF workload and the
    high-motion 4K stress clip at q 95/90 and 75/70, each for the plain form and, where a
    network is loaded, the learned form."""
    import torch

    from riv2_b200.synth import SynthClip
    dev = torch.device("cuda", dev_index)
    n = steps + warmup + 1
    f1080 = torch.from_numpy(frames_host[:n]).to(dev)
    cif = torch.from_numpy(SynthClip("cif", seed=2026).frames(max(n, 61))).to(dev)
    k4 = min(steps, 12)
    f4k = torch.from_numpy(SynthClip("4k", seed=2026).frames(k4 + warmup + 1)).to(dev)
    points = {"1080p_q95_90": (f1080, 1920, 1080, 95, 90, depth, 12, steps),
              "1080p_sr31": (f1080, 1920, 1080, 85, 80, depth, 31, steps),
              "1080p_depth0": (f1080, 1920, 1080, 85, 80, 0, 12, steps),
              "cif_q85_80": (cif, 352, 288, 85, 80, depth, 12, 60),
              "4k_q95_90": (f4k, 3840, 2160, 95, 90, depth, 12, k4),
              "4k_q75_70": (f4k, 3840, 2160, 75, 70, depth, 12, k4)}
    out = {}
    for name, (fr, w, h, iq, pq, d, sr, k) in points.items():
        k = min(k, fr.shape[0] - warmup - 1)
        row = {"plain": quick_fps(fr, w, h, iq, pq, d, 0, None, k, warmup, sr), "steps": k,
               "pipeline_depth": d, "search_range": sr, "quality": f"{iq}/{pq}"}
        if params is not None:
            row["learned"] = quick_fps(fr, w, h, iq, pq, d, 1, params, k, warmup, sr)
        out[name] = row
    return out


def cpu_baseline(frames_host, nframes, iq, pq):
    """The oracle (single-threaded restatement of the reference encoder, built here with
    -O3 -march=native) on a sample."""
    from oracle import oracle as O
    O.use_native_build()
    cfg = O.default_config(W_DISP, H_DISP, FPS)
    cfg.intra_quality, cfg.inter_quality = iq, pq
    cfg.keyframe_mode, cfg.keyframe_interval = 2, 1 << 40
    enc = O.OracleEncoder(cfg)
    enc.encode_rgb(frames_host[0], 0)
    t0 = time.perf_counter()
    for t in range(1, nframes + 1):
        enc.encode_rgb(frames_host[t], t * 20)
    dt = time.perf_counter() - t0
    return nframes / dt, dt


def _cpu_stream_worker(seed, nframes, iq, pq, barrier, results):
    """One independent CPU encode (spawned process): the key frame, then `nframes` P-frames
    timed from a barrier that all workers pass together."""
    frames = make_frames(nframes + 1, seed, 0)
    from oracle import oracle as O
    O.use_native_build()
    cfg = O.default_config(W_DISP, H_DISP, FPS)
    cfg.intra_quality, cfg.inter_quality = iq, pq
    cfg.keyframe_mode, cfg.keyframe_interval = 2, 1 << 40
    enc = O.OracleEncoder(cfg)
    enc.encode_rgb(frames[0], 0)
    barrier.wait(timeout=600)
    t0 = time.perf_counter()
    for t in range(1, nframes + 1):
        enc.encode_rgb(frames[t], t * 20)
    results.put((nframes, time.perf_counter() - t0))


def cpu_baseline_all_cores(seed, nframes, iq, pq, workers):
    """The CPU implementation with every host thread busy: the reference encoder is serial
    within a stream (raster-serial search, frames chained through the reconstruction), so
    the host's throughput is that of `workers` independent streams encoded at once.  Returns
    (frames/s over all streams, seconds of the slowest stream)."""
    import multiprocessing as mp
    ctx = mp.get_context("spawn")
    barrier = ctx.Barrier(workers)
    results = ctx.Queue()
    procs = [ctx.Process(target=_cpu_stream_worker, args=(seed, nframes, iq, pq, barrier, results))
             for _ in range(workers)]
    for pr in procs:
        pr.start()
    got = [results.get(timeout=900) for _ in range(workers)]
    for pr in procs:
        pr.join(timeout=60)
    slowest = max(dt for _, dt in got)
    return sum(n for n, _ in got) / slowest, slowest


# dram__bytes_read.sum + dram__bytes_write.sum of one steady-state k_search launch at this
# workload (ncu --set full, caches flushed before each pass, launch 7 of the bench
# command): 9,853,184 + 59,904 bytes.  The SAD table, the prediction, the pre-deblock
# reconstruction and the coefficients are produced and consumed inside the launch (or by the
# next one) and stay in L2.
SEARCH_TRAFFIC_BYTES = 9_853_184 + 59_904

Y_BYTES = 1920 * 1088            # one luma plane (storage size)
YUV_BYTES = Y_BYTES * 3 // 2     # one 4:2:0 frame


def launch_algorithmic_bytes(compact_bytes: float) -> dict:
    """Bytes each stage of one steady-state k_search launch reads and writes once, 1080p:
    * search + mode + AQ of frame t: read reference Y and current Y, write the per-MB records
      and outputs (8 + 20 B), ln variance and variance sums (12 B), and the luma prediction;
    * residual of frame t-1: read current YUV, luma prediction, reference chroma (chroma
      prediction), MB outputs and ln variances (24 B/MB); write the pre-deblock YUV, the
      coefficients (768 B/MB) and the skip / mask / EOB bytes (5 B/MB);
    * deblock of frame t-1: read the pre-deblock YUV and the mask, write the reference YUV;
    * compaction of frame t-1: read and write the compacted side info and coefficients
      (`compact_bytes`, the bench's measured device->host bytes per frame)."""
    n = MBS_PER_FRAME
    search = 2 * Y_BYTES + n * (28 + 12) + Y_BYTES
    residual = YUV_BYTES + Y_BYTES + Y_BYTES // 2 + n * 24 + YUV_BYTES + n * 768 + n * 5
    deblock = 2 * YUV_BYTES + n
    compact = 2 * compact_bytes
    return {"search_mode_aq": search, "residual": residual, "deblock": deblock, "compaction": int(compact),
            "total": int(search + residual + deblock + compact)}


def roofline_entry(stage_us_per_frame: float, compact_bytes: float):
    """One k_search launch: the wavefront search of frame t with the previous frame's
    residual, deblock and compaction in its worker CTAs.  Algorithmic bytes as in
    launch_algorithmic_bytes; the kernel is bound by the latency of its serial MB chain (120
    + 2 x 67 = 254 wavefront steps at 1080p), not by HBM, so the step time is reported
    beside the HBM fraction."""
    peaks = {}
    p = os.path.join(ROOT, "MEASURED_PEAKS.json")
    if os.path.exists(p):
        peaks = json.load(open(p))
    peak = float(peaks.get("hbm_gbs", 6650.0))
    parts = launch_algorithmic_bytes(compact_bytes)
    alg = parts["total"]
    achieved = alg / (stage_us_per_frame * 1e-6) / 1e9
    steps = (1920 // 16) + 2 * (1088 // 16 - 1)
    return {"bound": "hbm", "kernel": "k_search (wavefront search + RDO + mode + AQ of frame t; residual, deblock "
            "and compaction of frame t-1 in the worker CTAs)", "achieved": achieved,
            "peak": peak, "unit": "GB/s", "frac": achieved / peak, "traffic": SEARCH_TRAFFIC_BYTES,
            "algorithmic_bytes_per_launch": alg, "algorithmic_bytes_by_stage": parts, "launch_us": stage_us_per_frame,
            "peak_source": "measured" if "hbm_gbs" in peaks else "fallback",
            "critical_path": {"wavefront_steps": steps, "us_per_step": stage_us_per_frame / steps}}


def main():
    args = parse()
    ws, rank, local = dist_env()
    iq, pq = (int(x) for x in args.quality.split("/"))
    K, Wm = args.steps, args.warmup
    if args.impl == "reference":
        # rank 0 alone times the CPU implementation; other ranks exit without work.
        if rank != 0:
            return
        n = args.cpu_sample_frames
        frames = make_frames(n + 1, args.seed, 0)
        steps_vals = []
        for _ in range(max(1, min(K, 3))):
            fps, dt = cpu_baseline(frames, n, iq, pq)
            steps_vals.append(fps)
        fps = statistics.median(steps_vals)
        del frames
        # the host's capacity with every thread busy: independent streams, one per thread
        try:
            ncpu = len(os.sched_getaffinity(0))
        except AttributeError:
            ncpu = os.cpu_count() or 1
        workers = max(1, min(ncpu, args.cpu_workers))
        try:
            agg, slowest = cpu_baseline_all_cores(args.seed, n, iq, pq, workers)
            all_cores = {"value": agg, "unit": "frames/s", "streams": workers, "host_threads": ncpu,
                         "what": f"{workers} independent 1080p streams encoded at once, one per host thread "
                                 f"({n} P-frames each, timed from a common start; slowest {slowest:.1f} s)"}
        except Exception as ex:  # the single-stream figure above stands on its own
            all_cores = {"unavailable": f"{type(ex).__name__}: {ex}"}
        from oracle import oracle as O
        model = O.cpu_model()
        line = {"impl": "reference", "metric": METRIC, "value": fps, "unit": "frames/s", "n_gpus": ws, "steps": K,
                "warmup": Wm, "ms_per_step": 1000.0 / fps, "higher_is_better": True, "scaling": "weak",
                "vs_baseline": None, "dtype": "u8/i16/i32 (f32 AQ, f64 RDO)", "data": "synthetic",
                "config": {"workload": "1080p synthetic clip, q %d/%d, P-frames" % (iq, pq), "global_batch": 1,
                           "parallelism": "one stream on one host thread: the encoder is serial within a stream "
                                          "(raster-serial search, library-default features), so one thread is "
                                          "all this configuration can use"},
                "cpu_baseline": {"value": fps, "unit": "frames/s", "cores": 1, "kind": "port",
                                 "sample": f"{n} P-frames of the 1080p clip after its key frame, x{len(steps_vals)}",
                                 "cpu_model": model, "host_threads": ncpu,
                                 "build": "g++ -O3 -march=native -fwrapv -ffp-contract=off -fno-fast-math"},
                "cpu_all_cores": all_cores,
                "e2e": {"value": fps, "unit": "frames/s", "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0}}
        print(json.dumps(line))
        return

    dist = init_dist(ws, "nccl")
    import torch
    dev_index = local if torch.cuda.device_count() > 1 else 0
    if args.workload == "batch":  # the multi-clip workload alone, every clip over its whole length
        r = batch_point(dev_index, args.seed + rank, 0, Wm, full=True)
        ms = max_over_ranks(r["ms"], dist, torch.device("cuda", dev_index))
        if rank == 0:
            print(json.dumps({"metric": "multi-clip encode macroblocks/s (64 mixed-resolution clips, plain form)",
                              "value": r["mbs"] * ws / (ms / 1000.0), "unit": "macroblocks/s", "n_gpus": ws,
                              "steps": r["steps"], "warmup": Wm, "ms_per_step": ms / max(r["steps"], 1),
                              "higher_is_better": True, "scaling": "weak", "vs_baseline": None,
                              "dtype": "u8/i16/i32 (f32 AQ, f64 RDO)", "data": "synthetic",
                              "config": {"workload": r["what"], "parallelism": f"replicas x{ws}"}, "batch": r}))
        if dist is not None:
            dist.destroy_process_group()
        return
    frames = make_frames(K + Wm + 1, args.seed, rank)
    params = None
    if os.path.exists(args.weights):
        from riv2_b200 import proposal as P
        params = P.load_params(args.weights)
    forms = {"plain": run_ours(args, frames, dev_index, dist, 0)}
    if params is not None:
        forms["learned"] = run_ours(args, frames, dev_index, dist, 1, params)
    dvc = torch.device("cuda", dev_index)
    res = {}
    for name, r in forms.items():
        ms_v = max_over_ranks(r["ms_value"], dist, dvc)
        ms_e = max_over_ranks(r["ms_e2e"], dist, dvc)
        c0, c1 = r["c0"], r["c1"]
        pf = c1["pframes"] - c0["pframes"]
        ptimed = c1["timed_pframes"] - c0["timed_pframes"]  # stage timing events ride on sampled frames
        stage = [(b - a) / max(ptimed, 1) for a, b in zip(c0["stage_us_sum"], c1["stage_us_sum"])]
        res[name] = {
            "ms_v": ms_v, "ms_e": ms_e, "stage": stage, "launches": c1["launches"] - c0["launches"],
            "deferred": (c1["deferred_pframes"] - c0["deferred_pframes"]) / max(pf, 1),
            "h2d": (r["c1e"]["h2d_bytes"] - r["c0e"]["h2d_bytes"]) / K,
            "d2h": (r["c1e"]["d2h_bytes"] - r["c0e"]["d2h_bytes"]) / K,
            "host": dict(zip(["submit", "retire", "mv_coding", "dct_coding_sum", "write", "blocked"],
                             [round((b - a) / K, 3) for a, b in zip(c0["host_ms"], c1["host_ms"])])),
            "value": ws * K / (ms_v / 1000.0), "e2e": ws * K / (ms_e / 1000.0),
        }
    # quality of the two forms' streams of the same frames (decoded on the GPU; rank 0's clip)
    quality = None
    if "learned" in forms and rank == 0:
        from riv2_b200 import encoder as E
        sw, sh = W_DISP, (H_DISP + 15) // 16 * 16
        src_y = [E.stage_rgb_to_yuv(f, W_DISP, H_DISP, sw, sh)[: sw * sh].reshape(sh, sw) for f in frames]
        pp = psnr_y_of_stream(forms["plain"]["stream"], src_y, dev_index)
        pl = psnr_y_of_stream(forms["learned"]["stream"], src_y, dev_index)
        lc = forms["learned"]["learned_counters"]
        quality = {"psnr_y_plain_db": pp, "psnr_y_learned_db": pl, "delta_psnr_db": pl - pp,
                   "bytes_plain": forms["plain"]["stream_bytes"], "bytes_learned": forms["learned"]["stream_bytes"],
                   "delta_bitrate": forms["learned"]["stream_bytes"] / forms["plain"]["stream_bytes"] - 1.0,
                   "fallback_rate": lc["fallbacks"] / max(lc["mbs"], 1),
                   "shortcut_rate": lc["shortcuts"] / max(lc["mbs"], 1),
                   "frames": len(frames), "what": "the timed clip's key frame and P-frames, both streams decoded on "
                                                   "the GPU decoder, PSNR of the luma display area"}
    if rank != 0:
        if dist is not None:
            dist.destroy_process_group()
        return
    head = res.get("learned", res["plain"])
    cpu = None
    if ws == 1 and not args.no_cpu_baseline:
        fps, dt = cpu_baseline(frames, args.cpu_sample_frames, iq, pq)
        from oracle import oracle as O
        cpu = {"value": fps, "unit": "frames/s", "cores": 1, "kind": "port",
               "sample": f"{args.cpu_sample_frames} P-frames of the same 1080p clip after its key frame ({dt:.1f} s)",
               "cpu_model": O.cpu_model(), "build": "g++ -O3 -march=native -fwrapv -ffp-contract=off -fno-fast-math"}
    names = ["rgb_to_yuv", "sad_table", "search", "predict", "aq", "residual", "deblock", "compact", "total"]
    lnames = ["rgb_to_yuv", "proposal_network", "search_and_mode", "predict", "aq", "residual", "deblock", "compact",
              "total"]
    rp = res["plain"]
    learned = "learned" in res
    line = {
        "metric": METRIC, "value": head["value"] if learned else None, "unit": "frames/s", "n_gpus": ws, "steps": K,
        "warmup": Wm, "ms_per_step": head["ms_v"] / K, "higher_is_better": True, "scaling": "weak",
        "vs_baseline": None, "dtype": "u8/i16/i32 (f32 AQ, f64 RDO); bf16 network, f32 accumulation",
        "data": "synthetic",
        "config": {"workload": "1080p synthetic clip (1920x1080, 16 moving textured rects, pan, noise), GPU P-frame "
                               "encode, q %d/%d, search range 12, one key frame" % (iq, pq),
                   "global_batch": ws, "seq_len": K, "parallelism": f"replicas x{ws} (one clip per GPU)",
                   "form": ("learned proposal (network %s, fallback margin %d) vs plain"
                            % (os.path.relpath(args.weights, ROOT), args.margin)) if learned
                           else "plain only: no proposal-network weights at %s" % args.weights,
                   "pipeline_depth": args.pipeline_depth,
                   "l2": "inputs larger than L2: %d distinct RGB frames (%.0f MB) resident in HBM"
                         % (K + Wm + 1, (K + Wm + 1) * W_DISP * H_DISP * 3 / 1e6),
                   "macroblocks_per_s": head["value"] * MBS_PER_FRAME},
        "e2e": {"value": head["e2e"], "unit": "frames/s", "h2d_bytes_per_step": int(head["h2d"]),
                "d2h_bytes_per_step": int(head["d2h"])},
        "plain": {"value": rp["value"], "e2e": rp["e2e"], "ms_per_step": rp["ms_v"] / K,
                  "macroblocks_per_s": rp["value"] * MBS_PER_FRAME,
                  "gpu_stage_us_per_pframe": dict(zip(names, [round(x, 2) for x in rp["stage"]])),
                  "pframes_reconstructed_in_next_launch": round(rp["deferred"], 3),
                  "gpu_pipeline_fps": 1e6 / rp["stage"][8] if rp["stage"][8] > 0 else None,
                  "host_ms_per_frame": rp["host"], "gpu_launches": int(rp["launches"]),
                  "stream_bytes": forms["plain"]["stream_bytes"],
                  "streams_equal_value_vs_e2e": forms["plain"]["streams_equal"]},
        "gpu_launches": int(head["launches"]),
        "roofline": roofline_entry(rp["stage"][2], rp["d2h"]),
        "cpu_baseline": cpu,
        "clocks": forms["learned" if learned else "plain"]["clocks"],
        "clocks_e2e": forms["learned" if learned else "plain"]["clocks_e2e"],
        "decode": forms["plain"]["decode"],
    }
    if learned:
        rl = res["learned"]
        line["learned_vs_plain"] = dict({"value_ratio": rl["value"] / rp["value"], "e2e_ratio": rl["e2e"] / rp["e2e"]},
                                        **(quality or {}))
        line["learned_stage_us_per_pframe"] = dict(zip(lnames, [round(x, 2) for x in rl["stage"]]))
        line["learned_gpu_pipeline_fps"] = 1e6 / rl["stage"][8] if rl["stage"][8] > 0 else None
        line["learned_host_ms_per_frame"] = rl["host"]
        line["learned_streams_equal_value_vs_e2e"] = forms["learned"]["streams_equal"]
    if ws == 1 and not args.no_secondary:
        line["secondary"] = secondary_points(frames, dev_index, params, min(K, 20), min(Wm, 3), args.pipeline_depth)
        if args.batch_steps > 0:
            line["secondary"]["batch_64_clips"] = batch_point(dev_index, args.seed, args.batch_steps, 3)
    print(json.dumps(line))
    if dist is not None:
        dist.destroy_process_group()


if __name__ == "__main__":
    main()
