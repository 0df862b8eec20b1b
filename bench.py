#!/usr/bin/env python3
"""PyroWave B200 benchmark: microseconds per frame, encode + decode, 1080p 4:2:0 at 400000 bytes.

    python bench.py [--gpus N] [--steps K] [--warmup W] [--impl ours|reference] [--config 1080p|4k|4k444|720p]

One step = encode one frame and decode it again, on one GPU. Inputs are 16
seeded synthetic frames (gradient + band-limited noise + flat rectangles, the
generator in pyrowave_b200/synth.py) that stand in for the reference's private
game clips.

value : device-resident encode + decode (input planes already in HBM, decode
        from the encoder's device bitstream), timed per step with CUDA events on
        the stream the library launches on. The inputs rotate through distinct
        frames totalling more than twice the 126 MB L2 (--l2 flush instead
        writes 256 MiB between steps).
e2e   : the same frames through the reference-facing C API with host buffers:
        pyrowave_encoder_encode_cpu_synchronous (H2D inside), compute_num_packets
        + packetize (D2H), pyrowave_decoder_push_packet (host parse) and
        pyrowave_decoder_decode_cpu_buffer_synchronous (H2D payload, D2H planes).
Multi-GPU: one process per GPU (torchrun), independent replicas ("scaling":
"weak"): each rank codes its own frames; time = max over ranks.
--impl reference: the reference algorithm's CPU restatement (oracle/) on all
host cores, same workload and metric (the reference's own Vulkan path has no
device it can run on here).
"""
from __future__ import annotations

import argparse
import concurrent.futures
import json
import os
import statistics
import subprocess
import sys
import threading
import time

import numpy as np

ROOT = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, ROOT)

CONFIGS = {
    "1080p": dict(width=1920, height=1080, chroma444=False, budget=400000, seeds=list(range(1, 17)), rects=40, lines=0),
    "4k": dict(width=3840, height=2160, chroma444=False, budget=1200000, seeds=list(range(1, 17)), rects=40, lines=0),
    "4k444": dict(width=3840, height=2160, chroma444=True, budget=1200000, seeds=list(range(1, 5)), rects=200, lines=40),
    "720p": dict(width=1280, height=720, chroma444=False, budget=150000, seeds=[0], rects=40, lines=0),
}



def dist_info():
    ws = int(os.environ.get("WORLD_SIZE", "1"))
    rank = int(os.environ.get("RANK", "0"))
    local = int(os.environ.get("LOCAL_RANK", "0"))
    return ws, rank, local


def max_over_ranks(values, ws, device="cpu"):
    """Element-wise maximum of this rank's timings over all ranks; every rank
    gets the result (one all-reduce, the same on every rank). With one rank the
    values come back unchanged."""
    if ws <= 1:
        return [float(v) for v in values]
    import torch

    t = torch.tensor([float(v) for v in values], dtype=torch.float64, device=device)
    torch.distributed.all_reduce(t, op=torch.distributed.ReduceOp.MAX)
    return [float(x) for x in t.tolist()]


def whole_job_us_per_frame(max_ms, steps, ws):
    """Microseconds per frame of the whole job: every rank codes `steps`
    frames, and the job takes as long as its slowest rank."""
    return max_ms * 1e3 / (steps * ws)


def make_frames(cfg):
    from pyrowave_b200 import synth

    return [synth.synth_frame(cfg["width"], cfg["height"], cfg["chroma444"], s, cfg["rects"], cfg["lines"])
            for s in cfg["seeds"]]


def frames_fingerprint(frames):
    """8-byte blake2b over the frames' own fingerprints, in order."""
    import hashlib

    from pyrowave_b200 import synth

    h = hashlib.blake2b(digest_size=8)
    for f in frames:
        h.update(bytes.fromhex(synth.frame_hash(f)))
    return h.hexdigest()


def workload_config(cfg, frames, ws):
    """The `config` object of both arms' JSON lines: the same keys and values for the same workload."""
    c444 = cfg["chroma444"]
    return {"workload": f"encode+decode {cfg['width']}x{cfg['height']} {'4:4:4' if c444 else '4:2:0'} 8-bit, "
                        f"{cfg['budget']}-byte budget",
            "frames": len(frames), "frames_fingerprint": frames_fingerprint(frames),
            "budget_bytes": cfg["budget"], "parallelism": f"replicas x{ws}"}


# How the numbers of this line are tied to the reference's behaviour.
PARITY = {
    "bitstream_layer": "block layout, packetize and packet parser pinned to the reference's own "
                       "metal/pyrowave_bitstream.cpp, compiled from its tree (tests/test_oracle_pinning.py, "
                       "tests/golden/)",
    "shader_math": "DWT, quantiser and RD statistics, rate control, packing, dequantiser and inverse DWT: bit-exact "
                   "with the oracle's restatement of the reference shaders at every stage, on the frames of every "
                   "configuration of this line (tests/test_gpu_parity.py); the restatement itself is pinned only by "
                   "the reference's known-answer tests (pyrowave_c_test.cpp:147-158,288-379,440-535), since the "
                   "shaders need Vulkan, which no machine here has",
    "reference_precision": "REFERENCE_PRECISION (FP16 staging + FP16 levels 0-1) is bit-exact with the oracle's "
                           "restatement of the reference's precision 1, so its PSNR equals the restated "
                           "reference's (tests/test_gpu_psnr.py)",
}


def psnr_delta(cfg, frames, budget, mask):
    """Decoded PSNR of the given precision minus that of REFERENCE_PRECISION (the
    reference's arithmetic) at the same budget, per plane: mean over the frames
    and the frame with the largest difference."""
    import torch

    from pyrowave_b200 import capi

    w, h, c444 = cfg["width"], cfg["height"], cfg["chroma444"]
    chroma = capi.CHROMA_444 if c444 else capi.CHROMA_420
    dev = capi.Device()

    hvs = {}

    def coded(m):
        """PSNR per frame and plane, and the luma PSNR-HVS-M over all frames (the
        reference's metric on the GPU, pyrowave_cuda_psnr_hvs_m)."""
        enc = capi.Encoder(dev, w, h, chroma, m)
        dec = capi.Decoder(dev, w, h, chroma, m)
        errors = torch.zeros(16, dtype=torch.int64, device="cuda")
        res = []
        hvs_ms = 0.0
        for f in frames:
            d = [torch.from_numpy(p).cuda() for p in f]
            o = [torch.empty_like(p) for p in d]
            enc.encode_device([p.data_ptr() for p in d], [p.stride(0) for p in d], budget)
            s, mt, cap = enc.device_bitstream()
            dec.decode_blocks(mt, s + 8, cap - 2, [p.data_ptr() for p in o], [p.stride(0) for p in o])
            e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
            e0.record()
            capi.check(capi.psnr_hvs_m(w, h, d[0].data_ptr(), d[0].stride(0), o[0].data_ptr(), o[0].stride(0),
                                       errors.data_ptr()), "psnr_hvs_m")
            e1.record()
            e1.synchronize()
            hvs_ms += e0.elapsed_time(e1)
            res.append([_psnr(a, b.cpu().numpy()) for a, b in zip(f, o)])
        db = capi.psnr_hvs_m_db(errors.cpu().numpy().view(np.uint64),
                                capi.lib().pyrowave_psnr_hvs_m_pixels(w, h) * len(frames))
        hvs[m] = {"height_factor_1": round(float(db[0]), 3), "height_factor_2": round(float(db[8]), 3),
                  "height_factor_2.875": round(float(db[15]), 3),
                  "kernel_us_per_frame": round(hvs_ms * 1e3 / len(frames), 2)}
        enc.close()
        dec.close()
        return np.array(res)

    d = coded(mask) - coded(0x103)
    dev.close()
    worst = np.abs(d).max(axis=0)
    return {"mask": hex(mask), "against": "REFERENCE_PRECISION (0x103)", "frames": len(frames),
            "mean_y_cb_cr": [round(float(x), 4) for x in d.mean(axis=0)],
            "worst_frame_y_cb_cr": [round(float(x), 4) for x in worst],
            "within_0.02_db_mean": bool(np.abs(d.mean(axis=0)).max() <= 0.02),
            "psnr_hvs_m_luma_db": {"this_precision": hvs[mask], "reference_precision": hvs[0x103]}}


def _psnr(a, b):
    mse = float(np.mean((a.astype(np.float64) - b.astype(np.float64)) ** 2))
    return 99.0 if mse == 0 else 10.0 * np.log10(255.0 ** 2 / mse)


def algorithmic_bytes(cfg, fp16_mask):
    """Minimal bytes per frame of each kernel: every input byte read once, every output byte written once."""
    w, h, c444 = cfg["width"], cfg["height"], cfg["chroma444"]
    aw = max((w + 31) // 32 * 32, 128)
    ah = max((h + 31) // 32 * 32, 128)
    planes = [(w, h)] + ([(w, h)] * 2 if c444 else [(w // 2, h // 2)] * 2)

    def band_bytes(level):
        return ((aw // 2) >> level) * ((ah // 2) >> level) * (2 if (fp16_mask >> level) & 1 else 4)

    out = {}
    transmitted = 0
    for level in range(5):
        fin = fout = 0
        for c in range(3):
            first = 0 if (c == 0 or c444) else 1
            if level < first:
                continue
            src = planes[c][0] * planes[c][1] if level == first else band_bytes(level - 1)
            fin += src + 4 * band_bytes(level)            # forward: read input, write LL, HL, LH, HH
            fout += 4 * band_bytes(level) + src           # inverse: read 4 bands, write LL(level-1) or the plane
            transmitted += (4 if level == 4 else 3) * band_bytes(level)
        out[f"dwt{level}"] = fin
        out[f"idwt{level}"] = fout
    blocks8 = 0
    for level in range(5):
        bw, bh = (aw // 2) >> level, (ah // 2) >> level
        ncomp = 3 if (level > 0 or c444) else 1
        blocks8 += ((bw + 7) // 8) * ((bh + 7) // 8) * (4 if level == 4 else 3) * ncomp
    out["pack"] = transmitted + 4 * blocks8 + cfg["budget"]
    out["dequant"] = cfg["budget"] + transmitted
    # The DWT stage as a whole: 8-bit planes read once, transmitted coefficients written once.
    out["dwt_stage"] = sum(x * y for x, y in planes) + transmitted
    return out


class ClockSampler:
    """nvidia-smi clocks and throttle reasons, sampled every 50 ms with arrival
    times, so that only the samples taken while the GPU runs the measured
    workload (between mark_begin and mark_end) are summarised."""

    FIELDS = ("index,clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,clocks_event_reasons.hw_slowdown,"
              "clocks_event_reasons.hw_thermal_slowdown,clocks_event_reasons.sw_thermal_slowdown,"
              "clocks_event_reasons.sw_power_cap")
    INTERVAL_MS = 50

    def __init__(self, gpu_index: int):
        self.gpu_index = gpu_index
        self.proc = None
        self.lines = []  # (arrival time, csv line)
        self.begin = self.end = None

    def start(self):
        try:
            self.proc = subprocess.Popen(["nvidia-smi", "-i", str(self.gpu_index), f"--query-gpu={self.FIELDS}",
                                          "--format=csv,noheader,nounits", "-lms", str(self.INTERVAL_MS)],
                                         stdout=subprocess.PIPE, stderr=subprocess.DEVNULL, text=True)
            self.thread = threading.Thread(target=self._read, daemon=True)
            self.thread.start()
        except Exception:
            self.proc = None

    def _read(self):
        for line in self.proc.stdout:
            self.lines.append((time.perf_counter(), line.strip()))

    def wait_ready(self, timeout: float = 3.0):
        """Waits (bounded) for the first sample, so sampling runs before the load starts."""
        t0 = time.perf_counter()
        while self.proc is not None and not self.lines and time.perf_counter() - t0 < timeout:
            time.sleep(0.01)

    def mark_begin(self):
        self.begin = time.perf_counter()

    def mark_end(self):
        self.end = time.perf_counter()

    def stop(self):
        if self.proc is None:
            return {"sm_mhz": None, "sm_max_mhz": None, "reasons": ["nvidia-smi unavailable"]}
        time.sleep(2 * self.INTERVAL_MS / 1000)  # the sample in flight at mark_end
        self.proc.terminate()
        try:
            self.proc.wait(timeout=5)
        except Exception:
            self.proc.kill()
        lines = list(self.lines)
        in_region = lines
        if self.begin is not None and self.end is not None:
            # A sample printed up to one interval after mark_end was queried before it.
            last = self.end + self.INTERVAL_MS / 1000
            in_region = [(t, l) for t, l in lines if self.begin <= t <= last]
        used = in_region if in_region else lines
        sm, mx, reasons = [], None, set()
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        for _, line in used:
            parts = [p.strip() for p in line.split(",")]
            if len(parts) < 9:
                continue
            try:
                sm.append(float(parts[1]))
                mx = float(parts[2])
            except ValueError:
                continue
            for n, v in zip(names, parts[5:9]):
                if v.lower().startswith("active"):
                    reasons.add(n)
        return {"sm_mhz": statistics.median(sm) if sm else None, "sm_max_mhz": mx, "reasons": sorted(reasons),
                "samples": len(sm), "samples_under_load": len(in_region) if in_region is not lines else 0,
                "interval_ms": self.INTERVAL_MS}


def measured_peak():
    p = os.path.join(ROOT, "MEASURED_PEAKS.json")
    try:
        with open(p) as f:
            d = json.load(f)
        return float(d["hbm_gbs"]), "measured"
    except Exception:
        return 6650.0, "fallback"


# ---------------------------------------------------------------------------
def run_ours(args, cfg, ws, rank, local):
    import torch

    from pyrowave_b200 import capi

    torch.cuda.set_device(local)
    if ws > 1:
        import torch.distributed as dist
        from datetime import timedelta

        dist.init_process_group("nccl", timeout=timedelta(seconds=120), device_id=torch.device("cuda", local))
    frames = make_frames(cfg)
    w, h, c444, budget = cfg["width"], cfg["height"], cfg["chroma444"], cfg["budget"]
    chroma = capi.CHROMA_444 if c444 else capi.CHROMA_420

    dev = capi.Device()
    enc = capi.Encoder(dev, w, h, chroma, args.fp16_mask)
    dec = capi.Decoder(dev, w, h, chroma, args.fp16_mask)
    stream = torch.cuda.Stream()
    sid = stream.cuda_stream

    base = [[torch.from_numpy(p).cuda() for p in f] for f in frames]
    frame_bytes = sum(p.nbytes for p in frames[0])
    L2_BYTES = 126 * 1024 * 1024
    if args.l2 == "rotate":
        # Inputs larger than L2: enough distinct frames (shifted copies of the
        # seeded frames) that each step's input was evicted long before it is
        # read again.
        nframes = max(len(base), -(-2 * L2_BYTES // frame_bytes))
        d_frames = []
        for i in range(nframes):
            f = base[i % len(base)]
            k = i // len(base)
            d_frames.append([torch.roll(p, shifts=(3 * k, 5 * k), dims=(0, 1)).contiguous() if k else p for p in f])
        l2_note = f"inputs larger than L2: {nframes} distinct frames ({nframes * frame_bytes / 1e6:.0f} MB) rotated"
    else:
        d_frames = base
        l2_note = "flushed between steps (256 MiB write)"
    d_out = [torch.empty(p.shape, dtype=torch.uint8, device="cuda") for p in frames[0]]
    flush = torch.empty(256 << 20, dtype=torch.uint8, device="cuda") if args.l2 == "flush" else None
    torch.cuda.synchronize()

    def step(i):
        f = d_frames[i % len(d_frames)]
        enc.encode_device([p.data_ptr() for p in f], [p.stride(0) for p in f], budget, sid)
        s, m, cap = enc.device_bitstream()
        dec.decode_blocks(m, s + 8, cap - 2, [p.data_ptr() for p in d_out], [p.stride(0) for p in d_out], sid)

    for i in range(args.warmup):
        step(i)
    torch.cuda.synchronize()
    # Sanity: the last warm-up frame fits its budget.
    size = enc.size()
    assert 8 < size <= budget, size

    starts = [torch.cuda.Event(enable_timing=True) for _ in range(args.steps)]
    ends = [torch.cuda.Event(enable_timing=True) for _ in range(args.steps)]
    wall = {}

    def timed_pass(first):
        """Device milliseconds of `steps` steps. With rotated inputs (larger than
        L2) one event pair spans all steps, so any gap between steps counts; with
        an L2 flush between steps, the flushes are excluded by an event pair per
        step. The host wall clock over the same region is kept as a cross-check."""
        if ws > 1:
            torch.distributed.barrier()
        torch.cuda.synchronize()
        w0 = time.perf_counter()
        for i in range(args.steps):
            with torch.cuda.stream(stream):
                if flush is not None:
                    flush.fill_(i & 0xFF)  # evict the previous frame from the 126 MB L2
                if flush is not None or i == 0:
                    starts[i].record(stream)
            step(first + i)
            with torch.cuda.stream(stream):
                if flush is not None or i == args.steps - 1:
                    ends[i].record(stream)
        torch.cuda.synchronize()
        wall["ms"] = (time.perf_counter() - w0) * 1e3
        if ws > 1:
            torch.distributed.barrier()
        if flush is not None:
            return float(sum(s_.elapsed_time(e_) for s_, e_ in zip(starts, ends)))
        return float(starts[0].elapsed_time(ends[args.steps - 1]))

    # Timed region 1: the headline number (no extra events between kernels).
    # The clock samples cover it and about 0.3 s of the same untimed steps just
    # before it (64 at a time, then a synchronize, so the queue stays short):
    # the timed steps alone last too short for samples at 50 ms. The frame
    # order continues through the load steps into the timed ones, so no timed
    # frame is still in L2.
    sampler = ClockSampler(local)
    sampler.start()
    sampler.wait_ready()
    sampler.mark_begin()
    load_steps = 0
    t_load = time.perf_counter()
    while time.perf_counter() - t_load < 0.3:
        for _ in range(64):
            step(args.warmup + load_steps)
            load_steps += 1
        torch.cuda.synchronize()
    first_timed = args.warmup + load_steps
    plain_ms = timed_pass(first_timed)
    plain_wall_ms = wall["ms"]
    sampler.mark_end()
    clocks = sampler.stop()
    clocks["load_steps_before_timed"] = load_steps
    # Timed region 2: the same steps with a CUDA event after every kernel, for
    # the per-kernel durations behind the roofline.
    dev.set_stage_timing(True)
    dev.report_performance_stats(reset=True)
    total_ms = timed_pass(first_timed + args.steps)
    stage_lines = dev.report_performance_stats(reset=True)
    dev.set_stage_timing(False)
    stages = {}
    for line in stage_lines:
        tag, rest = line.split(":", 1)
        stages[tag.strip()] = float(rest.split("ms")[0])

    total_ms, plain_ms = max_over_ranks([total_ms, plain_ms], ws, "cuda")

    frames_total = args.steps * ws
    us_per_frame = whole_job_us_per_frame(plain_ms, args.steps, ws)

    # Roofline of the dominant kernel.
    alg = algorithmic_bytes(cfg, args.fp16_mask)
    peak, peak_kind = measured_peak()
    kernel_stages = {k: v for k, v in stages.items() if k in alg}
    dom = max(kernel_stages, key=kernel_stages.get) if kernel_stages else None
    roofline = None
    if dom:
        ms = kernel_stages[dom]
        achieved = alg[dom] / (ms * 1e-3) / 1e9
        roofline = {"bound": "hbm", "kernel": dom, "achieved": round(achieved, 1), "peak": peak, "unit": "GB/s",
                    "frac": round(achieved / peak, 4), "traffic": _ncu_traffic(dom, cfg), "peak_source": peak_kind,
                    "algorithmic_bytes": alg[dom], "avg_launch_us": round(ms * 1e3, 2)}
        limit = _ncu_limit(dom, cfg)
        if limit:
            roofline.update(limit)
    dwt_ms = sum(v for k, v in stages.items() if k.startswith("dwt"))
    dwt_stage = {"us": round(dwt_ms * 1e3, 2), "algorithmic_bytes": alg["dwt_stage"],
                 "achieved_gbs": round(alg["dwt_stage"] / (dwt_ms * 1e-3) / 1e9, 1) if dwt_ms else None}
    if dwt_ms:
        dwt_stage["frac_of_peak"] = round(dwt_stage["achieved_gbs"] / peak, 4)

    e2e = run_e2e(args, cfg, frames, dev) if (rank == 0 or ws > 1) and not getattr(args, "no_e2e", False) else None
    if ws > 1 and e2e is not None:
        e2e["total_s"] = max_over_ranks([e2e["total_s"]], ws, "cuda")[0]
    psnr = None
    if rank == 0 and not args.no_configs:
        psnr = psnr_delta(cfg, frames, budget, args.fp16_mask)
    cpu = None
    if rank == 0 and ws == 1 and not args.no_cpu_baseline:
        cpu = cpu_baseline(cfg, frames, args.cpu_seconds)
    batched = None
    if rank == 0 and ws == 1 and not args.no_batch:
        batched = run_batched(iters=10, frames_n=args.batch_frames)
    packet_decode = None
    if rank == 0 and ws == 1 and not args.no_configs:
        packet_decode = run_packet_decode(cfg, frames)
    serving = None
    if rank == 0 and ws == 1 and args.serve_seconds > 0:
        serving = run_serving(args.serve_seconds)
    secondary = None
    if rank == 0 and ws == 1 and not args.no_configs:
        secondary = run_secondary(steps=30, warmup=5)
    packing = None
    if rank == 0 and ws == 1 and not args.no_configs:
        packing = run_packing_analysis(cfg, frames)

    if rank == 0:
        line = {
            "metric": f"us/frame enc+dec {cfg['width']}x{cfg['height']} {'4:4:4' if c444 else '4:2:0'} @ {budget} B",
            "value": round(us_per_frame, 3),
            "unit": "us/frame",
            "n_gpus": ws,
            "steps": args.steps,
            "warmup": args.warmup,
            "ms_per_step": round(plain_ms / args.steps, 4),
            "higher_is_better": False,
            "scaling": "weak",
            "vs_baseline": None,
            "dtype": "f32" if args.fp16_mask == 0 else f"f32 (fp16 storage mask {args.fp16_mask:#x})",
            "data": "synthetic (seeded gradient + band-limited noise + rectangles, 16 frames)",
            "config": workload_config(cfg, frames, ws),
            "l2": l2_note,
            "wall_us_per_frame": round(plain_wall_ms * 1e3 / args.steps, 3),
            "e2e": None if e2e is None else {
                "value": round(e2e["total_s"] * 1e6 / (e2e["frames"] * ws), 2), "unit": "us/frame",
                "h2d_bytes_per_step": e2e["h2d"], "d2h_bytes_per_step": e2e["d2h"],
                "method": e2e["method"], "breakdown_us": e2e["breakdown_us"]},
            "parity": PARITY,
            "psnr_delta_db": psnr,
            "packing_analysis": packing,
            "gpu_launches": len(stages) * args.steps,  # one stage-timing tag per kernel launch
            "roofline": roofline,
            "dwt_stage": dwt_stage,
            "stages_us": {k: round(v * 1e3, 2) for k, v in stages.items()},
            "stage_event_overhead_us": round((total_ms - plain_ms) * 1e3 / args.steps, 2),
            "value_with_stage_events": round(total_ms * 1e3 / frames_total, 3),
            "bytes_per_frame": size,
            "clocks": clocks,
            "cpu_baseline": cpu,
            "batched": batched,
            "serving": serving,
            "configs": secondary,
            "device_packet_decode": packet_decode,
        }
        print(json.dumps(line), flush=True)
    if ws > 1:
        torch.distributed.barrier()
        torch.distributed.destroy_process_group()


BATCH_SIZES = [(1280, 720), (1366, 768), (1920, 1080), (2560, 1080), (2560, 1440), (3840, 2160)]


PACKING_LAYOUTS = ["32x32/2x2", "32x32/4x2", "32x32/2x4", "64x32/4x4", "64x64/8x4"]


def run_packing_analysis(cfg, frames):
    """Packing statistics of the workload's first frame, computed on the device
    (pyrowave_cuda_encoder_analyze_packing: the reference's disabled
    report_stats / analyze_alternative_packing pass, pyrowave_encoder.cpp:625-958):
    estimated bytes of five packet / sub-block shapes beside the coded bytes, and
    the byte entropy of each magnitude plane position."""
    from pyrowave_b200 import capi

    w, h, c444, budget = cfg["width"], cfg["height"], cfg["chroma444"], cfg["budget"]
    dev = capi.Device()
    enc = capi.Encoder(dev, w, h, capi.CHROMA_444 if c444 else capi.CHROMA_420)
    try:
        assert enc.encode_cpu(frames[0], budget) == capi.PYROWAVE_SUCCESS
        a = enc.analyze_packing()
    finally:
        enc.close()
        dev.close()
    coded = a["coded_bytes"]
    planes = int(np.count_nonzero(a["plane_bytes"]))
    return {"coded_bytes": coded, "significant": a["significant"],
            "layout_bytes": {n: int(b) for n, b in zip(PACKING_LAYOUTS, a["layout_bytes"])},
            "layout_vs_coded": {n: round(int(b) / coded, 4) if coded else None
                                for n, b in zip(PACKING_LAYOUTS, a["layout_bytes"])},
            "plane_bytes": [int(v) for v in a["plane_bytes"][:planes]],
            "plane_entropy": [round(float(v), 4) for v in a["plane_entropy"][:planes]]}


def run_packet_decode(cfg, frames, steps: int = 50, boundary: int = 8192):
    """Decode from received packets already in device memory: assembly on the
    GPU (pyrowave_cuda_decoder_decode_packets) against decoding the encoder's
    device-resident blocks (pyrowave_cuda_decoder_decode_blocks), us per frame."""
    import torch

    from pyrowave_b200 import capi

    w, h, c444, budget = cfg["width"], cfg["height"], cfg["chroma444"], cfg["budget"]
    chroma = capi.CHROMA_444 if c444 else capi.CHROMA_420
    dev = capi.Device()
    enc = capi.Encoder(dev, w, h, chroma)
    dec = capi.Decoder(dev, w, h, chroma)
    assert enc.encode_cpu(frames[0], budget) == capi.PYROWAVE_SUCCESS
    stream_bytes, packets = enc.packetize(boundary, budget)
    total = sum(sz for _, sz in packets)
    d_data = torch.from_numpy(np.ascontiguousarray(stream_bytes[:total])).cuda()
    d_desc = torch.from_numpy(np.array(packets, np.int64).reshape(-1)).cuda()
    out = [torch.empty(p.shape, dtype=torch.uint8, device="cuda") for p in frames[0]]
    ptrs, strides = [t.data_ptr() for t in out], [t.stride(0) for t in out]
    s, m, cap = enc.device_bitstream()
    stream = torch.cuda.Stream()
    torch.cuda.synchronize()  # inputs complete before the library's stream reads them

    def timed(fn):
        for _ in range(5):
            fn()
        torch.cuda.synchronize()
        e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        e0.record(stream)
        for _ in range(steps):
            fn()
        e1.record(stream)
        e1.synchronize()
        return e0.elapsed_time(e1) * 1e3 / steps

    packets_us = timed(lambda: capi.check(dec.decode_packets(d_data.data_ptr(), total, d_desc.data_ptr(), len(packets),
                                                             ptrs, strides, stream.cuda_stream), "decode_packets"))
    st = dec.packet_status()
    blocks_us = timed(lambda: dec.decode_blocks(m, s + 8, cap - 2, ptrs, strides, stream.cuda_stream))
    enc.close()
    dec.close()
    dev.close()
    return {"workload": f"decode {w}x{h} {'4:4:4' if c444 else '4:2:0'} from {len(packets)} packets of "
                        f"<= {boundary} B in device memory ({total} B)",
            "us_per_frame": round(packets_us, 2), "decode_blocks_us_per_frame": round(blocks_us, 2),
            "complete": bool(st.decoded_blocks >= st.total_blocks), "invalid_packets": int(st.invalid_packets)}


def run_batched(iters: int, frames_n: int = 64, seed: int = 7):
    """Batched form: frames_n frames of the six sizes, 4:2:0 and 4:4:4 mixed,
    budgets drawn uniformly from 150-250 Mbit/s at 60 fps; encode + decode of
    every frame per call. Compared with the same frames through frames_n
    single-frame encoders and decoders on the same device."""
    import torch

    from pyrowave_b200 import capi, synth

    rng = np.random.default_rng(seed)
    slots = []
    for i in range(frames_n):
        w, h = BATCH_SIZES[i % len(BATCH_SIZES)]
        c444 = (i // len(BATCH_SIZES)) % 2 == 1
        budget = int(rng.uniform(150e6, 250e6) / 8 / 60) & ~3
        slots.append((w, h, c444, budget))
    # One synthetic image per (size, chroma), shared by the slots that use it.
    content = {}
    for w, h, c444, _ in slots:
        if (w, h, c444) not in content:
            content[(w, h, c444)] = [torch.from_numpy(p).cuda()
                                     for p in synth.synth_frame(w, h, c444, 1000 + len(content))]
    inputs = [content[(w, h, c444)] for w, h, c444, _ in slots]
    outputs = [[torch.empty_like(p) for p in pl] for pl in inputs]
    in_ptrs = [[p.data_ptr() for p in pl] for pl in inputs]
    in_strides = [[p.stride(0) for p in pl] for pl in inputs]
    out_ptrs = [[p.data_ptr() for p in pl] for pl in outputs]
    out_strides = [[p.stride(0) for p in pl] for pl in outputs]
    budgets = [b for *_, b in slots]
    pixels = sum(w * h for w, h, _, _ in slots)

    dev = capi.Device()
    stream = torch.cuda.Stream()
    torch.cuda.synchronize()  # inputs complete before the library's stream reads them
    batch = capi.Batch(dev, [(w, h, capi.CHROMA_444 if c else capi.CHROMA_420, b) for w, h, c, b in slots])
    capi.check(batch.autotune(in_ptrs, in_strides, budgets, out_ptrs, out_strides, stream.cuda_stream), "autotune")

    def timed(fn):
        for _ in range(3):
            fn()
        torch.cuda.synchronize()
        e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        e0.record(stream)
        for _ in range(iters):
            fn()
        e1.record(stream)
        e1.synchronize()
        return e0.elapsed_time(e1) / iters  # ms per call

    def batched():
        capi.check(batch.encode(in_ptrs, in_strides, budgets, out_ptrs, out_strides, stream.cuda_stream), "batch")

    batch_ms = timed(batched)
    sizes = batch.sizes()
    chosen = batch.shape()
    # Both execution modes at their best shape among a few, for the record.
    modes = {}
    for name, kw in (("persistent", dict(persistent=True, small_level=chosen["small_level"], ctas_per_sm=0)),
                     ("per_stage", dict(persistent=False, small_level=chosen["small_level"], large_below=256))):
        batch.set_shape(**kw, stream=stream.cuda_stream)
        modes[name] = round(frames_n / (timed(batched) * 1e-3), 1)
    batch.set_shape(**{k: v for k, v in chosen.items()}, stream=stream.cuda_stream)

    encs, decs = [], []
    for w, h, c, _ in slots:
        chroma = capi.CHROMA_444 if c else capi.CHROMA_420
        encs.append(capi.Encoder(dev, w, h, chroma))
        decs.append(capi.Decoder(dev, w, h, chroma))

    def plain():
        for i in range(frames_n):
            encs[i].encode_device(in_ptrs[i], in_strides[i], budgets[i], stream.cuda_stream)
            s, m, cap = encs[i].device_bitstream()
            decs[i].decode_blocks(m, s + 8, cap - 2, out_ptrs[i], out_strides[i], stream.cuda_stream)

    plain_ms = timed(plain)
    result = {
        "workload": f"{frames_n} frames of {'/'.join(f'{w}x{h}' for w, h in BATCH_SIZES)}, 4:2:0 and 4:4:4 "
                    f"mixed, budgets 150-250 Mbit/s at 60 fps, encode + decode per frame",
        "frames_per_s": round(frames_n / (batch_ms * 1e-3), 1),
        "megapixels_per_s": round(pixels / (batch_ms * 1e-3) / 1e6, 1),
        "ms_per_call": round(batch_ms, 3),
        "plain_frames_per_s": round(frames_n / (plain_ms * 1e-3), 1),
        "speedup_vs_plain": round(plain_ms / batch_ms, 2),
        "bytes_within_budget": all(s <= b for s, b in zip(sizes, budgets)),
        "autotuned_shape": chosen,
        "frames_per_s_by_mode": modes,
    }
    for o in encs + decs:
        o.close()
    batch.close()
    dev.close()
    return result


def run_serving(seconds: float, streams_n: int = 32, pool_bytes: int = 16 << 30, seed: int = 11,
                saturation_seconds: float = 15.0, outstanding: int = 3):
    """Serving loop: streams_n streams with seeded Poisson frame arrivals at 60
    or 120 fps, sizes from the batched set (4:2:0 and 4:4:4), budgets 150-250
    Mbit/s; every frame is encoded and decoded on the device. Reports latency
    percentiles (submit to completion) and the aggregate frame rate at the
    offered load, then a saturation point: every stream keeps `outstanding`
    frames submitted at all times (offered load above capacity), which gives
    the loop's capacity and its latency there."""
    import torch

    from pyrowave_b200 import capi, synth

    rng = np.random.default_rng(seed)
    dev = capi.Device()
    server = capi.Server(dev, memory_pool_bytes=pool_bytes, max_in_flight=16)
    streams = []
    content = {}
    refused = 0
    for i in range(streams_n):
        w, h = BATCH_SIZES[int(rng.integers(len(BATCH_SIZES)))]
        c444 = bool(rng.integers(2))
        fps = 60.0 if rng.integers(2) == 0 else 120.0
        budget = int(rng.uniform(150e6, 250e6) / 8 / fps) & ~3
        code, sid = server.open_stream(w, h, capi.CHROMA_444 if c444 else capi.CHROMA_420, budget)
        if code != capi.PYROWAVE_SUCCESS:
            refused += 1
            continue
        key = (w, h, c444)
        if key not in content:
            content[key] = [torch.from_numpy(p).cuda() for p in synth.synth_frame(w, h, c444, 2000 + len(content))]
        inp = content[key]
        out = [torch.empty_like(p) for p in inp]
        streams.append(dict(sid=sid, fps=fps, budget=budget, inp=([p.data_ptr() for p in inp],
                                                                  [p.stride(0) for p in inp]),
                            out=([p.data_ptr() for p in out], [p.stride(0) for p in out]), keep=out,
                            next=float(rng.exponential(1.0 / fps))))
    torch.cuda.synchronize()  # inputs complete before the server's streams read them
    # Warm up every stream once (first-use allocation and graph capture).
    for st in streams:
        server.submit(st["sid"], *st["inp"], st["budget"], *st["out"])
    got = 0
    while got < len(streams):
        got += len(server.poll(timeout_us=100000))
    failures = 0

    # Offered load: Poisson arrivals.
    server.stats(reset=True)
    start = time.perf_counter()
    submitted = completed = 0
    nbytes = 0
    while True:
        now = time.perf_counter() - start
        if now >= seconds:
            break
        for st in streams:
            while st["next"] <= now:
                server.submit(st["sid"], *st["inp"], st["budget"], *st["out"])
                submitted += 1
                st["next"] += float(rng.exponential(1.0 / st["fps"]))
        for _, _, result, b, _ in server.poll(timeout_us=0):
            completed += 1
            nbytes += b
            failures += result != capi.PYROWAVE_SUCCESS
        time.sleep(0.0002)
    while completed < submitted:
        for _, _, result, b, _ in server.poll(timeout_us=100000):
            completed += 1
            nbytes += b
            failures += result != capi.PYROWAVE_SUCCESS
    elapsed = time.perf_counter() - start
    p50, p99, frames = server.stats(reset=True)
    offered = sum(st["fps"] for st in streams)

    # Saturation: a closed loop with `outstanding` frames per stream.
    by_sid = {st["sid"]: st for st in streams}
    sat_done = 0
    for st in streams:
        for _ in range(outstanding):
            server.submit(st["sid"], *st["inp"], st["budget"], *st["out"])
    t0 = time.perf_counter()
    while time.perf_counter() - t0 < saturation_seconds:
        for _, sid, result, _, _ in server.poll(timeout_us=1000):
            sat_done += 1
            failures += result != capi.PYROWAVE_SUCCESS
            st = by_sid[sid]
            server.submit(sid, *st["inp"], st["budget"], *st["out"])
    sat_elapsed = time.perf_counter() - t0
    s50, s99, _ = server.stats(reset=True)
    server.close()
    dev.close()
    return {
        "workload": f"{streams_n} streams, Poisson arrivals at 60/120 fps, sizes {len(BATCH_SIZES)}-way mixed, "
                    f"4:2:0 and 4:4:4, budgets 150-250 Mbit/s, {pool_bytes >> 30} GiB state pool, "
                    f"{seconds:g} s",
        "streams_admitted": len(streams), "streams_refused": refused,
        "offered_frames_per_s": round(offered, 1),
        "frames_per_s": round(completed / elapsed, 1),
        "p50_latency_us": round(p50, 1), "p99_latency_us": round(p99, 1),
        "frames": int(frames), "mean_bytes": round(nbytes / max(completed, 1), 1),
        "failed_requests": int(failures),
        "saturation": {"method": f"closed loop, {outstanding} frames outstanding per stream, "
                                 f"{saturation_seconds:g} s",
                       "frames_per_s": round(sat_done / sat_elapsed, 1),
                       "p50_latency_us": round(s50, 1), "p99_latency_us": round(s99, 1)},
    }


SECONDARY = [
    # (name, config, budget, precision mask)
    ("720p", "720p", 150000, 0),
    ("1080p_fp16_storage", "1080p", 400000, 0x3),
    ("1080p_reference_precision", "1080p", 400000, 0x103),
    ("4k", "4k", 1200000, 0),
    ("4k_fp16_storage", "4k", 1200000, 0x3),
    ("4k444_600000", "4k444", 600000, 0),
    ("4k444_1200000", "4k444", 1200000, 0),
    ("4k444_2400000", "4k444", 2400000, 0),
]


def measure_config(dev, cfg, budget, mask, steps, warmup):
    """Device-resident encode + decode of one configuration: us/frame over
    `steps` frames (inputs rotated through more than twice L2), then the same
    steps with per-kernel events for per-stage us and GB/s (algorithmic bytes)."""
    import torch

    from pyrowave_b200 import capi

    w, h, c444 = cfg["width"], cfg["height"], cfg["chroma444"]
    chroma = capi.CHROMA_444 if c444 else capi.CHROMA_420
    base = [[torch.from_numpy(p).cuda() for p in f] for f in make_frames(dict(cfg, seeds=cfg["seeds"][:2]))]
    frame_bytes = sum(p.numel() for p in base[0])
    n = max(len(base), -(-2 * (126 << 20) // frame_bytes))
    nb = len(base)
    frames = [[torch.roll(p, shifts=(3 * (i // nb), 5 * (i // nb)), dims=(0, 1)).contiguous() if i >= nb else p
               for p in base[i % nb]] for i in range(n)]
    out = [torch.empty_like(p) for p in base[0]]
    enc = capi.Encoder(dev, w, h, chroma, mask)
    dec = capi.Decoder(dev, w, h, chroma, mask)
    stream = torch.cuda.Stream()
    sid = stream.cuda_stream
    sizes = []
    torch.cuda.synchronize()  # inputs complete before the library's stream reads them

    def step(i):
        f = frames[i % len(frames)]
        enc.encode_device([p.data_ptr() for p in f], [p.stride(0) for p in f], budget, sid)
        s, m, cap = enc.device_bitstream()
        dec.decode_blocks(m, s + 8, cap - 2, [p.data_ptr() for p in out], [p.stride(0) for p in out], sid)

    for i in range(warmup):
        step(i)
        torch.cuda.synchronize()
        sizes.append(enc.size())

    def timed():
        e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        torch.cuda.synchronize()
        e0.record(stream)
        for i in range(steps):
            step(i)
        e1.record(stream)
        e1.synchronize()
        return e0.elapsed_time(e1) / steps

    ms = timed()
    dev.set_stage_timing(True)
    dev.report_performance_stats(reset=True)
    timed()
    stages = {}
    for line in dev.report_performance_stats(reset=True):
        tag, rest = line.split(":", 1)
        stages[tag.strip()] = float(rest.split("ms")[0])
    dev.set_stage_timing(False)
    alg = algorithmic_bytes(dict(cfg, budget=budget), mask & 0x1F)
    dwt_ms = sum(v for k, v in stages.items() if k.startswith("dwt"))
    enc.close()
    dec.close()
    psnr = None
    if mask != 0x103:
        psnr = psnr_delta(cfg, [[p.cpu().numpy() for p in f] for f in base], budget, mask)
    return {
        "workload": f"encode+decode {w}x{h} {'4:4:4' if c444 else '4:2:0'} 8-bit, {budget}-byte budget",
        "precision_mask": hex(mask), "us_per_frame": round(ms * 1e3, 2),
        "bytes_per_frame": max(sizes), "within_budget": all(0 < s <= budget for s in sizes),
        "stages_us": {k: round(v * 1e3, 2) for k, v in stages.items()},
        "stages_gbs": {k: round(alg[k] / (v * 1e-3) / 1e9, 1) for k, v in stages.items() if k in alg and v > 0},
        "dwt_stage_gbs": round(alg["dwt_stage"] / (dwt_ms * 1e-3) / 1e9, 1) if dwt_ms else None,
        "psnr_delta_db": psnr,
        "note": "stage times carry one event pair per kernel (launch gaps included)",
    }


def measure_transform(dev, cfg, steps: int = 30):
    """The forward transform alone (pyrowave_cuda_encoder_transform: five levels,
    no quantiser) with an event after every level: per-level us and GB/s of
    algorithmic bytes (8-bit input read once, all four bands written once per
    level), and the stage as a whole (input planes read once, transmitted
    coefficients written once) against the measured HBM peak."""
    import torch

    from pyrowave_b200 import capi

    w, h, c444 = cfg["width"], cfg["height"], cfg["chroma444"]
    chroma = capi.CHROMA_444 if c444 else capi.CHROMA_420
    base = [[torch.from_numpy(p).cuda() for p in f] for f in make_frames(dict(cfg, seeds=cfg["seeds"][:1]))]
    frame_bytes = sum(p.numel() for p in base[0])
    n = max(1, -(-2 * (126 << 20) // frame_bytes))
    frames = [[torch.roll(p, shifts=(3 * i, 5 * i), dims=(0, 1)).contiguous() if i else p for p in base[0]]
              for i in range(n)]
    enc = capi.Encoder(dev, w, h, chroma)
    stream = torch.cuda.Stream()
    torch.cuda.synchronize()  # inputs complete before the library's stream reads them
    for i in range(3):
        f = frames[i % n]
        enc.transform([p.data_ptr() for p in f], [p.stride(0) for p in f], stream.cuda_stream)
    torch.cuda.synchronize()
    dev.set_stage_timing(True)
    dev.report_performance_stats(reset=True)
    for i in range(steps):
        f = frames[i % n]
        enc.transform([p.data_ptr() for p in f], [p.stride(0) for p in f], stream.cuda_stream)
        torch.cuda.synchronize()
    stages = {}
    for line in dev.report_performance_stats(reset=True):
        tag, rest = line.split(":", 1)
        stages[tag.strip()] = float(rest.split("ms")[0])
    dev.set_stage_timing(False)
    # The stage as it runs without the per-level events (consecutive levels
    # overlapping through programmatic launches): one event pair per call.
    live_ms = 0.0
    for i in range(steps):
        f = frames[i % n]
        e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        with torch.cuda.stream(stream):
            torch.cuda._sleep(50000)  # keeps the stream busy while the host queues the levels
        e0.record(stream)
        enc.transform([p.data_ptr() for p in f], [p.stride(0) for p in f], stream.cuda_stream)
        e1.record(stream)
        e1.synchronize()
        live_ms += e0.elapsed_time(e1)
    live_ms /= steps
    enc.close()
    alg = algorithmic_bytes(cfg, 0)
    peak, peak_kind = measured_peak()
    levels = {k: v for k, v in stages.items() if k.startswith("xdwt")}
    total_ms = sum(levels.values())
    out = {"workload": f"forward transform alone, {w}x{h} {'4:4:4' if c444 else '4:2:0'}",
           "levels_us": {k: round(v * 1e3, 2) for k, v in levels.items()},
           "levels_gbs": {k: round(alg[k[1:]] / (v * 1e-3) / 1e9, 1) for k, v in levels.items() if v > 0},
           "stage_us": round(total_ms * 1e3, 2), "peak_gbs": peak, "peak_source": peak_kind}
    if total_ms:
        out["stage_gbs"] = round(alg["dwt_stage"] / (total_ms * 1e-3) / 1e9, 1)
        out["stage_frac_of_peak"] = round(out["stage_gbs"] / peak, 4)
        l0 = levels.get("xdwt0")
        if l0:
            out["level0_frac_of_peak"] = round(alg["dwt0"] / (l0 * 1e-3) / 1e9 / peak, 4)
    if live_ms > 0:
        out["stage_us_live"] = round(live_ms * 1e3, 2)
        out["stage_gbs_live"] = round(alg["dwt_stage"] / (live_ms * 1e-3) / 1e9, 1)
        out["stage_frac_of_peak_live"] = round(out["stage_gbs_live"] / peak, 4)
    return out


def run_secondary(steps, warmup):
    from pyrowave_b200 import capi

    dev = capi.Device()
    out = {}
    for name, cfg_name, budget, mask in SECONDARY:
        out[name] = measure_config(dev, CONFIGS[cfg_name], budget, mask, steps, warmup)
    for name in ("1080p", "4k444"):
        out[f"transform_only_{name}"] = measure_transform(dev, CONFIGS[name])
    dev.close()
    return out


def _ncu_entry(kernel, cfg):
    """The committed ncu figures of `kernel` at this workload (profiles/ncu_traffic.json):
    DRAM bytes per launch and, where captured, the share of issue slots busy and of
    DRAM throughput."""
    p = os.path.join(ROOT, "profiles", "ncu_traffic.json")
    try:
        with open(p) as f:
            d = json.load(f)
        key = f"{cfg['width']}x{cfg['height']}{'_444' if cfg['chroma444'] else ''}:{kernel}"
        e = d.get(key)
        return e if isinstance(e, dict) else ({"traffic": e} if e is not None else None)
    except Exception:
        return None


def _ncu_traffic(kernel, cfg):
    """DRAM bytes per launch of `kernel` from the committed ncu summary, if present."""
    e = _ncu_entry(kernel, cfg)
    return e.get("traffic") if e else None


def _ncu_limit(kernel, cfg):
    """What bounds `kernel` by its committed ncu figures: instruction issue when the
    issue slots are far busier than DRAM."""
    e = _ncu_entry(kernel, cfg)
    if not e or "issue_active_pct" not in e or "dram_pct" not in e:
        return None
    kind = "instruction issue" if e["issue_active_pct"] > 2 * e["dram_pct"] else "hbm"
    return {"limit": kind, "issue_slots_busy_pct": e["issue_active_pct"], "dram_throughput_pct": e["dram_pct"],
            "source": e.get("source", "profiles/ncu_traffic.json")}


E2E_PAIRS = 6  # encoder/decoder pairs (streams, host threads) in flight in the end-to-end measurement


def run_e2e(args, cfg, frames, dev):
    """Encode + decode through the reference-facing C API with host (pinned)
    buffers: pyrowave_encoder_encode_cpu_synchronous (input planes uploaded
    inside), compute_num_packets + packetize (the frame read back), one
    pyrowave_decoder_push_packet of the whole packetized frame (the parser
    walks the concatenated packets, as the reference's does) and
    pyrowave_decoder_decode_cpu_buffer_synchronous (payload uploaded, planes
    read back).

    The timed run keeps E2E_PAIRS encoder/decoder pairs, each on its own device
    object (its own CUDA stream) and host thread: a thread encodes its frame
    (which returns without waiting, pyrowave.h:445-447), packetizes, pushes and
    decodes it, then takes its next frame, so the frames of different threads
    overlap their copies and kernels (the C API calls release the interpreter
    lock). A sequential pass with one pair gives the per-call breakdown."""
    import concurrent.futures

    import torch

    from pyrowave_b200 import capi

    w, h, c444, budget = cfg["width"], cfg["height"], cfg["chroma444"], cfg["budget"]
    chroma = capi.CHROMA_444 if c444 else capi.CHROMA_420
    devs = [dev] + [capi.Device() for _ in range(E2E_PAIRS - 1)]
    pairs = [(capi.Encoder(d, w, h, chroma, args.fp16_mask), capi.Decoder(d, w, h, chroma, args.fp16_mask))
             for d in devs]
    pinned = [[torch.from_numpy(p).pin_memory().numpy() for p in f] for f in frames]
    outs = [[torch.empty(p.shape, dtype=torch.uint8).pin_memory().numpy() for p in frames[0]] for _ in pairs]
    bitstreams = [torch.empty(budget, dtype=torch.uint8).pin_memory().numpy() for _ in pairs]
    boundary = 8192
    packets = [(capi.Packet * 4096)() for _ in pairs]
    got = [capi.c_size_t() for _ in pairs]

    def encode(k, i):
        capi.check(pairs[k][0].encode_cpu(pinned[i % len(pinned)], budget), "encode_cpu_synchronous")

    def finish(k):
        enc, dec = pairs[k]
        bs = bitstreams[k]
        n = enc.compute_num_packets(boundary)
        assert n <= len(packets[k])
        capi.check(enc.L.pyrowave_encoder_packetize(enc.h, packets[k], boundary, capi.ctypes.byref(got[k]),
                                                    capi.ctypes.c_void_p(bs.ctypes.data), budget), "packetize")
        total = packets[k][got[k].value - 1].offset + packets[k][got[k].value - 1].size
        t_pk = time.perf_counter()
        capi.check(dec.push_packet_ptr(bs.ctypes.data, total), "push_packet")
        t_push = time.perf_counter()
        code, _ = dec.decode_cpu(outs[k])
        capi.check(code, "decode_cpu_buffer_synchronous")
        return total, t_pk, t_push

    # Sequential pass with one pair: per-call host times.
    for i in range(3):
        encode(0, i)
        finish(0)
    nseq = max(args.steps // 4, 10)
    acc = dict(encode=0.0, packetize=0.0, push_packet=0.0, decode=0.0)
    t_all = time.perf_counter()
    for i in range(nseq):
        t0 = time.perf_counter()
        encode(0, i)
        t1 = time.perf_counter()
        _, t_pk, t_push = finish(0)
        t2 = time.perf_counter()
        acc["encode"] += t1 - t0
        acc["packetize"] += t_pk - t1
        acc["push_packet"] += t_push - t_pk
        acc["decode"] += t2 - t_push
    seq_us = (time.perf_counter() - t_all) * 1e6 / nseq
    breakdown = {k: round(v * 1e6 / nseq, 1) for k, v in acc.items()}
    breakdown["sequential_total"] = round(seq_us, 1)
    breakdown["notes"] = ("encode: upload + launch, returns without waiting; packetize: waits for the encode, "
                          "reads the frame back, cuts packets; push_packet: host parse of the whole frame; "
                          "decode: payload upload, dequantise + inverse DWT, planes read back")

    # Timed run: one host thread per pair, frames dealt round robin.
    for i in range(2 * E2E_PAIRS):
        encode(i % E2E_PAIRS, i)
        finish(i % E2E_PAIRS)
    n = max(args.steps, 10)

    def worker(k):
        done = 0
        for i in range(k, n, E2E_PAIRS):
            encode(k, i)
            done += finish(k)[0]
        return done

    t0 = time.perf_counter()
    with concurrent.futures.ThreadPoolExecutor(E2E_PAIRS) as ex:
        total_bytes = sum(ex.map(worker, range(E2E_PAIRS)))
    t1 = time.perf_counter()
    blocks32 = pairs[0][0].layout().block_count_32x32
    for enc, dec in pairs:
        enc.close()
        dec.close()
    for d in devs[1:]:
        d.close()
    planes_bytes = sum(p.nbytes for p in frames[0])
    avg_stream = total_bytes // n
    return {"total_s": t1 - t0, "frames": n,
            "h2d": planes_bytes + avg_stream + 4 * blocks32,
            "d2h": planes_bytes + budget + 8 * blocks32 + 8,
            "method": f"{E2E_PAIRS} encoder/decoder pairs on {E2E_PAIRS} CUDA streams and host threads, frames "
                      "dealt round robin; per frame: encode (upload + launch), packetize, one push_packet of the "
                      "whole frame, decode (payload upload, kernels, planes read back)",
            "breakdown_us": breakdown}


def cpu_model() -> str:
    """The host CPU's model name (Linux /proc/cpuinfo), or "unknown"."""
    try:
        with open("/proc/cpuinfo") as f:
            for line in f:
                if line.startswith("model name"):
                    return line.split(":", 1)[1].strip()
    except OSError:
        pass
    return "unknown"


def _oracle_frame(O, f, w, h, c444, budget, mode):
    """One frame through the oracle (encode, packetize, parse, decode); seconds per stage."""
    t = {}
    o = O.Oracle(w, h, c444)
    t0 = time.perf_counter()
    pyr = o.dwt(f, mode)
    t1 = time.perf_counter()
    o.encode_pyramid(pyr, budget)
    t2 = time.perf_counter()
    stream, packets = o.packetize(8192, budget + 64)
    t3 = time.perf_counter()
    p = o.parser()
    for off, sz in packets:
        p.push(stream[off:off + sz].tobytes())
    offs, payload = p.get()
    t4 = time.perf_counter()
    coef = o.dequant(offs, payload, mode)
    t5 = time.perf_counter()
    o.idwt(coef, mode)
    t6 = time.perf_counter()
    t.update(dwt=t1 - t0, quant_rate_pack=t2 - t1, packetize=t3 - t2, parse=t4 - t3, dequant=t5 - t4, idwt=t6 - t5)
    return t


def cpu_baseline(cfg, frames, seconds, single_frames: int = 3):
    """The oracle (the reference algorithm restated in C++) on all host cores,
    plus a single-thread pass over a few frames with per-stage times."""
    import oracle as O

    cores = os.cpu_count() or 1
    w, h, c444, budget = cfg["width"], cfg["height"], cfg["chroma444"], cfg["budget"]

    def one(f):
        return _oracle_frame(O, f, w, h, c444, budget, O.MODE_F32)

    # Single thread: per-stage times (the first frame also warms the oracle's tables).
    one(frames[0])
    stages = {}
    t0 = time.perf_counter()
    for i in range(single_frames):
        for k, v in one(frames[i % len(frames)]).items():
            stages[k] = stages.get(k, 0.0) + v
    single_us = (time.perf_counter() - t0) * 1e6 / single_frames

    done = 0
    t0 = time.perf_counter()
    with concurrent.futures.ThreadPoolExecutor(max_workers=cores) as ex:
        while time.perf_counter() - t0 < seconds:
            list(ex.map(one, [frames[(done + k) % len(frames)] for k in range(cores)]))
            done += cores
    dt = time.perf_counter() - t0
    return {"value": round(dt * 1e6 / done, 1), "unit": "us/frame", "cores": cores, "kind": "port",
            "cpu_model": cpu_model(),
            "sample": f"{done} frames encoded+decoded on {cores} threads in {dt:.1f} s (oracle restatement, FP32); "
                      f"single thread: {single_frames} frames",
            "single_thread_us_per_frame": round(single_us, 1),
            "single_thread_stages_us": {k: round(v * 1e6 / single_frames, 1) for k, v in stages.items()}}


def run_reference(args, cfg, ws, rank):
    if rank != 0:
        return
    frames = make_frames(cfg)
    cores = os.cpu_count() or 1
    import oracle as O

    w, h, c444, budget = cfg["width"], cfg["height"], cfg["chroma444"], cfg["budget"]

    def one(f):
        o = O.Oracle(w, h, c444)
        o.encode(f, budget, O.MODE_REF16)
        stream, packets = o.packetize(8192, budget + 64)
        p = o.parser()
        for off, sz in packets:
            p.push(stream[off:off + sz].tobytes())
        offs, payload = p.get()
        o.idwt(o.dequant(offs, payload, O.MODE_REF16), O.MODE_REF16)

    per_step = cores  # one frame per host thread per step
    with concurrent.futures.ThreadPoolExecutor(max_workers=cores) as ex:
        for i in range(args.warmup):
            list(ex.map(one, [frames[(i * per_step + k) % len(frames)] for k in range(per_step)]))
        t0 = time.perf_counter()
        for i in range(args.steps):
            list(ex.map(one, [frames[(i * per_step + k) % len(frames)] for k in range(per_step)]))
        dt = time.perf_counter() - t0
    us = dt * 1e6 / (args.steps * per_step)
    line = {
        "impl": "reference",
        "metric": f"us/frame enc+dec {cfg['width']}x{cfg['height']} {'4:4:4' if c444 else '4:2:0'} @ {budget} B",
        "value": round(us, 1), "unit": "us/frame", "n_gpus": ws, "steps": args.steps, "warmup": args.warmup,
        "ms_per_step": round(dt * 1e3 / args.steps, 3), "higher_is_better": False, "scaling": "weak",
        "vs_baseline": None, "dtype": "f32 (fp16 staging, the reference's default precision)",
        "data": "synthetic (seeded gradient + band-limited noise + rectangles)",
        "config": workload_config(cfg, frames, ws),
        "cpu_baseline": {"value": round(us, 1), "unit": "us/frame", "cores": cores, "kind": "port",
                         "cpu_model": cpu_model(),
                         "sample": f"{args.steps * per_step} frames, {per_step} per step on {cores} threads "
                                   "(the reference's Vulkan path needs a graphics stack: unavailable on this box)"},
        "e2e": {"value": round(us, 1), "unit": "us/frame", "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0},
    }
    print(json.dumps(line), flush=True)


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=200)
    ap.add_argument("--warmup", type=int, default=10)
    ap.add_argument("--impl", default="ours", choices=["ours", "reference"])
    ap.add_argument("--config", default="1080p", choices=sorted(CONFIGS))
    ap.add_argument("--fp16-mask", type=lambda s: int(s, 0), default=0)
    ap.add_argument("--cpu-seconds", type=float, default=10.0)
    ap.add_argument("--no-cpu-baseline", action="store_true")
    ap.add_argument("--no-batch", action="store_true", help="skip the batched-form measurement")
    ap.add_argument("--no-e2e", action="store_true",
                    help="skip the end-to-end measurement through host buffers (profiling runs)")
    ap.add_argument("--batch-frames", type=int, default=64,
                    help="frames in the batched-form measurement (64: the batched benchmark's set)")
    ap.add_argument("--no-configs", action="store_true",
                    help="skip the other configurations (720p, FP16 storage, reference precision, 4K, 4K 4:4:4 sweep)")
    ap.add_argument("--serve-seconds", type=float, default=60.0,
                    help="duration of the serving-loop measurement (0: skip)")
    ap.add_argument("--l2", default="rotate", choices=["rotate", "flush"],
                    help="rotate: distinct inputs larger than L2; flush: 256 MiB write between steps")
    args = ap.parse_args()
    if args.warmup < 3:
        args.warmup = 3
    ws, rank, local = dist_info()
    cfg = CONFIGS[args.config]
    if args.impl == "reference":
        if args.steps > 50:
            args.steps = 20  # each reference step is a full frame per host core
        run_reference(args, cfg, ws, rank)
        return
    run_ours(args, cfg, ws, rank, local)


if __name__ == "__main__":
    main()
