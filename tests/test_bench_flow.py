"""bench.py's measurement flow on CPU, with the GPU parts replaced by stand-ins.

The stand-ins (CUDA events that report 0.1 ms per step, a no-op stream and
synchronize, coder objects that only count calls, a fixed end-to-end result)
let run_ours execute its whole control flow on a machine without a GPU: warm-up,
the clock-load steps, both timed passes, the roofline and the JSON line. It
checks the line's keys and the arithmetic behind `value`; it says nothing about
speed.
"""
import contextlib
import io
import json
import os
import sys
import types

import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
if ROOT not in sys.path:
    sys.path.insert(0, ROOT)

import bench  # noqa: E402

STEP_MS = 0.1
_clock = [0.0]  # fake device time: every encode_device call (one step) takes STEP_MS


class _Event:
    def __init__(self, enable_timing=False):
        self.t = 0.0

    def record(self, stream=None):
        self.t = _clock[0]

    def elapsed_time(self, other):
        return other.t - self.t


class _Stream:
    cuda_stream = 0


class _Coder:
    calls = 0

    def __init__(self, *a, **k):
        self.stage = False

    def encode_device(self, *a):
        _Coder.calls += 1
        _clock[0] += STEP_MS

    def device_bitstream(self):
        return 0, 0, 1000

    def decode_blocks(self, *a):
        pass

    def size(self):
        return 4000

    def set_stage_timing(self, on):
        self.stage = on

    def report_performance_stats(self, reset=False):
        tags = ["dwt0", "dwt1", "dwt2", "dwt3", "dwt4", "quant", "resolve", "pack", "dequant",
                "idwt4", "idwt3", "idwt2", "idwt1", "idwt0"]
        return [f"{t}: 0.0050 ms per frame" for t in tags]


@pytest.fixture
def fake_gpu(monkeypatch):
    import torch

    from pyrowave_b200 import capi

    monkeypatch.setattr(torch.cuda, "set_device", lambda *a: None)
    monkeypatch.setattr(torch.cuda, "synchronize", lambda *a: None)
    monkeypatch.setattr(torch.cuda, "Stream", lambda *a, **k: _Stream())
    monkeypatch.setattr(torch.cuda, "Event", _Event)
    monkeypatch.setattr(torch.cuda, "stream", lambda s: contextlib.nullcontext())
    monkeypatch.setattr(torch.Tensor, "cuda", lambda self, *a, **k: self)
    real_empty = torch.empty
    monkeypatch.setattr(torch, "empty", lambda *a, device=None, **k: real_empty(*a, **k))
    monkeypatch.setattr(capi, "Device", _Coder)
    monkeypatch.setattr(capi, "Encoder", _Coder)
    monkeypatch.setattr(capi, "Decoder", _Coder)
    monkeypatch.setattr(bench, "run_e2e", lambda *a: {"total_s": 0.004, "frames": 10, "h2d": 55296, "d2h": 55296,
                                                      "method": "stand-in", "breakdown_us": {}})
    monkeypatch.setattr(bench, "ClockSampler", _NoClocks)


class _NoClocks(bench.ClockSampler):
    def start(self):
        self.proc = None


def test_run_ours_json_line(fake_gpu):
    cfg = dict(width=256, height=144, chroma444=False, budget=20000, seeds=[1, 2], rects=4, lines=0)
    args = types.SimpleNamespace(steps=20, warmup=3, fp16_mask=0, l2="rotate", no_cpu_baseline=True,
                                 no_batch=True, no_configs=True, serve_seconds=0, cpu_seconds=0)
    out = io.StringIO()
    with contextlib.redirect_stdout(out):
        bench.run_ours(args, cfg, 1, 0, 0)
    line = json.loads(out.getvalue().strip().splitlines()[-1])
    for key in ("metric", "value", "unit", "n_gpus", "steps", "warmup", "ms_per_step", "higher_is_better",
                "scaling", "vs_baseline", "dtype", "data", "config", "e2e", "gpu_launches", "roofline",
                "clocks", "cpu_baseline"):
        assert key in line, key
    # 20 steps of 0.1 ms on one rank: 100 us per frame.
    assert line["value"] == pytest.approx(STEP_MS * 1e3)
    assert line["ms_per_step"] == pytest.approx(STEP_MS)
    assert line["n_gpus"] == 1 and line["steps"] == 20 and line["higher_is_better"] is False
    assert line["clocks"]["load_steps_before_timed"] >= 64
    assert line["gpu_launches"] == 14 * 20
    assert line["roofline"]["bound"] == "hbm" and line["roofline"]["frac"] > 0
    assert line["e2e"]["value"] == pytest.approx(0.004 * 1e6 / 10)
    assert len(line["config"]["frames_fingerprint"]) == 16
