"""The batched form against the oracle: frames of mixed sizes, chroma formats
and budgets coded in one call give, frame by frame, the oracle's packetized
bitstream and decoded planes, before and after autotuning.

The main case is the batched benchmark's frame set: the six sizes 1280x720,
1366x768, 1920x1080, 2560x1080, 2560x1440 and 3840x2160, in 4:2:0 and 4:4:4,
with budgets drawn from 150-250 Mbit/s at 60 frames/s."""
import concurrent.futures

import numpy as np
import pytest

from oracle_codec import oracle_frame, words_as_bytes
from pyrowave_b200 import capi, synth

pytestmark = pytest.mark.gpu

SIZES = [(1280, 720), (1366, 768), (1920, 1080), (2560, 1080), (2560, 1440), (3840, 2160)]


def _frame_set():
    rng = np.random.default_rng(17)
    out = []
    for c444 in (False, True):
        for w, h in SIZES:
            out.append((w, h, c444, int(rng.uniform(150e6, 250e6) / 8 / 60) & ~3))
    return out


FRAMES = _frame_set()


@pytest.fixture(scope="module")
def device(gpu):
    dev = capi.Device()
    yield dev
    dev.close()


def _ptrs(tensors):
    return [[t.data_ptr() for t in ts] for ts in tensors], [[t.stride(0) for t in ts] for ts in tensors]


class _DeviceWords:
    """A view of library-owned device memory for torch (CUDA array interface)."""

    def __init__(self, ptr, nwords):
        self.__cuda_array_interface__ = {"shape": (nwords,), "typestr": "<i4", "data": (ptr, False), "version": 3}


def _copy_device_words(ptr, nwords):
    import torch

    t = torch.as_tensor(_DeviceWords(ptr, nwords), device="cuda")
    return t.cpu().numpy().view(np.uint32).copy()


def _check_against_oracle(batch, frames, planes, outs, budgets, sequence, what):
    """Every frame's bitstream and decoded planes equal the oracle's for the same
    input, budget and sequence number (oracle runs in parallel threads)."""
    sizes = batch.sizes()
    with concurrent.futures.ThreadPoolExecutor(8) as ex:
        want = list(ex.map(lambda i: oracle_frame(frames[i][0], frames[i][1], frames[i][2], planes[i], budgets[i],
                                                  sequence), range(len(frames))))
    for i, (data, decoded) in enumerate(want):
        assert sizes[i] <= budgets[i]
        assert sizes[i] == data.size, f"{what} frame {i}: {sizes[i]} bytes, oracle {data.size}"
        s, _ = batch.device_bitstream(i)
        got = words_as_bytes(_copy_device_words(s, sizes[i] // 4))
        assert np.array_equal(got, data), f"{what} frame {i}: bitstream differs from the oracle"
        if outs is not None:
            for p in range(3):
                assert np.array_equal(outs[i][p].cpu().numpy(), decoded[p]), f"{what} frame {i} plane {p}"


def test_batch_matches_oracle(device):
    import torch

    planes = [synth.synth_frame(w, h, c444, 40 + i) for i, (w, h, c444, _) in enumerate(FRAMES)]
    dev_planes = [[torch.from_numpy(p).cuda() for p in pl] for pl in planes]
    budgets = [b for *_, b in FRAMES]
    infos = [(w, h, capi.CHROMA_444 if c444 else capi.CHROMA_420, b) for w, h, c444, b in FRAMES]
    batch = capi.Batch(device, infos)
    outs = [[torch.full_like(p, 0x55) for p in pl] for pl in dev_planes]
    in_ptrs, in_strides = _ptrs(dev_planes)
    out_ptrs, out_strides = _ptrs(outs)

    for call, scale in enumerate([1.0, 0.6]):
        b = [int(x * scale) for x in budgets]
        assert batch.encode(in_ptrs, in_strides, b, out_ptrs, out_strides) == capi.PYROWAVE_SUCCESS
        torch.cuda.synchronize()
        _check_against_oracle(batch, FRAMES, planes, outs, b, call + 1, f"call {call}")

    # The autotuner may pick other CTA shapes and does not advance the
    # sequence numbers; the next call's output is unchanged.
    b = [int(x * 0.8) for x in budgets]
    assert batch.autotune(in_ptrs, in_strides, b, out_ptrs, out_strides) == capi.PYROWAVE_SUCCESS
    assert batch.encode(in_ptrs, in_strides, b, out_ptrs, out_strides) == capi.PYROWAVE_SUCCESS
    torch.cuda.synchronize()
    _check_against_oracle(batch, FRAMES, planes, outs, b, 3, "after autotune")

    # Encode only (no outputs): the bitstreams alone.
    assert batch.encode(in_ptrs, in_strides, budgets, None, None) == capi.PYROWAVE_SUCCESS
    torch.cuda.synchronize()
    _check_against_oracle(batch, FRAMES, planes, None, budgets, 4, "encode only")
    batch.close()


def test_batch_small_and_odd_frames(device):
    """Frames below one 32x32 tile per band and odd sizes, mixed with a larger one."""
    import torch

    frames = [(34, 30, False, 65536), (130, 98, False, 20000), (200, 128, True, 30000), (640, 360, True, 60000)]
    planes = [synth.synth_frame(w, h, c444, 70 + i) for i, (w, h, c444, _) in enumerate(frames)]
    dev_planes = [[torch.from_numpy(p).cuda() for p in pl] for pl in planes]
    batch = capi.Batch(device, [(w, h, capi.CHROMA_444 if c else capi.CHROMA_420, b) for w, h, c, b in frames])
    outs = [[torch.zeros_like(p) for p in pl] for pl in dev_planes]
    in_ptrs, in_strides = _ptrs(dev_planes)
    out_ptrs, out_strides = _ptrs(outs)
    budgets = [b for *_, b in frames]
    assert batch.encode(in_ptrs, in_strides, budgets, out_ptrs, out_strides) == capi.PYROWAVE_SUCCESS
    torch.cuda.synchronize()
    _check_against_oracle(batch, frames, planes, outs, budgets, 1, "small frames")
    batch.close()


def test_batch_validation(device):
    import ctypes

    L = capi.lib()
    h = ctypes.c_void_p()
    bad = capi.PYROWAVE_ERROR_INVALID_ARGUMENT
    infos = (capi.BatchFrameInfo * 1)(capi.BatchFrameInfo(65, 64, capi.CHROMA_420, 1000))
    assert L.pyrowave_cuda_batch_create(device.h, infos, 1, ctypes.byref(h)) == bad
    infos = (capi.BatchFrameInfo * 1)(capi.BatchFrameInfo(64, 64, capi.CHROMA_420, 0))
    assert L.pyrowave_cuda_batch_create(device.h, infos, 1, ctypes.byref(h)) == bad
    assert L.pyrowave_cuda_batch_create(device.h, infos, 0, ctypes.byref(h)) == bad
    batch = capi.Batch(device, [(64, 64, capi.CHROMA_420, 4096)])
    import torch

    planes = [torch.zeros((64, 64), dtype=torch.uint8, device="cuda"), torch.zeros((32, 32), dtype=torch.uint8,
                                                                                   device="cuda"),
              torch.zeros((32, 32), dtype=torch.uint8, device="cuda")]
    ptrs, strides = _ptrs([planes])
    # Budget above the slot's maximum.
    assert batch.encode(ptrs, strides, [8192]) == bad
    assert batch.encode(ptrs, strides, [4096]) == capi.PYROWAVE_SUCCESS
    assert batch.sizes()[0] <= 4096
    batch.close()


@pytest.mark.parametrize("persistent", [False, True], ids=["per-stage", "persistent"])
def test_batch_frames_past_tensor_map_table(device, persistent):
    """Per-stage launches: frames past the batch's per-frame TMA map table (64
    frames) load their tiles with plain loads, the first 64 through their maps;
    the persistent launch loads every tile with plain loads. All give the
    oracle's bitstreams and planes, across 66 frames."""
    import torch

    big = (640, 360, True, 60000)
    shapes = [big] + [(64, 64, False, 4096)] * 63 + [big, (1280, 720, False, 150000)]
    planes = [synth.synth_frame(w, h, c444, 500 + i) for i, (w, h, c444, _) in enumerate(shapes)]
    dev_planes = [[torch.from_numpy(p).cuda() for p in pl] for pl in planes]
    infos = [(w, h, capi.CHROMA_444 if c444 else capi.CHROMA_420, b) for w, h, c444, b in shapes]
    batch = capi.Batch(device, infos)
    batch.set_shape(persistent=persistent, small_level=batch.shape()["small_level"], large_below=256)
    outs = [[torch.zeros_like(p) for p in pl] for pl in dev_planes]
    in_ptrs, in_strides = _ptrs(dev_planes)
    out_ptrs, out_strides = _ptrs(outs)
    budgets = [b for *_, b in shapes]
    assert batch.encode(in_ptrs, in_strides, budgets, out_ptrs, out_strides) == capi.PYROWAVE_SUCCESS
    torch.cuda.synchronize()
    sizes = batch.sizes()
    for i in (0, 1, 63, 64, 65):
        w, h, c444, budget = shapes[i]
        data, decoded = oracle_frame(w, h, c444, planes[i], budget, 1)
        assert sizes[i] == data.size
        bs, _ = batch.device_bitstream(i)
        assert np.array_equal(words_as_bytes(_copy_device_words(bs, sizes[i] // 4)), data), f"frame {i}"
        for p in range(3):
            assert np.array_equal(outs[i][p].cpu().numpy(), decoded[p]), f"frame {i} plane {p}"
    batch.close()


@pytest.mark.parametrize("shape", [
    dict(persistent=True, small_level=5, ctas_per_sm=2, large_first=True),
    dict(persistent=True, small_level=3, ctas_per_sm=4, large_first=False),
    dict(persistent=True, small_level=1, ctas_per_sm=3, large_first=False),
    dict(persistent=False, small_level=4, large_below=256),
    dict(persistent=False, small_level=5, large_below=0, branches=3),
    dict(persistent=False, small_level=2, large_below=256, branches=8),
    dict(persistent=False, small_level=5, large_below=0, branches=3, frame_graphs=True),
], ids=["persistent-fused-2cta-large-first", "persistent-small3-4cta", "persistent-small1-3cta", "per-stage",
        "per-stage-3-branches", "per-stage-branches-past-frames", "frame-graphs-3-streams"])
def test_batch_shapes_match_oracle(device, shape):
    """Every execution shape (one persistent launch with its CTA count, frame
    order and transform-only suffix; one launch per stage, in one or more
    concurrent groups of frames; or each frame's own encode and decode graphs
    over several streams) gives the oracle's bitstreams and planes."""
    import torch

    frames = [(1280, 720, False, 150000), (640, 360, True, 60000), (200, 128, True, 30000), (1920, 1080, False, 400000),
              (34, 30, False, 65536)]
    planes = [synth.synth_frame(w, h, c444, 80 + i) for i, (w, h, c444, _) in enumerate(frames)]
    dev_planes = [[torch.from_numpy(p).cuda() for p in pl] for pl in planes]
    batch = capi.Batch(device, [(w, h, capi.CHROMA_444 if c else capi.CHROMA_420, b) for w, h, c, b in frames])
    batch.set_shape(**shape)
    got = batch.shape()
    assert got["persistent"] == int(shape["persistent"]) and got["small_level"] == shape["small_level"]
    # At most one group of frames per frame.
    assert got["branches"] == (1 if shape["persistent"] else min(shape.get("branches", 1), len(frames)))
    assert got["frame_graphs"] == int(shape.get("frame_graphs", False))
    outs = [[torch.zeros_like(p) for p in pl] for pl in dev_planes]
    in_ptrs, in_strides = _ptrs(dev_planes)
    out_ptrs, out_strides = _ptrs(outs)
    budgets = [b for *_, b in frames]
    for call in range(2):
        assert batch.encode(in_ptrs, in_strides, budgets, out_ptrs, out_strides) == capi.PYROWAVE_SUCCESS
        torch.cuda.synchronize()
        _check_against_oracle(batch, frames, planes, outs, budgets, call + 1, f"{shape} call {call}")
    batch.close()
