"""The batched form: frames of mixed sizes, chroma formats and budgets through
one graph launch per call give the same bitstreams and decoded planes as the
single-frame encoder and decoder, before and after autotuning."""
import numpy as np
import pytest

from pyrowave_b200 import capi, synth

pytestmark = pytest.mark.gpu

# (width, height, 4:4:4, budget)
FRAMES = [
    (1280, 720, False, 150000),
    (130, 98, False, 20000),
    (200, 128, True, 30000),
    (640, 360, True, 60000),
    (34, 30, False, 65536),
    (1366, 768, False, 200000),
]


@pytest.fixture(scope="module")
def device(gpu):
    dev = capi.Device()
    yield dev
    dev.close()


def _inputs(seed_base):
    import torch

    planes = [synth.synth_frame(w, h, c444, seed_base + i) for i, (w, h, c444, _) in enumerate(FRAMES)]
    dev_planes = [[torch.from_numpy(p).cuda() for p in pl] for pl in planes]
    return planes, dev_planes


def _ptrs(tensors):
    return [[t.data_ptr() for t in ts] for ts in tensors], [[t.stride(0) for t in ts] for ts in tensors]


def _reference(device, dev_planes, budgets, calls):
    """Single-frame encoders run `calls` times (same budgets); returns the last stream bytes and decodes."""
    import torch

    streams, decoded = [], []
    for (w, h, c444, _), pl, budget in zip(FRAMES, dev_planes, budgets):
        chroma = capi.CHROMA_444 if c444 else capi.CHROMA_420
        enc = capi.Encoder(device, w, h, chroma)
        for _ in range(calls):
            enc.encode_device([p.data_ptr() for p in pl], [p.stride(0) for p in pl], budget)
        torch.cuda.synchronize()
        n = enc.size()
        s, m, _ = enc.device_bitstream()
        streams.append(_copy_device_words(s, n // 4))
        dec = capi.Decoder(device, w, h, chroma)
        outs = [torch.zeros_like(p) for p in pl]
        dec.decode_blocks(m, s + 8, n // 4 - 2, [t.data_ptr() for t in outs], [t.stride(0) for t in outs])
        torch.cuda.synchronize()
        decoded.append([t.cpu().numpy() for t in outs])
    return streams, decoded


class _DeviceWords:
    """A view of library-owned device memory for torch (CUDA array interface)."""

    def __init__(self, ptr, nwords):
        self.__cuda_array_interface__ = {"shape": (nwords,), "typestr": "<i4", "data": (ptr, False), "version": 3}


def _copy_device_words(ptr, nwords):
    import torch

    t = torch.as_tensor(_DeviceWords(ptr, nwords), device="cuda")
    return t.cpu().numpy().view(np.uint32).copy()


def test_batch_matches_single_frame(device):
    import torch

    planes, dev_planes = _inputs(40)
    budgets = [b for *_, b in FRAMES]
    infos = [(w, h, capi.CHROMA_444 if c444 else capi.CHROMA_420, 2 * b) for w, h, c444, b in FRAMES]
    batch = capi.Batch(device, infos)
    outs = [[torch.full_like(p, 0x55) for p in pl] for pl in dev_planes]
    in_ptrs, in_strides = _ptrs(dev_planes)
    out_ptrs, out_strides = _ptrs(outs)

    for call, scale in enumerate([1.0, 0.6]):
        b = [int(x * scale) for x in budgets]
        assert batch.encode(in_ptrs, in_strides, b, out_ptrs, out_strides) == capi.PYROWAVE_SUCCESS
        sizes = batch.sizes()
        ref_streams, ref_decoded = _reference(device, dev_planes, b, call + 1)
        for i in range(len(FRAMES)):
            assert sizes[i] <= b[i]
            s, _ = batch.device_bitstream(i)
            got = _copy_device_words(s, sizes[i] // 4)
            assert np.array_equal(got, ref_streams[i]), f"frame {i} call {call}: bitstream differs"
            for p in range(3):
                assert np.array_equal(outs[i][p].cpu().numpy(), ref_decoded[i][p]), f"frame {i} plane {p}"

    # The autotuner may pick other CTA shapes; the next call's output is unchanged.
    b = [int(x * 0.8) for x in budgets]
    assert batch.autotune(in_ptrs, in_strides, b, out_ptrs, out_strides) == capi.PYROWAVE_SUCCESS
    assert batch.encode(in_ptrs, in_strides, b, out_ptrs, out_strides) == capi.PYROWAVE_SUCCESS
    sizes = batch.sizes()
    ref_streams, ref_decoded = _reference(device, dev_planes, b, 3)
    for i in range(len(FRAMES)):
        s, _ = batch.device_bitstream(i)
        assert np.array_equal(_copy_device_words(s, sizes[i] // 4), ref_streams[i]), f"frame {i} after autotune"
        for p in range(3):
            assert np.array_equal(outs[i][p].cpu().numpy(), ref_decoded[i][p])
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


def test_batch_frames_past_tensor_map_table(device):
    """Frames past the batch's per-frame TMA map table (64 frames) load their
    tiles with plain loads; both kinds match the single-frame path."""
    import torch

    big = (640, 360, True, 60000)
    shapes = [big] + [(64, 64, False, 4096)] * 63 + [big, (1280, 720, False, 150000)]
    planes = [synth.synth_frame(w, h, c444, 500 + i) for i, (w, h, c444, _) in enumerate(shapes)]
    dev_planes = [[torch.from_numpy(p).cuda() for p in pl] for pl in planes]
    infos = [(w, h, capi.CHROMA_444 if c444 else capi.CHROMA_420, b) for w, h, c444, b in shapes]
    batch = capi.Batch(device, infos)
    outs = [[torch.zeros_like(p) for p in pl] for pl in dev_planes]
    in_ptrs, in_strides = _ptrs(dev_planes)
    out_ptrs, out_strides = _ptrs(outs)
    budgets = [b for *_, b in shapes]
    assert batch.encode(in_ptrs, in_strides, budgets, out_ptrs, out_strides) == capi.PYROWAVE_SUCCESS
    sizes = batch.sizes()
    for i in (0, 64, 65):
        w, h, c444, budget = shapes[i]
        chroma = capi.CHROMA_444 if c444 else capi.CHROMA_420
        enc = capi.Encoder(device, w, h, chroma)
        pl = dev_planes[i]
        enc.encode_device([p.data_ptr() for p in pl], [p.stride(0) for p in pl], budget)
        torch.cuda.synchronize()
        n = enc.size()
        s, m, _ = enc.device_bitstream()
        ref = _copy_device_words(s, n // 4)
        dec = capi.Decoder(device, w, h, chroma)
        ref_out = [torch.zeros_like(p) for p in pl]
        dec.decode_blocks(m, s + 8, n // 4 - 2, [t.data_ptr() for t in ref_out], [t.stride(0) for t in ref_out])
        torch.cuda.synchronize()
        bs, _ = batch.device_bitstream(i)
        assert sizes[i] == n
        assert np.array_equal(_copy_device_words(bs, sizes[i] // 4), ref), f"frame {i}: bitstream differs"
        for p in range(3):
            assert np.array_equal(outs[i][p].cpu().numpy(), ref_out[p].cpu().numpy()), f"frame {i} plane {p}"
    batch.close()
