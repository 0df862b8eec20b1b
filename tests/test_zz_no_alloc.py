"""pyrowave_cuda_decode_blocks_static: the decode entry point that allocates
nothing and keeps its coefficient pyramid in a fixed device array.

This file is collected last so that its GPU test also runs after every other
test of the session has used (and released) device memory.
"""
import ctypes

import numpy as np
import pytest

from pyrowave_b200 import capi, synth


def _dummy_planes(w, h):
    # Never dereferenced: every call below is rejected before any device work.
    return [1, 2, 3], [w, w, w]


def _call(w, h, chroma, num_words=16):
    ptrs, strides = _dummy_planes(w, h)
    return capi.decode_blocks_static(w, h, chroma, 0x1000, 0x2000, num_words, ptrs, strides)


def test_static_decode_rejects_before_device_work():
    bad = capi.PYROWAVE_ERROR_INVALID_ARGUMENT
    assert _call(0, 64, capi.CHROMA_420) == bad
    assert _call(65, 64, capi.CHROMA_420) == bad
    assert _call(64, 64, 5) == bad
    assert _call(64, 64, capi.CHROMA_420, num_words=1 << 33) == bad
    # Frames whose FP32 coefficient storage exceeds the 32 MiB array.
    assert _call(1920, 1080, capi.CHROMA_444) == bad
    assert _call(3840, 2160, capi.CHROMA_420) == bad
    assert _call(2560, 1600, capi.CHROMA_420) == bad
    L = capi.lib()
    assert L.pyrowave_cuda_decode_blocks_static(64, 64, capi.CHROMA_420, None, None, 0, None, None) == bad


def test_static_decode_size_limit_without_device():
    import torch

    if torch.cuda.is_available():
        pytest.skip("checks the no-device path")
    # Within the limit the call gets past validation and fails only for want of a device.
    assert _call(2560, 1440, capi.CHROMA_420) == capi.PYROWAVE_ERROR_GENERIC
    assert _call(1600, 900, capi.CHROMA_444) == capi.PYROWAVE_ERROR_GENERIC


@pytest.mark.gpu
def test_static_decode_matches_decoder_decode_blocks(gpu):
    import torch

    dev = capi.Device()
    # Frames of different layouts, so each call runs over whatever the one
    # before it left in the shared array; the last is the largest documented
    # frame that fits (2560x1440 4:2:0, close to the array's size).
    frames = [(1280, 720, capi.CHROMA_420, 150000, 1), (320, 240, capi.CHROMA_444, 30000, 2),
              (2560, 1440, capi.CHROMA_420, 500000, 3)]
    encoded = []
    for w, h, chroma, budget, seed in frames:
        enc = capi.Encoder(dev, w, h, chroma)
        planes = synth.synth_frame(w, h, chroma == capi.CHROMA_444, seed)
        d = [torch.from_numpy(p).cuda() for p in planes]
        enc.encode_device([p.data_ptr() for p in d], [p.stride(0) for p in d], budget)
        torch.cuda.synchronize()
        stream_ptr, meta_ptr, _ = enc.device_bitstream()
        total = enc.size()
        encoded.append((enc, w, h, chroma, planes, meta_ptr, stream_ptr + 8, total // 4 - 2))

    def alloc(planes):
        return [torch.full(p.shape, 0x55, dtype=torch.uint8, device="cuda") for p in planes]

    # Existing entry point, one decoder per frame.
    want = []
    for enc, w, h, chroma, planes, meta, words, n in encoded:
        dec = capi.Decoder(dev, w, h, chroma)
        out = alloc(planes)
        dec.decode_blocks(meta, words, n, [t.data_ptr() for t in out], [t.stride(0) for t in out])
        torch.cuda.synchronize()
        want.append([t.cpu().numpy() for t in out])
        dec.close()

    # The calls in a row on one stream, then compare each.
    got = []
    for enc, w, h, chroma, planes, meta, words, n in encoded:
        out = alloc(planes)
        code = capi.decode_blocks_static(w, h, chroma, meta, words, n, [t.data_ptr() for t in out],
                                         [t.stride(0) for t in out])
        assert code == capi.PYROWAVE_SUCCESS
        got.append(out)
    torch.cuda.synchronize()
    for (enc, w, h, chroma, planes, *_), out, ref in zip(encoded, got, want):
        for i in range(3):
            assert np.array_equal(out[i].cpu().numpy(), ref[i]), f"{w}x{h} plane {i}"
        # A real decode, not an untouched buffer.
        assert not np.all(ref[0] == 0x55)
    for e in encoded:
        e[0].close()
    dev.close()
