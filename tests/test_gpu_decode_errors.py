"""A decode whose inverse-transform tile load gave up cannot report success.

The inverse transform loads interior tiles with the tensor-memory accelerator
and waits for each load a bounded time; a load that does not complete marks
the decode as failed. The failure is injected on the host
(PYROWAVE_TEST_FAIL_TILE_WAIT=1 when a decoder builds its tile maps): each
completed load is then handled as a timed-out one, so the report path runs
without stalling or faulting the GPU. Every decode entry point must return an
error for such a frame, and a decoder built without the injection must not.
The frame is 1080p: its inverse levels have interior tiles, loaded this way
(the batched form's persistent launch loads every tile without the
accelerator, so its test runs the batch as one launch per stage).
"""
import os

import numpy as np
import pytest

from pyrowave_b200 import capi, synth

pytestmark = pytest.mark.gpu

W, H, BUDGET = 1920, 1080, 400000


@pytest.fixture(scope="module")
def device(gpu):
    dev = capi.Device()
    yield dev
    dev.close()


class _injected:
    """Sets the injection variable for the objects created inside the block."""

    def __enter__(self):
        os.environ["PYROWAVE_TEST_FAIL_TILE_WAIT"] = "1"

    def __exit__(self, *exc):
        os.environ.pop("PYROWAVE_TEST_FAIL_TILE_WAIT", None)


def _encoded(device):
    import torch

    planes = synth.synth_frame(W, H, False, 3)
    enc = capi.Encoder(device, W, H, capi.CHROMA_420)
    assert enc.encode_cpu(planes, BUDGET) == capi.PYROWAVE_SUCCESS
    stream, packets = enc.packetize(1 << 30, BUDGET)
    d = [torch.from_numpy(p).cuda() for p in planes]
    torch.cuda.synchronize()  # the library works on its own stream
    enc.encode_device([p.data_ptr() for p in d], [p.stride(0) for p in d], BUDGET)
    torch.cuda.synchronize()
    return enc, planes, stream, packets


def _decode_all_ways(dec, enc, planes, stream, packets):
    """Result codes of: host-buffer decode, device-block decode + get_error,
    device packet assembly + get_packet_status."""
    import torch

    for off, sz in packets:
        assert dec.push_packet(stream[off:off + sz]) == capi.PYROWAVE_SUCCESS
    sync_code, _ = dec.decode_cpu()

    outs = [torch.zeros(p.shape, dtype=torch.uint8, device="cuda") for p in planes]
    torch.cuda.synchronize()
    s, m, _ = enc.device_bitstream()
    n = enc.size()
    dec.decode_blocks(m, s + 8, n // 4 - 2, [t.data_ptr() for t in outs], [t.stride(0) for t in outs])
    blocks_code, bits = dec.error()

    total = sum(sz for _, sz in packets)
    d_data = torch.from_numpy(np.ascontiguousarray(stream[:total])).cuda()
    d_desc = torch.from_numpy(np.array(packets, np.int64).reshape(-1)).cuda()
    torch.cuda.synchronize()
    assert dec.decode_packets(d_data.data_ptr(), total, d_desc.data_ptr(), len(packets),
                              [t.data_ptr() for t in outs], [t.stride(0) for t in outs]) == capi.PYROWAVE_SUCCESS
    st = capi.PacketStatus()
    packets_code = capi.lib().pyrowave_cuda_decoder_get_packet_status(dec.h, st)
    return sync_code, blocks_code, bits, packets_code


def test_tile_wait_failure_reaches_every_decode_entry_point(device):
    enc, planes, stream, packets = _encoded(device)
    with _injected():
        bad = capi.Decoder(device, W, H, capi.CHROMA_420)
        sync_code, blocks_code, bits, packets_code = _decode_all_ways(bad, enc, planes, stream, packets)
    assert sync_code == capi.PYROWAVE_ERROR_GENERIC
    assert blocks_code == capi.PYROWAVE_ERROR_GENERIC and bits == 1
    assert packets_code == capi.PYROWAVE_ERROR_GENERIC
    bad.close()

    good = capi.Decoder(device, W, H, capi.CHROMA_420)
    sync_code, blocks_code, bits, packets_code = _decode_all_ways(good, enc, planes, stream, packets)
    assert (sync_code, blocks_code, bits, packets_code) == (capi.PYROWAVE_SUCCESS, capi.PYROWAVE_SUCCESS, 0,
                                                            capi.PYROWAVE_SUCCESS)
    good.close()
    enc.close()


def test_tile_wait_failure_fails_the_batch(device):
    import torch

    planes = synth.synth_frame(W, H, False, 4)
    d = [torch.from_numpy(p).cuda() for p in planes]
    outs = [torch.zeros_like(p) for p in d]
    args = ([[p.data_ptr() for p in d]], [[p.stride(0) for p in d]], [BUDGET], [[t.data_ptr() for t in outs]],
            [[t.stride(0) for t in outs]])
    torch.cuda.synchronize()
    with _injected():
        bad = capi.Batch(device, [(W, H, capi.CHROMA_420, BUDGET)])
    # One launch per stage: its 256-thread inverse levels load tiles with the accelerator.
    bad.set_shape(persistent=False, small_level=bad.shape()["small_level"], large_below=256)
    assert bad.encode(*args) == capi.PYROWAVE_SUCCESS
    with pytest.raises(capi.PyrowaveError):
        bad.sizes()
    # Encode without decode does not run the inverse transform.
    assert bad.encode(*args[:3]) == capi.PYROWAVE_SUCCESS
    assert bad.sizes()[0] <= BUDGET
    bad.close()
    good = capi.Batch(device, [(W, H, capi.CHROMA_420, BUDGET)])
    good.set_shape(persistent=False, small_level=good.shape()["small_level"], large_below=256)
    assert good.encode(*args) == capi.PYROWAVE_SUCCESS
    assert good.sizes()[0] <= BUDGET
    good.close()
