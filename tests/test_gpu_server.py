"""The serving loop: each stream's results are the same alone and in a mix of
concurrent streams (bit-exact), streams are admitted by memory, and latency
statistics are reported."""
import time

import numpy as np
import pytest

from pyrowave_b200 import capi, synth

pytestmark = pytest.mark.gpu

# (width, height, 4:4:4, budget)
STREAMS = [(640, 360, False, 40000), (1280, 720, True, 150000), (320, 240, False, 12000)]
FRAMES_PER_STREAM = 4


@pytest.fixture(scope="module")
def device(gpu):
    dev = capi.Device()
    yield dev
    dev.close()


def _frames(si):
    import torch

    w, h, c444, _ = STREAMS[si]
    return [[torch.from_numpy(p).cuda() for p in synth.synth_frame(w, h, c444, 100 * si + k)]
            for k in range(FRAMES_PER_STREAM)]


def _serve(device, which, interleave):
    """Run the frames of the streams in `which` through one server; returns
    {stream index: [(bytes, decoded planes) per frame]}."""
    import torch

    server = capi.Server(device, memory_pool_bytes=4 << 30, max_in_flight=4)
    ids, frames, outs = {}, {}, {}
    for si in which:
        w, h, c444, budget = STREAMS[si]
        code, sid = server.open_stream(w, h, capi.CHROMA_444 if c444 else capi.CHROMA_420, budget)
        assert code == capi.PYROWAVE_SUCCESS
        ids[si] = sid
        frames[si] = _frames(si)
        outs[si] = [[torch.full_like(p, 0x55) for p in f] for f in frames[si]]
    order = [(si, k) for k in range(FRAMES_PER_STREAM) for si in which] if interleave else \
        [(si, k) for si in which for k in range(FRAMES_PER_STREAM)]
    req = {}
    for si, k in order:
        f, o = frames[si][k], outs[si][k]
        rid = server.submit(ids[si], [p.data_ptr() for p in f], [p.stride(0) for p in f], STREAMS[si][3],
                            [p.data_ptr() for p in o], [p.stride(0) for p in o])
        req[rid] = (si, k)
    done = {}
    deadline = time.time() + 60
    while len(done) < len(order) and time.time() < deadline:
        for rid, sid, result, nbytes, lat in server.poll(timeout_us=100000):
            assert result == capi.PYROWAVE_SUCCESS
            assert lat > 0
            done[rid] = nbytes
    assert len(done) == len(order)
    torch.cuda.synchronize()
    result = {si: [None] * FRAMES_PER_STREAM for si in which}
    for rid, (si, k) in req.items():
        result[si][k] = (done[rid], [p.cpu().numpy() for p in outs[si][k]])
    p50, p99, n = server.stats()
    assert n == len(order) and 0 < p50 <= p99
    server.close()
    return result


def test_same_alone_and_in_mix(device):
    mixed = _serve(device, [0, 1, 2], interleave=True)
    for si in range(len(STREAMS)):
        alone = _serve(device, [si], interleave=False)
        for k in range(FRAMES_PER_STREAM):
            a_bytes, a_planes = alone[si][k]
            m_bytes, m_planes = mixed[si][k]
            assert a_bytes == m_bytes and a_bytes <= STREAMS[si][3]
            for p in range(3):
                assert np.array_equal(a_planes[p], m_planes[p]), f"stream {si} frame {k} plane {p}"
                assert not np.all(a_planes[p] == 0x55)


def test_admission_by_memory(device):
    # A pool that holds one 1280x720 stream (about 16.5 MB of state) but not two.
    server = capi.Server(device, memory_pool_bytes=24 << 20, max_in_flight=2)
    code, a = server.open_stream(1280, 720, capi.CHROMA_420, 150000)
    assert code == capi.PYROWAVE_SUCCESS
    code, _ = server.open_stream(1280, 720, capi.CHROMA_420, 150000)
    assert code == capi.PYROWAVE_ERROR_OUT_OF_DEVICE_MEMORY
    assert server.close_stream(a) == capi.PYROWAVE_SUCCESS
    deadline = time.time() + 10
    while time.time() < deadline:
        code, b = server.open_stream(1280, 720, capi.CHROMA_420, 150000)
        if code == capi.PYROWAVE_SUCCESS:
            break
        time.sleep(0.01)
    assert code == capi.PYROWAVE_SUCCESS
    assert server.close_stream(12345) == capi.PYROWAVE_ERROR_INVALID_ARGUMENT
    server.close()
