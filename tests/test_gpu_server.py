"""The serving loop: each stream's results equal the oracle's coding of the
same frames, alone and in a mix of concurrent streams (bit-exact), streams are
admitted by memory, and latency statistics are reported."""
import concurrent.futures
import time

import numpy as np
import pytest

from oracle_codec import oracle_frame
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


def _host_frames(si):
    w, h, c444, _ = STREAMS[si]
    return [synth.synth_frame(w, h, c444, 100 * si + k) for k in range(FRAMES_PER_STREAM)]


def _frames(si):
    import torch

    return [[torch.from_numpy(p).cuda() for p in f] for f in _host_frames(si)]


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
    torch.cuda.synchronize()  # the server's streams do not order with torch's
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


def _oracle_streams():
    """{stream: [(bytes, decoded planes) per frame]} of the oracle: frame k of a
    stream is its encoder's (k + 1)-th frame."""
    jobs = [(si, k) for si in range(len(STREAMS)) for k in range(FRAMES_PER_STREAM)]
    frames = {si: _host_frames(si) for si in range(len(STREAMS))}

    def one(job):
        si, k = job
        w, h, c444, budget = STREAMS[si]
        data, planes = oracle_frame(w, h, c444, frames[si][k], budget, k + 1)
        return data.size, planes

    with concurrent.futures.ThreadPoolExecutor(8) as ex:
        res = list(ex.map(one, jobs))
    out = {si: [None] * FRAMES_PER_STREAM for si in range(len(STREAMS))}
    for (si, k), r in zip(jobs, res):
        out[si][k] = r
    return out


def test_same_alone_and_in_mix(device):
    want = _oracle_streams()
    mixed = _serve(device, [0, 1, 2], interleave=True)
    for si in range(len(STREAMS)):
        alone = _serve(device, [si], interleave=False)
        for k in range(FRAMES_PER_STREAM):
            o_bytes, o_planes = want[si][k]
            a_bytes, a_planes = alone[si][k]
            m_bytes, m_planes = mixed[si][k]
            assert a_bytes == m_bytes == o_bytes and a_bytes <= STREAMS[si][3]
            for p in range(3):
                assert np.array_equal(a_planes[p], o_planes[p]), f"stream {si} frame {k} plane {p} alone"
                assert np.array_equal(m_planes[p], o_planes[p]), f"stream {si} frame {k} plane {p} in the mix"


def test_admission_by_memory(device):
    """A pool that holds one 1280x720 working set (about 16.5 MB) but not two:
    both streams open, their frames are admitted one working set at a time
    (the idle stream's set is released for the other's frame), and every frame
    still equals the oracle's coding of it, its sequence numbers carried over."""
    import torch

    pool = 24 << 20
    server = capi.Server(device, memory_pool_bytes=pool, max_in_flight=2)
    w, h, budget = 1280, 720, 150000
    code, big = server.open_stream(3840, 2160, capi.CHROMA_444, 2400000)
    assert code == capi.PYROWAVE_ERROR_OUT_OF_DEVICE_MEMORY  # one working set exceeds the pool
    ids = []
    for _ in range(2):
        code, sid = server.open_stream(w, h, capi.CHROMA_420, budget)
        assert code == capi.PYROWAVE_SUCCESS
        ids.append(sid)
    frames = [[synth.synth_frame(w, h, False, 300 + 10 * j + k) for k in range(3)] for j in range(2)]
    dev_frames = [[[torch.from_numpy(p).cuda() for p in f] for f in fr] for fr in frames]
    outs = [[[torch.zeros_like(p) for p in f] for f in fr] for fr in dev_frames]
    torch.cuda.synchronize()
    req = {}
    for k in range(3):
        for j, sid in enumerate(ids):
            f, o = dev_frames[j][k], outs[j][k]
            rid = server.submit(sid, [p.data_ptr() for p in f], [p.stride(0) for p in f], budget,
                                [p.data_ptr() for p in o], [p.stride(0) for p in o])
            req[rid] = (j, k)
    done = {}
    deadline = time.time() + 60
    while len(done) < len(req) and time.time() < deadline:
        for rid, sid, result, nbytes, lat in server.poll(timeout_us=100000):
            assert result == capi.PYROWAVE_SUCCESS
            done[rid] = nbytes
    assert len(done) == len(req)
    used, peak, releases = server.memory()
    assert 0 < peak <= pool and releases >= 1
    torch.cuda.synchronize()
    for rid, (j, k) in req.items():
        data, planes = oracle_frame(w, h, False, frames[j][k], budget, k + 1)
        assert done[rid] == data.size, (j, k)
        for p in range(3):
            assert np.array_equal(outs[j][k][p].cpu().numpy(), planes[p]), (j, k, p)
    assert server.close_stream(ids[0]) == capi.PYROWAVE_SUCCESS
    assert server.close_stream(12345) == capi.PYROWAVE_ERROR_INVALID_ARGUMENT
    server.close()
