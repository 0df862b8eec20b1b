"""Device-side packet assembly (pyrowave_cuda_decoder_decode_packets) against the
oracle: the oracle parser (a restatement of pyrowave_decoder.cpp:126-262, itself
pinned to the reference's own compiled parser) fed the same packets in the same
order, then the oracle's dequantiser and inverse transform. Decoded planes must
be bit-identical, and the readiness and rejected-packet counts must agree. The
library's host parser (pyrowave_decoder_clear + pyrowave_decoder_push_packet per
packet + pyrowave_cuda_decoder_decode) is held to the same answers."""
import numpy as np
import pytest

import oracle as O
from oracle_codec import oracle_decode
from pyrowave_b200 import capi, synth

pytestmark = pytest.mark.gpu


@pytest.fixture(scope="module")
def device(gpu):
    dev = capi.Device()
    yield dev
    dev.close()


def _frame_packets(enc, planes, budget, boundary):
    assert enc.encode_cpu(planes, budget) == capi.PYROWAVE_SUCCESS
    stream, packets = enc.packetize(boundary, budget)
    return [bytes(stream[off:off + sz]) for off, sz in packets]


def _host_decode(dec, packets, shapes):
    import torch

    dec.clear()
    invalid = sum(dec.push_packet(np.frombuffer(p, np.uint8)) != capi.PYROWAVE_SUCCESS for p in packets)
    ready, partial = dec.is_ready(False), dec.is_ready(True)  # before the decode marks the frame decoded
    out = [torch.full(s, 0x33, dtype=torch.uint8, device="cuda") for s in shapes]
    dec.decode_device([t.data_ptr() for t in out], [t.stride(0) for t in out])
    torch.cuda.synchronize()
    return [t.cpu().numpy() for t in out], invalid, ready, partial


def _device_decode(dec, packets, shapes, misalign=()):
    import torch

    # Packets placed at 4-byte aligned offsets, in a shuffled layout (the
    # descriptors, not the layout, give the push order).
    order = list(range(len(packets)))[::-1]
    offsets = [0] * len(packets)
    pos = 0
    for i in order:
        pos += 4 if i in misalign else 0
        offsets[i] = pos + (2 if i in misalign else 0)
        pos = offsets[i] + len(packets[i])
        pos = (pos + 3) & ~3
    buf = np.zeros(pos + 16, np.uint8)
    for i, p in enumerate(packets):
        buf[offsets[i]:offsets[i] + len(p)] = np.frombuffer(p, np.uint8)
    desc = np.array([[offsets[i], len(p)] for i, p in enumerate(packets)], np.uint64).reshape(-1)
    d_buf = torch.from_numpy(buf).cuda()
    d_desc = torch.from_numpy(desc.view(np.int64)).cuda()
    out = [torch.full(s, 0x33, dtype=torch.uint8, device="cuda") for s in shapes]
    code = dec.decode_packets(d_buf.data_ptr(), buf.nbytes, d_desc.data_ptr(), len(packets),
                              [t.data_ptr() for t in out], [t.stride(0) for t in out])
    assert code == capi.PYROWAVE_SUCCESS
    st = dec.packet_status()
    torch.cuda.synchronize()
    return [t.cpu().numpy() for t in out], st


def _cases(pa, pb, rng):
    """Packet lists in push order: name -> list."""
    cases = {
        "in order": pa,
        "shuffled": [pa[i] for i in rng.permutation(len(pa))],
        "duplicates": pa + [pa[i] for i in rng.choice(len(pa), len(pa) // 2)],
        "partial 70%": [pa[i] for i in sorted(rng.choice(len(pa), int(len(pa) * 0.7), replace=False))],
        "partial 30%": [pa[i] for i in sorted(rng.choice(len(pa), max(1, int(len(pa) * 0.3)), replace=False))],
        "newer sequence midway": pa[: len(pa) // 2] + pb + pa[len(pa) // 2:],
        "interleaved": [p for pair in zip(pa, pb) for p in pair],
        "older after newer": pb + pa,
        "first packet only": pa[:1],
    }
    # Malformed packets: truncated in the middle of a block, a block index past
    # the frame, a mismatched sequence header.
    big = max(range(len(pa)), key=lambda i: len(pa[i]))
    trunc = pa[big][: len(pa[big]) - 6]
    bad_index = bytearray(pa[big])
    first_block = 8 if (bad_index[3] & 0x80) else 0
    bad_index[first_block + 5:first_block + 8] = b"\xff\xff\xff"
    bad_header = bytearray(pa[0])
    bad_header[0] ^= 0x01  # width - 1
    cases["malformed"] = [bytes(bad_header)] + pa[1:big] + [trunc, bytes(bad_index)] + pa[big + 1:]
    return cases


@pytest.mark.parametrize("w,h,c444,budget,boundary", [(640, 360, False, 40000, 2048), (200, 128, True, 30000, 512),
                                                       (1920, 1080, False, 400000, 8192)])
def test_device_assembly_matches_host_parser(device, w, h, c444, budget, boundary):
    chroma = capi.CHROMA_444 if c444 else capi.CHROMA_420
    enc = capi.Encoder(device, w, h, chroma)
    pa = _frame_packets(enc, synth.synth_frame(w, h, c444, 3), budget, boundary)
    pb = _frame_packets(enc, synth.synth_frame(w, h, c444, 4), budget, boundary)
    assert len(pa) > 4
    shapes = [p.shape for p in synth.synth_frame(w, h, c444, 3)]
    host = capi.Decoder(device, w, h, chroma)
    dev_dec = capi.Decoder(device, w, h, chroma)
    o = O.Oracle(w, h, c444)
    rng = np.random.default_rng(5)
    for name, packets in _cases(pa, pb, rng).items():
        # The oracle: parser state, counts and decoded planes.
        op = o.parser()
        o_invalid = sum(not op.push(pkt) for pkt in packets)
        o_ready, o_partial = op.ready(False), op.ready(True)
        o_planes = oracle_decode(o, packets)

        d_planes, st = _device_decode(dev_dec, packets, shapes)
        h_planes, h_invalid, h_ready, h_partial = _host_decode(host, packets, shapes)
        for i in range(3):
            assert np.array_equal(d_planes[i], o_planes[i]), f"{name}: device plane {i} differs from the oracle"
            assert np.array_equal(h_planes[i], o_planes[i]), f"{name}: host-parser plane {i} differs from the oracle"
        assert st.invalid_packets == o_invalid == h_invalid, name
        ready = st.sequence != 0xffffffff and st.decoded_blocks >= st.total_blocks
        partial = st.sequence != 0xffffffff and (ready or st.decoded_blocks > st.total_blocks // 2)
        assert (ready, partial) == (o_ready, o_partial) == (h_ready, h_partial), \
            (name, st.decoded_blocks, st.total_blocks)


def test_device_assembly_misaligned_and_invalid_arguments(device):
    """A packet not at a 4-byte offset is rejected as a whole (the rest of the
    frame still assembles); invalid arguments are refused before any work."""
    import torch

    w, h = 320, 240
    enc = capi.Encoder(device, w, h, capi.CHROMA_420)
    pa = _frame_packets(enc, synth.synth_frame(w, h, False, 9), 20000, 1024)
    shapes = [p.shape for p in synth.synth_frame(w, h, False, 9)]
    dec = capi.Decoder(device, w, h, capi.CHROMA_420)
    _, st = _device_decode(dec, pa, shapes, misalign={len(pa) - 1})
    assert st.invalid_packets == 1
    out = [torch.empty(s, dtype=torch.uint8, device="cuda") for s in shapes]
    ptrs, strides = [t.data_ptr() for t in out], [t.stride(0) for t in out]
    buf = torch.zeros(64, dtype=torch.uint8, device="cuda")
    desc = torch.zeros(2, dtype=torch.int64, device="cuda")
    assert dec.decode_packets(buf.data_ptr(), 64, desc.data_ptr(), 0, ptrs, strides) == \
        capi.PYROWAVE_ERROR_INVALID_ARGUMENT
    assert dec.decode_packets(buf.data_ptr() + 2, 60, desc.data_ptr(), 1, ptrs, strides) == \
        capi.PYROWAVE_ERROR_INVALID_ARGUMENT
