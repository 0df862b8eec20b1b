"""Behaviour of the C API on a CUDA device: argument validation, input formats,
the packet parser and partial / empty frames.

Validation rules follow pyrowave_c.cpp:1058-1088 (encode) and :1345-1373
(decode) of the reference; the parser follows pyrowave_decoder.cpp:154-262 and
is checked against the oracle's restatement of it packet by packet.
"""
import ctypes

import numpy as np
import pytest

import oracle as O
from pyrowave_b200 import capi, synth

pytestmark = pytest.mark.gpu


@pytest.fixture(scope="module")
def device(gpu):
    dev = capi.Device()
    yield dev
    dev.close()


def _create_encoder(device, w, h, chroma):
    info = capi.EncoderCreateInfo(device.h, w, h, chroma)
    hdl = ctypes.c_void_p()
    code = capi.lib().pyrowave_encoder_create(ctypes.byref(info), ctypes.byref(hdl))
    if code == capi.PYROWAVE_SUCCESS:
        capi.lib().pyrowave_encoder_destroy(hdl)
    return code


def test_create_validation(device):
    assert _create_encoder(device, 64, 64, capi.CHROMA_420) == capi.PYROWAVE_SUCCESS
    assert _create_encoder(device, 65, 64, capi.CHROMA_420) == capi.PYROWAVE_ERROR_INVALID_ARGUMENT
    assert _create_encoder(device, 64, 63, capi.CHROMA_420) == capi.PYROWAVE_ERROR_INVALID_ARGUMENT
    assert _create_encoder(device, 65, 63, capi.CHROMA_444) == capi.PYROWAVE_SUCCESS
    assert _create_encoder(device, 0, 64, capi.CHROMA_444) == capi.PYROWAVE_ERROR_INVALID_ARGUMENT
    assert _create_encoder(device, 64, 64, 7) == capi.PYROWAVE_ERROR_INVALID_ARGUMENT


def test_encode_validation(device):
    w, h = 96, 64
    enc = capi.Encoder(device, w, h, capi.CHROMA_420)
    planes = synth.synth_frame(w, h, False, 1)
    L = capi.lib()

    def run(mutate, budget=20000, fmt=capi.FORMAT_YUV420P):
        buf, keep = capi.cpu_buffer(planes, w, h, fmt)
        mutate(buf)
        rc = capi.RateControl(budget)
        return L.pyrowave_encoder_encode_cpu_synchronous(enc.h, ctypes.byref(buf), ctypes.byref(rc))

    ok = capi.PYROWAVE_SUCCESS
    bad = capi.PYROWAVE_ERROR_INVALID_ARGUMENT
    assert run(lambda b: None) == ok
    assert run(lambda b: setattr(b, "width", w + 2)) == bad
    assert run(lambda b: setattr(b, "height", h - 2)) == bad
    assert run(lambda b: None, fmt=capi.FORMAT_YUV444P) == bad
    assert run(lambda b: None, fmt=9) == bad
    assert run(lambda b: b.row_stride_in_bytes.__setitem__(1, w // 2 - 1)) == bad
    assert run(lambda b: b.plane_size_in_bytes.__setitem__(2, b.plane_size_in_bytes[2] - 1)) == bad
    assert run(lambda b: b.data.__setitem__(0, None)) == bad
    assert run(lambda b: None, budget=0) == bad
    assert L.pyrowave_encoder_encode_cpu_synchronous(enc.h, None, None) == bad
    # A rejected call leaves the encoder usable.
    assert run(lambda b: None) == ok


def test_decode_validation(device):
    w, h = 96, 64
    dec = capi.Decoder(device, w, h, capi.CHROMA_420)
    code, _ = dec.decode_cpu(fmt=capi.FORMAT_NV12)
    assert code == capi.PYROWAVE_ERROR_INVALID_ARGUMENT
    code, _ = dec.decode_cpu(fmt=capi.FORMAT_YUV444P)
    assert code == capi.PYROWAVE_ERROR_INVALID_ARGUMENT
    short = [np.zeros((h, w), np.uint8), np.zeros((h // 2, w // 2 - 1), np.uint8), np.zeros((h // 2, w // 2), np.uint8)]
    code, _ = dec.decode_cpu(planes=short)
    assert code == capi.PYROWAVE_ERROR_INVALID_ARGUMENT
    code, _ = dec.decode_cpu()
    assert code == capi.PYROWAVE_SUCCESS


def test_nv12_equals_planar(device):
    w, h, budget = 320, 180, 25000
    y, cb, cr = synth.synth_frame(w, h, False, 3)
    cbcr = np.stack([cb, cr], axis=-1).reshape(h // 2, w)
    a = capi.Encoder(device, w, h, capi.CHROMA_420)
    b = capi.Encoder(device, w, h, capi.CHROMA_420)
    assert a.encode_cpu([y, cb, cr], budget) == capi.PYROWAVE_SUCCESS
    assert b.encode_cpu([y, cbcr, None], budget, fmt=capi.FORMAT_NV12) == capi.PYROWAVE_SUCCESS
    sa, pa = a.packetize(4096, budget)
    sb, pb = b.packetize(4096, budget)
    assert pa == pb
    n = sum(p[1] for p in pa)
    assert np.array_equal(sa[:n], sb[:n])


def test_empty_decoder_is_mid_grey(device):
    # pyrowave_c_test.cpp:105-162: nothing pushed, decoding gives 0x7f / 0x80.
    dec = capi.Decoder(device, 16, 16, capi.CHROMA_420)
    assert not dec.is_ready()
    code, out = dec.decode_cpu()
    assert code == capi.PYROWAVE_SUCCESS
    for p in out:
        assert np.isin(p, [0x7F, 0x80]).all()


def _encode(device, w, h, c444, seed, budget, boundary, encoder=None):
    enc = encoder or capi.Encoder(device, w, h, capi.CHROMA_444 if c444 else capi.CHROMA_420)
    planes = synth.synth_frame(w, h, c444, seed)
    assert enc.encode_cpu(planes, budget) == capi.PYROWAVE_SUCCESS
    stream, packets = enc.packetize(boundary, budget)
    return enc, planes, [stream[o:o + s].copy() for o, s in packets]


def _oracle_decode(o, parser):
    offs, payload = parser.get()
    return o.idwt(o.dequant(offs, payload, O.MODE_F32), O.MODE_F32)


def test_partial_frame(device):
    w, h = 256, 192
    _, planes, pkts = _encode(device, w, h, False, 9, 60000, 2048)
    assert len(pkts) > 4
    dec = capi.Decoder(device, w, h, capi.CHROMA_420)
    o = O.Oracle(w, h, False)
    p = o.parser()
    keep = pkts[: (3 * len(pkts)) // 4]
    for pk in keep:
        assert dec.push_packet(pk) == capi.PYROWAVE_SUCCESS
        assert p.push(pk.tobytes())
        assert dec.is_ready(False) == p.ready(False)
        assert dec.is_ready(True) == p.ready(True)
    code, out = dec.decode_cpu()
    assert code == capi.PYROWAVE_SUCCESS
    want = _oracle_decode(o, p)
    for i in range(3):
        assert np.array_equal(out[i], want[i])
    # Decoding marks the frame as consumed.
    assert not dec.is_ready(True)


def test_out_of_order_and_duplicate_packets(device):
    w, h = 200, 130
    _, planes, pkts = _encode(device, w, h, False, 12, 40000, 1500)
    rng = np.random.default_rng(5)
    order = rng.permutation(len(pkts)).tolist() + [0, len(pkts) - 1]
    dec = capi.Decoder(device, w, h, capi.CHROMA_420)
    ref = capi.Decoder(device, w, h, capi.CHROMA_420)
    for i in order:
        assert dec.push_packet(pkts[i]) == capi.PYROWAVE_SUCCESS
    for pk in pkts:
        assert ref.push_packet(pk) == capi.PYROWAVE_SUCCESS
    assert dec.is_ready() and ref.is_ready()
    a = dec.decode_cpu()[1]
    b = ref.decode_cpu()[1]
    for i in range(3):
        assert np.array_equal(a[i], b[i])


def test_sequence_handling(device):
    """A newer sequence restarts the frame; packets of an older one are dropped."""
    w, h = 128, 128
    enc = capi.Encoder(device, w, h, capi.CHROMA_420)
    frames = [_encode(device, w, h, False, 20 + k, 20000, 1024, encoder=enc)[2] for k in range(3)]
    dec = capi.Decoder(device, w, h, capi.CHROMA_420)
    o = O.Oracle(w, h, False)
    p = o.parser()
    # half of frame 1, all of frame 3 (sequence 3), then stale frame 2 packets (sequence 2)
    stream = frames[0][: len(frames[0]) // 2] + frames[2] + frames[1]
    for pk in stream:
        assert (dec.push_packet(pk) == capi.PYROWAVE_SUCCESS) == p.push(pk.tobytes())
        assert dec.is_ready() == p.ready()
    code, out = dec.decode_cpu()
    assert code == capi.PYROWAVE_SUCCESS
    want = _oracle_decode(o, p)
    for i in range(3):
        assert np.array_equal(out[i], want[i])


def _mutations(pkts, rng):
    """Damaged packets: truncated, bit-flipped headers, random bytes, bad block indices."""
    out = []
    for pk in pkts:
        out.append(pk)
        if len(pk) > 12:
            cut = int(rng.integers(1, len(pk) - 1))
            out.append(pk[:cut])
        flip = pk.copy()
        k = int(rng.integers(0, min(len(flip), 8)))
        flip[k] ^= np.uint8(1 << int(rng.integers(0, 8)))
        out.append(flip)
        if len(pk) >= 8:
            idx = pk.copy()
            idx[5:8] = 0xFF  # block index far out of range
            out.append(idx)
    out.append(rng.integers(0, 256, 64, dtype=np.uint8))
    out.append(np.zeros(0, np.uint8))
    out.append(np.zeros(4, np.uint8))
    return out


@pytest.mark.parametrize("seed", [0, 1, 2])
def test_parser_fuzz_matches_oracle_parser(device, seed):
    w, h = 160, 96
    _, planes, pkts = _encode(device, w, h, False, 30 + seed, 30000, 700)
    rng = np.random.default_rng(seed)
    dec = capi.Decoder(device, w, h, capi.CHROMA_420)
    o = O.Oracle(w, h, False)
    p = o.parser()
    for pk in _mutations(pkts, rng):
        got = dec.push_packet(pk) == capi.PYROWAVE_SUCCESS
        want = p.push(pk.tobytes())
        assert got == want
        assert dec.is_ready(True) == p.ready(True)
    # Whatever was accepted decodes like the oracle decodes it (bounds-checked payload reads).
    code, out = dec.decode_cpu()
    assert code == capi.PYROWAVE_SUCCESS
    want = _oracle_decode(o, p)
    for i in range(3):
        assert np.array_equal(out[i], want[i])


def test_stage_timing_report(device):
    w, h = 256, 256
    dev = capi.Device()
    dev.set_stage_timing(True)
    enc = capi.Encoder(dev, w, h, capi.CHROMA_420)
    planes = synth.synth_frame(w, h, False, 2)
    for _ in range(3):
        assert enc.encode_cpu(planes, 20000) == capi.PYROWAVE_SUCCESS
        enc.packetize(1 << 20, 20000)
    lines = dev.report_performance_stats(True)
    assert any("dwt" in s for s in lines), lines
    enc.close()
    dev.close()
