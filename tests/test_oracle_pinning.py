"""Pins the CPU oracle before it is trusted as the checker.

1. Against the reference's own code: the Granite-free bitstream library
   (metal/pyrowave_bitstream.cpp) built into oracle/_ref, when present, and the
   golden fixtures generated from it (tests/golden/, always present).
2. Against the known-answer tests of the reference's test suite
   (pyrowave_c_test.cpp): near-lossless 34x30 round trip, 4K stability run
   (budget fill, PSNR bounds, readiness exactly at the last packet), empty
   decoder output.
3. Internal invariants: IEEE half conversion, the exact bucket index, the
   budget never exceeded.
"""
import hashlib
import json
import math
import os
from fractions import Fraction

import numpy as np
import pytest

import oracle as O
from pyrowave_b200 import synth

GOLDEN = os.path.join(os.path.dirname(__file__), "golden")


def sha(a):
    return hashlib.sha256(np.ascontiguousarray(a).tobytes()).hexdigest()


@pytest.fixture(scope="module")
def golden():
    with open(os.path.join(GOLDEN, "reference_bitstream.json")) as f:
        g = json.load(f)
    arrays = dict(np.load(os.path.join(GOLDEN, "reference_bitstream.npz")))
    return g, arrays


# --- golden fixtures from the reference's own bitstream code -------------------
def test_layout_matches_reference_golden(golden):
    g, _ = golden
    for lay in g["layouts"]:
        o = O.Oracle(lay["width"], lay["height"], bool(lay["chroma444"]))
        assert (o.blocks8, o.blocks32) == (lay["blocks8"], lay["blocks32"])
        assert (o.aligned_width, o.aligned_height) == (lay["aligned_width"], lay["aligned_height"])
        assert o.block_info().reshape(-1).tolist() == lay["block_info"]
        assert sha(o.block_mapping()) == lay["mapping_sha256"]


def test_packetize_matches_reference_golden(golden):
    g, arrays = golden
    meta = arrays["pk_meta"]
    words = arrays["ps_stream"][8:].view(np.uint32)
    o = O.Oracle(1280, 720, False)
    o.set_encoded(meta, words, 5)
    for case in g["packetize"]:
        assert o.compute_num_packets(case["boundary"]) == case["num_packets"]
        stream, packets = o.packetize(case["boundary"], case["size"])
        assert packets.tolist() == case["packets"], case
        assert sha(stream) == case["stream_sha256"], case


def _reseq(data: bytes, seq: int) -> bytes:
    a = np.frombuffer(data, np.uint8).copy()
    w0 = a[:4].view(np.uint32)
    w0[0] = (w0[0] & ~np.uint32(7 << 28)) | np.uint32(seq << 28)
    return a.tobytes()


def test_parser_matches_reference_golden(golden):
    g, arrays = golden
    stream, packets = arrays["ps_stream"], arrays["ps_packets"]
    full = [stream[o:o + s].tobytes() for o, s in packets]
    third = full[2][: 4 * ((full[2][2] | (full[2][3] << 8)) & 0xFFF)]
    bad = bytearray(full[0])
    blk = np.frombuffer(bytes(bad[8:16]), np.uint32).copy()
    blk[1] = (blk[1] & 0xFF) | (0xFFFFFF << 8)
    bad[8:16] = blk.tobytes()
    dims = bytearray(full[0])
    w0 = np.frombuffer(bytes(dims[:4]), np.uint32).copy()
    w0[0] = (w0[0] & ~np.uint32(0x3FFF)) | np.uint32(99)
    dims[:4] = w0.tobytes()
    scenarios = {
        "in_order": full,
        "reversed": full[::-1],
        "duplicates": full[:3] + full[:3] + full[3:],
        "drop_half": full[::2],
        "truncated": [full[0], full[1][:-4]],
        "older_sequence": full[:2] + [_reseq(third, 4)],
        "newer_sequence": full[:2] + [_reseq(third, 6)],
        "block_index_out_of_range": [bytes(bad)],
        "dimension_mismatch": [bytes(dims)],
        "trailing_bytes": [full[0] + b"\x01\x02\x03"],
    }
    o = O.Oracle(1280, 720, False)
    for case in g["parser"]:
        p = o.parser()
        log = []
        for data in scenarios[case["name"]]:
            ok = p.push(data)
            log.append([int(ok), int(p.ready(False)), int(p.ready(True)), p.decoded_blocks(), p.total_blocks()])
        offs, payload = p.get()
        assert log == case["log"], case["name"]
        assert sha(offs) == case["offsets_sha256"], case["name"]
        assert sha(payload) == case["payload_sha256"], case["name"]


def test_quant_code_helpers_match_reference_golden(golden):
    g, _ = golden
    qr = O.Oracle(64, 64)
    # decode_quant is exercised through the tables: resolutions are 1 / decode(encode(1 / r)).
    tables, _ = qr.quant_tables()
    for b in range(0, 13):
        code = g["quant_code"]["encode"][str(2.0 ** -b)]
        assert code == ((b + 4) << 3)
        assert g["quant_code"]["decode"][code] == 2.0 ** -b
    assert set(np.unique(tables[tables > 0])).issubset({2.0 ** k for k in range(7, 13)})


@pytest.mark.skipif(not O.ref_available(), reason="reference tree not built into oracle/_ref")
def test_oracle_encode_packetize_parse_against_reference_code():
    w, h = 1280, 720
    planes = synth.synth_frame(w, h, False, 0)
    o = O.Oracle(w, h, False)
    r = O.RefBitstream(w, h, False)
    o.encode(planes, 150000)
    meta, words = o.meta(), o.bitstream_words()
    for boundary in (64, 1400, 8192, 1 << 20):
        a, pa = o.packetize(boundary, 200000)
        b, pb = r.packetize(meta, words, boundary, 200000)
        assert np.array_equal(pa, pb) and np.array_equal(a, b)
        p = o.parser()
        r.parser_reset()
        for off, sz in pa:
            x = a[off:off + sz].tobytes()
            assert p.push(x) == r.push(x)
            assert p.ready() == r.ready()
        oo, op = p.get()
        ro, rp = r.parser_get()
        assert np.array_equal(oo, ro) and np.array_equal(op, rp)


# --- known-answer tests of pyrowave_c_test.cpp -----------------------------------
def _roundtrip(w, h, c444, planes, budget, boundary, mode=O.MODE_F32):
    o = O.Oracle(w, h, c444)
    o.encode(planes, budget, mode)
    stream, packets = o.packetize(boundary, budget + 64)
    p = o.parser()
    ready = []
    for off, sz in packets:
        assert p.push(stream[off:off + sz].tobytes())
        ready.append(p.ready(False))
    offs, payload = p.get()
    out = o.idwt(o.dequant(offs, payload, mode), mode)
    return packets, ready, out


@pytest.mark.parametrize("c444", [False, True])
@pytest.mark.parametrize("mode", [O.MODE_F32, O.MODE_REF16])
def test_known_answer_near_lossless_34x30(c444, mode):
    # pyrowave_c_test.cpp:220-383: 64 KiB budget, one packet, every sample within 1.
    planes = synth.gradient_frame(34, 30, c444)
    packets, ready, out = _roundtrip(34, 30, c444, planes, 64 * 1024, 64 * 1024, mode)
    assert len(packets) == 1 and packets[0][0] == 0
    assert ready == [True]
    for a, b in zip(planes, out):
        assert int(np.abs(a.astype(int) - b.astype(int)).max()) <= 1


def test_known_answer_4k_stability():
    # pyrowave_c_test.cpp:385-548: 4K 4:2:0 mirror gradient at 500000 bytes,
    # 8 KiB packets: 95%..100% fill, ready exactly at the last packet, 40 < PSNR < 60 dB.
    w, h = 3840, 2160
    planes = synth.mirror_gradient_frame(w, h)
    packets, ready, out = _roundtrip(w, h, False, planes, 500000, 8192)
    total = sum(int(s) for _, s in packets)
    assert len(packets) > 1
    assert 95 * 500000 // 100 <= total <= 500000
    assert ready[-1] and not any(ready[:-1])
    for a, b in zip(planes, out):
        assert 40.0 < O.psnr(a, b) < 60.0


def test_known_answer_empty_decoder_is_mid_grey():
    # pyrowave_c_test.cpp:105-162: nothing pushed, decode gives 0x7f/0x80.
    o = O.Oracle(16, 16, False)
    offsets = np.full(o.blocks32, 0xFFFFFFFF, np.uint32)
    out = o.idwt(o.dequant(offsets, np.zeros(0, np.uint32)))
    for p in out:
        assert np.isin(p, [0x7F, 0x80]).all()


# --- invariants ----------------------------------------------------------------
def test_float_to_half_is_ieee_rne():
    rng = np.random.default_rng(1)
    vals = np.concatenate([rng.standard_normal(20000).astype(np.float32) * s for s in (1e-7, 1e-3, 1.0, 1e3, 7e4)])
    vals = np.concatenate([vals, np.array([0.0, -0.0, 65504.0, 65519.99, 65520.0, 2.0 ** -24, 2.0 ** -25,
                                           3 * 2.0 ** -26, 6.1e-5], np.float32)])
    with np.errstate(over="ignore"):  # values from 65520 up round to infinity, as intended
        ref = vals.astype(np.float16).view(np.uint16)
    got = np.array([O.float_to_half(float(v)) for v in vals], np.uint16)
    assert np.array_equal(got, ref)


def test_bucket_index_is_exact():
    # uint(max(60 + 2*log2(r) + 0.5, 0)) evaluated with exact rational thresholds.
    rng = np.random.default_rng(2)
    for _ in range(3000):
        d0 = float(np.float32(rng.uniform(0, 1000)))
        d = float(np.float32(d0 + rng.exponential(50.0)))
        c0 = float(rng.integers(1, 500))
        c = float(rng.integers(0, int(c0)))
        got = O.bucket_index(d, c, d0, c0)
        num = max(float(np.float32(d) - np.float32(d0)), 0.0)
        r = float(np.float32(np.float32(num) / np.float32(c0 - c)))
        if r <= 0:
            assert got == 0
            continue
        # floor(60.5 + 2*log2(r)) is the largest k with r^4 >= 2^(2k - 121), in exact arithmetic.
        r4 = Fraction(r) ** 4
        k = math.floor(60.5 + 2 * math.log2(r))
        while r4 < Fraction(2) ** (2 * k - 121):
            k -= 1
        while r4 >= Fraction(2) ** (2 * (k + 1) - 121):
            k += 1
        expect = max(k, 0)
        assert got == expect, (d, c, d0, c0, r)


@pytest.mark.parametrize("budget", [1200, 4000, 20000, 60000, 150000])
def test_rate_control_never_exceeds_budget(budget):
    w, h = 320, 240
    planes = synth.synth_frame(w, h, False, 5)
    o = O.Oracle(w, h, False)
    o.encode(planes, budget)
    words = o.meta()[:, 1].astype(np.int64).sum()
    assert 8 + 4 * words <= (budget & ~3)
