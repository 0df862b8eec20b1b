"""Parity of the sm_100a encode/decode path with the CPU oracle.

Every stage of the path is compared bit for bit with the oracle's restatement
of the reference algorithm on the same seeded frames:

  DWT coefficients          shaders/dwt.comp + dwt_common.h (forward lifting)
  8x8 code words, RD table  shaders/wavelet_quant.comp (quantiser + per-32x32 RD data)
  histogram, quant drops    shaders/analyze_rate_control.comp, resolve_rate_control.comp
  block metadata, bytes     shaders/block_packing.comp + pyrowave_encoder.cpp:1085-1109
  decoded planes            shaders/wavelet_dequant.comp + shaders/idwt.comp

The cases include every configuration the benchmark reports: 1080p 4:2:0 at
400000 bytes with FP32 storage (seeds from both ends of its 16-frame set),
4K 4:2:0 at 1200000 bytes with FP32 and FP16 level 0-1 storage, and 4K 4:4:4
with the dense generator (200 rectangles, 1-pixel lines) at 600000 and
2400000 bytes. Each benchmark frame is pinned by its fingerprint, so these are
the frames the benchmark codes.

All calls go through the C-ABI library (libpyrowave-shared.so.0).
"""
import numpy as np
import pytest

import oracle as O
from pyrowave_b200 import capi, synth

pytestmark = pytest.mark.gpu

# (width, height, 4:4:4, budget bytes, seed, FP16 level mask, rectangles, lines, frame fingerprint or None)
CASES = [
    (1280, 720, False, 150000, 0, 0, 40, 0, "ca29b7e9c4fab120"),
    (34, 30, False, 65536, 0, 0, 40, 0, None),
    (34, 30, True, 65536, 0, 0, 40, 0, None),
    (130, 98, False, 20000, 5, 0, 40, 0, None),
    (200, 128, True, 30000, 6, 0, 40, 0, None),
    (1000, 562, False, 60000, 7, 0x1F, 40, 0, None),
    (1920, 1080, False, 400000, 1, 3, 40, 0, "3ff3f07e40a6491f"),
    # 1080p benchmark workload, FP32 storage (the headline configuration).
    (1920, 1080, False, 400000, 1, 0, 40, 0, "3ff3f07e40a6491f"),
    (1920, 1080, False, 400000, 8, 0, 40, 0, "0b14888ed34de5d9"),
    (1920, 1080, False, 400000, 16, 0, 40, 0, "5a629d5f15facfa2"),
    # 4K 4:2:0 benchmark workload, FP32 and FP16 (levels 0-1) storage.
    (3840, 2160, False, 1200000, 1, 0, 40, 0, "141d31e7daf8c1a9"),
    (3840, 2160, False, 1200000, 2, 3, 40, 0, "1f9bb18edb08fb69"),
    # 4K 4:4:4 benchmark generator, budget sweep ends and middle.
    (3840, 2160, True, 600000, 1, 0, 200, 40, "56a528decd878230"),
    (3840, 2160, True, 1200000, 3, 0, 200, 40, "f2411da1edc69dc3"),
    (3840, 2160, True, 2400000, 2, 0, 200, 40, "6f0c2e3064ec0195"),
]


def _ids(c):
    return f"{c[0]}x{c[1]}-{'444' if c[2] else '420'}-{c[3]}B-seed{c[4]}-fp16mask{c[5]}" + ("-dense" if c[6] > 40 else "")


@pytest.fixture(scope="module")
def device(gpu):
    dev = capi.Device()
    yield dev
    dev.close()


def _to_dev(planes):
    """Device copies, complete before the library (which works on its own stream) reads them."""
    import torch

    out = [torch.from_numpy(np.ascontiguousarray(p)).cuda() for p in planes]
    torch.cuda.synchronize()
    return out


def _mismatch(name, got, want):
    got = np.asarray(got)
    want = np.asarray(want)
    if got.shape != want.shape:
        return f"{name}: shape {got.shape} != {want.shape}"
    bad = np.argwhere(got != want)
    if len(bad):
        return f"{name}: {len(bad)} elements differ, first at {bad[:3].tolist()}"
    return None


@pytest.mark.parametrize("case", CASES, ids=[_ids(c) for c in CASES])
def test_encode_decode_bit_exact(device, case):
    import torch

    w, h, c444, budget, seed, fp16, rects, lines, fingerprint = case
    chroma = capi.CHROMA_444 if c444 else capi.CHROMA_420
    planes = synth.synth_frame(w, h, c444, seed, rects, lines)
    if fingerprint:
        assert synth.frame_hash(planes) == fingerprint, "not the benchmark's frame"
    enc = capi.Encoder(device, w, h, chroma, fp16)
    lay = enc.layout()
    o = O.Oracle(w, h, c444, fp16)
    assert lay.block_count_32x32 == o.blocks32
    assert lay.pyramid_size == o.pyramid_size
    errors = []

    # A different frame and budget first, so the second encode runs through the
    # per-call updates of the captured graph rather than its first capture.
    other = _to_dev(synth.synth_frame(w, h, c444, seed + 100, rects, lines))
    enc.encode_device([p.data_ptr() for p in other], [p.stride(0) for p in other], budget // 2)
    dplanes = _to_dev(planes)
    enc.encode_device([p.data_ptr() for p in dplanes], [p.stride(0) for p in dplanes], budget)
    torch.cuda.synchronize()

    pyr = torch.zeros(lay.pyramid_size, dtype=torch.float32, device="cuda")
    enc.read_wavelet(pyr.data_ptr())
    torch.cuda.synchronize()
    gpu_pyr = pyr.cpu().numpy()
    ora_pyr = o.dwt(planes, O.MODE_F32)
    errors.append(_mismatch("dwt bits", gpu_pyr.view(np.uint32), ora_pyr.view(np.uint32)))

    o.encode_pyramid(ora_pyr, budget, sequence=2)
    d = enc.debug()
    assert int(d["error_flags"][0]) == 0, "device consistency check failed"
    errors.append(_mismatch("code words", d["code_words"], o.code_words()))
    rc, dist, bk = o.rd()
    errors.append(_mismatch("rd cost", d["rd_cost"].astype(np.uint32), rc))
    errors.append(_mismatch("rd dist", d["rd_dist"].view(np.uint32), dist.view(np.uint32)))
    errors.append(_mismatch("rd bucket", d["rd_bucket"].astype(np.uint32), bk))
    scan, consumed = o.histogram()
    errors.append(_mismatch("consumed", d["consumed"], [consumed]))
    errors.append(_mismatch("histogram scan", np.cumsum(d["histogram"].astype(np.uint64)).astype(np.uint32), scan))
    errors.append(_mismatch("quant", d["quant"], o.quant()))
    errors.append(_mismatch("block meta", d["block_meta"], o.meta()))

    # Host-buffer API: encode -> packetize, against the oracle's packetizer.
    assert enc.encode_cpu(planes, budget) == capi.PYROWAVE_SUCCESS
    boundary = 8192
    stream, packets = enc.packetize(boundary, budget)
    o.encode_pyramid(ora_pyr, budget, sequence=3)  # third encode of this encoder
    ostream, opackets = o.packetize(boundary, budget)
    total = sum(p[1] for p in packets)
    assert total <= budget
    errors.append(_mismatch("packets", np.array(packets, np.int64).reshape(-1, 2), opackets))
    errors.append(_mismatch("stream bytes", stream[:total], ostream[:total]))

    # Host-buffer decode through the packet parser.
    dec = capi.Decoder(device, w, h, chroma, fp16)
    for off, sz in packets:
        assert dec.push_packet(stream[off:off + sz]) == capi.PYROWAVE_SUCCESS
    assert dec.is_ready()
    code, out = dec.decode_cpu()
    assert code == capi.PYROWAVE_SUCCESS
    p = o.parser()
    for off, sz in packets:
        assert p.push(stream[off:off + sz].tobytes())
    offs, payload = p.get()
    oout = o.idwt(o.dequant(offs, payload, O.MODE_F32), O.MODE_F32)
    for i in range(3):
        errors.append(_mismatch(f"decoded plane {i}", out[i], oout[i]))

    # Device-resident decode straight from the encoder's device bitstream.
    s, m, _ = enc.device_bitstream()
    outs = [torch.zeros(pl.shape, dtype=torch.uint8, device="cuda") for pl in planes]
    dec2 = capi.Decoder(device, w, h, chroma, fp16)
    dec2.decode_blocks(m, s + 8, total // 4 - 2, [t.data_ptr() for t in outs], [t.stride(0) for t in outs])
    assert dec2.error() == (capi.PYROWAVE_SUCCESS, 0)
    torch.cuda.synchronize()
    for i in range(3):
        errors.append(_mismatch(f"device decode plane {i}", outs[i].cpu().numpy(), oout[i]))

    errors = [e for e in errors if e]
    assert not errors, "\n".join(errors)


@pytest.mark.parametrize("w,h,c444,budget,seed", [(1920, 1080, False, 400000, 1), (1920, 1080, False, 400000, 2),
                                                  (200, 128, True, 30000, 6)])
def test_reference_precision_bit_exact(device, w, h, c444, budget, seed):
    """REFERENCE_PRECISION (FP16 lifting stages, FP16 levels 0-1) against the
    oracle's restatement of the reference's precision 1: pyramid, packets and
    decoded planes bit for bit, hence the same PSNR at the same budget."""
    import torch

    chroma = capi.CHROMA_444 if c444 else capi.CHROMA_420
    planes = synth.synth_frame(w, h, c444, seed)
    mode = capi.REFERENCE_PRECISION
    enc = capi.Encoder(device, w, h, chroma, mode)
    o = O.Oracle(w, h, c444, 3)
    d = _to_dev(planes)
    enc.encode_device([p.data_ptr() for p in d], [p.stride(0) for p in d], budget)
    pyr = torch.zeros(enc.layout().pyramid_size, dtype=torch.float32, device="cuda")
    enc.read_wavelet(pyr.data_ptr())
    torch.cuda.synchronize()
    ref_pyr = o.dwt(planes, O.MODE_REF16)
    errors = [_mismatch("dwt bits", pyr.cpu().numpy().view(np.uint32), ref_pyr.view(np.uint32))]

    assert enc.encode_cpu(planes, budget) == capi.PYROWAVE_SUCCESS
    stream, packets = enc.packetize(8192, budget)
    o.encode_pyramid(ref_pyr, budget, sequence=2)
    ostream, opackets = o.packetize(8192, budget)
    total = sum(p[1] for p in packets)
    assert total <= budget
    errors.append(_mismatch("packets", np.array(packets, np.int64).reshape(-1, 2), opackets))
    errors.append(_mismatch("stream bytes", stream[:total], ostream[:total]))

    dec = capi.Decoder(device, w, h, chroma, mode)
    for off, sz in packets:
        assert dec.push_packet(stream[off:off + sz]) == capi.PYROWAVE_SUCCESS
    code, out = dec.decode_cpu()
    assert code == capi.PYROWAVE_SUCCESS
    p = o.parser()
    for off, sz in packets:
        assert p.push(stream[off:off + sz].tobytes())
    offs, payload = p.get()
    oout = o.idwt(o.dequant(offs, payload, O.MODE_REF16), O.MODE_REF16)
    for i in range(3):
        errors.append(_mismatch(f"decoded plane {i}", out[i], oout[i]))
    errors = [e for e in errors if e]
    assert not errors, "\n".join(errors)


@pytest.mark.parametrize("w,h,c444", [(1280, 720, False), (640, 480, True)])
def test_dwt_accuracy_vs_fp64(device, w, h, c444):
    """The FP32 transform stays within 1e-5 of an FP64 evaluation of the same lifting."""
    import torch

    planes = synth.synth_frame(w, h, c444, 11)
    chroma = capi.CHROMA_444 if c444 else capi.CHROMA_420
    enc = capi.Encoder(device, w, h, chroma)
    d = _to_dev(planes)
    enc.encode_device([p.data_ptr() for p in d], [p.stride(0) for p in d], 100000)
    pyr = torch.zeros(enc.layout().pyramid_size, dtype=torch.float32, device="cuda")
    enc.read_wavelet(pyr.data_ptr())
    torch.cuda.synchronize()
    ref = O.Oracle(w, h, c444).dwt(planes, O.MODE_F64)
    assert float(np.abs(pyr.cpu().numpy().astype(np.float64) - ref).max()) < 1e-5


@pytest.mark.parametrize("budget", [4096, 12000, 40000, 150000, 2000000])
def test_budget_sweep_bit_exact(device, budget):
    """Rate control from starved to unconstrained budgets matches the oracle byte for byte."""
    w, h = 640, 360
    planes = synth.synth_frame(w, h, False, 21)
    enc = capi.Encoder(device, w, h, capi.CHROMA_420)
    assert enc.encode_cpu(planes, budget) == capi.PYROWAVE_SUCCESS
    stream, packets = enc.packetize(1 << 30, budget)
    total = sum(p[1] for p in packets)
    assert total <= budget
    o = O.Oracle(w, h, False)
    o.encode(planes, budget, sequence=1)
    ostream, opackets = o.packetize(1 << 30, budget)
    assert np.array_equal(np.array(packets, np.int64).reshape(-1, 2), opackets)
    assert np.array_equal(stream[:total], ostream[:total])


@pytest.mark.parametrize("quant_scale", [-1.0, 0.5, 2.0])
def test_pre_transformed_input(device, quant_scale):
    """encode_pre_transformed on the oracle's pyramid equals the oracle's encode of it."""
    import torch

    w, h = 512, 288
    planes = synth.synth_frame(w, h, False, 4)
    o = O.Oracle(w, h, False)
    pyr = o.dwt(planes, O.MODE_F32)
    enc = capi.Encoder(device, w, h, capi.CHROMA_420)
    dpyr = torch.from_numpy(pyr).cuda()
    budget = 30000
    enc.encode_pre_transformed(dpyr.data_ptr(), budget, quant_scale)
    stream, packets = enc.packetize(1 << 30, budget)
    total = sum(p[1] for p in packets)
    o.encode_pyramid(pyr, budget, sequence=1, quant_scale=quant_scale)
    ostream, _ = o.packetize(1 << 30, budget)
    assert np.array_equal(stream[:total], ostream[:total])


def test_decode_pyramid_matches_oracle_idwt(device):
    import torch

    w, h = 320, 240
    planes = synth.synth_frame(w, h, True, 8)
    o = O.Oracle(w, h, True)
    pyr = o.dwt(planes, O.MODE_F32)
    dec = capi.Decoder(device, w, h, capi.CHROMA_444)
    outs = [torch.zeros(p.shape, dtype=torch.uint8, device="cuda") for p in planes]
    dpyr = torch.from_numpy(pyr).cuda()
    dec.decode_pyramid(dpyr.data_ptr(), [t.data_ptr() for t in outs], [t.stride(0) for t in outs])
    torch.cuda.synchronize()
    want = o.idwt(pyr, O.MODE_F32)
    for i in range(3):
        assert np.array_equal(outs[i].cpu().numpy(), want[i])
    # Lossless round trip of the transform alone.
    for i in range(3):
        assert int(np.abs(want[i].astype(int) - planes[i].astype(int)).max()) <= 1


def test_4k_stability(device):
    """Repeated encodes of a 4K frame fill 95-100% of the budget and stay decodable."""
    w, h, budget = 3840, 2160, 500000
    planes = synth.mirror_gradient_frame(w, h)
    enc = capi.Encoder(device, w, h, capi.CHROMA_420)
    dec = capi.Decoder(device, w, h, capi.CHROMA_420)
    for it in range(3):
        assert enc.encode_cpu(planes, budget) == capi.PYROWAVE_SUCCESS
        stream, packets = enc.packetize(8192, budget)
        total = sum(p[1] for p in packets)
        assert len(packets) > 1
        assert 95 * budget // 100 <= total <= budget
        ready = []
        for off, sz in packets:
            assert dec.push_packet(stream[off:off + sz]) == capi.PYROWAVE_SUCCESS
            ready.append(dec.is_ready())
        assert ready[-1] and not any(ready[:-1])
        code, out = dec.decode_cpu()
        assert code == capi.PYROWAVE_SUCCESS
        assert 40.0 < O.psnr(planes[0], out[0]) < 60.0


def test_tensor_maps_follow_reused_addresses(device):
    """Encoders and decoders created and destroyed in turn, with different
    frame sizes, so the device addresses of their TMA tensor maps are reused
    for maps of other buffers: every transform still reads its own buffers
    (bit-exact pyramids and decoded planes)."""
    import torch

    shapes = [(1280, 720, False), (640, 480, True), (1920, 1080, False), (1280, 720, False), (960, 544, True)]
    for k, (w, h, c444) in enumerate(shapes * 2):
        chroma = capi.CHROMA_444 if c444 else capi.CHROMA_420
        planes = synth.synth_frame(w, h, c444, 40 + k)
        enc = capi.Encoder(device, w, h, chroma)
        d = _to_dev(planes)
        enc.encode_device([p.data_ptr() for p in d], [p.stride(0) for p in d], 60000)
        pyr = torch.zeros(enc.layout().pyramid_size, dtype=torch.float32, device="cuda")
        enc.read_wavelet(pyr.data_ptr())
        torch.cuda.synchronize()
        o = O.Oracle(w, h, c444)
        ref = o.dwt(planes, O.MODE_F32)
        err = _mismatch(f"dwt bits {w}x{h} #{k}", pyr.cpu().numpy().view(np.uint32), ref.view(np.uint32))
        assert err is None, err
        dec = capi.Decoder(device, w, h, chroma)
        outs = [torch.zeros(pl.shape, dtype=torch.uint8, device="cuda") for pl in planes]
        dec.decode_pyramid(pyr.data_ptr(), [t.data_ptr() for t in outs], [t.stride(0) for t in outs])
        torch.cuda.synchronize()
        want = o.idwt(ref, O.MODE_F32)
        for i in range(3):
            err = _mismatch(f"idwt plane {i} {w}x{h} #{k}", outs[i].cpu().numpy(), want[i])
            assert err is None, err
        enc.close()
        dec.close()


@pytest.mark.parametrize("w,h,c444", [(1920, 1080, False), (640, 360, True)])
def test_transform_only_matches_oracle(device, w, h, c444):
    """pyrowave_cuda_encoder_transform (the forward levels without the quantiser)
    gives the oracle's pyramid bit for bit."""
    import torch

    planes = synth.synth_frame(w, h, c444, 31)
    chroma = capi.CHROMA_444 if c444 else capi.CHROMA_420
    enc = capi.Encoder(device, w, h, chroma)
    d = _to_dev(planes)
    enc.transform([p.data_ptr() for p in d], [p.stride(0) for p in d])
    pyr = torch.zeros(enc.layout().pyramid_size, dtype=torch.float32, device="cuda")
    enc.read_wavelet(pyr.data_ptr())
    torch.cuda.synchronize()
    ref = O.Oracle(w, h, c444).dwt(planes, O.MODE_F32)
    err = _mismatch("transform-only pyramid", pyr.cpu().numpy().view(np.uint32), ref.view(np.uint32))
    assert err is None, err


def _frame16(w, h, c444, seed):
    """A 16-bit frame: the 8-bit synthetic frame widened, with seeded low bits."""
    rng = np.random.default_rng(seed)
    return [(p.astype(np.uint16) << 8) | rng.integers(0, 256, p.shape, dtype=np.uint16)
            for p in synth.synth_frame(w, h, c444, seed)]


@pytest.mark.parametrize("w,h,c444,budget", [(640, 360, False, 60000), (333, 197, True, 40000),
                                              (1920, 1080, False, 400000)])
def test_sixteen_bit_planes_bit_exact(device, w, h, c444, budget):
    """16-bit (R16_UNORM) input and output, the reference's high bit depth path
    (encode.cpp:152, decode.cpp:215): host-buffer and device-plane encodes give
    the oracle's stream, and both decodes give the oracle's 16-bit planes."""
    import torch

    chroma = capi.CHROMA_444 if c444 else capi.CHROMA_420
    planes = _frame16(w, h, c444, 12)
    o = O.Oracle(w, h, c444)
    pyr = o.dwt(planes, O.MODE_F32)
    o.encode_pyramid(pyr, budget, sequence=1)
    ostream, opackets = o.packetize(1 << 30, budget)
    total = int(sum(int(sz) for _, sz in opackets))
    want = o.idwt16(o.dequant(*_parse_all(o, ostream[:total])), O.MODE_F32)

    enc = capi.Encoder(device, w, h, chroma)
    assert enc.encode_cpu(planes, budget) == capi.PYROWAVE_SUCCESS
    stream, packets = enc.packetize(1 << 30, budget)
    assert sum(p[1] for p in packets) == total
    assert np.array_equal(stream[:total], ostream[:total]), "16-bit host encode differs from the oracle"

    dec = capi.Decoder(device, w, h, chroma)
    assert dec.push_packet(stream[:total]) == capi.PYROWAVE_SUCCESS
    code, out = dec.decode_cpu(wide=True)
    assert code == capi.PYROWAVE_SUCCESS
    for i in range(3):
        assert out[i].dtype == np.uint16
        err = _mismatch(f"16-bit decoded plane {i}", out[i], want[i])
        assert err is None, err

    # Device planes: encode16 (second frame of the encoder, sequence 2) and decode_blocks16.
    d = [torch.from_numpy(p.view(np.int16)).cuda() for p in planes]
    enc.encode_device16([p.data_ptr() for p in d], [p.stride(0) * 2 for p in d], budget)
    torch.cuda.synchronize()
    s, m, _ = enc.device_bitstream()
    n = enc.size()
    assert n == total
    outs = [torch.zeros(p.shape, dtype=torch.int16, device="cuda") for p in planes]
    dec2 = capi.Decoder(device, w, h, chroma)
    dec2.decode_blocks16(m, s + 8, n // 4 - 2, [t.data_ptr() for t in outs], [t.stride(0) * 2 for t in outs])
    assert dec2.error() == (capi.PYROWAVE_SUCCESS, 0)
    torch.cuda.synchronize()
    for i in range(3):
        err = _mismatch(f"16-bit device plane {i}", outs[i].cpu().numpy().view(np.uint16), want[i])
        assert err is None, err


def _parse_all(o, data):
    p = o.parser()
    assert p.push(data.tobytes())
    return p.get()
