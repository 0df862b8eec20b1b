"""Packing analysis on the device (pyrowave_cuda_encoder_analyze_packing) against
the oracle's restatement of the reference's disabled statistics pass
(pyrowave_encoder.cpp:625-958: analyze_cost over 64x64 regions for five
packet / block / sub-block shapes, coded bytes per band, plane-byte histograms).

The two sides reach the quantised integers by different routes: the kernel from
the encoder's device buffers (the quantiser's magnitudes, code words and the
rate-control quant drops), the oracle by parsing the packetized stream with its
restated parser and reading every block's planes back. Every count must agree
exactly; the plane entropies must equal the byte entropy of the histogram."""
import numpy as np
import pytest

import oracle as O
from pyrowave_b200 import capi, synth

pytestmark = pytest.mark.gpu

CASES = [
    # w, h, 4:4:4, budget, seed, rects, lines
    (1280, 720, False, 150000, 0, 40, 0),
    (1920, 1080, False, 400000, 1, 40, 0),
    (1920, 1080, False, 30000, 2, 40, 0),      # most blocks dropped by rate control
    (960, 544, True, 300000, 3, 200, 24),      # 4:4:4 with the dense rectangle + line generator
    (34, 30, False, 65536, 4, 40, 0),          # bands narrower than one 64x64 region
    (1366, 768, True, 2000000, 5, 40, 0),      # high rate: many planes per sub-block
]


@pytest.fixture(scope="module")
def device(gpu):
    dev = capi.Device()
    yield dev
    dev.close()


def _entropy(hist):
    out = np.zeros(16)
    for j in range(16):
        t = hist[j].sum()
        if t:
            p = hist[j][hist[j] > 0].astype(np.float64) / float(t)
            out[j] = -(p * np.log2(p)).sum() / 8.0
    return out


@pytest.mark.parametrize("w,h,c444,budget,seed,rects,lines", CASES)
def test_analysis_matches_oracle(device, w, h, c444, budget, seed, rects, lines):
    planes = synth.synth_frame(w, h, c444, seed, rects=rects, lines=lines)
    chroma = capi.CHROMA_444 if c444 else capi.CHROMA_420
    enc = capi.Encoder(device, w, h, chroma)
    try:
        assert enc.encode_cpu(planes, budget) == capi.PYROWAVE_SUCCESS
        got = enc.analyze_packing()
        # Twice in a row: the accumulators are cleared per call.
        again = enc.analyze_packing()
        stream, packets = enc.packetize(2048, budget)
    finally:
        enc.close()
    total = sum(s for _, s in packets)
    assert total <= budget

    o = O.Oracle(w, h, c444)
    p = o.parser()
    for off, sz in packets:
        assert p.push(stream[off:off + sz].tobytes())
    offs, payload = p.get()
    want = o.analyze_packing(offs, payload)

    for k in ("layout_bytes", "band_bytes", "plane_histogram"):
        assert np.array_equal(got[k], want[k]), k
        assert np.array_equal(again[k], want[k]), k
    assert got["significant"] == want["significant"]
    assert got["coded_bytes"] == total - 8  # the stream minus its sequence header
    assert np.array_equal(got["plane_bytes"], want["plane_histogram"].sum(axis=1))
    np.testing.assert_allclose(got["plane_entropy"], _entropy(want["plane_histogram"]), rtol=1e-12, atol=1e-15)
    # The estimate for the current shape (32x32 packets, 4x2 sub-blocks) is within
    # a few percent of what the packer really wrote (it rounds signs per 8x8
    # block where the stream packs them per 32x32 block and pads to words).
    if total > 10000:
        assert abs(int(got["layout_bytes"][1]) - (total - 8)) < 0.05 * total


def test_analysis_before_encode_rejected(device):
    enc = capi.Encoder(device, 256, 144, capi.CHROMA_420)
    try:
        a = capi.PackingAnalysis()
        import ctypes

        assert enc.L.pyrowave_cuda_encoder_analyze_packing(enc.h, ctypes.byref(a)) == capi.PYROWAVE_ERROR_INVALID_ARGUMENT
        assert enc.L.pyrowave_cuda_encoder_analyze_packing(enc.h, None) == capi.PYROWAVE_ERROR_INVALID_ARGUMENT
    finally:
        enc.close()
