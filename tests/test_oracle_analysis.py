"""The oracle's packing analysis (a restatement of the reference's disabled
statistics pass, pyrowave_encoder.cpp:625-958) on CPU: the counts it derives
from a parsed stream agree with what the stream and the oracle's own decoder
say independently."""
import numpy as np
import pytest

import oracle as O
from pyrowave_b200 import synth


def _parsed(w, h, c444, budget, seed):
    planes = synth.synth_frame(w, h, c444, seed)
    o = O.Oracle(w, h, c444)
    o.encode(planes, budget, sequence=1)
    stream, packets = o.packetize(2048, budget)
    p = o.parser()
    for off, sz in packets:
        assert p.push(stream[off:off + sz].tobytes())
    offs, payload = p.get()
    return o, offs, payload, sum(s for _, s in packets)


@pytest.mark.parametrize("w,h,c444,budget,seed", [(320, 240, False, 20000, 1), (256, 160, True, 60000, 2),
                                                   (34, 30, False, 65536, 3), (320, 240, False, 600, 4)])
def test_analysis_counts(w, h, c444, budget, seed):
    o, offs, payload, total = _parsed(w, h, c444, budget, seed)
    a = o.analyze_packing(offs, payload)
    # Coded bytes per band add up to the frame minus its 8-byte sequence header.
    assert int(a["band_bytes"].sum()) == total - 8
    # Nonzero coefficients are exactly the nonzero values the dequantiser produces.
    pyr = o.dequant(offs, payload)
    assert a["significant"] == int(np.count_nonzero(pyr))
    # Absent bands (4:2:0 chroma at level 0, LL above the last level) hold nothing.
    if not c444:
        assert not a["band_bytes"][1:, 0].any()
    assert not a["band_bytes"][:, :4, 0].any()
    lay = a["layout_bytes"]
    if a["significant"] == 0:
        assert not lay.any()
    else:
        assert (lay > 0).all()


def test_analysis_of_empty_stream_is_zero():
    o = O.Oracle(64, 64, False)
    offs = np.full(o.blocks32, 0xFFFFFFFF, np.uint32)
    a = o.analyze_packing(offs, np.zeros(0, np.uint32))
    assert not a["layout_bytes"].any() and not a["band_bytes"].any() and a["significant"] == 0
    assert not a["plane_histogram"].any()
