"""PSNR-HVS-M on the GPU (pyrowave_cuda_psnr_hvs_m) against the oracle's
restatement of the reference metric: the 16 fixed-point error sums are
identical integers, for decoded frames of the codec and odd plane sizes, and
sums accumulate over frames."""
import numpy as np
import pytest

import oracle as O
from pyrowave_b200 import capi, synth

pytestmark = pytest.mark.gpu


def _gpu_errors(ref, dist, errors=None):
    import torch

    a = torch.from_numpy(np.ascontiguousarray(ref)).cuda()
    b = torch.from_numpy(np.ascontiguousarray(dist)).cuda()
    if errors is None:
        errors = torch.zeros(16, dtype=torch.int64, device="cuda")
    h, w = ref.shape
    assert capi.psnr_hvs_m(w, h, a.data_ptr(), a.stride(0), b.data_ptr(), b.stride(0),
                           errors.data_ptr()) == capi.PYROWAVE_SUCCESS
    torch.cuda.synchronize()
    return errors


def _decoded_luma(w, h, c444, seed, budget):
    o = O.Oracle(w, h, c444)
    planes = synth.synth_frame(w, h, c444, seed)
    o.encode(planes, budget, sequence=1)
    stream, packets = o.packetize(1 << 30, budget)
    p = o.parser()
    for off, sz in packets:
        p.push(stream[int(off):int(off) + int(sz)].tobytes())
    offs, payload = p.get()
    return planes[0], o.idwt(o.dequant(offs, payload))[0]


@pytest.mark.parametrize("w,h,c444,seed,budget", [(1920, 1080, False, 1, 400000), (333, 197, True, 5, 20000),
                                                   (1280, 720, False, 0, 150000)])
def test_psnr_hvs_m_matches_oracle(gpu, w, h, c444, seed, budget):
    ref, dist = _decoded_luma(w, h, c444, seed, budget)
    got = _gpu_errors(ref, dist).cpu().numpy().view(np.uint64)
    want = O.psnr_hvs_m_errors(ref, dist)
    assert np.array_equal(got, want), (got, want)
    db = capi.psnr_hvs_m_db(got, capi.lib().pyrowave_psnr_hvs_m_pixels(w, h))
    assert np.all(np.isfinite(db)) and np.all(db > 20)


def test_psnr_hvs_m_accumulates_and_rejects(gpu):
    import torch

    ref, dist = _decoded_luma(640, 360, False, 9, 30000)
    ref2, dist2 = _decoded_luma(640, 360, False, 10, 30000)
    errors = _gpu_errors(ref, dist)
    _gpu_errors(ref2, dist2, errors)
    want = O.psnr_hvs_m_errors(ref, dist) + O.psnr_hvs_m_errors(ref2, dist2)
    assert np.array_equal(errors.cpu().numpy().view(np.uint64), want)
    # Identical planes add nothing.
    before = errors.clone()
    _gpu_errors(ref, ref, errors)
    assert torch.equal(before, errors)
    bad = capi.PYROWAVE_ERROR_INVALID_ARGUMENT
    assert capi.psnr_hvs_m(0, 360, 1, 640, 2, 640, errors.data_ptr()) == bad
    assert capi.psnr_hvs_m(640, 360, 1, 639, 2, 640, errors.data_ptr()) == bad
    assert capi.psnr_hvs_m(640, 360, 1, 640, 2, 640, errors.data_ptr() + 4) == bad
