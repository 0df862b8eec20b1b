"""PSNR-HVS-M restatement (shaders/psnr_hvs_m.comp, psnr.cpp:25-28,126-224,245-320
of the reference) on the CPU: its 8-point DCT is the orthonormal DCT-II, its
tables follow the CSF formula, and its sums behave as an error measure. The
library's host conversion to dB agrees with the oracle's."""
import math

import numpy as np

import oracle as O
from pyrowave_b200 import capi, synth


def _dct2_orthonormal(x):
    n = len(x)
    k = np.arange(n)[:, None]
    i = np.arange(n)[None, :]
    basis = np.cos(np.pi * (2 * i + 1) * k / (2 * n)) * np.sqrt(2.0 / n)
    basis[0] /= np.sqrt(2.0)
    return basis @ np.asarray(x, np.float64)


def test_dct8_is_orthonormal_dct2():
    rng = np.random.default_rng(3)
    for _ in range(50):
        x = rng.uniform(-1, 1, 8).astype(np.float32)
        got = O.hvs_dct8(x).astype(np.float64)
        want = _dct2_orthonormal(x)
        # The butterfly network leaves the sign of some odd coefficients to its
        # own convention; magnitudes are the DCT-II's.
        assert np.allclose(np.abs(got), np.abs(want), atol=2e-6), (got, want)
    # DC of a constant signal, energy preserved.
    assert abs(O.hvs_dct8(np.ones(8, np.float32))[0] - math.sqrt(8)) < 1e-6


def test_tables_follow_the_csf_formula():
    h = 1080
    t = O.psnr_hvs_m_tables(h).astype(np.float64)
    for f in (0, 7, 15):
        nyq = h * (1 + f / 8) * np.pi / 360
        for y in range(8):
            for x in range(8):
                cpd = np.hypot((x + 0.5) / 8, (y + 0.5) / 8) * nyq
                csf = 2.6 * 2.6 * (0.0192 + 0.114 * cpd) * np.exp(-(0.114 * cpd) ** 1.1)
                assert abs(t[f, 0, y, x] - csf) <= 1e-5 * abs(csf) + 1e-9
        assert t[f, 1, 0, 0] == 0.0 and t[f, 2, 0, 0] == 0.0
        assert np.isclose(t[f, 1].max(), 1.0, rtol=1e-6)  # normalised by the largest CSF value squared
        nz = t[f, 1] > 0
        assert np.allclose(t[f, 2][nz], 1.0 / t[f, 1][nz], rtol=1e-6)


def test_error_sums_behave():
    y = synth.synth_frame(320, 180, False, 4)[0]
    assert not O.psnr_hvs_m_errors(y, y).any()
    rng = np.random.default_rng(1)
    small = np.clip(y.astype(int) + rng.integers(-2, 3, y.shape), 0, 255).astype(np.uint8)
    large = np.clip(y.astype(int) + rng.integers(-12, 13, y.shape), 0, 255).astype(np.uint8)
    e_small, e_large = O.psnr_hvs_m_errors(y, small), O.psnr_hvs_m_errors(y, large)
    assert (e_large > e_small).all() and (e_small > 0).all()
    assert O.psnr_hvs_m_pixels(320, 180) == 80 * 45 * 64
    assert O.psnr_hvs_m_pixels(321, 181) == 81 * 46 * 64


def test_library_conversion_matches_oracle():
    y = synth.synth_frame(256, 144, False, 2)[0]
    d = np.clip(y.astype(int) + 3, 0, 255).astype(np.uint8)
    e = O.psnr_hvs_m_errors(y, d)
    px = O.psnr_hvs_m_pixels(256, 144)
    assert capi.lib().pyrowave_psnr_hvs_m_pixels(256, 144) == px
    for full in (True, False):
        assert np.allclose(capi.psnr_hvs_m_db(e, px, full), O.psnr_hvs_m_db(e, px, full), rtol=0, atol=1e-12)
