"""bench.py's algorithmic-byte accounting, which every roofline figure divides by.

DWT stage bytes per frame = the 8-bit input read once plus every subband
coefficient written once. The expected totals are computed independently from
the aligned frame sizes (1280x736, 1920x1088, 3840x2176): input bytes +
coefficients x 4 bytes (x 2 with FP16 storage).
"""
import os
import sys

import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
if ROOT not in sys.path:
    sys.path.insert(0, ROOT)

import bench  # noqa: E402


@pytest.mark.parametrize("name, input_bytes, coefs", [
    ("720p", 1_382_400, 1_413_120),
    ("1080p", 3_110_400, 3_133_440),
    ("4k", 12_441_600, 12_533_760),
    ("4k444", 24_883_200, 25_067_520),
])
def test_dwt_stage_bytes(name, input_bytes, coefs):
    alg = bench.algorithmic_bytes(bench.CONFIGS[name], 0)
    assert alg["dwt_stage"] == input_bytes + 4 * coefs
    # The five levels' outputs are all coefficients the frame holds at some level.
    assert alg["dwt0"] <= alg["dwt_stage"]


def test_fp16_storage_halves_coefficient_bytes():
    alg = bench.algorithmic_bytes(bench.CONFIGS["1080p"], 0x1F)
    assert alg["dwt_stage"] == 3_110_400 + 2 * 3_133_440


def test_level0_luma_bytes_1080p():
    # Luma 1920x1080 read once, four 960x544 FP32 bands written once.
    alg = bench.algorithmic_bytes(bench.CONFIGS["1080p"], 0)
    assert alg["dwt0"] == 1920 * 1080 + 4 * 960 * 544 * 4
