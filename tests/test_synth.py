"""The seeded frame generator: SplitMix64 against its published outputs, and
fingerprints of benchmark frames, so every harness and machine codes the same
frames."""
from pyrowave_b200 import synth


def test_splitmix64_known_answer():
    # SplitMix64 from state 0 (Steele, Lea & Flood 2014; the sequence Java's SplittableRandom uses).
    assert [int(x) for x in synth.splitmix64(0, 3)] == [0xE220A8397B1DCDAF, 0x6E789E6AA1B965F4, 0x06C45D188009454F]


def test_benchmark_frame_fingerprints():
    cases = [
        ((1280, 720, False, 0, 40, 0), "ca29b7e9c4fab120"),    # 720p workload, seed 0
        ((1920, 1080, False, 1, 40, 0), "3ff3f07e40a6491f"),   # 1080p workload, first seed
        ((3840, 2160, True, 1, 200, 40), "56a528decd878230"),  # 4K 4:4:4 workload, first seed
    ]
    for args, expect in cases:
        assert synth.frame_hash(synth.synth_frame(*args)) == expect, args
