"""Seeded synthetic YCbCr frames (stand-in for the reference's private game clips).

The generator is deterministic across machines: every random number comes from
SplitMix64 (Steele, Lea & Flood, "Fast splittable pseudorandom number
generators", OOPSLA 2014) evaluated with numpy uint64 arithmetic, and all
floating point work is float64 before the final rounding to 8 bits.

A frame is
  * a smooth 2D gradient (random direction and level per plane),
  * plus band-limited Gaussian noise (white noise through a separable [1,2,1]
    binomial filter applied twice, rescaled to the requested sigma),
  * overpainted by N sharp-edged flat rectangles,
  * optionally overpainted by 1-pixel line patterns (alternating rows or columns),
clamped to [16, 235] for luma and [16, 240] for chroma.
"""
from __future__ import annotations

import hashlib

import numpy as np

_M1 = np.uint64(0xBF58476D1CE4E5B9)
_M2 = np.uint64(0x94D049BB133111EB)
_GOLDEN = np.uint64(0x9E3779B97F4A7C15)


def _mix(z: np.ndarray) -> np.ndarray:
    z = z.astype(np.uint64, copy=True)
    with np.errstate(over="ignore"):
        z ^= z >> np.uint64(30)
        z *= _M1
        z ^= z >> np.uint64(27)
        z *= _M2
        z ^= z >> np.uint64(31)
    return z


def splitmix64(seed: int, count: int, stream: int = 0) -> np.ndarray:
    """count outputs of SplitMix64 started at seed, for an independent stream id."""
    with np.errstate(over="ignore"):
        base = np.uint64(seed & 0xFFFFFFFFFFFFFFFF) + np.uint64(stream) * np.uint64(0xD1B54A32D192ED03)
        idx = np.arange(1, count + 1, dtype=np.uint64)
        return _mix(base + idx * _GOLDEN)


def uniform(seed: int, count: int, stream: int) -> np.ndarray:
    """Uniform doubles in (0, 1) from the top 53 bits."""
    u = splitmix64(seed, count, stream) >> np.uint64(11)
    return (u.astype(np.float64) + 0.5) * (1.0 / 9007199254740992.0)


def gaussian(seed: int, shape, stream: int) -> np.ndarray:
    n = int(np.prod(shape))
    m = (n + 1) // 2
    u1 = uniform(seed, m, stream)
    u2 = uniform(seed, m, stream + 1)
    r = np.sqrt(-2.0 * np.log(u1))
    z = np.concatenate([r * np.cos(2.0 * np.pi * u2), r * np.sin(2.0 * np.pi * u2)])[:n]
    return z.reshape(shape)


def _binomial_blur(a: np.ndarray) -> np.ndarray:
    p = np.pad(a, 1, mode="reflect")
    h = 0.25 * p[:, :-2] + 0.5 * p[:, 1:-1] + 0.25 * p[:, 2:]
    return 0.25 * h[:-2, :] + 0.5 * h[1:-1, :] + 0.25 * h[2:, :]


def synth_plane(width: int, height: int, seed: int, plane: int, luma: bool, rects: int = 40,
                lines: int = 0, noise_sigma: float = 6.0) -> np.ndarray:
    lo, hi = (16.0, 235.0) if luma else (16.0, 240.0)
    s = 97 * plane + 11
    params = uniform(seed, 8, s)
    yy, xx = np.meshgrid(np.arange(height, dtype=np.float64), np.arange(width, dtype=np.float64), indexing="ij")
    angle = 2.0 * np.pi * params[0]
    t = (np.cos(angle) * xx / max(width, 1) + np.sin(angle) * yy / max(height, 1))
    if luma:
        base = 48.0 + 140.0 * (0.5 + 0.5 * t) + 20.0 * params[1]
    else:
        base = 128.0 + 60.0 * t * (params[1] - 0.5) * 2.0

    noise = gaussian(seed, (height, width), s + 2)
    noise = _binomial_blur(_binomial_blur(noise))
    std = float(noise.std())
    if std > 0:
        noise *= noise_sigma / std
    img = base + noise

    if rects > 0:
        r = uniform(seed, rects * 5, s + 4).reshape(rects, 5)
        for i in range(rects):
            cx, cy, rw, rh, val = r[i]
            w = max(1, int(rw * width * 0.25))
            h = max(1, int(rh * height * 0.25))
            x0 = int(cx * max(width - w, 1))
            y0 = int(cy * max(height - h, 1))
            img[y0:y0 + h, x0:x0 + w] = lo + (hi - lo) * val

    if lines > 0:
        r = uniform(seed, lines * 6, s + 5).reshape(lines, 6)
        for i in range(lines):
            cx, cy, rw, rh, v0, orient = r[i]
            w = max(2, int(rw * width * 0.15))
            h = max(2, int(rh * height * 0.15))
            x0 = int(cx * max(width - w, 1))
            y0 = int(cy * max(height - h, 1))
            a = lo + (hi - lo) * v0
            b = hi + lo - a
            region = img[y0:y0 + h, x0:x0 + w]
            if orient < 0.5:
                region[0::2, :] = a
                region[1::2, :] = b
            else:
                region[:, 0::2] = a
                region[:, 1::2] = b

    return np.clip(np.rint(img), lo, hi).astype(np.uint8)


def synth_frame(width: int, height: int, chroma444: bool, seed: int, rects: int = 40, lines: int = 0):
    """Y, Cb, Cr planes (chroma is width/2 x height/2 for 4:2:0)."""
    cw, ch = (width, height) if chroma444 else (width // 2, height // 2)
    y = synth_plane(width, height, seed, 0, True, rects, lines)
    cb = synth_plane(cw, ch, seed, 1, False, rects, lines)
    cr = synth_plane(cw, ch, seed, 2, False, rects, lines)
    return [y, cb, cr]


def frame_hash(planes) -> str:
    """Fingerprint (8-byte blake2b, hex) of the three planes."""
    h = hashlib.blake2b(digest_size=8)
    for p in planes:
        h.update(np.ascontiguousarray(p).tobytes())
    return h.hexdigest()


def gradient_frame(width: int, height: int, chroma444: bool):
    """The reference test's gradient input (pyrowave_c_test.cpp:288-308)."""
    yy, xx = np.meshgrid(np.arange(height), np.arange(width), indexing="ij")
    luma = ((3 * xx + 5 * yy) & 0xFF).astype(np.uint8)
    cb = ((7 * xx + 3 * yy) & 0xFF).astype(np.uint8)
    cr = ((3 * xx + 5 * yy) & 0xFF).astype(np.uint8)
    if chroma444:
        return [luma, cb, cr]
    return [luma, cb[: height // 2, : width // 2].copy(), cr[: height // 2, : width // 2].copy()]


def mirror_gradient_frame(width: int, height: int):
    """The reference stability test's 4:2:0 input (pyrowave_c_test.cpp:440-456):
    luma mirror(3x+5y), Cb mirror(5y+7x), Cr mirror(7x+3y)."""

    def mirror(v):
        v = v & 511
        return np.where(v > 255, 511 - v, v).astype(np.uint8)

    yy, xx = np.meshgrid(np.arange(height), np.arange(width), indexing="ij")
    luma = mirror(3 * xx + 5 * yy)
    cy, cx = np.meshgrid(np.arange(height // 2), np.arange(width // 2), indexing="ij")
    cb = mirror(cy * 5 + cx * 7)
    cr = mirror(7 * cx + cy * 3)
    return [luma, cb, cr]
