"""Whole-frame coding through the CPU oracle (test infrastructure): what a
frame's packetized bitstream and decoded planes must be, for the tests that
check the library's batched form, device packet assembly and serving loop."""
import numpy as np

import oracle as O


def oracle_frame(w, h, c444, planes, budget, sequence, mode=O.MODE_F32, fp16_mask=0):
    """Encodes `planes` within `budget` bytes as the encoder's frame number
    `sequence` (its 3-bit sequence field), then parses and decodes the result.
    Returns (packetized frame bytes: the 8-byte header and the coded blocks in
    block order, decoded planes)."""
    o = O.Oracle(w, h, c444, fp16_mask)
    o.encode(planes, budget, mode, sequence=sequence & 7)
    stream, packets = o.packetize(1 << 30, budget)
    total = int(sum(int(sz) for _, sz in packets))
    data = stream[:total].copy()
    return data, oracle_decode(o, [data.tobytes()], mode)


def oracle_decode(o, packets, mode=O.MODE_F32):
    """Decoded planes of the oracle parser after pushing `packets` in order
    (rejected packets keep what they added before the fault, as the parser does)."""
    p = o.parser()
    for pkt in packets:
        p.push(pkt)
    offs, payload = p.get()
    return o.idwt(o.dequant(offs, payload, mode), mode)


def words_as_bytes(words: np.ndarray) -> np.ndarray:
    return np.ascontiguousarray(words, np.uint32).view(np.uint8)
