"""Generate the golden fixtures in this folder from the reference's own code.

    python tests/golden/make_golden.py

Requires oracle/_ref/libref_bitstream.so, i.e. the reference's Granite-free
bitstream code (metal/pyrowave_bitstream.cpp) compiled in place by
`make -C oracle`. The reference has no stored golden vectors of its own, so
these fixtures record what its block layout, packetizer, packet parser and
quant-code helpers produce on deterministic inputs. tests/test_oracle_pinning.py then
pins the oracle against them on machines without the reference tree.
"""
from __future__ import annotations

import hashlib
import json
import os
import sys

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(os.path.dirname(HERE))
sys.path.insert(0, ROOT)

import oracle as O  # noqa: E402

LAYOUT_SIZES = [(16, 16, 0), (34, 30, 0), (34, 30, 1), (1, 1, 1), (33, 17, 1), (130, 98, 0), (1280, 720, 0),
                (1366, 768, 0), (1920, 1080, 0), (1920, 1080, 1), (2560, 1080, 0), (2560, 1440, 1),
                (3840, 2160, 0), (3840, 2160, 1), (16384, 16, 1), (16384, 16384, 0)]


def sha(a: np.ndarray) -> str:
    return hashlib.sha256(np.ascontiguousarray(a).tobytes()).hexdigest()


def synthetic_meta(blocks: int, seed: int):
    """Per-block word counts (0 = empty) and a bitstream whose block headers are well formed."""
    rng = np.random.default_rng(seed)
    words = rng.integers(0, 24, blocks).astype(np.uint32)
    words[words < 8] = 0
    meta = np.zeros((blocks, 2), np.uint32)
    out = []
    off = 0
    for b in range(blocks):
        meta[b] = (off, words[b])
        if words[b]:
            blk = rng.integers(0, 2**32, int(words[b]), dtype=np.uint64).astype(np.uint32)
            ballot = int(rng.integers(1, 65536))
            blk[0] = (ballot & 0xFFFF) | (int(words[b]) << 16) | (5 << 28)
            blk[1] = (int(rng.integers(0, 256)) & 0xFF) | (b << 8)
            out.append(blk)
            off += int(words[b])
    return meta, (np.concatenate(out) if out else np.zeros(0, np.uint32))


def main():
    if not O.ref_available():
        raise SystemExit("oracle/_ref/libref_bitstream.so is missing: run `make -C oracle` where the reference tree exists")
    golden = {"layouts": [], "packetize": [], "parser": [], "quant_code": {}, "subdivision": []}
    arrays = {}

    for (w, h, c444) in LAYOUT_SIZES:
        r = O.RefBitstream(w, h, bool(c444))
        info = r.block_info()
        mapping = r.block_mapping()
        golden["layouts"].append({
            "width": w, "height": h, "chroma444": c444, "blocks8": r.blocks8, "blocks32": r.blocks32,
            "aligned_width": r.aligned_width, "aligned_height": r.aligned_height,
            "block_info": info.reshape(-1).tolist(), "mapping_sha256": sha(mapping),
        })

    # Packetize + parse on the 1280x720 4:2:0 layout with synthetic blocks.
    r = O.RefBitstream(1280, 720, False)
    meta, words = synthetic_meta(r.blocks32, seed=7)
    arrays["pk_meta"] = meta
    for boundary in (40, 1000, 1400, 8192, 65536, 1 << 22):
        for size in (8, 1000, 200000):
            stream, packets = r.packetize(meta, words, boundary, size)
            golden["packetize"].append({
                "boundary": boundary, "size": size, "num_packets": r.compute_num_packets(meta, boundary),
                "packets": packets.tolist(), "stream_sha256": sha(stream),
            })

    # Parser scenarios on a complete stream (sequence 5 in every header).
    stream, packets = r.packetize(meta, words, 8192, 200000)
    # Give the start-of-frame header sequence 5 as well so that it belongs to the same frame.
    hdr = stream[:8].copy().view(np.uint32)
    hdr[0] = (hdr[0] & ~np.uint32(7 << 28)) | np.uint32(5 << 28)
    stream[:8] = hdr.view(np.uint8)
    # The blocks are laid out in index order, so the stream minus its 8-byte
    # header is also the concatenated block words the packetizer consumed.
    assert np.array_equal(stream[8:8 + 4 * words.size].view(np.uint32), words)
    arrays["ps_stream"] = stream[: 8 + 4 * words.size]
    arrays["ps_packets"] = packets

    def scenario(name, pushes):
        r.parser_reset()
        log = []
        for data in pushes:
            ok = r.push(data)
            log.append([int(ok), int(r.ready(False)), int(r.ready(True)), r.decoded_blocks(), r.total_blocks()])
        offs, payload = r.parser_get()
        golden["parser"].append({"name": name, "log": log, "offsets_sha256": sha(offs), "payload_sha256": sha(payload),
                                 "payload_words": int(payload.size)})

    full = [stream[o:o + s].tobytes() for o, s in packets]
    scenario("in_order", full)
    scenario("reversed", full[::-1])
    scenario("duplicates", full[:3] + full[:3] + full[3:])
    scenario("drop_half", full[::2])
    trunc = bytearray(full[1])
    scenario("truncated", [full[0], bytes(trunc[:-4])])
    # Block header from an older sequence (4) after sequence 5: dropped. From a newer one (6): restart.
    def reseq(data: bytes, seq: int) -> bytes:
        a = np.frombuffer(data, np.uint8).copy()
        w0 = a[:4].view(np.uint32)
        w0[0] = (w0[0] & ~np.uint32(7 << 28)) | np.uint32(seq << 28)
        return a.tobytes()
    scenario("older_sequence", full[:2] + [reseq(full[2][: 4 * ((full[2][2] | (full[2][3] << 8)) & 0xFFF)], 4)])
    scenario("newer_sequence", full[:2] + [reseq(full[2][: 4 * ((full[2][2] | (full[2][3] << 8)) & 0xFFF)], 6)])
    bad = bytearray(full[0])
    bad_block = np.frombuffer(bytes(bad[8:16]), np.uint32).copy()
    bad_block[1] = (bad_block[1] & 0xFF) | (0xFFFFFF << 8)
    bad[8:16] = bad_block.tobytes()
    scenario("block_index_out_of_range", [bytes(bad)])
    wrong_dims = bytearray(full[0])
    w0 = np.frombuffer(bytes(wrong_dims[:4]), np.uint32).copy()
    w0[0] = (w0[0] & ~np.uint32(0x3FFF)) | np.uint32(99)
    wrong_dims[:4] = w0.tobytes()
    scenario("dimension_mismatch", [bytes(wrong_dims)])
    scenario("trailing_bytes", [full[0] + b"\x01\x02\x03"])

    # Quant codes.
    golden["quant_code"]["decode"] = [float(O.ref_decode_quant(c)) for c in range(200)]
    golden["quant_code"]["encode"] = {str(2.0 ** -b): O.ref_encode_quant(2.0 ** -b) for b in range(0, 17)}
    golden["subdivision"] = [[n, O.ref_block_count_per_subdivision(n)] for n in (1, 15, 16, 17, 100, 1473, 3261, 12429, 24669, 65535)]

    with open(os.path.join(HERE, "reference_bitstream.json"), "w") as f:
        json.dump(golden, f, indent=0, sort_keys=True)
    np.savez_compressed(os.path.join(HERE, "reference_bitstream.npz"), **arrays)
    print("wrote", os.path.join(HERE, "reference_bitstream.json"))


if __name__ == "__main__":
    main()
