"""Python binding of the PyroWave CPU oracle.

TEST INFRASTRUCTURE ONLY: imported by tests/, by ``__graft_entry__.smoke()`` and
by the ``cpu_baseline`` / ``--impl reference`` legs of ``bench.py``. The product
(``pyrowave_b200``) never imports it.

``Oracle`` wraps ``liboracle.so`` (a C++ restatement of the reference's encode /
decode path, see ``pyrowave_oracle.cpp``). ``RefBitstream`` wraps
``_ref/libref_bitstream.so``, which is the reference's own Granite-free C++
(``metal/pyrowave_bitstream.cpp``) compiled in place; it exists only where the
reference tree was available at build time.
"""
from __future__ import annotations

import ctypes
import os
from ctypes import POINTER, c_char_p, c_float, c_int, c_int32, c_int64, c_size_t, c_uint, c_uint16, c_uint32, c_uint64, c_void_p

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
LIB_PATH = os.path.join(HERE, "liboracle.so")
REF_LIB_PATH = os.path.join(HERE, "_ref", "libref_bitstream.so")

MODE_F32 = 0
MODE_REF16 = 1
MODE_F64 = 2

_lib = None
_ref = None


def build(reference: str | None = None) -> None:
    """Compile the oracle (and _ref when the reference tree is present)."""
    import subprocess

    cmd = ["make", "-s", "-C", HERE]
    if reference:
        cmd.append(f"REFERENCE={reference}")
    subprocess.run(cmd, check=True)


def _ptr(a: np.ndarray):
    return a.ctypes.data_as(c_void_p)


def lib():
    global _lib
    if _lib is None:
        if not os.path.exists(LIB_PATH):
            build()
        L = ctypes.CDLL(LIB_PATH)
        L.oracle_create.restype = c_void_p
        L.oracle_create.argtypes = [c_int, c_int, c_int, c_uint]
        L.oracle_destroy.argtypes = [c_void_p]
        for name in ("oracle_aligned_width", "oracle_aligned_height", "oracle_block_count_8x8", "oracle_block_count_32x32"):
            getattr(L, name).restype = c_int
            getattr(L, name).argtypes = [c_void_p]
        L.oracle_pyramid_size.restype = c_size_t
        L.oracle_pyramid_size.argtypes = [c_void_p]
        L.oracle_psnr_hvs_m.argtypes = [c_void_p, c_int, c_void_p, c_int, c_int, c_int, c_void_p]
        L.oracle_psnr_hvs_m.restype = None
        L.oracle_psnr_hvs_m_tables.argtypes = [c_int, c_void_p]
        L.oracle_psnr_hvs_m_tables.restype = None
        L.oracle_psnr_hvs_m_pixels.argtypes = [c_int, c_int]
        L.oracle_psnr_hvs_m_pixels.restype = c_uint64
        L.oracle_hvs_dct8.argtypes = [c_void_p, c_void_p]
        L.oracle_hvs_dct8.restype = None
        L.oracle_block_info.argtypes = [c_void_p, c_void_p]
        L.oracle_block_mapping.argtypes = [c_void_p, c_void_p]
        L.oracle_band_offsets.argtypes = [c_void_p, c_void_p]
        L.oracle_quant_tables.argtypes = [c_void_p, c_void_p, c_void_p]
        L.oracle_dwt.restype = c_int
        L.oracle_dwt.argtypes = [c_void_p, c_void_p, c_void_p, c_int, c_void_p]
        L.oracle_dwt_f64.restype = c_int
        L.oracle_dwt_f64.argtypes = [c_void_p, c_void_p, c_void_p, c_void_p]
        L.oracle_encode_pyramid.restype = c_int
        L.oracle_encode_pyramid.argtypes = [c_void_p, c_void_p, c_uint64, c_uint32, c_float]
        for name in ("oracle_get_code_words", "oracle_get_block_stats", "oracle_get_quant", "oracle_get_meta", "oracle_get_bitstream"):
            getattr(L, name).argtypes = [c_void_p, c_void_p]
        L.oracle_get_rd.argtypes = [c_void_p, c_void_p, c_void_p, c_void_p]
        L.oracle_get_histogram.argtypes = [c_void_p, c_void_p, c_void_p]
        L.oracle_get_bitstream_words.restype = c_size_t
        L.oracle_get_bitstream_words.argtypes = [c_void_p]
        L.oracle_set_encoded.argtypes = [c_void_p, c_void_p, c_void_p, c_size_t, c_uint32]
        L.oracle_compute_num_packets.restype = c_size_t
        L.oracle_compute_num_packets.argtypes = [c_void_p, c_size_t]
        L.oracle_packetize.restype = c_size_t
        L.oracle_packetize.argtypes = [c_void_p, c_void_p, c_size_t, c_void_p, c_size_t]
        L.oracle_parser_create.restype = c_void_p
        L.oracle_parser_create.argtypes = [c_void_p]
        L.oracle_parser_destroy.argtypes = [c_void_p]
        L.oracle_parser_clear.argtypes = [c_void_p]
        L.oracle_parser_push_packet.restype = c_int
        L.oracle_parser_push_packet.argtypes = [c_void_p, c_void_p, c_size_t]
        L.oracle_parser_decode_is_ready.restype = c_int
        L.oracle_parser_decode_is_ready.argtypes = [c_void_p, c_int]
        L.oracle_parser_mark_decoded.argtypes = [c_void_p]
        L.oracle_parser_payload_words.restype = c_size_t
        L.oracle_parser_payload_words.argtypes = [c_void_p]
        L.oracle_parser_get.argtypes = [c_void_p, c_void_p, c_void_p]
        L.oracle_parser_decoded_blocks.restype = c_int
        L.oracle_parser_decoded_blocks.argtypes = [c_void_p]
        L.oracle_parser_total_blocks.restype = c_int
        L.oracle_parser_total_blocks.argtypes = [c_void_p]
        L.oracle_dequant.restype = c_int
        L.oracle_dequant.argtypes = [c_void_p, c_void_p, c_void_p, c_size_t, c_int, c_void_p]
        L.oracle_idwt.restype = c_int
        L.oracle_idwt.argtypes = [c_void_p, c_void_p, c_int, c_void_p, c_void_p]
        L.oracle_idwt_f64.restype = c_int
        L.oracle_idwt_f64.argtypes = [c_void_p, c_void_p, c_void_p, c_void_p]
        L.oracle_dwt16.restype = c_int
        L.oracle_dwt16.argtypes = [c_void_p, c_void_p, c_void_p, c_int, c_void_p]
        L.oracle_idwt16.restype = c_int
        L.oracle_idwt16.argtypes = [c_void_p, c_void_p, c_int, c_void_p, c_void_p]
        L.oracle_analyze_packing.restype = c_int
        L.oracle_analyze_packing.argtypes = [c_void_p, c_void_p, c_void_p, c_size_t, c_void_p, c_void_p, c_void_p,
                                             c_void_p]
        L.oracle_float_to_half.restype = c_uint16
        L.oracle_float_to_half.argtypes = [c_float]
        L.oracle_half_to_float.restype = c_float
        L.oracle_half_to_float.argtypes = [c_uint16]
        L.oracle_bucket_index.restype = c_uint32
        L.oracle_bucket_index.argtypes = [c_float, c_float, c_float, c_float]
        _lib = L
    return _lib


def _plane_args(planes):
    arrs = [np.ascontiguousarray(p, dtype=np.uint8) for p in planes]
    ptrs = (c_void_p * 3)(*[a.ctypes.data for a in arrs])
    strides = (c_int * 3)(*[a.shape[1] for a in arrs])
    return arrs, ptrs, strides


class Oracle:
    """One frame geometry (width, height, chroma) of the CPU restatement."""

    def __init__(self, width: int, height: int, chroma444: bool = False, fp16_level_mask: int = 0):
        self.L = lib()
        self.h = self.L.oracle_create(width, height, int(chroma444), fp16_level_mask)
        if not self.h:
            raise ValueError("invalid oracle geometry")
        self.width, self.height, self.chroma444 = width, height, chroma444
        self.aligned_width = self.L.oracle_aligned_width(self.h)
        self.aligned_height = self.L.oracle_aligned_height(self.h)
        self.blocks8 = self.L.oracle_block_count_8x8(self.h)
        self.blocks32 = self.L.oracle_block_count_32x32(self.h)
        self.pyramid_size = self.L.oracle_pyramid_size(self.h)
        self.sequence = 0

    def __del__(self):
        if getattr(self, "h", None):
            self.L.oracle_destroy(self.h)
            self.h = None

    # --- layout -------------------------------------------------------------
    def block_info(self) -> np.ndarray:
        out = np.zeros((3, 5, 4, 4), np.int32)
        self.L.oracle_block_info(self.h, _ptr(out))
        return out

    def block_mapping(self) -> np.ndarray:
        out = np.zeros((self.blocks32, 4), np.int32)
        self.L.oracle_block_mapping(self.h, _ptr(out))
        return out

    def band_offsets(self) -> np.ndarray:
        out = np.zeros((3, 5, 4), np.int64)
        self.L.oracle_band_offsets(self.h, _ptr(out))
        return out

    def quant_tables(self):
        qr = np.zeros((3, 5, 4), np.float32)
        rdo = np.zeros((3, 5, 4), np.float32)
        self.L.oracle_quant_tables(self.h, _ptr(qr), _ptr(rdo))
        return qr, rdo

    def plane_shapes(self):
        if self.chroma444:
            return [(self.height, self.width)] * 3
        return [(self.height, self.width), (self.height // 2, self.width // 2), (self.height // 2, self.width // 2)]

    # --- transform ------------------------------------------------------------
    def dwt(self, planes, mode: int = MODE_F32) -> np.ndarray:
        """Forward transform of 8-bit planes, or of 16-bit (R16_UNORM) planes when they are uint16."""
        if np.asarray(planes[0]).dtype == np.uint16:
            arrs = [np.ascontiguousarray(p, np.uint16) for p in planes]
            ptrs = (c_void_p * 3)(*[a.ctypes.data for a in arrs])
            strides = (c_int * 3)(*[a.shape[1] for a in arrs])
            out = np.zeros(self.pyramid_size, np.float32)
            if self.L.oracle_dwt16(self.h, ptrs, strides, mode, _ptr(out)) != 0:
                raise RuntimeError("oracle_dwt16 failed")
            return out
        arrs, ptrs, strides = _plane_args(planes)
        if mode == MODE_F64:
            out = np.zeros(self.pyramid_size, np.float64)
            rc = self.L.oracle_dwt_f64(self.h, ptrs, strides, _ptr(out))
        else:
            out = np.zeros(self.pyramid_size, np.float32)
            rc = self.L.oracle_dwt(self.h, ptrs, strides, mode, _ptr(out))
        if rc != 0:
            raise RuntimeError("oracle_dwt failed")
        return out

    def idwt16(self, pyramid: np.ndarray, mode: int = MODE_F32):
        """Inverse transform into 16-bit (R16_UNORM) planes."""
        outs = [np.zeros(s, np.uint16) for s in self.plane_shapes()]
        ptrs = (c_void_p * 3)(*[a.ctypes.data for a in outs])
        strides = (c_int * 3)(*[a.shape[1] for a in outs])
        p = np.ascontiguousarray(pyramid, np.float32)
        if self.L.oracle_idwt16(self.h, _ptr(p), mode, ptrs, strides) != 0:
            raise RuntimeError("oracle_idwt16 failed")
        return outs

    def idwt(self, pyramid: np.ndarray, mode: int = MODE_F32):
        outs = [np.zeros(s, np.uint8) for s in self.plane_shapes()]
        ptrs = (c_void_p * 3)(*[a.ctypes.data for a in outs])
        strides = (c_int * 3)(*[a.shape[1] for a in outs])
        if mode == MODE_F64:
            p = np.ascontiguousarray(pyramid, np.float64)
            rc = self.L.oracle_idwt_f64(self.h, _ptr(p), ptrs, strides)
        else:
            p = np.ascontiguousarray(pyramid, np.float32)
            rc = self.L.oracle_idwt(self.h, _ptr(p), mode, ptrs, strides)
        if rc != 0:
            raise RuntimeError("oracle_idwt failed")
        return outs

    # --- encoder --------------------------------------------------------------
    def encode_pyramid(self, pyramid: np.ndarray, budget: int, sequence: int | None = None, quant_scale: float = -1.0):
        if sequence is None:
            self.sequence = (self.sequence + 1) & 7
            sequence = self.sequence
        p = np.ascontiguousarray(pyramid, np.float32)
        rc = self.L.oracle_encode_pyramid(self.h, _ptr(p), budget, sequence, quant_scale)
        if rc != 0:
            raise ValueError(f"oracle_encode_pyramid returned {rc}")

    def encode(self, planes, budget: int, mode: int = MODE_F32, sequence: int | None = None):
        pyr = self.dwt(planes, mode)
        self.encode_pyramid(pyr, budget, sequence)
        return pyr

    def code_words(self):
        out = np.zeros(self.blocks8, np.uint32)
        self.L.oracle_get_code_words(self.h, _ptr(out))
        return out

    def block_stats(self):
        out = np.zeros((self.blocks8, 17), np.uint32)
        self.L.oracle_get_block_stats(self.h, _ptr(out))
        return out

    def rd(self):
        rc = np.zeros((self.blocks32, 16), np.uint32)
        d = np.zeros((self.blocks32, 16), np.float32)
        b = np.zeros((self.blocks32, 16), np.uint32)
        self.L.oracle_get_rd(self.h, _ptr(rc), _ptr(d), _ptr(b))
        return rc, d, b

    def histogram(self):
        scan = np.zeros(2048, np.uint32)
        consumed = np.zeros(1, np.uint32)
        self.L.oracle_get_histogram(self.h, _ptr(scan), _ptr(consumed))
        return scan, int(consumed[0])

    def quant(self):
        out = np.zeros(self.blocks32, np.int32)
        self.L.oracle_get_quant(self.h, _ptr(out))
        return out

    def meta(self):
        out = np.zeros((self.blocks32, 2), np.uint32)
        self.L.oracle_get_meta(self.h, _ptr(out))
        return out

    def bitstream_words(self):
        n = self.L.oracle_get_bitstream_words(self.h)
        out = np.zeros(n, np.uint32)
        if n:
            self.L.oracle_get_bitstream(self.h, _ptr(out))
        return out

    def set_encoded(self, meta: np.ndarray, words: np.ndarray, sequence: int):
        m = np.ascontiguousarray(meta, np.uint32)
        w = np.ascontiguousarray(words, np.uint32)
        if w.size == 0:
            w = np.zeros(1, np.uint32)
            n = 0
        else:
            n = w.size
        self.L.oracle_set_encoded(self.h, _ptr(m), _ptr(w), n, sequence)

    def compute_num_packets(self, boundary: int) -> int:
        return int(self.L.oracle_compute_num_packets(self.h, boundary))

    def packetize(self, boundary: int, size: int):
        n = self.compute_num_packets(boundary)
        packets = np.zeros((max(n, 1), 2), np.uint64)
        out = np.zeros(size, np.uint8)
        got = self.L.oracle_packetize(self.h, _ptr(packets), boundary, _ptr(out), size)
        return out, packets[:got].astype(np.int64)

    # --- decoder --------------------------------------------------------------
    def dequant(self, offsets: np.ndarray, payload: np.ndarray, mode: int = MODE_F32) -> np.ndarray:
        out = np.zeros(self.pyramid_size, np.float32)
        off = np.ascontiguousarray(offsets, np.uint32)
        pay = np.ascontiguousarray(payload, np.uint32)
        if pay.size == 0:
            pay = np.zeros(1, np.uint32)
            nwords = 0
        else:
            nwords = pay.size
        self.L.oracle_dequant(self.h, _ptr(off), _ptr(pay), nwords, mode, _ptr(out))
        return out

    def analyze_packing(self, offsets: np.ndarray, payload: np.ndarray) -> dict:
        """Packing statistics of a parsed frame (pyrowave_encoder.cpp:625-958): the
        estimated bytes of the five alternative layouts, coded bytes per band,
        the nonzero count and the plane-byte histograms."""
        off = np.ascontiguousarray(offsets, np.uint32)
        pay = np.ascontiguousarray(payload, np.uint32)
        nwords = pay.size
        if pay.size == 0:
            pay = np.zeros(1, np.uint32)
        layouts = np.zeros(5, np.uint64)
        bands = np.zeros((3, 5, 4), np.uint64)
        sig = np.zeros(1, np.uint64)
        hist = np.zeros((16, 256), np.uint32)
        self.L.oracle_analyze_packing(self.h, _ptr(off), _ptr(pay), nwords, _ptr(layouts), _ptr(bands), _ptr(sig),
                                      _ptr(hist))
        return {"layout_bytes": layouts, "band_bytes": bands, "significant": int(sig[0]), "plane_histogram": hist}

    def parser(self):
        return Parser(self)


class Parser:
    """Restated packet parser (pyrowave_decoder.cpp:126-262)."""

    def __init__(self, oracle: Oracle):
        self.o = oracle
        self.L = oracle.L
        self.h = self.L.oracle_parser_create(oracle.h)

    def __del__(self):
        if getattr(self, "h", None):
            self.L.oracle_parser_destroy(self.h)
            self.h = None

    def clear(self):
        self.L.oracle_parser_clear(self.h)

    def push(self, data) -> bool:
        buf = np.ascontiguousarray(np.frombuffer(bytes(data), np.uint8)) if not isinstance(data, np.ndarray) else np.ascontiguousarray(data, np.uint8)
        if buf.size == 0:
            buf2 = np.zeros(1, np.uint8)
            return self.L.oracle_parser_push_packet(self.h, _ptr(buf2), 0) == 0
        return self.L.oracle_parser_push_packet(self.h, _ptr(buf), buf.size) == 0

    def ready(self, allow_partial: bool = False) -> bool:
        return bool(self.L.oracle_parser_decode_is_ready(self.h, int(allow_partial)))

    def mark_decoded(self):
        self.L.oracle_parser_mark_decoded(self.h)

    def get(self):
        n = self.L.oracle_parser_payload_words(self.h)
        offsets = np.zeros(self.o.blocks32, np.uint32)
        payload = np.zeros(max(n, 1), np.uint32)
        self.L.oracle_parser_get(self.h, _ptr(offsets), _ptr(payload))
        return offsets, payload[:n]

    def decoded_blocks(self):
        return self.L.oracle_parser_decoded_blocks(self.h)

    def total_blocks(self):
        return self.L.oracle_parser_total_blocks(self.h)


def float_to_half(v: float) -> int:
    return int(lib().oracle_float_to_half(v))


def half_to_float(h: int) -> float:
    return float(lib().oracle_half_to_float(h))


def bucket_index(d, cost, d_base, cost_base) -> int:
    return int(lib().oracle_bucket_index(d, cost, d_base, cost_base))


# ---------------------------------------------------------------------------
def ref_available() -> bool:
    return os.path.exists(REF_LIB_PATH)


def ref_lib():
    global _ref
    if _ref is None:
        R = ctypes.CDLL(REF_LIB_PATH)
        R.ref_layout_create.restype = c_void_p
        R.ref_layout_create.argtypes = [c_int, c_int, c_int]
        R.ref_layout_destroy.argtypes = [c_void_p]
        R.ref_layout_counts.argtypes = [c_void_p, c_void_p]
        R.ref_layout_block_info.argtypes = [c_void_p, c_void_p]
        R.ref_layout_block_mapping.argtypes = [c_void_p, c_void_p]
        R.ref_block_count_per_subdivision.restype = c_int
        R.ref_block_count_per_subdivision.argtypes = [c_int]
        R.ref_compute_num_packets.restype = c_size_t
        R.ref_compute_num_packets.argtypes = [c_void_p, c_void_p, c_size_t]
        R.ref_packetize.restype = c_size_t
        R.ref_packetize.argtypes = [c_void_p, c_void_p, c_size_t, c_size_t, c_void_p, c_size_t, c_void_p, c_void_p]
        R.ref_decode_quant.restype = c_float
        R.ref_decode_quant.argtypes = [c_uint32]
        R.ref_encode_quant.restype = c_uint32
        R.ref_encode_quant.argtypes = [c_float]
        R.ref_parser_create.restype = c_void_p
        R.ref_parser_create.argtypes = [c_void_p]
        R.ref_parser_destroy.argtypes = [c_void_p]
        R.ref_parser_clear.argtypes = [c_void_p]
        R.ref_parser_push_packet.restype = c_int
        R.ref_parser_push_packet.argtypes = [c_void_p, c_void_p, c_size_t]
        R.ref_parser_decode_is_ready.restype = c_int
        R.ref_parser_decode_is_ready.argtypes = [c_void_p, c_int]
        R.ref_parser_mark_decoded.argtypes = [c_void_p]
        R.ref_parser_payload_words.restype = c_size_t
        R.ref_parser_payload_words.argtypes = [c_void_p]
        R.ref_parser_get.argtypes = [c_void_p, c_void_p, c_void_p]
        R.ref_parser_decoded_blocks.restype = c_int
        R.ref_parser_decoded_blocks.argtypes = [c_void_p]
        R.ref_parser_total_blocks.restype = c_int
        R.ref_parser_total_blocks.argtypes = [c_void_p]
        _ref = R
    return _ref


class RefBitstream:
    """The reference's BlockLayout / packetize / BitstreamParser (metal/pyrowave_bitstream.cpp)."""

    def __init__(self, width: int, height: int, chroma444: bool = False):
        self.R = ref_lib()
        self.h = self.R.ref_layout_create(width, height, int(chroma444))
        if not self.h:
            raise ValueError("invalid geometry")
        c = np.zeros(4, np.int32)
        self.R.ref_layout_counts(self.h, _ptr(c))
        self.blocks8, self.blocks32, self.aligned_width, self.aligned_height = (int(v) for v in c)
        self.parser_h = None

    def __del__(self):
        if getattr(self, "parser_h", None):
            self.R.ref_parser_destroy(self.parser_h)
        if getattr(self, "h", None):
            self.R.ref_layout_destroy(self.h)

    def block_info(self):
        out = np.zeros((3, 5, 4, 4), np.int32)
        self.R.ref_layout_block_info(self.h, _ptr(out))
        return out

    def block_mapping(self):
        out = np.zeros((self.blocks32, 4), np.int32)
        self.R.ref_layout_block_mapping(self.h, _ptr(out))
        return out

    def compute_num_packets(self, meta: np.ndarray, boundary: int) -> int:
        m = np.ascontiguousarray(meta, np.uint32)
        return int(self.R.ref_compute_num_packets(self.h, _ptr(m), boundary))

    def packetize(self, meta: np.ndarray, words: np.ndarray, boundary: int, size: int):
        m = np.ascontiguousarray(meta, np.uint32)
        w = np.ascontiguousarray(words, np.uint32)
        if w.size == 0:
            w = np.zeros(1, np.uint32)
        n = self.compute_num_packets(m, boundary)
        packets = np.zeros((max(n, 1), 2), np.uint64)
        out = np.zeros(size, np.uint8)
        got = self.R.ref_packetize(self.h, _ptr(packets), max(n, 1), boundary, _ptr(out), size, _ptr(m), _ptr(w))
        return out, packets[:got].astype(np.int64)

    def parser_reset(self):
        if self.parser_h:
            self.R.ref_parser_destroy(self.parser_h)
        self.parser_h = self.R.ref_parser_create(self.h)

    def push(self, data) -> bool:
        if not self.parser_h:
            self.parser_reset()
        buf = np.ascontiguousarray(np.frombuffer(bytes(data), np.uint8))
        if buf.size == 0:
            return self.R.ref_parser_push_packet(self.parser_h, _ptr(np.zeros(1, np.uint8)), 0) == 0
        return self.R.ref_parser_push_packet(self.parser_h, _ptr(buf), buf.size) == 0

    def ready(self, allow_partial=False) -> bool:
        return bool(self.R.ref_parser_decode_is_ready(self.parser_h, int(allow_partial)))

    def parser_get(self):
        n = self.R.ref_parser_payload_words(self.parser_h)
        offsets = np.zeros(self.blocks32, np.uint32)
        payload = np.zeros(max(n, 1), np.uint32)
        self.R.ref_parser_get(self.parser_h, _ptr(offsets), _ptr(payload))
        return offsets, payload[:n]

    def decoded_blocks(self):
        return self.R.ref_parser_decoded_blocks(self.parser_h)

    def total_blocks(self):
        return self.R.ref_parser_total_blocks(self.parser_h)


def ref_encode_quant(v: float) -> int:
    return int(ref_lib().ref_encode_quant(v))


def ref_decode_quant(code: int) -> float:
    return float(ref_lib().ref_decode_quant(code))


def ref_block_count_per_subdivision(n: int) -> int:
    return int(ref_lib().ref_block_count_per_subdivision(n))


def psnr_hvs_m_errors(ref: np.ndarray, dist: np.ndarray) -> np.ndarray:
    """Per height factor (1 + i/8, i = 0..15) fixed-point (2^-24) PSNR-HVS-M error
    sums of a distorted luma plane against its reference (psnr_hvs_m.comp)."""
    L = lib()
    a = np.ascontiguousarray(ref, np.uint8)
    b = np.ascontiguousarray(dist, np.uint8)
    out = np.zeros(16, np.uint64)
    L.oracle_psnr_hvs_m(_ptr(a), a.shape[1], _ptr(b), b.shape[1], a.shape[1], a.shape[0], _ptr(out))
    return out


def psnr_hvs_m_tables(height: int) -> np.ndarray:
    """(16 factors, 3 tables {csf, mask, inv_mask}, 8, 8) floats of psnr.cpp's per-factor set-up."""
    out = np.zeros(16 * 192, np.float32)
    lib().oracle_psnr_hvs_m_tables(height, _ptr(out))
    return out.reshape(16, 3, 8, 8)


def psnr_hvs_m_pixels(width: int, height: int) -> int:
    return int(lib().oracle_psnr_hvs_m_pixels(width, height))


def hvs_dct8(x) -> np.ndarray:
    a = np.ascontiguousarray(x, np.float32)
    out = np.zeros(8, np.float32)
    lib().oracle_hvs_dct8(_ptr(a), _ptr(out))
    return out


def psnr_hvs_m_db(errors: np.ndarray, pixels: int, full_range: bool = True) -> np.ndarray:
    """psnr.cpp:220-240: 10 log10(pixels * peak / error) per height factor."""
    peak = 1.0 if full_range else (223.0 * 223.0) / (255.0 * 255.0)
    e = np.ldexp(errors.astype(np.float64), -24)
    with np.errstate(divide="ignore"):
        return 10.0 * np.log10(pixels * peak / e)


def psnr(a: np.ndarray, b: np.ndarray) -> float:
    d = a.astype(np.float64) - b.astype(np.float64)
    mse = float(np.mean(d * d))
    if mse == 0:
        return float("inf")
    return 10.0 * np.log10(255.0 * 255.0 / mse)
