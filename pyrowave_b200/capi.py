"""ctypes binding of libpyrowave-shared.so.0 (include/pyrowave.h + include/pyrowave_cuda.h).

This is the Python-side mirror of the reference's C API: the same entry points,
argument meaning and result codes. Every call goes through the C ABI; there is
no other compute path. Loading fails loudly when the library is missing.
"""
from __future__ import annotations

import ctypes
import os
import weakref
from ctypes import (POINTER, Structure, c_bool, c_float, c_int, c_int32, c_size_t, c_uint8, c_uint16, c_uint32,
                    c_void_p)

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
LIB_PATH = os.path.join(HERE, "libpyrowave-shared.so.0")

PYROWAVE_SUCCESS = 0
PYROWAVE_TIMEOUT = 1
PYROWAVE_ERROR_GENERIC = -1
PYROWAVE_ERROR_INVALID_ARGUMENT = -2
PYROWAVE_ERROR_OUT_OF_HOST_MEMORY = -3
PYROWAVE_ERROR_OUT_OF_DEVICE_MEMORY = -4
PYROWAVE_ERROR_NO_VULKAN = -5
PYROWAVE_ERROR_NOT_IMPLEMENTED = -6

CHROMA_420 = 0
CHROMA_444 = 1

# Precision flag of pyrowave_cuda_*_set_precision: lifting staged through FP16
# as in the reference's precision 1; REFERENCE_PRECISION adds FP16 storage of
# levels 0-1, which together reproduce that precision.
PRECISION_STAGE16 = 0x100
REFERENCE_PRECISION = PRECISION_STAGE16 | 0x3

FORMAT_NV12 = 0
FORMAT_YUV420P = 1
FORMAT_YUV444P = 2
# 16-bit planar extensions (pyrowave_cuda.h): R16_UNORM samples.
FORMAT_YUV420P16 = 0x101
FORMAT_YUV444P16 = 0x102

# Every exported symbol of include/pyrowave.h and include/pyrowave_cuda.h.
API_SYMBOLS = [
    "pyrowave_get_api_version", "pyrowave_create_default_device", "pyrowave_create_device_by_compat",
    "pyrowave_create_device", "pyrowave_device_set_command_buffer", "pyrowave_device_report_performance_stats",
    "pyrowave_device_get_vk_device_handles", "pyrowave_device_confirm_interop_support",
    "pyrowave_device_set_queue_type", "pyrowave_device_destroy", "pyrowave_sync_object_create",
    "pyrowave_sync_object_get_semaphore", "pyrowave_sync_object_export_handle", "pyrowave_sync_object_cpu_wait",
    "pyrowave_sync_object_cpu_signal", "pyrowave_sync_object_destroy", "pyrowave_image_create",
    "pyrowave_image_get_handle", "pyrowave_image_get_image_view", "pyrowave_image_destroy",
    "pyrowave_encoder_create", "pyrowave_encoder_encode_gpu_synchronous", "pyrowave_encoder_encode_cpu_synchronous",
    "pyrowave_encoder_compute_num_packets", "pyrowave_encoder_packetize", "pyrowave_encoder_destroy",
    "pyrowave_decoder_device_prefers_fragment_path", "pyrowave_decoder_create", "pyrowave_decoder_clear",
    "pyrowave_decoder_push_packet", "pyrowave_decoder_decode_is_ready", "pyrowave_decoder_decode_gpu_buffer",
    "pyrowave_decoder_decode_cpu_buffer_synchronous", "pyrowave_decoder_destroy",
    # CUDA extension
    "pyrowave_cuda_device_set_stage_timing", "pyrowave_cuda_encoder_set_precision", "pyrowave_cuda_decoder_set_precision", "pyrowave_cuda_encoder_get_layout",
    "pyrowave_cuda_decoder_get_layout", "pyrowave_cuda_encoder_encode", "pyrowave_cuda_encoder_get_device_bitstream",
    "pyrowave_cuda_encoder_get_size", "pyrowave_cuda_encoder_encode_pre_transformed",
    "pyrowave_cuda_encoder_read_wavelet", "pyrowave_cuda_encoder_read_debug", "pyrowave_cuda_encoder_analyze_packing", "pyrowave_cuda_encoder_transform", "pyrowave_cuda_decoder_decode",
    "pyrowave_cuda_decoder_decode_blocks", "pyrowave_cuda_decoder_read_wavelet", "pyrowave_cuda_decoder_decode_pyramid",
    "pyrowave_cuda_decoder_decode_packets", "pyrowave_cuda_decoder_get_packet_status",
    "pyrowave_cuda_decoder_get_error", "pyrowave_cuda_decode_blocks_static",
    "pyrowave_cuda_psnr_hvs_m", "pyrowave_psnr_hvs_m_pixels", "pyrowave_psnr_hvs_m_from_errors",
    "pyrowave_cuda_encoder_encode16", "pyrowave_cuda_decoder_decode_blocks16",
    "pyrowave_cuda_batch_create", "pyrowave_cuda_batch_destroy", "pyrowave_cuda_batch_encode",
    "pyrowave_cuda_batch_get_device_bitstream", "pyrowave_cuda_batch_get_sizes", "pyrowave_cuda_batch_autotune",
    "pyrowave_cuda_batch_get_shape", "pyrowave_cuda_batch_set_shape",
    "pyrowave_cuda_server_create", "pyrowave_cuda_server_destroy", "pyrowave_cuda_server_open_stream",
    "pyrowave_cuda_server_close_stream", "pyrowave_cuda_server_submit", "pyrowave_cuda_server_poll",
    "pyrowave_cuda_server_stats", "pyrowave_cuda_server_get_memory",
]

# Coefficient storage limit of pyrowave_cuda_decode_blocks_static (PYROWAVE_CUDA_STATIC_DECODE_SCRATCH_BYTES).
STATIC_DECODE_SCRATCH_BYTES = 32 << 20


class PyrowaveError(RuntimeError):
    def __init__(self, what: str, code: int):
        super().__init__(f"{what} failed with pyrowave_result {code}")
        self.code = code


class EncoderCreateInfo(Structure):
    _fields_ = [("device", c_void_p), ("width", c_int), ("height", c_int), ("chroma", c_int)]


class DecoderCreateInfo(Structure):
    _fields_ = [("device", c_void_p), ("width", c_int), ("height", c_int), ("chroma", c_int), ("fragment_path", c_bool)]


class CpuBuffer(Structure):
    _fields_ = [("data", c_void_p * 3), ("row_stride_in_bytes", c_size_t * 3), ("plane_size_in_bytes", c_size_t * 3),
                ("width", c_int), ("height", c_int), ("format", c_int)]


class RateControl(Structure):
    _fields_ = [("maximum_bitstream_size", c_size_t)]


class Packet(Structure):
    _fields_ = [("offset", c_size_t), ("size", c_size_t)]


class PacketStatus(Structure):
    _fields_ = [("decoded_blocks", c_uint32), ("total_blocks", c_uint32), ("sequence", c_uint32),
                ("invalid_packets", c_uint32)]


class CudaPlanes(Structure):
    _fields_ = [("data", c_void_p * 3), ("row_stride_in_bytes", c_size_t * 3)]


class CudaLayout(Structure):
    _fields_ = [("width", c_int), ("height", c_int), ("chroma444", c_int), ("aligned_width", c_int),
                ("aligned_height", c_int), ("block_count_8x8", c_int), ("block_count_32x32", c_int),
                ("pyramid_size", c_size_t), ("fp16_level_mask", c_uint32)]


class CudaEncoderDebug(Structure):
    _fields_ = [("code_words", c_void_p), ("rd_cost", c_void_p), ("rd_bucket", c_void_p), ("rd_dist", c_void_p),
                ("histogram", c_void_p), ("consumed", c_void_p), ("quant", c_void_p), ("block_meta", c_void_p),
                ("error_flags", c_void_p)]


class PackingAnalysis(Structure):
    _fields_ = [("layout_bytes", ctypes.c_uint64 * 5), ("band_bytes", ctypes.c_uint64 * 60),
                ("coded_bytes", ctypes.c_uint64), ("significant", ctypes.c_uint64),
                ("plane_bytes", ctypes.c_uint64 * 16), ("plane_entropy", ctypes.c_double * 16),
                ("plane_histogram", c_uint32 * 4096)]


class BatchFrameInfo(Structure):
    _fields_ = [("width", ctypes.c_int), ("height", ctypes.c_int), ("chroma", ctypes.c_int),
                ("maximum_bitstream_size", c_size_t)]


class ServerInfo(Structure):
    _fields_ = [("memory_pool_bytes", c_size_t), ("max_in_flight", c_uint32)]


class ServerCompletion(Structure):
    _fields_ = [("request_id", ctypes.c_uint64), ("stream_id", c_uint32), ("result", c_int32), ("bytes", c_size_t),
                ("latency_us", ctypes.c_double)]


MESSAGE_CB = ctypes.CFUNCTYPE(None, c_void_p, ctypes.c_char_p)

_lib = None


def library_path() -> str:
    return LIB_PATH


def lib():
    """Load the C-ABI library. Raises if it has not been built."""
    global _lib
    if _lib is not None:
        return _lib
    if not os.path.exists(LIB_PATH):
        raise RuntimeError(
            f"{LIB_PATH} is missing: build it with `python -m pyrowave_b200.build` (there is no fallback path)")
    L = ctypes.CDLL(LIB_PATH)
    L.pyrowave_get_api_version.argtypes = [POINTER(c_uint32)] * 3
    L.pyrowave_get_api_version.restype = None
    L.pyrowave_create_default_device.argtypes = [POINTER(c_void_p)]
    L.pyrowave_device_destroy.argtypes = [c_void_p]
    L.pyrowave_device_destroy.restype = None
    L.pyrowave_device_report_performance_stats.argtypes = [c_void_p, MESSAGE_CB, c_void_p, c_bool]
    L.pyrowave_device_report_performance_stats.restype = None
    L.pyrowave_device_set_queue_type.argtypes = [c_void_p, c_int]
    L.pyrowave_device_confirm_interop_support.argtypes = [c_void_p]
    L.pyrowave_device_confirm_interop_support.restype = c_bool
    L.pyrowave_decoder_device_prefers_fragment_path.argtypes = [c_void_p]
    L.pyrowave_decoder_device_prefers_fragment_path.restype = c_bool
    L.pyrowave_encoder_create.argtypes = [POINTER(EncoderCreateInfo), POINTER(c_void_p)]
    L.pyrowave_encoder_destroy.argtypes = [c_void_p]
    L.pyrowave_encoder_destroy.restype = None
    L.pyrowave_encoder_encode_cpu_synchronous.argtypes = [c_void_p, POINTER(CpuBuffer), POINTER(RateControl)]
    L.pyrowave_encoder_encode_gpu_synchronous.argtypes = [c_void_p, c_void_p, c_void_p, c_void_p, POINTER(RateControl)]
    L.pyrowave_encoder_compute_num_packets.argtypes = [c_void_p, c_size_t, POINTER(c_size_t)]
    L.pyrowave_encoder_packetize.argtypes = [c_void_p, POINTER(Packet), c_size_t, POINTER(c_size_t), c_void_p, c_size_t]
    L.pyrowave_decoder_create.argtypes = [POINTER(DecoderCreateInfo), POINTER(c_void_p)]
    L.pyrowave_decoder_destroy.argtypes = [c_void_p]
    L.pyrowave_decoder_destroy.restype = None
    L.pyrowave_decoder_clear.argtypes = [c_void_p]
    L.pyrowave_decoder_clear.restype = None
    L.pyrowave_decoder_push_packet.argtypes = [c_void_p, c_void_p, c_size_t]
    L.pyrowave_decoder_decode_is_ready.argtypes = [c_void_p, c_bool]
    L.pyrowave_decoder_decode_is_ready.restype = c_bool
    L.pyrowave_decoder_decode_cpu_buffer_synchronous.argtypes = [c_void_p, POINTER(CpuBuffer)]
    L.pyrowave_decoder_decode_gpu_buffer.argtypes = [c_void_p, c_void_p, c_void_p, c_void_p]
    L.pyrowave_cuda_device_set_stage_timing.argtypes = [c_void_p, c_bool]
    L.pyrowave_cuda_encoder_set_precision.argtypes = [c_void_p, c_uint32]
    L.pyrowave_cuda_decoder_set_precision.argtypes = [c_void_p, c_uint32]
    L.pyrowave_cuda_encoder_get_layout.argtypes = [c_void_p, POINTER(CudaLayout)]
    L.pyrowave_cuda_decoder_get_layout.argtypes = [c_void_p, POINTER(CudaLayout)]
    L.pyrowave_cuda_encoder_encode.argtypes = [c_void_p, POINTER(CudaPlanes), POINTER(RateControl), c_void_p]
    L.pyrowave_cuda_encoder_get_device_bitstream.argtypes = [c_void_p, POINTER(c_void_p), POINTER(c_void_p),
                                                             POINTER(c_size_t)]
    L.pyrowave_cuda_encoder_get_size.argtypes = [c_void_p, POINTER(c_size_t)]
    L.pyrowave_cuda_encoder_encode_pre_transformed.argtypes = [c_void_p, c_void_p, POINTER(RateControl), c_float,
                                                               c_void_p]
    L.pyrowave_cuda_encoder_read_wavelet.argtypes = [c_void_p, c_void_p, c_void_p]
    L.pyrowave_cuda_encoder_transform.argtypes = [c_void_p, POINTER(CudaPlanes), c_void_p]
    L.pyrowave_cuda_encoder_read_debug.argtypes = [c_void_p, POINTER(CudaEncoderDebug)]
    L.pyrowave_cuda_encoder_analyze_packing.argtypes = [c_void_p, POINTER(PackingAnalysis)]
    L.pyrowave_cuda_decoder_decode.argtypes = [c_void_p, POINTER(CudaPlanes), c_void_p]
    L.pyrowave_cuda_decoder_decode_blocks.argtypes = [c_void_p, c_void_p, c_void_p, c_size_t, POINTER(CudaPlanes),
                                                      c_void_p]
    L.pyrowave_cuda_decoder_read_wavelet.argtypes = [c_void_p, c_void_p, c_void_p]
    L.pyrowave_cuda_decoder_decode_packets.argtypes = [c_void_p, c_void_p, c_size_t, c_void_p, c_uint32,
                                                       POINTER(CudaPlanes), c_void_p]
    L.pyrowave_cuda_decoder_get_packet_status.argtypes = [c_void_p, POINTER(PacketStatus)]
    L.pyrowave_cuda_decoder_get_error.argtypes = [c_void_p, POINTER(c_uint32)]
    L.pyrowave_cuda_encoder_encode16.argtypes = [c_void_p, POINTER(CudaPlanes), POINTER(RateControl), c_void_p]
    L.pyrowave_cuda_decoder_decode_blocks16.argtypes = [c_void_p, c_void_p, c_void_p, c_size_t, POINTER(CudaPlanes),
                                                        c_void_p]
    L.pyrowave_cuda_psnr_hvs_m.argtypes = [c_int, c_int, c_void_p, c_size_t, c_void_p, c_size_t, c_void_p, c_void_p]
    L.pyrowave_psnr_hvs_m_pixels.argtypes = [c_int, c_int]
    L.pyrowave_psnr_hvs_m_pixels.restype = ctypes.c_uint64
    L.pyrowave_psnr_hvs_m_from_errors.argtypes = [c_void_p, ctypes.c_uint64, c_bool, c_void_p]
    L.pyrowave_psnr_hvs_m_from_errors.restype = None
    L.pyrowave_cuda_decoder_decode_pyramid.argtypes = [c_void_p, c_void_p, POINTER(CudaPlanes), c_void_p]
    L.pyrowave_cuda_decode_blocks_static.argtypes = [ctypes.c_int, ctypes.c_int, ctypes.c_int, c_void_p, c_void_p,
                                                     c_size_t, POINTER(CudaPlanes), c_void_p]
    L.pyrowave_cuda_batch_create.argtypes = [c_void_p, POINTER(BatchFrameInfo), c_uint32, POINTER(c_void_p)]
    L.pyrowave_cuda_batch_destroy.argtypes = [c_void_p]
    L.pyrowave_cuda_batch_destroy.restype = None
    L.pyrowave_cuda_batch_encode.argtypes = [c_void_p, POINTER(CudaPlanes), POINTER(c_size_t), POINTER(CudaPlanes),
                                             c_void_p]
    L.pyrowave_cuda_batch_get_device_bitstream.argtypes = [c_void_p, c_uint32, POINTER(c_void_p), POINTER(c_void_p)]
    L.pyrowave_cuda_batch_get_sizes.argtypes = [c_void_p, POINTER(c_size_t)]
    L.pyrowave_cuda_batch_autotune.argtypes = [c_void_p, POINTER(CudaPlanes), POINTER(c_size_t), POINTER(CudaPlanes),
                                               c_void_p]
    L.pyrowave_cuda_batch_get_shape.argtypes = [c_void_p, c_void_p]
    L.pyrowave_cuda_batch_set_shape.argtypes = [c_void_p, c_void_p, c_void_p]
    L.pyrowave_cuda_server_create.argtypes = [c_void_p, POINTER(ServerInfo), POINTER(c_void_p)]
    L.pyrowave_cuda_server_destroy.argtypes = [c_void_p]
    L.pyrowave_cuda_server_destroy.restype = None
    L.pyrowave_cuda_server_open_stream.argtypes = [c_void_p, c_int, c_int, c_int, c_size_t, POINTER(c_uint32)]
    L.pyrowave_cuda_server_close_stream.argtypes = [c_void_p, c_uint32]
    L.pyrowave_cuda_server_submit.argtypes = [c_void_p, c_uint32, POINTER(CudaPlanes), c_size_t, POINTER(CudaPlanes),
                                              POINTER(ctypes.c_uint64)]
    L.pyrowave_cuda_server_poll.argtypes = [c_void_p, POINTER(ServerCompletion), c_uint32, POINTER(c_uint32),
                                            c_uint32]
    L.pyrowave_cuda_server_stats.argtypes = [c_void_p, POINTER(ctypes.c_double), POINTER(ctypes.c_double),
                                             POINTER(ctypes.c_uint64), c_bool]
    L.pyrowave_cuda_server_get_memory.argtypes = [c_void_p, POINTER(c_size_t), POINTER(c_size_t),
                                                  POINTER(ctypes.c_uint64)]
    for name in API_SYMBOLS:
        getattr(L, name)  # every declared entry point must resolve
    _lib = L
    return L


def check(code: int, what: str):
    if code != PYROWAVE_SUCCESS:
        raise PyrowaveError(what, code)


def api_version():
    L = lib()
    a, b, c = c_uint32(), c_uint32(), c_uint32()
    L.pyrowave_get_api_version(ctypes.byref(a), ctypes.byref(b), ctypes.byref(c))
    return a.value, b.value, c.value


def _ptr(a):
    return ctypes.c_void_p(a.ctypes.data)


class Device:
    """pyrowave_device: binds the current CUDA device."""

    def __init__(self):
        self.L = lib()
        h = c_void_p()
        check(self.L.pyrowave_create_default_device(ctypes.byref(h)), "pyrowave_create_default_device")
        self.h = h
        self._children = weakref.WeakSet()

    def adopt(self, child):
        """Encoders, decoders and batches made on this device: closed before it."""
        self._children.add(child)

    def close(self):
        if self.h:
            # The C API requires every object of a device to be destroyed first.
            for child in list(self._children):
                child.close()
            self.L.pyrowave_device_destroy(self.h)
            self.h = None

    def __del__(self):
        self.close()

    def set_stage_timing(self, enable: bool):
        check(self.L.pyrowave_cuda_device_set_stage_timing(self.h, enable), "set_stage_timing")

    def report_performance_stats(self, reset: bool = True):
        out = []
        cb = MESSAGE_CB(lambda ud, msg: out.append(msg.decode()))
        self.L.pyrowave_device_report_performance_stats(self.h, cb, None, reset)
        return out


def _plane_shapes(width, height, chroma):
    if chroma == CHROMA_444:
        return [(height, width)] * 3
    return [(height, width), (height // 2, width // 2), (height // 2, width // 2)]


def cpu_buffer(planes, width, height, fmt):
    buf = CpuBuffer()
    keep = []
    for i, p in enumerate(planes):
        if p is None:
            continue
        a = np.ascontiguousarray(p) if not p.flags.c_contiguous else p
        keep.append(a)
        buf.data[i] = a.ctypes.data
        buf.row_stride_in_bytes[i] = a.strides[0]
        buf.plane_size_in_bytes[i] = a.strides[0] * a.shape[0]
    buf.width = width
    buf.height = height
    buf.format = fmt
    return buf, keep


class Encoder:
    """pyrowave_encoder (reference pyrowave.h:442-481)."""

    def __init__(self, device: Device, width: int, height: int, chroma: int = CHROMA_420, fp16_level_mask: int = 0):
        self.L = lib()
        self.device = device
        device.adopt(self)
        info = EncoderCreateInfo(device.h, width, height, chroma)
        h = c_void_p()
        check(self.L.pyrowave_encoder_create(ctypes.byref(info), ctypes.byref(h)), "pyrowave_encoder_create")
        self.h = h
        self.width, self.height, self.chroma = width, height, chroma
        if fp16_level_mask:
            check(self.L.pyrowave_cuda_encoder_set_precision(self.h, fp16_level_mask), "set_precision")

    def close(self):
        if self.h:
            self.L.pyrowave_encoder_destroy(self.h)
            self.h = None

    def __del__(self):
        self.close()

    def layout(self) -> CudaLayout:
        lay = CudaLayout()
        check(self.L.pyrowave_cuda_encoder_get_layout(self.h, ctypes.byref(lay)), "get_layout")
        return lay

    def encode_cpu(self, planes, budget: int, fmt: int | None = None) -> int:
        if fmt is None:
            wide = np.asarray(planes[0]).dtype == np.uint16
            if self.chroma == CHROMA_444:
                fmt = FORMAT_YUV444P16 if wide else FORMAT_YUV444P
            else:
                fmt = FORMAT_YUV420P16 if wide else FORMAT_YUV420P
        buf, keep = cpu_buffer(planes, self.width, self.height, fmt)
        rc = RateControl(budget)
        return self.L.pyrowave_encoder_encode_cpu_synchronous(self.h, ctypes.byref(buf), ctypes.byref(rc))

    def compute_num_packets(self, boundary: int) -> int:
        n = c_size_t()
        check(self.L.pyrowave_encoder_compute_num_packets(self.h, boundary, ctypes.byref(n)), "compute_num_packets")
        return n.value

    def packetize(self, boundary: int, size: int):
        n = self.compute_num_packets(boundary)
        packets = (Packet * max(n, 1))()
        out = np.zeros(size, np.uint8)
        got = c_size_t()
        check(self.L.pyrowave_encoder_packetize(self.h, packets, boundary, ctypes.byref(got), _ptr(out), size),
              "packetize")
        return out, [(packets[i].offset, packets[i].size) for i in range(got.value)]

    # --- CUDA extension --------------------------------------------------------
    def encode_device(self, plane_ptrs, strides, budget: int, stream: int = 0):
        cp = CudaPlanes()
        for i in range(3):
            cp.data[i] = plane_ptrs[i]
            cp.row_stride_in_bytes[i] = strides[i]
        rc = RateControl(budget)
        check(self.L.pyrowave_cuda_encoder_encode(self.h, ctypes.byref(cp), ctypes.byref(rc), c_void_p(stream)),
              "pyrowave_cuda_encoder_encode")

    def encode_device16(self, plane_ptrs, strides, budget: int, stream: int = 0):
        """pyrowave_cuda_encoder_encode16: 16-bit (R16_UNORM) device planes; strides in bytes."""
        cp = CudaPlanes()
        for i in range(3):
            cp.data[i] = plane_ptrs[i]
            cp.row_stride_in_bytes[i] = strides[i]
        rc = RateControl(budget)
        check(self.L.pyrowave_cuda_encoder_encode16(self.h, ctypes.byref(cp), ctypes.byref(rc), c_void_p(stream)),
              "pyrowave_cuda_encoder_encode16")

    def transform(self, plane_ptrs, strides, stream: int = 0):
        """pyrowave_cuda_encoder_transform: the five forward levels alone (no quantiser)."""
        cp = CudaPlanes()
        for i in range(3):
            cp.data[i] = plane_ptrs[i]
            cp.row_stride_in_bytes[i] = strides[i]
        check(self.L.pyrowave_cuda_encoder_transform(self.h, ctypes.byref(cp), c_void_p(stream)),
              "pyrowave_cuda_encoder_transform")

    def encode_pre_transformed(self, pyramid_dev_ptr: int, budget: int, quant_scale: float = -1.0, stream: int = 0):
        rc = RateControl(budget)
        check(self.L.pyrowave_cuda_encoder_encode_pre_transformed(self.h, c_void_p(pyramid_dev_ptr), ctypes.byref(rc),
                                                                  quant_scale, c_void_p(stream)),
              "encode_pre_transformed")

    def read_wavelet(self, pyramid_dev_ptr: int, stream: int = 0):
        check(self.L.pyrowave_cuda_encoder_read_wavelet(self.h, c_void_p(pyramid_dev_ptr), c_void_p(stream)),
              "read_wavelet")

    def device_bitstream(self):
        s, m, cap = c_void_p(), c_void_p(), c_size_t()
        check(self.L.pyrowave_cuda_encoder_get_device_bitstream(self.h, ctypes.byref(s), ctypes.byref(m),
                                                                ctypes.byref(cap)), "get_device_bitstream")
        return s.value, m.value, cap.value

    def size(self) -> int:
        n = c_size_t()
        check(self.L.pyrowave_cuda_encoder_get_size(self.h, ctypes.byref(n)), "get_size")
        return n.value

    def debug(self):
        lay = self.layout()
        n8, n32 = lay.block_count_8x8, lay.block_count_32x32
        d = {
            "code_words": np.zeros(n8, np.uint32),
            "rd_cost": np.zeros((n32, 16), np.uint16),
            "rd_bucket": np.zeros((n32, 16), np.uint8),
            "rd_dist": np.zeros((n32, 16), np.float32),
            "histogram": np.zeros(2048, np.uint32),
            "consumed": np.zeros(1, np.uint32),
            "quant": np.zeros(n32, np.int32),
            "block_meta": np.zeros((n32, 2), np.uint32),
            "error_flags": np.zeros(1, np.uint32),
        }
        dbg = CudaEncoderDebug(*[d[k].ctypes.data for k in ("code_words", "rd_cost", "rd_bucket", "rd_dist", "histogram",
                                                            "consumed", "quant", "block_meta", "error_flags")])
        check(self.L.pyrowave_cuda_encoder_read_debug(self.h, ctypes.byref(dbg)), "read_debug")
        return d

    def analyze_packing(self) -> dict:
        """Packing statistics of the last encode (pyrowave_cuda_encoder_analyze_packing)."""
        a = PackingAnalysis()
        check(self.L.pyrowave_cuda_encoder_analyze_packing(self.h, ctypes.byref(a)), "analyze_packing")
        return {
            "layout_bytes": np.ctypeslib.as_array(a.layout_bytes).copy(),
            "band_bytes": np.ctypeslib.as_array(a.band_bytes).reshape(3, 5, 4).copy(),
            "coded_bytes": int(a.coded_bytes),
            "significant": int(a.significant),
            "plane_bytes": np.ctypeslib.as_array(a.plane_bytes).copy(),
            "plane_entropy": np.ctypeslib.as_array(a.plane_entropy).copy(),
            "plane_histogram": np.ctypeslib.as_array(a.plane_histogram).reshape(16, 256).copy(),
        }


class Decoder:
    """pyrowave_decoder (reference pyrowave.h:485-539)."""

    def __init__(self, device: Device, width: int, height: int, chroma: int = CHROMA_420, fp16_level_mask: int = 0):
        self.L = lib()
        self.device = device
        device.adopt(self)
        info = DecoderCreateInfo(device.h, width, height, chroma, False)
        h = c_void_p()
        check(self.L.pyrowave_decoder_create(ctypes.byref(info), ctypes.byref(h)), "pyrowave_decoder_create")
        self.h = h
        self.width, self.height, self.chroma = width, height, chroma
        if fp16_level_mask:
            check(self.L.pyrowave_cuda_decoder_set_precision(self.h, fp16_level_mask), "set_precision")

    def close(self):
        if self.h:
            self.L.pyrowave_decoder_destroy(self.h)
            self.h = None

    def __del__(self):
        self.close()

    def layout(self) -> CudaLayout:
        lay = CudaLayout()
        check(self.L.pyrowave_cuda_decoder_get_layout(self.h, ctypes.byref(lay)), "get_layout")
        return lay

    def clear(self):
        self.L.pyrowave_decoder_clear(self.h)

    def push_packet(self, data) -> int:
        buf = np.frombuffer(bytes(data), np.uint8) if not isinstance(data, np.ndarray) else np.ascontiguousarray(data)
        if buf.size == 0:
            return self.L.pyrowave_decoder_push_packet(self.h, None, 0)
        return self.L.pyrowave_decoder_push_packet(self.h, _ptr(buf), buf.size)

    def push_packet_ptr(self, ptr: int, size: int) -> int:
        """pyrowave_decoder_push_packet on `size` bytes at host address `ptr` (no copy in Python)."""
        return self.L.pyrowave_decoder_push_packet(self.h, c_void_p(ptr), size)

    def is_ready(self, allow_partial: bool = False) -> bool:
        return bool(self.L.pyrowave_decoder_decode_is_ready(self.h, allow_partial))

    def decode_cpu(self, planes=None, fmt: int | None = None, wide: bool = False):
        """Synchronous decode into host planes (uint16 planes, or wide=True: 16-bit output)."""
        if planes is not None:
            wide = np.asarray(planes[0]).dtype == np.uint16
        if fmt is None:
            if self.chroma == CHROMA_444:
                fmt = FORMAT_YUV444P16 if wide else FORMAT_YUV444P
            else:
                fmt = FORMAT_YUV420P16 if wide else FORMAT_YUV420P
        if planes is None:
            planes = [np.zeros(s, np.uint16 if wide else np.uint8)
                      for s in _plane_shapes(self.width, self.height, self.chroma)]
        buf, keep = cpu_buffer(planes, self.width, self.height, fmt)
        code = self.L.pyrowave_decoder_decode_cpu_buffer_synchronous(self.h, ctypes.byref(buf))
        return code, planes

    def decode_device(self, plane_ptrs, strides, stream: int = 0):
        cp = CudaPlanes()
        for i in range(3):
            cp.data[i] = plane_ptrs[i]
            cp.row_stride_in_bytes[i] = strides[i]
        check(self.L.pyrowave_cuda_decoder_decode(self.h, ctypes.byref(cp), c_void_p(stream)), "cuda_decoder_decode")

    def decode_blocks(self, meta_ptr: int, words_ptr: int, num_words: int, plane_ptrs, strides, stream: int = 0):
        cp = CudaPlanes()
        for i in range(3):
            cp.data[i] = plane_ptrs[i]
            cp.row_stride_in_bytes[i] = strides[i]
        check(self.L.pyrowave_cuda_decoder_decode_blocks(self.h, c_void_p(meta_ptr), c_void_p(words_ptr), num_words,
                                                         ctypes.byref(cp), c_void_p(stream)), "decode_blocks")

    def decode_blocks16(self, meta_ptr: int, words_ptr: int, num_words: int, plane_ptrs, strides, stream: int = 0):
        """pyrowave_cuda_decoder_decode_blocks16: into 16-bit device planes; strides in bytes."""
        cp = CudaPlanes()
        for i in range(3):
            cp.data[i] = plane_ptrs[i]
            cp.row_stride_in_bytes[i] = strides[i]
        check(self.L.pyrowave_cuda_decoder_decode_blocks16(self.h, c_void_p(meta_ptr), c_void_p(words_ptr),
                                                           num_words, ctypes.byref(cp), c_void_p(stream)),
              "decode_blocks16")

    def decode_packets(self, data_ptr: int, data_size: int, packets_ptr: int, count: int, plane_ptrs, strides,
                       stream: int = 0) -> int:
        """pyrowave_cuda_decoder_decode_packets: assemble a frame from device-resident packets
        ({offset, size} u64 pairs at packets_ptr) on the GPU and decode it. Returns the result code."""
        cp = CudaPlanes()
        for i in range(3):
            cp.data[i] = plane_ptrs[i]
            cp.row_stride_in_bytes[i] = strides[i]
        return self.L.pyrowave_cuda_decoder_decode_packets(self.h, c_void_p(data_ptr), data_size, c_void_p(packets_ptr),
                                                           count, ctypes.byref(cp), c_void_p(stream))

    def error(self):
        """pyrowave_cuda_decoder_get_error: (result code, error bits) of the last decode (waits for it)."""
        bits = c_uint32(0)
        code = self.L.pyrowave_cuda_decoder_get_error(self.h, ctypes.byref(bits))
        return code, int(bits.value)

    def packet_status(self) -> PacketStatus:
        st = PacketStatus()
        check(self.L.pyrowave_cuda_decoder_get_packet_status(self.h, ctypes.byref(st)), "get_packet_status")
        return st

    def decode_pyramid(self, pyramid_ptr: int, plane_ptrs, strides, stream: int = 0):
        cp = CudaPlanes()
        for i in range(3):
            cp.data[i] = plane_ptrs[i]
            cp.row_stride_in_bytes[i] = strides[i]
        check(self.L.pyrowave_cuda_decoder_decode_pyramid(self.h, c_void_p(pyramid_ptr), ctypes.byref(cp),
                                                          c_void_p(stream)), "decode_pyramid")

    def read_wavelet(self, pyramid_dev_ptr: int, stream: int = 0):
        check(self.L.pyrowave_cuda_decoder_read_wavelet(self.h, c_void_p(pyramid_dev_ptr), c_void_p(stream)),
              "decoder_read_wavelet")


def psnr_hvs_m(width: int, height: int, ref_ptr: int, ref_stride: int, dist_ptr: int, dist_stride: int,
               errors_ptr: int, stream: int = 0) -> int:
    """pyrowave_cuda_psnr_hvs_m: add the 16 fixed-point error sums into the device array at errors_ptr."""
    return lib().pyrowave_cuda_psnr_hvs_m(width, height, c_void_p(ref_ptr), ref_stride, c_void_p(dist_ptr),
                                          dist_stride, c_void_p(errors_ptr), c_void_p(stream))


def psnr_hvs_m_db(errors, pixels: int, full_range: bool = True) -> np.ndarray:
    """pyrowave_psnr_hvs_m_from_errors on host copies of the sums."""
    e = np.ascontiguousarray(errors, np.uint64)
    out = np.zeros(16, np.float64)
    lib().pyrowave_psnr_hvs_m_from_errors(_ptr(e), pixels, full_range, _ptr(out))
    return out


def decode_blocks_static(width: int, height: int, chroma: int, meta_ptr: int, words_ptr: int, num_words: int,
                         plane_ptrs, strides, stream: int = 0) -> int:
    """pyrowave_cuda_decode_blocks_static: decode device-resident blocks with no decoder object and no
    allocation. Returns the pyrowave_result code."""
    cp = CudaPlanes()
    for i in range(3):
        cp.data[i] = plane_ptrs[i]
        cp.row_stride_in_bytes[i] = strides[i]
    return lib().pyrowave_cuda_decode_blocks_static(width, height, chroma, c_void_p(meta_ptr), c_void_p(words_ptr),
                                                    num_words, ctypes.byref(cp), c_void_p(stream))


def _planes_array(plane_ptr_lists, stride_lists):
    arr = (CudaPlanes * len(plane_ptr_lists))()
    for i, (ptrs, strides) in enumerate(zip(plane_ptr_lists, stride_lists)):
        for p in range(3):
            arr[i].data[p] = ptrs[p]
            arr[i].row_stride_in_bytes[p] = strides[p]
    return arr


class Batch:
    """pyrowave_cuda_batch: many frames of any sizes through one graph launch per call."""

    def __init__(self, device: Device, frames):
        """frames: list of (width, height, chroma, maximum_bitstream_size)."""
        self.L = lib()
        self.device = device
        device.adopt(self)
        infos = (BatchFrameInfo * len(frames))(*[BatchFrameInfo(w, h, c, m) for w, h, c, m in frames])
        h = c_void_p()
        check(self.L.pyrowave_cuda_batch_create(device.h, infos, len(frames), ctypes.byref(h)), "batch_create")
        self.h = h
        self.count = len(frames)

    def close(self):
        if self.h:
            self.L.pyrowave_cuda_batch_destroy(self.h)
            self.h = None

    def __del__(self):
        self.close()

    def _args(self, inputs, input_strides, budgets, outputs, output_strides):
        ins = _planes_array(inputs, input_strides)
        outs = _planes_array(outputs, output_strides) if outputs is not None else None
        b = (c_size_t * self.count)(*budgets)
        return ins, b, outs

    def encode(self, inputs, input_strides, budgets, outputs=None, output_strides=None, stream: int = 0) -> int:
        ins, b, outs = self._args(inputs, input_strides, budgets, outputs, output_strides)
        return self.L.pyrowave_cuda_batch_encode(self.h, ins, b, outs, c_void_p(stream))

    def autotune(self, inputs, input_strides, budgets, outputs=None, output_strides=None, stream: int = 0) -> int:
        ins, b, outs = self._args(inputs, input_strides, budgets, outputs, output_strides)
        return self.L.pyrowave_cuda_batch_autotune(self.h, ins, b, outs, c_void_p(stream))

    def device_bitstream(self, index: int):
        s, m = c_void_p(), c_void_p()
        check(self.L.pyrowave_cuda_batch_get_device_bitstream(self.h, index, ctypes.byref(s), ctypes.byref(m)),
              "batch_get_device_bitstream")
        return s.value, m.value

    def sizes(self):
        out = (c_size_t * self.count)()
        check(self.L.pyrowave_cuda_batch_get_sizes(self.h, out), "batch_get_sizes")
        return list(out)

    def shape(self) -> dict:
        sh = BatchShape()
        check(self.L.pyrowave_cuda_batch_get_shape(self.h, ctypes.byref(sh)), "batch_get_shape")
        return {k: int(getattr(sh, k)) for k, _ in BatchShape._fields_}

    def set_shape(self, persistent=True, small_level=5, large_below=0, ctas_per_sm=0, large_first=False,
                  branches=1, frame_graphs=False, stream: int = 0):
        sh = BatchShape(int(persistent), small_level, large_below, ctas_per_sm, int(large_first), branches,
                        int(frame_graphs))
        check(self.L.pyrowave_cuda_batch_set_shape(self.h, ctypes.byref(sh), c_void_p(stream)), "batch_set_shape")


class BatchShape(Structure):
    _fields_ = [("persistent", c_uint32), ("small_level", c_int32), ("large_below", c_int32),
                ("ctas_per_sm", c_int32), ("large_first", c_uint32), ("branches", c_uint32),
                ("frame_graphs", c_uint32)]


class Server:
    """pyrowave_cuda_server: continuous batching of encode + decode requests from many streams."""

    def __init__(self, device: Device, memory_pool_bytes: int, max_in_flight: int = 8):
        self.L = lib()
        self.device = device
        device.adopt(self)
        info = ServerInfo(memory_pool_bytes, max_in_flight)
        h = c_void_p()
        check(self.L.pyrowave_cuda_server_create(device.h, ctypes.byref(info), ctypes.byref(h)), "server_create")
        self.h = h

    def close(self):
        if self.h:
            self.L.pyrowave_cuda_server_destroy(self.h)
            self.h = None

    def __del__(self):
        self.close()

    def open_stream(self, width: int, height: int, chroma: int, maximum_bitstream_size: int):
        """Returns (result code, stream id)."""
        sid = c_uint32()
        code = self.L.pyrowave_cuda_server_open_stream(self.h, width, height, chroma, maximum_bitstream_size,
                                                       ctypes.byref(sid))
        return code, sid.value

    def close_stream(self, stream_id: int) -> int:
        return self.L.pyrowave_cuda_server_close_stream(self.h, stream_id)

    def submit(self, stream_id: int, in_ptrs, in_strides, budget: int, out_ptrs=None, out_strides=None):
        ins = _planes_array([in_ptrs], [in_strides])
        outs = _planes_array([out_ptrs], [out_strides]) if out_ptrs is not None else None
        rid = ctypes.c_uint64()
        check(self.L.pyrowave_cuda_server_submit(self.h, stream_id, ins, budget, outs, ctypes.byref(rid)),
              "server_submit")
        return rid.value

    def poll(self, capacity: int = 256, timeout_us: int = 0):
        arr = (ServerCompletion * capacity)()
        n = c_uint32()
        check(self.L.pyrowave_cuda_server_poll(self.h, arr, capacity, ctypes.byref(n), timeout_us), "server_poll")
        return [(arr[i].request_id, arr[i].stream_id, arr[i].result, arr[i].bytes, arr[i].latency_us)
                for i in range(n.value)]

    def memory(self):
        """(pool bytes in use, peak, working sets released to admit other streams' frames)."""
        used, peak, rel = c_size_t(), c_size_t(), ctypes.c_uint64()
        check(self.L.pyrowave_cuda_server_get_memory(self.h, ctypes.byref(used), ctypes.byref(peak),
                                                     ctypes.byref(rel)), "server_get_memory")
        return used.value, peak.value, rel.value

    def stats(self, reset: bool = False):
        p50, p99, frames = ctypes.c_double(), ctypes.c_double(), ctypes.c_uint64()
        check(self.L.pyrowave_cuda_server_stats(self.h, ctypes.byref(p50), ctypes.byref(p99), ctypes.byref(frames),
                                                reset), "server_stats")
        return p50.value, p99.value, frames.value
