/*
 * PyroWave CUDA extension API (B200 implementation only).
 *
 * The reference exposes its GPU path through Vulkan images and semaphores
 * (pyrowave.h:457-462, :528-532 of the reference). On B200 the same role is
 * played by CUDA device pointers and a CUDA stream: these entry points encode
 * from and decode to device memory, ordered on the caller's stream, with no
 * host round trip. All types are plain C; the stream is a cudaStream_t.
 *
 * Also declared here are the introspection entry points the parity tests use:
 * encoding a caller-provided wavelet pyramid (the reference's
 * Encoder::encode_pre_transformed, pyrowave_encoder.hpp:44-47) and reading the
 * pyramid and the rate-control decisions back.
 */
#ifndef PYROWAVE_CUDA_H_
#define PYROWAVE_CUDA_H_

#include "pyrowave.h"

#ifdef __cplusplus
extern "C" {
#endif

typedef struct CUstream_st *pyrowave_cuda_stream; /* cudaStream_t */

/* Three 8-bit planes in device memory. For 4:2:0 the chroma planes are
 * (width/2) x (height/2). */
typedef struct pyrowave_cuda_planes
{
	void *data[3];
	size_t row_stride_in_bytes[3];
} pyrowave_cuda_planes;

typedef struct pyrowave_cuda_layout
{
	int width, height, chroma444;
	int aligned_width, aligned_height;
	int block_count_8x8, block_count_32x32;
	size_t pyramid_size;       /* coefficients of all transmitted bands (canonical layout) */
	uint32_t fp16_level_mask;  /* bit L set: level L coefficients stored as FP16 */
} pyrowave_cuda_layout;

/* Per-kernel GPU timing with CUDA events recorded on the launching stream
 * ("dwt0".."dwt4", "resolve", "pack", "dequant", "idwt4".."idwt0"), reported
 * through pyrowave_device_report_performance_stats. Off by default (also
 * enabled by the environment variable PYROWAVE_STAGE_TIMING=1). */
PYROWAVE_PUBLIC_API pyrowave_result pyrowave_cuda_device_set_stage_timing(pyrowave_device device, bool enable);

/* Coefficient storage precision per decomposition level. Default 0 (FP32 at
 * every level); 0x3 matches the reference's default precision layout (FP16 for
 * levels 0-1). Must be called before the first encode / decode.
 * PYROWAVE_CUDA_PRECISION_STAGE16 added to the mask also rounds every lifting
 * input and output to FP16, as the reference's precision 1 stages its shared
 * memory in FP16 (dwt_common.h:45-47); 0x3 | STAGE16 reproduces that precision
 * (pyrowave_common.cpp:133-157). Encoder and decoder of one stream should agree. */
#define PYROWAVE_CUDA_PRECISION_STAGE16 0x100u
PYROWAVE_PUBLIC_API pyrowave_result pyrowave_cuda_encoder_set_precision(pyrowave_encoder encoder, uint32_t fp16_level_mask);
PYROWAVE_PUBLIC_API pyrowave_result pyrowave_cuda_decoder_set_precision(pyrowave_decoder decoder, uint32_t fp16_level_mask);

PYROWAVE_PUBLIC_API pyrowave_result pyrowave_cuda_encoder_get_layout(pyrowave_encoder encoder, pyrowave_cuda_layout *layout);
PYROWAVE_PUBLIC_API pyrowave_result pyrowave_cuda_decoder_get_layout(pyrowave_decoder decoder, pyrowave_cuda_layout *layout);

/* 16-bit planes (R16_UNORM samples, little-endian uint16: the reference's
 * high bit depth input and output, encode.cpp:152 and decode.cpp:215 of the
 * reference) for pyrowave_encoder_encode_cpu_synchronous and
 * pyrowave_decoder_decode_cpu_buffer_synchronous: row strides and plane sizes
 * in bytes, as for the 8-bit formats. These values extend the reference's
 * pyrowave_cpu_buffer_format, which has no 16-bit planar formats. */
#define PYROWAVE_CPU_BUFFER_FORMAT_YUV420P16 ((pyrowave_cpu_buffer_format)0x101)
#define PYROWAVE_CPU_BUFFER_FORMAT_YUV444P16 ((pyrowave_cpu_buffer_format)0x102)

/* Encode device planes on `stream`; returns without waiting. The packetized
 * frame (8-byte start-of-frame header followed by the coded 32x32 blocks in
 * block index order, exactly what pyrowave_encoder_packetize emits with an
 * unbounded packet size) stays in device memory until the next encode. */
PYROWAVE_PUBLIC_API pyrowave_result pyrowave_cuda_encoder_encode(pyrowave_encoder encoder,
                                                                 const pyrowave_cuda_planes *planes,
                                                                 const pyrowave_rate_control *rate_control,
                                                                 pyrowave_cuda_stream stream);

/* As pyrowave_cuda_encoder_encode, from 16-bit planes (R16_UNORM samples, each
 * row_stride_in_bytes a multiple of 2 and at least 2 * width). */
PYROWAVE_PUBLIC_API pyrowave_result pyrowave_cuda_encoder_encode16(pyrowave_encoder encoder,
                                                                   const pyrowave_cuda_planes *planes,
                                                                   const pyrowave_rate_control *rate_control,
                                                                   pyrowave_cuda_stream stream);

/* Device view of the last encode: stream = packetized frame (words), block_meta
 * = {offset_u32, num_words} per 32x32 block (the reference's BitstreamPacket
 * table, offsets relative to stream + 2). Valid once `stream` work completes. */
PYROWAVE_PUBLIC_API pyrowave_result pyrowave_cuda_encoder_get_device_bitstream(pyrowave_encoder encoder,
                                                                               const uint32_t **stream,
                                                                               const uint32_t **block_meta,
                                                                               size_t *capacity_words);

/* Bytes of the last packetized frame (waits for the encode). */
PYROWAVE_PUBLIC_API pyrowave_result pyrowave_cuda_encoder_get_size(pyrowave_encoder encoder, size_t *bytes);

/* Encode a wavelet pyramid given in device memory in the canonical layout
 * (transmitted bands in block-index order, each band row-major and unpadded).
 * quant_scale < 0 uses the per-band resolutions; >= 0 overrides them
 * (reference pyrowave_encoder.cpp:449,251). */
PYROWAVE_PUBLIC_API pyrowave_result pyrowave_cuda_encoder_encode_pre_transformed(pyrowave_encoder encoder,
                                                                                 const float *pyramid,
                                                                                 const pyrowave_rate_control *rate_control,
                                                                                 float quant_scale,
                                                                                 pyrowave_cuda_stream stream);

/* The forward transform alone: the five CDF 9/7 levels of `planes` into the
 * encoder's pyramid (read back with pyrowave_cuda_encoder_read_wavelet), with
 * no quantiser, rate control or packing: the reference's DWT stage
 * (pyrowave_encoder.cpp:490-594) by itself, for measuring it apart from the
 * quantiser the encoder fuses into its large levels. With stage timing on, the
 * levels report as "xdwt0".."xdwt4". Queued on `stream`; does not wait. */
PYROWAVE_PUBLIC_API pyrowave_result pyrowave_cuda_encoder_transform(pyrowave_encoder encoder,
                                                                   const pyrowave_cuda_planes *planes,
                                                                   pyrowave_cuda_stream stream);

/* Copy the last encode's wavelet pyramid (canonical layout, device memory). */
PYROWAVE_PUBLIC_API pyrowave_result pyrowave_cuda_encoder_read_wavelet(pyrowave_encoder encoder, float *pyramid,
                                                                       pyrowave_cuda_stream stream);

/* Host copies of the last encode's decisions (waits). Any pointer may be NULL.
 * code_words: per 8x8; rd_cost/rd_bucket/rd_dist: 16 per 32x32; histogram: 2048
 * savings counters (not scanned); quant: per 32x32; block_meta: 2 per 32x32. */
typedef struct pyrowave_cuda_encoder_debug
{
	uint32_t *code_words;
	uint16_t *rd_cost;
	uint8_t *rd_bucket;
	float *rd_dist;
	uint32_t *histogram;
	uint32_t *consumed;
	int32_t *quant;
	uint32_t *block_meta;
	uint32_t *error_flags;
} pyrowave_cuda_encoder_debug;

PYROWAVE_PUBLIC_API pyrowave_result pyrowave_cuda_encoder_read_debug(pyrowave_encoder encoder,
                                                                     const pyrowave_cuda_encoder_debug *debug);

/* Packing statistics of the last encode, computed on the device (waits for the
 * encode, then for its own kernel). The reference keeps this analysis as
 * disabled code (pyrowave_encoder.cpp:625-958, Encoder::Impl::report_stats and
 * analyze_alternative_packing); here it covers the current block format:
 *   layout_bytes: estimated bytes of the frame's coded bands packed as 32x32
 *     packets with 2x2, 4x2 (the current shape) and 2x4 sub-blocks, 64x32
 *     packets with 4x4 and 64x64 packets with 8x4 sub-blocks (the reference's
 *     analyze_cost over 64x64 regions of the quantised integers);
 *   band_bytes: coded bytes (block words x 4) per component, level and band;
 *     coded_bytes their sum (the frame minus its 8-byte sequence header);
 *   significant: nonzero coefficients (one sign bit each);
 *   plane_histogram[j]: the plane bytes at position j of their sub-block's run
 *     of magnitude planes (0: most significant); plane_bytes[j] their count and
 *     plane_entropy[j] their byte entropy in bits / 8 (1.0: incompressible).
 * The first call on an encoder allocates its region table and accumulators. */
typedef struct pyrowave_cuda_packing_analysis
{
	uint64_t layout_bytes[5];
	uint64_t band_bytes[3][5][4];
	uint64_t coded_bytes;
	uint64_t significant;
	uint64_t plane_bytes[16];
	double plane_entropy[16];
	uint32_t plane_histogram[16][256];
} pyrowave_cuda_packing_analysis;

PYROWAVE_PUBLIC_API pyrowave_result pyrowave_cuda_encoder_analyze_packing(pyrowave_encoder encoder,
                                                                          pyrowave_cuda_packing_analysis *analysis);

/* Decode the packets pushed so far into device planes on `stream` (uploads the
 * parsed payload, then dequantises and inverse transforms). */
PYROWAVE_PUBLIC_API pyrowave_result pyrowave_cuda_decoder_decode(pyrowave_decoder decoder,
                                                                 const pyrowave_cuda_planes *planes,
                                                                 pyrowave_cuda_stream stream);

/* Decode coded blocks already in device memory: block_meta = {offset_u32,
 * num_words} per 32x32 block (num_words == 0: block missing), words = the
 * concatenated block words the offsets index. Nothing touches the host. */
PYROWAVE_PUBLIC_API pyrowave_result pyrowave_cuda_decoder_decode_blocks(pyrowave_decoder decoder,
                                                                        const uint32_t *block_meta,
                                                                        const uint32_t *words, size_t num_words,
                                                                        const pyrowave_cuda_planes *planes,
                                                                        pyrowave_cuda_stream stream);

/* As pyrowave_cuda_decoder_decode_blocks, into 16-bit planes (R16_UNORM samples,
 * each row_stride_in_bytes a multiple of 2 and at least 2 * width). */
PYROWAVE_PUBLIC_API pyrowave_result pyrowave_cuda_decoder_decode_blocks16(pyrowave_decoder decoder,
                                                                          const uint32_t *block_meta,
                                                                          const uint32_t *words, size_t num_words,
                                                                          const pyrowave_cuda_planes *planes,
                                                                          pyrowave_cuda_stream stream);

/* Assemble a frame from received packets on the GPU and decode it: the
 * device-side counterpart of pyrowave_decoder_clear, then
 * pyrowave_decoder_push_packet for every packet in order
 * (pyrowave_decoder.cpp:126-262), then pyrowave_decoder_decode_gpu_buffer.
 * `data` holds the packets in device memory (4-byte aligned, at most 4 GiB);
 * `packets` is a device array of `count` {offset, size} byte ranges of `data`,
 * in push order, each offset a multiple of 4. The sequence rules of the
 * reference parser apply (a newer sequence restarts the frame, packets of an
 * older one are ignored from that point of the packet on, the first copy of a
 * block wins); blocks not received decode as zero. A packet the host parser
 * would reject keeps what it added before the fault, as push_packet does,
 * except that a block announcing fewer than two words is left missing. Nothing
 * waits: the outcome is read with pyrowave_cuda_decoder_get_packet_status. */
typedef struct pyrowave_cuda_packet_status
{
	uint32_t decoded_blocks;  /* distinct blocks of the assembled frame */
	uint32_t total_blocks;    /* blocks its sequence header announced (the layout's count without one) */
	uint32_t sequence;        /* 3-bit sequence of the frame, 0xffffffff when no packet was accepted */
	uint32_t invalid_packets; /* packets pyrowave_decoder_push_packet would have rejected */
} pyrowave_cuda_packet_status;

PYROWAVE_PUBLIC_API pyrowave_result pyrowave_cuda_decoder_decode_packets(pyrowave_decoder decoder, const void *data,
                                                                         size_t data_size,
                                                                         const pyrowave_packet *packets,
                                                                         uint32_t count,
                                                                         const pyrowave_cuda_planes *planes,
                                                                         pyrowave_cuda_stream stream);

/* Outcome of the last pyrowave_cuda_decoder_decode_packets (waits for it).
 * The frame was complete when decoded_blocks >= total_blocks; the reference's
 * partial-frame rule (pyrowave_decoder_decode_is_ready with
 * allow_partial_frame) accepts more than half. */
PYROWAVE_PUBLIC_API pyrowave_result pyrowave_cuda_decoder_get_packet_status(pyrowave_decoder decoder,
                                                                            pyrowave_cuda_packet_status *status);

/* Outcome of the decoder's last decode on the GPU (any of pyrowave_cuda_decoder_decode,
 * _decode_blocks, _decode_packets, _decode_pyramid; waits for it). The inverse
 * transform loads interior tiles with the tensor-memory accelerator and gives
 * up a tile whose load does not complete within a bounded wait; such a frame
 * is not valid. Returns PYROWAVE_ERROR_GENERIC and sets bit 0 of *error_bits
 * (may be NULL) when that happened, PYROWAVE_SUCCESS otherwise.
 * pyrowave_decoder_decode_cpu_buffer_synchronous and
 * pyrowave_cuda_decoder_get_packet_status report the same condition through
 * their own result. No counterpart in the reference (its Vulkan decode has no
 * bounded waits). */
PYROWAVE_PUBLIC_API pyrowave_result pyrowave_cuda_decoder_get_error(pyrowave_decoder decoder, uint32_t *error_bits);

/* Copy the last decode's dequantised pyramid (canonical layout, device memory). */
PYROWAVE_PUBLIC_API pyrowave_result pyrowave_cuda_decoder_read_wavelet(pyrowave_decoder decoder, float *pyramid,
                                                                       pyrowave_cuda_stream stream);

/* Inverse transform of a canonical pyramid in device memory into device planes. */
PYROWAVE_PUBLIC_API pyrowave_result pyrowave_cuda_decoder_decode_pyramid(pyrowave_decoder decoder, const float *pyramid,
                                                                         const pyrowave_cuda_planes *planes,
                                                                         pyrowave_cuda_stream stream);

/* Largest FP32 coefficient storage pyrowave_cuda_decode_blocks_static accepts:
 * 32 MiB, enough for 4:2:0 frames up to 2560x1440 (1920x1080 needs 17.7 MB;
 * 1920x1080 4:4:4 and 3840x2160 do not fit). */
#define PYROWAVE_CUDA_STATIC_DECODE_SCRATCH_BYTES (32u << 20)

/* Decode coded blocks already in device memory (same block_meta / words
 * format as pyrowave_cuda_decoder_decode_blocks) into device planes, without
 * a decoder object and without allocating any memory, host or device.
 *
 * There is no counterpart in the reference: its decoder always owns buffers
 * it allocates. This entry point is for callers that cannot allocate when
 * they decode: a process whose device memory is fully budgeted up front, a
 * real-time thread that must not enter an allocator, or an application that
 * hands its CUDA memory to its own arena and wants no other owner on the GPU.
 *
 * Scratch: the coefficient pyramid is kept in one fixed device array of
 * PYROWAVE_CUDA_STATIC_DECODE_SCRATCH_BYTES inside this library, reserved by
 * CUDA when the library's device code is loaded on a device. Frames whose
 * coefficient storage is larger are rejected with
 * PYROWAVE_ERROR_INVALID_ARGUMENT. Nothing in the array has to start at zero:
 * every coefficient the inverse transform reads is written earlier in the
 * same call (a missing block decodes as zeros).
 *
 * Device address: every call looks up the array's address on the current
 * device (cudaGetSymbolAddress), which allocates nothing once the library's
 * device code is loaded there. With lazy module loading, the CUDA default,
 * the first call on a device is where CUDA loads that code and reserves the
 * array: that call can fail, with PYROWAVE_ERROR_OUT_OF_DEVICE_MEMORY when
 * the device has no room for it. Make that first call before any stream
 * capture is in progress, for example with a small decode at start-up. After
 * a device reset the next call looks the array up again.
 *
 * Overlapping calls race: every call on a device uses the same array, so two
 * calls whose work can overlap on the GPU (different streams without an event
 * between them, or concurrent host threads) corrupt each other's output.
 * Issue the calls in one stream, or order them with events.
 *
 * width, height and chroma follow pyrowave_decoder_create's rules; planes
 * follow pyrowave_cuda_decoder_decode_blocks. Work is queued on `stream`
 * (0: the legacy default stream); the call does not wait for it. */
PYROWAVE_PUBLIC_API pyrowave_result pyrowave_cuda_decode_blocks_static(int width, int height,
                                                                       pyrowave_chroma_subsampling chroma,
                                                                       const uint32_t *block_meta,
                                                                       const uint32_t *words, size_t num_words,
                                                                       const pyrowave_cuda_planes *planes,
                                                                       pyrowave_cuda_stream stream);

/* ------------------------------------------------------------------------
 * PSNR-HVS-M: the reference's perceptual quality metric (shaders/psnr_hvs_m.comp
 * and its driver psnr.cpp:25-28,126-224,245-320: a port of Ponomarenko's
 * PSNR-HVS-M with the reference's own contrast sensitivity function) of a
 * distorted luma plane against its reference, on 8x8 windows at a stride of 4,
 * for 16 viewing distances (height factors 1 + i/8, i = 0..15).
 *
 * pyrowave_cuda_psnr_hvs_m adds each factor's error sum, in fixed point with
 * 2^-24 units, into `errors` (16 uint64_t in device memory, 8-byte aligned,
 * zeroed by the caller; several frames may accumulate). Both planes are 8-bit,
 * width x height, in device memory. Queued on `stream`; allocates nothing.
 * pyrowave_psnr_hvs_m_pixels gives the pixel count one frame adds (64 per
 * window, as the reference counts); pyrowave_psnr_hvs_m_from_errors turns
 * host copies of the sums into dB, with the limited-range peak of 223/255
 * unless full_range. */
PYROWAVE_PUBLIC_API pyrowave_result pyrowave_cuda_psnr_hvs_m(int width, int height, const uint8_t *reference,
                                                             size_t reference_stride, const uint8_t *distorted,
                                                             size_t distorted_stride, uint64_t *errors,
                                                             pyrowave_cuda_stream stream);
PYROWAVE_PUBLIC_API uint64_t pyrowave_psnr_hvs_m_pixels(int width, int height);
PYROWAVE_PUBLIC_API void pyrowave_psnr_hvs_m_from_errors(const uint64_t *errors, uint64_t total_pixels, bool full_range,
                                                         double *psnr);

/* ------------------------------------------------------------------------
 * Batched form: encode (and optionally decode) many frames of any sizes,
 * chroma formats and budgets with one CUDA graph launch per call: every stage
 * runs once over all frames' tiles or blocks. Each frame's bitstream is
 * identical to what a pyrowave_encoder of the same size produces for the same
 * input and budget on its n-th call. No counterpart in the reference. */
typedef struct pyrowave_cuda_batch_opaque *pyrowave_cuda_batch;

typedef struct pyrowave_cuda_batch_frame_info
{
	int width, height;
	pyrowave_chroma_subsampling chroma;
	size_t maximum_bitstream_size; /* largest per-call budget of this frame, bytes */
} pyrowave_cuda_batch_frame_info;

/* Create a batch of `count` frame slots (at most 256). Device memory is
 * allocated here, once. */
PYROWAVE_PUBLIC_API pyrowave_result pyrowave_cuda_batch_create(pyrowave_device device,
                                                               const pyrowave_cuda_batch_frame_info *frames,
                                                               uint32_t count, pyrowave_cuda_batch *batch);
PYROWAVE_PUBLIC_API void pyrowave_cuda_batch_destroy(pyrowave_cuda_batch batch);

/* Encode frame i from inputs[i] within budgets[i] bytes (<= its maximum) for
 * every slot; when `outputs` is not NULL, also decode every frame's new
 * bitstream into outputs[i]. Queued on `stream` (NULL: the device's stream);
 * the call does not wait. A call may overwrite the previous call's results. */
PYROWAVE_PUBLIC_API pyrowave_result pyrowave_cuda_batch_encode(pyrowave_cuda_batch batch,
                                                               const pyrowave_cuda_planes *inputs,
                                                               const size_t *budgets,
                                                               const pyrowave_cuda_planes *outputs,
                                                               pyrowave_cuda_stream stream);

/* Device view of frame i's last bitstream (as pyrowave_cuda_encoder_get_device_bitstream). */
PYROWAVE_PUBLIC_API pyrowave_result pyrowave_cuda_batch_get_device_bitstream(pyrowave_cuda_batch batch, uint32_t index,
                                                                             const uint32_t **stream,
                                                                             const uint32_t **block_meta);

/* Bytes of every frame's last bitstream (waits for the last call). */
PYROWAVE_PUBLIC_API pyrowave_result pyrowave_cuda_batch_get_sizes(pyrowave_cuda_batch batch, size_t *bytes);

/* How a batch runs its calls. persistent = 1 (the default): one persistent
 * kernel per call runs every stage of every frame, taking (frame, stage, item)
 * work items in order from a counter, each item waiting (bounded) for its
 * frame's previous stage; ctas_per_sm resident CTAs per SM (0: as many as fit)
 * and large_first = 1 orders each stage's frames largest first. persistent = 0:
 * one launch per stage over all frames, levels with fewer than large_below
 * tiles on 1024-thread CTAs. Both: forward levels >= small_level only
 * transform, and their blocks are quantised afterwards. The bitstreams do not
 * depend on the shape. */
typedef struct pyrowave_cuda_batch_shape
{
	uint32_t persistent;
	int32_t small_level;
	int32_t large_below;
	int32_t ctas_per_sm;
	uint32_t large_first;
	/* Per-stage launches: the frames split into this many groups (1 to 8),
	 * each group its own chain of stage launches, the chains running
	 * concurrently (parallel paths of the call's graph). Frame graphs: the
	 * number of streams the frames are spread over. */
	uint32_t branches;
	/* Nonzero (with persistent = 0): every frame through its own single-frame
	 * encode and decode graphs (as pyrowave_cuda_encoder_encode and
	 * pyrowave_cuda_decoder_decode_blocks), the frames dealt round robin over
	 * `branches` streams that fork from and join into the call's stream. */
	uint32_t frame_graphs;
} pyrowave_cuda_batch_shape;

PYROWAVE_PUBLIC_API pyrowave_result pyrowave_cuda_batch_get_shape(pyrowave_cuda_batch batch,
                                                                  pyrowave_cuda_batch_shape *shape);
/* Waits for the batch's last call, then switches to `shape`. */
PYROWAVE_PUBLIC_API pyrowave_result pyrowave_cuda_batch_set_shape(pyrowave_cuda_batch batch,
                                                                  const pyrowave_cuda_batch_shape *shape,
                                                                  pyrowave_cuda_stream stream);

/* Choose the batch's shape by timing the candidates on these inputs (the
 * batch's autotuner) and keep the fastest: persistent launches with 2 to 4
 * resident CTAs per SM and both frame orders, per-stage launches with
 * three thresholds for 1024-thread CTAs and 1, 2, 4 or 8 concurrent groups of
 * frames, each with the transform-only suffix starting at levels 5 down to 2,
 * and frame graphs over 4 or 8 streams. The bitstreams do not depend on the choice,
 * and the tuning calls do not advance the frames' sequence numbers. Waits. */
PYROWAVE_PUBLIC_API pyrowave_result pyrowave_cuda_batch_autotune(pyrowave_cuda_batch batch,
                                                                 const pyrowave_cuda_planes *inputs,
                                                                 const size_t *budgets,
                                                                 const pyrowave_cuda_planes *outputs,
                                                                 pyrowave_cuda_stream stream);

/* ------------------------------------------------------------------------
 * Serving loop: continuous batching of encode + decode requests from many
 * video streams on one GPU. No counterpart in the reference.
 *
 * Each stream's state is a device-resident working set: an encoder and a
 * decoder with their buffers, which stays on the device between the stream's
 * frames. Requests are admitted by memory: a frame whose stream has no working
 * set starts only once the memory pool has room for one, after releasing the
 * working sets of idle streams (least recently used first) if needed; until
 * then it waits in its stream's queue while other requests run. Submitted
 * frames are queued per stream; a dispatcher thread starts every frame whose
 * stream is idle as soon as one of `max_in_flight` CUDA streams is free and
 * admission allows, so the kernels of different requests overlap on the
 * device. Frames of one stream run in submission order; each result is the
 * same as encoding and decoding that stream alone, also when its working set
 * was released and created again between frames. */
typedef struct pyrowave_cuda_server_opaque *pyrowave_cuda_server;

typedef struct pyrowave_cuda_server_info
{
	size_t memory_pool_bytes; /* device memory for per-stream state */
	uint32_t max_in_flight;   /* frames on the GPU at once (1..64) */
} pyrowave_cuda_server_info;

typedef struct pyrowave_cuda_server_completion
{
	uint64_t request_id;
	uint32_t stream_id;
	int32_t result;           /* pyrowave_result of the request */
	size_t bytes;             /* bitstream bytes of the frame */
	double latency_us;        /* submit to completion, host clock */
} pyrowave_cuda_server_completion;

PYROWAVE_PUBLIC_API pyrowave_result pyrowave_cuda_server_create(pyrowave_device device,
                                                                const pyrowave_cuda_server_info *info,
                                                                pyrowave_cuda_server *server);
/* Waits for every submitted frame, then frees everything. */
PYROWAVE_PUBLIC_API void pyrowave_cuda_server_destroy(pyrowave_cuda_server server);

/* Opens a stream. PYROWAVE_ERROR_OUT_OF_DEVICE_MEMORY when one working set
 * of this frame size and budget is larger than the whole pool; no memory is
 * taken until the stream's first frame is admitted. */
PYROWAVE_PUBLIC_API pyrowave_result pyrowave_cuda_server_open_stream(pyrowave_cuda_server server, int width, int height,
                                                                     pyrowave_chroma_subsampling chroma,
                                                                     size_t maximum_bitstream_size,
                                                                     uint32_t *stream_id);
/* Releases the stream's memory once its queued frames have finished. */
PYROWAVE_PUBLIC_API pyrowave_result pyrowave_cuda_server_close_stream(pyrowave_cuda_server server, uint32_t stream_id);

/* Queue one frame: encode `input` (device planes) within `budget` bytes, then
 * decode the new bitstream into `output` (device planes, may be NULL). Both
 * buffers must stay valid until the completion is reported. Thread-safe.
 * Finished requests wait for pyrowave_cuda_server_poll: with 2^20 requests
 * queued, running or finished but not yet polled, submit refuses more with
 * PYROWAVE_ERROR_OUT_OF_HOST_MEMORY. */
PYROWAVE_PUBLIC_API pyrowave_result pyrowave_cuda_server_submit(pyrowave_cuda_server server, uint32_t stream_id,
                                                                const pyrowave_cuda_planes *input, size_t budget,
                                                                const pyrowave_cuda_planes *output,
                                                                uint64_t *request_id);

/* Up to `capacity` finished requests; waits up to timeout_us for the first. */
PYROWAVE_PUBLIC_API pyrowave_result pyrowave_cuda_server_poll(pyrowave_cuda_server server,
                                                              pyrowave_cuda_server_completion *completions,
                                                              uint32_t capacity, uint32_t *count,
                                                              uint32_t timeout_us);

/* Pool bytes held by working sets now and at most so far, and how many
 * working sets were released to admit another stream's frame. */
PYROWAVE_PUBLIC_API pyrowave_result pyrowave_cuda_server_get_memory(pyrowave_cuda_server server, size_t *used_bytes,
                                                                    size_t *peak_bytes, uint64_t *releases);

/* Latency percentiles (microseconds) and count of the requests finished since
 * the last reset. The percentiles cover the most recent 2^20 of those requests. */
PYROWAVE_PUBLIC_API pyrowave_result pyrowave_cuda_server_stats(pyrowave_cuda_server server, double *p50_us,
                                                               double *p99_us, uint64_t *frames, bool reset);

#ifdef __cplusplus
}
#endif

#endif
