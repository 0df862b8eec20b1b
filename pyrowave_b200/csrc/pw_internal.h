// Internal definitions shared by the host library and the sm_100a kernels.
//
// Frame geometry follows the bitstream definition (bitstream.md:99-152 and the
// block index order at :472-511 of the reference). Device layout chosen here:
//   * every band is a row-major 2D array whose pitch and row count are padded to
//     multiples of 32, so every 8x8 and 32x32 block is addressable without
//     bounds checks; the forward transform writes zeros into the padding, which
//     reproduces the reference quantiser's clamp-to-border sampling;
//   * levels are stored in FP32 or FP16 (per-level mask), each in its own buffer;
//   * the encoder emits the packetized bitstream directly: a 2-word sequence
//     header followed by the coded 32x32 blocks in block index order, placed by
//     a device prefix scan instead of the reference's atomic allocation.
#pragma once

#include <cstddef>
#include <cstdint>

#include <cuda.h>
#include <cuda_fp16.h>
#include <cuda_runtime.h>

struct pyrowave_device_opaque;
struct pyrowave_encoder_opaque;

namespace pw
{
// The CUDA device a pyrowave_device was created on. Library threads of their
// own (the serving loop's dispatcher) make it current before any CUDA call.
int device_ordinal(const pyrowave_device_opaque *device);

// An encoder's frame counter (mod 8, the 3-bit sequence number of its last
// frame). The serving loop carries a stream's counter over to a new encoder
// when the stream's working set was released and is created again.
uint32_t encoder_frames(const pyrowave_encoder_opaque *encoder);
void encoder_set_frames(pyrowave_encoder_opaque *encoder, uint32_t frames);

constexpr int kLevels = 5;
constexpr int kComponents = 3;
constexpr int kAlignment = 32;
constexpr int kMinImageSize = 128;
constexpr int kBuckets = 128;
constexpr int kSubdivisions = 16;
constexpr int kHistSize = kBuckets * kSubdivisions;
constexpr int kMaxBlockWords = 1024; // a 32x32 block can need at most ~640 words
constexpr int kQPlanesOffset = 16;
constexpr int kQuantScaleOffset = 20;
constexpr int kMaxScaleExp = 4;

// Magnitudes are clamped below 2^15 after scaling, keeping the statistics of an
// 8x8 block within 16 entries (q = 0..14 plus "drop all"). Real 8-bit content
// stays far below this (the reference's own table has 15 entries).
constexpr float kMaxScaledMagnitude = 32767.0f;

struct BandDesc
{
	int32_t present;          // transmitted band (LL only at the last level)
	int64_t offset;           // element offset of the band in its level's storage buffer
	int32_t block8_offset;    // first global 8x8 block index
	int32_t block8_stride;    // 8x8 blocks per row
	int32_t block32_offset;   // first global 32x32 block index
	int32_t block32_stride;   // 32x32 blocks per row
	float quant_resolution;   // 1 / decode_quant(encode_quant(1 / resolution)): quantiser scale
	float rdo_scale;          // CSF distortion weight / 256
	uint32_t quant_code;      // encode_quant(1 / resolution): the 32x32 header's quant code
};

struct LevelDesc
{
	int32_t width, height;    // band size at this level
	int32_t pitch, rows;      // padded to multiples of 32
	int32_t tiles_x, tiles_y; // 32x32 band tiles
	int32_t blocks8_x, blocks8_y;
	int32_t fp16;             // 1: coefficients of this level are stored as FP16
	int32_t stage16;          // 1: lifting inputs and outputs rounded to FP16 (reference precision 1)
};

struct Geometry
{
	int32_t width, height, chroma444;
	int32_t aligned_width, aligned_height;
	int32_t block_count_8x8, block_count_32x32;
	int32_t blocks_per_subdivision, subdivision_shift;
	int32_t plane_width[3], plane_height[3];
	LevelDesc level[kLevels];
	BandDesc band[kComponents][kLevels][4];
	int64_t storage_elems32, storage_elems16;
};

// Which band a 32x32 block (in block index order) belongs to: packed
// level | comp << 3 | band << 5 | bx << 8 | by << 20.
__host__ __device__ inline uint32_t pack_job(int level, int comp, int band, int bx, int by)
{
	return uint32_t(level) | (uint32_t(comp) << 3) | (uint32_t(band) << 5) | (uint32_t(bx) << 8) | (uint32_t(by) << 20);
}
__host__ __device__ inline void unpack_job(uint32_t j, int &level, int &comp, int &band, int &bx, int &by)
{
	level = int(j & 7u);
	comp = int((j >> 3) & 3u);
	band = int((j >> 5) & 3u);
	bx = int((j >> 8) & 0xfffu);
	by = int(j >> 20);
}

// The resolve kernel runs one CTA per slice of blocks: a rate-control
// subdivision, or a 1024-block part of a larger one (subdivisions hold a power
// of two of blocks), one thread per block of the slice between 256 and 1024;
// the batched form always uses 1024.
constexpr int kMaxResolveSlices = 128;
constexpr int kResolveBatchThreads = 1024;
__host__ __device__ inline int resolve_slice_blocks(int blocks, int blocks_per_subdivision)
{
	int per = 1024; // a power of two, at least blocks / kMaxResolveSlices
	while (per * kMaxResolveSlices < blocks)
		per *= 2;
	return blocks_per_subdivision < per ? blocks_per_subdivision : per;
}
inline int resolve_slices(int blocks, int blocks_per_subdivision)
{
	const int per = resolve_slice_blocks(blocks, blocks_per_subdivision);
	const int n = (blocks + per - 1) / per;
	return n < 1 ? 1 : n;
}

// Rate-control scratch, one per encoder instance (device memory), cleared
// before every frame.
struct RateControlState
{
	uint32_t histogram[kHistSize]; // savings per (bucket, subdivision)
	uint32_t consumed;             // words at quant 0
	uint32_t error;                // nonzero when a consistency check failed
	uint32_t total_words;          // coded words after rate control (blocks only)
	uint32_t non_zero_blocks;
	int32_t xstar;                 // first partially applied bucket*16+subdivision (-1 none)
	uint32_t sequence;
	uint32_t decode_error;         // kDecodeError* bits of the batched form's decode of this frame
	uint32_t fused_done;           // tile dataflow: fused forward-level CTAs whose quantiser finished
	// Per resolve slice: words << 32 | non-empty blocks << 1 | 1 once published.
	unsigned long long slice_total[kMaxResolveSlices];
};

// Error bits of a decoder's error word.
constexpr uint32_t kDecodeErrorTileWait = 1u;  // an inverse-transform tile load did not complete in time

// Per-decode device state of a decoder, cleared by the dequantiser (or by a
// clear before an inverse-only decode).
struct DecodeState
{
	uint32_t error; // kDecodeError* bits
	uint32_t pad[3];
};

// Error bits of RateControlState::error.
constexpr uint32_t kErrorStreamCapacity = 1u; // the coded frame does not fit the stream buffer
constexpr uint32_t kErrorWordCount = 2u;      // a packed block's size differs from the rate-control estimate
constexpr uint32_t kErrorSliceWait = 4u;      // a resolve slice gave up waiting for a preceding slice's total
constexpr uint32_t kErrorTileWait = 8u;       // a forward-transform tile load did not complete in time
constexpr uint32_t kErrorLevelWait = 16u;     // a work item gave up waiting for the tiles or items it depends on

// Buffers the encode kernels read and write.
struct EncodeBuffers
{
	float *coef32;
	__half *coef16;
	// Per 32x32 block, 1024 values: the quantiser's scaled coefficients as
	// sign-magnitude (|int(v)| in bits 0-14, v < 0 in bit 15), eight per 4x2
	// sub-block at [block * 1024 + 8 * (sub + 8 * col8 + 32 * row8) + i], so the
	// packer reads a sub-block as one 16-byte vector instead of re-quantising.
	uint16_t *mag16;
	uint32_t *code_words;   // per 8x8: q=0 code word (plane codes | Q planes << 16 | scale << 20)
	uint16_t *rd_cost;      // per 32x32 x 16: words when quantised by q
	uint8_t *rd_bucket;     // per 32x32 x 16: bucket index of the step to q
	float *rd_dist;         // per 32x32 x 16: summed distortion
	RateControlState *rc;
	int32_t *quant;         // per 32x32: chosen quant drop
	uint32_t *block_meta;   // per 32x32: {offset_u32 relative to the first block word, num_words}
	uint32_t *stream;       // packetized output: 2-word sequence header, then blocks
	uint32_t stream_capacity_words;
	const uint32_t *jobs;   // per 32x32: pack_job(...)
	// Tile dataflow of the single-frame encode (null: every kernel waits for the
	// whole previous grid). One counter per (level, component, transform tile),
	// cleared with the rate-control state before the frame: each CTA that stores
	// part of a tile adds one after its stores, and a consumer reads a tile only
	// once its counter is complete, so a level starts on the tiles whose inputs
	// exist while the finer level's quantisers still run.
	uint32_t *tile_done;
};

// TMA map of one transform level: the frame's FP32 coefficient storage viewed
// as rows of one level's pitch, every band of that level starting on a row.
// Passed as a kernel parameter (grid constant): a map in global memory at an
// address that earlier held another map can be served stale by the TMA unit's
// descriptor cache.
struct alignas(64) LevelTileMap
{
	CUtensorMap map;
	uint32_t valid;     // bit c: component c's interior tiles load through the map
	int32_t row[3][4];  // first row of band b of component c (forward: the LL input, b = 0)
	// Fault injection for tests (inverse maps only): every tile load that
	// completes is handled as if its bounded wait had run out, which exercises
	// the error report without stalling the GPU. Set from the environment
	// variable PYROWAVE_TEST_FAIL_TILE_WAIT=1 when a decoder builds its maps.
	uint32_t test_fail_wait;
};
// The batched form's maps of one level, per frame (frames past the table use
// plain loads).
constexpr int kBatchTileMapFrames = 64;
struct alignas(64) BatchTileMaps
{
	LevelTileMap frame[kBatchTileMapFrames];
};

struct PlaneInput
{
	const uint8_t *data[3];
	int32_t pitch[3];   // bytes between rows
	int32_t xstride[3]; // bytes between samples (2 for the interleaved CbCr plane of NV12 and for 16-bit planes)
	int32_t sample16;   // 1: 16-bit little-endian samples (R16_UNORM), else 8-bit (R8_UNORM)
};

struct PlaneOutput
{
	uint8_t *data[3];
	int32_t pitch[3];   // bytes between rows
	int32_t sample16;   // 1: write 16-bit samples (R16_UNORM), else 8-bit
};

struct DecodeInput
{
	const uint32_t *offsets;    // per 32x32 block, UINT32_MAX = missing (reference format), or nullptr
	const uint32_t *block_meta; // alternatively {offset, num_words} pairs; num_words == 0 = missing
	const unsigned long long *keys; // alternatively packet-assembly keys: word offset in the low 30 bits, ~0 = missing
	uint32_t *error;            // kDecodeError* bits, or nullptr
	DecodeState *state;         // the decoder's per-decode state (small-levels inverse launch), or nullptr
	const uint32_t *payload;    // concatenated block words
	uint32_t payload_words;
	const uint32_t *jobs;
	float *coef32;
	__half *coef16;
};

// ---------------------------------------------------------------------------
// Kernel parameter blocks. Everything a kernel needs about the frame layout
// arrives by value with the launch, so no kernel starts with a chain of
// dependent loads of layout metadata.
struct BandParam
{
	int64_t offset;                       // storage offset of the band (elements)
	int32_t block8_offset, block8_stride; // global 8x8 numbering
	int32_t block32_offset, block32_stride;
	float quant_resolution, rdo_scale;
	uint32_t quant_code, pad;
};

// One forward or inverse level.
struct LevelParams
{
	LevelDesc L;            // this level
	LevelDesc P;            // the finer level (level - 1): forward input LL / inverse output LL
	int32_t level, chroma444, subdivision_shift;
	int32_t width, height, aligned_width, aligned_height;
	int32_t plane_width[3], plane_height[3];
	int64_t prev_ll[3];     // offset of LL at level - 1 per component
	BandParam band[3][4];   // this level's four bands per component
	// Tile dataflow of the single-frame encode (used when EncodeBuffers::tile_done
	// is set): this level's tile counters start at done_offset (component-major,
	// tiles in row-major order), the finer level's at prev_done_offset, and each
	// finer tile is complete once prev_parts CTAs have counted it.
	int32_t done_offset, prev_done_offset, prev_parts, pad_done;
};

// One transmitted band, for kernels that walk the 32x32 blocks of all bands.
struct BandEntry
{
	int64_t offset;
	int32_t block32_offset;
	int32_t block32_stride;
	int32_t block8_offset, block8_stride;
	float quant_resolution;
	uint32_t quant_code;
	float rdo_scale;
	int32_t level, comp;
	// Tile dataflow: the counter of the transform tile holding block rel of this
	// band is done_index + rel (tiles and blocks share their row-major order);
	// it is complete at done_parts.
	int32_t done_index, done_parts;
};

constexpr int kMaxBands = 48;
struct BlockParams
{
	LevelDesc level[kLevels];
	int32_t nbands, block_count_32x32, subdivision_shift;
	int32_t width, height, chroma444; // frame size and chroma format (sequence header)
	BandEntry band[kMaxBands]; // in block index order
};

struct ResolveParams
{
	int32_t block_count_32x32, blocks_per_subdivision, subdivision_shift;
	int32_t width, height, chroma444;
	uint32_t target_words, sequence;
	uint32_t fused_ctas; // tile dataflow: forward-level CTAs with a fused quantiser to wait for (0: none)
};

// cudaLaunchKernelEx configuration, optionally marked as a programmatic
// dependent launch of the preceding kernel on the stream.
struct LaunchConfig
{
	cudaLaunchConfig_t cfg;
	cudaLaunchAttribute attr;
	LaunchConfig(dim3 grid, dim3 block, cudaStream_t stream, bool programmatic);
	LaunchConfig(const LaunchConfig &) = delete;
};

// Packing analysis (statistics of a coded frame beside the hot path): device
// accumulators of packing_analysis_kernel, cleared by the launcher. Layouts:
// 32x32 packets with 2x2, 4x2 and 2x4 sub-blocks, 64x32 with 4x4, 64x64 with 8x4.
constexpr int kPackingLayouts = 5;
struct PackingAnalysisAccum
{
	unsigned long long layout_bytes[kPackingLayouts];
	unsigned long long band_bytes[kComponents * kLevels * 4]; // (component * 5 + level) * 4 + band
	unsigned long long significant;
	uint32_t plane_histogram[16 * 256];
};
// regions: 5 ints per 64x64 region of a coded band (four 32x32 block indices,
// -1 beyond the band, then the band's slot).
cudaError_t launch_packing_analysis(const BlockParams &p, const EncodeBuffers &buf, const int32_t *regions,
                                    int num_regions, PackingAnalysisAccum *acc, cudaStream_t stream);

// Frame layout without the job table; allocates nothing.
bool make_geometry(Geometry &g, int width, int height, bool chroma444, uint32_t fp16_mask);
LevelParams make_level_params(const Geometry &g, int level);
BlockParams make_block_params(const Geometry &g);
ResolveParams make_resolve_params(const Geometry &g, uint32_t target_words, uint32_t sequence);

// ---------------------------------------------------------------------------
// Batched form: the frames of a batch (any sizes and chroma formats) go
// through every stage in one launch per stage. Each frame's fixed parameters
// sit in a device table of BatchFrame, its per-call inputs in BatchFrameIO;
// each launch maps its CTAs to (frame, work item of that frame) through a
// table of batch_cta() words.
struct BatchFrame
{
	LevelParams lp[kLevels];
	BlockParams bp;
	EncodeBuffers eb;
	DecodeInput di;      // decodes the frame's own bitstream (eb.block_meta, eb.stream + 2)
	int32_t block_count;  // 32x32 blocks
	int32_t slices;       // resolve CTAs
	int32_t small_blocks; // blocks of the levels the batch quantises after the transform
	int32_t pad;
};

struct BatchFrameIO
{
	PlaneInput in;
	PlaneOutput out;
	ResolveParams rp; // target words and sequence number of this call
};

__host__ __device__ inline uint32_t batch_cta(int frame, int local) { return (uint32_t(frame) << 24) | uint32_t(local); }
constexpr int kMaxBatchFrames = 256;

// The batched form's persistent launch: one kernel runs every stage of every
// frame. Its work items are (frame, stage, item) words in a fixed order; CTAs
// take them from a ticket counter, and an item first waits until every item
// of its frame's gating stage (the nearest earlier stage with items) has
// finished. Stages of a frame in dependency order:
constexpr int kStageDwt0 = 0;     // forward level L is stage kStageDwt0 + L (levels 0..4)
constexpr int kStageQuant = 5;    // quantiser of the transform-only levels, two 32x32 blocks per item
constexpr int kStageResolve = 6;  // rate-control slices
constexpr int kStagePack = 7;     // two 32x32 blocks per item
constexpr int kStageDequant = 8;  // two 32x32 blocks per item
constexpr int kStageIdwt4 = 9;    // inverse level L is stage kStageIdwt4 + 4 - L
constexpr int kBatchStages = 14;
constexpr int kBatchLocalBits = 19;
__host__ __device__ inline uint32_t batch_work(int frame, int stage, int local)
{
	return (uint32_t(frame) << 24) | (uint32_t(stage) << kBatchLocalBits) | uint32_t(local);
}
constexpr uint32_t kNoGate = 0xffffffffu;

struct BatchRunParams
{
	const BatchFrame *frames;
	const BatchFrameIO *io;
	const uint32_t *work;  // work items in ticket order
	const uint32_t *gates; // per frame and stage: gating stage << 24 | its item count, or kNoGate
	uint32_t *ticket;      // zero at launch
	uint32_t *done;        // per frame and stage: items finished, zero at launch
	int32_t nwork;
	int32_t small_level;   // forward levels >= this only transform; kStageQuant quantises their blocks
};
constexpr int kBatchPersistentThreads = 256;
// Resident CTAs per SM of the persistent kernel (its register and shared-memory limit).
int batch_persistent_max_ctas_per_sm();
void launch_batch_persistent(const BatchRunParams &rp, int ctas, cudaStream_t stream);

// Host-side kernel launchers (implemented in the .cu files). Every launch but
// the first of a sequence may start early (programmatic dependent launch):
// kernels wait for their predecessor with griddepcontrol before touching
// global memory.
// Levels with fewer tiles than this (all components) are "small": their
// transforms run 1024-thread CTAs, and the encoder quantises their bands in one
// launch across the whole GPU after the last level instead of inside the
// transform of each level.
constexpr int kSmallLevelTiles = 256;
// Fused quantiser modes of a forward level launch: 0 none, 1 fused, and
// kFusedSplitTail (levels of fewer than kSplitTailTiles tiles, about two waves
// of 256-thread CTAs): a last quantiser round with idle groups runs on the
// whole CTA instead.
constexpr int kFusedSplitTail = 2;
constexpr int kSplitTailTiles = 2 * 148 * 4;
// CTAs per tile of a small transform-only level (row stripes of the tile).
constexpr int kDwtStripeCtas = 4;
// Bounded waits of the tile dataflow (each poll sleeps about 64 ns or more):
// about a second at most, after which the waiting CTA records kErrorLevelWait
// and carries on.
constexpr uint32_t kDataflowWaitSpins = 1u << 20;
int forward_fused_mode(const LevelParams &p, bool fused_quant);
void launch_dwt_forward_level(const LevelParams &p, const PlaneInput &in, const EncodeBuffers &buf,
                              const LevelTileMap *maps, bool fused_quant,
                              bool programmatic, cudaStream_t stream);
// Quantise and analyse the first nblocks 32x32 blocks (block index order) from storage.
void launch_quant_pretransformed(const BlockParams &p, const EncodeBuffers &buf, int nblocks, bool programmatic,
                                 cudaStream_t stream);
// Largest thread-block cluster the resolve uses on this device (8 or 16);
// queried once, outside stream capture, before the first launch_resolve.
int resolve_cluster_max();
void launch_resolve(const ResolveParams &p, const EncodeBuffers &buf, cudaStream_t stream);
void launch_pack(const BlockParams &p, const EncodeBuffers &buf, cudaStream_t stream);
// Dequantise blocks [first, first + count) (block index order).
void launch_dequant(const BlockParams &p, const DecodeInput &in, int first, int count, bool programmatic,
                    cudaStream_t stream);
void launch_idwt_level(const LevelParams &p, const DecodeInput &in, const PlaneOutput &out, const LevelTileMap *maps,
                       bool programmatic,
                       cudaStream_t stream);
void launch_pyramid_io(const BlockParams &p, float *canonical, float *coef32, __half *coef16, bool to_canonical,
                       cudaStream_t stream);

// Device-side packet assembly (pw_packets.cu). The first four fields of
// PacketStatus are the public pyrowave_cuda_packet_status.
struct PacketStatus
{
	uint32_t decoded_blocks;  // distinct blocks kept
	uint32_t total_blocks;    // blocks the frame's sequence header announced, else the layout's count
	uint32_t sequence;        // 3-bit sequence of the assembled frame, 0xffffffff: none
	uint32_t invalid_packets; // packets the host parser would reject
	uint32_t restart_packet, restart_item; // position of the last restart
	uint32_t pad[2];
};

struct PacketParams
{
	const uint32_t *data;             // the received packets (device memory, 4-byte aligned)
	unsigned long long data_bytes;
	const unsigned long long *packets; // {offset, size} in bytes per packet (pyrowave_packet), device memory
	int32_t count;
	int32_t width, height, chroma444, block_count;
	uint32_t *tables;                 // count x 9 x {state | error << 4 | restart << 8, total}
	uint8_t *state_before;            // count
	uint32_t *summaries;              // count x 8 words: each packet's item summary
	uint32_t *items;                  // data_bytes / 4: packet p's item positions at its own first word on
	unsigned long long *first;        // block_count: smallest (packet, item, word offset) key, ~0 = missing
	uint32_t *counter;                // CTAs of the table pass done (zero between calls)
	PacketStatus *status;
};

constexpr int kMaxPackets = 1 << 20;
void launch_packet_assembly(const PacketParams &pp, cudaStream_t stream);

// Batched launchers: `cta_map` holds one batch_cta() word per CTA.
// large_ctas selects the 1024-thread variant of a level; `maps` (may be null)
// holds the level's per-frame TMA maps.
void launch_dwt_forward_batch(const BatchFrame *frames, const BatchFrameIO *io, const uint32_t *cta_map, int nctas,
                              int level, const BatchTileMaps *maps, bool fused_quant, bool large_ctas,
                              bool programmatic, cudaStream_t stream);
void launch_quant_blocks_batch(const BatchFrame *frames, const uint32_t *cta_map, int nctas, bool programmatic,
                               cudaStream_t stream);
void launch_resolve_batch(const BatchFrame *frames, const BatchFrameIO *io, const uint32_t *cta_map, int nctas,
                          cudaStream_t stream);
void launch_pack_batch(const BatchFrame *frames, const uint32_t *cta_map, int nctas, cudaStream_t stream);
void launch_dequant_batch(const BatchFrame *frames, const uint32_t *cta_map, int nctas, bool programmatic,
                          cudaStream_t stream);
void launch_idwt_batch(const BatchFrame *frames, const BatchFrameIO *io, const uint32_t *cta_map, int nctas, int level,
                       const BatchTileMaps *maps, bool large_ctas, bool programmatic, cudaStream_t stream);

} // namespace pw
