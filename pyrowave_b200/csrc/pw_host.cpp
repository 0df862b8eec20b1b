// Host side of the B200 PyroWave library: frame geometry, encoder and decoder
// objects, the packet parser and the C API of include/pyrowave.h and
// include/pyrowave_cuda.h.
//
// Reference interfaces replaced (file:line in the reference tree):
//   C API                   pyrowave.h:73-539, pyrowave_c.cpp:32-1498
//   geometry / block tables pyrowave_common.cpp:191-241 (and bitstream.md:472-511)
//   quant tables            pyrowave_encoder.cpp:107-172
//   encode sequence         pyrowave_encoder.cpp:1153-1183
//   packetize               pyrowave_encoder.cpp:596-623,1048-1115
//   packet parser           pyrowave_decoder.cpp:126-262,780-794,832-840
//   decode sequence         pyrowave_decoder.cpp:796-830
#include "pw_internal.h"

#include <cudaTypedefs.h>

#include "pyrowave.h"
#include "pyrowave_cuda.h"

#include <algorithm>
#include <array>
#include <cmath>
#include <cstdio>
#include <cstdlib>
#include <cstring>
#include <mutex>
#include <new>
#include <string>
#include <vector>

using namespace pw;

namespace
{
int align_up(int v, int a) { return (v + a - 1) & ~(a - 1); }

// CUDA error reporting: failures are logged to stderr when PYROWAVE_DEBUG is
// set (the reference logs through Granite only with VULKAN_DEBUG,
// pyrowave_c.cpp:17-29).
bool debug_enabled()
{
	static const bool on = [] {
		const char *e = getenv("PYROWAVE_DEBUG");
		return e && atoi(e) != 0;
	}();
	return on;
}

bool cuda_ok(cudaError_t e, const char *what)
{
	if (e == cudaSuccess)
		return true;
	if (debug_enabled())
		fprintf(stderr, "pyrowave: %s failed: %s\n", what, cudaGetErrorString(e));
	return false;
}

// Consumes (and reports) the error state left by preceding kernel launches.
bool launches_ok(const char *what) { return cuda_ok(cudaGetLastError(), what); }

uint32_t float_bits(float f)
{
	uint32_t u;
	memcpy(&u, &f, 4);
	return u;
}

// 32x32 header quant code (pyrowave_common.hpp:135-145 / bitstream.md:441-449).
uint32_t encode_quant(float decoder_q_scale)
{
	uint32_t v = float_bits(decoder_q_scale);
	int e = int((v >> 23) & 0xffu) - 127 - kMaxScaleExp;
	int m = int((v >> 20) & 7u);
	e = std::min(std::max(-e, 0), 31);
	return uint32_t((e << 3) | m) & 0xffu;
}

float decode_quant(uint32_t code)
{
	int e = kMaxScaleExp - int(code >> 3);
	int m = int(code & 7u);
	return std::ldexp(float(8 + m), e - 3);
}

// Initial quantiser resolution: a flat spectrum with noise-power normalisation,
// 8 bits plus 2 for LL, 1 for HL/LH, plus the level, one less for chroma,
// capped at 4096 (pyrowave_encoder.cpp:144-172).
float noise_normalized_resolution(int level, int comp, int band)
{
	int bits = 8 + (band == 0 ? 2 : (band < 3 ? 1 : 0)) + level - (comp != 0 ? 1 : 0);
	return float(1 << bits);
}

float quant_resolution(int level, int comp, int band)
{
	return std::min(4096.0f, noise_normalized_resolution(level, comp, band));
}

// Contrast-sensitivity weighting of the RD distortion (pyrowave_encoder.cpp:107-142):
// band centre frequency in cycles per degree at 96 dpi and 1 m viewing distance,
// CSF 2.6 (0.0192 + 0.114 f) exp(-(0.114 f)^1.1), chroma discounted 0.6 at 4:2:0,
// squared because distortion is measured in power.
float rdo_distortion_scale(int level, int comp, int band, bool chroma444)
{
	const float hx = (band & 1) ? 0.75f : 0.25f;
	const float vy = (band & 2) ? 0.75f : 0.25f;
	const float cpd_nyquist = 0.34f * 1.0f * 96.0f;
	float cpd = std::sqrt(hx * hx + vy * vy) * cpd_nyquist * std::exp2(-float(level));
	cpd = std::max(cpd, 8.0f);
	float csf = 2.6f * (0.0192f + 0.114f * cpd) * std::exp(-std::pow(0.114f * cpd, 1.1f));
	if (comp != 0 && level != kLevels - 1 && !chroma444)
		csf *= 0.6f;
	float weighted = csf * noise_normalized_resolution(level, comp, band);
	return weighted * weighted;
}

bool has_level(int comp, int level, bool chroma444) { return !(level == 0 && comp != 0 && !chroma444); }

// Frame geometry, padded band storage and the block tables.
// Layout only: band sizes, storage offsets and block numbering (no job table).
bool build_geometry(Geometry &g, int width, int height, bool chroma444, uint32_t fp16_mask)
{
	if (width <= 0 || height <= 0 || width > 16384 || height > 16384)
		return false;
	memset(&g, 0, sizeof(g));
	g.width = width;
	g.height = height;
	g.chroma444 = chroma444 ? 1 : 0;
	g.aligned_width = std::max(align_up(width, kAlignment), kMinImageSize);
	g.aligned_height = std::max(align_up(height, kAlignment), kMinImageSize);
	for (int c = 0; c < 3; c++)
	{
		g.plane_width[c] = (c == 0 || chroma444) ? width : width / 2;
		g.plane_height[c] = (c == 0 || chroma444) ? height : height / 2;
	}
	for (int level = 0; level < kLevels; level++)
	{
		LevelDesc &L = g.level[level];
		L.width = std::max(1, (g.aligned_width / 2) >> level);
		L.height = std::max(1, (g.aligned_height / 2) >> level);
		L.pitch = align_up(L.width, 32);
		L.rows = align_up(L.height, 32);
		L.tiles_x = L.pitch / 32;
		L.tiles_y = L.rows / 32;
		L.blocks8_x = (L.width + 7) / 8;
		L.blocks8_y = (L.height + 7) / 8;
		L.fp16 = (fp16_mask >> level) & 1u;
		L.stage16 = (fp16_mask & PYROWAVE_CUDA_PRECISION_STAGE16) ? 1 : 0;
	}

	// Storage: every band of every (component, level) that exists, LL included.
	int64_t off32 = 0, off16 = 0;
	for (int level = 0; level < kLevels; level++)
		for (int comp = 0; comp < kComponents; comp++)
		{
			if (!has_level(comp, level, chroma444))
				continue;
			const LevelDesc &L = g.level[level];
			for (int band = 0; band < 4; band++)
			{
				int64_t &off = L.fp16 ? off16 : off32;
				g.band[comp][level][band].offset = off;
				off += int64_t(L.pitch) * L.rows;
			}
		}
	g.storage_elems32 = off32;
	g.storage_elems16 = off16;

	// Block index order (bitstream.md:472-511): level 4 -> 0, component, band.
	int count8 = 0, count32 = 0;
	for (int level = kLevels - 1; level >= 0; level--)
		for (int comp = 0; comp < kComponents; comp++)
		{
			if (!has_level(comp, level, chroma444))
				continue;
			for (int band = (level == kLevels - 1 ? 0 : 1); band < 4; band++)
			{
				const LevelDesc &L = g.level[level];
				BandDesc &B = g.band[comp][level][band];
				B.present = 1;
				B.block8_offset = count8;
				B.block8_stride = L.blocks8_x;
				B.block32_offset = count32;
				B.block32_stride = (L.width + 31) / 32;
				float qr = quant_resolution(level, comp, band);
				B.quant_code = encode_quant(1.0f / qr);
				B.quant_resolution = 1.0f / decode_quant(B.quant_code);
				B.rdo_scale = rdo_distortion_scale(level, comp, band, chroma444) * (1.0f / 256.0f);
				const int by32n = (L.height + 31) / 32;
				count32 += B.block32_stride * by32n;
				count8 += L.blocks8_x * L.blocks8_y;
			}
		}
	g.block_count_8x8 = count8;
	g.block_count_32x32 = count32;
	// Blocks per subdivision: next power of two of ceil(count / 16) (pyrowave_encoder.cpp:21-26).
	int per = (count32 + kSubdivisions - 1) / kSubdivisions;
	int pot = 1, shift = 0;
	while (pot < per)
	{
		pot *= 2;
		shift++;
	}
	g.blocks_per_subdivision = pot;
	g.subdivision_shift = shift;
	return true;
}

// Layout plus the per-32x32 job table in block index order.
bool build_geometry(Geometry &g, std::vector<uint32_t> &jobs, int width, int height, bool chroma444, uint32_t fp16_mask)
{
	if (!build_geometry(g, width, height, chroma444, fp16_mask))
		return false;
	jobs.clear();
	for (int level = kLevels - 1; level >= 0; level--)
		for (int comp = 0; comp < kComponents; comp++)
			for (int band = 0; band < 4; band++)
			{
				const BandDesc &B = g.band[comp][level][band];
				if (!B.present)
					continue;
				const int by32n = (g.level[level].height + 31) / 32;
				for (int by = 0; by < by32n; by++)
					for (int bx = 0; bx < B.block32_stride; bx++)
						jobs.push_back(pack_job(level, comp, band, bx, by));
			}
	return true;
}

// The small levels (fewer than kSmallLevelTiles tiles) are the coarsest ones;
// their blocks come first in block index order (level 4 -> 0), so they are
// the prefix [0, blocks) of the blocks.
void small_level_split(const Geometry &g, int &level_out, int &blocks)
{
	level_out = kLevels;
	for (int level = kLevels - 1; level >= 0; level--)
	{
		const int tiles = g.level[level].tiles_x * g.level[level].tiles_y * ((level == 0 && !g.chroma444) ? 1 : 3);
		if (tiles >= kSmallLevelTiles)
			break;
		level_out = level;
	}
	blocks = level_out == kLevels ? 0
	         : level_out == 0     ? g.block_count_32x32
	                              : g.band[0][level_out - 1][1].block32_offset;
}

// Per-band resolution override of encode_pre_transformed (pyrowave_encoder.cpp:449,251).
void apply_quant_scale_override(Geometry &g, float quant_scale)
{
	for (int comp = 0; comp < kComponents; comp++)
		for (int level = 0; level < kLevels; level++)
			for (int band = 0; band < 4; band++)
			{
				BandDesc &B = g.band[comp][level][band];
				if (!B.present)
					continue;
				float qr = quant_scale < 0.0f ? quant_resolution(level, comp, band) : quant_scale;
				B.quant_code = encode_quant(1.0f / qr);
				B.quant_resolution = 1.0f / decode_quant(B.quant_code);
			}
}

template <typename T> T *dev_alloc(size_t count, bool &ok)
{
	if (count == 0)
		count = 1;
	void *p = nullptr;
	if (cudaMalloc(&p, count * sizeof(T)) != cudaSuccess)
	{
		ok = false;
		(void)cudaGetLastError();
		return nullptr;
	}
	return static_cast<T *>(p);
}

template <typename T> T *host_alloc(size_t count, bool &ok)
{
	if (count == 0)
		count = 1;
	void *p = nullptr;
	if (cudaMallocHost(&p, count * sizeof(T)) != cudaSuccess)
	{
		ok = false;
		(void)cudaGetLastError();
		return nullptr;
	}
	return static_cast<T *>(p);
}

void dev_free(void *p)
{
	if (p)
		cudaFree(p);
}
void host_free(void *p)
{
	if (p)
		cudaFreeHost(p);
}

struct StageTimer
{
	const char *tag;
	double total_ms = 0.0;
	uint64_t frames = 0;
};

} // namespace

// ---------------------------------------------------------------------------
// Kernel parameter blocks derived from the geometry.
namespace pw
{
static BandParam band_param(const Geometry &g, int comp, int level, int band)
{
	const BandDesc &B = g.band[comp][level][band];
	BandParam p = {};
	p.offset = B.offset;
	p.block8_offset = B.block8_offset;
	p.block8_stride = B.block8_stride;
	p.block32_offset = B.block32_offset;
	p.block32_stride = B.block32_stride;
	p.quant_resolution = B.quant_resolution;
	p.rdo_scale = B.rdo_scale;
	p.quant_code = B.quant_code;
	return p;
}

LevelParams make_level_params(const Geometry &g, int level)
{
	LevelParams p = {};
	p.L = g.level[level];
	p.P = level > 0 ? g.level[level - 1] : g.level[0];
	p.level = level;
	p.chroma444 = g.chroma444;
	p.subdivision_shift = g.subdivision_shift;
	p.width = g.width;
	p.height = g.height;
	p.aligned_width = g.aligned_width;
	p.aligned_height = g.aligned_height;
	for (int c = 0; c < 3; c++)
	{
		p.plane_width[c] = g.plane_width[c];
		p.plane_height[c] = g.plane_height[c];
		p.prev_ll[c] = level > 0 ? g.band[c][level - 1][0].offset : 0;
		for (int b = 0; b < 4; b++)
			p.band[c][b] = band_param(g, c, level, b);
	}
	return p;
}

BlockParams make_block_params(const Geometry &g)
{
	BlockParams p = {};
	for (int level = 0; level < kLevels; level++)
		p.level[level] = g.level[level];
	p.block_count_32x32 = g.block_count_32x32;
	p.subdivision_shift = g.subdivision_shift;
	p.width = g.width;
	p.height = g.height;
	p.chroma444 = g.chroma444;
	for (int level = kLevels - 1; level >= 0; level--)
		for (int comp = 0; comp < kComponents; comp++)
			for (int band = 0; band < 4; band++)
			{
				const BandDesc &B = g.band[comp][level][band];
				if (!B.present || p.nbands >= kMaxBands)
					continue;
				BandEntry &e = p.band[p.nbands++];
				e.offset = B.offset;
				e.block32_offset = B.block32_offset;
				e.block32_stride = B.block32_stride;
				e.block8_offset = B.block8_offset;
				e.block8_stride = B.block8_stride;
				e.quant_resolution = B.quant_resolution;
				e.quant_code = B.quant_code;
				e.rdo_scale = B.rdo_scale;
				e.level = level;
				e.comp = comp;
			}
	return p;
}

// Tile dataflow of the single-frame encode: one counter per (level, component,
// transform tile), components and tiles in order within a level. Fills in the
// counters' offsets and the count at which each level's tiles are complete
// (the CTAs storing one tile: row stripes for the small transform-only levels,
// as launch_dwt_forward_level launches them), and the number of forward-level
// CTAs with a fused quantiser. Returns the number of counters.
int setup_tile_dataflow(const Geometry &g, int small_level, LevelParams (&lp)[kLevels], BlockParams &bp,
                        uint32_t &fused_ctas)
{
	int32_t offset[kLevels] = {}, parts[kLevels] = {};
	int total = 0;
	fused_ctas = 0;
	for (int level = 0; level < kLevels; level++)
	{
		const int comps = (level == 0 && !g.chroma444) ? 1 : kComponents;
		const int tiles = comps * g.level[level].tiles_x * g.level[level].tiles_y;
		offset[level] = total;
		total += tiles;
		const bool transform_only = level >= small_level;
		parts[level] = (transform_only && tiles < kSmallLevelTiles) ? kDwtStripeCtas : 1;
		if (!transform_only)
			fused_ctas += uint32_t(tiles);
	}
	for (int level = 0; level < kLevels; level++)
	{
		lp[level].done_offset = offset[level];
		lp[level].prev_done_offset = level > 0 ? offset[level - 1] : 0;
		lp[level].prev_parts = level > 0 ? parts[level - 1] : 0;
	}
	for (int i = 0; i < bp.nbands; i++)
	{
		BandEntry &e = bp.band[i];
		const LevelDesc &L = g.level[e.level];
		const int comp = (e.level == 0 && !g.chroma444) ? 0 : e.comp;
		e.done_index = offset[e.level] + comp * L.tiles_x * L.tiles_y;
		e.done_parts = parts[e.level];
	}
	return total;
}

ResolveParams make_resolve_params(const Geometry &g, uint32_t target_words, uint32_t sequence)
{
	ResolveParams p = {};
	p.block_count_32x32 = g.block_count_32x32;
	p.blocks_per_subdivision = g.blocks_per_subdivision;
	p.subdivision_shift = g.subdivision_shift;
	p.width = g.width;
	p.height = g.height;
	p.chroma444 = g.chroma444;
	p.target_words = target_words;
	p.sequence = sequence;
	return p;
}

bool make_geometry(Geometry &g, int width, int height, bool chroma444, uint32_t fp16_mask)
{
	return build_geometry(g, width, height, chroma444, fp16_mask);
}
} // namespace pw

// ---------------------------------------------------------------------------
struct pyrowave_device_opaque
{
	int cuda_device = 0;
	cudaStream_t stream = nullptr;
	bool stage_timing = false;
	std::mutex lock;
	std::vector<StageTimer> timers;

	void add_time(const char *tag, double ms)
	{
		std::lock_guard<std::mutex> g(lock);
		for (auto &t : timers)
			if (strcmp(t.tag, tag) == 0)
			{
				t.total_ms += ms;
				t.frames++;
				return;
			}
		timers.push_back({tag, ms, 1});
	}
};

namespace pw
{
int device_ordinal(const pyrowave_device_opaque *device) { return device ? device->cuda_device : 0; }
} // namespace pw

namespace
{
// Per-stage GPU timing with CUDA events (the reference's register_time_interval,
// pyrowave_encoder.cpp:277,335,411,486,591; surfaced by report_performance_stats).
struct StageEvents
{
	static constexpr int kMax = 16;
	cudaEvent_t ev[kMax + 1] = {};
	const char *tags[kMax] = {};
	int count = 0;
	bool pending = false;
	bool created = false;

	// Outside stream capture: create the events once timing is on.
	void prepare(pyrowave_device_opaque *dev)
	{
		if (!dev->stage_timing || created)
			return;
		for (auto &e : ev)
			cuda_ok(cudaEventCreate(&e), "cudaEventCreate");
		created = true;
	}
	// Inside stream capture the records become event-record graph nodes
	// (cudaEventRecordExternal), replayed with every launch of the graph;
	// outside a capture (captured = false) they are plain records.
	bool captured = true;
	void record(cudaStream_t s, cudaEvent_t e)
	{
		if (captured)
			cuda_ok(cudaEventRecordWithFlags(e, s, cudaEventRecordExternal), "cudaEventRecordWithFlags");
		else
			cuda_ok(cudaEventRecord(e, s), "cudaEventRecord");
	}
	void begin(pyrowave_device_opaque *dev, cudaStream_t s, bool in_capture = true)
	{
		if (!dev->stage_timing || !created)
			return;
		count = 0;
		captured = in_capture;
		record(s, ev[0]);
	}
	void mark(pyrowave_device_opaque *dev, cudaStream_t s, const char *tag)
	{
		if (!dev->stage_timing || !created || count >= kMax)
			return;
		tags[count++] = tag;
		record(s, ev[count]);
	}
	// The events of the captured sequence were launched (they are graph nodes).
	void launched(pyrowave_device_opaque *dev)
	{
		if (dev->stage_timing && created && count > 0)
			pending = true;
	}
	void collect(pyrowave_device_opaque *dev)
	{
		if (!pending)
			return;
		pending = false;
		if (!cuda_ok(cudaEventSynchronize(ev[count]), "cudaEventSynchronize"))
			return;
		for (int i = 0; i < count; i++)
		{
			float ms = 0.0f;
			if (cuda_ok(cudaEventElapsedTime(&ms, ev[i], ev[i + 1]), "cudaEventElapsedTime"))
				dev->add_time(tags[i], ms);
		}
	}
	void destroy()
	{
		if (created)
			for (auto &e : ev)
				cudaEventDestroy(e);
		created = false;
	}
};
} // namespace

namespace
{
// A kernel node of a captured graph, with the launch parameters it was
// captured with; its arguments are replaced per call.
struct KernelNode
{
	cudaGraphNode_t node = nullptr;
	cudaKernelNodeParams params = {};
};

// The node the last captured operation on `s` created.
bool last_captured_node(cudaStream_t s, KernelNode &kn)
{
	cudaStreamCaptureStatus st;
	const cudaGraphNode_t *deps = nullptr;
	size_t n = 0;
	if (!cuda_ok(cudaStreamGetCaptureInfo(s, &st, nullptr, nullptr, &deps, &n), "cudaStreamGetCaptureInfo") ||
	    st != cudaStreamCaptureStatusActive || n == 0)
		return false;
	kn.node = deps[n - 1];
	return cuda_ok(cudaGraphKernelNodeGetParams(kn.node, &kn.params), "cudaGraphKernelNodeGetParams");
}

// Replace the arguments of a kernel node in an instantiated graph; the types
// of `args` must be exactly the kernel's parameter types.
template <typename... A> bool set_kernel_args(cudaGraphExec_t exec, const KernelNode &kn, A &...args)
{
	void *arr[] = {static_cast<void *>(&args)...};
	cudaKernelNodeParams p = kn.params;
	p.kernelParams = arr;
	p.extra = nullptr;
	return cuda_ok(cudaGraphExecKernelNodeSetParams(exec, kn.node, &p), "cudaGraphExecKernelNodeSetParams");
}

// One encode or decode sequence captured as a CUDA graph: a single launch
// per frame instead of one per kernel.
struct CapturedGraph
{
	cudaGraph_t graph = nullptr;
	cudaGraphExec_t exec = nullptr;
	uint64_t key = ~0ull;
	bool valid() const { return exec != nullptr; }
	void destroy()
	{
		if (exec)
			cudaGraphExecDestroy(exec);
		if (graph)
			cudaGraphDestroy(graph);
		exec = nullptr;
		graph = nullptr;
		key = ~0ull;
	}
	bool begin(cudaStream_t s)
	{
		destroy();
		launches_ok("work queued before graph capture");
		return cuda_ok(cudaStreamBeginCapture(s, cudaStreamCaptureModeThreadLocal), "cudaStreamBeginCapture");
	}
	bool end(cudaStream_t s, uint64_t k)
	{
		if (!cuda_ok(cudaStreamEndCapture(s, &graph), "cudaStreamEndCapture"))
		{
			graph = nullptr;
			return false;
		}
		if (!cuda_ok(cudaGraphInstantiate(&exec, graph, cudaGraphInstantiateFlagUseNodePriority), "cudaGraphInstantiate"))
		{
			exec = nullptr;
			return false;
		}
		key = k;
		return true;
	}
};
} // namespace

PFN_cuTensorMapEncodeTiled_v12000 tensor_map_encoder()
{
	static PFN_cuTensorMapEncodeTiled_v12000 encode = [] {
		void *fn = nullptr;
		cudaDriverEntryPointQueryResult q;
		if (cudaGetDriverEntryPoint("cuTensorMapEncodeTiled", &fn, cudaEnableDefault, &q) != cudaSuccess ||
		    q != cudaDriverEntryPointSuccess)
			fn = nullptr;
		return reinterpret_cast<PFN_cuTensorMapEncodeTiled_v12000>(fn);
	}();
	return encode;
}

// 2D FP32 tensor map over a frame's whole FP32 coefficient storage, viewed as
// rows of `pitch` samples.
bool encode_storage_map(CUtensorMap &map, float *coef32, int64_t storage_elems, int pitch, uint32_t box_w,
                        uint32_t box_h)
{
	const auto encode = tensor_map_encoder();
	const cuuint64_t dims[2] = {cuuint64_t(pitch), cuuint64_t(storage_elems / pitch)};
	const cuuint64_t strides[1] = {cuuint64_t(pitch) * 4};
	const cuuint32_t box[2] = {box_w, box_h};
	const cuuint32_t elem[2] = {1, 1};
	return encode && encode(&map, CU_TENSOR_MAP_DATA_TYPE_FLOAT32, 2, coef32, dims, strides, box, elem,
	                        CU_TENSOR_MAP_INTERLEAVE_NONE, CU_TENSOR_MAP_SWIZZLE_NONE, CU_TENSOR_MAP_L2_PROMOTION_L2_128B,
	                        CU_TENSOR_MAP_FLOAT_OOB_FILL_NONE) == CUDA_SUCCESS;
}

// Per-level TMA maps of a frame. Forward level l reads its LL input (level
// l - 1) as boxes of 72 rows x 76 samples; inverse level l reads its four bands
// as boxes of 36 rows x 40 samples. A component's tiles use the map (valid bit)
// when its level is FP32, large enough to have interior tiles, and each band it
// reads starts on a row of the level's pitch; otherwise they use plain loads,
// as do all tiles when the driver offers no tensor-map encoder. Either table
// may be null.
void build_tile_maps(const Geometry &g, const LevelParams (&lp)[kLevels], float *coef32, LevelTileMap *fwd,
                     LevelTileMap *inv)
{
	for (int level = 0; level < kLevels; level++)
	{
		if (fwd)
			fwd[level] = LevelTileMap{};
		if (inv)
			inv[level] = LevelTileMap{};
	}
	if (!tensor_map_encoder() || !coef32 || g.storage_elems32 <= 0)
		return;
	for (int level = 0; level < kLevels; level++)
	{
		const LevelParams &p = lp[level];
		if (fwd && level > 0 && !p.P.fp16 && p.P.pitch >= 76 && p.P.rows >= 72)
		{
			LevelTileMap &m = fwd[level];
			uint32_t valid = 0;
			for (int comp = 0; comp < kComponents; comp++)
			{
				if (level == 1 && comp != 0 && !g.chroma444)
					continue; // 4:2:0 chroma enters at level 1 from its plane
				if (p.prev_ll[comp] % p.P.pitch == 0)
				{
					m.row[comp][0] = int32_t(p.prev_ll[comp] / p.P.pitch);
					valid |= 1u << comp;
				}
			}
			if (valid && encode_storage_map(m.map, coef32, g.storage_elems32, p.P.pitch, 76, 72))
				m.valid = valid;
		}
		if (inv && !p.L.fp16 && p.L.pitch >= 40 && p.L.rows >= 36)
		{
			LevelTileMap &m = inv[level];
			uint32_t valid = 0;
			for (int comp = 0; comp < kComponents; comp++)
			{
				if (level == 0 && comp != 0 && !g.chroma444)
					continue;
				bool rows_ok = true;
				for (int band = 0; band < 4; band++)
				{
					rows_ok = rows_ok && p.band[comp][band].offset % p.L.pitch == 0;
					m.row[comp][band] = int32_t(p.band[comp][band].offset / p.L.pitch);
				}
				if (rows_ok)
					valid |= 1u << comp;
			}
			if (valid && encode_storage_map(m.map, coef32, g.storage_elems32, p.L.pitch, 40, 36))
				m.valid = valid;
			const char *fail = getenv("PYROWAVE_TEST_FAIL_TILE_WAIT");
			m.test_fail_wait = fail && atoi(fail) != 0 ? 1u : 0u;
		}
	}
}

struct pyrowave_encoder_opaque
{
	pyrowave_device device = nullptr;
	Geometry g = {};
	std::vector<uint32_t> jobs;
	uint32_t fp16_mask = 0;
	bool allocated = false;

	LevelParams lp[kLevels] = {}; // kernel parameter blocks derived from g
	BlockParams bp = {};
	float *coef32 = nullptr;
	__half *coef16 = nullptr;
	uint16_t *mag16 = nullptr;
	uint32_t *code_words = nullptr;
	uint16_t *rd_cost = nullptr;
	uint8_t *rd_bucket = nullptr;
	float *rd_dist = nullptr;
	RateControlState *rc = nullptr;
	int32_t *quant = nullptr;
	uint32_t *block_meta = nullptr;
	uint32_t *stream_buf = nullptr;
	uint32_t stream_capacity = 0;
	uint32_t *jobs_d = nullptr;
	LevelTileMap in_maps[kLevels] = {}; // TMA maps of the forward transform's LL inputs
	uint8_t *in_planes[3] = {};
	int in_pitch[3] = {};

	uint32_t *h_meta = nullptr;
	uint32_t *h_stream = nullptr;
	uint32_t h_stream_capacity = 0;
	uint32_t *h_total = nullptr;
	cudaEvent_t done = nullptr;
	cudaEvent_t encoded = nullptr; // recorded after every encode launch (device path included)
	bool has_frame = false;     // a completed CPU-visible encode exists
	bool has_device_frame = false;
	uint32_t sequence_count = 0;
	StageEvents timing;
	CapturedGraph graph;
	KernelNode node_dwt[kLevels];
	int small_level = kLevels; // levels >= this: transform only, then one quantiser launch over their blocks
	int small_blocks = 0;      // 32x32 blocks of those levels (a prefix in block index order)
	KernelNode node_resolve;
	// Tile dataflow of the captured encode: counters right after the rate-control
	// state in the same allocation (one clear covers both).
	int tile_counters = 0;
	uint32_t fused_ctas = 0;
	// Packing analysis (allocated by its first call): the 64x64 region table and
	// the device accumulators.
	int32_t *analysis_regions = nullptr;
	int analysis_region_count = 0;
	PackingAnalysisAccum *analysis_acc = nullptr;
	uint32_t *tile_done() const { return reinterpret_cast<uint32_t *>(rc + 1); }
	size_t rc_bytes() const { return sizeof(RateControlState) + size_t(tile_counters) * 4; }

	EncodeBuffers buffers() const
	{
		EncodeBuffers b;
		b.coef32 = coef32;
		b.coef16 = coef16;
		b.mag16 = mag16;
		b.code_words = code_words;
		b.rd_cost = rd_cost;
		b.rd_bucket = rd_bucket;
		b.rd_dist = rd_dist;
		b.rc = rc;
		b.quant = quant;
		b.block_meta = block_meta;
		b.stream = stream_buf;
		b.stream_capacity_words = stream_capacity;
		b.jobs = jobs_d;
		b.tile_done = nullptr; // set only for the captured single-frame encode
		return b;
	}

	void release()
	{
		if (device)
			cudaStreamSynchronize(device->stream);
		dev_free(coef32);
		dev_free(coef16);
		dev_free(mag16);
		dev_free(code_words);
		dev_free(rd_cost);
		dev_free(rd_bucket);
		dev_free(rd_dist);
		dev_free(rc);
		dev_free(quant);
		dev_free(block_meta);
		dev_free(stream_buf);
		dev_free(jobs_d);
		dev_free(analysis_regions);
		dev_free(analysis_acc);
		analysis_regions = nullptr;
		analysis_acc = nullptr;
		analysis_region_count = 0;
		for (auto &p : in_planes)
			dev_free(p);
		host_free(h_meta);
		host_free(h_stream);
		host_free(h_total);
		if (done)
			cudaEventDestroy(done);
		done = nullptr;
		if (encoded)
			cudaEventDestroy(encoded);
		encoded = nullptr;
		timing.destroy();
		graph.destroy();
		coef32 = nullptr;
		coef16 = nullptr;
		mag16 = nullptr;
		code_words = nullptr;
		rd_cost = nullptr;
		rd_bucket = nullptr;
		rd_dist = nullptr;
		rc = nullptr;
		quant = nullptr;
		block_meta = nullptr;
		stream_buf = nullptr;
		stream_capacity = 0;
		jobs_d = nullptr;
		for (auto &p : in_planes)
			p = nullptr;
		h_meta = h_stream = h_total = nullptr;
		h_stream_capacity = 0;
		has_frame = has_device_frame = false;
		allocated = false;
	}

	pyrowave_result allocate()
	{
		if (allocated)
			return PYROWAVE_SUCCESS;
		if (!build_geometry(g, jobs, g.width, g.height, g.chroma444 != 0, fp16_mask))
			return PYROWAVE_ERROR_INVALID_ARGUMENT;
		for (int level = 0; level < kLevels; level++)
			lp[level] = make_level_params(g, level);
		bp = make_block_params(g);
		small_level_split(g, small_level, small_blocks);
		tile_counters = setup_tile_dataflow(g, small_level, lp, bp, fused_ctas);
		(void)resolve_cluster_max();
		bool ok = true;
		coef32 = dev_alloc<float>(size_t(g.storage_elems32), ok);
		coef16 = dev_alloc<__half>(size_t(g.storage_elems16), ok);
		mag16 = dev_alloc<uint16_t>(size_t(g.block_count_32x32) * 1024, ok);
		code_words = dev_alloc<uint32_t>(size_t(g.block_count_8x8), ok);
		rd_cost = dev_alloc<uint16_t>(size_t(g.block_count_32x32) * 16, ok);
		rd_bucket = dev_alloc<uint8_t>(size_t(g.block_count_32x32) * 16, ok);
		rd_dist = dev_alloc<float>(size_t(g.block_count_32x32) * 16, ok);
		rc = reinterpret_cast<RateControlState *>(dev_alloc<uint8_t>(rc_bytes(), ok));
		quant = dev_alloc<int32_t>(size_t(g.block_count_32x32), ok);
		block_meta = dev_alloc<uint32_t>(size_t(g.block_count_32x32) * 2, ok);
		jobs_d = dev_alloc<uint32_t>(jobs.size(), ok);
		h_meta = host_alloc<uint32_t>(size_t(g.block_count_32x32) * 2, ok);
		h_total = host_alloc<uint32_t>(4, ok);
		if (ok && cudaEventCreateWithFlags(&done, cudaEventDisableTiming) != cudaSuccess)
			ok = false;
		if (ok && cudaEventCreateWithFlags(&encoded, cudaEventDisableTiming) != cudaSuccess)
			ok = false;
		if (!ok)
		{
			release();
			return PYROWAVE_ERROR_OUT_OF_DEVICE_MEMORY;
		}
		cudaMemcpy(jobs_d, jobs.data(), jobs.size() * 4, cudaMemcpyHostToDevice);
		build_tile_maps(g, lp, coef32, in_maps, nullptr);
		allocated = true;
		return PYROWAVE_SUCCESS;
	}

	pyrowave_result ensure_stream_capacity(uint32_t words)
	{
		if (words <= stream_capacity)
			return PYROWAVE_SUCCESS;
		cudaStreamSynchronize(device->stream);
		dev_free(stream_buf);
		bool ok = true;
		stream_buf = dev_alloc<uint32_t>(words, ok);
		stream_capacity = ok ? words : 0;
		return ok ? PYROWAVE_SUCCESS : PYROWAVE_ERROR_OUT_OF_DEVICE_MEMORY;
	}

	pyrowave_result ensure_host_capacity(uint32_t words)
	{
		if (words <= h_stream_capacity)
			return PYROWAVE_SUCCESS;
		host_free(h_stream);
		bool ok = true;
		h_stream = host_alloc<uint32_t>(words, ok);
		h_stream_capacity = ok ? words : 0;
		return ok ? PYROWAVE_SUCCESS : PYROWAVE_ERROR_OUT_OF_HOST_MEMORY;
	}

	pyrowave_result ensure_input_planes()
	{
		if (in_planes[0])
			return PYROWAVE_SUCCESS;
		bool ok = true;
		for (int c = 0; c < 3; c++)
		{
			// Rows are sized for 16-bit samples and for the interleaved CbCr plane of NV12.
			in_pitch[c] = align_up(2 * g.plane_width[c], 128);
			in_planes[c] = dev_alloc<uint8_t>(size_t(in_pitch[c]) * g.plane_height[c], ok);
		}
		return ok ? PYROWAVE_SUCCESS : PYROWAVE_ERROR_OUT_OF_DEVICE_MEMORY;
	}

	// Validates the budget (pyrowave_c.cpp:957-961) and returns the target in
	// words after the 8-byte sequence header (pyrowave_encoder.cpp:289-324).
	static bool budget_words(const pyrowave_rate_control *rc, uint32_t &target_words, uint32_t &capacity_words)
	{
		if (!rc)
			return false;
		uint64_t target = uint64_t(rc->maximum_bitstream_size) & ~uint64_t(3);
		if (target == 0 || target > 0xffffffffull)
			return false;
		uint64_t payload = target >= 8 ? target - 8 : target;
		target_words = uint32_t(payload / 4);
		capacity_words = target_words + 2;
		return true;
	}

	ResolveParams dataflow_resolve_params(uint32_t target_words) const
	{
		ResolveParams rp = make_resolve_params(g, target_words, sequence_count);
		rp.fused_ctas = fused_ctas;
		return rp;
	}

	// Queue the encode of resident input planes (pyrowave_encoder.cpp:1153-1183).
	pyrowave_result enqueue(const PlaneInput &in, const pyrowave_rate_control *rc_in, cudaStream_t s)
	{
		uint32_t target_words, capacity;
		if (!budget_words(rc_in, target_words, capacity))
			return PYROWAVE_ERROR_INVALID_ARGUMENT;
		pyrowave_result r = ensure_stream_capacity(capacity);
		if (r != PYROWAVE_SUCCESS)
			return r;
		sequence_count = (sequence_count + 1) & 7u;
		EncodeBuffers b = buffers();
		b.tile_done = tile_done();
		timing.collect(device);
		timing.prepare(device);
		const uint64_t key = uint64_t(stream_capacity) | (device->stage_timing ? (1ull << 40) : 0ull);
		if (!graph.valid() || graph.key != key)
		{
			// Capture the frame's kernel sequence once (pyrowave_encoder.cpp:1153-1183:
			// clear, DWT + quant + analyze per level, resolve, pack).
			if (!graph.begin(s))
				return PYROWAVE_ERROR_GENERIC;
			bool ok = true;
			timing.begin(device, s);
			cudaMemsetAsync(rc, 0, rc_bytes(), s);
			static const char *const dwt_tags[kLevels] = {"dwt0", "dwt1", "dwt2", "dwt3", "dwt4"};
			const bool pdl = !device->stage_timing; // event nodes between kernels break programmatic edges
			// The small levels (few tiles each) transform only, each level one launch;
			// one launch then quantises all their blocks, so no level's quantiser
			// waits on the critical path of the transforms.
			for (int level = 0; level < kLevels; level++)
			{
				launch_dwt_forward_level(lp[level], in, b, &in_maps[level], level < small_level, pdl && level > 0, s);
				ok = ok && last_captured_node(s, node_dwt[level]);
				timing.mark(device, s, dwt_tags[level]);
			}
			if (small_blocks > 0)
			{
				launch_quant_pretransformed(bp, b, small_blocks, pdl, s);
				timing.mark(device, s, "quant");
			}
			launch_resolve(dataflow_resolve_params(target_words), b, s);
			ok = ok && last_captured_node(s, node_resolve);
			timing.mark(device, s, "resolve");
			launch_pack(bp, b, s);
			timing.mark(device, s, "pack");
			ok = graph.end(s, key) && ok;
			if (!ok)
			{
				graph.destroy();
				(void)cudaGetLastError();
				return PYROWAVE_ERROR_GENERIC;
			}
		}
		else
		{
			PlaneInput pin = in;
			ResolveParams rp = dataflow_resolve_params(target_words);
			bool ok = true;
			for (int level = 0; level < kLevels; level++)
			{
				int fused = forward_fused_mode(lp[level], level < small_level);
				ok = ok && set_kernel_args(graph.exec, node_dwt[level], lp[level], pin, b, fused, in_maps[level]);
			}
			ok = ok && set_kernel_args(graph.exec, node_resolve, rp, b);
			if (!ok)
			{
				graph.destroy();
				(void)cudaGetLastError();
				return PYROWAVE_ERROR_GENERIC;
			}
		}
		if (!cuda_ok(cudaGraphLaunch(graph.exec, s), "cudaGraphLaunch"))
			return PYROWAVE_ERROR_GENERIC;
		timing.launched(device);
		cudaEventRecord(encoded, s);
		has_device_frame = true;
		return PYROWAVE_SUCCESS;
	}

	// Copy the result to pinned host memory for compute_num_packets / packetize.
	pyrowave_result queue_readback(cudaStream_t s)
	{
		pyrowave_result r = ensure_host_capacity(stream_capacity);
		if (r != PYROWAVE_SUCCESS)
			return r;
		cudaMemcpyAsync(h_meta, block_meta, size_t(g.block_count_32x32) * 8, cudaMemcpyDeviceToHost, s);
		cudaMemcpyAsync(h_total, &rc->error, 8, cudaMemcpyDeviceToHost, s); // error, total_words
		cudaMemcpyAsync(h_stream, stream_buf, size_t(stream_capacity) * 4, cudaMemcpyDeviceToHost, s);
		cudaEventRecord(done, s);
		has_frame = true;
		return PYROWAVE_SUCCESS;
	}

	bool wait()
	{
		if (!has_frame)
			return false;
		cudaEventSynchronize(done);
		return true;
	}
};

namespace pw
{
uint32_t encoder_frames(const pyrowave_encoder_opaque *encoder) { return encoder ? encoder->sequence_count : 0; }
void encoder_set_frames(pyrowave_encoder_opaque *encoder, uint32_t frames)
{
	if (encoder)
		encoder->sequence_count = frames & 7u;
}
} // namespace pw

// Growable array of 32-bit words in page-locked host memory: the parser's
// payload, uploaded without a staging copy when the caller waits for the decode.
struct PinnedWords
{
	uint32_t *ptr = nullptr;
	size_t n = 0, cap = 0;
	PinnedWords() = default;
	PinnedWords(const PinnedWords &) = delete;
	PinnedWords &operator=(const PinnedWords &) = delete;
	~PinnedWords()
	{
		if (ptr)
			cudaFreeHost(ptr);
	}
	size_t size() const { return n; }
	bool empty() const { return n == 0; }
	uint32_t *data() { return ptr; }
	const uint32_t *data() const { return ptr; }
	void clear() { n = 0; }
	bool reserve(size_t c)
	{
		if (c <= cap)
			return true;
		uint32_t *np = nullptr;
		if (cudaHostAlloc(reinterpret_cast<void **>(&np), c * 4, cudaHostAllocDefault) != cudaSuccess)
			return false;
		if (n)
			memcpy(np, ptr, n * 4);
		if (ptr)
			cudaFreeHost(ptr);
		ptr = np;
		cap = c;
		return true;
	}
	bool resize(size_t m)
	{
		if (m > cap && !reserve(std::max(m, cap * 2)))
			return false;
		n = m;
		return true;
	}
};

struct pyrowave_decoder_opaque
{
	pyrowave_device device = nullptr;
	Geometry g = {};
	std::vector<uint32_t> jobs;
	uint32_t fp16_mask = 0;
	bool allocated = false;

	LevelParams lp[kLevels] = {};
	BlockParams bp = {};
	float *coef32 = nullptr;
	__half *coef16 = nullptr;
	uint32_t *jobs_d = nullptr;
	uint32_t *offsets_d = nullptr;
	uint32_t *payload_d = nullptr;
	size_t payload_capacity = 0;
	uint8_t *out_planes[3] = {};
	int out_pitch[3] = {};
	uint32_t *h_upload = nullptr;
	size_t h_upload_capacity = 0;
	StageEvents timing;
	CapturedGraph graph_full, graph_idwt;
	KernelNode node_dequant;
	KernelNode node_idwt_full[kLevels], node_idwt_only[kLevels];

	LevelTileMap band_maps[kLevels] = {}; // TMA maps of the FP32 bands (inverse transform tile loads)
	DecodeState *state_d = nullptr;  // per-decode state: error bits
	uint32_t *error_d = nullptr;     // &state_d->error: kDecodeError* bits of the last decode (cleared by each decode)
	uint32_t *h_error = nullptr;     // page-locked copy of error_d
	cudaEvent_t decode_done = nullptr; // recorded after every decode launch
	bool decode_pending = false;
	// Device-side packet assembly (pw_packets.cu): per-packet tables, grown on demand.
	uint32_t *pk_tables = nullptr;
	uint8_t *pk_state = nullptr;
	uint32_t *pk_summaries = nullptr;
	size_t pk_capacity = 0; // packets
	uint32_t *pk_items = nullptr;
	size_t pk_items_capacity = 0; // words
	unsigned long long *pk_first = nullptr;
	PacketStatus *pk_status = nullptr;
	PacketStatus *pk_status_h = nullptr;
	uint32_t *pk_counter = nullptr;
	cudaEvent_t pk_done = nullptr;
	bool pk_pending = false;

	// Parser state (pyrowave_decoder.cpp:24-39).
	std::vector<uint32_t> offsets;
	PinnedWords payload;
	int decoded_blocks = 0;
	int total_blocks_in_sequence = 0;
	uint32_t last_seq = UINT32_MAX;
	bool decoded_frame_for_current_sequence = false;

	void clear()
	{
		std::fill(offsets.begin(), offsets.end(), UINT32_MAX);
		decoded_blocks = 0;
		last_seq = UINT32_MAX;
		decoded_frame_for_current_sequence = false;
		total_blocks_in_sequence = g.block_count_32x32;
		payload.clear();
	}

	// Append one coded block; the first copy of a block index wins.
	bool add_block(const uint8_t *data, uint32_t block_index, uint32_t payload_words)
	{
		uint32_t &off = offsets[block_index];
		if (off != UINT32_MAX)
			return true;
		decoded_blocks++;
		off = uint32_t(payload.size());
		if (payload_words < 2)
			return false;
		size_t base = payload.size();
		if (!payload.resize(base + payload_words))
			return false;
		memcpy(payload.data() + base, data, size_t(payload_words) * 4);
		return true;
	}

	// Packet parser with the reference's sequence handling (pyrowave_decoder.cpp:154-262):
	// a start-of-frame or block header from an older sequence (3-bit wrapping
	// difference > 3) is dropped, a newer one restarts the frame.
	bool push_packet(const uint8_t *data, size_t size)
	{
		while (size >= 8)
		{
			uint32_t w0, w1;
			memcpy(&w0, data, 4);
			memcpy(&w1, data + 4, 4);
			const uint32_t seq = (w0 >> 28) & 7u;
			if ((w0 >> 31) & 1u)
			{
				// BitstreamSequenceHeader (bitstream.md:250-265).
				const uint32_t chroma_resolution = (w1 >> 26) & 1u;
				if (chroma_resolution != uint32_t(g.chroma444))
					return false;
				const uint32_t diff = (seq - last_seq) & 7u;
				if (last_seq != UINT32_MAX && diff > 3)
					return true;
				if (last_seq == UINT32_MAX || diff != 0)
				{
					clear();
					last_seq = seq;
				}
				const uint32_t code = (w1 >> 24) & 3u;
				if (code != 0)
					return false;
				if (int(w0 & 0x3fffu) + 1 != g.width || int((w0 >> 14) & 0x3fffu) + 1 != g.height)
					return false;
				total_blocks_in_sequence = int(w1 & 0xffffffu);
				data += 8;
				size -= 8;
				continue;
			}
			const uint32_t words = (w0 >> 16) & 0xfffu;
			const size_t packet_size = size_t(words) * 4;
			if (packet_size > size)
				return false;
			bool restart;
			if (last_seq == UINT32_MAX)
				restart = true;
			else
			{
				const uint32_t diff = (seq - last_seq) & 7u;
				if (diff > 3)
					return true;
				restart = diff != 0;
			}
			if (restart)
			{
				clear();
				last_seq = seq;
			}
			const uint32_t block_index = (w1 >> 8) & 0xffffffu;
			if (block_index >= uint32_t(g.block_count_32x32))
				return false;
			if (!add_block(data, block_index, words))
				return false;
			data += packet_size;
			size -= packet_size;
		}
		return size == 0;
	}

	bool decode_is_ready(bool allow_partial) const
	{
		if (decoded_frame_for_current_sequence || last_seq == UINT32_MAX)
			return false;
		if (decoded_blocks < total_blocks_in_sequence)
			if (!allow_partial || decoded_blocks <= total_blocks_in_sequence / 2)
				return false;
		return true;
	}

	void release()
	{
		if (device)
			cudaStreamSynchronize(device->stream);
		dev_free(coef32);
		dev_free(coef16);
		dev_free(jobs_d);
		dev_free(offsets_d);
		dev_free(payload_d);
		for (auto &p : out_planes)
			dev_free(p);
		host_free(h_upload);
		dev_free(pk_tables);
		dev_free(pk_state);
		dev_free(pk_summaries);
		dev_free(pk_items);
		dev_free(pk_first);
		dev_free(state_d);
		state_d = nullptr;
		error_d = nullptr;
		host_free(h_error);
		h_error = nullptr;
		if (decode_done)
			cudaEventDestroy(decode_done);
		decode_done = nullptr;
		decode_pending = false;
		dev_free(pk_status);
		dev_free(pk_counter);
		host_free(pk_status_h);
		if (pk_done)
			cudaEventDestroy(pk_done);
		pk_tables = nullptr;
		pk_state = nullptr;
		pk_summaries = nullptr;
		pk_items = nullptr;
		pk_items_capacity = 0;
		pk_first = nullptr;
		pk_status = nullptr;
		pk_counter = nullptr;
		pk_status_h = nullptr;
		pk_done = nullptr;
		pk_capacity = 0;
		pk_pending = false;
		timing.destroy();
		graph_full.destroy();
		graph_idwt.destroy();
		coef32 = nullptr;
		coef16 = nullptr;
		jobs_d = offsets_d = payload_d = nullptr;
		payload_capacity = 0;
		for (auto &p : out_planes)
			p = nullptr;
		h_upload = nullptr;
		h_upload_capacity = 0;
		allocated = false;
	}

	pyrowave_result allocate()
	{
		if (allocated)
			return PYROWAVE_SUCCESS;
		if (!build_geometry(g, jobs, g.width, g.height, g.chroma444 != 0, fp16_mask))
			return PYROWAVE_ERROR_INVALID_ARGUMENT;
		for (int level = 0; level < kLevels; level++)
			lp[level] = make_level_params(g, level);
		bp = make_block_params(g);
		bool ok = true;
		coef32 = dev_alloc<float>(size_t(g.storage_elems32), ok);
		coef16 = dev_alloc<__half>(size_t(g.storage_elems16), ok);
		jobs_d = dev_alloc<uint32_t>(jobs.size(), ok);
		offsets_d = dev_alloc<uint32_t>(size_t(g.block_count_32x32), ok);
		if (!ok)
		{
			release();
			return PYROWAVE_ERROR_OUT_OF_DEVICE_MEMORY;
		}
		cudaMemcpy(jobs_d, jobs.data(), jobs.size() * 4, cudaMemcpyHostToDevice);
		state_d = dev_alloc<DecodeState>(1, ok);
		error_d = state_d ? &state_d->error : nullptr;
		h_error = host_alloc<uint32_t>(1, ok);
		if (state_d)
			cudaMemset(state_d, 0, sizeof(DecodeState));
		if (ok && cudaEventCreateWithFlags(&decode_done, cudaEventDisableTiming) != cudaSuccess)
			ok = false;
		build_tile_maps(g, lp, coef32, nullptr, band_maps);
		if (!ok)
		{
			release();
			return PYROWAVE_ERROR_OUT_OF_DEVICE_MEMORY;
		}
		if (offsets.size() != size_t(g.block_count_32x32))
		{
			offsets.assign(size_t(g.block_count_32x32), UINT32_MAX);
			payload.reserve(1 << 18);
			clear();
		}
		allocated = true;
		return PYROWAVE_SUCCESS;
	}

	pyrowave_result ensure_payload(size_t words)
	{
		words += 4; // keep one extra word for sign reads at the very end
		if (words > payload_capacity)
		{
			dev_free(payload_d);
			bool ok = true;
			size_t cap = std::max<size_t>(words * 2, 1 << 16);
			payload_d = dev_alloc<uint32_t>(cap, ok);
			payload_capacity = ok ? cap : 0;
			if (!ok)
				return PYROWAVE_ERROR_OUT_OF_DEVICE_MEMORY;
		}
		size_t need = words + size_t(g.block_count_32x32);
		if (need > h_upload_capacity)
		{
			host_free(h_upload);
			bool ok = true;
			size_t cap = std::max<size_t>(need * 2, 1 << 16);
			h_upload = host_alloc<uint32_t>(cap, ok);
			h_upload_capacity = ok ? cap : 0;
			if (!ok)
				return PYROWAVE_ERROR_OUT_OF_HOST_MEMORY;
		}
		return PYROWAVE_SUCCESS;
	}

	pyrowave_result ensure_output_planes()
	{
		if (out_planes[0])
			return PYROWAVE_SUCCESS;
		bool ok = true;
		for (int c = 0; c < 3; c++)
		{
			out_pitch[c] = align_up(2 * g.plane_width[c], 128); // room for 16-bit samples
			out_planes[c] = dev_alloc<uint8_t>(size_t(out_pitch[c]) * g.plane_height[c], ok);
		}
		return ok ? PYROWAVE_SUCCESS : PYROWAVE_ERROR_OUT_OF_DEVICE_MEMORY;
	}

	// Dequantise + inverse transform (pyrowave_decoder.cpp:796-830).
	// Dequantise + inverse transform (pyrowave_decoder.cpp:796-830), as one graph launch.
	bool run(const DecodeInput &in_args, const PlaneOutput &out, cudaStream_t s, bool dequant)
	{
		DecodeInput in = in_args;
		in.error = error_d;
		in.state = state_d;
		timing.collect(device);
		timing.prepare(device);
		CapturedGraph &graph = dequant ? graph_full : graph_idwt;
		const uint64_t key = device->stage_timing ? 1ull : 0ull;
		if (!graph.valid() || graph.key != key)
		{
			if (!graph.begin(s))
				return false;
			bool ok = true;
			timing.begin(device, s);
			const bool pdl = !device->stage_timing; // event nodes between kernels break programmatic edges
			// The dequantiser clears the decode state before any inverse level runs;
			// without it the graph starts with a clear of its own.
			if (!dequant)
				cudaMemsetAsync(state_d, 0, sizeof(DecodeState), s);
			if (dequant)
			{
				launch_dequant(bp, in, 0, g.block_count_32x32, false, s);
				ok = ok && last_captured_node(s, node_dequant);
				timing.mark(device, s, "dequant");
			}
			// Programmatic launches follow a kernel only (not the clear of an inverse-only decode).
			static const char *const idwt_tags[kLevels] = {"idwt0", "idwt1", "idwt2", "idwt3", "idwt4"};
			for (int level = kLevels - 1; level >= 0; level--)
			{
				launch_idwt_level(lp[level], in, out, &band_maps[level], pdl && (dequant || level < kLevels - 1), s);
				ok = ok && last_captured_node(s, dequant ? node_idwt_full[level] : node_idwt_only[level]);
				timing.mark(device, s, idwt_tags[level]);
			}
			ok = graph.end(s, key) && ok;
			if (!ok)
			{
				graph.destroy();
				(void)cudaGetLastError();
				return false;
			}
		}
		else
		{
			DecodeInput din = in;
			PlaneOutput pout = out;
			bool ok = true;
			if (dequant)
			{
				int first = 0;
				ok = set_kernel_args(graph.exec, node_dequant, bp, din, first);
			}
			for (int level = 0; level < kLevels; level++)
				ok = ok && set_kernel_args(graph.exec, dequant ? node_idwt_full[level] : node_idwt_only[level], lp[level],
				                           din, pout, band_maps[level]);
			if (!ok)
			{
				graph.destroy();
				(void)cudaGetLastError();
				return false;
			}
		}
		if (!cuda_ok(cudaGraphLaunch(graph.exec, s), "cudaGraphLaunch"))
			return false;
		timing.launched(device);
		cudaEventRecord(decode_done, s);
		decode_pending = true;
		decoded_frame_for_current_sequence = true;
		return true;
	}

	// Error bits of the last decode (waits for it); 0 when none was launched.
	bool last_error(uint32_t &bits)
	{
		bits = 0;
		if (!decode_pending)
			return true;
		if (!cuda_ok(cudaEventSynchronize(decode_done), "cudaEventSynchronize") ||
		    !cuda_ok(cudaMemcpy(h_error, error_d, sizeof(uint32_t), cudaMemcpyDeviceToHost), "cudaMemcpy"))
			return false;
		bits = *h_error;
		return true;
	}

	// Upload the parsed frame and decode it.
	// Assemble the frame from packets in device memory on the GPU, then decode it.
	pyrowave_result decode_packets(const void *data, size_t data_bytes, const pyrowave_packet *packets, uint32_t count,
	                               const PlaneOutput &out, cudaStream_t s)
	{
		bool ok = true;
		if (!pk_first)
		{
			pk_first = dev_alloc<unsigned long long>(size_t(g.block_count_32x32), ok);
			pk_status = dev_alloc<PacketStatus>(1, ok);
			pk_counter = dev_alloc<uint32_t>(1, ok);
			pk_status_h = host_alloc<PacketStatus>(1, ok);
			if (ok && cudaMemset(pk_counter, 0, sizeof(uint32_t)) != cudaSuccess)
				ok = false;
			if (ok && cudaEventCreateWithFlags(&pk_done, cudaEventDisableTiming) != cudaSuccess)
				ok = false;
		}
		if (ok && count > pk_capacity)
		{
			cudaStreamSynchronize(s);
			dev_free(pk_tables);
			dev_free(pk_state);
			dev_free(pk_summaries);
			const size_t cap = std::max<size_t>(count, 256);
			pk_tables = dev_alloc<uint32_t>(cap * 18, ok);
			pk_state = dev_alloc<uint8_t>(cap, ok);
			pk_summaries = dev_alloc<uint32_t>(cap * 8, ok);
			pk_capacity = ok ? cap : 0;
		}
		const size_t data_words = (data_bytes + 3) / 4;
		if (ok && data_words > pk_items_capacity)
		{
			cudaStreamSynchronize(s);
			dev_free(pk_items);
			const size_t cap = std::max<size_t>(data_words, 1 << 16);
			pk_items = dev_alloc<uint32_t>(cap, ok);
			pk_items_capacity = ok ? cap : 0;
		}
		if (!ok)
			return PYROWAVE_ERROR_OUT_OF_DEVICE_MEMORY;
		PacketParams pp = {};
		pp.data = static_cast<const uint32_t *>(data);
		pp.data_bytes = data_bytes;
		pp.packets = reinterpret_cast<const unsigned long long *>(packets);
		pp.count = int32_t(count);
		pp.width = g.width;
		pp.height = g.height;
		pp.chroma444 = g.chroma444;
		pp.block_count = g.block_count_32x32;
		pp.tables = pk_tables;
		pp.state_before = pk_state;
		pp.summaries = pk_summaries;
		pp.items = pk_items;
		pp.first = pk_first;
		pp.counter = pk_counter;
		pp.status = pk_status;
		launch_packet_assembly(pp, s);
		DecodeInput in = {};
		in.keys = pk_first;
		in.payload = pp.data;
		in.payload_words = uint32_t(data_bytes / 4);
		in.jobs = jobs_d;
		in.coef32 = coef32;
		in.coef16 = coef16;
		if (!run(in, out, s, true))
			return PYROWAVE_ERROR_GENERIC;
		cudaEventRecord(pk_done, s);
		pk_pending = true;
		return launches_ok("kernel launch") ? PYROWAVE_SUCCESS : PYROWAVE_ERROR_GENERIC;
	}

	// `waits`: the caller synchronizes with `s` before the parser can change,
	// so the payload is uploaded straight from the parser's page-locked array;
	// otherwise it is staged first.
	pyrowave_result decode_parsed(const PlaneOutput &out, cudaStream_t s, bool waits = false)
	{
		pyrowave_result r = ensure_payload(payload.size());
		if (r != PYROWAVE_SUCCESS)
			return r;
		const size_t nb = size_t(g.block_count_32x32);
		memcpy(h_upload, offsets.data(), nb * 4);
		cudaMemcpyAsync(offsets_d, h_upload, nb * 4, cudaMemcpyHostToDevice, s);
		if (!payload.empty())
		{
			const uint32_t *src = payload.data();
			if (!waits)
			{
				memcpy(h_upload + nb, payload.data(), payload.size() * 4);
				src = h_upload + nb;
			}
			cudaMemcpyAsync(payload_d, src, payload.size() * 4, cudaMemcpyHostToDevice, s);
		}
		DecodeInput in = {};
		in.offsets = offsets_d;
		in.payload = payload_d;
		in.payload_words = uint32_t(payload.size());
		in.jobs = jobs_d;
		in.coef32 = coef32;
		in.coef16 = coef16;
		if (!run(in, out, s, true))
			return PYROWAVE_ERROR_GENERIC;
		return launches_ok("kernel launch") ? PYROWAVE_SUCCESS : PYROWAVE_ERROR_GENERIC;
	}
};

// ---------------------------------------------------------------------------
namespace
{
cudaStream_t pick_stream(pyrowave_device dev, pyrowave_cuda_stream s)
{
	return s ? reinterpret_cast<cudaStream_t>(s) : dev->stream;
}

bool plane_dims(pyrowave_chroma_subsampling chroma, int width, int height, int plane, int &w, int &h)
{
	w = width;
	h = height;
	if (plane != 0 && chroma == PYROWAVE_CHROMA_SUBSAMPLING_420)
	{
		w /= 2;
		h /= 2;
	}
	return true;
}

pyrowave_result fill_layout(const Geometry &g, uint32_t mask, pyrowave_cuda_layout *layout)
{
	if (!layout)
		return PYROWAVE_ERROR_INVALID_ARGUMENT;
	layout->width = g.width;
	layout->height = g.height;
	layout->chroma444 = g.chroma444;
	layout->aligned_width = g.aligned_width;
	layout->aligned_height = g.aligned_height;
	layout->block_count_8x8 = g.block_count_8x8;
	layout->block_count_32x32 = g.block_count_32x32;
	size_t n = 0;
	for (int level = 0; level < kLevels; level++)
		for (int comp = 0; comp < kComponents; comp++)
			for (int band = 0; band < 4; band++)
				if (g.band[comp][level][band].present)
					n += size_t(g.level[level].width) * g.level[level].height;
	layout->pyramid_size = n;
	layout->fp16_level_mask = mask & 0x1fu;
	return PYROWAVE_SUCCESS;
}
} // namespace

extern "C" {

void pyrowave_get_api_version(uint32_t *major, uint32_t *minor, uint32_t *patch)
{
	*major = PYROWAVE_API_VERSION_MAJOR;
	*minor = PYROWAVE_API_VERSION_MINOR;
	*patch = PYROWAVE_API_VERSION_PATCH;
}

pyrowave_result pyrowave_create_default_device(pyrowave_device *device)
{
	if (!device)
		return PYROWAVE_ERROR_INVALID_ARGUMENT;
	int count = 0;
	if (cudaGetDeviceCount(&count) != cudaSuccess || count == 0)
	{
		(void)cudaGetLastError();
		return PYROWAVE_ERROR_NO_VULKAN;
	}
	auto *dev = new (std::nothrow) pyrowave_device_opaque;
	if (!dev)
		return PYROWAVE_ERROR_OUT_OF_HOST_MEMORY;
	cudaGetDevice(&dev->cuda_device);
	// The library's own stream runs at the highest priority, so its kernels go
	// first when other work shares the GPU.
	int least = 0, greatest = 0;
	cudaDeviceGetStreamPriorityRange(&least, &greatest);
	// A blocking stream: work a caller queues on the legacy default stream (its
	// uploads, or the buffers it prepares) is ordered with the library's work.
	if (cudaStreamCreateWithPriority(&dev->stream, cudaStreamDefault, greatest) != cudaSuccess)
	{
		delete dev;
		return PYROWAVE_ERROR_GENERIC;
	}
	const char *env = getenv("PYROWAVE_STAGE_TIMING");
	dev->stage_timing = env && atoi(env) != 0;
	*device = dev;
	return PYROWAVE_SUCCESS;
}

pyrowave_result pyrowave_create_device(const pyrowave_device_create_info *, pyrowave_device *)
{
	return PYROWAVE_ERROR_NO_VULKAN;
}

pyrowave_result pyrowave_create_device_by_compat(uint32_t vid, uint32_t pid, const pyrowave_uuid *device_uuid,
                                                 const pyrowave_uuid *, const pyrowave_luid *,
                                                 pyrowave_device *device)
{
	if (!device)
		return PYROWAVE_ERROR_INVALID_ARGUMENT;
	if (vid != 0 && vid != 0x10de)
		return PYROWAVE_ERROR_NO_VULKAN;
	(void)pid;
	if (device_uuid)
	{
		int count = 0;
		cudaGetDeviceCount(&count);
		bool found = false;
		for (int i = 0; i < count && !found; i++)
		{
			cudaDeviceProp prop;
			if (cudaGetDeviceProperties(&prop, i) == cudaSuccess &&
			    memcmp(prop.uuid.bytes, device_uuid->uuid, 16) == 0)
			{
				cudaSetDevice(i);
				found = true;
			}
		}
		if (!found)
			return PYROWAVE_ERROR_NO_VULKAN;
	}
	return pyrowave_create_default_device(device);
}

void pyrowave_device_report_performance_stats(pyrowave_device device, pyrowave_message_cb cb, void *userdata, bool reset)
{
	if (!device || !cb)
		return;
	std::lock_guard<std::mutex> g(device->lock);
	for (auto &t : device->timers)
	{
		char msg[256];
		snprintf(msg, sizeof(msg), "%s: %.4f ms per frame\n", t.tag, t.frames ? t.total_ms / double(t.frames) : 0.0);
		cb(userdata, msg);
	}
	if (reset)
		device->timers.clear();
}

void pyrowave_device_get_vk_device_handles(pyrowave_device, VkInstance *vk_instance,
                                           VkPhysicalDevice *vk_physical_device, VkDevice *vk_device)
{
	if (vk_instance)
		*vk_instance = nullptr;
	if (vk_physical_device)
		*vk_physical_device = nullptr;
	if (vk_device)
		*vk_device = nullptr;
}

void pyrowave_device_set_command_buffer(pyrowave_device, VkCommandBuffer) {}

pyrowave_result pyrowave_device_set_queue_type(pyrowave_device device, VkQueueFlagBits)
{
	return device ? PYROWAVE_SUCCESS : PYROWAVE_ERROR_INVALID_ARGUMENT;
}

bool pyrowave_device_confirm_interop_support(pyrowave_device) { return false; }

pyrowave_result pyrowave_cuda_device_set_stage_timing(pyrowave_device device, bool enable)
{
	if (!device)
		return PYROWAVE_ERROR_INVALID_ARGUMENT;
	device->stage_timing = enable;
	return PYROWAVE_SUCCESS;
}

void pyrowave_device_destroy(pyrowave_device device)
{
	if (!device)
		return;
	cudaStreamSynchronize(device->stream);
	cudaStreamDestroy(device->stream);
	delete device;
}

pyrowave_result pyrowave_sync_object_create(const pyrowave_sync_object_create_info *, pyrowave_sync_object *sync)
{
	if (sync)
		*sync = nullptr;
	return PYROWAVE_ERROR_NOT_IMPLEMENTED;
}
VkSemaphore pyrowave_sync_object_get_semaphore(pyrowave_sync_object) { return nullptr; }
pyrowave_result pyrowave_sync_object_export_handle(pyrowave_sync_object, pyrowave_os_handle *)
{
	return PYROWAVE_ERROR_NOT_IMPLEMENTED;
}
pyrowave_result pyrowave_sync_object_cpu_wait(pyrowave_sync_object, uint64_t, uint64_t)
{
	return PYROWAVE_ERROR_NOT_IMPLEMENTED;
}
pyrowave_result pyrowave_sync_object_cpu_signal(pyrowave_sync_object, uint64_t) { return PYROWAVE_ERROR_NOT_IMPLEMENTED; }
void pyrowave_sync_object_destroy(pyrowave_sync_object) {}

pyrowave_result pyrowave_image_create(const pyrowave_image_create_info *, pyrowave_image *image)
{
	if (image)
		*image = nullptr;
	return PYROWAVE_ERROR_NOT_IMPLEMENTED;
}
VkImage pyrowave_image_get_handle(pyrowave_image) { return nullptr; }
pyrowave_result pyrowave_image_get_image_view(pyrowave_image, VkImageAspectFlagBits, VkImageUsageFlagBits,
                                              pyrowave_image_view *)
{
	return PYROWAVE_ERROR_NOT_IMPLEMENTED;
}
void pyrowave_image_destroy(pyrowave_image) {}

// --- encoder ---------------------------------------------------------------
pyrowave_result pyrowave_encoder_create(const pyrowave_encoder_create_info *info, pyrowave_encoder *encoder)
{
	if (!info || !encoder || !info->device)
		return PYROWAVE_ERROR_INVALID_ARGUMENT;
	if (info->width <= 0 || info->height <= 0)
		return PYROWAVE_ERROR_INVALID_ARGUMENT;
	if (info->chroma == PYROWAVE_CHROMA_SUBSAMPLING_420 && ((info->width & 1) || (info->height & 1)))
		return PYROWAVE_ERROR_INVALID_ARGUMENT;
	if (info->chroma != PYROWAVE_CHROMA_SUBSAMPLING_420 && info->chroma != PYROWAVE_CHROMA_SUBSAMPLING_444)
		return PYROWAVE_ERROR_INVALID_ARGUMENT;
	auto *enc = new (std::nothrow) pyrowave_encoder_opaque;
	if (!enc)
		return PYROWAVE_ERROR_OUT_OF_HOST_MEMORY;
	enc->device = info->device;
	std::vector<uint32_t> jobs;
	if (!build_geometry(enc->g, jobs, info->width, info->height, info->chroma == PYROWAVE_CHROMA_SUBSAMPLING_444, 0))
	{
		delete enc;
		return PYROWAVE_ERROR_GENERIC;
	}
	*encoder = enc;
	return PYROWAVE_SUCCESS;
}

pyrowave_result pyrowave_encoder_encode_gpu_synchronous(pyrowave_encoder, const pyrowave_gpu_sync_operation *,
                                                        const pyrowave_gpu_sync_operation *, const pyrowave_gpu_buffers *,
                                                        const pyrowave_rate_control *)
{
	return PYROWAVE_ERROR_NOT_IMPLEMENTED;
}

pyrowave_result pyrowave_encoder_encode_cpu_synchronous(pyrowave_encoder encoder, const pyrowave_cpu_buffer *buffers,
                                                        const pyrowave_rate_control *rate_control)
{
	if (!encoder || !buffers || !rate_control)
		return PYROWAVE_ERROR_INVALID_ARGUMENT;
	const Geometry &g = encoder->g;
	const pyrowave_chroma_subsampling chroma =
	    g.chroma444 ? PYROWAVE_CHROMA_SUBSAMPLING_444 : PYROWAVE_CHROMA_SUBSAMPLING_420;
	// Validation order and rules of pyrowave_c.cpp:1058-1088; the 16-bit planar
	// formats (an extension) follow the rules of their 8-bit counterparts.
	const bool wide = buffers->format == PYROWAVE_CPU_BUFFER_FORMAT_YUV420P16 ||
	                  buffers->format == PYROWAVE_CPU_BUFFER_FORMAT_YUV444P16;
	const pyrowave_cpu_buffer_format fmt = buffers->format == PYROWAVE_CPU_BUFFER_FORMAT_YUV420P16
	                                           ? PYROWAVE_CPU_BUFFER_FORMAT_YUV420P
	                                       : buffers->format == PYROWAVE_CPU_BUFFER_FORMAT_YUV444P16
	                                           ? PYROWAVE_CPU_BUFFER_FORMAT_YUV444P
	                                           : buffers->format;
	const int num_planes = fmt == PYROWAVE_CPU_BUFFER_FORMAT_NV12 ? 2 : 3;
	if (buffers->width != g.width || buffers->height != g.height)
		return PYROWAVE_ERROR_INVALID_ARGUMENT;
	if (chroma == PYROWAVE_CHROMA_SUBSAMPLING_420 && fmt == PYROWAVE_CPU_BUFFER_FORMAT_YUV444P)
		return PYROWAVE_ERROR_INVALID_ARGUMENT;
	if (chroma == PYROWAVE_CHROMA_SUBSAMPLING_444 && fmt != PYROWAVE_CPU_BUFFER_FORMAT_YUV444P)
		return PYROWAVE_ERROR_INVALID_ARGUMENT;
	if (fmt != PYROWAVE_CPU_BUFFER_FORMAT_NV12 && fmt != PYROWAVE_CPU_BUFFER_FORMAT_YUV420P &&
	    fmt != PYROWAVE_CPU_BUFFER_FORMAT_YUV444P)
		return PYROWAVE_ERROR_INVALID_ARGUMENT;
	for (int p = 0; p < num_planes; p++)
	{
		int w, h;
		plane_dims(chroma, g.width, g.height, p, w, h);
		const size_t bpp = ((num_planes == 2 && p == 1) || wide) ? 2 : 1;
		if (wide && ((buffers->row_stride_in_bytes[p] & 1u) || (reinterpret_cast<uintptr_t>(buffers->data[p]) & 1u)))
			return PYROWAVE_ERROR_INVALID_ARGUMENT;
		if (buffers->row_stride_in_bytes[p] < size_t(w) * bpp)
			return PYROWAVE_ERROR_INVALID_ARGUMENT;
		// stride * h > plane size, written so that an absurd stride cannot wrap around
		if (h > 0 && buffers->row_stride_in_bytes[p] > buffers->plane_size_in_bytes[p] / size_t(h))
			return PYROWAVE_ERROR_INVALID_ARGUMENT;
		if (!buffers->data[p])
			return PYROWAVE_ERROR_INVALID_ARGUMENT;
	}
	uint32_t tw, cap;
	if (!pyrowave_encoder_opaque::budget_words(rate_control, tw, cap))
		return PYROWAVE_ERROR_INVALID_ARGUMENT;

	pyrowave_result r = encoder->allocate();
	if (r != PYROWAVE_SUCCESS)
		return r;
	r = encoder->ensure_input_planes();
	if (r != PYROWAVE_SUCCESS)
		return r;
	cudaStream_t s = encoder->device->stream;
	PlaneInput in = {};
	if (num_planes == 2)
	{
		// NV12: the interleaved CbCr plane is uploaded once and read with a
		// 2-byte sample stride (Cb = byte 0, Cr = byte 1).
		int w, h;
		plane_dims(chroma, g.width, g.height, 0, w, h);
		cudaMemcpy2DAsync(encoder->in_planes[0], encoder->in_pitch[0], buffers->data[0], buffers->row_stride_in_bytes[0],
		                  size_t(w), size_t(h), cudaMemcpyHostToDevice, s);
		plane_dims(chroma, g.width, g.height, 1, w, h);
		cudaMemcpy2DAsync(encoder->in_planes[1], size_t(encoder->in_pitch[1]), buffers->data[1],
		                  buffers->row_stride_in_bytes[1], size_t(w) * 2, size_t(h), cudaMemcpyHostToDevice, s);
		in.data[0] = encoder->in_planes[0];
		in.pitch[0] = encoder->in_pitch[0];
		in.xstride[0] = 1;
		in.data[1] = encoder->in_planes[1];
		in.data[2] = encoder->in_planes[1] + 1;
		in.pitch[1] = in.pitch[2] = encoder->in_pitch[1];
		in.xstride[1] = in.xstride[2] = 2;
	}
	else
	{
		const size_t bps = wide ? 2 : 1; // bytes per sample
		in.sample16 = wide ? 1 : 0;
		for (int p = 0; p < 3; p++)
		{
			int w, h;
			plane_dims(chroma, g.width, g.height, p, w, h);
			const size_t stride = buffers->row_stride_in_bytes[p];
			const size_t row = size_t(w) * bps;
			in.data[p] = encoder->in_planes[p];
			in.xstride[p] = int32_t(bps);
			if (stride <= size_t(encoder->in_pitch[p]))
			{
				// One linear copy (row padding included) at the source's own pitch:
				// a pitched copy of narrow rows runs far below the link's bandwidth.
				cudaMemcpyAsync(encoder->in_planes[p], buffers->data[p], stride * size_t(h - 1) + row,
				                cudaMemcpyHostToDevice, s);
				in.pitch[p] = int32_t(stride);
			}
			else
			{
				cudaMemcpy2DAsync(encoder->in_planes[p], encoder->in_pitch[p], buffers->data[p], stride, row,
				                  size_t(h), cudaMemcpyHostToDevice, s);
				in.pitch[p] = encoder->in_pitch[p];
			}
		}
	}
	r = encoder->enqueue(in, rate_control, s);
	if (r != PYROWAVE_SUCCESS)
		return r;
	return encoder->queue_readback(s);
}

pyrowave_result pyrowave_encoder_compute_num_packets(pyrowave_encoder encoder, size_t packet_boundary, size_t *num_packets)
{
	if (!encoder || !num_packets)
		return PYROWAVE_ERROR_INVALID_ARGUMENT;
	if (!encoder->wait())
		return PYROWAVE_ERROR_GENERIC;
	const uint32_t *meta = encoder->h_meta;
	size_t n = 0, in_packet = 8;
	for (int i = 0; i < encoder->g.block_count_32x32; i++)
	{
		const size_t bytes = size_t(meta[2 * i + 1]) * 4;
		if (!bytes)
			continue;
		if (in_packet + bytes > packet_boundary)
		{
			in_packet = 0;
			n++;
		}
		in_packet += bytes;
	}
	if (in_packet)
		n++;
	*num_packets = n;
	return PYROWAVE_SUCCESS;
}

pyrowave_result pyrowave_encoder_packetize(pyrowave_encoder encoder, pyrowave_packet *packets, size_t packet_boundary,
                                           size_t *out_packets, void *bitstream, size_t size)
{
	if (!encoder || !out_packets || !bitstream || !packets)
		return PYROWAVE_ERROR_INVALID_ARGUMENT;
	if (!encoder->wait())
		return PYROWAVE_ERROR_GENERIC;
	if (encoder->h_total[0] != 0)
		return PYROWAVE_ERROR_GENERIC; // device-side consistency check failed
	// The device stream already holds header + blocks contiguously in block
	// order, which is what the packet loop of pyrowave_encoder.cpp:1085-1109
	// produces; only the packet boundaries are computed here.
	const uint32_t *meta = encoder->h_meta;
	size_t n = 0, in_packet = 0, packet_offset = 0, output_offset = 0;
	if (size < 8)
	{
		*out_packets = 0;
		return PYROWAVE_SUCCESS;
	}
	output_offset = 8;
	in_packet = 8;
	bool truncated = false;
	for (int i = 0; i < encoder->g.block_count_32x32; i++)
	{
		const size_t bytes = size_t(meta[2 * i + 1]) * 4;
		if (!bytes)
			continue;
		if (in_packet + bytes > packet_boundary)
		{
			packets[n].offset = packet_offset;
			packets[n].size = in_packet;
			n++;
			in_packet = 0;
			packet_offset = output_offset;
		}
		// An output buffer that is too small ends packetization early
		// (metal/pyrowave_bitstream.cpp:367-368 of the reference).
		if (output_offset + bytes > size)
		{
			truncated = true;
			break;
		}
		output_offset += bytes;
		in_packet += bytes;
	}
	if (!truncated && in_packet)
	{
		packets[n].offset = packet_offset;
		packets[n].size = in_packet;
		n++;
	}
	memcpy(bitstream, encoder->h_stream, output_offset);
	*out_packets = n;
	return PYROWAVE_SUCCESS;
}

void pyrowave_encoder_destroy(pyrowave_encoder encoder)
{
	if (!encoder)
		return;
	encoder->release();
	delete encoder;
}

// --- decoder ---------------------------------------------------------------
bool pyrowave_decoder_device_prefers_fragment_path(pyrowave_device) { return false; }

pyrowave_result pyrowave_decoder_create(const pyrowave_decoder_create_info *info, pyrowave_decoder *decoder)
{
	if (!info || !decoder || !info->device)
		return PYROWAVE_ERROR_INVALID_ARGUMENT;
	if (info->width <= 0 || info->height <= 0)
		return PYROWAVE_ERROR_INVALID_ARGUMENT;
	if (info->chroma == PYROWAVE_CHROMA_SUBSAMPLING_420 && ((info->width & 1) || (info->height & 1)))
		return PYROWAVE_ERROR_INVALID_ARGUMENT;
	if (info->chroma != PYROWAVE_CHROMA_SUBSAMPLING_420 && info->chroma != PYROWAVE_CHROMA_SUBSAMPLING_444)
		return PYROWAVE_ERROR_INVALID_ARGUMENT;
	auto *dec = new (std::nothrow) pyrowave_decoder_opaque;
	if (!dec)
		return PYROWAVE_ERROR_OUT_OF_HOST_MEMORY;
	dec->device = info->device;
	if (!build_geometry(dec->g, dec->jobs, info->width, info->height,
	                    info->chroma == PYROWAVE_CHROMA_SUBSAMPLING_444, 0))
	{
		delete dec;
		return PYROWAVE_ERROR_INVALID_ARGUMENT;
	}
	dec->offsets.assign(size_t(dec->g.block_count_32x32), UINT32_MAX);
	dec->clear();
	*decoder = dec;
	return PYROWAVE_SUCCESS;
}

void pyrowave_decoder_clear(pyrowave_decoder decoder)
{
	if (decoder)
		decoder->clear();
}

pyrowave_result pyrowave_decoder_push_packet(pyrowave_decoder decoder, const void *data, size_t size)
{
	if (!decoder || (!data && size))
		return PYROWAVE_ERROR_INVALID_ARGUMENT;
	return decoder->push_packet(static_cast<const uint8_t *>(data), size) ? PYROWAVE_SUCCESS
	                                                                      : PYROWAVE_ERROR_INVALID_ARGUMENT;
}

bool pyrowave_decoder_decode_is_ready(pyrowave_decoder decoder, bool allow_partial_frame)
{
	return decoder && decoder->decode_is_ready(allow_partial_frame);
}

pyrowave_result pyrowave_decoder_decode_gpu_buffer(pyrowave_decoder, const pyrowave_gpu_sync_operation *,
                                                   const pyrowave_gpu_sync_operation *, const pyrowave_gpu_buffers *)
{
	return PYROWAVE_ERROR_NOT_IMPLEMENTED;
}

pyrowave_result pyrowave_decoder_decode_cpu_buffer_synchronous(pyrowave_decoder decoder, const pyrowave_cpu_buffer *buffers)
{
	if (!decoder || !buffers)
		return PYROWAVE_ERROR_INVALID_ARGUMENT;
	const Geometry &g = decoder->g;
	const pyrowave_chroma_subsampling chroma =
	    g.chroma444 ? PYROWAVE_CHROMA_SUBSAMPLING_444 : PYROWAVE_CHROMA_SUBSAMPLING_420;
	// Validation of pyrowave_c.cpp:1345-1373; the 16-bit planar formats (an
	// extension) follow the rules of their 8-bit counterparts.
	const bool wide = buffers->format == PYROWAVE_CPU_BUFFER_FORMAT_YUV420P16 ||
	                  buffers->format == PYROWAVE_CPU_BUFFER_FORMAT_YUV444P16;
	const pyrowave_cpu_buffer_format fmt = buffers->format == PYROWAVE_CPU_BUFFER_FORMAT_YUV420P16
	                                           ? PYROWAVE_CPU_BUFFER_FORMAT_YUV420P
	                                       : buffers->format == PYROWAVE_CPU_BUFFER_FORMAT_YUV444P16
	                                           ? PYROWAVE_CPU_BUFFER_FORMAT_YUV444P
	                                           : buffers->format;
	const size_t bps = wide ? 2 : 1;
	if (buffers->width != g.width || buffers->height != g.height)
		return PYROWAVE_ERROR_INVALID_ARGUMENT;
	if (fmt == PYROWAVE_CPU_BUFFER_FORMAT_NV12)
		return PYROWAVE_ERROR_INVALID_ARGUMENT;
	if (chroma == PYROWAVE_CHROMA_SUBSAMPLING_420 && fmt == PYROWAVE_CPU_BUFFER_FORMAT_YUV444P)
		return PYROWAVE_ERROR_INVALID_ARGUMENT;
	if (chroma == PYROWAVE_CHROMA_SUBSAMPLING_444 && fmt != PYROWAVE_CPU_BUFFER_FORMAT_YUV444P)
		return PYROWAVE_ERROR_INVALID_ARGUMENT;
	if (fmt != PYROWAVE_CPU_BUFFER_FORMAT_YUV420P && fmt != PYROWAVE_CPU_BUFFER_FORMAT_YUV444P)
		return PYROWAVE_ERROR_INVALID_ARGUMENT;
	for (int p = 0; p < 3; p++)
	{
		int w, h;
		plane_dims(chroma, g.width, g.height, p, w, h);
		if (buffers->row_stride_in_bytes[p] < size_t(w) * bps)
			return PYROWAVE_ERROR_INVALID_ARGUMENT;
		if (wide && ((buffers->row_stride_in_bytes[p] & 1u) || (reinterpret_cast<uintptr_t>(buffers->data[p]) & 1u)))
			return PYROWAVE_ERROR_INVALID_ARGUMENT;
		// stride * h > plane size, written so that an absurd stride cannot wrap around
		if (h > 0 && buffers->row_stride_in_bytes[p] > buffers->plane_size_in_bytes[p] / size_t(h))
			return PYROWAVE_ERROR_INVALID_ARGUMENT;
		if (!buffers->data[p])
			return PYROWAVE_ERROR_INVALID_ARGUMENT;
	}
	pyrowave_result r = decoder->allocate();
	if (r != PYROWAVE_SUCCESS)
		return r;
	r = decoder->ensure_output_planes();
	if (r != PYROWAVE_SUCCESS)
		return r;
	cudaStream_t s = decoder->device->stream;
	PlaneOutput out = {};
	out.sample16 = wide ? 1 : 0;
	bool linear[3];
	for (int p = 0; p < 3; p++)
	{
		int w, h;
		plane_dims(chroma, g.width, g.height, p, w, h);
		// Unpadded host rows: decode at that pitch and copy back in one piece
		// (a pitched copy of narrow rows runs far below the link's bandwidth).
		linear[p] = buffers->row_stride_in_bytes[p] == size_t(w) * bps;
		out.data[p] = decoder->out_planes[p];
		out.pitch[p] = linear[p] ? int32_t(size_t(w) * bps) : decoder->out_pitch[p];
	}
	r = decoder->decode_parsed(out, s, true);
	if (r != PYROWAVE_SUCCESS)
		return r;
	for (int p = 0; p < 3; p++)
	{
		int w, h;
		plane_dims(chroma, g.width, g.height, p, w, h);
		const size_t row = size_t(w) * bps;
		if (linear[p])
			cudaMemcpyAsync(buffers->data[p], decoder->out_planes[p], row * size_t(h), cudaMemcpyDeviceToHost, s);
		else
			cudaMemcpy2DAsync(buffers->data[p], buffers->row_stride_in_bytes[p], decoder->out_planes[p],
			                  decoder->out_pitch[p], row, size_t(h), cudaMemcpyDeviceToHost, s);
	}
	cudaMemcpyAsync(decoder->h_error, decoder->error_d, sizeof(uint32_t), cudaMemcpyDeviceToHost, s);
	if (cudaStreamSynchronize(s) != cudaSuccess)
		return PYROWAVE_ERROR_GENERIC;
	// A tile load of the inverse transform that did not complete in time.
	if (*decoder->h_error != 0)
		return PYROWAVE_ERROR_GENERIC;
	return PYROWAVE_SUCCESS;
}

void pyrowave_decoder_destroy(pyrowave_decoder decoder)
{
	if (!decoder)
		return;
	decoder->release();
	delete decoder;
}

// --- CUDA extension ----------------------------------------------------------
pyrowave_result pyrowave_cuda_encoder_set_precision(pyrowave_encoder encoder, uint32_t fp16_level_mask)
{
	if (!encoder || (fp16_level_mask & ~(0x1fu | PYROWAVE_CUDA_PRECISION_STAGE16)))
		return PYROWAVE_ERROR_INVALID_ARGUMENT;
	if (encoder->allocated && fp16_level_mask != encoder->fp16_mask)
		encoder->release();
	encoder->fp16_mask = fp16_level_mask;
	return PYROWAVE_SUCCESS;
}

pyrowave_result pyrowave_cuda_decoder_set_precision(pyrowave_decoder decoder, uint32_t fp16_level_mask)
{
	if (!decoder || (fp16_level_mask & ~(0x1fu | PYROWAVE_CUDA_PRECISION_STAGE16)))
		return PYROWAVE_ERROR_INVALID_ARGUMENT;
	if (decoder->allocated && fp16_level_mask != decoder->fp16_mask)
		decoder->release();
	decoder->fp16_mask = fp16_level_mask;
	return PYROWAVE_SUCCESS;
}

pyrowave_result pyrowave_cuda_encoder_get_layout(pyrowave_encoder encoder, pyrowave_cuda_layout *layout)
{
	if (!encoder)
		return PYROWAVE_ERROR_INVALID_ARGUMENT;
	return fill_layout(encoder->g, encoder->fp16_mask, layout);
}

pyrowave_result pyrowave_cuda_decoder_get_layout(pyrowave_decoder decoder, pyrowave_cuda_layout *layout)
{
	if (!decoder)
		return PYROWAVE_ERROR_INVALID_ARGUMENT;
	return fill_layout(decoder->g, decoder->fp16_mask, layout);
}

static pyrowave_result encode_device_planes(pyrowave_encoder encoder, const pyrowave_cuda_planes *planes,
                                            const pyrowave_rate_control *rate_control, pyrowave_cuda_stream stream,
                                            bool wide)
{
	if (!encoder || !planes || !rate_control)
		return PYROWAVE_ERROR_INVALID_ARGUMENT;
	pyrowave_result r = encoder->allocate();
	if (r != PYROWAVE_SUCCESS)
		return r;
	const Geometry &g = encoder->g;
	const size_t bps = wide ? 2 : 1;
	PlaneInput in = {};
	in.sample16 = wide ? 1 : 0;
	for (int p = 0; p < 3; p++)
	{
		if (!planes->data[p] || planes->row_stride_in_bytes[p] < size_t(g.plane_width[p]) * bps ||
		    planes->row_stride_in_bytes[p] > 0x7fffffffu)
			return PYROWAVE_ERROR_INVALID_ARGUMENT;
		if (wide && ((planes->row_stride_in_bytes[p] & 1u) || (reinterpret_cast<uintptr_t>(planes->data[p]) & 1u)))
			return PYROWAVE_ERROR_INVALID_ARGUMENT;
		in.data[p] = static_cast<const uint8_t *>(planes->data[p]);
		in.pitch[p] = int32_t(planes->row_stride_in_bytes[p]);
		in.xstride[p] = int32_t(bps);
	}
	return encoder->enqueue(in, rate_control, pick_stream(encoder->device, stream));
}

pyrowave_result pyrowave_cuda_encoder_encode(pyrowave_encoder encoder, const pyrowave_cuda_planes *planes,
                                             const pyrowave_rate_control *rate_control, pyrowave_cuda_stream stream)
{
	return encode_device_planes(encoder, planes, rate_control, stream, false);
}

pyrowave_result pyrowave_cuda_encoder_encode16(pyrowave_encoder encoder, const pyrowave_cuda_planes *planes,
                                               const pyrowave_rate_control *rate_control, pyrowave_cuda_stream stream)
{
	return encode_device_planes(encoder, planes, rate_control, stream, true);
}

pyrowave_result pyrowave_cuda_encoder_get_device_bitstream(pyrowave_encoder encoder, const uint32_t **stream,
                                                           const uint32_t **block_meta, size_t *capacity_words)
{
	if (!encoder || !encoder->has_device_frame)
		return PYROWAVE_ERROR_GENERIC;
	if (stream)
		*stream = encoder->stream_buf;
	if (block_meta)
		*block_meta = encoder->block_meta;
	if (capacity_words)
		*capacity_words = encoder->stream_capacity;
	return PYROWAVE_SUCCESS;
}

pyrowave_result pyrowave_cuda_encoder_get_size(pyrowave_encoder encoder, size_t *bytes)
{
	if (!encoder || !bytes || !encoder->has_device_frame)
		return PYROWAVE_ERROR_INVALID_ARGUMENT;
	// The encode ran on the caller's stream, which need not be ordered with the
	// copy below: wait for it first.
	uint32_t v[2] = {0, 0};
	if (!cuda_ok(cudaEventSynchronize(encoder->encoded), "cudaEventSynchronize") ||
	    cudaMemcpy(v, &encoder->rc->error, 8, cudaMemcpyDeviceToHost) != cudaSuccess)
		return PYROWAVE_ERROR_GENERIC;
	if (v[0] != 0)
		return PYROWAVE_ERROR_GENERIC;
	*bytes = 8 + size_t(v[1]) * 4;
	return PYROWAVE_SUCCESS;
}

pyrowave_result pyrowave_cuda_encoder_encode_pre_transformed(pyrowave_encoder encoder, const float *pyramid,
                                                             const pyrowave_rate_control *rate_control,
                                                             float quant_scale, pyrowave_cuda_stream stream)
{
	if (!encoder || !pyramid || !rate_control)
		return PYROWAVE_ERROR_INVALID_ARGUMENT;
	pyrowave_result r = encoder->allocate();
	if (r != PYROWAVE_SUCCESS)
		return r;
	uint32_t target_words, capacity;
	if (!pyrowave_encoder_opaque::budget_words(rate_control, target_words, capacity))
		return PYROWAVE_ERROR_INVALID_ARGUMENT;
	r = encoder->ensure_stream_capacity(capacity);
	if (r != PYROWAVE_SUCCESS)
		return r;
	cudaStream_t s = pick_stream(encoder->device, stream);
	Geometry g = encoder->g;
	apply_quant_scale_override(g, quant_scale);
	encoder->sequence_count = (encoder->sequence_count + 1) & 7u;
	EncodeBuffers b = encoder->buffers();
	const BlockParams bp = make_block_params(g);
	cudaMemsetAsync(encoder->rc, 0, sizeof(RateControlState), s);
	launch_pyramid_io(bp, const_cast<float *>(pyramid), encoder->coef32, encoder->coef16, false, s);
	launch_quant_pretransformed(bp, b, bp.block_count_32x32, true, s);
	launch_resolve(make_resolve_params(g, target_words, encoder->sequence_count), b, s);
	launch_pack(bp, b, s);
	if (!launches_ok("kernel launch"))
		return PYROWAVE_ERROR_GENERIC;
	cudaEventRecord(encoder->encoded, s);
	encoder->has_device_frame = true;
	return encoder->queue_readback(s);
}

pyrowave_result pyrowave_cuda_encoder_transform(pyrowave_encoder encoder, const pyrowave_cuda_planes *planes,
                                                pyrowave_cuda_stream stream)
{
	if (!encoder || !planes)
		return PYROWAVE_ERROR_INVALID_ARGUMENT;
	pyrowave_result r = encoder->allocate();
	if (r != PYROWAVE_SUCCESS)
		return r;
	const Geometry &g = encoder->g;
	PlaneInput in = {};
	for (int p = 0; p < 3; p++)
	{
		if (!planes->data[p] || planes->row_stride_in_bytes[p] < size_t(g.plane_width[p]) ||
		    planes->row_stride_in_bytes[p] > 0x7fffffffu)
			return PYROWAVE_ERROR_INVALID_ARGUMENT;
		in.data[p] = static_cast<const uint8_t *>(planes->data[p]);
		in.pitch[p] = int32_t(planes->row_stride_in_bytes[p]);
		in.xstride[p] = 1;
	}
	cudaStream_t s = pick_stream(encoder->device, stream);
	pyrowave_device_opaque *dev = encoder->device;
	StageEvents &timing = encoder->timing;
	timing.collect(dev);
	timing.prepare(dev);
	timing.begin(dev, s, false);
	static const char *const tags[kLevels] = {"xdwt0", "xdwt1", "xdwt2", "xdwt3", "xdwt4"};
	const EncodeBuffers b = encoder->buffers();
	for (int level = 0; level < kLevels; level++)
	{
		launch_dwt_forward_level(encoder->lp[level], in, b, &encoder->in_maps[level], false,
		                         level > 0 && !dev->stage_timing, s);
		timing.mark(dev, s, tags[level]);
	}
	timing.launched(dev);
	return launches_ok("kernel launch") ? PYROWAVE_SUCCESS : PYROWAVE_ERROR_GENERIC;
}

pyrowave_result pyrowave_cuda_encoder_read_wavelet(pyrowave_encoder encoder, float *pyramid, pyrowave_cuda_stream stream)
{
	if (!encoder || !pyramid || !encoder->allocated)
		return PYROWAVE_ERROR_INVALID_ARGUMENT;
	launch_pyramid_io(encoder->bp, pyramid, encoder->coef32, encoder->coef16, true, pick_stream(encoder->device, stream));
	return launches_ok("kernel launch") ? PYROWAVE_SUCCESS : PYROWAVE_ERROR_GENERIC;
}

pyrowave_result pyrowave_cuda_encoder_read_debug(pyrowave_encoder encoder, const pyrowave_cuda_encoder_debug *d)
{
	if (!encoder || !d || !encoder->allocated)
		return PYROWAVE_ERROR_INVALID_ARGUMENT;
	if (cudaDeviceSynchronize() != cudaSuccess)
		return PYROWAVE_ERROR_GENERIC;
	const Geometry &g = encoder->g;
	const size_t n8 = size_t(g.block_count_8x8), n32 = size_t(g.block_count_32x32);
	if (d->code_words)
		cudaMemcpy(d->code_words, encoder->code_words, n8 * 4, cudaMemcpyDeviceToHost);
	if (d->rd_cost)
		cudaMemcpy(d->rd_cost, encoder->rd_cost, n32 * 32, cudaMemcpyDeviceToHost);
	if (d->rd_bucket)
		cudaMemcpy(d->rd_bucket, encoder->rd_bucket, n32 * 16, cudaMemcpyDeviceToHost);
	if (d->rd_dist)
		cudaMemcpy(d->rd_dist, encoder->rd_dist, n32 * 64, cudaMemcpyDeviceToHost);
	if (d->histogram)
		cudaMemcpy(d->histogram, encoder->rc->histogram, kHistSize * 4, cudaMemcpyDeviceToHost);
	if (d->consumed)
		cudaMemcpy(d->consumed, &encoder->rc->consumed, 4, cudaMemcpyDeviceToHost);
	if (d->quant)
		cudaMemcpy(d->quant, encoder->quant, n32 * 4, cudaMemcpyDeviceToHost);
	if (d->block_meta)
		cudaMemcpy(d->block_meta, encoder->block_meta, n32 * 8, cudaMemcpyDeviceToHost);
	if (d->error_flags)
		cudaMemcpy(d->error_flags, &encoder->rc->error, 4, cudaMemcpyDeviceToHost);
	return cudaGetLastError() == cudaSuccess ? PYROWAVE_SUCCESS : PYROWAVE_ERROR_GENERIC;
}

// The reference's disabled statistics pass (pyrowave_encoder.cpp:625-958) on the
// device: every 64x64 region of every coded band, in the reference's band order
// (component, level, band), as four 32x32 block indices.
pyrowave_result pyrowave_cuda_encoder_analyze_packing(pyrowave_encoder encoder, pyrowave_cuda_packing_analysis *a)
{
	if (!encoder || !a || !encoder->allocated || !encoder->has_device_frame)
		return PYROWAVE_ERROR_INVALID_ARGUMENT;
	if (cudaEventSynchronize(encoder->encoded) != cudaSuccess)
		return PYROWAVE_ERROR_GENERIC;
	const Geometry &g = encoder->g;
	if (!encoder->analysis_acc)
	{
		std::vector<int32_t> regions;
		for (int comp = 0; comp < kComponents; comp++)
			for (int level = 0; level < kLevels; level++)
				for (int band = 0; band < 4; band++)
				{
					const BandDesc &B = g.band[comp][level][band];
					if (!B.present)
						continue;
					const int bw = g.level[level].tiles_x, bh = g.level[level].tiles_y;
					for (int ry = 0; ry < (bh + 1) / 2; ry++)
						for (int rx = 0; rx < (bw + 1) / 2; rx++)
						{
							for (int q = 0; q < 4; q++)
							{
								const int bx = 2 * rx + (q & 1), by = 2 * ry + (q >> 1);
								regions.push_back(bx < bw && by < bh ? B.block32_offset + by * B.block32_stride + bx : -1);
							}
							regions.push_back((comp * kLevels + level) * 4 + band);
						}
				}
		bool ok = true;
		int32_t *table = dev_alloc<int32_t>(regions.size(), ok);
		PackingAnalysisAccum *acc = dev_alloc<PackingAnalysisAccum>(1, ok);
		if (!ok || cudaMemcpy(table, regions.data(), regions.size() * 4, cudaMemcpyHostToDevice) != cudaSuccess)
		{
			dev_free(table);
			dev_free(acc);
			(void)cudaGetLastError();
			return PYROWAVE_ERROR_OUT_OF_DEVICE_MEMORY;
		}
		encoder->analysis_regions = table;
		encoder->analysis_acc = acc;
		encoder->analysis_region_count = int(regions.size() / 5);
	}
	cudaStream_t stream = encoder->device->stream;
	PackingAnalysisAccum host = {};
	if (launch_packing_analysis(encoder->bp, encoder->buffers(), encoder->analysis_regions,
	                            encoder->analysis_region_count, encoder->analysis_acc, stream) != cudaSuccess ||
	    cudaMemcpyAsync(&host, encoder->analysis_acc, sizeof(host), cudaMemcpyDeviceToHost, stream) != cudaSuccess ||
	    cudaStreamSynchronize(stream) != cudaSuccess)
	{
		(void)cudaGetLastError();
		return PYROWAVE_ERROR_GENERIC;
	}
	memset(a, 0, sizeof(*a));
	for (int i = 0; i < kPackingLayouts; i++)
		a->layout_bytes[i] = host.layout_bytes[i];
	for (int i = 0; i < kComponents * kLevels * 4; i++)
	{
		(&a->band_bytes[0][0][0])[i] = host.band_bytes[i];
		a->coded_bytes += host.band_bytes[i];
	}
	a->significant = host.significant;
	for (int j = 0; j < 16; j++)
	{
		uint64_t total = 0;
		for (int b = 0; b < 256; b++)
		{
			a->plane_histogram[j][b] = host.plane_histogram[j * 256 + b];
			total += host.plane_histogram[j * 256 + b];
		}
		a->plane_bytes[j] = total;
		// Byte entropy of the plane, as a fraction of 8 bits (pyrowave_encoder.cpp:932-950).
		double h = 0.0;
		for (int b = 0; b < 256 && total; b++)
		{
			const uint32_t n = host.plane_histogram[j * 256 + b];
			if (n)
			{
				const double pr = double(n) / double(total);
				h -= pr * std::log2(pr);
			}
		}
		a->plane_entropy[j] = h / 8.0;
	}
	return PYROWAVE_SUCCESS;
}

pyrowave_result pyrowave_cuda_decoder_decode(pyrowave_decoder decoder, const pyrowave_cuda_planes *planes,
                                             pyrowave_cuda_stream stream)
{
	if (!decoder || !planes)
		return PYROWAVE_ERROR_INVALID_ARGUMENT;
	pyrowave_result r = decoder->allocate();
	if (r != PYROWAVE_SUCCESS)
		return r;
	PlaneOutput out = {};
	for (int p = 0; p < 3; p++)
	{
		if (!planes->data[p] || planes->row_stride_in_bytes[p] < size_t(decoder->g.plane_width[p]) ||
		    planes->row_stride_in_bytes[p] > 0x7fffffffu)
			return PYROWAVE_ERROR_INVALID_ARGUMENT;
		out.data[p] = static_cast<uint8_t *>(planes->data[p]);
		out.pitch[p] = int32_t(planes->row_stride_in_bytes[p]);
	}
	return decoder->decode_parsed(out, pick_stream(decoder->device, stream));
}

static pyrowave_result decode_device_blocks(pyrowave_decoder decoder, const uint32_t *block_meta,
                                            const uint32_t *words, size_t num_words,
                                            const pyrowave_cuda_planes *planes, pyrowave_cuda_stream stream,
                                            bool wide);

pyrowave_result pyrowave_cuda_decoder_decode_blocks(pyrowave_decoder decoder, const uint32_t *block_meta,
                                                    const uint32_t *words, size_t num_words,
                                                    const pyrowave_cuda_planes *planes, pyrowave_cuda_stream stream)
{
	return decode_device_blocks(decoder, block_meta, words, num_words, planes, stream, false);
}

pyrowave_result pyrowave_cuda_decoder_decode_blocks16(pyrowave_decoder decoder, const uint32_t *block_meta,
                                                      const uint32_t *words, size_t num_words,
                                                      const pyrowave_cuda_planes *planes, pyrowave_cuda_stream stream)
{
	return decode_device_blocks(decoder, block_meta, words, num_words, planes, stream, true);
}

static pyrowave_result decode_device_blocks(pyrowave_decoder decoder, const uint32_t *block_meta,
                                            const uint32_t *words, size_t num_words,
                                            const pyrowave_cuda_planes *planes, pyrowave_cuda_stream stream,
                                            bool wide)
{
	if (!decoder || !block_meta || !words || !planes || num_words > 0xffffffffu)
		return PYROWAVE_ERROR_INVALID_ARGUMENT;
	pyrowave_result r = decoder->allocate();
	if (r != PYROWAVE_SUCCESS)
		return r;
	const size_t bps = wide ? 2 : 1;
	PlaneOutput out = {};
	out.sample16 = wide ? 1 : 0;
	for (int p = 0; p < 3; p++)
	{
		if (!planes->data[p] || planes->row_stride_in_bytes[p] < size_t(decoder->g.plane_width[p]) * bps ||
		    planes->row_stride_in_bytes[p] > 0x7fffffffu)
			return PYROWAVE_ERROR_INVALID_ARGUMENT;
		if (wide && ((planes->row_stride_in_bytes[p] & 1u) || (reinterpret_cast<uintptr_t>(planes->data[p]) & 1u)))
			return PYROWAVE_ERROR_INVALID_ARGUMENT;
		out.data[p] = static_cast<uint8_t *>(planes->data[p]);
		out.pitch[p] = int32_t(planes->row_stride_in_bytes[p]);
	}
	DecodeInput in = {};
	in.offsets = nullptr;
	in.block_meta = block_meta;
	in.payload = words;
	in.payload_words = uint32_t(num_words);
	in.jobs = decoder->jobs_d;
	in.coef32 = decoder->coef32;
	in.coef16 = decoder->coef16;
	if (!decoder->run(in, out, pick_stream(decoder->device, stream), true))
		return PYROWAVE_ERROR_GENERIC;
	return launches_ok("kernel launch") ? PYROWAVE_SUCCESS : PYROWAVE_ERROR_GENERIC;
}

pyrowave_result pyrowave_cuda_decoder_decode_packets(pyrowave_decoder decoder, const void *data, size_t data_size,
                                                     const pyrowave_packet *packets, uint32_t count,
                                                     const pyrowave_cuda_planes *planes, pyrowave_cuda_stream stream)
{
	if (!decoder || !data || !packets || !planes || count == 0 || count > uint32_t(kMaxPackets) ||
	    data_size > 0xffffffffull || (reinterpret_cast<uintptr_t>(data) & 3u) != 0 ||
	    (reinterpret_cast<uintptr_t>(packets) & 7u) != 0)
		return PYROWAVE_ERROR_INVALID_ARGUMENT;
	pyrowave_result r = decoder->allocate();
	if (r != PYROWAVE_SUCCESS)
		return r;
	PlaneOutput out = {};
	for (int p = 0; p < 3; p++)
	{
		if (!planes->data[p] || planes->row_stride_in_bytes[p] < size_t(decoder->g.plane_width[p]) ||
		    planes->row_stride_in_bytes[p] > 0x7fffffffu)
			return PYROWAVE_ERROR_INVALID_ARGUMENT;
		out.data[p] = static_cast<uint8_t *>(planes->data[p]);
		out.pitch[p] = int32_t(planes->row_stride_in_bytes[p]);
	}
	return decoder->decode_packets(data, data_size, packets, count, out, pick_stream(decoder->device, stream));
}

pyrowave_result pyrowave_cuda_decoder_get_packet_status(pyrowave_decoder decoder, pyrowave_cuda_packet_status *status)
{
	if (!decoder || !status || !decoder->pk_pending)
		return PYROWAVE_ERROR_INVALID_ARGUMENT;
	if (!cuda_ok(cudaEventSynchronize(decoder->pk_done), "cudaEventSynchronize") ||
	    !cuda_ok(cudaMemcpy(decoder->pk_status_h, decoder->pk_status, sizeof(PacketStatus), cudaMemcpyDeviceToHost),
	             "cudaMemcpy"))
		return PYROWAVE_ERROR_GENERIC;
	const PacketStatus &st = *decoder->pk_status_h;
	status->decoded_blocks = st.decoded_blocks;
	status->total_blocks = st.total_blocks;
	status->sequence = st.sequence;
	status->invalid_packets = st.invalid_packets;
	uint32_t bits = 0;
	if (!decoder->last_error(bits) || bits != 0)
		return PYROWAVE_ERROR_GENERIC;
	return PYROWAVE_SUCCESS;
}

pyrowave_result pyrowave_cuda_decoder_get_error(pyrowave_decoder decoder, uint32_t *error_bits)
{
	if (!decoder)
		return PYROWAVE_ERROR_INVALID_ARGUMENT;
	uint32_t bits = 0;
	const bool ok = decoder->last_error(bits);
	if (error_bits)
		*error_bits = bits;
	return ok && bits == 0 ? PYROWAVE_SUCCESS : PYROWAVE_ERROR_GENERIC;
}

pyrowave_result pyrowave_cuda_decoder_read_wavelet(pyrowave_decoder decoder, float *pyramid, pyrowave_cuda_stream stream)
{
	if (!decoder || !pyramid || !decoder->allocated)
		return PYROWAVE_ERROR_INVALID_ARGUMENT;
	launch_pyramid_io(decoder->bp, pyramid, decoder->coef32, decoder->coef16, true, pick_stream(decoder->device, stream));
	return launches_ok("kernel launch") ? PYROWAVE_SUCCESS : PYROWAVE_ERROR_GENERIC;
}

pyrowave_result pyrowave_cuda_decoder_decode_pyramid(pyrowave_decoder decoder, const float *pyramid,
                                                     const pyrowave_cuda_planes *planes, pyrowave_cuda_stream stream)
{
	if (!decoder || !pyramid || !planes)
		return PYROWAVE_ERROR_INVALID_ARGUMENT;
	pyrowave_result r = decoder->allocate();
	if (r != PYROWAVE_SUCCESS)
		return r;
	PlaneOutput out = {};
	for (int p = 0; p < 3; p++)
	{
		if (!planes->data[p] || planes->row_stride_in_bytes[p] < size_t(decoder->g.plane_width[p]))
			return PYROWAVE_ERROR_INVALID_ARGUMENT;
		out.data[p] = static_cast<uint8_t *>(planes->data[p]);
		out.pitch[p] = int32_t(planes->row_stride_in_bytes[p]);
	}
	cudaStream_t s = pick_stream(decoder->device, stream);
	launch_pyramid_io(decoder->bp, const_cast<float *>(pyramid), decoder->coef32, decoder->coef16, false, s);
	DecodeInput in = {};
	in.jobs = decoder->jobs_d;
	in.coef32 = decoder->coef32;
	in.coef16 = decoder->coef16;
	if (!decoder->run(in, out, s, false))
		return PYROWAVE_ERROR_GENERIC;
	return launches_ok("kernel launch") ? PYROWAVE_SUCCESS : PYROWAVE_ERROR_GENERIC;
}
}

// ---------------------------------------------------------------------------
// Batched form. Every frame of the batch owns the same buffers an encoder
// owns. A call is one CUDA graph launch: upload of the per-call table, the
// clears of the rate-control states and the work counters, then one
// persistent kernel that runs every stage of every frame from a list of
// (frame, stage, item) work words (batch_persistent_kernel). The per-stage
// kernels (one launch per stage over all frames, CTAs mapped to frames through
// tables of batch_cta() words) remain as a second execution mode among the
// autotuner's candidates.
namespace
{
// Execution choices of one batch (the autotuner's search space).
struct BatchShape
{
	bool persistent = true;     // one persistent launch, or one launch per stage
	int small_level = kLevels;  // levels >= this: transform only, quantised after the last level
	int large_below = 0;        // per-stage mode: levels with fewer tiles run 1024-thread CTAs
	int ctas_per_sm = 0;        // persistent mode: resident CTAs per SM (0: as many as fit)
	bool large_first = false;   // persistent mode: within a stage, frames in decreasing size
	int branches = 1;           // per-stage mode: groups of frames, each its own chain of launches;
	                            // frame-graph mode: streams the frames are spread over
	bool frame_graphs = false;  // each frame through its own single-frame encode and decode graphs
};
constexpr int kMaxBatchBranches = 8;
} // namespace

struct pyrowave_cuda_batch_opaque
{
	pyrowave_device device = nullptr;
	int count = 0;
	std::vector<Geometry> geo;
	std::vector<uint32_t> capacity_words; // stream buffer per frame
	std::vector<uint32_t> sequence;
	std::vector<BatchFrame> frames_h;
	std::vector<void *> owned; // device allocations
	BatchFrame *frames_d = nullptr;
	BatchFrameIO *io_d = nullptr;
	BatchFrameIO *io_h[2] = {};
	cudaEvent_t io_free[2] = {};
	int slot = 0;
	RateControlState *rc_d = nullptr;
	// Per frame, the words of RateControlState from `error` to `decode_error`.
	static constexpr int kTotalsWords =
	    int((offsetof(RateControlState, decode_error) - offsetof(RateControlState, error)) / 4) + 1;
	uint32_t *h_totals = nullptr;
	cudaStream_t last_stream = nullptr;
	bool has_result = false;

	// CTA maps, one device array; per branch (group of frames), per-stage ranges.
	uint32_t *maps_d = nullptr;
	std::vector<uint32_t> maps_h;
	struct StageRanges
	{
		int level_off[kLevels] = {}, level_n[kLevels] = {};
		int quant_off = 0, quant_n = 0, resolve_off = 0, resolve_n = 0, block_off = 0, block_n = 0;
	};
	std::vector<StageRanges> ranges;
	int level_tiles[kLevels] = {}; // all frames' tiles per level
	// Per-stage mode with branches: one stream per branch joins the capture
	// through fork / join events (the branches become parallel graph paths).
	cudaStream_t branch_stream[kMaxBatchBranches] = {};
	cudaEvent_t fork_event = nullptr, join_event[kMaxBatchBranches] = {};
	// Frame-graph mode: one single-frame encoder and decoder per frame (created
	// on first use, stream buffers sized for the frame's largest budget).
	std::vector<pyrowave_encoder> frame_enc;
	std::vector<pyrowave_decoder> frame_dec;
	bool result_frame_graphs = false; // the last call ran in frame-graph mode
	// Per-level TMA maps of the first kBatchTileMapFrames frames (kernel parameters).
	std::vector<BatchTileMaps> fwd_maps = std::vector<BatchTileMaps>(kLevels);
	std::vector<BatchTileMaps> inv_maps = std::vector<BatchTileMaps>(kLevels);

	BatchShape shape;
	CapturedGraph graphs[2][2]; // [slot][with decode]

	// Persistent mode: work lists (encode only, encode + decode), per-frame
	// stage gates, and the ticket / finished-item counters cleared per call.
	uint32_t *work_d[2] = {};
	int work_n[2] = {};
	uint32_t *gates_d = nullptr;
	uint32_t *sync_d = nullptr; // ticket, then count x kBatchStages finished counters
	int sm_count = 148;

	template <typename T> T *alloc(size_t n, bool &ok)
	{
		T *p = dev_alloc<T>(n, ok);
		if (p)
			owned.push_back(p);
		return p;
	}

	~pyrowave_cuda_batch_opaque()
	{
		if (device)
			cudaStreamSynchronize(device->stream);
		if (last_stream)
			cudaStreamSynchronize(last_stream);
		for (auto &row : graphs)
			for (auto &gr : row)
				gr.destroy();
		for (void *p : owned)
			dev_free(p);
		for (int i = 0; i < 2; i++)
		{
			host_free(io_h[i]);
			if (io_free[i])
				cudaEventDestroy(io_free[i]);
		}
		host_free(h_totals);
		for (pyrowave_encoder e : frame_enc)
			pyrowave_encoder_destroy(e);
		for (pyrowave_decoder d : frame_dec)
			pyrowave_decoder_destroy(d);
		for (int i = 0; i < kMaxBatchBranches; i++)
		{
			if (branch_stream[i])
				cudaStreamDestroy(branch_stream[i]);
			if (join_event[i])
				cudaEventDestroy(join_event[i]);
		}
		if (fork_event)
			cudaEventDestroy(fork_event);
	}

	// Frames of each branch: largest first, each to the branch with the least
	// work so far (samples coded), so the branches end close together.
	std::vector<std::vector<int>> branch_frames() const
	{
		const int nb = std::max(1, std::min(shape.persistent || shape.frame_graphs ? 1 : shape.branches, count));
		std::vector<std::vector<int>> out(static_cast<size_t>(nb));
		std::vector<int> order(static_cast<size_t>(count));
		std::vector<double> load(size_t(nb), 0.0);
		for (int f = 0; f < count; f++)
			order[size_t(f)] = f;
		auto work = [&](int f) { return double(geo[f].width) * geo[f].height * (geo[f].chroma444 ? 3.0 : 1.5); };
		std::stable_sort(order.begin(), order.end(), [&](int a, int b) { return work(a) > work(b); });
		for (int f : order)
		{
			const size_t g = size_t(std::min_element(load.begin(), load.end()) - load.begin());
			out[g].push_back(f);
			load[g] += work(f);
		}
		for (auto &v : out)
			std::sort(v.begin(), v.end());
		return out;
	}

	void build_maps()
	{
		maps_h.clear();
		for (int level = 0; level < kLevels; level++)
		{
			level_tiles[level] = 0;
			for (int f = 0; f < count; f++)
				level_tiles[level] += geo[f].level[level].tiles_x * geo[f].level[level].tiles_y *
				                      ((level == 0 && !geo[f].chroma444) ? 1 : 3);
		}
		const std::vector<std::vector<int>> groups = branch_frames();
		ranges.assign(groups.size(), StageRanges{});
		for (size_t g = 0; g < groups.size(); g++)
		{
			StageRanges &r = ranges[g];
			const std::vector<int> &fs = groups[g];
			for (int level = 0; level < kLevels; level++)
			{
				r.level_off[level] = int(maps_h.size());
				for (int f : fs)
				{
					const LevelDesc &L = geo[f].level[level];
					const int ncomp = (level == 0 && !geo[f].chroma444) ? 1 : 3;
					for (int i = 0; i < L.tiles_x * L.tiles_y * ncomp; i++)
						maps_h.push_back(batch_cta(f, i));
				}
				r.level_n[level] = int(maps_h.size()) - r.level_off[level];
			}
			r.quant_off = int(maps_h.size());
			for (int f : fs)
				for (int i = 0; i < (frames_h[f].small_blocks + 1) / 2; i++)
					maps_h.push_back(batch_cta(f, i));
			r.quant_n = int(maps_h.size()) - r.quant_off;
			r.resolve_off = int(maps_h.size());
			for (int f : fs)
				for (int i = 0; i < frames_h[f].slices; i++)
					maps_h.push_back(batch_cta(f, i));
			r.resolve_n = int(maps_h.size()) - r.resolve_off;
			r.block_off = int(maps_h.size());
			for (int f : fs)
				for (int i = 0; i < frames_h[f].block_count; i++)
					maps_h.push_back(batch_cta(f, i));
			r.block_n = int(maps_h.size()) - r.block_off;
		}
	}

	// One branch's stage launches (per-stage mode) on stream s; the first launch
	// follows the fork without a programmatic edge.
	void launch_stages(const StageRanges &r, bool decode, bool first_programmatic, cudaStream_t s)
	{
		bool pdl = first_programmatic;
		for (int level = 0; level < kLevels; level++)
		{
			if (r.level_n[level] == 0)
				continue;
			launch_dwt_forward_batch(frames_d, io_d, maps_d + r.level_off[level], r.level_n[level], level,
			                         &fwd_maps[level], level < shape.small_level, large(level), pdl, s);
			pdl = true;
		}
		if (r.quant_n > 0)
			launch_quant_blocks_batch(frames_d, maps_d + r.quant_off, r.quant_n, pdl, s);
		launch_resolve_batch(frames_d, io_d, maps_d + r.resolve_off, r.resolve_n, s);
		launch_pack_batch(frames_d, maps_d + r.block_off, r.block_n, s);
		if (decode)
		{
			launch_dequant_batch(frames_d, maps_d + r.block_off, r.block_n, true, s);
			for (int level = kLevels - 1; level >= 0; level--)
				if (r.level_n[level] > 0)
					launch_idwt_batch(frames_d, io_d, maps_d + r.level_off[level], r.level_n[level], level,
					                  &inv_maps[level], large(level), true, s);
		}
	}

	// Items of each stage of frame f (persistent mode).
	void stage_counts(int f, int (&n)[kBatchStages]) const
	{
		const Geometry &g = geo[f];
		const BatchFrame &fr = frames_h[f];
		for (int level = 0; level < kLevels; level++)
		{
			const int tiles = g.level[level].tiles_x * g.level[level].tiles_y * ((level == 0 && !g.chroma444) ? 1 : 3);
			n[kStageDwt0 + level] = tiles;
			n[kStageIdwt4 + 4 - level] = tiles;
		}
		n[kStageQuant] = (fr.small_blocks + 1) / 2;
		n[kStageResolve] = fr.slices;
		n[kStagePack] = (fr.block_count + 1) / 2;
		n[kStageDequant] = (fr.block_count + 1) / 2;
	}

	// Work lists and gates of the persistent mode: stage by stage, every frame's
	// items (frames in index order, or largest first); an item is gated by the
	// nearest earlier stage of its frame that has items.
	void build_work(std::vector<uint32_t> (&work)[2], std::vector<uint32_t> &gates) const
	{
		std::vector<int> order(static_cast<size_t>(count));
		for (int f = 0; f < count; f++)
			order[size_t(f)] = f;
		if (shape.large_first)
			std::stable_sort(order.begin(), order.end(), [&](int a, int b) {
				return geo[a].storage_elems32 > geo[b].storage_elems32;
			});
		std::vector<std::array<int, kBatchStages>> n(static_cast<size_t>(count));
		gates.assign(size_t(count) * kBatchStages, kNoGate);
		for (int f = 0; f < count; f++)
		{
			int c[kBatchStages];
			stage_counts(f, c);
			int prev = -1;
			for (int st = 0; st < kBatchStages; st++)
			{
				n[size_t(f)][size_t(st)] = c[st];
				if (prev >= 0)
					gates[size_t(f) * kBatchStages + st] = (uint32_t(prev) << 24) | uint32_t(c[prev]);
				if (c[st] > 0)
					prev = st;
			}
		}
		for (int d = 0; d < 2; d++)
		{
			work[d].clear();
			const int last = d ? kBatchStages : kStageDequant;
			for (int st = 0; st < last; st++)
				for (int f : order)
					for (int i = 0; i < n[size_t(f)][size_t(st)]; i++)
						work[d].push_back(batch_work(f, st, i));
		}
	}

	int persistent_ctas() const
	{
		const int fit = batch_persistent_max_ctas_per_sm();
		const int per_sm = shape.ctas_per_sm > 0 ? std::min(shape.ctas_per_sm, fit) : fit;
		return std::max(1, per_sm) * sm_count;
	}

	// Per-frame blocks of the levels >= small_level (a prefix in block index order).
	void apply_shape(const BatchShape &s)
	{
		shape = s;
		for (int f = 0; f < count; f++)
		{
			const Geometry &g = geo[f];
			frames_h[f].small_blocks = s.small_level >= kLevels ? 0
			                           : s.small_level == 0     ? g.block_count_32x32
			                                                    : g.band[0][s.small_level - 1][1].block32_offset;
		}
		for (auto &row : graphs)
			for (auto &gr : row)
				gr.destroy();
	}

	// Upload the frame table, the CTA maps and the work lists (after apply_shape).
	bool upload(cudaStream_t s)
	{
		build_maps();
		const size_t nstreams = shape.frame_graphs ? size_t(std::max(1, std::min(shape.branches, count))) : ranges.size();
		for (size_t g = 0; g < nstreams && nstreams > 1; g++)
		{
			if (!branch_stream[g] &&
			    !cuda_ok(cudaStreamCreateWithFlags(&branch_stream[g], cudaStreamNonBlocking), "cudaStreamCreate"))
				return false;
			if (!join_event[g] &&
			    !cuda_ok(cudaEventCreateWithFlags(&join_event[g], cudaEventDisableTiming), "cudaEventCreate"))
				return false;
		}
		if (!fork_event && !cuda_ok(cudaEventCreateWithFlags(&fork_event, cudaEventDisableTiming), "cudaEventCreate"))
			return false;
		(void)batch_persistent_max_ctas_per_sm(); // kernel attributes, set outside any capture
		bool ok = true;
		std::vector<uint32_t> work[2], gates;
		build_work(work, gates);
		for (int d = 0; d < 2; d++)
		{
			if (work_d[d])
			{
				dev_free(work_d[d]);
				owned.erase(std::find(owned.begin(), owned.end(), static_cast<void *>(work_d[d])));
			}
			work_d[d] = alloc<uint32_t>(std::max<size_t>(work[d].size(), 1), ok);
			work_n[d] = int(work[d].size());
		}
		if (!gates_d)
			gates_d = alloc<uint32_t>(gates.size(), ok);
		if (!sync_d)
			sync_d = alloc<uint32_t>(1 + size_t(count) * kBatchStages, ok);
		if (!ok)
			return false;
		for (int d = 0; d < 2; d++)
			if (!work[d].empty() &&
			    !cuda_ok(cudaMemcpyAsync(work_d[d], work[d].data(), work[d].size() * 4, cudaMemcpyHostToDevice, s),
			             "cudaMemcpyAsync"))
				return false;
		if (!cuda_ok(cudaMemcpyAsync(gates_d, gates.data(), gates.size() * 4, cudaMemcpyHostToDevice, s),
		             "cudaMemcpyAsync"))
			return false;
		if (!frames_d)
			frames_d = alloc<BatchFrame>(size_t(count), ok);
		if (maps_d)
		{
			dev_free(maps_d);
			owned.erase(std::find(owned.begin(), owned.end(), static_cast<void *>(maps_d)));
		}
		maps_d = alloc<uint32_t>(maps_h.size(), ok);
		if (!ok)
			return false;
		return cuda_ok(cudaMemcpyAsync(frames_d, frames_h.data(), sizeof(BatchFrame) * size_t(count),
		                               cudaMemcpyHostToDevice, s), "cudaMemcpyAsync") &&
		       cuda_ok(cudaMemcpyAsync(maps_d, maps_h.data(), maps_h.size() * 4, cudaMemcpyHostToDevice, s),
		               "cudaMemcpyAsync") &&
		       cuda_ok(cudaStreamSynchronize(s), "cudaStreamSynchronize");
	}

	bool large(int level) const { return level >= shape.small_level || level_tiles[level] < shape.large_below; }

	// The stages of one call, captured into graphs[slot][decode].
	bool capture(int slot_index, bool decode, cudaStream_t s)
	{
		CapturedGraph &graph = graphs[slot_index][decode ? 1 : 0];
		if (graph.valid())
			return true;
		if (!graph.begin(s))
			return false;
		bool ok = cuda_ok(cudaMemcpyAsync(io_d, io_h[slot_index], sizeof(BatchFrameIO) * size_t(count),
		                                  cudaMemcpyHostToDevice, s), "cudaMemcpyAsync");
		ok = ok && cuda_ok(cudaMemsetAsync(rc_d, 0, sizeof(RateControlState) * size_t(count), s), "cudaMemsetAsync");
		if (shape.persistent)
		{
			ok = ok && cuda_ok(cudaMemsetAsync(sync_d, 0, (1 + size_t(count) * kBatchStages) * 4, s),
			                   "cudaMemsetAsync");
			BatchRunParams rp = {};
			rp.frames = frames_d;
			rp.io = io_d;
			rp.work = work_d[decode ? 1 : 0];
			rp.gates = gates_d;
			rp.ticket = sync_d;
			rp.done = sync_d + 1;
			rp.nwork = work_n[decode ? 1 : 0];
			rp.small_level = shape.small_level;
			launch_batch_persistent(rp, persistent_ctas(), s);
			ok = launches_ok("kernel launch") && ok;
			ok = graph.end(s, 0) && ok;
			if (!ok)
				graph.destroy();
			return ok;
		}
		if (ranges.size() <= 1)
			launch_stages(ranges[0], decode, false, s);
		else
		{
			// Fork: every branch stream waits for the clears above; join: the
			// capturing stream waits for every branch.
			ok = ok && cuda_ok(cudaEventRecord(fork_event, s), "cudaEventRecord");
			for (size_t g = 0; g < ranges.size() && ok; g++)
			{
				ok = cuda_ok(cudaStreamWaitEvent(branch_stream[g], fork_event, 0), "cudaStreamWaitEvent");
				launch_stages(ranges[g], decode, false, branch_stream[g]);
				ok = ok && cuda_ok(cudaEventRecord(join_event[g], branch_stream[g]), "cudaEventRecord") &&
				     cuda_ok(cudaStreamWaitEvent(s, join_event[g], 0), "cudaStreamWaitEvent");
			}
		}
		ok = launches_ok("kernel launch") && ok;
		ok = graph.end(s, 0) && ok;
		if (!ok)
			graph.destroy();
		return ok;
	}

	bool ensure_frame_coders()
	{
		if (!frame_enc.empty())
			return true;
		for (int f = 0; f < count; f++)
		{
			const Geometry &g = geo[f];
			pyrowave_encoder_create_info ei = {device, g.width, g.height,
			                                   g.chroma444 ? PYROWAVE_CHROMA_SUBSAMPLING_444
			                                               : PYROWAVE_CHROMA_SUBSAMPLING_420};
			pyrowave_decoder_create_info di = {};
			di.device = device;
			di.width = g.width;
			di.height = g.height;
			di.chroma = ei.chroma;
			pyrowave_encoder e = nullptr;
			pyrowave_decoder d = nullptr;
			if (pyrowave_encoder_create(&ei, &e) != PYROWAVE_SUCCESS)
				return false;
			frame_enc.push_back(e);
			if (pyrowave_decoder_create(&di, &d) != PYROWAVE_SUCCESS)
				return false;
			frame_dec.push_back(d);
			// Buffers now, sized for the largest budget the batch accepts, so no
			// call reallocates while other frames' work is in flight.
			if (e->allocate() != PYROWAVE_SUCCESS || e->ensure_stream_capacity(capacity_words[f]) != PYROWAVE_SUCCESS ||
			    d->allocate() != PYROWAVE_SUCCESS)
				return false;
		}
		return true;
	}

	// Frame-graph mode: every frame's encode (and decode) through its own
	// single-frame graphs, the frames dealt round robin over the branch
	// streams, which fork from and join into s. Each frame's totals and decode
	// error word are read back on its stream.
	pyrowave_result run_frame_graphs(const pyrowave_cuda_planes *inputs, const size_t *budgets,
	                                 const pyrowave_cuda_planes *outputs, cudaStream_t s)
	{
		if (!ensure_frame_coders())
			return PYROWAVE_ERROR_OUT_OF_DEVICE_MEMORY;
		const int nb = std::max(1, std::min(shape.branches, count));
		if (!cuda_ok(cudaEventRecord(fork_event, s), "cudaEventRecord"))
			return PYROWAVE_ERROR_GENERIC;
		for (int k = 0; k < nb; k++)
			if (!cuda_ok(cudaStreamWaitEvent(branch_stream[k], fork_event, 0), "cudaStreamWaitEvent"))
				return PYROWAVE_ERROR_GENERIC;
		pyrowave_result r = PYROWAVE_SUCCESS;
		for (int f = 0; f < count && r == PYROWAVE_SUCCESS; f++)
		{
			cudaStream_t bs = branch_stream[f % nb];
			const pyrowave_cuda_stream ps = reinterpret_cast<pyrowave_cuda_stream>(bs);
			encoder_set_frames(frame_enc[size_t(f)], (sequence[f] + 7u) & 7u); // the encode advances it to sequence[f]
			const pyrowave_rate_control rc = {budgets[f]};
			r = pyrowave_cuda_encoder_encode(frame_enc[size_t(f)], &inputs[f], &rc, ps);
			uint32_t *tot = h_totals + size_t(f) * kTotalsWords;
			if (r == PYROWAVE_SUCCESS &&
			    !cuda_ok(cudaMemcpyAsync(tot, &frame_enc[size_t(f)]->rc->error, kTotalsWords * 4, cudaMemcpyDeviceToHost,
			                             bs),
			             "cudaMemcpyAsync"))
				r = PYROWAVE_ERROR_GENERIC;
			if (r == PYROWAVE_SUCCESS && outputs)
			{
				const uint32_t *words = nullptr, *meta = nullptr;
				size_t cap = 0;
				r = pyrowave_cuda_encoder_get_device_bitstream(frame_enc[size_t(f)], &words, &meta, &cap);
				if (r == PYROWAVE_SUCCESS)
					r = pyrowave_cuda_decoder_decode_blocks(frame_dec[size_t(f)], meta, words + 2, cap - 2, &outputs[f], ps);
				if (r == PYROWAVE_SUCCESS &&
				    !cuda_ok(cudaMemcpyAsync(tot + kTotalsWords - 1, frame_dec[size_t(f)]->error_d, 4,
				                             cudaMemcpyDeviceToHost, bs),
				             "cudaMemcpyAsync"))
					r = PYROWAVE_ERROR_GENERIC;
			}
		}
		// Join every branch, also after a failed frame, so the stream state stays whole.
		for (int k = 0; k < nb; k++)
			if (!cuda_ok(cudaEventRecord(join_event[k], branch_stream[k]), "cudaEventRecord") ||
			    !cuda_ok(cudaStreamWaitEvent(s, join_event[k], 0), "cudaStreamWaitEvent"))
				r = PYROWAVE_ERROR_GENERIC;
		last_stream = s;
		has_result = r == PYROWAVE_SUCCESS;
		result_frame_graphs = true;
		return r;
	}

	pyrowave_result run(const pyrowave_cuda_planes *inputs, const size_t *budgets, const pyrowave_cuda_planes *outputs,
	                    cudaStream_t s)
	{
		// Validate everything before touching any state.
		for (int f = 0; f < count; f++)
		{
			const Geometry &g = geo[f];
			for (int p = 0; p < 3; p++)
			{
				if (!inputs[f].data[p] || inputs[f].row_stride_in_bytes[p] < size_t(g.plane_width[p]) ||
				    inputs[f].row_stride_in_bytes[p] > 0x7fffffffu)
					return PYROWAVE_ERROR_INVALID_ARGUMENT;
				if (outputs && (!outputs[f].data[p] || outputs[f].row_stride_in_bytes[p] < size_t(g.plane_width[p]) ||
				                outputs[f].row_stride_in_bytes[p] > 0x7fffffffu))
					return PYROWAVE_ERROR_INVALID_ARGUMENT;
			}
			const uint64_t target = uint64_t(budgets[f]) & ~uint64_t(3);
			if (target == 0 || target > 0xffffffffull || (target >= 8 ? (target - 8) / 4 : target / 4) + 2 >
			                                                 capacity_words[f])
				return PYROWAVE_ERROR_INVALID_ARGUMENT;
		}
		const int k = slot;
		slot ^= 1;
		// The pinned table of this slot was last read by the call before the previous one.
		if (!cuda_ok(cudaEventSynchronize(io_free[k]), "cudaEventSynchronize"))
			return PYROWAVE_ERROR_GENERIC;
		for (int f = 0; f < count; f++)
		{
			BatchFrameIO &io = io_h[k][f];
			io = {};
			for (int p = 0; p < 3; p++)
			{
				io.in.data[p] = static_cast<const uint8_t *>(inputs[f].data[p]);
				io.in.pitch[p] = int32_t(inputs[f].row_stride_in_bytes[p]);
				io.in.xstride[p] = 1;
				if (outputs)
				{
					io.out.data[p] = static_cast<uint8_t *>(outputs[f].data[p]);
					io.out.pitch[p] = int32_t(outputs[f].row_stride_in_bytes[p]);
				}
			}
			const uint64_t target = uint64_t(budgets[f]) & ~uint64_t(3);
			sequence[f] = (sequence[f] + 1) & 7u;
			io.rp = make_resolve_params(geo[f], uint32_t((target >= 8 ? target - 8 : target) / 4), sequence[f]);
		}
		if (shape.frame_graphs)
			return run_frame_graphs(inputs, budgets, outputs, s);
		result_frame_graphs = false;
		if (!capture(k, outputs != nullptr, s))
			return PYROWAVE_ERROR_GENERIC;
		if (!cuda_ok(cudaGraphLaunch(graphs[k][outputs ? 1 : 0].exec, s), "cudaGraphLaunch") ||
		    !cuda_ok(cudaEventRecord(io_free[k], s), "cudaEventRecord"))
			return PYROWAVE_ERROR_GENERIC;
		// {error, total_words, ..., decode_error} of every frame, for get_sizes.
		if (!cuda_ok(cudaMemcpy2DAsync(h_totals, kTotalsWords * 4, &rc_d[0].error, sizeof(RateControlState),
		                               kTotalsWords * 4, size_t(count), cudaMemcpyDeviceToHost, s),
		             "cudaMemcpy2DAsync"))
			return PYROWAVE_ERROR_GENERIC;
		last_stream = s;
		has_result = true;
		return PYROWAVE_SUCCESS;
	}
};

extern "C" {

pyrowave_result pyrowave_cuda_batch_create(pyrowave_device device, const pyrowave_cuda_batch_frame_info *frames,
                                           uint32_t count, pyrowave_cuda_batch *batch)
{
	if (!device || !frames || !batch || count == 0 || count > uint32_t(kMaxBatchFrames))
		return PYROWAVE_ERROR_INVALID_ARGUMENT;
	for (uint32_t f = 0; f < count; f++)
	{
		const auto &fi = frames[f];
		if (fi.width <= 0 || fi.height <= 0)
			return PYROWAVE_ERROR_INVALID_ARGUMENT;
		if (fi.chroma != PYROWAVE_CHROMA_SUBSAMPLING_420 && fi.chroma != PYROWAVE_CHROMA_SUBSAMPLING_444)
			return PYROWAVE_ERROR_INVALID_ARGUMENT;
		if (fi.chroma == PYROWAVE_CHROMA_SUBSAMPLING_420 && ((fi.width & 1) || (fi.height & 1)))
			return PYROWAVE_ERROR_INVALID_ARGUMENT;
		const uint64_t target = uint64_t(fi.maximum_bitstream_size) & ~uint64_t(3);
		if (target == 0 || target > 0xffffffffull)
			return PYROWAVE_ERROR_INVALID_ARGUMENT;
	}
	auto *b = new (std::nothrow) pyrowave_cuda_batch_opaque;
	if (!b)
		return PYROWAVE_ERROR_OUT_OF_HOST_MEMORY;
	b->device = device;
	b->count = int(count);
	b->geo.resize(count);
	b->frames_h.resize(count);
	b->capacity_words.resize(count);
	b->sequence.assign(count, 0);
	bool ok = true;
	b->rc_d = b->alloc<RateControlState>(count, ok);
	for (uint32_t f = 0; f < count && ok; f++)
	{
		const auto &fi = frames[f];
		Geometry &g = b->geo[f];
		if (!make_geometry(g, fi.width, fi.height, fi.chroma == PYROWAVE_CHROMA_SUBSAMPLING_444, 0))
		{
			delete b;
			return PYROWAVE_ERROR_INVALID_ARGUMENT;
		}
		const uint64_t target = uint64_t(fi.maximum_bitstream_size) & ~uint64_t(3);
		b->capacity_words[f] = uint32_t((target >= 8 ? target - 8 : target) / 4) + 2;
		BatchFrame &fr = b->frames_h[f];
		fr = {};
		for (int level = 0; level < kLevels; level++)
			fr.lp[level] = make_level_params(g, level);
		fr.bp = make_block_params(g);
		const size_t n8 = size_t(g.block_count_8x8), n32 = size_t(g.block_count_32x32);
		EncodeBuffers &eb = fr.eb;
		eb.coef32 = b->alloc<float>(size_t(g.storage_elems32), ok);
		eb.coef16 = nullptr;
		eb.mag16 = b->alloc<uint16_t>(n32 * 1024, ok);
		eb.code_words = b->alloc<uint32_t>(n8, ok);
		eb.rd_cost = b->alloc<uint16_t>(n32 * 16, ok);
		eb.rd_bucket = b->alloc<uint8_t>(n32 * 16, ok);
		eb.rd_dist = b->alloc<float>(n32 * 16, ok);
		eb.rc = b->rc_d ? b->rc_d + f : nullptr;
		eb.quant = b->alloc<int32_t>(n32, ok);
		eb.block_meta = b->alloc<uint32_t>(n32 * 2, ok);
		eb.stream = b->alloc<uint32_t>(b->capacity_words[f], ok);
		eb.stream_capacity_words = b->capacity_words[f];
		eb.jobs = nullptr;
		DecodeInput &di = fr.di;
		di.offsets = nullptr;
		di.keys = nullptr;
		di.error = eb.rc ? &eb.rc->decode_error : nullptr;
		di.block_meta = eb.block_meta;
		di.payload = eb.stream ? eb.stream + 2 : nullptr;
		di.payload_words = b->capacity_words[f] - 2;
		di.coef32 = eb.coef32;
		di.coef16 = nullptr;
		if (ok && f < uint32_t(kBatchTileMapFrames))
		{
			LevelTileMap fwd[kLevels], inv[kLevels];
			build_tile_maps(g, fr.lp, eb.coef32, fwd, inv);
			for (int level = 0; level < kLevels; level++)
			{
				b->fwd_maps[level].frame[f] = fwd[level];
				b->inv_maps[level].frame[f] = inv[level];
			}
		}
		fr.block_count = g.block_count_32x32;
		fr.slices = resolve_slices(g.block_count_32x32, g.blocks_per_subdivision);
	}
	b->io_d = b->alloc<BatchFrameIO>(count, ok);
	for (int i = 0; i < 2 && ok; i++)
	{
		b->io_h[i] = host_alloc<BatchFrameIO>(count, ok);
		ok = ok && cudaEventCreateWithFlags(&b->io_free[i], cudaEventDisableTiming) == cudaSuccess;
	}
	b->h_totals = host_alloc<uint32_t>(size_t(count) * pyrowave_cuda_batch_opaque::kTotalsWords, ok);
	if (!ok)
	{
		(void)cudaGetLastError();
		delete b;
		return PYROWAVE_ERROR_OUT_OF_DEVICE_MEMORY;
	}
	// Default shape: the single-frame rule applied to the batch's tile counts.
	BatchShape shape;
	int tiles[kLevels] = {};
	for (int f = 0; f < b->count; f++)
		for (int level = 0; level < kLevels; level++)
			tiles[level] += b->geo[f].level[level].tiles_x * b->geo[f].level[level].tiles_y *
			                ((level == 0 && !b->geo[f].chroma444) ? 1 : 3);
	for (int level = kLevels - 1; level >= 0 && tiles[level] < kSmallLevelTiles; level--)
		shape.small_level = level;
	shape.large_below = kSmallLevelTiles;
	int sms = 0;
	if (cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, device->cuda_device) == cudaSuccess && sms > 0)
		b->sm_count = sms;
	b->apply_shape(shape);
	if (!b->upload(device->stream))
	{
		delete b;
		return PYROWAVE_ERROR_GENERIC;
	}
	*batch = b;
	return PYROWAVE_SUCCESS;
}

void pyrowave_cuda_batch_destroy(pyrowave_cuda_batch batch) { delete batch; }

pyrowave_result pyrowave_cuda_batch_encode(pyrowave_cuda_batch batch, const pyrowave_cuda_planes *inputs,
                                           const size_t *budgets, const pyrowave_cuda_planes *outputs,
                                           pyrowave_cuda_stream stream)
{
	if (!batch || !inputs || !budgets)
		return PYROWAVE_ERROR_INVALID_ARGUMENT;
	return batch->run(inputs, budgets, outputs, pick_stream(batch->device, stream));
}

pyrowave_result pyrowave_cuda_batch_get_device_bitstream(pyrowave_cuda_batch batch, uint32_t index,
                                                         const uint32_t **stream, const uint32_t **block_meta)
{
	if (!batch || index >= uint32_t(batch->count) || !stream || !block_meta)
		return PYROWAVE_ERROR_INVALID_ARGUMENT;
	if (batch->result_frame_graphs)
	{
		size_t cap = 0;
		return pyrowave_cuda_encoder_get_device_bitstream(batch->frame_enc[index], stream, block_meta, &cap);
	}
	*stream = batch->frames_h[index].eb.stream;
	*block_meta = batch->frames_h[index].eb.block_meta;
	return PYROWAVE_SUCCESS;
}

pyrowave_result pyrowave_cuda_batch_get_sizes(pyrowave_cuda_batch batch, size_t *bytes)
{
	if (!batch || !bytes || !batch->has_result)
		return PYROWAVE_ERROR_INVALID_ARGUMENT;
	if (!cuda_ok(cudaStreamSynchronize(batch->last_stream), "cudaStreamSynchronize"))
		return PYROWAVE_ERROR_GENERIC;
	for (int f = 0; f < batch->count; f++)
	{
		const uint32_t *t = batch->h_totals + size_t(f) * pyrowave_cuda_batch_opaque::kTotalsWords;
		// Encoder consistency check, or a decode tile load that did not complete in time.
		if (t[0] != 0 || t[pyrowave_cuda_batch_opaque::kTotalsWords - 1] != 0)
			return PYROWAVE_ERROR_GENERIC;
		bytes[f] = 8 + size_t(t[1]) * 4;
	}
	return PYROWAVE_SUCCESS;
}

pyrowave_result pyrowave_cuda_batch_get_shape(pyrowave_cuda_batch batch, pyrowave_cuda_batch_shape *shape)
{
	if (!batch || !shape)
		return PYROWAVE_ERROR_INVALID_ARGUMENT;
	shape->persistent = batch->shape.persistent ? 1u : 0u;
	shape->small_level = batch->shape.small_level;
	shape->large_below = batch->shape.large_below;
	shape->ctas_per_sm = batch->shape.persistent ? batch->persistent_ctas() / batch->sm_count : 0;
	shape->large_first = batch->shape.large_first ? 1u : 0u;
	shape->branches = batch->shape.persistent ? 1u
	                  : batch->shape.frame_graphs ? uint32_t(std::max(1, std::min(batch->shape.branches, batch->count)))
	                                              : uint32_t(batch->ranges.size());
	shape->frame_graphs = batch->shape.frame_graphs ? 1u : 0u;
	return PYROWAVE_SUCCESS;
}

pyrowave_result pyrowave_cuda_batch_set_shape(pyrowave_cuda_batch batch, const pyrowave_cuda_batch_shape *shape,
                                              pyrowave_cuda_stream stream)
{
	if (!batch || !shape || shape->small_level < 0 || shape->small_level > kLevels || shape->ctas_per_sm < 0 ||
	    shape->large_below < 0 || shape->branches > uint32_t(kMaxBatchBranches))
		return PYROWAVE_ERROR_INVALID_ARGUMENT;
	BatchShape s;
	s.persistent = shape->persistent != 0;
	s.small_level = shape->small_level;
	s.large_below = shape->large_below;
	s.ctas_per_sm = shape->ctas_per_sm;
	s.large_first = shape->large_first != 0;
	s.branches = std::max(1, int(shape->branches));
	s.frame_graphs = shape->frame_graphs != 0 && !s.persistent;
	cudaStream_t st = pick_stream(batch->device, stream);
	if (batch->last_stream && !cuda_ok(cudaStreamSynchronize(batch->last_stream), "cudaStreamSynchronize"))
		return PYROWAVE_ERROR_GENERIC;
	batch->apply_shape(s);
	return batch->upload(st) ? PYROWAVE_SUCCESS : PYROWAVE_ERROR_GENERIC;
}

pyrowave_result pyrowave_cuda_batch_autotune(pyrowave_cuda_batch batch, const pyrowave_cuda_planes *inputs,
                                             const size_t *budgets, const pyrowave_cuda_planes *outputs,
                                             pyrowave_cuda_stream stream)
{
	if (!batch || !inputs || !budgets)
		return PYROWAVE_ERROR_INVALID_ARGUMENT;
	cudaStream_t s = pick_stream(batch->device, stream);
	const std::vector<uint32_t> sequence = batch->sequence; // tuning calls do not count
	cudaEvent_t e0 = nullptr, e1 = nullptr;
	if (!cuda_ok(cudaEventCreate(&e0), "cudaEventCreate") || !cuda_ok(cudaEventCreate(&e1), "cudaEventCreate"))
		return PYROWAVE_ERROR_GENERIC;
	// Candidates. Persistent launch: where the transform-only suffix of levels
	// starts (its blocks quantised in a stage of their own), resident CTAs per
	// SM, and the order of frames within a stage. Per-stage launches: the same
	// suffix, below how many tiles a level runs 1024-thread CTAs, and how many
	// concurrent groups of frames. Each is timed over a few calls; the fastest
	// is kept.
	std::vector<BatchShape> cands;
	for (int small = kLevels; small >= 2; small--)
	{
		for (int per_sm = 2; per_sm <= std::max(2, batch_persistent_max_ctas_per_sm()); per_sm++)
			for (int large_first = 0; large_first < 2; large_first++)
			{
				BatchShape c;
				c.persistent = true;
				c.small_level = small;
				c.ctas_per_sm = per_sm;
				c.large_first = large_first != 0;
				cands.push_back(c);
			}
		if (small == kLevels)
			for (int br : {4, 8})
			{
				// Frame graphs do not depend on the suffix or the CTA threshold.
				if (br > batch->count)
					continue;
				BatchShape c;
				c.persistent = false;
				c.frame_graphs = true;
				c.branches = br;
				cands.push_back(c);
			}
		for (int lb : {0, 256, 1024})
			for (int br : {1, 2, 4, 8})
			{
				if (br > batch->count || (br > 1 && lb == 1024))
					continue;
				BatchShape c;
				c.persistent = false;
				c.small_level = small;
				c.large_below = lb;
				c.branches = br;
				cands.push_back(c);
			}
	}
	BatchShape best = batch->shape;
	float best_ms = 0.0f;
	bool have_best = false;
	pyrowave_result r = PYROWAVE_SUCCESS;
	for (const BatchShape &cand : cands)
	{
		if (r != PYROWAVE_SUCCESS)
			break;
		batch->apply_shape(cand);
		if (!batch->upload(s))
		{
			r = PYROWAVE_ERROR_GENERIC;
			break;
		}
		for (int w = 0; w < 2 && r == PYROWAVE_SUCCESS; w++)
			r = batch->run(inputs, budgets, outputs, s);
		if (r != PYROWAVE_SUCCESS)
			break;
		cudaEventRecord(e0, s);
		for (int it = 0; it < 4 && r == PYROWAVE_SUCCESS; it++)
			r = batch->run(inputs, budgets, outputs, s);
		cudaEventRecord(e1, s);
		float ms = 0.0f;
		if (r != PYROWAVE_SUCCESS || !cuda_ok(cudaEventSynchronize(e1), "cudaEventSynchronize") ||
		    !cuda_ok(cudaEventElapsedTime(&ms, e0, e1), "cudaEventElapsedTime"))
		{
			r = r != PYROWAVE_SUCCESS ? r : PYROWAVE_ERROR_GENERIC;
			break;
		}
		if (!have_best || ms < best_ms)
		{
			best_ms = ms;
			best = cand;
			have_best = true;
		}
	}
	cudaEventDestroy(e0);
	cudaEventDestroy(e1);
	batch->apply_shape(best);
	batch->sequence = sequence;
	if (!batch->upload(s))
		return PYROWAVE_ERROR_GENERIC;
	return r;
}
}
