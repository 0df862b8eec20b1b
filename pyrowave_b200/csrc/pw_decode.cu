// Decoder kernels for sm_100a: dequantiser and inverse CDF 9/7 level.
//
// Reference behaviour followed (file:line in the reference tree):
//   dequantiser   shaders/wavelet_dequant.comp:100-391 (STORAGE_MODE 0), pyrowave_decoder.cpp:280-381
//   inverse level shaders/idwt.comp:25-214, pyrowave_decoder.cpp:699-778
//
// Every payload read is bounds-checked against the payload size: the payload
// comes from the network and a malformed packet must decode to garbage, never
// to an out-of-bounds access. Reads past the end return zero.
#include "pw_decode_body.cuh"

namespace pw
{
namespace
{
// One 32x32 block per 64-thread CTA, two sub-blocks per thread: twice the
// blocks resident per SM of 128-thread CTAs (a 1080p frame's 3261 blocks in
// one wave).
constexpr int kDequantThreads = 64;
__global__ void __launch_bounds__(kDequantThreads) dequant_kernel(const BlockParams p, const DecodeInput in, const int first)
{
	__shared__ DequantShared sh;
	// Only the launch that starts at block 0 clears the decode's error word.
	dequant_body<128 / kDequantThreads>(sh, p, in, first + int(blockIdx.x), blockIdx.x == 0 && first == 0, 1);
}

// Batched form: one CTA per (frame, block), decoding the frame's own bitstream.
__global__ void __launch_bounds__(128) dequant_batch_kernel(const BatchFrame *frames, const uint32_t *cta_map)
{
	__shared__ BlockParams s_p;
	__shared__ DecodeInput s_in;
	int f, local;
	batch_item(cta_map, f, local);
	load_params(s_p, frames[f].bp);
	load_params(s_in, frames[f].di);
	__syncthreads();
	__shared__ DequantShared sh;
	dequant_body(sh, s_p, s_in, local, local == 0, 1);
}

// 256-thread CTAs: three per SM (80 registers) for levels of about one wave,
// four per SM (64 registers) for levels of several waves, each measured the
// faster of the two there; 1024-thread CTAs keep 32 registers.
template <int kThreads> constexpr int kIdwtMinBlocks = kThreads >= 1024 ? 2 : 3;
constexpr int kIdwtManyTiles = 2 * 148 * 4; // levels with at least this many tiles use four CTAs per SM

template <int kThreads, int kMinBlocks = kIdwtMinBlocks<kThreads>>
__global__ void __launch_bounds__(kThreads, kMinBlocks) idwt_kernel(const LevelParams p, const DecodeInput in, const PlaneOutput out,
                                                                     const __grid_constant__ LevelTileMap maps)
{
	__shared__ IdwtShared sh;
	idwt_body<kThreads>(sh, p, in, out, &maps, int(blockIdx.x), int(blockIdx.y));
}

// Small levels (fewer tiles than SMs): four 256-thread CTAs per tile, one per
// stripe of 16 output rows (blockIdx.x = tile * 4 + stripe).
constexpr int kIdwtStripes = 4;
// Same parameters as idwt_kernel (graph nodes are updated with one argument
// list); the stripes load with plain vector loads, not tensor maps.
__global__ void __launch_bounds__(256, 4) idwt_stripes_kernel(const LevelParams p, const DecodeInput in, const PlaneOutput out,
                                                              const __grid_constant__ LevelTileMap maps)
{
	(void)maps;
	__shared__ IdwtShared sh;
	idwt_body<256, kIdwtStripes>(sh, p, in, out, nullptr, int(blockIdx.x) / kIdwtStripes, int(blockIdx.y),
	                             int(blockIdx.x) % kIdwtStripes);
}

// Batched form: one CTA per (frame, component, tile) of this level.
template <int kThreads, int kMinBlocks = kIdwtMinBlocks<kThreads>>
__global__ void __launch_bounds__(kThreads, kMinBlocks) idwt_batch_kernel(const BatchFrame *frames, const BatchFrameIO *io,
                                                              const uint32_t *cta_map, const int level,
                                                              const __grid_constant__ BatchTileMaps maps)
{
	__shared__ LevelParams s_p;
	__shared__ DecodeInput s_in;
	__shared__ PlaneOutput s_out;
	int f, local;
	batch_item(cta_map, f, local);
	load_params(s_p, frames[f].lp[level]);
	load_params(s_in, frames[f].di);
	load_params(s_out, io[f].out);
	__syncthreads();
	const int ntiles = s_p.L.tiles_x * s_p.L.tiles_y;
	__shared__ IdwtShared sh;
	idwt_body<kThreads>(sh, s_p, s_in, s_out, f < kBatchTileMapFrames ? &maps.frame[f] : nullptr, local % ntiles,
	                    local / ntiles);
}

// Canonical pyramid (all transmitted bands, band-major, unpadded) <-> padded storage.
__global__ void pyramid_io_kernel(const BlockParams p, float *canonical, float *coef32, __half *coef16,
                                  int to_canonical)
{
	const int k = blockIdx.y;
	const BandEntry &B = p.band[k];
	const LevelDesc &L = p.level[B.level];
	int64_t canon = 0;
	for (int j = 0; j < k; j++)
		canon += int64_t(p.level[p.band[j].level].width) * p.level[p.band[j].level].height;
	const int64_t n = int64_t(L.width) * L.height;
	for (int64_t i = int64_t(blockIdx.x) * blockDim.x + threadIdx.x; i < n; i += int64_t(gridDim.x) * blockDim.x)
	{
		const int y = int(i / L.width), x = int(i - int64_t(y) * L.width);
		const int64_t s = B.offset + int64_t(y) * L.pitch + x;
		if (to_canonical)
			canonical[canon + i] = L.fp16 ? __half2float(coef16[s]) : coef32[s];
		else
		{
			const float v = canonical[canon + i];
			if (L.fp16)
				coef16[s] = __float2half_rn(v);
			else
				coef32[s] = v;
		}
	}
}
} // namespace

void launch_dequant(const BlockParams &p, const DecodeInput &in, int first, int count, bool programmatic,
                    cudaStream_t stream)
{
	LaunchConfig lc(dim3(count), dim3(kDequantThreads), stream, programmatic);
	cudaLaunchKernelEx(&lc.cfg, dequant_kernel, p, in, first);
}

// SMs of the current device (queried once).
int device_sm_count()
{
	static int cached = 0;
	if (cached == 0)
	{
		int dev = 0, n = 0;
		if (cudaGetDevice(&dev) != cudaSuccess || cudaDeviceGetAttribute(&n, cudaDevAttrMultiProcessorCount, dev) != cudaSuccess ||
		    n <= 0)
		{
			(void)cudaGetLastError();
			n = 148;
		}
		cached = n;
	}
	return cached;
}

// Levels that fit one wave at three CTAs per SM run the 80-register CTAs (the
// faster per tile); larger levels run four 64-register CTAs per SM, so a level
// just above one wave at three (1080p level 0: 510 tiles) still runs in one.
void launch_idwt_level(const LevelParams &p, const DecodeInput &in, const PlaneOutput &out, const LevelTileMap *maps,
                       bool programmatic, cudaStream_t stream)
{
	const dim3 grid(p.L.tiles_x * p.L.tiles_y, (p.level == 0 && !p.chroma444) ? 1 : 3);
	LevelTileMap m = {};
	if (maps)
		m = *maps;
	if (int(grid.x * grid.y) < kSmallLevelTiles)
	{
		LaunchConfig lc(dim3(grid.x * kIdwtStripes, grid.y), dim3(256), stream, programmatic);
		cudaLaunchKernelEx(&lc.cfg, idwt_stripes_kernel, p, in, out, m);
	}
	else if (int(grid.x * grid.y) <= 3 * device_sm_count())
	{
		LaunchConfig lc(grid, dim3(256), stream, programmatic);
		cudaLaunchKernelEx(&lc.cfg, idwt_kernel<256>, p, in, out, m);
	}
	else
	{
		LaunchConfig lc(grid, dim3(256), stream, programmatic);
		cudaLaunchKernelEx(&lc.cfg, idwt_kernel<256, 4>, p, in, out, m);
	}
}

void launch_pyramid_io(const BlockParams &p, float *canonical, float *coef32, __half *coef16, bool to_canonical,
                       cudaStream_t stream)
{
	pyramid_io_kernel<<<dim3(64, p.nbands), 256, 0, stream>>>(p, canonical, coef32, coef16, to_canonical ? 1 : 0);
}

void launch_dequant_batch(const BatchFrame *frames, const uint32_t *cta_map, int nctas, bool programmatic,
                          cudaStream_t stream)
{
	LaunchConfig lc(dim3(nctas), dim3(128), stream, programmatic);
	cudaLaunchKernelEx(&lc.cfg, dequant_batch_kernel, frames, cta_map);
}

void launch_idwt_batch(const BatchFrame *frames, const BatchFrameIO *io, const uint32_t *cta_map, int nctas, int level,
                       const BatchTileMaps *maps, bool large_ctas, bool programmatic, cudaStream_t stream)
{
	static const BatchTileMaps none = {};
	const BatchTileMaps &m = maps ? *maps : none;
	if (large_ctas)
	{
		LaunchConfig lc(dim3(nctas), dim3(1024), stream, programmatic);
		cudaLaunchKernelEx(&lc.cfg, idwt_batch_kernel<1024>, frames, io, cta_map, level, m);
	}
	else if (nctas < kIdwtManyTiles)
	{
		LaunchConfig lc(dim3(nctas), dim3(256), stream, programmatic);
		cudaLaunchKernelEx(&lc.cfg, idwt_batch_kernel<256>, frames, io, cta_map, level, m);
	}
	else
	{
		LaunchConfig lc(dim3(nctas), dim3(256), stream, programmatic);
		cudaLaunchKernelEx(&lc.cfg, idwt_batch_kernel<256, 4>, frames, io, cta_map, level, m);
	}
}

} // namespace pw

// ---------------------------------------------------------------------------
// Decode without allocation (pyrowave_cuda_decode_blocks_static).
//
// The coefficient pyramid of the decode lives in one file-scope device array
// instead of memory owned by a decoder object. In host code the array's name
// only stands in for it: the device address is looked up with
// cudaGetSymbolAddress, with the caller's device current, on every call. The
// lookup allocates nothing once this library's device code is loaded on the
// device; with lazy module loading (the CUDA default) the first lookup on a
// device is where CUDA reserves the array, so it can fail there for lack of
// memory. Looking it up each time keeps a device reset (which unloads the
// module and may move the array) from leaving a stale address behind.
#include "pyrowave_cuda.h"

namespace
{
constexpr size_t kStaticScratchBytes = PYROWAVE_CUDA_STATIC_DECODE_SCRATCH_BYTES;
static __device__ __align__(256) float g_static_pyramid[kStaticScratchBytes / sizeof(float)];

// Device address of the array on the current device, or the failure.
pyrowave_result static_pyramid_on_current_device(float *&ptr)
{
	ptr = nullptr;
	const cudaError_t e = cudaGetSymbolAddress(reinterpret_cast<void **>(&ptr), g_static_pyramid);
	if (e != cudaSuccess || !ptr)
	{
		(void)cudaGetLastError();
		ptr = nullptr;
		return e == cudaErrorMemoryAllocation ? PYROWAVE_ERROR_OUT_OF_DEVICE_MEMORY : PYROWAVE_ERROR_GENERIC;
	}
	return PYROWAVE_SUCCESS;
}
} // namespace

extern "C" pyrowave_result pyrowave_cuda_decode_blocks_static(int width, int height,
                                                              pyrowave_chroma_subsampling chroma,
                                                              const uint32_t *block_meta, const uint32_t *words,
                                                              size_t num_words, const pyrowave_cuda_planes *planes,
                                                              pyrowave_cuda_stream stream)
{
	using namespace pw;
	// Frame rules of pyrowave_decoder_create, buffer rules of pyrowave_cuda_decoder_decode_blocks.
	if (width <= 0 || height <= 0)
		return PYROWAVE_ERROR_INVALID_ARGUMENT;
	if (chroma != PYROWAVE_CHROMA_SUBSAMPLING_420 && chroma != PYROWAVE_CHROMA_SUBSAMPLING_444)
		return PYROWAVE_ERROR_INVALID_ARGUMENT;
	if (chroma == PYROWAVE_CHROMA_SUBSAMPLING_420 && ((width & 1) || (height & 1)))
		return PYROWAVE_ERROR_INVALID_ARGUMENT;
	if (!block_meta || !words || !planes || num_words > 0xffffffffu)
		return PYROWAVE_ERROR_INVALID_ARGUMENT;
	Geometry g;
	if (!make_geometry(g, width, height, chroma == PYROWAVE_CHROMA_SUBSAMPLING_444, 0))
		return PYROWAVE_ERROR_INVALID_ARGUMENT;
	if (size_t(g.storage_elems32) * sizeof(float) > kStaticScratchBytes)
		return PYROWAVE_ERROR_INVALID_ARGUMENT;
	PlaneOutput out = {};
	for (int p = 0; p < 3; p++)
	{
		if (!planes->data[p] || planes->row_stride_in_bytes[p] < size_t(g.plane_width[p]) ||
		    planes->row_stride_in_bytes[p] > 0x7fffffffu)
			return PYROWAVE_ERROR_INVALID_ARGUMENT;
		out.data[p] = static_cast<uint8_t *>(planes->data[p]);
		out.pitch[p] = int32_t(planes->row_stride_in_bytes[p]);
	}
	float *scratch = nullptr;
	const pyrowave_result looked_up = static_pyramid_on_current_device(scratch);
	if (looked_up != PYROWAVE_SUCCESS)
		return looked_up;

	DecodeInput in = {};
	in.block_meta = block_meta;
	in.payload = words;
	in.payload_words = uint32_t(num_words);
	in.coef32 = scratch;
	in.coef16 = nullptr; // every level is FP32 here
	const cudaStream_t s = reinterpret_cast<cudaStream_t>(stream);
	launch_dequant(make_block_params(g), in, 0, g.block_count_32x32, false, s);
	for (int level = kLevels - 1; level >= 0; level--)
		launch_idwt_level(make_level_params(g, level), in, out, nullptr, true, s);
	return cudaGetLastError() == cudaSuccess ? PYROWAVE_SUCCESS : PYROWAVE_ERROR_GENERIC;
}
