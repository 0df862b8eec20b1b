// Packing analysis of an encoded frame on the device.
//
// The reference carries a disabled statistics pass (pyrowave_encoder.cpp:625-958,
// Encoder::Impl::report_stats and analyze_alternative_packing) that reads a
// frame's quantised coefficients back and estimates what other packet, block and
// sub-block shapes would have cost, next to the coded bytes per band and the
// byte histograms of each bit plane. This kernel computes the same statistics
// for the current block format straight from the encoder's device buffers: the
// quantiser's 16-bit magnitudes, the code words and the rate-control quant
// drops give each coefficient's integer exactly as the packer codes it (bits
// [quant, quant + planes) of the magnitude), and the plane bytes are the ones
// the packer writes. It is a reporting tool beside the hot path, not part of it.
#include "pw_internal.h"

#include "pw_device.cuh"

namespace pw
{
namespace
{
constexpr int kAnalysisThreads = 256;

struct AnalysisShared
{
	uint16_t v[64][64];       // the region's integer magnitudes (row-major)
	uint32_t hist[16][256];   // plane bytes by position in their sub-block's run of planes
	uint8_t sub_bits[1024];   // per sub-block of the layout being costed: magnitude bits
	uint8_t sub_nnz[1024];    //   and significant values
	uint32_t packet_any[4];   // per packet of that layout: any significant value
	unsigned long long cost[kPackingLayouts];
	unsigned int significant;
};

__device__ __forceinline__ int magnitude_bits(uint32_t v) { return 32 - __clz(v); }

// analyze_cost<PW, PH, SW, SH> (pyrowave_encoder.cpp:650-713) of the region in
// shared memory, added into sh.cost[which]: 8 bytes per PW x PH packet holding a
// significant value; per (PW/4) x (PH/4) block holding one, 2 bits of plane
// code per SW x SH sub-block and a byte of Q bits and scale, then every
// sub-block's planes at max(its magnitude bits, Q bits) with Q bits the block's
// magnitude bits minus 3, and one sign bit per significant value, in bytes.
// Sub-blocks are costed one per thread, then blocks one per thread.
template <int PW, int PH, int SW, int SH>
__device__ void layout_cost(AnalysisShared &sh, int which)
{
	constexpr int BW = PW / 4, BH = PH / 4;
	constexpr int NSX = BW / SW, NS = NSX * (BH / SH);
	constexpr int NBX = 64 / BW, NB = NBX * (64 / BH);
	constexpr int NPX = 64 / PW, NP = NPX * (64 / PH);
	static_assert(NB * NS <= 1024 && NP <= 4, "layout fits the shared arrays");
	for (int s = threadIdx.x; s < NB * NS; s += kAnalysisThreads)
	{
		const int b = s / NS, k = s - b * NS;
		const int x0 = (b % NBX) * BW + (k % NSX) * SW, y0 = (b / NBX) * BH + (k / NSX) * SH;
		uint32_t m = 0, n = 0;
#pragma unroll
		for (int y = 0; y < SH; y++)
#pragma unroll
			for (int x = 0; x < SW; x++)
			{
				const uint32_t val = sh.v[y0 + y][x0 + x];
				m = max(m, val);
				n += val != 0 ? 1u : 0u;
			}
		sh.sub_bits[s] = uint8_t(magnitude_bits(m));
		sh.sub_nnz[s] = uint8_t(n);
	}
	__syncthreads();
	uint32_t cost = 0;
	for (int b = threadIdx.x; b < NB; b += kAnalysisThreads)
	{
		int bits = 0, nnz = 0;
		for (int k = 0; k < NS; k++)
		{
			bits = max(bits, int(sh.sub_bits[b * NS + k]));
			nnz += sh.sub_nnz[b * NS + k];
		}
		if (bits == 0)
			continue;
		const int q_bits = max(bits - 3, 0);
		int weight = 0;
		for (int k = 0; k < NS; k++)
			weight += SW * SH * max(int(sh.sub_bits[b * NS + k]), q_bits);
		cost += uint32_t(2 * NS / 8 + 1 + (weight + nnz + 7) / 8);
		const int bx = b % NBX, by = b / NBX;
		sh.packet_any[(by * BH / PH) * NPX + bx * BW / PW] = 1u;
	}
#pragma unroll
	for (int off = 16; off > 0; off >>= 1)
		cost += __shfl_xor_sync(0xffffffffu, cost, off);
	if ((threadIdx.x & 31) == 0 && cost != 0)
		atomicAdd(&sh.cost[which], (unsigned long long)cost);
	__syncthreads();
	if (threadIdx.x == 0)
	{
		unsigned long long headers = 0;
		for (int p = 0; p < NP; p++)
		{
			headers += sh.packet_any[p] ? 8u : 0u;
			sh.packet_any[p] = 0;
		}
		sh.cost[which] += headers;
	}
	__syncthreads();
}

// One CTA per 64x64 region of a coded band: regions[5 * r + q] is the 32x32
// block at quadrant q (x = q & 1, y = q >> 1; -1 beyond the band) and
// regions[5 * r + 4] the band's slot (component * 5 + level) * 4 + band.
__global__ void __launch_bounds__(kAnalysisThreads) packing_analysis_kernel(const BlockParams p, const EncodeBuffers buf,
                                                                            const int32_t *regions,
                                                                            PackingAnalysisAccum *acc)
{
	__shared__ AnalysisShared sh;
	const int t = threadIdx.x;
	for (int i = t; i < 16 * 256; i += kAnalysisThreads)
		(&sh.hist[0][0])[i] = 0;
	if (t < 4)
		sh.packet_any[t] = 0;
	if (t < kPackingLayouts)
		sh.cost[t] = 0;
	if (t == 0)
		sh.significant = 0;
	__syncthreads();

	const int32_t *region = regions + 5 * int64_t(blockIdx.x);
	const int q = t >> 6, qx = (q & 1) * 32, qy = (q >> 1) * 32;
	const int blk = region[q];
	uint32_t words = 0;
	int quant = 0;
	if (blk >= 0)
	{
		words = __ldcg(reinterpret_cast<const uint2 *>(buf.block_meta) + blk).y;
		quant = __ldcg(&buf.quant[blk]);
	}
	unsigned int significant = 0;
#pragma unroll
	for (int h = 0; h < 2; h++)
	{
		const int sb = (t & 63) + 64 * h, sub = sb & 7, lx = (sb >> 3) & 3, ly = sb >> 5;
		uint32_t mag[8] = {};
		uint32_t planes = 0;
		if (blk >= 0 && words != 0)
		{
			const BandEntry &B = p.band[find_band(p, blk)];
			const LevelDesc &L = p.level[B.level];
			const int rel = blk - B.block32_offset;
			const int by32 = rel / B.block32_stride, bx32 = rel - by32 * B.block32_stride;
			const int x8 = bx32 * 4 + lx, y8 = by32 * 4 + ly;
			const uint32_t cw0 = (x8 < L.blocks8_x && y8 < L.blocks8_y)
			                         ? __ldcg(&buf.code_words[B.block8_offset + y8 * B.block8_stride + x8])
			                         : 0u;
			const uint32_t cw = quantize_code_word(cw0, quant);
			if ((cw & 0xffffu) != 0)
				planes = ((cw >> (2 * sub)) & 3u) + ((cw >> kQPlanesOffset) & 0xfu);
			if (planes != 0)
			{
				const uint4 w4 = __ldcg(
				    reinterpret_cast<const uint4 *>(buf.mag16 + int64_t(blk) * 1024 + 8 * (sub + 8 * lx + 32 * ly)));
				const uint32_t w[4] = {w4.x, w4.y, w4.z, w4.w};
#pragma unroll
				for (int i = 0; i < 8; i++)
					mag[i] = (w[i >> 1] >> (16 * (i & 1))) & 0x7fffu;
				for (uint32_t pl = 0; pl < planes && pl < 16; pl++)
				{
					const uint32_t bit = uint32_t(quant) + planes - 1u - pl; // most significant plane first
					uint32_t byte = 0;
#pragma unroll
					for (int i = 0; i < 8; i++)
						byte |= (bit < 32 ? (mag[i] >> bit) & 1u : 0u) << i;
					atomicAdd(&sh.hist[pl][byte], 1u);
				}
			}
		}
		const uint32_t keep = planes >= 32 ? 0xffffffffu : (1u << planes) - 1u;
		const int x0 = qx + lx * 8 + sub_x(sub), y0 = qy + ly * 8 + sub_y(sub);
#pragma unroll
		for (int i = 0; i < 8; i++)
		{
			const uint32_t val = planes != 0 ? (mag[i] >> quant) & keep : 0u;
			sh.v[y0 + (i & 1)][x0 + (i >> 1)] = uint16_t(val);
			significant += val != 0 ? 1u : 0u;
		}
	}
	if ((t & 63) == 0 && blk >= 0 && words != 0)
		atomicAdd(&acc->band_bytes[region[4]], (unsigned long long)words * 4ull);
#pragma unroll
	for (int off = 16; off > 0; off >>= 1)
		significant += __shfl_xor_sync(0xffffffffu, significant, off);
	if ((t & 31) == 0 && significant != 0)
		atomicAdd(&sh.significant, significant);
	__syncthreads();

	layout_cost<32, 32, 2, 2>(sh, 0);
	layout_cost<32, 32, 4, 2>(sh, 1);
	layout_cost<32, 32, 2, 4>(sh, 2);
	layout_cost<64, 32, 4, 4>(sh, 3);
	layout_cost<64, 64, 8, 4>(sh, 4);

	if (t < kPackingLayouts && sh.cost[t] != 0)
		atomicAdd(&acc->layout_bytes[t], sh.cost[t]);
	if (t == 0 && sh.significant != 0)
		atomicAdd(&acc->significant, (unsigned long long)sh.significant);
	for (int i = t; i < 16 * 256; i += kAnalysisThreads)
	{
		const uint32_t n = (&sh.hist[0][0])[i];
		if (n != 0)
			atomicAdd(&acc->plane_histogram[i], n);
	}
}
} // namespace

cudaError_t launch_packing_analysis(const BlockParams &p, const EncodeBuffers &buf, const int32_t *regions,
                                    int num_regions, PackingAnalysisAccum *acc, cudaStream_t stream)
{
	cudaError_t e = cudaMemsetAsync(acc, 0, sizeof(PackingAnalysisAccum), stream);
	if (e != cudaSuccess || num_regions == 0)
		return e;
	packing_analysis_kernel<<<num_regions, kAnalysisThreads, 0, stream>>>(p, buf, regions, acc);
	return cudaGetLastError();
}
} // namespace pw
