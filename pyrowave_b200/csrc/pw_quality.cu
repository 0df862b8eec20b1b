// PSNR-HVS-M quality metric for sm_100a: the reference's perceptual metric
// (shaders/psnr_hvs_m.comp:1-225, with the host tables of psnr.cpp:25-28,
// 126-224 and the 16 height factors of psnr.cpp:245-320) over a luma plane
// and its reference, without allocating anything.
//
// Work split: a half-warp per 8x8 window (windows at a stride of 4 samples).
// Its 16 lanes stage the two windows in shared memory (UNORM values from a
// per-CTA table of x / 255), eight of them sum the four quadrants of both
// windows for the masking's variances, all 16 run the row and then the column
// DCTs (one 8-point DCT each), then each lane stores four coefficients' squares
// and absolute differences for the window, and lane f evaluates height factor
// f: the masking of both windows and the CSF-weighted error of the window
// pair, reading the coefficient terms and its factor's tables four at a time.
// The per-factor fixed-point (2^-24)
// error sums are integers, so their accumulation (per lane, per CTA in shared
// memory, then one global atomic per factor and CTA) is exact in any order.
// Every floating-point operation is one rounded IEEE operation in the order
// of the reference shader (the library builds with --fmad=false), which is
// also the oracle's order, so the sums are bit-identical to the oracle's.
#include "pw_device.cuh"

#include "pyrowave_cuda.h"

#include <algorithm>
#include <cmath>

namespace pw
{
namespace
{
constexpr int kHvsFactors = 16;
constexpr int kHvsThreads = 256;
constexpr int kHvsSlots = kHvsThreads / 16; // windows per CTA and round
constexpr int kHvsPitch = 68;               // floats per factor row of the shared tables (16-byte rows, no bank conflicts)

// The tables of all factors, factor-minor: entry [y * 8 + x][f], so the 16
// lanes of a window read 16 consecutive words.
struct HvsParams
{
	float csf[64][kHvsFactors];
	float mask[64][kHvsFactors];
	float inv_mask[64][kHvsFactors];
	int32_t width, height, nbx, nby;
};

__device__ __forceinline__ void butterfly(float &a, float &b)
{
	const float pos = __fadd_rn(a, b), neg = __fsub_rn(a, b);
	a = pos;
	b = neg;
}

__device__ __forceinline__ void rotate(float &a, float &b, float c, float s)
{
	const float pos = __fadd_rn(__fmul_rn(a, c), __fmul_rn(b, s));
	const float neg = __fsub_rn(__fmul_rn(b, c), __fmul_rn(a, s));
	a = pos;
	b = neg;
}

// 8-point DCT by butterflies (psnr_hvs_m.comp:58-97): s in signal order, out in frequency order.
__device__ __forceinline__ void dct8(float (&s)[8], float (&out)[8])
{
	const float c7 = 0.19509032201612833f, s7 = 0.9807852804032304f;
	const float c6 = 0.38268343236508984f, s6 = 0.9238795325112867f;
	const float c5 = 0.5555702330196023f, s5 = 0.8314696123025452f;
	const float r1 = __fsqrt_rn(0.125f), r2 = __fsqrt_rn(0.25f);
	butterfly(s[0], s[7]);
	butterfly(s[1], s[6]);
	butterfly(s[2], s[5]);
	butterfly(s[3], s[4]);
	butterfly(s[0], s[3]);
	butterfly(s[1], s[2]);
	butterfly(s[0], s[1]);
	rotate(s[2], s[3], c6, s6);
	rotate(s[4], s[7], c7, s7);
	rotate(s[5], s[6], c5, s5);
	butterfly(s[4], s[5]);
	butterfly(s[6], s[7]);
	butterfly(s[5], s[6]);
	out[0] = __fmul_rn(s[0], r1);
	out[1] = __fmul_rn(s[4], r2);
	out[2] = __fmul_rn(s[2], r2);
	out[3] = __fmul_rn(s[5], r1);
	out[4] = __fmul_rn(s[1], r1);
	out[5] = __fmul_rn(s[6], r1);
	out[6] = __fmul_rn(s[3], r2);
	out[7] = __fmul_rn(s[7], -r2);
}

__device__ __forceinline__ float vari(float e, float e2, int count) // psnr_hvs_m.comp:104-107
{
	return __fdiv_rn(fmaxf(__fsub_rn(__fmul_rn(e2, float(count)), __fmul_rn(e, e)), 0.0f), float(count - 1));
}

// Sum and sum of squares of quadrant (y, x) = (q >> 1, q & 1) of a window, in
// the row-major order of psnr_hvs_m.comp:115-126.
__device__ __forceinline__ void quadrant_sums(const float (&sig)[8][9], int q, float &e, float &e2)
{
	const int y0 = (q >> 1) * 4, x0 = (q & 1) * 4;
	e = 0.0f;
	e2 = 0.0f;
	for (int suby = 0; suby < 4; suby++)
		for (int subx = 0; subx < 4; subx++)
		{
			const float v = sig[y0 + suby][x0 + subx];
			e = __fadd_rn(e, v);
			e2 = __fadd_rn(e2, __fmul_rn(v, v));
		}
}

// The factor-independent part of maskeff (psnr_hvs_m.comp:109-153) from the
// quadrant sums {e, e2} in quadrant order (0,0), (0,1), (1,0), (1,1): the
// totals add them in that order, the variance ratio in the shader's order
// (0,0), (1,0), (0,1), (1,1).
__device__ float window_pop(const float (&quad)[4][2])
{
	float sum_e_total = 0.0f, sum_e2_total = 0.0f;
	for (int q = 0; q < 4; q++)
	{
		sum_e_total = __fadd_rn(sum_e_total, quad[q][0]);
		sum_e2_total = __fadd_rn(sum_e2_total, quad[q][1]);
	}
	float pop = vari(sum_e_total, sum_e2_total, 64);
	if (pop != 0.0f)
	{
		float v = __fadd_rn(vari(quad[0][0], quad[0][1], 16), vari(quad[2][0], quad[2][1], 16));
		v = __fadd_rn(v, vari(quad[1][0], quad[1][1], 16));
		v = __fadd_rn(v, vari(quad[3][0], quad[3][1], 16));
		pop = __fdiv_rn(v, pop);
	}
	return pop;
}

__global__ void __launch_bounds__(kHvsThreads) psnr_hvs_m_kernel(const __grid_constant__ HvsParams hp,
                                                                 const uint8_t *ref, const int ref_pitch,
                                                                 const uint8_t *dist, const int dist_pitch,
                                                                 unsigned long long *errors)
{
	// Tables factor-major ([f][k], rows of kHvsPitch): lane f reads four
	// consecutive coefficients of its own row as one 16-byte load.
	__shared__ __align__(16) float s_csf[kHvsFactors][kHvsPitch], s_mask[kHvsFactors][kHvsPitch],
	    s_inv[kHvsFactors][kHvsPitch];
	__shared__ float s_unorm[256];
	__shared__ float s_sig[kHvsSlots][2][8][9]; // [window][image][y][x], then the 2D DCT in place
	// Per window and coefficient: a^2, b^2 and |a - b| of the two DCTs.
	__shared__ __align__(16) float s_a2[kHvsSlots][64], s_b2[kHvsSlots][64], s_diff[kHvsSlots][64];
	__shared__ float s_quad[kHvsSlots][2][4][2];
	__shared__ float s_pop[kHvsSlots][2];
	__shared__ unsigned long long s_err[kHvsFactors];
	for (int i = threadIdx.x; i < 64 * kHvsFactors; i += kHvsThreads)
	{
		const int k = i / kHvsFactors, f = i % kHvsFactors;
		s_csf[f][k] = (&hp.csf[0][0])[i];
		s_mask[f][k] = (&hp.mask[0][0])[i];
		s_inv[f][k] = (&hp.inv_mask[0][0])[i];
	}
	for (int i = threadIdx.x; i < 256; i += kHvsThreads)
		s_unorm[i] = __fdiv_rn(float(i), 255.0f);
	if (threadIdx.x < kHvsFactors)
		s_err[threadIdx.x] = 0ull;
	__syncthreads();

	const int lane = threadIdx.x & 31, l = lane & 15;
	const int slot = threadIdx.x >> 4;
	const unsigned half_mask = (lane < 16) ? 0x0000ffffu : 0xffff0000u;
	float(&sig)[2][8][9] = s_sig[slot];
	const int nwin = hp.nbx * hp.nby;
	unsigned long long acc = 0ull; // factor l
	for (int base = int(blockIdx.x) * kHvsSlots; base < nwin; base += int(gridDim.x) * kHvsSlots)
	{
		const int win = base + slot;
		const bool valid = win < nwin;
		const int wx = valid ? (win % hp.nbx) * 4 : 0, wy = valid ? (win / hp.nbx) * 4 : 0;
		// Both windows: 128 samples, UNORM to float; outside the plane reads zero.
		for (int k = l; k < 128; k += 16)
		{
			const int img = k >> 6, y = (k >> 3) & 7, x = k & 7;
			const int px = wx + x, py = wy + y;
			float v = 0.0f;
			if (valid && px < hp.width && py < hp.height)
				v = s_unorm[img == 0 ? ref[size_t(py) * ref_pitch + px] : dist[size_t(py) * dist_pitch + px]];
			sig[img][y][x] = v;
		}
		__syncwarp(half_mask);
		if (l < 8)
			quadrant_sums(sig[l >> 2], l & 3, s_quad[slot][l >> 2][l & 3][0], s_quad[slot][l >> 2][l & 3][1]);
		__syncwarp(half_mask);
		if (l < 2)
			s_pop[slot][l] = window_pop(s_quad[slot][l]);
		// Row DCTs (lanes 0-7 the reference window, 8-15 the distorted one), then column DCTs.
		{
			const int img = l >> 3, r = l & 7;
			float s[8], d[8];
			for (int i = 0; i < 8; i++)
				s[i] = sig[img][r][i];
			dct8(s, d);
			for (int i = 0; i < 8; i++)
				sig[img][r][i] = d[i];
			__syncwarp(half_mask);
			for (int i = 0; i < 8; i++)
				s[i] = sig[img][i][r];
			dct8(s, d);
			for (int i = 0; i < 8; i++)
				sig[img][i][r] = d[i];
		}
		__syncwarp(half_mask);
		{
			float a2[4], b2[4], df[4];
#pragma unroll
			for (int j = 0; j < 4; j++)
			{
				const int k = 4 * l + j;
				const float a = sig[0][k >> 3][k & 7], b = sig[1][k >> 3][k & 7];
				a2[j] = __fmul_rn(a, a);
				b2[j] = __fmul_rn(b, b);
				df[j] = fabsf(__fsub_rn(a, b));
			}
			*reinterpret_cast<float4 *>(&s_a2[slot][4 * l]) = make_float4(a2[0], a2[1], a2[2], a2[3]);
			*reinterpret_cast<float4 *>(&s_b2[slot][4 * l]) = make_float4(b2[0], b2[1], b2[2], b2[3]);
			*reinterpret_cast<float4 *>(&s_diff[slot][4 * l]) = make_float4(df[0], df[1], df[2], df[3]);
		}
		__syncwarp(half_mask);
		// Height factor l: masking of both windows (maskeff), then the weighted error (dct_error).
		{
			float ma = 0.0f, mb = 0.0f;
#pragma unroll 4
			for (int k = 0; k < 64; k += 4)
			{
				const float4 A = *reinterpret_cast<const float4 *>(&s_a2[slot][k]);
				const float4 B = *reinterpret_cast<const float4 *>(&s_b2[slot][k]);
				const float4 M = *reinterpret_cast<const float4 *>(&s_mask[l][k]);
				ma = __fadd_rn(ma, __fmul_rn(A.x, M.x));
				mb = __fadd_rn(mb, __fmul_rn(B.x, M.x));
				ma = __fadd_rn(ma, __fmul_rn(A.y, M.y));
				mb = __fadd_rn(mb, __fmul_rn(B.y, M.y));
				ma = __fadd_rn(ma, __fmul_rn(A.z, M.z));
				mb = __fadd_rn(mb, __fmul_rn(B.z, M.z));
				ma = __fadd_rn(ma, __fmul_rn(A.w, M.w));
				mb = __fadd_rn(mb, __fmul_rn(B.w, M.w));
			}
			const float mask_a = __fdiv_rn(__fsqrt_rn(__fmul_rn(ma, s_pop[slot][0])), 32.0f);
			const float mask_b = __fdiv_rn(__fsqrt_rn(__fmul_rn(mb, s_pop[slot][1])), 32.0f);
			const float mask = fmaxf(mask_a, mask_b);
			float total = 0.0f;
#pragma unroll 4
			for (int k = 0; k < 64; k += 4)
			{
				const float4 E = *reinterpret_cast<const float4 *>(&s_diff[slot][k]);
				const float4 I = *reinterpret_cast<const float4 *>(&s_inv[l][k]);
				const float4 C = *reinterpret_cast<const float4 *>(&s_csf[l][k]);
				const float e[4] = {E.x, E.y, E.z, E.w}, inv[4] = {I.x, I.y, I.z, I.w}, csf[4] = {C.x, C.y, C.z, C.w};
#pragma unroll
				for (int j = 0; j < 4; j++)
				{
					const float w = __fmul_rn(fmaxf(__fsub_rn(e[j], __fmul_rn(mask, inv[j])), 0.0f), csf[j]);
					total = __fadd_rn(total, __fmul_rn(w, w));
				}
			}
			if (valid)
				acc += __float2ull_rz(__fmul_rn(total, 16777216.0f)); // ldexp(total, 24), truncated
		}
		__syncwarp(half_mask);
	}
	atomicAdd(&s_err[l], acc);
	__syncthreads();
	if (threadIdx.x < kHvsFactors && s_err[threadIdx.x])
		atomicAdd(errors + threadIdx.x, s_err[threadIdx.x]);
}

// Host tables of one plane height (psnr.cpp:25-28,151-195), written in the
// same operation order as the oracle's so both get the same floats.
float contrast_sensitivity(float cpd)
{
	return 2.6f * (0.0192f + 0.114f * cpd) * std::exp(-std::pow(0.114f * cpd, 1.1f));
}

void hvs_tables(int height, HvsParams &hp)
{
	for (int f = 0; f < kHvsFactors; f++)
	{
		const float height_factor = 1.0f + float(f) / 8.0f; // psnr.cpp:245-248
		const float pi = 3.14159265358979323846f;
		const float nyquist_cpd = float(height) * height_factor * pi / 360.0f;
		float csf[8][8];
		for (int y = 0; y < 8; y++)
			for (int x = 0; x < 8; x++)
			{
				const float H = (float(x) + 0.5f) / 8.0f;
				const float V = (float(y) + 0.5f) / 8.0f;
				const float cpd = std::sqrt(H * H + V * V);
				csf[y][x] = 2.6f * contrast_sensitivity(cpd * nyquist_cpd);
			}
		float max_csf = 0.0f;
		for (auto &row : csf)
			for (float v : row)
				max_csf = std::max(max_csf, v);
		float norm = 1.0f / max_csf;
		norm *= norm;
		for (int y = 0; y < 8; y++)
			for (int x = 0; x < 8; x++)
			{
				const float m = (y || x) ? csf[y][x] * csf[y][x] * norm : 0.0f;
				hp.csf[y * 8 + x][f] = csf[y][x];
				hp.mask[y * 8 + x][f] = m;
				hp.inv_mask[y * 8 + x][f] = (y || x) ? 1.0f / m : 0.0f;
			}
	}
}
} // namespace
} // namespace pw

extern "C" {

uint64_t pyrowave_psnr_hvs_m_pixels(int width, int height)
{
	if (width <= 0 || height <= 0)
		return 0;
	const uint64_t bx = uint64_t((width - 1) / 4 + 1), by = uint64_t((height - 1) / 4 + 1);
	return bx * by * 64;
}

void pyrowave_psnr_hvs_m_from_errors(const uint64_t *errors, uint64_t total_pixels, bool full_range, double *psnr)
{
	if (!errors || !psnr)
		return;
	// psnr.cpp:220-240: errors are fixed point 2^-24; limited range scales the peak to 223/255.
	const double peak = full_range ? 1.0 : (223.0 * 223.0) / (255.0 * 255.0);
	for (int i = 0; i < pw::kHvsFactors; i++)
	{
		const double e = std::ldexp(double(errors[i]), -24);
		psnr[i] = e > 0.0 ? 10.0 * std::log10(double(total_pixels) * peak / e) : INFINITY;
	}
}

pyrowave_result pyrowave_cuda_psnr_hvs_m(int width, int height, const uint8_t *reference, size_t reference_stride,
                                         const uint8_t *distorted, size_t distorted_stride, uint64_t *errors,
                                         pyrowave_cuda_stream stream)
{
	using namespace pw;
	if (width <= 0 || height <= 0 || !reference || !distorted || !errors)
		return PYROWAVE_ERROR_INVALID_ARGUMENT;
	if (reference_stride < size_t(width) || distorted_stride < size_t(width) || reference_stride > 0x7fffffffu ||
	    distorted_stride > 0x7fffffffu || (reinterpret_cast<uintptr_t>(errors) & 7u) != 0)
		return PYROWAVE_ERROR_INVALID_ARGUMENT;
	// The tables depend only on the plane height; each calling thread keeps the
	// last height's (about 1000 exp/pow evaluations otherwise per call).
	thread_local int table_height = -1;
	thread_local HvsParams hp;
	if (table_height != height)
	{
		hvs_tables(height, hp);
		table_height = height;
	}
	hp.width = width;
	hp.height = height;
	hp.nbx = (width - 1) / 4 + 1;
	hp.nby = (height - 1) / 4 + 1;
	const int nwin = hp.nbx * hp.nby;
	// A few CTAs per SM, each looping over windows: every CTA copies the tables
	// into shared memory once.
	int device = 0, sms = 148;
	if (cudaGetDevice(&device) != cudaSuccess ||
	    cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, device) != cudaSuccess)
		return PYROWAVE_ERROR_GENERIC;
	const int grid = std::max(1, std::min((nwin + kHvsSlots - 1) / kHvsSlots, sms * 4));
	psnr_hvs_m_kernel<<<grid, kHvsThreads, 0, reinterpret_cast<cudaStream_t>(stream)>>>(
	    hp, reference, int(reference_stride), distorted, int(distorted_stride),
	    reinterpret_cast<unsigned long long *>(errors));
	return cudaGetLastError() == cudaSuccess ? PYROWAVE_SUCCESS : PYROWAVE_ERROR_GENERIC;
}
}
