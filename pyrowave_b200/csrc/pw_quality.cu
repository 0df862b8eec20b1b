// PSNR-HVS-M quality metric for sm_100a: the reference's perceptual metric
// (shaders/psnr_hvs_m.comp:1-225, with the host tables of psnr.cpp:25-28,
// 126-224 and the 16 height factors of psnr.cpp:245-320) over a luma plane
// and its reference, without allocating anything.
//
// Work split: a half-warp per 8x8 window (windows at a stride of 4 samples).
// Its 16 lanes stage the two windows in shared memory, eight of them run the
// row and then the column DCTs of both windows (one 8-point DCT each), and
// then lane f evaluates height factor f: the masking of both windows and the
// CSF-weighted error of the window pair. The per-factor fixed-point (2^-24)
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
constexpr int kHvsThreads = 128;
constexpr int kHvsSlots = kHvsThreads / 16; // windows per CTA and round

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

// The factor-independent part of maskeff (psnr_hvs_m.comp:109-153).
__device__ float window_pop(const float (&sig)[8][9])
{
	float sum_e2[2][2], sum_e[2][2];
	float sum_e2_total = 0.0f, sum_e_total = 0.0f;
	for (int y = 0; y < 2; y++)
		for (int x = 0; x < 2; x++)
		{
			float e = 0.0f, e2 = 0.0f;
			for (int suby = 0; suby < 4; suby++)
				for (int subx = 0; subx < 4; subx++)
				{
					const float v = sig[y * 4 + suby][x * 4 + subx];
					e = __fadd_rn(e, v);
					e2 = __fadd_rn(e2, __fmul_rn(v, v));
				}
			sum_e[y][x] = e;
			sum_e2[y][x] = e2;
			sum_e_total = __fadd_rn(sum_e_total, e);
			sum_e2_total = __fadd_rn(sum_e2_total, e2);
		}
	float pop = vari(sum_e_total, sum_e2_total, 64);
	if (pop != 0.0f)
	{
		float q = __fadd_rn(vari(sum_e[0][0], sum_e2[0][0], 16), vari(sum_e[1][0], sum_e2[1][0], 16));
		q = __fadd_rn(q, vari(sum_e[0][1], sum_e2[0][1], 16));
		q = __fadd_rn(q, vari(sum_e[1][1], sum_e2[1][1], 16));
		pop = __fdiv_rn(q, pop);
	}
	return pop;
}

__global__ void __launch_bounds__(kHvsThreads) psnr_hvs_m_kernel(const __grid_constant__ HvsParams hp,
                                                                 const uint8_t *ref, const int ref_pitch,
                                                                 const uint8_t *dist, const int dist_pitch,
                                                                 unsigned long long *errors)
{
	__shared__ float s_csf[64][kHvsFactors], s_mask[64][kHvsFactors], s_inv[64][kHvsFactors];
	__shared__ float s_sig[kHvsSlots][2][8][9]; // [window][image][y][x], then the 2D DCT in place
	__shared__ float s_pop[kHvsSlots][2];
	__shared__ unsigned long long s_err[kHvsFactors];
	for (int i = threadIdx.x; i < 64 * kHvsFactors; i += kHvsThreads)
	{
		(&s_csf[0][0])[i] = (&hp.csf[0][0])[i];
		(&s_mask[0][0])[i] = (&hp.mask[0][0])[i];
		(&s_inv[0][0])[i] = (&hp.inv_mask[0][0])[i];
	}
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
			{
				const uint8_t u = img == 0 ? ref[size_t(py) * ref_pitch + px] : dist[size_t(py) * dist_pitch + px];
				v = __fdiv_rn(float(u), 255.0f);
			}
			sig[img][y][x] = v;
		}
		__syncwarp(half_mask);
		if (l < 2)
			s_pop[slot][l] = window_pop(sig[l]);
		__syncwarp(half_mask);
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
		// Height factor l: masking of both windows (maskeff), then the weighted error (dct_error).
		{
			float ma = 0.0f, mb = 0.0f;
			for (int k = 0; k < 64; k++)
			{
				const float a = sig[0][k >> 3][k & 7], b = sig[1][k >> 3][k & 7];
				ma = __fadd_rn(ma, __fmul_rn(__fmul_rn(a, a), s_mask[k][l]));
				mb = __fadd_rn(mb, __fmul_rn(__fmul_rn(b, b), s_mask[k][l]));
			}
			const float mask_a = __fdiv_rn(__fsqrt_rn(__fmul_rn(ma, s_pop[slot][0])), 32.0f);
			const float mask_b = __fdiv_rn(__fsqrt_rn(__fmul_rn(mb, s_pop[slot][1])), 32.0f);
			const float mask = fmaxf(mask_a, mask_b);
			float total = 0.0f;
			for (int k = 0; k < 64; k++)
			{
				const float e = fabsf(__fsub_rn(sig[0][k >> 3][k & 7], sig[1][k >> 3][k & 7]));
				const float m = __fmul_rn(mask, s_inv[k][l]);
				const float w = __fmul_rn(fmaxf(__fsub_rn(e, m), 0.0f), s_csf[k][l]);
				total = __fadd_rn(total, __fmul_rn(w, w));
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
	HvsParams hp;
	hvs_tables(height, hp);
	hp.width = width;
	hp.height = height;
	hp.nbx = (width - 1) / 4 + 1;
	hp.nby = (height - 1) / 4 + 1;
	const int nwin = hp.nbx * hp.nby;
	const int grid = std::max(1, std::min((nwin + kHvsSlots - 1) / kHvsSlots, 148 * 16));
	psnr_hvs_m_kernel<<<grid, kHvsThreads, 0, reinterpret_cast<cudaStream_t>(stream)>>>(
	    hp, reference, int(reference_stride), distorted, int(distorted_stride),
	    reinterpret_cast<unsigned long long *>(errors));
	return cudaGetLastError() == cudaSuccess ? PYROWAVE_SUCCESS : PYROWAVE_ERROR_GENERIC;
}
}
