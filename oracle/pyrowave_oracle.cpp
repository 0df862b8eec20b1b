// PyroWave CPU oracle -- TEST INFRASTRUCTURE ONLY (the checker, never the product).
//
// A line-by-line CPU restatement of the reference's encode/decode path. Every
// function cites the reference file:line it follows. Arithmetic conventions,
// chosen so that the CUDA implementation can be compared bit for bit:
//   * FP32 operations are IEEE round-to-nearest operations with no implicit
//     contraction (build with -ffp-contract=off), no fast-math. Where a shader
//     statement is a multiply-add (a lifting step x += c * (a + b), the squared
//     sums of dot()), it is one fused multiply-add (std::fmaf), which is what
//     an FMA-capable GPU compiles those statements to.
//   * Subgroup float reductions use the xor-butterfly order (lanes 1,2,4,8).
//   * FP16 conversions are IEEE round-to-nearest-even.
//   * The rate-control bucket index uses the exactly rounded value of
//     60 + 2*log2(r) instead of a GPU log2 approximation (see bucket_index()).
#include "pyrowave_oracle.h"

#include <algorithm>
#include <cmath>
#include <cstdio>
#include <cstdlib>
#include <cstring>
#include <type_traits>
#include <vector>

namespace
{
// ---------------------------------------------------------------------------
// Constants: pyrowave_common.hpp:112-124, bitstream.md:99-106
constexpr int DecompositionLevels = 5;
constexpr int Alignment = 1 << DecompositionLevels;
constexpr int MinimumImageSize = 4 << DecompositionLevels;
constexpr int NumComponents = 3;
constexpr int MaxScaleExp = 4;
// constants.h:4-8
constexpr int Q_PLANES_OFFSET = 16;
constexpr int QUANT_SCALE_OFFSET = 20;
// dwt_quant_scale.h:12
constexpr uint32_t ENCODE_QUANT_IDENTITY = 6;
// pyrowave_encoder.cpp:17-19
constexpr int BlockSpaceSubdivision = 16;
constexpr int NumRDOBuckets = 128;

// Lifting constants: dwt_common.h:37-42 (GLSL float literals, so rounded to float;
// inv_K is a float division of the two literals).
const float ALPHA = -1.586134342059924f;
const float BETA = -0.052980118572961f;
const float GAMMA = 0.882911075530934f;
const float DELTA = 0.443506852043971f;
const float KF = 1.230174104914001f;
const float INV_KF = 1.0f / 1.230174104914001f;

const double ALPHA_D = -1.586134342059924;
const double BETA_D = -0.052980118572961;
const double GAMMA_D = 0.882911075530934;
const double DELTA_D = 0.443506852043971;
const double K_D = 1.230174104914001;

int align_up(int v, int a) { return (v + a - 1) & ~(a - 1); }

int find_msb(uint32_t v) { return v ? 31 - __builtin_clz(v) : -1; }
int popcount(uint32_t v) { return __builtin_popcount(v); }

uint32_t f2u(float f) { uint32_t u; memcpy(&u, &f, 4); return u; }
float u2f(uint32_t u) { float f; memcpy(&f, &u, 4); return f; }

// IEEE binary16 round-to-nearest-even.
uint16_t float_to_half(float f)
{
	uint32_t x = f2u(f);
	uint32_t sign = (x >> 16) & 0x8000u;
	uint32_t a = x & 0x7fffffffu;
	if (a >= 0x7f800000u)
		return uint16_t(sign | 0x7c00u | (a > 0x7f800000u ? 0x200u : 0u));
	if (a >= 0x477ff000u) // >= 65520 rounds to infinity
		return uint16_t(sign | 0x7c00u);
	if (a < 0x38800000u) // below the smallest normal half
	{
		if (a <= 0x33000000u) // <= 2^-25 rounds to zero (the tie goes to even 0)
			return uint16_t(sign);
		uint32_t e = a >> 23;
		uint32_t mant = (a & 0x7fffffu) | 0x800000u;
		uint32_t shift = 126u - e;
		uint32_t k = mant >> shift;
		uint32_t rem = mant & ((1u << shift) - 1u);
		uint32_t half = 1u << (shift - 1u);
		if (rem > half || (rem == half && (k & 1u)))
			k++;
		return uint16_t(sign | k);
	}
	uint32_t h = ((((a >> 23) - 127u + 15u) << 10) | ((a & 0x7fffffu) >> 13));
	uint32_t rem = a & 0x1fffu;
	if (rem > 0x1000u || (rem == 0x1000u && (h & 1u)))
		h++;
	return uint16_t(sign | h);
}

float half_to_float(uint16_t h)
{
	uint32_t sign = uint32_t(h & 0x8000u) << 16;
	uint32_t e = (h >> 10) & 0x1fu;
	uint32_t m = h & 0x3ffu;
	if (e == 0)
	{
		float v = float(m) * (1.0f / 16777216.0f);
		return sign ? -v : v;
	}
	if (e == 31)
		return u2f(sign | 0x7f800000u | (m << 13));
	return u2f(sign | ((e - 15u + 127u) << 23) | (m << 13));
}

float round_half(float v) { return half_to_float(float_to_half(v)); }

// pyrowave_common.hpp:126-133 / bitstream.md:441-449. Written with ldexp so that
// quant codes outside the encoder's range stay defined: (8+m) * 2^(20+e) / 2^23.
float decode_quant(uint32_t quant_code)
{
	int e = MaxScaleExp - int(quant_code >> 3);
	int m = int(quant_code & 7u);
	return std::ldexp(float(8 + m), e - 3);
}

// pyrowave_common.hpp:135-145
uint32_t encode_quant(float decoder_q_scale)
{
	uint32_t v = f2u(decoder_q_scale);
	int e = int((v >> 23) & 0xffu) - 127 - MaxScaleExp;
	int m = int((v >> 20) & 7u);
	e = -e;
	if (e < 0)
		e = 0;
	if (e > 31)
		e = 31;
	return uint32_t((e << 3) | m) & 0xffu;
}

// dwt_quant_scale.h:6-19
float decode_quant_scale(uint32_t code) { return float(code) / 8.0f + 0.25f; }
uint32_t encode_quant_scale(float scale) { return uint32_t(std::ceil((scale - 0.25f) * 8.0f)); }

// analyze_rate_control.comp:73-83. index = 60 + 2*log2(r); return uint(max(index + 0.5, 0)).
// Evaluated exactly: with r = m * 2^e (m in [1,2)), floor(60.5 + 2e + 2*log2(m))
// = 60 + 2e + [m >= 2^0.25] + [m >= 2^0.75]. The thresholds are the smallest
// floats >= 2^0.25 (0x3f9837f1) and >= 2^0.75 (0x3fd744fd); since m is a float,
// comparing against them is the same as comparing against the irrational values.
uint32_t bucket_index(float d, float cost, float d_base, float cost_base)
{
	if (cost == cost_base)
		return 0;
	float num = std::max(d - d_base, 0.0f);
	float den = cost_base - cost;
	float r = num / den;
	if (!(r > 0.0f))
		return 0;
	uint32_t bits = f2u(r);
	uint32_t exp_field = bits >> 23;
	if (exp_field == 0)
		return 0; // subnormal: 2*log2(r) < -250
	if (exp_field >= 255)
		return 255;
	int e = int(exp_field) - 127;
	uint32_t mant = bits & 0x7fffffu;
	int idx = 60 + 2 * e + (mant >= 0x1837f1u ? 1 : 0) + (mant >= 0x5744fdu ? 1 : 0);
	return idx < 0 ? 0u : uint32_t(idx);
}

// dwt_swizzle.h:16-23 (unswizzle8x8), used as (subblock << 3).
void subblock_origin(int subblock, int &x, int &y)
{
	y = (subblock & 3) * 2;
	x = (subblock >> 2) * 4;
}

// Pixel order inside a 4x2 sub-block: bitstream.md:362-368.
void pixel_offset(int pixel, int &dx, int &dy)
{
	dx = pixel >> 1;
	dy = pixel & 1;
}

// ---------------------------------------------------------------------------
// Sampler index semantics.
//
// MIRRORED_REPEAT over [0, n): Vulkan spec address mode.
int mirrored_repeat(int i, int n)
{
	int p = 2 * n;
	int t = i % p;
	if (t < 0)
		t += p;
	return t < n ? t : p - 1 - t;
}

// dwt.comp:27-36 (generate_mirror_uv + textureGather on a mirrored-repeat
// sampler), resolved per sample: the coordinate adjustments are made on the
// even sample of each gathered pair. resolution = real texture size,
// aligned = padded size (equal above level 0).
int fwd_index(int p, int resolution, int aligned)
{
	int x = p & ~1;
	int idx;
	if (x < 0)
		idx = p - 1;
	else if (x + 1 >= 2 * aligned - resolution)
		idx = p + 1 + 2 * (resolution - aligned);
	else
		idx = std::min(p, resolution);
	return mirrored_repeat(idx, resolution);
}

// idwt.comp:25-32: low-pass (even) samples and high-pass (odd) samples of a band of size n.
int inv_index_low(int p, int n)
{
	return mirrored_repeat(p < 0 ? p - 1 : p, n);
}

int inv_index_high(int p, int n)
{
	int q = p & ~1;
	return mirrored_repeat(q + 1 >= n ? p + 1 : p, n);
}

// ---------------------------------------------------------------------------
// One-dimensional lifting on an extended array e[0 .. 2n+8) whose element j
// holds signal position j - 4. Step ranges cover every position whose
// neighbours exist; the in-range outputs equal those of dwt.comp:91-138 /
// idwt.comp:82-127 because each step uses the same operands in the same order.
template <typename T> struct Lift;

template <> struct Lift<float>
{
	static float add(float a, float b) { return a + b; }
	static void fwd(float *e, int len)
	{
		for (int j = 1; j + 1 < len; j += 2) e[j] = std::fmaf(ALPHA, e[j - 1] + e[j + 1], e[j]);
		for (int j = 2; j + 1 < len; j += 2) e[j] = std::fmaf(BETA, e[j - 1] + e[j + 1], e[j]);
		for (int j = 3; j + 1 < len; j += 2) e[j] = std::fmaf(GAMMA, e[j - 1] + e[j + 1], e[j]);
		for (int j = 4; j + 1 < len; j += 2) e[j] = std::fmaf(DELTA, e[j - 1] + e[j + 1], e[j]);
	}
	static void inv(float *e, int len)
	{
		for (int j = 2; j + 1 < len; j += 2) e[j] = std::fmaf(-DELTA, e[j - 1] + e[j + 1], e[j]);
		for (int j = 3; j + 1 < len; j += 2) e[j] = std::fmaf(-GAMMA, e[j - 1] + e[j + 1], e[j]);
		for (int j = 4; j + 1 < len; j += 2) e[j] = std::fmaf(-BETA, e[j - 1] + e[j + 1], e[j]);
		for (int j = 5; j + 1 < len; j += 2) e[j] = std::fmaf(-ALPHA, e[j - 1] + e[j + 1], e[j]);
	}
	static float low_scale() { return INV_KF; }
	static float high_scale() { return KF; }
	static float inv_low_scale() { return KF; }
	static float inv_high_scale() { return INV_KF; }
};

template <> struct Lift<double>
{
	static void fwd(double *e, int len)
	{
		for (int j = 1; j + 1 < len; j += 2) e[j] += ALPHA_D * (e[j - 1] + e[j + 1]);
		for (int j = 2; j + 1 < len; j += 2) e[j] += BETA_D * (e[j - 1] + e[j + 1]);
		for (int j = 3; j + 1 < len; j += 2) e[j] += GAMMA_D * (e[j - 1] + e[j + 1]);
		for (int j = 4; j + 1 < len; j += 2) e[j] += DELTA_D * (e[j - 1] + e[j + 1]);
	}
	static void inv(double *e, int len)
	{
		for (int j = 2; j + 1 < len; j += 2) e[j] -= DELTA_D * (e[j - 1] + e[j + 1]);
		for (int j = 3; j + 1 < len; j += 2) e[j] -= GAMMA_D * (e[j - 1] + e[j + 1]);
		for (int j = 4; j + 1 < len; j += 2) e[j] -= BETA_D * (e[j - 1] + e[j + 1]);
		for (int j = 5; j + 1 < len; j += 2) e[j] -= ALPHA_D * (e[j - 1] + e[j + 1]);
	}
	static double low_scale() { return 1.0 / K_D; }
	static double high_scale() { return K_D; }
	static double inv_low_scale() { return K_D; }
	static double inv_high_scale() { return 1.0 / K_D; }
};

constexpr int APRON = 4;

// A 2D plane of samples with the real size and the aligned size the sampler logic uses.
template <typename T> struct Plane
{
	int width = 0, height = 0; // real texture size
	std::vector<T> data;
	T at(int x, int y) const { return data[size_t(y) * size_t(width) + size_t(x)]; }
};

// One forward level (dwt.comp:195-233): H lifting on every needed row, then V
// lifting on every column. Returns LL, HL, LH, HH of size (aligned/2)^2.
// round16: reference precision-1 FP16 staging (dwt_common.h:44-47).
template <typename T>
void forward_level(const Plane<T> &src, int aligned_w, int aligned_h, bool round16, std::vector<T> out[4])
{
	int nx = aligned_w / 2, ny = aligned_h / 2;
	auto stage = [&](T v) -> T {
		if (round16)
			return T(round_half(float(v)));
		return v;
	};

	// H pass over each source row that is reachable through the row index map.
	std::vector<T> lo(size_t(src.height) * nx), hi(size_t(src.height) * nx);
	std::vector<T> e(2 * nx + 2 * APRON);
	for (int r = 0; r < src.height; r++)
	{
		for (int j = 0; j < 2 * nx + 2 * APRON; j++)
			e[j] = stage(src.at(fwd_index(j - APRON, src.width, aligned_w), r));
		Lift<T>::fwd(e.data(), int(e.size()));
		for (int k = 0; k < nx; k++)
		{
			T a = e[APRON + 2 * k] * Lift<T>::low_scale();
			T b = e[APRON + 2 * k + 1] * Lift<T>::high_scale();
			lo[size_t(r) * nx + k] = stage(a);
			hi[size_t(r) * nx + k] = stage(b);
		}
	}

	for (int b = 0; b < 4; b++)
		out[b].assign(size_t(nx) * ny, T(0));

	std::vector<T> col(2 * ny + 2 * APRON);
	for (int pass = 0; pass < 2; pass++)
	{
		const std::vector<T> &h = pass == 0 ? lo : hi;
		std::vector<T> &low_band = out[pass == 0 ? 0 : 1];  // LL or HL
		std::vector<T> &high_band = out[pass == 0 ? 2 : 3]; // LH or HH
		for (int k = 0; k < nx; k++)
		{
			for (int j = 0; j < 2 * ny + 2 * APRON; j++)
				col[j] = h[size_t(fwd_index(j - APRON, src.height, aligned_h)) * nx + k];
			Lift<T>::fwd(col.data(), int(col.size()));
			for (int y = 0; y < ny; y++)
			{
				low_band[size_t(y) * nx + k] = stage(col[APRON + 2 * y] * Lift<T>::low_scale());
				high_band[size_t(y) * nx + k] = stage(col[APRON + 2 * y + 1] * Lift<T>::high_scale());
			}
		}
	}
}

// One inverse level (idwt.comp:182-214): V lifting per band column, then H
// lifting per output row. Output has size (2*nx, 2*ny).
template <typename T>
void inverse_level(const std::vector<T> bands[4], int nx, int ny, bool round16, std::vector<T> &out)
{
	auto stage = [&](T v) -> T {
		if (round16)
			return T(round_half(float(v)));
		return v;
	};
	auto band_at = [&](int b, int x, int y) -> T { return stage(bands[b][size_t(y) * nx + x]); };

	// V pass: lowx column from LL/LH, highx column from HL/HH.
	std::vector<T> lowx(size_t(2 * ny) * nx), highx(size_t(2 * ny) * nx);
	std::vector<T> col(2 * ny + 2 * APRON);
	for (int pass = 0; pass < 2; pass++)
	{
		int b_low = pass == 0 ? 0 : 1;  // LL or HL (vertical low)
		int b_high = pass == 0 ? 2 : 3; // LH or HH (vertical high)
		std::vector<T> &dst = pass == 0 ? lowx : highx;
		for (int k = 0; k < nx; k++)
		{
			for (int j = 0; j < 2 * ny + 2 * APRON; j++)
			{
				int p = j - APRON;
				int py = p >> 1; // arithmetic shift: floor
				if ((p & 1) == 0)
					col[j] = band_at(b_low, k, inv_index_low(py, ny)) * Lift<T>::inv_low_scale();
				else
					col[j] = band_at(b_high, k, inv_index_high(py, ny)) * Lift<T>::inv_high_scale();
			}
			Lift<T>::inv(col.data(), int(col.size()));
			for (int y = 0; y < 2 * ny; y++)
				dst[size_t(y) * nx + k] = stage(col[APRON + y]);
		}
	}

	out.assign(size_t(2 * nx) * size_t(2 * ny), T(0));
	std::vector<T> row(2 * nx + 2 * APRON);
	for (int y = 0; y < 2 * ny; y++)
	{
		for (int j = 0; j < 2 * nx + 2 * APRON; j++)
		{
			int p = j - APRON;
			int px = p >> 1;
			if ((p & 1) == 0)
				row[j] = lowx[size_t(y) * nx + inv_index_low(px, nx)] * Lift<T>::inv_low_scale();
			else
				row[j] = highx[size_t(y) * nx + inv_index_high(px, nx)] * Lift<T>::inv_high_scale();
		}
		Lift<T>::inv(row.data(), int(row.size()));
		for (int x = 0; x < 2 * nx; x++)
			out[size_t(y) * 2 * nx + x] = stage(row[APRON + x]);
	}
}

// ---------------------------------------------------------------------------
// Structures of the reference encoder (pyrowave_common.hpp:93-110).
struct QuantStats
{
	uint16_t square_error_fp16;
	uint16_t encode_cost_bits;
};
// The reference's BlockStats (pyrowave_common.hpp:99-103) holds 15 entries and
// relies on num_planes <= 14. Scaled magnitudes are clamped below 2^15 here (a
// no-op for 8-bit content) and the table has 16 entries, so that every index
// min(q, num_planes) with q <= 15 stays inside it.
constexpr float MaxScaledMagnitude = 32767.0f;
struct BlockStats
{
	uint32_t num_planes;
	QuantStats errors[16];
};
static_assert(sizeof(BlockStats) == 68, "BlockStats layout");

struct BandInfo
{
	int block_offset_8x8 = -1, block_stride_8x8 = 0;
	int block_offset_32x32 = -1, block_stride_32x32 = 0;
	int64_t pyramid_offset = -1;
};

struct BlockMapping
{
	int block_offset_8x8, block_stride_8x8, block_width_8x8, block_height_8x8;
};

struct RDOperation
{
	int32_t quant;
	uint32_t block_offset_saving;
};
} // namespace

struct oracle_codec
{
	int width = 0, height = 0;
	bool chroma444 = false;
	unsigned fp16_mask = 0;
	int aligned_width = 0, aligned_height = 0;
	int block_count_8x8 = 0, block_count_32x32 = 0;
	size_t pyramid_size = 0;
	BandInfo bands[NumComponents][DecompositionLevels][4];
	std::vector<BlockMapping> mapping;

	// Encoder results.
	std::vector<uint32_t> code_words;      // BlockMeta.code_word per 8x8
	std::vector<uint32_t> payload_offset;  // BlockMeta.offset per 8x8
	std::vector<BlockStats> stats;         // per 8x8
	std::vector<uint8_t> payload;          // q=0 payload bytes
	std::vector<uint32_t> rate_cost;       // per 32x32 x 16, in words
	std::vector<float> distortion;         // per 32x32 x 16
	std::vector<uint32_t> bucket;          // per 32x32 x 16
	std::vector<uint32_t> savings_scan;    // 2048
	uint32_t consumed_payload = 0;
	std::vector<int32_t> quant;            // per 32x32
	std::vector<uint32_t> meta;            // per 32x32 x {offset_u32, num_words}
	std::vector<uint32_t> bitstream;       // words, in block index order
	uint32_t sequence = 0;

	int level_width(int level) const { return std::max(1, (aligned_width / 2) >> level); }
	int level_height(int level) const { return std::max(1, (aligned_height / 2) >> level); }
	bool has_band(int c, int level, int band) const
	{
		if (level == 0 && c != 0 && !chroma444)
			return false;
		if (band == 0 && level != DecompositionLevels - 1)
			return false;
		return true;
	}
	bool level_fp16(int level) const { return (fp16_mask >> level) & 1u; }
};

namespace
{
// pyrowave_common.cpp:212-241 (init_block_meta / accumulate_block_mapping);
// metal/pyrowave_bitstream.cpp:23-95 has the same derivation without Vulkan.
void init_layout(oracle_codec &c)
{
	c.aligned_width = std::max(align_up(c.width, Alignment), MinimumImageSize);
	c.aligned_height = std::max(align_up(c.height, Alignment), MinimumImageSize);
	c.block_count_8x8 = 0;
	c.block_count_32x32 = 0;
	c.pyramid_size = 0;
	c.mapping.clear();
	for (int level = DecompositionLevels - 1; level >= 0; level--)
	{
		for (int comp = 0; comp < NumComponents; comp++)
		{
			if (level == 0 && comp != 0 && !c.chroma444)
				continue;
			for (int band = (level == DecompositionLevels - 1 ? 0 : 1); band < 4; band++)
			{
				int w = c.level_width(level), h = c.level_height(level);
				int bx8 = (w + 7) / 8, by8 = (h + 7) / 8;
				int bx32 = (w + 31) / 32;
				BandInfo &info = c.bands[comp][level][band];
				info.block_offset_8x8 = c.block_count_8x8;
				info.block_stride_8x8 = bx8;
				info.block_offset_32x32 = c.block_count_32x32;
				info.block_stride_32x32 = bx32;
				info.pyramid_offset = int64_t(c.pyramid_size);
				c.pyramid_size += size_t(w) * size_t(h);

				int bx32b = (bx8 + 3) / 4, by32b = (by8 + 3) / 4;
				for (int y = 0; y < by32b; y++)
					for (int x = 0; x < bx32b; x++)
					{
						BlockMapping m;
						m.block_offset_8x8 = c.block_count_8x8 + 4 * y * bx8 + 4 * x;
						m.block_stride_8x8 = bx8;
						m.block_width_8x8 = std::min(4, bx8 - 4 * x);
						m.block_height_8x8 = std::min(4, by8 - 4 * y);
						c.mapping.push_back(m);
						c.block_count_32x32++;
					}
				c.block_count_8x8 += bx8 * by8;
			}
		}
	}
}

// pyrowave_encoder.cpp:152-172
float noise_power_normalized_quant_resolution(int level, int component, int band)
{
	int bits = 8; // precision >= 1
	if (band == 0)
		bits += 2;
	else if (band < 3)
		bits += 1;
	bits += level;
	if (component != 0)
		bits--;
	return float(1 << bits);
}

// pyrowave_encoder.cpp:144-150
float quant_resolution(int level, int component, int band)
{
	return std::min<float>(4096.0f, noise_power_normalized_quant_resolution(level, component, band));
}

// pyrowave_encoder.cpp:107-142
float rdo_distortion_scale(const oracle_codec &c, int level, int component, int band)
{
	float horiz_midpoint = (band & 1) ? 0.75f : 0.25f;
	float vert_midpoint = (band & 2) ? 0.75f : 0.25f;
	constexpr float dpi = 96.0f;
	constexpr float viewing_distance = 1.0f;
	constexpr float cpd_nyquist = 0.34f * viewing_distance * dpi;
	float cpd = std::sqrt(horiz_midpoint * horiz_midpoint + vert_midpoint * vert_midpoint) *
	            cpd_nyquist * std::exp2(-float(level));
	cpd = std::max(cpd, 8.0f);
	float csf = 2.6f * (0.0192f + 0.114f * cpd) * std::exp(-std::pow(0.114f * cpd, 1.1f));
	if (component != 0 && level != DecompositionLevels - 1)
	{
		if (!c.chroma444)
			csf *= 0.6f;
	}
	float resolution = noise_power_normalized_quant_resolution(level, component, band);
	float weighted_resolution = csf * resolution;
	return weighted_resolution * weighted_resolution;
}

// ---------------------------------------------------------------------------
// wavelet_quant.comp
struct SubblockResult
{
	float square_error;
	int encode_cost_early;
	int block4x2_shifted;
	int quality_planes;
};

// Clustered (8-lane) xor-butterfly float sum in lane order.
float butterfly8(const float v[8])
{
	float a0 = v[0] + v[1], a1 = v[2] + v[3], a2 = v[4] + v[5], a3 = v[6] + v[7];
	float b0 = a0 + a1, b1 = a2 + a3;
	return b0 + b1;
}

float butterfly16(const float v[16])
{
	float a[8], b[4], c[2];
	for (int i = 0; i < 8; i++)
		a[i] = v[2 * i] + v[2 * i + 1];
	for (int i = 0; i < 4; i++)
		b[i] = a[2 * i] + a[2 * i + 1];
	for (int i = 0; i < 2; i++)
		c[i] = b[2 * i] + b[2 * i + 1];
	return c[0] + c[1];
}

float dot4(const float *e)
{
	float s = e[0] * e[0];
	s = std::fmaf(e[1], e[1], s);
	s = std::fmaf(e[2], e[2], s);
	s = std::fmaf(e[3], e[3], s);
	return s;
}

// wavelet_quant.comp:113-128 (per lane part; the clustered count is done by the caller).
float compute_square_error(const float v_in[8], int q, float rdo_scale, int &num_significant)
{
	float err[8];
	num_significant = 0;
	for (int i = 0; i < 8; i++)
	{
		float v = std::fabs(v_in[i]);
		float iv = std::floor(std::ldexp(v, -q)); // floor and trunc agree for v >= 0
		if (iv != 0.0f)
			num_significant++;
		if (iv != 0.0f)
			iv += 0.5f;
		iv = std::trunc(std::ldexp(iv, q));
		err[i] = v - iv;
	}
	float d = dot4(err) + dot4(err + 4);
	return d * rdo_scale;
}

// wavelet_quant.comp:139-165 (per lane part).
SubblockResult compute_quant_stats(const float v[8], int q, int msb, int block4x2_max, float inv_quant_squared,
                                   float rdo_scale, int &num_significant)
{
	block4x2_max >>= q;
	SubblockResult r;
	r.square_error = compute_square_error(v, q, rdo_scale, num_significant) * inv_quant_squared;
	r.block4x2_shifted = block4x2_max;
	r.encode_cost_early = block4x2_max > 0 ? 1 : 0;
	msb -= q;
	r.quality_planes = 0;
	if (msb >= 3)
	{
		r.quality_planes = msb - 2;
		r.encode_cost_early = r.quality_planes + 1;
		r.block4x2_shifted >>= r.quality_planes;
	}
	r.encode_cost_early += find_msb(uint32_t(r.block4x2_shifted)) + 1;
	return r;
}

// wavelet_quant.comp:95-111
void compute_quant_scale(float max_wave_texels, uint32_t &quant_code, float &quant_scale)
{
	if (max_wave_texels < 1.0f)
	{
		quant_code = ENCODE_QUANT_IDENTITY;
		quant_scale = 1.0f;
	}
	else
	{
		int e;
		std::frexp(max_wave_texels - 0.25f, &e);
		float target_max = float(1 << e) - 0.25f;
		float inv_scale = max_wave_texels / target_max;
		quant_code = encode_quant_scale(inv_scale);
		quant_scale = 1.0f / decode_quant_scale(quant_code);
	}
}

// wavelet_quant.comp:172-290 for one 8x8 block. texels[s][i]: sub-block s, pixel i,
// already multiplied by quant_resolution (wavelet_quant.comp:311-312).
void encode_payload_8x8(oracle_codec &c, uint32_t block_index, float texels[8][8], float rdo_scale,
                        float quant_resolution_value)
{
	float max_sub[8];
	float max_wave = 0.0f;
	for (int s = 0; s < 8; s++)
	{
		float m = 0.0f;
		for (int i = 0; i < 8; i++)
			m = std::max(m, std::fabs(texels[s][i]));
		max_sub[s] = m;
		max_wave = std::max(max_wave, m);
	}

	uint32_t quant_code;
	float quant_scale;
	compute_quant_scale(max_wave, quant_code, quant_scale);
	for (int s = 0; s < 8; s++)
	{
		for (int i = 0; i < 8; i++)
		{
			float t = texels[s][i] * quant_scale;
			texels[s][i] = std::min(std::max(t, -MaxScaledMagnitude), MaxScaledMagnitude);
		}
		max_sub[s] = std::min(max_sub[s] * quant_scale, MaxScaledMagnitude);
	}
	max_wave = std::min(max_wave * quant_scale, MaxScaledMagnitude);

	float overall_quant_scale = quant_resolution_value * quant_scale;
	float inv_quant = 1.0f / overall_quant_scale;
	float inv_quant_squared = inv_quant * inv_quant;

	int abs_q[8][8];
	int block4x2_max[8];
	for (int s = 0; s < 8; s++)
	{
		for (int i = 0; i < 8; i++)
			abs_q[s][i] = std::abs(int(texels[s][i]));
		block4x2_max[s] = int(max_sub[s]);
	}
	int max_absolute_value = int(max_wave);

	BlockStats &st = c.stats[block_index];
	if (max_absolute_value == 0)
	{
		c.code_words[block_index] = 0;
		c.payload_offset[block_index] = 0;
		st.num_planes = 0;
		st.errors[0] = {0, 0};
		return;
	}

	int msb = find_msb(uint32_t(max_absolute_value));

	SubblockResult r0[8];
	int nsig0 = 0;
	for (int s = 0; s < 8; s++)
	{
		int ns;
		r0[s] = compute_quant_stats(texels[s], 0, msb, block4x2_max[s], inv_quant_squared, rdo_scale, ns);
		nsig0 += ns;
	}
	int cost_sum0 = 0;
	for (int s = 0; s < 8; s++)
		cost_sum0 += std::max(r0[s].encode_cost_early - 1, 0);
	uint32_t cost_late0 = uint32_t(8 * cost_sum0 + nsig0);

	int quality_planes = r0[0].quality_planes; // identical on all lanes
	uint32_t code_word = uint32_t(quality_planes) << Q_PLANES_OFFSET;
	code_word = (code_word & ~(0xfu << QUANT_SCALE_OFFSET)) | ((quant_code & 0xfu) << QUANT_SCALE_OFFSET);
	uint32_t plane_codes[8];
	for (int s = 0; s < 8; s++)
	{
		plane_codes[s] = uint32_t(find_msb(uint32_t(r0[s].block4x2_shifted)) + 1);
		code_word |= plane_codes[s] << (2 * s);
	}

	// Payload allocation: deterministic (8x8 index order) instead of the atomic at
	// wavelet_quant.comp:213-215; the layout of this scratch buffer does not reach the bitstream.
	uint32_t global_offset = uint32_t(c.payload.size());
	c.code_words[block_index] = code_word;
	c.payload_offset[block_index] = global_offset;
	st.num_planes = uint32_t(msb + 1);
	st.errors[0] = {0, uint16_t(cost_late0)};

	for (int q = 1; q <= msb; q++)
	{
		float se[8];
		int nsig = 0, cost_sum = 0;
		for (int s = 0; s < 8; s++)
		{
			int ns;
			SubblockResult r = compute_quant_stats(texels[s], q, msb, block4x2_max[s], inv_quant_squared, rdo_scale, ns);
			se[s] = r.square_error;
			nsig += ns;
			cost_sum += std::max(r.encode_cost_early - 1, 0);
		}
		float square_error = butterfly8(se);
		st.errors[q] = {float_to_half(std::min(square_error, 60000.0f)), uint16_t(8 * cost_sum + nsig)};
	}

	float total[8];
	for (int s = 0; s < 8; s++)
	{
		float d = dot4(texels[s]) + dot4(texels[s] + 4);
		total[s] = d * inv_quant_squared;
	}
	float square_error = butterfly8(total);
	st.errors[msb + 1] = {float_to_half(std::min(60000.0f, square_error)), 0};

	// Sign byte + magnitude planes per sub-block (wavelet_quant.comp:258-289).
	for (int s = 0; s < 8; s++)
	{
		bool need_sign = r0[s].block4x2_shifted != 0 || quality_planes != 0;
		if (!need_sign)
			continue;
		uint32_t sgn = 0;
		for (int i = 0; i < 8; i++)
			if (texels[s][i] < 0.0f)
				sgn |= 1u << i;
		c.payload.push_back(uint8_t(sgn));
		int plane_iterations = quality_planes + int(plane_codes[s]);
		for (int q = plane_iterations - 1; q >= 0; q--)
		{
			uint32_t b = 0;
			for (int i = 0; i < 8; i++)
				b |= uint32_t((abs_q[s][i] >> q) & 1) << i;
			c.payload.push_back(uint8_t(b));
		}
	}
}

// wavelet_quant.comp:292-316 over one band. The band is read with border
// (zero) addressing outside its extent (pyrowave_common.cpp:273-277).
void quant_band(oracle_codec &c, const float *band, int w, int h, const BandInfo &info, float quant_res, float rdo_scale)
{
	int bx8 = (w + 7) / 8, by8 = (h + 7) / 8;
	for (int by = 0; by < by8; by++)
		for (int bx = 0; bx < bx8; bx++)
		{
			float texels[8][8];
			for (int s = 0; s < 8; s++)
			{
				int sx, sy;
				subblock_origin(s, sx, sy);
				for (int i = 0; i < 8; i++)
				{
					int dx, dy;
					pixel_offset(i, dx, dy);
					int x = bx * 8 + sx + dx, y = by * 8 + sy + dy;
					float v = (x < w && y < h) ? band[size_t(y) * w + x] : 0.0f;
					texels[s][i] = v * quant_res;
				}
			}
			uint32_t block_index = uint32_t(info.block_offset_8x8 + by * info.block_stride_8x8 + bx);
			encode_payload_8x8(c, block_index, texels, rdo_scale, quant_res);
		}
}

// analyze_rate_control.comp:85-99
void inclusive_max_clustered16(uint32_t v[16])
{
	for (int l = 0; l < 16; l++)
		v[l] = std::min(v[l], uint32_t(128 - 16 + l));
	for (int i = 1; i < 16; i *= 2)
	{
		uint32_t nv[16];
		for (int l = 0; l < 16; l++)
		{
			uint32_t up = l >= i ? v[l - i] + uint32_t(i) : 0u;
			nv[l] = std::max(v[l], up);
		}
		memcpy(v, nv, sizeof(nv));
	}
}

int block_count_per_subdivision(int num_blocks)
{
	int per = align_up(num_blocks, BlockSpaceSubdivision) / BlockSpaceSubdivision;
	int pot = 1;
	while (pot < per)
		pot *= 2;
	return pot;
}

// analyze_rate_control.comp:101-220 for every 32x32 block of one band.
void analyze_band(oracle_codec &c, int w, int h, const BandInfo &info, std::vector<RDOperation> &ops,
                  std::vector<uint32_t> &total_savings, uint32_t num_blocks_aligned, uint32_t shamt)
{
	int bx8 = (w + 7) / 8, by8 = (h + 7) / 8;
	int bx32 = (w + 31) / 32, by32 = (h + 31) / 32;
	for (int by = 0; by < by32; by++)
		for (int bx = 0; bx < bx32; bx++)
		{
			uint32_t block_index = uint32_t(info.block_offset_32x32 + by * info.block_stride_32x32 + bx);
			uint32_t rate_cost[16];
			float dist[16];
			for (int i = 0; i < 16; i++)
			{
				float d[16];
				uint32_t cost_total = 0;
				for (int lane = 0; lane < 16; lane++)
				{
					int lx = lane & 3, ly = lane >> 2;
					int x8 = 4 * bx + lx, y8 = 4 * by + ly;
					float dd = 0.0f;
					uint32_t cost = 0;
					if (x8 < bx8 && y8 < by8)
					{
						const BlockStats &st = c.stats[size_t(info.block_offset_8x8 + info.block_stride_8x8 * y8 + x8)];
						const QuantStats &qs = st.errors[std::min<uint32_t>(uint32_t(i), st.num_planes)];
						dd = half_to_float(qs.square_error_fp16);
						cost = qs.encode_cost_bits;
					}
					if (cost != 0)
						cost += 24;
					d[lane] = dd;
					cost_total += cost;
				}
				if (cost_total != 0)
					cost_total += 64;
				rate_cost[i] = (cost_total + 31) >> 5;
				dist[i] = butterfly16(d);
			}

			uint32_t b[16];
			for (int l = 0; l < 16; l++)
				b[l] = bucket_index(dist[l], float(rate_cost[l]), dist[0], float(rate_cost[0]));
			b[0] = 0;
			inclusive_max_clustered16(b);

			for (int l = 0; l < 16; l++)
			{
				c.rate_cost[size_t(block_index) * 16 + l] = rate_cost[l];
				c.distortion[size_t(block_index) * 16 + l] = dist[l];
				c.bucket[size_t(block_index) * 16 + l] = b[l];
			}

			c.consumed_payload += rate_cost[0];
			for (int l = 1; l < 16; l++)
			{
				uint32_t saving = rate_cost[l - 1] - rate_cost[l];
				if (saving != 0)
				{
					uint32_t subdivision = block_index >> shamt;
					total_savings[b[l] * BlockSpaceSubdivision + subdivision] += saving;
					ops[block_index + b[l] * num_blocks_aligned] = {int32_t(l), block_index | (saving << 16)};
				}
			}
		}
}

// block_packing.comp:97-105
uint32_t compute_required_8x8_size(uint32_t control_word)
{
	int q_bits = int((control_word >> Q_PLANES_OFFSET) & 0xfu);
	uint32_t lsbs = control_word & 0x5555u;
	uint32_t msbs = control_word & 0xaaaau;
	msbs |= msbs >> 1;
	return uint32_t(popcount(lsbs) + popcount(msbs) + q_bits * 8);
}

// block_packing.comp:107-142
uint32_t quantize_code_word(uint32_t control_word, int quant)
{
	if (quant != 0 && control_word != 0)
	{
		int q_bits = int((control_word >> Q_PLANES_OFFSET) & 0xfu);
		int sub_quant = std::min(q_bits, quant);
		q_bits -= sub_quant;
		quant -= sub_quant;
		if (quant != 0)
		{
			quant = std::min(quant, 3);
			uint32_t plane0 = control_word & 0x5555u;
			uint32_t plane1 = (control_word & 0xaaaau) >> 1;
			uint32_t plane2 = plane0 & plane1;
			do
			{
				plane0 = plane1;
				plane1 = plane2;
				plane2 = 0;
				quant--;
			} while (quant != 0);
			plane0 &= ~plane1;
			uint32_t new_control_word = plane0 | (plane1 << 1);
			control_word = (control_word & ~0xffffu) | (new_control_word & 0xffffu);
		}
		control_word = (control_word & ~(0xfu << Q_PLANES_OFFSET)) | (uint32_t(q_bits) << Q_PLANES_OFFSET);
	}
	return control_word;
}

// block_packing.comp:161-167
uint32_t modify_quant_code(uint32_t code, int quant)
{
	int e = int((code >> 3) & 31u);
	e = std::max(e - quant, 0);
	return (code & ~(31u << 3)) | (uint32_t(e) << 3);
}

// block_packing.comp:224-379 for one 32x32 block; words appended to c.bitstream
// in block index order (the reference allocates with an atomic, which only
// changes where the block sits before packetize reorders by block index).
void pack_block(oracle_codec &c, int bx, int by, int w, int h, const BandInfo &info, uint32_t quant_res_code)
{
	int bx8 = (w + 7) / 8, by8 = (h + 7) / 8;
	uint32_t block_index = uint32_t(info.block_offset_32x32 + by * info.block_stride_32x32 + bx);
	int quant = c.quant[block_index];

	uint32_t code_word[16], in_code[16], in_offset[16], num_bits[16];
	bool active[16];
	uint32_t ballot = 0;
	for (int lane = 0; lane < 16; lane++)
	{
		int x8 = 4 * bx + (lane & 3), y8 = 4 * by + (lane >> 2);
		uint32_t cw = 0, off = 0, nb = 0;
		if (x8 < bx8 && y8 < by8)
		{
			uint32_t bi = uint32_t(info.block_offset_8x8 + info.block_stride_8x8 * y8 + x8);
			cw = c.code_words[bi];
			off = c.payload_offset[bi];
			const BlockStats &st = c.stats[bi];
			nb = st.errors[std::min<uint32_t>(st.num_planes, uint32_t(quant))].encode_cost_bits;
		}
		in_code[lane] = cw;
		in_offset[lane] = off;
		num_bits[lane] = nb;
		code_word[lane] = quantize_code_word(cw, quant);
		active[lane] = (code_word[lane] & 0xffffu) != 0;
		if (active[lane])
			ballot |= 1u << lane;
	}

	uint32_t total_bits = 0, plane_bytes_total = 0, sign_bits_total = 0;
	uint32_t plane_bytes[16], sign_bits[16];
	for (int lane = 0; lane < 16; lane++)
	{
		plane_bytes[lane] = compute_required_8x8_size(code_word[lane]);
		sign_bits[lane] = num_bits[lane] - plane_bytes[lane] * 8;
		uint32_t with_meta = num_bits[lane];
		if (with_meta != 0)
			with_meta += 24;
		total_bits += with_meta;
		plane_bytes_total += plane_bytes[lane];
		sign_bits_total += sign_bits[lane];
	}
	uint32_t words = (total_bits + 31) / 32;
	if (words != 0)
		words += 2;

	uint32_t offset = uint32_t(c.bitstream.size());
	c.meta[size_t(block_index) * 2 + 0] = offset;
	c.meta[size_t(block_index) * 2 + 1] = words;
	if (words == 0)
		return;

	std::vector<uint8_t> bytes(size_t(words) * 4, 0);
	uint32_t w0 = (ballot & 0xffffu) | (words << 16) | ((c.sequence & 7u) << 28);
	uint32_t w1 = modify_quant_code(quant_res_code, quant) | (block_index << 8);
	memcpy(&bytes[0], &w0, 4);
	memcpy(&bytes[4], &w1, 4);

	uint32_t n = uint32_t(popcount(ballot));
	uint32_t planes_base = 8 + 3 * n;
	uint32_t sign_base = planes_base + plane_bytes_total;
	uint32_t plane_cursor = planes_base;
	uint32_t sign_cursor = 0;
	uint32_t compact = 0;
	for (int lane = 0; lane < 16; lane++)
	{
		if (!active[lane])
			continue;
		uint16_t cw16 = uint16_t(code_word[lane]);
		memcpy(&bytes[8 + 2 * compact], &cw16, 2);
		bytes[8 + 2 * n + compact] = uint8_t(code_word[lane] >> 16);
		compact++;

		uint32_t in_q_bits = (in_code[lane] >> Q_PLANES_OFFSET) & 0xfu;
		uint32_t out_q_bits = (code_word[lane] >> Q_PLANES_OFFSET) & 0xfu;
		uint32_t input_offset = in_offset[lane];
		for (int bit_offset = 0; bit_offset < 16; bit_offset += 2)
		{
			uint32_t out_planes = ((code_word[lane] >> bit_offset) & 3u) + out_q_bits;
			uint32_t in_planes = ((in_code[lane] >> bit_offset) & 3u) + in_q_bits;
			if (in_planes != 0)
				in_planes++;
			if (out_planes != 0)
			{
				uint32_t sign_plane = c.payload[input_offset];
				uint32_t significant = 0;
				for (uint32_t p = 0; p < out_planes; p++)
				{
					uint8_t b = c.payload[input_offset + 1 + p];
					significant |= b;
					bytes[plane_cursor++] = b;
				}
				for (int bit = 0; bit < 8; bit++)
				{
					if (significant & (1u << bit))
					{
						if ((sign_plane >> bit) & 1u)
							bytes[sign_base + (sign_cursor >> 3)] |= uint8_t(1u << (sign_cursor & 7u));
						sign_cursor++;
					}
				}
			}
			input_offset += in_planes;
		}
	}
	(void)sign_bits_total;

	size_t base = c.bitstream.size();
	c.bitstream.resize(base + words);
	memcpy(&c.bitstream[base], bytes.data(), bytes.size());
}

// ---------------------------------------------------------------------------
// wavelet_dequant.comp:100-160,168-175,220-391 (STORAGE_MODE 0) for one 32x32 block.
void dequant_block(const oracle_codec &c, const uint32_t *offsets, const uint32_t *payload, size_t payload_words,
                   uint32_t block_index, float *band, int w, int h, int bx, int by, int storage_mode16)
{
	auto store = [&](int x, int y, float v) {
		if (x < w && y < h)
			band[size_t(y) * w + x] = storage_mode16 ? round_half(v) : v;
	};
	uint32_t offset_u32 = offsets[block_index];
	if (offset_u32 == ~0u)
	{
		for (int y = 0; y < 32; y++)
			for (int x = 0; x < 32; x++)
				store(bx * 32 + x, by * 32 + y, 0.0f);
		return;
	}
	const uint8_t *p8 = reinterpret_cast<const uint8_t *>(payload);
	size_t payload_bytes = payload_words * 4;
	auto rd8 = [&](size_t i) -> uint32_t { return i < payload_bytes ? p8[i] : 0u; };
	auto rd16 = [&](size_t i) -> uint32_t { return rd8(2 * i) | (rd8(2 * i + 1) << 8); };
	auto rd32 = [&](size_t i) -> uint32_t { return i < payload_words ? payload[i] : 0u; };

	uint32_t ballot = rd32(offset_u32) & 0xffffu;
	uint32_t q_code = rd32(size_t(offset_u32) + 1) & 0xffu;
	uint32_t nballot = uint32_t(popcount(ballot));

	uint32_t plane_offsets[16];
	uint32_t byte_scan = uint32_t(offset_u32) * 4 + 8 + 3 * nballot;
	for (int l = 0; l < 16; l++)
	{
		uint32_t cw = 0, q_bits = 0;
		if ((ballot >> l) & 1u)
		{
			uint32_t local = uint32_t(popcount(ballot & ((1u << l) - 1u)));
			cw = rd16(size_t(offset_u32) * 2 + 4 + local);
			q_bits = rd8(size_t(offset_u32) * 4 + 8 + nballot * 2 + local) & 0xfu;
		}
		uint32_t lsbs = cw & 0x5555u, msbs = cw & 0xaaaau;
		msbs |= msbs >> 1;
		uint32_t cost = uint32_t(popcount(lsbs) + popcount(msbs)) + q_bits * 8;
		plane_offsets[l] = byte_scan;
		byte_scan += cost;
	}
	uint32_t sign_bit = 8 * byte_scan;

	float q = decode_quant(q_code);
	for (int l = 0; l < 16; l++)
	{
		int lx = l & 3, ly = l >> 2;
		for (int s = 0; s < 8; s++)
		{
			int sx, sy;
			subblock_origin(s, sx, sy);
			float v[8] = {};
			if ((ballot >> l) & 1u)
			{
				uint32_t local = uint32_t(popcount(ballot & ((1u << l) - 1u)));
				uint32_t cw = rd16(size_t(offset_u32) * 2 + 4 + local);
				uint32_t cw2 = rd8(size_t(offset_u32) * 4 + 8 + nballot * 2 + local);
				uint32_t q_bits = cw2 & 0xfu;
				if (cw != 0)
				{
					int bit_offset = 2 * s;
					uint32_t lsbs = cw & 0x5555u, msbs = cw & 0xaaaau;
					msbs |= msbs >> 1;
					uint32_t mask = bit_offset ? ((1u << bit_offset) - 1u) : 0u;
					uint32_t byte_offset = uint32_t(popcount(lsbs & mask) + popcount(msbs & mask)) +
					                       q_bits * uint32_t(s) + plane_offsets[l];
					uint32_t local_cw = (cw >> bit_offset) & 3u;
					int plane_iterations = int(q_bits + local_cw);
					int dec[8] = {};
					for (int pq = plane_iterations - 1; pq >= 0; pq--)
					{
						uint32_t pl = rd8(byte_offset++);
						for (int b = 0; b < 8; b++)
							dec[b] |= int((pl >> b) & 1u) << pq;
					}
					for (int b = 0; b < 8; b++)
					{
						float f = float(dec[b]);
						if (f != 0.0f)
							f += 0.5f;
						v[b] = f;
					}
				}
				float inv_scale = q * decode_quant_scale((cw2 >> (QUANT_SCALE_OFFSET - 16)) & 0xfu);
				for (int b = 0; b < 8; b++)
					v[b] = v[b] * inv_scale;
			}
			// Signs in pixel order at the running significant position.
			for (int b = 0; b < 8; b++)
			{
				if (v[b] != 0.0f)
				{
					uint32_t word = rd32(sign_bit / 32);
					uint32_t bit = (word >> (sign_bit & 31u)) & 1u;
					v[b] = v[b] * (1.0f - 2.0f * float(bit));
					sign_bit++;
				}
			}
			for (int b = 0; b < 8; b++)
			{
				int dx, dy;
				pixel_offset(b, dx, dy);
				store(bx * 32 + lx * 8 + sx + dx, by * 32 + ly * 8 + sy + dy, v[b]);
			}
		}
	}
}

// UNORM texel of an 8-bit (R8_UNORM) or 16-bit (R16_UNORM, encode.cpp:152) plane.
template <typename S> constexpr float unorm_max() { return sizeof(S) == 1 ? 255.0f : 65535.0f; }

// The DWT input: UNORM value minus the DC shift of 0.5 (dwt.comp:48,66,75,85).
// `stride` is in samples.
template <typename T, typename S>
void load_plane(Plane<T> &p, const S *data, int stride, int w, int h, bool round16)
{
	p.width = w;
	p.height = h;
	p.data.resize(size_t(w) * h);
	for (int y = 0; y < h; y++)
		for (int x = 0; x < w; x++)
		{
			T v;
			if (std::is_same<T, double>::value)
				v = T(double(data[size_t(y) * stride + x]) / double(unorm_max<S>()) - 0.5);
			else
			{
				float f = float(data[size_t(y) * stride + x]) / unorm_max<S>();
				f = f - 0.5f;
				v = T(f);
			}
			p.data[size_t(y) * w + x] = round16 ? T(round_half(float(v))) : v;
		}
}

template <typename T> T store_round(const oracle_codec &c, int level, T v, int mode)
{
	if (std::is_same<T, double>::value)
		return v;
	if (mode == ORACLE_MODE_F32 && c.level_fp16(level))
		return T(round_half(float(v)));
	return v;
}

template <typename T, typename S = uint8_t>
int run_dwt(oracle_codec &c, const S *const planes[3], const int strides[3], int mode, T *out)
{
	bool round16 = mode == ORACLE_MODE_REF16;
	for (int comp = 0; comp < NumComponents; comp++)
	{
		Plane<T> input;
		int start_level = (comp != 0 && !c.chroma444) ? 1 : 0;
		int pw = c.width, ph = c.height;
		if (start_level == 1)
		{
			pw /= 2;
			ph /= 2;
		}
		// The input plane keeps its real size; the sampler logic pads it to the
		// aligned size (pyrowave_encoder.cpp:509-581).
		load_plane(input, planes[comp], strides[comp], pw, ph, round16);
		int aw = c.aligned_width >> start_level, ah = c.aligned_height >> start_level;
		for (int level = start_level; level < DecompositionLevels; level++)
		{
			std::vector<T> bands[4];
			forward_level(input, aw, ah, round16, bands);
			int nx = aw / 2, ny = ah / 2;
			for (int b = 0; b < 4; b++)
				for (auto &v : bands[b])
					v = store_round(c, level, v, mode);
			for (int b = 0; b < 4; b++)
			{
				const BandInfo &info = c.bands[comp][level][b];
				if (!c.has_band(comp, level, b))
					continue;
				memcpy(out + info.pyramid_offset, bands[b].data(), sizeof(T) * bands[b].size());
			}
			input.width = nx;
			input.height = ny;
			input.data = std::move(bands[0]);
			aw = nx;
			ah = ny;
		}
	}
	return 0;
}

// The final store adds the DC shift back and converts to UNORM with the
// store's clamp (idwt.comp:208-211); `strides` in samples.
template <typename T, typename S = uint8_t>
int run_idwt(oracle_codec &c, const T *pyramid, int mode, S *const planes[3], const int strides[3])
{
	bool round16 = mode == ORACLE_MODE_REF16;
	for (int comp = 0; comp < NumComponents; comp++)
	{
		int end_level = (comp != 0 && !c.chroma444) ? 1 : 0;
		int pw = c.width, ph = c.height;
		if (end_level == 1)
		{
			pw /= 2;
			ph /= 2;
		}
		std::vector<T> ll;
		{
			const BandInfo &info = c.bands[comp][DecompositionLevels - 1][0];
			size_t n = size_t(c.level_width(DecompositionLevels - 1)) * c.level_height(DecompositionLevels - 1);
			ll.assign(pyramid + info.pyramid_offset, pyramid + info.pyramid_offset + n);
		}
		for (int level = DecompositionLevels - 1; level >= end_level; level--)
		{
			int nx = c.level_width(level), ny = c.level_height(level);
			std::vector<T> bands[4];
			bands[0] = ll;
			for (int b = 1; b < 4; b++)
			{
				const BandInfo &info = c.bands[comp][level][b];
				bands[b].assign(pyramid + info.pyramid_offset, pyramid + info.pyramid_offset + size_t(nx) * ny);
			}
			std::vector<T> out;
			inverse_level(bands, nx, ny, round16, out);
			if (level == end_level)
			{
				int ow = 2 * nx;
				for (int y = 0; y < ph; y++)
					for (int x = 0; x < pw; x++)
					{
						T v = out[size_t(y) * ow + x];
						S u;
						if (std::is_same<T, double>::value)
						{
							double f = double(v) + 0.5;
							f = std::min(std::max(f, 0.0), 1.0);
							u = S(int(f * double(unorm_max<S>()) + 0.5));
						}
						else
						{
							float f = float(v) + 0.5f;
							f = std::min(std::max(f, 0.0f), 1.0f);
							u = S(int(f * unorm_max<S>() + 0.5f));
						}
						planes[comp][size_t(y) * strides[comp] + x] = u;
					}
			}
			else
			{
				for (auto &v : out)
					v = store_round(c, level - 1, v, mode);
				ll = std::move(out);
			}
		}
	}
	return 0;
}
} // namespace

// ---------------------------------------------------------------------------
// Packet parser: pyrowave_decoder.cpp:126-262 (push_packet / decode_packet),
// :780-794 (decode_is_ready), :832-840 (clear).
struct oracle_parser
{
	const oracle_codec *codec = nullptr;
	std::vector<uint32_t> offsets;
	std::vector<uint32_t> payload;
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
		total_blocks_in_sequence = codec->block_count_32x32;
		payload.clear();
	}

	bool decode_packet(const uint8_t *data, uint32_t block_index, uint32_t payload_words)
	{
		uint32_t &offset = offsets[block_index];
		if (offset == UINT32_MAX)
		{
			decoded_blocks++;
			offset = uint32_t(payload.size());
		}
		else
			return true;
		if (2 > payload_words)
			return false;
		size_t base = payload.size();
		payload.resize(base + payload_words);
		memcpy(&payload[base], data, size_t(payload_words) * 4);
		return true;
	}

	bool push_packet(const uint8_t *data, size_t size)
	{
		while (size >= 8)
		{
			uint32_t w0, w1;
			memcpy(&w0, data, 4);
			memcpy(&w1, data + 4, 4);
			uint32_t header_sequence = (w0 >> 28) & 7u;
			uint32_t extended = (w0 >> 31) & 1u;
			if (extended)
			{
				uint32_t width_minus_1 = w0 & 0x3fffu;
				uint32_t height_minus_1 = (w0 >> 14) & 0x3fffu;
				uint32_t total_blocks = w1 & 0xffffffu;
				uint32_t code = (w1 >> 24) & 3u;
				uint32_t chroma_resolution = (w1 >> 26) & 1u;
				if (chroma_resolution != (codec->chroma444 ? 1u : 0u))
					return false;
				// BitstreamHeader::sequence (bits 28-30 of word 0) is read through the
				// plain header view, as the reference does (pyrowave_decoder.cpp:177).
				uint8_t diff = uint8_t((header_sequence - last_seq) & 7u);
				if (last_seq != UINT32_MAX && diff > 3)
					return true;
				if (last_seq == UINT32_MAX || diff != 0)
				{
					clear();
					last_seq = header_sequence;
				}
				if (code == 0)
				{
					if (int(width_minus_1 + 1) != codec->width || int(height_minus_1 + 1) != codec->height)
						return false;
					total_blocks_in_sequence = int(total_blocks);
				}
				else
					return false;
				data += 8;
				size -= 8;
				continue;
			}

			uint32_t payload_words = (w0 >> 16) & 0xfffu;
			size_t packet_size = size_t(payload_words) * 4;
			if (packet_size > size)
				return false;

			bool restart;
			if (last_seq == UINT32_MAX)
				restart = true;
			else
			{
				uint8_t diff = uint8_t((header_sequence - last_seq) & 7u);
				if (diff > 3)
					return true;
				restart = diff != 0;
			}
			if (restart)
			{
				clear();
				last_seq = header_sequence;
			}
			uint32_t block_index = (w1 >> 8) & 0xffffffu;
			if (block_index >= uint32_t(codec->block_count_32x32))
				return false;
			if (!decode_packet(data, block_index, payload_words))
				return false;
			data += packet_size;
			size -= packet_size;
		}
		return size == 0;
	}

	bool decode_is_ready(bool allow_partial_frame) const
	{
		if (decoded_frame_for_current_sequence)
			return false;
		if (last_seq == UINT32_MAX)
			return false;
		if (decoded_blocks < total_blocks_in_sequence)
			if (!allow_partial_frame || decoded_blocks <= total_blocks_in_sequence / 2)
				return false;
		return true;
	}
};

extern "C" {

oracle_codec *oracle_create(int width, int height, int chroma444, unsigned fp16_level_mask)
{
	if (width <= 0 || height <= 0 || width > 16384 || height > 16384)
		return nullptr;
	if (!chroma444 && ((width & 1) || (height & 1)))
		return nullptr;
	auto *c = new oracle_codec;
	c->width = width;
	c->height = height;
	c->chroma444 = chroma444 != 0;
	c->fp16_mask = fp16_level_mask;
	init_layout(*c);
	return c;
}

void oracle_destroy(oracle_codec *codec) { delete codec; }
int oracle_aligned_width(const oracle_codec *c) { return c->aligned_width; }
int oracle_aligned_height(const oracle_codec *c) { return c->aligned_height; }
int oracle_block_count_8x8(const oracle_codec *c) { return c->block_count_8x8; }
int oracle_block_count_32x32(const oracle_codec *c) { return c->block_count_32x32; }
size_t oracle_pyramid_size(const oracle_codec *c) { return c->pyramid_size; }

void oracle_block_info(const oracle_codec *c, int32_t *out)
{
	for (int comp = 0; comp < 3; comp++)
		for (int level = 0; level < 5; level++)
			for (int band = 0; band < 4; band++)
			{
				const BandInfo &b = c->bands[comp][level][band];
				int32_t *o = out + ((comp * 5 + level) * 4 + band) * 4;
				bool present = c->has_band(comp, level, band);
				o[0] = present ? b.block_offset_8x8 : -1;
				o[1] = present ? b.block_stride_8x8 : -1;
				o[2] = present ? b.block_offset_32x32 : -1;
				o[3] = present ? b.block_stride_32x32 : -1;
			}
}

void oracle_block_mapping(const oracle_codec *c, int32_t *out)
{
	for (size_t i = 0; i < c->mapping.size(); i++)
	{
		out[4 * i + 0] = c->mapping[i].block_offset_8x8;
		out[4 * i + 1] = c->mapping[i].block_stride_8x8;
		out[4 * i + 2] = c->mapping[i].block_width_8x8;
		out[4 * i + 3] = c->mapping[i].block_height_8x8;
	}
}

void oracle_band_offsets(const oracle_codec *c, int64_t *out)
{
	for (int comp = 0; comp < 3; comp++)
		for (int level = 0; level < 5; level++)
			for (int band = 0; band < 4; band++)
				out[(comp * 5 + level) * 4 + band] =
				    c->has_band(comp, level, band) ? c->bands[comp][level][band].pyramid_offset : -1;
}

void oracle_quant_tables(const oracle_codec *c, float *qr, float *rdo)
{
	for (int comp = 0; comp < 3; comp++)
		for (int level = 0; level < 5; level++)
			for (int band = 0; band < 4; band++)
			{
				int i = (comp * 5 + level) * 4 + band;
				qr[i] = quant_resolution(level, comp, band);
				rdo[i] = rdo_distortion_scale(*c, level, comp, band) * (1.0f / 256.0f);
			}
}

int oracle_dwt(oracle_codec *c, const uint8_t *const planes[3], const int strides[3], int mode, float *out)
{
	if (mode != ORACLE_MODE_F32 && mode != ORACLE_MODE_REF16)
		return -1;
	return run_dwt<float>(*c, planes, strides, mode, out);
}

int oracle_dwt_f64(oracle_codec *c, const uint8_t *const planes[3], const int strides[3], double *out)
{
	return run_dwt<double>(*c, planes, strides, ORACLE_MODE_F64, out);
}

int oracle_dwt16(oracle_codec *c, const uint16_t *const planes[3], const int strides[3], int mode, float *out)
{
	if (mode != ORACLE_MODE_F32 && mode != ORACLE_MODE_REF16)
		return -1;
	return run_dwt<float, uint16_t>(*c, planes, strides, mode, out);
}

// pyrowave_encoder.cpp:1117-1183 minus the DWT: quant -> analyze -> finalize ->
// resolve -> block packing over every band in dispatch order.
int oracle_encode_pyramid(oracle_codec *c, const float *pyramid, uint64_t maximum_bitstream_size, uint32_t sequence,
                          float quant_scale)
{
	// pyrowave_c.cpp:957-961
	uint64_t target = maximum_bitstream_size & ~uint64_t(3);
	if (target > UINT32_MAX || target == 0)
		return -2;

	c->sequence = sequence & 7u;
	c->code_words.assign(c->block_count_8x8, 0);
	c->payload_offset.assign(c->block_count_8x8, 0);
	c->stats.assign(c->block_count_8x8, BlockStats{});
	c->payload.clear();
	c->rate_cost.assign(size_t(c->block_count_32x32) * 16, 0);
	c->distortion.assign(size_t(c->block_count_32x32) * 16, 0.0f);
	c->bucket.assign(size_t(c->block_count_32x32) * 16, 0);
	c->consumed_payload = 0;
	c->quant.assign(c->block_count_32x32, 0);
	c->meta.assign(size_t(c->block_count_32x32) * 2, 0);
	c->bitstream.clear();

	// Quant: pyrowave_encoder.cpp:433-479 (+ the pre-transformed override at :449).
	for (int level = 0; level < DecompositionLevels; level++)
		for (int comp = 0; comp < NumComponents; comp++)
			for (int band = 0; band < 4; band++)
			{
				if (!c->has_band(comp, level, band))
					continue;
				float qres = quant_scale < 0.0f ? quant_resolution(level, comp, band) : quant_scale;
				float push_qres = 1.0f / decode_quant(encode_quant(1.0f / qres));
				float rdo = rdo_distortion_scale(*c, level, comp, band) * (1.0f / 256.0f);
				const BandInfo &info = c->bands[comp][level][band];
				quant_band(*c, pyramid + info.pyramid_offset, c->level_width(level), c->level_height(level), info,
				           push_qres, rdo);
			}

	// Analyze: pyrowave_encoder.cpp:340-413
	int nbps = block_count_per_subdivision(c->block_count_32x32);
	uint32_t num_blocks_aligned = uint32_t(nbps * BlockSpaceSubdivision);
	uint32_t shamt = uint32_t(find_msb(uint32_t(nbps)));
	std::vector<RDOperation> ops(size_t(NumRDOBuckets) * num_blocks_aligned, RDOperation{0, 0});
	std::vector<uint32_t> total_savings(NumRDOBuckets * BlockSpaceSubdivision, 0);
	for (int level = 0; level < DecompositionLevels; level++)
		for (int comp = 0; comp < NumComponents; comp++)
			for (int band = 0; band < 4; band++)
			{
				if (!c->has_band(comp, level, band))
					continue;
				analyze_band(*c, c->level_width(level), c->level_height(level), c->bands[comp][level][band], ops,
				             total_savings, num_blocks_aligned, shamt);
			}

	// Finalize: analyze_rate_control_finalize.comp (inclusive scan of 2048 counters).
	for (size_t i = 1; i < total_savings.size(); i++)
		total_savings[i] += total_savings[i - 1];
	c->savings_scan = total_savings;

	// Resolve: resolve_rate_control.comp:38-81 with pyrowave_encoder.cpp:289-324.
	uint64_t target_payload_size = target;
	if (target_payload_size >= 8)
		target_payload_size -= 8;
	uint32_t target_words = uint32_t(target_payload_size / 4);
	for (int x = 0; x < NumRDOBuckets * BlockSpaceSubdivision; x++)
	{
		int32_t required = int32_t(c->consumed_payload) - int32_t(target_words);
		if (x != 0)
		{
			int32_t prev = int32_t(total_savings[x - 1]);
			if (int32_t(total_savings[x]) == prev)
				continue;
			required -= prev;
		}
		else if (total_savings[x] == 0)
			continue;
		if (required <= 0)
			continue;
		uint32_t total_saved = 0;
		for (int i = 0; i < nbps && total_saved < uint32_t(required); i++)
		{
			const RDOperation &op = ops[size_t(x) * nbps + i];
			uint32_t saving = op.block_offset_saving >> 16;
			uint32_t block_offset = op.block_offset_saving & 0xffffu;
			if (total_saved < uint32_t(required) && saving != 0)
				c->quant[block_offset] = std::max(c->quant[block_offset], op.quant);
			total_saved += saving;
		}
	}

	// Block packing: pyrowave_encoder.cpp:229-270. Blocks are emitted in block index
	// order, so bands are walked in index order here.
	std::vector<std::pair<int, int>> order; // unused placeholder for clarity
	(void)order;
	for (int level = DecompositionLevels - 1; level >= 0; level--)
		for (int comp = 0; comp < NumComponents; comp++)
			for (int band = 0; band < 4; band++)
			{
				if (!c->has_band(comp, level, band))
					continue;
				int w = c->level_width(level), h = c->level_height(level);
				float qres = quant_scale < 0.0f ? quant_resolution(level, comp, band) : quant_scale;
				uint32_t code = encode_quant(1.0f / qres);
				const BandInfo &info = c->bands[comp][level][band];
				int bx32 = (w + 31) / 32, by32 = (h + 31) / 32;
				for (int by = 0; by < by32; by++)
					for (int bx = 0; bx < bx32; bx++)
						pack_block(*c, bx, by, w, h, info, code);
			}
	return 0;
}

void oracle_get_code_words(const oracle_codec *c, uint32_t *out)
{
	memcpy(out, c->code_words.data(), c->code_words.size() * 4);
}

void oracle_get_block_stats(const oracle_codec *c, uint32_t *out)
{
	memcpy(out, c->stats.data(), c->stats.size() * sizeof(BlockStats));
}

void oracle_get_rd(const oracle_codec *c, uint32_t *rate_cost, float *distortion, uint32_t *bucket)
{
	memcpy(rate_cost, c->rate_cost.data(), c->rate_cost.size() * 4);
	memcpy(distortion, c->distortion.data(), c->distortion.size() * 4);
	memcpy(bucket, c->bucket.data(), c->bucket.size() * 4);
}

void oracle_get_histogram(const oracle_codec *c, uint32_t *scan2048, uint32_t *consumed)
{
	memcpy(scan2048, c->savings_scan.data(), c->savings_scan.size() * 4);
	*consumed = c->consumed_payload;
}

void oracle_get_quant(const oracle_codec *c, int32_t *out) { memcpy(out, c->quant.data(), c->quant.size() * 4); }
void oracle_get_meta(const oracle_codec *c, uint32_t *out) { memcpy(out, c->meta.data(), c->meta.size() * 4); }
size_t oracle_get_bitstream_words(const oracle_codec *c) { return c->bitstream.size(); }
void oracle_get_bitstream(const oracle_codec *c, uint32_t *out)
{
	memcpy(out, c->bitstream.data(), c->bitstream.size() * 4);
}

// Replace the encoder output (per-block meta + block words) with given data,
// so that packetize can be checked on arbitrary block tables.
void oracle_set_encoded(oracle_codec *c, const uint32_t *meta, const uint32_t *words, size_t nwords, uint32_t sequence)
{
	c->meta.assign(meta, meta + size_t(c->block_count_32x32) * 2);
	c->bitstream.assign(words, words + nwords);
	c->sequence = sequence & 7u;
}

// pyrowave_encoder.cpp:596-623
size_t oracle_compute_num_packets(const oracle_codec *c, size_t packet_boundary)
{
	size_t num_packets = 0, size_in_packet = 8;
	for (int i = 0; i < c->block_count_32x32; i++)
	{
		size_t packet_size = size_t(c->meta[2 * i + 1]) * 4;
		if (!packet_size)
			continue;
		if (size_in_packet + packet_size > packet_boundary)
		{
			size_in_packet = 0;
			num_packets++;
		}
		size_in_packet += packet_size;
	}
	if (size_in_packet)
		num_packets++;
	return num_packets;
}

// pyrowave_encoder.cpp:1048-1115. The sequence header carries the encoder's
// sequence counter (the reference reads it back from block 0's header).
size_t oracle_packetize(const oracle_codec *c, uint64_t *packets, size_t packet_boundary, uint8_t *out, size_t size)
{
	size_t num_packets = 0, size_in_packet = 0, packet_offset = 0, output_offset = 0;
	uint32_t non_zero = 0;
	for (int i = 0; i < c->block_count_32x32; i++)
		if (c->meta[2 * i + 1] != 0)
			non_zero++;
	uint32_t w0 = uint32_t(c->width - 1) | (uint32_t(c->height - 1) << 14) | ((c->sequence & 7u) << 28) | (1u << 31);
	uint32_t w1 = (non_zero & 0xffffffu) | (0u << 24) | ((c->chroma444 ? 1u : 0u) << 26);
	if (size < 8)
		return 0;
	memcpy(out, &w0, 4);
	memcpy(out + 4, &w1, 4);
	output_offset = 8;
	size_in_packet = 8;
	for (int i = 0; i < c->block_count_32x32; i++)
	{
		size_t packet_size = size_t(c->meta[2 * i + 1]) * 4;
		if (!packet_size)
			continue;
		if (size_in_packet + packet_size > packet_boundary)
		{
			packets[2 * num_packets + 0] = packet_offset;
			packets[2 * num_packets + 1] = size_in_packet;
			num_packets++;
			size_in_packet = 0;
			packet_offset = output_offset;
		}
		if (output_offset + packet_size > size)
			return num_packets;
		memcpy(out + output_offset, c->bitstream.data() + c->meta[2 * i], packet_size);
		output_offset += packet_size;
		size_in_packet += packet_size;
	}
	if (size_in_packet)
	{
		packets[2 * num_packets + 0] = packet_offset;
		packets[2 * num_packets + 1] = size_in_packet;
		num_packets++;
	}
	return num_packets;
}

oracle_parser *oracle_parser_create(const oracle_codec *codec)
{
	auto *p = new oracle_parser;
	p->codec = codec;
	p->offsets.resize(codec->block_count_32x32);
	p->clear();
	return p;
}

void oracle_parser_destroy(oracle_parser *p) { delete p; }
void oracle_parser_clear(oracle_parser *p) { p->clear(); }
int oracle_parser_push_packet(oracle_parser *p, const void *data, size_t size)
{
	return p->push_packet(static_cast<const uint8_t *>(data), size) ? 0 : -1;
}
int oracle_parser_decode_is_ready(const oracle_parser *p, int allow_partial) { return p->decode_is_ready(allow_partial != 0); }
void oracle_parser_mark_decoded(oracle_parser *p) { p->decoded_frame_for_current_sequence = true; }
size_t oracle_parser_payload_words(const oracle_parser *p) { return p->payload.size(); }
void oracle_parser_get(const oracle_parser *p, uint32_t *offsets, uint32_t *payload)
{
	memcpy(offsets, p->offsets.data(), p->offsets.size() * 4);
	if (!p->payload.empty())
		memcpy(payload, p->payload.data(), p->payload.size() * 4);
}
int oracle_parser_decoded_blocks(const oracle_parser *p) { return p->decoded_blocks; }
int oracle_parser_total_blocks(const oracle_parser *p) { return p->total_blocks_in_sequence; }

// pyrowave_decoder.cpp:280-381: dequant every band. Storage rounding: F32 mode
// follows the level mask; REF16 mode stores levels 0-1 in FP16 (the reference's
// precision 1 images, pyrowave_common.cpp:133-170).
int oracle_dequant(const oracle_codec *c, const uint32_t *offsets, const uint32_t *payload, size_t payload_words, int mode,
                   float *out)
{
	for (int level = 0; level < DecompositionLevels; level++)
		for (int comp = 0; comp < NumComponents; comp++)
			for (int band = 0; band < 4; band++)
			{
				if (!c->has_band(comp, level, band))
					continue;
				int w = c->level_width(level), h = c->level_height(level);
				const BandInfo &info = c->bands[comp][level][band];
				int r16 = mode == ORACLE_MODE_REF16 ? (level < 2) : (mode == ORACLE_MODE_F32 ? c->level_fp16(level) : 0);
				for (int by = 0; by < (h + 31) / 32; by++)
					for (int bx = 0; bx < (w + 31) / 32; bx++)
					{
						uint32_t bi = uint32_t(info.block_offset_32x32 + by * info.block_stride_32x32 + bx);
						dequant_block(*c, offsets, payload, payload_words, bi, out + info.pyramid_offset, w, h, bx, by, r16);
					}
			}
	return 0;
}

int oracle_idwt(oracle_codec *c, const float *pyramid, int mode, uint8_t *const planes[3], const int strides[3])
{
	if (mode != ORACLE_MODE_F32 && mode != ORACLE_MODE_REF16)
		return -1;
	return run_idwt<float>(*c, pyramid, mode, planes, strides);
}

int oracle_idwt_f64(oracle_codec *c, const double *pyramid, uint8_t *const planes[3], const int strides[3])
{
	return run_idwt<double>(*c, pyramid, ORACLE_MODE_F64, planes, strides);
}

int oracle_idwt16(oracle_codec *c, const float *pyramid, int mode, uint16_t *const planes[3], const int strides[3])
{
	if (mode != ORACLE_MODE_F32 && mode != ORACLE_MODE_REF16)
		return -1;
	return run_idwt<float, uint16_t>(*c, pyramid, mode, planes, strides);
}

uint16_t oracle_float_to_half(float v) { return float_to_half(v); }
float oracle_half_to_float(uint16_t h) { return half_to_float(h); }
uint32_t oracle_bucket_index(float d, float cost, float d_base, float cost_base)
{
	return bucket_index(d, cost, d_base, cost_base);
}
}

// ---------------------------------------------------------------------------
// PSNR-HVS-M of a luma plane against a reference luma plane: the reference's
// quality metric (shaders/psnr_hvs_m.comp:1-225, a port of Ponomarenko's
// psnrhvsm.m with its own contrast sensitivity function), with the host-side
// tables of psnr.cpp:25-28 (CSF), 126-224 (per height factor: CSF, masking
// coefficients and their inverses, the 8x8 windows at a stride of 4) and
// 245-320 (16 height factors 1 + i/8, fixed-point 2^-24 error sums, the
// 10*log10 of pixels * peak / error). Every floating-point operation is one
// rounded IEEE operation in the written order (no contraction), so the CUDA
// kernel can reproduce the sums bit for bit. Samples outside the plane read as
// zero (a texel fetch with robust image access).
namespace
{
constexpr int kHvsFactors = 16;

struct HvsTables
{
	float csf[8][8];
	float mask[8][8];
	float inv_mask[8][8];
};

float hvs_contrast_sensitivity(float cpd) // psnr.cpp:25-28
{
	return 2.6f * (0.0192f + 0.114f * cpd) * std::exp(-std::pow(0.114f * cpd, 1.1f));
}

void hvs_tables(int height, int factor, HvsTables &t) // psnr.cpp:151-195
{
	const float height_factor = 1.0f + float(factor) / 8.0f;
	const float pi = 3.14159265358979323846f;
	const float nyquist_cpd = float(height) * height_factor * pi / 360.0f;
	for (int y = 0; y < 8; y++)
		for (int x = 0; x < 8; x++)
		{
			const float H = (float(x) + 0.5f) / 8.0f;
			const float V = (float(y) + 0.5f) / 8.0f;
			const float cpd = std::sqrt(H * H + V * V);
			t.csf[y][x] = 2.6f * hvs_contrast_sensitivity(cpd * nyquist_cpd);
		}
	float max_csf = 0.0f;
	for (auto &row : t.csf)
		for (float v : row)
			max_csf = std::max(max_csf, v);
	float norm = 1.0f / max_csf;
	norm *= norm;
	for (int y = 0; y < 8; y++)
		for (int x = 0; x < 8; x++)
			t.mask[y][x] = t.csf[y][x] * t.csf[y][x] * norm;
	t.mask[0][0] = 0.0f;
	for (int y = 0; y < 8; y++)
		for (int x = 0; x < 8; x++)
			t.inv_mask[y][x] = (y || x) ? 1.0f / t.mask[y][x] : 0.0f;
}

void hvs_butterfly(float &a, float &b)
{
	const float pos = a + b, neg = a - b;
	a = pos;
	b = neg;
}

void hvs_rotate(float &a, float &b, float c, float s)
{
	const float pos = a * c + b * s, neg = b * c - a * s;
	a = pos;
	b = neg;
}

void hvs_dct8(float dct[8], float sig[8]) // psnr_hvs_m.comp:58-97
{
	const float c7 = 0.19509032201612833f, s7 = 0.9807852804032304f;
	const float c6 = 0.38268343236508984f, s6 = 0.9238795325112867f;
	const float c5 = 0.5555702330196023f, s5 = 0.8314696123025452f;
	const float r1 = std::sqrt(1.0f / 8.0f), r2 = std::sqrt(2.0f / 8.0f);
	hvs_butterfly(sig[0], sig[7]);
	hvs_butterfly(sig[1], sig[6]);
	hvs_butterfly(sig[2], sig[5]);
	hvs_butterfly(sig[3], sig[4]);
	hvs_butterfly(sig[0], sig[3]);
	hvs_butterfly(sig[1], sig[2]);
	hvs_butterfly(sig[0], sig[1]);
	hvs_rotate(sig[2], sig[3], c6, s6);
	hvs_rotate(sig[4], sig[7], c7, s7);
	hvs_rotate(sig[5], sig[6], c5, s5);
	hvs_butterfly(sig[4], sig[5]);
	hvs_butterfly(sig[6], sig[7]);
	hvs_butterfly(sig[5], sig[6]);
	sig[0] *= r1;
	sig[1] *= r1;
	sig[2] *= r2;
	sig[3] *= r2;
	sig[4] *= r2;
	sig[5] *= r1;
	sig[6] *= r1;
	sig[7] *= -r2;
	dct[0] = sig[0];
	dct[1] = sig[4];
	dct[2] = sig[2];
	dct[3] = sig[5];
	dct[4] = sig[1];
	dct[5] = sig[6];
	dct[6] = sig[3];
	dct[7] = sig[7];
}

void hvs_dct8x8(float dct[8][8], float sig[8][8]) // psnr_hvs_m.comp:155-171
{
	for (int row = 0; row < 8; row++)
	{
		float s[8];
		memcpy(s, sig[row], sizeof(s));
		hvs_dct8(dct[row], s);
	}
	for (int col = 0; col < 8; col++)
	{
		float s[8], d[8];
		for (int i = 0; i < 8; i++)
			s[i] = dct[i][col];
		hvs_dct8(d, s);
		for (int i = 0; i < 8; i++)
			dct[i][col] = d[i];
	}
}

float hvs_vari(float e, float e2, int count) // psnr_hvs_m.comp:104-107
{
	return std::max(e2 * float(count) - e * e, 0.0f) / float(count - 1);
}

// The factor-independent part of maskeff (psnr_hvs_m.comp:109-153): the ratio
// of the quadrant variances to the block variance.
float hvs_pop(float sig[8][8])
{
	float sum_e2[2][2], sum_e[2][2];
	float sum_e2_total = 0.0f, sum_e_total = 0.0f;
	for (int y = 0; y < 2; y++)
		for (int x = 0; x < 2; x++)
		{
			sum_e2[y][x] = 0.0f;
			sum_e[y][x] = 0.0f;
			for (int suby = 0; suby < 4; suby++)
				for (int subx = 0; subx < 4; subx++)
				{
					const float v = sig[y * 4 + suby][x * 4 + subx];
					sum_e[y][x] += v;
					sum_e2[y][x] += v * v;
				}
			sum_e_total += sum_e[y][x];
			sum_e2_total += sum_e2[y][x];
		}
	float pop = hvs_vari(sum_e_total, sum_e2_total, 64);
	if (pop != 0.0f)
		pop = (hvs_vari(sum_e[0][0], sum_e2[0][0], 16) + hvs_vari(sum_e[1][0], sum_e2[1][0], 16) +
		       hvs_vari(sum_e[0][1], sum_e2[0][1], 16) + hvs_vari(sum_e[1][1], sum_e2[1][1], 16)) /
		      pop;
	return pop;
}

float hvs_maskeff(const float dct[8][8], float pop, const HvsTables &t) // psnr_hvs_m.comp:109-153
{
	float m = 0.0f;
	for (int y = 0; y < 8; y++)
		for (int x = 0; x < 8; x++)
			m += dct[y][x] * dct[y][x] * t.mask[y][x];
	return std::sqrt(m * pop) / 32.0f;
}

float hvs_dct_error(const float a[8][8], const float b[8][8], float mask, const HvsTables &t) // :173-195
{
	float total = 0.0f;
	for (int y = 0; y < 8; y++)
		for (int x = 0; x < 8; x++)
		{
			float e = std::fabs(a[y][x] - b[y][x]);
			const float masking = mask * t.inv_mask[y][x];
			e = std::max(e - masking, 0.0f);
			const float w = e * t.csf[y][x];
			total += w * w;
		}
	return total;
}

void hvs_window(const uint8_t *plane, int stride, int w, int h, int x0, int y0, float sig[8][8])
{
	for (int y = 0; y < 8; y++)
		for (int x = 0; x < 8; x++)
		{
			const int px = x0 + x, py = y0 + y;
			sig[y][x] = (px < w && py < h) ? float(plane[size_t(py) * size_t(stride) + size_t(px)]) / 255.0f : 0.0f;
		}
}
} // namespace

extern "C" {
void oracle_psnr_hvs_m_tables(int height, float *out)
{
	for (int f = 0; f < kHvsFactors; f++)
	{
		HvsTables t;
		hvs_tables(height, f, t);
		memcpy(out + size_t(f) * 192, &t, sizeof(t));
	}
}

uint64_t oracle_psnr_hvs_m_pixels(int width, int height)
{
	const uint64_t bx = uint64_t((width - 1) / 4 + 1), by = uint64_t((height - 1) / 4 + 1);
	return bx * by * 64;
}

// Adds each height factor's fixed-point error sum (2^-24 units) into errors[16]. psnr_hvs_m.comp:197-225
void oracle_psnr_hvs_m(const uint8_t *ref, int ref_stride, const uint8_t *dist, int dist_stride, int width,
                       int height, uint64_t *errors)
{
	HvsTables tables[kHvsFactors];
	for (int f = 0; f < kHvsFactors; f++)
		hvs_tables(height, f, tables[f]);
	const int nbx = (width - 1) / 4 + 1, nby = (height - 1) / 4 + 1;
	for (int by = 0; by < nby; by++)
		for (int bx = 0; bx < nbx; bx++)
		{
			float sig[8][8], dct_a[8][8], dct_b[8][8];
			hvs_window(ref, ref_stride, width, height, bx * 4, by * 4, sig);
			const float pop_a = hvs_pop(sig);
			hvs_dct8x8(dct_a, sig);
			hvs_window(dist, dist_stride, width, height, bx * 4, by * 4, sig);
			const float pop_b = hvs_pop(sig);
			hvs_dct8x8(dct_b, sig);
			for (int f = 0; f < kHvsFactors; f++)
			{
				const float mask = std::max(hvs_maskeff(dct_a, pop_a, tables[f]), hvs_maskeff(dct_b, pop_b, tables[f]));
				const float e = hvs_dct_error(dct_a, dct_b, mask, tables[f]);
				errors[f] += uint64_t(std::ldexp(e, 24));
			}
		}
}

// dct8 of psnr_hvs_m.comp, exposed for the test that pins it to the orthonormal DCT-II.
void oracle_hvs_dct8(const float *in, float *out)
{
	float s[8];
	memcpy(s, in, sizeof(s));
	hvs_dct8(out, s);
}
}

// ---------------------------------------------------------------------------
// Packing analysis: the reference's disabled statistics pass
// (pyrowave_encoder.cpp:625-958, Encoder::Impl::report_stats and
// analyze_alternative_packing) restated for the current block format. It reads
// a decoded frame's integer coefficients back out of the bitstream and
// estimates what other packet / block / sub-block shapes would cost.
namespace
{
constexpr int kLayouts = 5;

int magnitude_bits(uint32_t v) { return v ? 32 - __builtin_clz(v) : 0; }

// analyze_cost<PacketW, PacketH, SubW, SubH> of pyrowave_encoder.cpp:650-713 on
// one 64x64 region of quantised magnitudes: 8 bytes per packet holding any
// significant value; per block (a packet's 4x4 grid) with one, 2 bits of plane
// code per sub-block plus a byte of Q bits and scale, then the planes (each
// sub-block at max(its magnitude bits, Q bits), Q bits = magnitude bits of the
// block minus 3) and a sign bit per significant value, rounded up to bytes.
template <int PW, int PH, int SW, int SH>
uint64_t analyze_cost(const uint16_t (&v)[64][64])
{
	constexpr int BW = PW / 4, BH = PH / 4, NS = (BW / SW) * (BH / SH);
	uint64_t cost = 0;
	for (int py = 0; py < 64; py += PH)
		for (int px = 0; px < 64; px += PW)
		{
			bool any = false;
			for (int y = 0; y < PH; y++)
				for (int x = 0; x < PW; x++)
					any |= v[py + y][px + x] != 0;
			if (any)
				cost += 8;
		}
	for (int by = 0; by < 64; by += BH)
		for (int bx = 0; bx < 64; bx += BW)
		{
			uint32_t mag = 0;
			int nnz = 0;
			for (int y = 0; y < BH; y++)
				for (int x = 0; x < BW; x++)
				{
					mag = std::max<uint32_t>(mag, v[by + y][bx + x]);
					nnz += v[by + y][bx + x] != 0;
				}
			if (mag == 0)
				continue;
			cost += 2 * NS / 8 + 1;
			const int q_bits = std::max(magnitude_bits(mag) - 3, 0);
			int weight_bits = 0;
			for (int sy = 0; sy < BH; sy += SH)
				for (int sx = 0; sx < BW; sx += SW)
				{
					uint32_t smag = 0;
					for (int y = 0; y < SH; y++)
						for (int x = 0; x < SW; x++)
							smag = std::max<uint32_t>(smag, v[by + sy + y][bx + sx + x]);
					weight_bits += SW * SH * std::max(magnitude_bits(smag), q_bits);
				}
			cost += uint64_t((weight_bits + nnz + 7) / 8);
		}
	return cost;
}

// The integer magnitudes of one coded 32x32 block, read from the stream the way
// the dequantiser reads it (dequant_block above), into out (zeros when absent),
// with each plane byte counted in hist by its position in the sub-block's run of
// planes (0: most significant). Returns the block's word count (0 when absent).
uint32_t decode_block_magnitudes(const uint32_t *offsets, const uint32_t *payload, size_t payload_words,
                                 uint32_t block_index, uint16_t (&out)[32][32], uint32_t *hist, uint64_t &significant)
{
	memset(out, 0, sizeof(out));
	const uint32_t offset_u32 = offsets[block_index];
	if (offset_u32 == ~0u)
		return 0;
	const uint8_t *p8 = reinterpret_cast<const uint8_t *>(payload);
	const size_t payload_bytes = payload_words * 4;
	auto rd8 = [&](size_t i) -> uint32_t { return i < payload_bytes ? p8[i] : 0u; };
	auto rd16 = [&](size_t i) -> uint32_t { return rd8(2 * i) | (rd8(2 * i + 1) << 8); };
	auto rd32 = [&](size_t i) -> uint32_t { return i < payload_words ? payload[i] : 0u; };

	const uint32_t header = rd32(offset_u32);
	const uint32_t ballot = header & 0xffffu, words = (header >> 16) & 0xfffu;
	const uint32_t nballot = uint32_t(popcount(ballot));
	uint32_t byte_pos = offset_u32 * 4 + 8 + 3 * nballot;
	for (int l = 0; l < 16; l++)
	{
		if (!((ballot >> l) & 1u))
			continue;
		const uint32_t local = uint32_t(popcount(ballot & ((1u << l) - 1u)));
		const uint32_t cw = rd16(size_t(offset_u32) * 2 + 4 + local);
		const uint32_t q_bits = rd8(size_t(offset_u32) * 4 + 8 + nballot * 2 + local) & 0xfu;
		const int lx = l & 3, ly = l >> 2;
		for (int s = 0; s < 8; s++)
		{
			const int planes = int(q_bits + ((cw >> (2 * s)) & 3u));
			uint32_t dec[8] = {};
			for (int j = 0; j < planes; j++)
			{
				const uint32_t pl = rd8(byte_pos++);
				if (j < 16)
					hist[j * 256 + pl]++;
				for (int b = 0; b < 8; b++)
					dec[b] |= ((pl >> b) & 1u) << (planes - 1 - j);
			}
			int sx, sy;
			subblock_origin(s, sx, sy);
			for (int b = 0; b < 8; b++)
			{
				int dx, dy;
				pixel_offset(b, dx, dy);
				out[ly * 8 + sy + dy][lx * 8 + sx + dx] = uint16_t(dec[b]);
				significant += dec[b] != 0;
			}
		}
	}
	return words;
}
} // namespace

extern "C" {
// Packing statistics of one decoded frame (offsets and payload as the parser
// returns them). layout_bytes[5]: analyze_cost over every 64x64 region of every
// coded band (pyrowave_encoder.cpp:717-829) for 32x32 packets with 2x2, 4x2 and
// 2x4 sub-blocks, 64x32 with 4x4 and 64x64 with 8x4; band_bytes[(c * 5 + level)
// * 4 + band]: coded bytes (block words x 4, pyrowave_encoder.cpp:869-912);
// hist[16 * 256]: plane bytes by position (pyrowave_encoder.cpp:884-895).
int oracle_analyze_packing(const oracle_codec *c, const uint32_t *offsets, const uint32_t *payload,
                           size_t payload_words, uint64_t *layout_bytes, uint64_t *band_bytes, uint64_t *significant,
                           uint32_t *hist)
{
	memset(layout_bytes, 0, kLayouts * sizeof(uint64_t));
	memset(band_bytes, 0, NumComponents * DecompositionLevels * 4 * sizeof(uint64_t));
	memset(hist, 0, 16 * 256 * sizeof(uint32_t));
	*significant = 0;
	uint16_t region[64][64];
	uint16_t block[32][32];
	for (int comp = 0; comp < NumComponents; comp++)
		for (int level = 0; level < DecompositionLevels; level++)
			for (int band = 0; band < 4; band++)
			{
				if (!c->has_band(comp, level, band))
					continue;
				const BandInfo &info = c->bands[comp][level][band];
				const int bw = (c->level_width(level) + 31) / 32, bh = (c->level_height(level) + 31) / 32;
				for (int ry = 0; ry < (bh + 1) / 2; ry++)
					for (int rx = 0; rx < (bw + 1) / 2; rx++)
					{
						memset(region, 0, sizeof(region));
						for (int q = 0; q < 4; q++)
						{
							const int bx = 2 * rx + (q & 1), by = 2 * ry + (q >> 1);
							if (bx >= bw || by >= bh)
								continue;
							const uint32_t bi = uint32_t(info.block_offset_32x32 + by * info.block_stride_32x32 + bx);
							const uint32_t words =
							    decode_block_magnitudes(offsets, payload, payload_words, bi, block, hist, *significant);
							band_bytes[(comp * DecompositionLevels + level) * 4 + band] += uint64_t(words) * 4;
							for (int y = 0; y < 32; y++)
								memcpy(&region[(q >> 1) * 32 + y][(q & 1) * 32], block[y], sizeof(block[y]));
						}
						layout_bytes[0] += analyze_cost<32, 32, 2, 2>(region);
						layout_bytes[1] += analyze_cost<32, 32, 4, 2>(region);
						layout_bytes[2] += analyze_cost<32, 32, 2, 4>(region);
						layout_bytes[3] += analyze_cost<64, 32, 4, 4>(region);
						layout_bytes[4] += analyze_cost<64, 64, 8, 4>(region);
					}
			}
	return 0;
}
}
