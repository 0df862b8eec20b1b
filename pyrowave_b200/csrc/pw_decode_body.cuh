// Device bodies of the decoder stages, shared by the per-stage kernels
// (pw_decode.cu) and the batched form's persistent kernel (pw_encode.cu):
// the dequantiser of one 32x32 block and the inverse transform of one tile.
//
// Reference behaviour followed (file:line in the reference tree):
//   dequantiser   shaders/wavelet_dequant.comp:100-391 (STORAGE_MODE 0), pyrowave_decoder.cpp:280-381
//   inverse level shaders/idwt.comp:25-214, pyrowave_decoder.cpp:699-778
//
// Every payload read is bounds-checked against the payload size: the payload
// comes from the network and a malformed packet must decode to garbage, never
// to an out-of-bounds access. Reads past the end return zero.
#pragma once

#include "pw_device.cuh"

namespace pw
{
namespace
{
struct PayloadReader
{
	const uint32_t *words;
	uint32_t nwords;
	__device__ __forceinline__ uint32_t w32(uint32_t i) const { return i < nwords ? __ldcg(words + i) : 0u; }
	__device__ __forceinline__ uint32_t u8(uint32_t i) const { return (w32(i >> 2) >> (8u * (i & 3u))) & 0xffu; }
	__device__ __forceinline__ uint32_t u16(uint32_t i) const { return (w32(i >> 1) >> (16u * (i & 1u))) & 0xffffu; }
};

// A block's words staged in shared memory: words [base, base + count) of the
// payload come from `s`, anything else from the bounds-checked global reader,
// so reads of a malformed block behave exactly as with PayloadReader alone.
struct StagedReader
{
	const uint32_t *s;
	uint32_t base, count;
	PayloadReader g;
	__device__ __forceinline__ uint32_t w32(uint32_t i) const
	{
		const uint32_t r = i - base;
		return r < count ? s[r] : g.w32(i);
	}
	__device__ __forceinline__ uint32_t u8(uint32_t i) const { return (w32(i >> 2) >> (8u * (i & 3u))) & 0xffu; }
	__device__ __forceinline__ uint32_t u16(uint32_t i) const { return (w32(i >> 1) >> (16u * (i & 1u))) & 0xffffu; }
};

constexpr uint32_t kSpeculativeWords = 128; // staged with the header when the block size is not yet known

// s[i] = payload word off + i for i in [begin, end), by kThreads threads with
// up to eight loads per thread in flight together.
template <int kThreads = 128>
__device__ __forceinline__ void stage_words(uint32_t *s, const PayloadReader &g, uint32_t off, uint32_t begin,
                                            uint32_t end, int t)
{
	for (uint32_t base = begin + uint32_t(t); base < end; base += kThreads * 8)
	{
		uint32_t v[8];
#pragma unroll
		for (int u = 0; u < 8; u++)
		{
			const uint32_t i = base + uint32_t(kThreads) * u;
			v[u] = i < end ? g.w32(off + i) : 0u;
		}
#pragma unroll
		for (int u = 0; u < 8; u++)
		{
			const uint32_t i = base + uint32_t(kThreads) * u;
			if (i < end)
				s[i] = v[u];
		}
	}
}

// The barrier of a block's thread group: hardware barrier `bar` of 128
// threads, or the whole CTA when a CTA holds one smaller group.
template <int kSubs> __device__ __forceinline__ void block_sync(int bar)
{
	if constexpr (kSubs == 1)
		group_sync(bar);
	else
		__syncthreads();
}

__device__ __forceinline__ void store_coef(float *c32, __half *c16, bool fp16, int64_t idx, float v)
{
	if (fp16)
		c16[idx] = __float2half_rn(v);
	else
		c32[idx] = v;
}

// One 32x32 block per thread group; thread = one 4x2 sub-block (the
// reference's mapping, wavelet_dequant.comp:222-238), or kSubs sub-blocks two
// 8x8 rows apart. The group with `clear_error` set clears the decode's error
// word: every inverse level runs after the dequantiser has completed, so the
// clear precedes any error report.
struct DequantShared
{
	uint32_t s_words[kMaxBlockWords];
	uint32_t s_plane_off[16];
	uint32_t s_sign_base;
	uint32_t s_sig[4];
};

// One 32x32 block on a group of 128 / kSubs threads: with kSubs = 1 the group
// is threadIdx.x & 127, synchronised with hardware barrier `bar`; with kSubs =
// 2 the whole 64-thread CTA, each thread decoding the sub-blocks of 8x8 rows
// ly and ly + 2.
template <int kSubs = 1>
__device__ __forceinline__ void dequant_body(DequantShared &sh, const BlockParams &p, const DecodeInput &in,
                                             const int blk, const bool clear_error, const int bar)
{
	static_assert(kSubs == 1 || kSubs == 2, "one or two sub-blocks per thread");
	constexpr int kGroup = 128 / kSubs;
	constexpr int kRowStep = 4 / kSubs;
	uint32_t *const s_words = sh.s_words;
	uint32_t *const s_plane_off = sh.s_plane_off;
	uint32_t &s_sign_base = sh.s_sign_base;
	uint32_t *const s_sig = sh.s_sig;
	pdl_trigger();
	const int k = find_band(p, blk);
	const BandEntry &B = p.band[k];
	const LevelDesc &L = p.level[B.level];
	const int rel = blk - B.block32_offset;
	const int by32 = rel / B.block32_stride, bx32 = rel - by32 * B.block32_stride;
	const bool f16 = L.fp16 != 0;
	const int t = threadIdx.x & (kGroup - 1), lane = t & 31;
	const int sub = t & 7, lx = (t >> 3) & 3, ly0 = t >> 5;
	const int ox = bx32 * 32 + lx * 8 + sub_x(sub);
	pdl_wait();
	if (clear_error && t == 0 && in.error)
		*in.error = 0u;
	if (clear_error && in.state && t < int(sizeof(DecodeState) / 4))
		reinterpret_cast<uint32_t *>(in.state)[t] = 0u;

	uint32_t off, words = 0;
	const bool sized_by_header = in.offsets || in.keys;
	if (in.keys)
	{
		const unsigned long long key = __ldcg(in.keys + blk);
		off = key == ~0ull ? 0xffffffffu : uint32_t(key & 0x3fffffffull);
	}
	else if (in.offsets)
		off = __ldcg(in.offsets + blk);
	else
	{
		const uint2 m = __ldcg(reinterpret_cast<const uint2 *>(in.block_meta) + blk);
		off = m.y ? m.x : 0xffffffffu;
		words = m.y;
	}

	if (off == 0xffffffffu)
	{
		// Missing block: all coefficients are zero (wavelet_dequant.comp:242-248).
		const float zero[8] = {0.f, 0.f, 0.f, 0.f, 0.f, 0.f, 0.f, 0.f};
#pragma unroll
		for (int h = 0; h < kSubs; h++)
		{
			const int oy = by32 * 32 + (ly0 + h * kRowStep) * 8 + sub_y(sub);
			store_subblock(in.coef32, in.coef16, f16, B.offset + int64_t(oy) * L.pitch + ox, L.pitch, zero);
		}
		return;
	}

	// Stage the block's words in shared memory with all loads in flight at
	// once; every read below is then a shared-memory read. With only an offset
	// table the size comes from the block header, so the first
	// kSpeculativeWords are fetched together with it.
	const PayloadReader grd{in.payload, in.payload_words};
	uint32_t staged;
	if (sized_by_header)
	{
		stage_words<kGroup>(s_words, grd, off, 0, kSpeculativeWords, t);
		block_sync<kSubs>(bar);
		words = (s_words[0] >> 16) & 0xfffu;
		staged = min(max(words, kSpeculativeWords), uint32_t(kMaxBlockWords));
		stage_words<kGroup>(s_words, grd, off, kSpeculativeWords, staged, t);
	}
	else
	{
		staged = min(words, uint32_t(kMaxBlockWords));
		stage_words<kGroup>(s_words, grd, off, 0, staged, t);
	}
	block_sync<kSubs>(bar);
	const StagedReader rd{s_words, off, staged, grd};
	const uint32_t ballot = rd.w32(off) & 0xffffu;
	const uint32_t q_code = rd.w32(off + 1) & 0xffu;
	const uint32_t n = uint32_t(__popc(ballot));

	if (t < 16)
	{
		uint32_t cw = 0, qb = 0;
		if ((ballot >> t) & 1u)
		{
			const uint32_t local = uint32_t(__popc(ballot & ((1u << t) - 1u)));
			cw = rd.u16(off * 2 + 4 + local);
			qb = rd.u8(off * 4 + 8 + n * 2 + local) & 0xfu;
		}
		const uint32_t lsbs = cw & 0x5555u;
		uint32_t msbs = cw & 0xaaaau;
		msbs |= msbs >> 1;
		const uint32_t cost = uint32_t(__popc(lsbs) + __popc(msbs)) + qb * 8u;
		uint32_t inc = cost;
#pragma unroll
		for (int o = 1; o < 16; o *= 2)
		{
			const uint32_t y = __shfl_up_sync(0x0000ffffu, inc, o);
			if (t >= o)
				inc += y;
		}
		const uint32_t base = off * 4 + 8 + 3 * n;
		s_plane_off[t] = base + inc - cost;
		if (t == 15)
			s_sign_base = 8u * (base + inc);
	}
	block_sync<kSubs>(bar);

	float v[kSubs][8];
#pragma unroll
	for (int h = 0; h < kSubs; h++)
	{
		const int grp = (ly0 + h * kRowStep) * 4 + lx;
#pragma unroll
		for (int i = 0; i < 8; i++)
			v[h][i] = 0.0f;
		if ((ballot >> grp) & 1u)
		{
			const uint32_t local = uint32_t(__popc(ballot & ((1u << grp) - 1u)));
			const uint32_t cw = rd.u16(off * 2 + 4 + local);
			const uint32_t cw2 = rd.u8(off * 4 + 8 + n * 2 + local);
			const uint32_t qb = cw2 & 0xfu;
			if (cw != 0)
			{
				const uint32_t mask = (1u << (2 * sub)) - 1u;
				const uint32_t lsbs = cw & 0x5555u;
				uint32_t msbs = cw & 0xaaaau;
				msbs |= msbs >> 1;
				uint32_t byte_offset =
				    uint32_t(__popc(lsbs & mask) + __popc(msbs & mask)) + qb * uint32_t(sub) + s_plane_off[grp];
				const int planes = int(qb + ((cw >> (2 * sub)) & 3u));
				uint32_t dec[8] = {0, 0, 0, 0, 0, 0, 0, 0};
				if (planes <= 16)
				{
					// Plane bytes (most significant first) as the rows of two 8x8 bit
					// matrices; transposed, byte i holds coefficient i's magnitude bits.
					unsigned long long lo = 0, hi = 0;
					for (int pl = planes - 1; pl >= 0; pl--)
					{
						const unsigned long long bits = rd.u8(byte_offset++);
						if (pl < 8)
							lo |= bits << (8 * pl);
						else
							hi |= bits << (8 * (pl - 8));
					}
					lo = transpose8x8(lo);
					hi = transpose8x8(hi);
#pragma unroll
					for (int i = 0; i < 8; i++)
						dec[i] = uint32_t((lo >> (8 * i)) & 0xffu) | (uint32_t((hi >> (8 * i)) & 0xffu) << 8);
				}
				else
				{
					// Only a malformed header gives more than 16 planes.
					for (int pl = planes - 1; pl >= 0; pl--)
					{
						const uint32_t bits = rd.u8(byte_offset++);
#pragma unroll
						for (int i = 0; i < 8; i++)
							dec[i] |= ((bits >> i) & 1u) << pl;
					}
				}
#pragma unroll
				for (int i = 0; i < 8; i++)
				{
					float f = float(dec[i]);
					if (f != 0.0f)
						f = __fadd_rn(f, 0.5f);
					v[h][i] = f;
				}
			}
			const float inv_scale = __fmul_rn(decode_quant(q_code), decode_quant_scale((cw2 >> 4) & 0xfu));
#pragma unroll
			for (int i = 0; i < 8; i++)
				v[h][i] = __fmul_rn(v[h][i], inv_scale);
		}
	}

	// Sign bits: position = number of significant coefficients before this one
	// (in sub-block order: 8x8 rows, then the 32 sub-blocks of a row).
	uint32_t nsig[kSubs], inc[kSubs];
#pragma unroll
	for (int h = 0; h < kSubs; h++)
	{
		nsig[h] = 0;
#pragma unroll
		for (int i = 0; i < 8; i++)
			nsig[h] += v[h][i] != 0.0f ? 1u : 0u;
		inc[h] = nsig[h];
#pragma unroll
		for (int o = 1; o < 32; o *= 2)
		{
			const uint32_t y = __shfl_up_sync(0xffffffffu, inc[h], o);
			if (lane >= o)
				inc[h] += y;
		}
		if (lane == 31)
			s_sig[ly0 + h * kRowStep] = inc[h];
	}
	block_sync<kSubs>(bar);
#pragma unroll
	for (int h = 0; h < kSubs; h++)
	{
		const int ly = ly0 + h * kRowStep;
		uint32_t bitpos = s_sign_base + inc[h] - nsig[h];
		for (int w = 0; w < ly; w++)
			bitpos += s_sig[w];
		// This thread's (at most 8) sign bits are consecutive: one 64-bit window.
		const uint32_t sw = bitpos >> 5, shift = bitpos & 31u;
		const uint64_t window = (uint64_t(rd.w32(sw + 1)) << 32 | rd.w32(sw)) >> shift;
		int nth = 0;
#pragma unroll
		for (int i = 0; i < 8; i++)
		{
			if (v[h][i] != 0.0f)
			{
				if ((window >> nth) & 1u)
					v[h][i] = -v[h][i];
				nth++;
			}
		}
		const int oy = by32 * 32 + ly * 8 + sub_y(sub);
		store_subblock(in.coef32, in.coef16, f16, B.offset + int64_t(oy) * L.pitch + ox, L.pitch, v[h]);
	}
}

constexpr int kBandTile = 36; // 32 band samples + 2 on each side
constexpr int kBandTilePitch = 37;
// Band tiles are stored as rows of 40 samples from 4 before the tile (16-byte
// aligned in the band, so an interior tile is one TMA box per band): band
// sample j of the tile (0 = 2 before it) is at column j + kBandCol0.
constexpr int kBandRow = 40;
constexpr int kBandCol0 = 2;
constexpr uint32_t kBandBoxBytes = kBandTile * kBandRow * 4;
constexpr uint32_t kTmaMaxPolls = 1u << 20; // bounded wait for a tile load

struct IdwtShared
{
	int yl[kBandTile], yh[kBandTile], xl[kBandTile], xh[kBandTile];
	alignas(128) float band[4][kBandTile][kBandRow];
	float v[2][64][kBandTilePitch]; // after vertical lifting: [horizontal low/high][output row][band column]
	uint64_t tile_bar;             // completion of the TMA tile loads
};

// One inverse level for a 64x64 output tile (32x32 band tile) of one component.
// Large levels run 256-thread CTAs, several per SM; the batched form's small
// levels run 1024-thread CTAs whose lifting items cover half as many outputs.
// With kStripes = 4 a CTA computes one stripe of 16 output rows of the tile
// (small levels: four times the CTAs, each with a quarter of the lifting and
// a third of the loads), with the same arithmetic per output.
template <int kThreads, int kStripes = 1>
__device__ __forceinline__ void idwt_body(IdwtShared &sh, const LevelParams &p, const DecodeInput &in,
                                          const PlaneOutput &out, const LevelTileMap *maps, const int tile,
                                          const int comp_index, const int stripe = 0)
{
	constexpr int kOut = kThreads >= 1024 ? 8 : 16; // outputs per lifting item
	constexpr int kSegs = 64 / kOut;
	constexpr int kWin = kOut + 8;
	static_assert(kStripes == 1 || (kStripes == kSegs && kOut == 16), "a stripe is one lifting segment of 16 rows");
	// Band tile rows this CTA reads: all 36, or the 12 that the stripe's segment spans.
	constexpr int kRows = kStripes == 1 ? kBandTile : kWin / 2;
	const int row0 = kStripes == 1 ? 0 : stripe * (kOut / 2);
	pdl_trigger();
	const int level = p.level;
	const int comp = (level == 0 && !p.chroma444) ? 0 : comp_index;
	const LevelDesc &L = p.L;
	const int tx = tile % L.tiles_x, ty = tile / L.tiles_x;
	const int nx = L.width, ny = L.height;
	const bool final_level = level == 0 || (level == 1 && comp != 0 && !p.chroma444);

	for (int k = threadIdx.x; k < 4 * kBandTile; k += kThreads)
	{
		const int j = k % kBandTile, which = k / kBandTile;
		const int px = tx * 32 - 2 + j, py = ty * 32 - 2 + j;
		if (which == 0)
			sh.xl[j] = inv_index_low(px, nx);
		else if (which == 1)
			sh.xh[j] = inv_index_high(px, nx);
		else if (which == 2)
			sh.yl[j] = inv_index_low(py, ny);
		else
			sh.yh[j] = inv_index_high(py, ny);
	}
	const bool f16 = L.fp16 != 0;
	const int64_t o0 = p.band[comp][0].offset, o1 = p.band[comp][1].offset, o2 = p.band[comp][2].offset,
	              o3 = p.band[comp][3].offset;
	// Interior tiles read every band sample at its own position: rows of 40
	// samples from 4 before the tile (16-byte aligned). Interior FP32 tiles of a
	// decoder with tensor maps take one TMA box per band (barrier and maps made
	// ready before the dependency wait); other interior tiles load 10 vectors per
	// row, all in flight at once. Edge tiles use the mirrored index tables.
	const int bx0 = tx * 32 - 2, by0 = ty * 32 - 2;
	const bool interior = bx0 - 2 >= 0 && by0 >= 0 && bx0 + 38 <= nx && by0 + kBandTile <= ny;
	const bool use_tma = kThreads == 256 && kStripes == 1 && interior && maps && ((maps->valid >> comp) & 1u) && !f16 &&
	                     !L.stage16;
	if (use_tma && threadIdx.x == 0)
	{
		mbarrier_init(&sh.tile_bar, 1);
		prefetch_tensor_map(&maps->map);
	}
	__syncthreads();
	pdl_wait();

	if (use_tma)
	{
		if (threadIdx.x == 0)
		{
			mbarrier_expect_tx(&sh.tile_bar, 4 * kBandBoxBytes);
#pragma unroll
			for (int b = 0; b < 4; b++)
				tma_load_2d(&sh.band[b][0][0], &maps->map, bx0 - kBandCol0, maps->row[comp][b] + by0, &sh.tile_bar);
		}
		const bool done = mbarrier_wait(&sh.tile_bar, 0, kTmaMaxPolls) && !maps->test_fail_wait;
		if (__syncthreads_or(!done))
		{
			// Give up on this tile: record it, and keep the CTA alive (its shared
			// memory is the copy's destination) for one more bounded wait.
			if (threadIdx.x == 0 && in.error)
				atomicOr(in.error, kDecodeErrorTileWait);
			(void)mbarrier_wait(&sh.tile_bar, 0, kTmaMaxPolls);
			return;
		}
	}
	else if (interior)
	{
		constexpr int kVecPerRow = 10;
		constexpr int kVecs = 4 * kRows * kVecPerRow; // 1440 for a whole tile
		constexpr int kIters = (kVecs + kThreads - 1) / kThreads;
		float4 v[kIters];
#pragma unroll
		for (int u = 0; u < kIters; u++)
		{
			const int k = threadIdx.x + u * kThreads;
			const int b = k / (kRows * kVecPerRow);
			const int r = k - b * kRows * kVecPerRow;
			const int i = row0 + r / kVecPerRow, j = r % kVecPerRow;
			if (k >= kVecs)
			{
				v[u] = make_float4(0.f, 0.f, 0.f, 0.f);
				continue;
			}
			const int64_t bo = b == 0 ? o0 : (b == 1 ? o1 : (b == 2 ? o2 : o3));
			const int64_t idx = bo + int64_t(by0 + i) * L.pitch + (bx0 - 2) + 4 * j;
			if (f16)
			{
				uint2 hv = __ldcg(reinterpret_cast<const uint2 *>(in.coef16 + idx));
				const float2 a = __half22float2(*reinterpret_cast<__half2 *>(&hv.x));
				const float2 c = __half22float2(*reinterpret_cast<__half2 *>(&hv.y));
				v[u] = make_float4(a.x, a.y, c.x, c.y);
			}
			else
				v[u] = __ldcg(reinterpret_cast<const float4 *>(in.coef32 + idx));
		}
#pragma unroll
		for (int u = 0; u < kIters; u++)
		{
			const int k = threadIdx.x + u * kThreads;
			if (k >= kVecs)
				continue;
			const int b = k / (kRows * kVecPerRow);
			const int r = k - b * kRows * kVecPerRow;
			const int i = row0 + r / kVecPerRow, j = r % kVecPerRow;
			float4 f = v[u];
			if (L.stage16)
			{
				f.x = round_to_half(f.x);
				f.y = round_to_half(f.y);
				f.z = round_to_half(f.z);
				f.w = round_to_half(f.w);
			}
			*reinterpret_cast<float4 *>(&sh.band[b][i][4 * j]) = f;
		}
	}
	else
	{
		constexpr int kN = 4 * kRows * kBandTile;
		constexpr int kIdwtGen = (kN + kThreads - 1) / kThreads; // every load in flight at once
		for (int base = threadIdx.x; base < kN; base += kThreads * kIdwtGen)
		{
			float v[kIdwtGen];
#pragma unroll
			for (int u = 0; u < kIdwtGen; u++)
			{
				const int k = base + u * kThreads;
				const int b = k / (kRows * kBandTile);
				const int r = k - b * kRows * kBandTile;
				const int i = row0 + r / kBandTile, j = r % kBandTile;
				const int yy = (b >> 1) ? sh.yh[i] : sh.yl[i];
				const int xx = (b & 1) ? sh.xh[j] : sh.xl[j];
				const int64_t bo = b == 0 ? o0 : (b == 1 ? o1 : (b == 2 ? o2 : o3));
				v[u] = k < kN ? (f16 ? __half2float(__ldcg(in.coef16 + bo + int64_t(yy) * L.pitch + xx))
				                     : __ldcg(in.coef32 + bo + int64_t(yy) * L.pitch + xx))
				              : 0.0f;
			}
#pragma unroll
			for (int u = 0; u < kIdwtGen; u++)
			{
				const int k = base + u * kThreads;
				if (k < kN)
				{
					const int b = k / (kRows * kBandTile);
					const int r = k - b * kRows * kBandTile;
					const int i = row0 + r / kBandTile, j = r % kBandTile;
					sh.band[b][i][j + kBandCol0] = L.stage16 ? round_to_half(v[u]) : v[u];
				}
			}
		}
	}
	__syncthreads();

	// Vertical lifting: 36 band columns x {horizontal low: LL/LH, horizontal high: HL/HH} x kSegs segments
	// (the stripe's segment only).
	constexpr int kVSegs = kStripes == 1 ? kSegs : 1;
	for (int item = threadIdx.x; item < kBandTile * 2 * kVSegs; item += kThreads)
	{
		const int col = item % kBandTile;
		const int which = (item / kBandTile) & 1;
		const int seg = kStripes == 1 ? item / (2 * kBandTile) : stripe;
		const int b_low = which ? 1 : 0, b_high = which ? 3 : 2;
		float e[kWin];
#pragma unroll
		for (int jj = 0; jj < kWin; jj++)
		{
			const int q = seg * kOut + jj;
			const int i = q >> 1;
			e[jj] = (q & 1) ? __fmul_rn(sh.band[b_high][i][col + kBandCol0], kInvK)
			                : __fmul_rn(sh.band[b_low][i][col + kBandCol0], kK);
		}
		lift_inverse(e);
#pragma unroll
		for (int jj = 4; jj < 4 + kOut; jj++)
			sh.v[which][seg * kOut + jj - 4][col] = L.stage16 ? round_to_half(e[jj]) : e[jj];
	}
	__syncthreads();

	// Horizontal lifting: 64 output rows (the stripe's 16) x kSegs segments of kOut outputs.
	constexpr int kHRows = kStripes == 1 ? 64 : kOut;
	for (int item = threadIdx.x; item < kHRows * kSegs; item += kThreads)
	{
		const int row = (kStripes == 1 ? 0 : stripe * kOut) + item % kHRows, seg = item / kHRows;
		float e[kWin];
#pragma unroll
		for (int jj = 0; jj < kWin; jj++)
		{
			const int q = seg * kOut + jj;
			const int i = q >> 1;
			e[jj] = (q & 1) ? __fmul_rn(sh.v[1][row][i], kInvK) : __fmul_rn(sh.v[0][row][i], kK);
		}
		lift_inverse(e);
		if (L.stage16)
		{
#pragma unroll
			for (int jj = 4; jj < 4 + kOut; jj++)
				e[jj] = round_to_half(e[jj]);
		}
		const int gy = ty * 64 + row;
		const int gx0 = tx * 64 + seg * kOut;
		if (final_level)
		{
			const int pw = p.plane_width[comp], ph = p.plane_height[comp];
			uint8_t *const plane = comp == 0 ? out.data[0] : (comp == 1 ? out.data[1] : out.data[2]);
			const int opitch = comp == 0 ? out.pitch[0] : (comp == 1 ? out.pitch[1] : out.pitch[2]);
			if (gy < ph && out.sample16)
			{
				// 16-bit samples (R16_UNORM store: clamp, then round to 1/65535).
				uint16_t *dst = reinterpret_cast<uint16_t *>(plane + size_t(gy) * opitch);
#pragma unroll
				for (int jj = 4; jj < 4 + kOut; jj++)
				{
					float f = __fadd_rn(e[jj], 0.5f);
					f = fminf(fmaxf(f, 0.0f), 1.0f);
					const int gx = gx0 + jj - 4;
					if (gx < pw)
						dst[gx] = uint16_t(int(__fadd_rn(__fmul_rn(f, 65535.0f), 0.5f)));
				}
			}
			else if (gy < ph)
			{
				uint8_t *dst = plane + size_t(gy) * opitch;
				uint32_t packed[kOut / 4];
#pragma unroll
				for (int w = 0; w < kOut / 4; w++)
					packed[w] = 0;
#pragma unroll
				for (int jj = 4; jj < 4 + kOut; jj++)
				{
					float f = __fadd_rn(e[jj], 0.5f);
					f = fminf(fmaxf(f, 0.0f), 1.0f);
					const uint32_t u = uint32_t(int(__fadd_rn(__fmul_rn(f, 255.0f), 0.5f)));
					packed[(jj - 4) >> 2] |= u << (8 * ((jj - 4) & 3));
				}
				if (gx0 + kOut <= pw && (reinterpret_cast<uintptr_t>(dst + gx0) & (kOut - 1)) == 0)
				{
					if constexpr (kOut == 16)
						*reinterpret_cast<uint4 *>(dst + gx0) = make_uint4(packed[0], packed[1], packed[2], packed[3]);
					else
						*reinterpret_cast<uint2 *>(dst + gx0) = make_uint2(packed[0], packed[1]);
				}
				else
				{
#pragma unroll
					for (int jj = 0; jj < kOut; jj++)
						if (gx0 + jj < pw)
							dst[gx0 + jj] = uint8_t(packed[jj >> 2] >> (8 * (jj & 3)));
				}
			}
		}
		else
		{
			const LevelDesc &P = p.P;
			const int64_t ll = comp == 0 ? p.prev_ll[0] : (comp == 1 ? p.prev_ll[1] : p.prev_ll[2]);
			const bool pf16 = P.fp16 != 0;
			if (gy < P.height)
			{
				const int64_t base = ll + int64_t(gy) * P.pitch + gx0;
				if (gx0 + kOut <= P.width)
				{
					if (pf16)
					{
#pragma unroll
						for (int v = 0; v < kOut / 8; v++)
						{
							uint32_t hw[4];
#pragma unroll
							for (int k = 0; k < 4; k++)
							{
								__half2 h2 = __floats2half2_rn(e[4 + 8 * v + 2 * k], e[5 + 8 * v + 2 * k]);
								hw[k] = *reinterpret_cast<uint32_t *>(&h2);
							}
							*reinterpret_cast<uint4 *>(in.coef16 + base + 8 * v) = make_uint4(hw[0], hw[1], hw[2], hw[3]);
						}
					}
					else
					{
#pragma unroll
						for (int k = 0; k < kOut / 4; k++)
							*reinterpret_cast<float4 *>(in.coef32 + base + 4 * k) =
							    make_float4(e[4 + 4 * k], e[5 + 4 * k], e[6 + 4 * k], e[7 + 4 * k]);
					}
				}
				else
				{
#pragma unroll
					for (int jj = 4; jj < 4 + kOut; jj++)
					{
						const int gx = gx0 + jj - 4;
						if (gx < P.width)
							store_coef(in.coef32, in.coef16, pf16, ll + int64_t(gy) * P.pitch + gx, e[jj]);
					}
				}
			}
		}
	}
}

} // namespace
} // namespace pw
