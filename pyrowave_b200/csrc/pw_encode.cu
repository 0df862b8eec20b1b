// Encoder kernels for sm_100a: fused forward CDF 9/7 level + quantiser + RD
// analysis, the single-CTA rate-control resolve, and block packing.
//
// Reference behaviour followed (file:line in the reference tree):
//   forward level      shaders/dwt.comp:38-234 (tile + apron, H then V lifting)
//   quantiser / stats  shaders/wavelet_quant.comp:72-316
//   RD analysis        shaders/analyze_rate_control.comp:73-220
//   finalize/resolve   shaders/analyze_rate_control_finalize.comp:14-38,
//                      shaders/resolve_rate_control.comp:38-81, pyrowave_encoder.cpp:283-338
//   block packing      shaders/block_packing.comp:97-379
//   packetize layout   pyrowave_encoder.cpp:1048-1115
#include "pw_decode_body.cuh"

namespace pw
{
namespace
{
constexpr int kTileIn = 72;  // 64 input samples + 4-sample apron on each side
// Rows of 76 samples: 16-byte aligned, so the horizontal lifting reads its
// window as float4 vectors without bank conflicts (76 = 4 * 19, 19 odd), and an
// interior tile of a level above 0 is one TMA box (72 rows of 76 samples).
constexpr int kInPitch = 76;
constexpr uint32_t kInBoxBytes = kTileIn * kInPitch * 4;
constexpr int kHPitch = 65;
constexpr int kBandPitch = 33;

// Reduction scratch of one 128-thread quantiser group (one 32x32 block).
struct QuantGroupShared
{
	float dist[4][16];
	uint32_t cost[4][16];
};

// ---------------------------------------------------------------------------
// Quantiser + RD analysis of one 32x32 block held in shared memory.
//
// A group of 128 * S threads handles the block. Thread t owns one 4x2
// sub-block, sub = t & 7, in 8x8 column lx = (t >> 3) & 3 and 8x8 row
// ly = (t >> 5) & 3 (one warp per 8x8 row, the reference's mapping,
// wavelet_quant.comp:294-306), and the statistics of every S-th quant level
// starting at 1 + (t >> 7): with S = 2 two threads share a sub-block's levels,
// halving the serial loop. Each level's values are computed by exactly one
// thread, in the same order, so the results do not depend on S.
//
// Every thread of the CTA must call this the same number of times (it contains
// __syncthreads); `active` is false for groups without a block this round.
template <int S>
__device__ __forceinline__ void quant_analyze_block(const float *tile, int tile_pitch, bool active, int t,
                                                    QuantGroupShared &sh, const LevelDesc &L, const BandParam &B,
                                                    int subdivision_shift, int bx32, int by32,
                                                    const EncodeBuffers &buf)
{
	const int sub = t & 7, lx = (t >> 3) & 3, ly = (t >> 5) & 3;
	const int r = t >> 7; // quant levels q with (q - 1) % S == r are this thread's
	const int lane = threadIdx.x & 31;
	const int x8 = bx32 * 4 + lx, y8 = by32 * 4 + ly;
	const bool in_range = active && x8 < L.blocks8_x && y8 < L.blocks8_y;
	const float qres = active ? B.quant_resolution : 1.0f;

	float v[8];
	const int ox = lx * 8 + sub_x(sub), oy = ly * 8 + sub_y(sub);
#pragma unroll
	for (int i = 0; i < 8; i++)
	{
		float c = in_range ? tile[(oy + (i & 1)) * tile_pitch + ox + (i >> 1)] : 0.0f;
		v[i] = __fmul_rn(c, qres);
	}

	// 8x8 maximum and quant scale (wavelet_quant.comp:174-181).
	float max_sub = 0.0f;
#pragma unroll
	for (int i = 0; i < 8; i++)
		max_sub = fmaxf(max_sub, fabsf(v[i]));
	float max_wave = max_sub;
	max_wave = fmaxf(max_wave, __shfl_xor_sync(0xffffffffu, max_wave, 1));
	max_wave = fmaxf(max_wave, __shfl_xor_sync(0xffffffffu, max_wave, 2));
	max_wave = fmaxf(max_wave, __shfl_xor_sync(0xffffffffu, max_wave, 4));

	uint32_t qcode;
	float qs;
	compute_quant_scale(max_wave, qcode, qs);
#pragma unroll
	for (int i = 0; i < 8; i++)
		v[i] = fminf(fmaxf(__fmul_rn(v[i], qs), -kMaxScaledMagnitude), kMaxScaledMagnitude);
	max_sub = fminf(__fmul_rn(max_sub, qs), kMaxScaledMagnitude);
	max_wave = fminf(__fmul_rn(max_wave, qs), kMaxScaledMagnitude);

	// The packer's input: the scaled values as sign-magnitude (|int(v)| <= 32767),
	// one 16-byte store per sub-block, written by the first thread of each.
	if (active && r == 0 && buf.mag16)
	{
		uint32_t w[4];
#pragma unroll
		for (int j = 0; j < 4; j++)
		{
			const uint32_t a = uint32_t(int(fabsf(v[2 * j]))) | (v[2 * j] < 0.0f ? 0x8000u : 0u);
			const uint32_t b = uint32_t(int(fabsf(v[2 * j + 1]))) | (v[2 * j + 1] < 0.0f ? 0x8000u : 0u);
			w[j] = a | (b << 16);
		}
		const int blk = B.block32_offset + by32 * B.block32_stride + bx32;
		*reinterpret_cast<uint4 *>(buf.mag16 + int64_t(blk) * 1024 + 8 * (t & 127)) = make_uint4(w[0], w[1], w[2], w[3]);
	}

	const float overall = __fmul_rn(qres, qs);
	const float inv_quant = __fdiv_rn(1.0f, overall);
	const float iqs = __fmul_rn(inv_quant, inv_quant);
	const float rdo = active ? B.rdo_scale : 0.0f;
	const int block4x2_max = int(max_sub);
	const int max_abs = int(max_wave);
	const int msb = find_msb(uint32_t(max_abs));

	// Stats at q = 0 (wavelet_quant.comp:139-165,205-238).
	int qp0 = 0, shifted0 = block4x2_max, cost_early0 = block4x2_max > 0 ? 1 : 0;
	if (msb >= 3)
	{
		qp0 = msb - 2;
		cost_early0 = qp0 + 1;
		shifted0 >>= qp0;
	}
	cost_early0 += find_msb(uint32_t(shifted0)) + 1;
	// compute_square_error (wavelet_quant.comp:113-128) reconstructs each value
	// quantised at q as trunc((floor(|v| / 2^q) + 0.5) * 2^q) when nonzero. With
	// m = int(|v|) (|v| < 2^15), floor(|v| / 2^q) = m >> q and, for q >= 1, the
	// reconstruction is the integer ((m >> q) << q) + 2^(q-1): the same values,
	// computed without floating-point rounding steps.
	float av[8];
	int nsig0 = 0;
#pragma unroll
	for (int i = 0; i < 8; i++)
	{
		av[i] = fabsf(v[i]);
		nsig0 += av[i] >= 1.0f ? 1 : 0; // int(|v|) != 0
	}
	int csum0 = max(cost_early0 - 1, 0) * 8 + nsig0;
	csum0 += __shfl_xor_sync(0xffffffffu, csum0, 1);
	csum0 += __shfl_xor_sync(0xffffffffu, csum0, 2);
	csum0 += __shfl_xor_sync(0xffffffffu, csum0, 4);

	uint32_t plane_code = uint32_t(find_msb(uint32_t(shifted0)) + 1);
	uint32_t cw = plane_code << (2 * sub);
	cw |= __shfl_xor_sync(0xffffffffu, cw, 1);
	cw |= __shfl_xor_sync(0xffffffffu, cw, 2);
	cw |= __shfl_xor_sync(0xffffffffu, cw, 4);
	cw |= (uint32_t(qp0) << kQPlanesOffset) | ((qcode & 0xfu) << kQuantScaleOffset);
	if (max_abs == 0)
		cw = 0;

	// Distortion of dropping every plane (wavelet_quant.comp:253-256).
	float drop;
	{
		float s0 = __fmul_rn(v[0], v[0]);
		s0 = __fmaf_rn(v[1], v[1], s0);
		s0 = __fmaf_rn(v[2], v[2], s0);
		s0 = __fmaf_rn(v[3], v[3], s0);
		float s1 = __fmul_rn(v[4], v[4]);
		s1 = __fmaf_rn(v[5], v[5], s1);
		s1 = __fmaf_rn(v[6], v[6], s1);
		s1 = __fmaf_rn(v[7], v[7], s1);
		drop = __fmul_rn(__fadd_rn(s0, s1), iqs);
		drop = __fadd_rn(drop, __shfl_xor_sync(0xffffffffu, drop, 1));
		drop = __fadd_rn(drop, __shfl_xor_sync(0xffffffffu, drop, 2));
		drop = __fadd_rn(drop, __shfl_xor_sync(0xffffffffu, drop, 4));
		drop = __half2float(__float2half_rn(fminf(60000.0f, drop)));
	}

	// Lane `sub` keeps the 8x8's entries for quant levels i = sub and sub + 8:
	// errors[min(i, num_planes)] of the reference's BlockStats.
	float d_lo = 0.0f, d_hi = drop;
	uint32_t c_lo = (sub == 0) ? uint32_t(csum0) : 0u, c_hi = 0u;
	if (sub != 0 && sub > msb)
		d_lo = drop;

	const int warp_msb = __reduce_max_sync(0xffffffffu, max(msb, 0));
	// Magnitudes as pairs (i, i + 4): the two lanes of a pair accumulate the two
	// halves of the squared error, e0 over i = 0..3 and e1 over i = 4..7, in the
	// same order as eight scalar steps would.
	f32x2 avp[4];
#pragma unroll
	for (int j = 0; j < 4; j++)
		avp[j] = f2_pack(av[j], av[j + 4]);
	for (int q = 1 + r; q <= warp_msb; q += S)
	{
		// compute_square_error + compute_quant_stats at q (wavelet_quant.comp:113-165).
		// R = floor(|v| / 2^q) * 2^q in float arithmetic, exactly: adding
		// M = 2^(23+q) with round-toward-zero keeps the multiples of 2^q (the
		// spacing of floats in [M, 2M), and |v| < 2^15 < M), and subtracting M
		// again is exact. The reconstruction R + 2^(q-1) is an exact integer, so
		// err equals the integer formulation above. With sg = min(R, 1) (1 when
		// significant), err = (|v| - R) - sg * 2^(q-1): the difference and the
		// fused multiply-add are exact, so they round to themselves. The count
		// of significant values is a sum of zeros and ones, exact in any order.
		const float hq = __int_as_float((126 + q) << 23);
		const float mq = __int_as_float((150 + q) << 23);
		const f32x2 mq2 = f2_pack(mq, mq), neg_hq2 = f2_pack(-hq, -hq);
		f32x2 nsig2 = 0ull, e2 = 0ull;
#pragma unroll
		for (int j = 0; j < 4; j++)
		{
			const f32x2 R = f2_sub_rn(f2_add_rz(avp[j], mq2), mq2);
			float r_lo, r_hi;
			f2_unpack(R, r_lo, r_hi);
			const f32x2 sg = f2_pack(fminf(r_lo, 1.0f), fminf(r_hi, 1.0f));
			nsig2 = j == 0 ? sg : f2_add_rn(nsig2, sg);
			const f32x2 err = f2_fma_rn(sg, neg_hq2, f2_sub_rn(avp[j], R));
			e2 = j == 0 ? f2_mul_rn(err, err) : f2_fma_rn(err, err, e2);
		}
		float e0, e1, n_lo, n_hi;
		f2_unpack(e2, e0, e1);
		f2_unpack(nsig2, n_lo, n_hi);
		const int nsig = int(n_lo) + int(n_hi);
		float se = __fmul_rn(__fmul_rn(__fadd_rn(e0, e1), rdo), iqs);
		se = __fadd_rn(se, __shfl_xor_sync(0xffffffffu, se, 1));
		se = __fadd_rn(se, __shfl_xor_sync(0xffffffffu, se, 2));
		se = __fadd_rn(se, __shfl_xor_sync(0xffffffffu, se, 4));

		const int m = msb - q;
		int shifted = block4x2_max >> q;
		int ce = shifted > 0 ? 1 : 0;
		if (m >= 3)
		{
			const int qp = m - 2;
			ce = qp + 1;
			shifted >>= qp;
		}
		ce += find_msb(uint32_t(shifted)) + 1;
		int csum = max(ce - 1, 0) * 8 + nsig;
		csum += __shfl_xor_sync(0xffffffffu, csum, 1);
		csum += __shfl_xor_sync(0xffffffffu, csum, 2);
		csum += __shfl_xor_sync(0xffffffffu, csum, 4);

		if (q <= msb)
		{
			const float d = __half2float(__float2half_rn(fminf(se, 60000.0f)));
			if (q == sub)
			{
				d_lo = d;
				c_lo = uint32_t(csum);
			}
			if (q == sub + 8)
			{
				d_hi = d;
				c_hi = uint32_t(csum);
			}
		}
	}
	if (max_abs == 0)
	{
		d_lo = d_hi = 0.0f;
		c_lo = c_hi = 0u;
	}

	// Per-32x32 sums (analyze_rate_control.comp:169-215): +24 bits per coded
	// 8x8, butterfly over the 16 8x8 blocks in index order lx + 4 * ly.
	if (c_lo != 0)
		c_lo += 24;
	if (c_hi != 0)
		c_hi += 24;
	d_lo = __fadd_rn(d_lo, __shfl_xor_sync(0xffffffffu, d_lo, 8));
	d_lo = __fadd_rn(d_lo, __shfl_xor_sync(0xffffffffu, d_lo, 16));
	d_hi = __fadd_rn(d_hi, __shfl_xor_sync(0xffffffffu, d_hi, 8));
	d_hi = __fadd_rn(d_hi, __shfl_xor_sync(0xffffffffu, d_hi, 16));
	c_lo += __shfl_xor_sync(0xffffffffu, c_lo, 8);
	c_lo += __shfl_xor_sync(0xffffffffu, c_lo, 16);
	c_hi += __shfl_xor_sync(0xffffffffu, c_hi, 8);
	c_hi += __shfl_xor_sync(0xffffffffu, c_hi, 16);
	// The thread that computed level sub (level 0: residue 0) and sub + 8 stores them.
	const bool own_lo = sub == 0 ? r == 0 : (sub - 1) % S == r;
	const bool own_hi = (sub + 7) % S == r;
	if (lane < 8)
	{
		if (own_lo)
		{
			sh.dist[ly][sub] = d_lo;
			sh.cost[ly][sub] = c_lo;
		}
		if (own_hi)
		{
			sh.dist[ly][sub + 8] = d_hi;
			sh.cost[ly][sub + 8] = c_hi;
		}
	}
	if (in_range && sub == 0 && r == 0)
		buf.code_words[B.block8_offset + y8 * B.block8_stride + x8] = cw;
	__syncthreads();

	if (active && t < 16)
	{
		const int i = t;
		const float d = __fadd_rn(__fadd_rn(sh.dist[0][i], sh.dist[1][i]), __fadd_rn(sh.dist[2][i], sh.dist[3][i]));
		uint32_t c = sh.cost[0][i] + sh.cost[1][i] + sh.cost[2][i] + sh.cost[3][i];
		if (c != 0)
			c += 64;
		const uint32_t rate = (c + 31) >> 5;
		const unsigned m16 = 0x0000ffffu;
		const float d0 = __shfl_sync(m16, d, 0);
		const uint32_t r0 = __shfl_sync(m16, rate, 0);
		uint32_t bk = bucket_index(d, float(rate), d0, float(r0));
		if (i == 0)
			bk = 0;
		// inclusive_max_clustered16 (analyze_rate_control.comp:85-99)
		bk = min(bk, uint32_t(128 - 16 + i));
#pragma unroll
		for (int off = 1; off < 16; off *= 2)
		{
			const uint32_t up = __shfl_up_sync(m16, bk, off) + uint32_t(off);
			if (i >= off)
				bk = max(bk, up);
		}
		const uint32_t rate_prev = __shfl_up_sync(m16, rate, 1);
		const uint32_t block_index = uint32_t(B.block32_offset + by32 * B.block32_stride + bx32);
		buf.rd_cost[block_index * 16 + i] = uint16_t(rate);
		buf.rd_bucket[block_index * 16 + i] = uint8_t(bk);
		buf.rd_dist[block_index * 16 + i] = d;
		if (i == 0)
			atomicAdd(&buf.rc->consumed, rate);
		else
		{
			const uint32_t saving = rate_prev - rate;
			if (saving != 0)
			{
				const uint32_t subdivision = block_index >> subdivision_shift;
				atomicAdd(&buf.rc->histogram[bk * kSubdivisions + subdivision], saving);
			}
		}
	}
	__syncthreads();
}

struct DwtShared
{
	int xidx[kTileIn];
	int yidx[kTileIn];
	alignas(128) float in[kTileIn][kInPitch]; // input tile, later the four 32x32 band tiles
	float h[kTileIn][kHPitch];   // after horizontal lifting: low in 0..31, high in 32..63
	QuantGroupShared q[4];
	float unorm[256];            // unorm8_centered(u) for every byte value
	uint64_t tile_bar;           // completion of the TMA tile load
};

__device__ __forceinline__ float unorm8_centered(uint32_t u)
{
	return __fsub_rn(__fdiv_rn(float(u), 255.0f), 0.5f);
}

// Work split of the forward level for a CTA of kThreads threads. Large levels
// run many 256-thread CTAs per SM; the small levels, with fewer tiles than
// SMs, run 1024-thread CTAs that cut every serial phase: shorter lifting
// windows per thread and all bands quantised in one round with two threads per
// 4x2 sub-block.
template <int kThreads> struct DwtSplit
{
	static constexpr int kSegPairs = kThreads >= 1024 ? 4 : 8; // output pairs per lifting item
	static constexpr int kSegs = 32 / kSegPairs;                // items per row / column
	static constexpr int kWin = 2 * kSegPairs + 8;              // lifting window (4 apron samples each side)
	static constexpr int kQSplit = kThreads >= 1024 ? 2 : 1;    // threads per 4x2 sub-block in the quantiser
	static constexpr int kGroupThreads = 128 * kQSplit;         // threads per quantised 32x32 block
	static constexpr int kGroups = kThreads / kGroupThreads;    // 32x32 blocks quantised at once
	static constexpr int kMinBlocks = kThreads >= 1024 ? 1 : (kThreads >= 384 ? 2 : 4); // CTAs per SM to fit
};

// CTA size of the large levels (several CTAs per SM). 384-thread CTAs, which
// quantise the three high bands of a tile in one round, measured no faster.
constexpr int kLargeLevelThreads = 256;

// Tile dataflow: waits (bounded) until every tile of the finer level whose LL
// samples this CTA reads has been stored. The rows and columns read are those
// of the index tables (mirrored at the edges), so the tiles are the ranges
// their minimum and maximum fall in: at most 4 x 4 for a whole tile. Called by
// every thread after the index tables are built; ends with a CTA barrier.
template <int kRowsIn>
__device__ __forceinline__ void wait_finer_tiles(const DwtShared &sh, const LevelParams &p, const EncodeBuffers &buf,
                                                 const int comp, const int r0)
{
	if (threadIdx.x < 32)
	{
		const int lane = threadIdx.x;
		int ylo = 0x7fffffff, yhi = 0, xlo = 0x7fffffff, xhi = 0;
		for (int i = lane; i < kRowsIn; i += 32)
		{
			ylo = min(ylo, sh.yidx[r0 + i]);
			yhi = max(yhi, sh.yidx[r0 + i]);
		}
		for (int i = lane; i < kTileIn; i += 32)
		{
			xlo = min(xlo, sh.xidx[i]);
			xhi = max(xhi, sh.xidx[i]);
		}
		const int ty0 = __reduce_min_sync(0xffffffffu, ylo) >> 5, ty1 = __reduce_max_sync(0xffffffffu, yhi) >> 5;
		const int tx0 = __reduce_min_sync(0xffffffffu, xlo) >> 5, tx1 = __reduce_max_sync(0xffffffffu, xhi) >> 5;
		const int w = tx1 - tx0 + 1, n = w * (ty1 - ty0 + 1);
		const uint32_t *base = buf.tile_done + p.prev_done_offset + comp * p.P.tiles_x * p.P.tiles_y;
		bool ok = true;
		for (int k = lane; k < n && ok; k += 32)
			ok = wait_counter(base + (ty0 + k / w) * p.P.tiles_x + tx0 + k % w, uint32_t(p.prev_parts));
		if (!__all_sync(0xffffffffu, ok) && lane == 0)
			atomicOr(&buf.rc->error, kErrorLevelWait);
	}
	__syncthreads();
}

// One forward level for one 32x32 band tile of one component (64x64 input
// samples): `tile` in row-major tile order, `comp_index` the component among
// those at this level. Run by every thread of a kThreads-thread CTA. With
// kStripes > 1 (transform only) the CTA computes one stripe of 32 / kStripes
// band rows of the tile, one vertical lifting segment: it loads and lifts
// horizontally only the input rows that segment spans.
template <int kThreads, int kStripes = 1>
__device__ __forceinline__ void dwt_forward_body(DwtShared &sh, const LevelParams &p, const PlaneInput &in,
                                                 const EncodeBuffers &buf, const LevelTileMap *maps, const int fused,
                                                 const int tile, const int comp_index, const int stripe = 0)
{
	using Split = DwtSplit<kThreads>;
	static_assert(kStripes == 1 || kStripes == Split::kSegs, "a stripe is one vertical lifting segment");
	// Input rows this CTA loads and lifts horizontally: all 72, or the window of its stripe.
	constexpr int kRowsIn = kStripes == 1 ? kTileIn : Split::kWin;
	const int r0 = kStripes == 1 ? 0 : stripe * 2 * Split::kSegPairs;
	constexpr int kGen = (kRowsIn * kTileIn + kThreads - 1) / kThreads; // gathered loads per thread
	pdl_trigger();
	const int level = p.level;
	const int comp = (level == 0 && !p.chroma444) ? 0 : comp_index;
	const LevelDesc &L = p.L;
	const int tx = tile % L.tiles_x, ty = tile / L.tiles_x;
	const bool from_plane = level == 0 || (level == 1 && comp != 0 && !p.chroma444);

	int res_w, res_h, al_w, al_h;
	if (from_plane)
	{
		res_w = p.plane_width[comp];
		res_h = p.plane_height[comp];
		al_w = level == 0 ? p.aligned_width : p.aligned_width >> 1;
		al_h = level == 0 ? p.aligned_height : p.aligned_height >> 1;
	}
	else
	{
		res_w = al_w = p.P.width;
		res_h = al_h = p.P.height;
	}

	// Tile load. A tile whose 72x72 window lies inside the source maps every
	// sample to itself: an FP32 level above 0 with a tensor map is one TMA box
	// (barrier and map made ready before the dependency wait); otherwise whole
	// rows are read with vector loads, all in flight at once. Edge tiles go
	// through the mirrored index tables in batches of independent loads.
	const int x0 = tx * 64 - 4, y0 = ty * 64 - 4;
	const bool interior = x0 >= 0 && y0 >= 0 && x0 + kTileIn <= res_w && y0 + kTileIn <= res_h;
	const bool use_tma = kStripes == 1 && !from_plane && interior && maps && ((maps->valid >> comp) & 1u) && !p.P.fp16;
	const CUtensorMap *tmap = use_tma ? &maps->map : nullptr;
	constexpr int kVecPerRow = kTileIn / 4;     // 18 vectors of 4 samples
	constexpr int kVecs = kVecPerRow * kRowsIn; // 1296 for a whole tile
	constexpr int kVecIters = (kVecs + kThreads - 1) / kThreads;
	const uint8_t *src = comp == 0 ? in.data[0] : (comp == 1 ? in.data[1] : in.data[2]);
	const int pitch = comp == 0 ? in.pitch[0] : (comp == 1 ? in.pitch[1] : in.pitch[2]);
	const int xs = comp == 0 ? in.xstride[0] : (comp == 1 ? in.xstride[1] : in.xstride[2]);
	const bool vec_ok = from_plane && interior && xs == 1 && !in.sample16 &&
	                    ((reinterpret_cast<uintptr_t>(src) | uintptr_t(pitch)) & 3u) == 0;
	// An interior tile of an 8-bit input plane is read first, before the index
	// tables and before the dependency wait: the planes are complete before the
	// frame's first kernel, so the load latency overlaps the set-up (and, at
	// level 1, the end of level 0).
	uint32_t pv[kVecIters];
	if (vec_ok)
	{
#pragma unroll
		for (int u = 0; u < kVecIters; u++)
		{
			const int k = threadIdx.x + u * kThreads;
			const int ii = k / kVecPerRow, i = r0 + ii, j = k - ii * kVecPerRow;
			pv[u] = k < kVecs ? __ldg(reinterpret_cast<const uint32_t *>(src + size_t(y0 + i) * pitch + x0) + j) : 0u;
		}
	}

	for (int k = threadIdx.x; k < 2 * kTileIn; k += kThreads)
	{
		if (k < kTileIn)
			sh.xidx[k] = fwd_index(tx * 64 - 4 + k, res_w, al_w);
		else
			sh.yidx[k - kTileIn] = fwd_index(ty * 64 - 4 + (k - kTileIn), res_h, al_h);
	}
	if (from_plane)
		for (int u = threadIdx.x; u < 256; u += kThreads)
		{
			const float f = unorm8_centered(uint32_t(u));
			sh.unorm[u] = L.stage16 ? round_to_half(f) : f;
		}
	if (use_tma && threadIdx.x == 0)
	{
		mbarrier_init(&sh.tile_bar, 1);
		prefetch_tensor_map(tmap);
	}
	__syncthreads();
	if (buf.tile_done)
	{
		// Tile dataflow: the input planes are complete before the frame's first
		// kernel; the finer level's LL is read once the tiles it comes from are.
		if (!from_plane)
			wait_finer_tiles<kRowsIn>(sh, p, buf, comp, r0);
	}
	else
		pdl_wait();
	if (from_plane)
	{
		if (in.sample16)
		{
			// 16-bit samples (R16_UNORM): u / 65535 - 0.5, gathered through the index tables.
			for (int base = threadIdx.x; base < kRowsIn * kTileIn; base += kThreads * kGen)
			{
				uint32_t v[kGen];
#pragma unroll
				for (int u = 0; u < kGen; u++)
				{
					const int k = base + u * kThreads;
					const int ii = k / kTileIn, i = r0 + ii, j = k - ii * kTileIn;
					v[u] = k < kRowsIn * kTileIn
					           ? uint32_t(*reinterpret_cast<const uint16_t *>(src + size_t(sh.yidx[i]) * pitch +
					                                                          size_t(sh.xidx[j]) * xs))
					           : 0u;
				}
#pragma unroll
				for (int u = 0; u < kGen; u++)
				{
					const int k = base + u * kThreads;
					if (k < kRowsIn * kTileIn)
					{
						const int ii = k / kTileIn, i = r0 + ii, j = k - ii * kTileIn;
						const float f = __fsub_rn(__fdiv_rn(float(v[u]), 65535.0f), 0.5f);
						sh.in[i][j] = L.stage16 ? round_to_half(f) : f;
					}
				}
			}
		}
		else if (vec_ok)
		{
#pragma unroll
			for (int u = 0; u < kVecIters; u++)
			{
				const int k = threadIdx.x + u * kThreads;
				if (k < kVecs)
				{
					const int ii = k / kVecPerRow, i = r0 + ii, j = k - ii * kVecPerRow;
#pragma unroll
					for (int b = 0; b < 4; b++)
						sh.in[i][4 * j + b] = sh.unorm[(pv[u] >> (8 * b)) & 0xffu];
				}
			}
		}
		else
		{
			for (int base = threadIdx.x; base < kRowsIn * kTileIn; base += kThreads * kGen)
			{
				uint32_t v[kGen];
#pragma unroll
				for (int u = 0; u < kGen; u++)
				{
					const int k = base + u * kThreads;
					const int ii = k / kTileIn, i = r0 + ii, j = k - ii * kTileIn;
					v[u] = k < kRowsIn * kTileIn ? src[size_t(sh.yidx[i]) * pitch + size_t(sh.xidx[j]) * xs] : 0u;
				}
#pragma unroll
				for (int u = 0; u < kGen; u++)
				{
					const int k = base + u * kThreads;
					if (k < kRowsIn * kTileIn)
					{
						const int ii = k / kTileIn, i = r0 + ii, j = k - ii * kTileIn;
						sh.in[i][j] = sh.unorm[v[u] & 0xffu];
					}
				}
			}
		}
	}
	else if (use_tma)
	{
		if (threadIdx.x == 0)
		{
			if (buf.tile_done)
				fence_proxy_async_global(); // LL stored by other CTAs, observed through the counters
			mbarrier_expect_tx(&sh.tile_bar, kInBoxBytes);
			tma_load_2d(&sh.in[0][0], tmap, x0, maps->row[comp][0] + y0, &sh.tile_bar);
		}
		const bool done = mbarrier_wait(&sh.tile_bar, 0, kTmaMaxPolls);
		if (__syncthreads_or(!done))
		{
			// Give up on this tile: record it, and keep the CTA alive (its shared
			// memory is the copy's destination) for one more bounded wait.
			if (threadIdx.x == 0)
				atomicOr(&buf.rc->error, kErrorTileWait);
			(void)mbarrier_wait(&sh.tile_bar, 0, kTmaMaxPolls);
			return;
		}
	}
	else
	{
		const LevelDesc &P = p.P;
		const int64_t ll = comp == 0 ? p.prev_ll[0] : (comp == 1 ? p.prev_ll[1] : p.prev_ll[2]);
		const bool f16 = P.fp16 != 0;
		if (interior)
		{
			float4 v[kVecIters];
#pragma unroll
			for (int u = 0; u < kVecIters; u++)
			{
				const int k = threadIdx.x + u * kThreads;
				const int ii = k / kVecPerRow, i = r0 + ii, j = k - ii * kVecPerRow;
				const int64_t idx = ll + int64_t(y0 + i) * P.pitch + x0 + 4 * j;
				if (k >= kVecs)
					v[u] = make_float4(0.f, 0.f, 0.f, 0.f);
				else if (f16)
				{
					uint2 hv = __ldcg(reinterpret_cast<const uint2 *>(buf.coef16 + idx));
					const float2 a = __half22float2(*reinterpret_cast<__half2 *>(&hv.x));
					const float2 b = __half22float2(*reinterpret_cast<__half2 *>(&hv.y));
					v[u] = make_float4(a.x, a.y, b.x, b.y);
				}
				else
					v[u] = __ldcg(reinterpret_cast<const float4 *>(buf.coef32 + idx));
			}
#pragma unroll
			for (int u = 0; u < kVecIters; u++)
			{
				const int k = threadIdx.x + u * kThreads;
				if (k < kVecs)
				{
					const int ii = k / kVecPerRow, i = r0 + ii, j = k - ii * kVecPerRow;
					*reinterpret_cast<float4 *>(&sh.in[i][4 * j]) = v[u];
				}
			}
		}
		else
		{
			for (int base = threadIdx.x; base < kRowsIn * kTileIn; base += kThreads * kGen)
			{
				float v[kGen];
#pragma unroll
				for (int u = 0; u < kGen; u++)
				{
					const int k = base + u * kThreads;
					const int ii = k / kTileIn, i = r0 + ii, j = k - ii * kTileIn;
					v[u] = k < kRowsIn * kTileIn
					           ? load_coef(buf.coef32, buf.coef16, f16, ll + int64_t(sh.yidx[i]) * P.pitch + sh.xidx[j])
					           : 0.0f;
				}
#pragma unroll
				for (int u = 0; u < kGen; u++)
				{
					const int k = base + u * kThreads;
					if (k < kRowsIn * kTileIn)
					{
						const int ii = k / kTileIn, i = r0 + ii, j = k - ii * kTileIn;
						sh.in[i][j] = v[u];
					}
				}
			}
		}
	}
	__syncthreads();

	// Horizontal lifting: 72 rows (the stripe's 24) x kSegs segments of kSegPairs output pairs.
	constexpr int kSegPairs = Split::kSegPairs, kWin = Split::kWin;
	for (int item = threadIdx.x; item < kRowsIn * Split::kSegs; item += kThreads)
	{
		const int row = r0 + item % kRowsIn, seg = item / kRowsIn;
		float e[kWin];
#pragma unroll
		for (int j = 0; j < kWin; j += 4)
		{
			const float4 q = *reinterpret_cast<const float4 *>(&sh.in[row][seg * 2 * kSegPairs + j]);
			e[j] = q.x;
			e[j + 1] = q.y;
			e[j + 2] = q.z;
			e[j + 3] = q.w;
		}
		lift_forward(e);
#pragma unroll
		for (int k = 0; k < kSegPairs; k++)
		{
			float lo = __fmul_rn(e[4 + 2 * k], kInvK), hi = __fmul_rn(e[5 + 2 * k], kK);
			if (L.stage16)
			{
				lo = round_to_half(lo);
				hi = round_to_half(hi);
			}
			sh.h[row][seg * kSegPairs + k] = lo;
			sh.h[row][32 + seg * kSegPairs + k] = hi;
		}
	}
	__syncthreads();

	// Vertical lifting: 64 columns x kSegs segments. Columns 0..31 hold the
	// horizontal low band (-> LL, LH), 32..63 the high band (-> HL, HH).
	float(*bands)[32][kBandPitch] = reinterpret_cast<float(*)[32][kBandPitch]>(&sh.in[0][0]);
	constexpr int kVSegs = kStripes == 1 ? Split::kSegs : 1;
	for (int item = threadIdx.x; item < 64 * kVSegs; item += kThreads)
	{
		const int col = item & 63, seg = kStripes == 1 ? item >> 6 : stripe;
		float e[kWin];
#pragma unroll
		for (int j = 0; j < kWin; j++)
			e[j] = sh.h[seg * 2 * kSegPairs + j][col];
		lift_forward(e);
		const int c = col & 31;
		const int b_low = col < 32 ? 0 : 1, b_high = col < 32 ? 2 : 3;
		const int gx = tx * 32 + c;
#pragma unroll
		for (int k = 0; k < kSegPairs; k++)
		{
			const int r = seg * kSegPairs + k;
			const int gy = ty * 32 + r;
			float lo = __fmul_rn(e[4 + 2 * k], kInvK);
			float hi = __fmul_rn(e[5 + 2 * k], kK);
			if (gx >= L.width || gy >= L.height)
				lo = hi = 0.0f;
			else if (L.fp16 || L.stage16)
			{
				lo = round_to_half(lo);
				hi = round_to_half(hi);
			}
			bands[b_low][r][c] = lo;
			bands[b_high][r][c] = hi;
		}
	}
	__syncthreads();

	// Store all four bands (LL feeds the next level): 4 x 32 rows (the stripe's rows) x 8 vectors.
	constexpr int kBandRows = 32 / kStripes;
	for (int item = threadIdx.x; item < 4 * kBandRows * 8; item += kThreads)
	{
		const int b = item / (kBandRows * 8), r = stripe * kBandRows + (item >> 3) % kBandRows, c4 = (item & 7) * 4;
		const int64_t idx = p.band[comp][b].offset + int64_t(ty * 32 + r) * L.pitch + tx * 32 + c4;
		if (L.fp16)
		{
			__half2 h0 = __floats2half2_rn(bands[b][r][c4 + 0], bands[b][r][c4 + 1]);
			__half2 h1 = __floats2half2_rn(bands[b][r][c4 + 2], bands[b][r][c4 + 3]);
			uint2 u;
			u.x = *reinterpret_cast<uint32_t *>(&h0);
			u.y = *reinterpret_cast<uint32_t *>(&h1);
			*reinterpret_cast<uint2 *>(buf.coef16 + idx) = u;
		}
		else
		{
			float4 f = make_float4(bands[b][r][c4 + 0], bands[b][r][c4 + 1], bands[b][r][c4 + 2], bands[b][r][c4 + 3]);
			*reinterpret_cast<float4 *>(buf.coef32 + idx) = f;
		}
	}

	if (buf.tile_done)
		cta_count_done(buf.tile_done + p.done_offset + comp * L.tiles_x * L.tiles_y + tile);
	if (kStripes > 1 || !fused)
		return;

	// Quantise the transmitted bands of this tile: HL, LH, HH (+ LL at the last
	// level), kGroups bands per round. With fused == kFusedSplitTail, a last
	// round that would leave groups idle (HH after HL and LH in a 256-thread
	// CTA) instead runs its band on the whole CTA with twice the threads per
	// sub-block: same results, a shorter serial chain for levels of few waves.
	const int first_band = level == kLevels - 1 ? 0 : 1;
	const int nb = 4 - first_band;
	const int grp = threadIdx.x / Split::kGroupThreads, t = threadIdx.x % Split::kGroupThreads;
	bool split_tail = false;
	if constexpr (kThreads == kLargeLevelThreads)
		split_tail = fused == kFusedSplitTail && (nb % Split::kGroups) != 0;
	const int rounds = split_tail ? nb / Split::kGroups : (nb + Split::kGroups - 1) / Split::kGroups;
	for (int round = 0; round < rounds; round++)
	{
		const int bi = round * Split::kGroups + grp;
		const bool active = bi < nb;
		const int band = active ? first_band + bi : first_band;
		quant_analyze_block<Split::kQSplit>(&bands[band][0][0], kBandPitch, active, t, sh.q[grp], L,
		                                    p.band[comp][band], p.subdivision_shift, tx, ty, buf);
	}
	if constexpr (kThreads == kLargeLevelThreads)
	{
		if (split_tail)
		{
			const int band = first_band + rounds * Split::kGroups;
			quant_analyze_block<2 * Split::kQSplit>(&bands[band][0][0], kBandPitch, true, int(threadIdx.x), sh.q[0],
			                                        L, p.band[comp][band], p.subdivision_shift, tx, ty, buf);
		}
	}
	// Tile dataflow: the resolve waits for every fused quantiser (the last
	// round ended with a CTA barrier after its statistics were stored).
	if (buf.tile_done && threadIdx.x == 0)
	{
		__threadfence();
		atomicAdd(&buf.rc->fused_done, 1u);
	}
}

template <int kThreads>
__global__ void __launch_bounds__(kThreads, DwtSplit<kThreads>::kMinBlocks)
    dwt_forward_kernel(const LevelParams p, const PlaneInput in, const EncodeBuffers buf, const int fused,
                       const __grid_constant__ LevelTileMap maps)
{
	__shared__ DwtShared sh;
	dwt_forward_body<kThreads>(sh, p, in, buf, &maps, fused, int(blockIdx.x), int(blockIdx.y));
}

// Small transform-only levels (fewer tiles than SMs): four 256-thread CTAs per
// tile, one per stripe of 8 band rows (blockIdx.x = tile * 4 + stripe). Same
// parameters as dwt_forward_kernel (graph nodes are updated with one argument
// list); the stripes load with plain vector loads, not tensor maps.
constexpr int kDwtStripes = DwtSplit<kLargeLevelThreads>::kSegs;
__global__ void __launch_bounds__(kLargeLevelThreads, 4)
    dwt_stripes_kernel(const LevelParams p, const PlaneInput in, const EncodeBuffers buf, const int fused,
                       const __grid_constant__ LevelTileMap maps)
{
	(void)fused;
	(void)maps;
	__shared__ DwtShared sh;
	dwt_forward_body<kLargeLevelThreads, kDwtStripes>(sh, p, in, buf, nullptr, 0, int(blockIdx.x) / kDwtStripes,
	                                                  int(blockIdx.y), int(blockIdx.x) % kDwtStripes);
}

// Batched form: one CTA per (frame, component, tile) of this level.
template <int kThreads>
__global__ void __launch_bounds__(kThreads, DwtSplit<kThreads>::kMinBlocks)
    dwt_forward_batch_kernel(const BatchFrame *frames, const BatchFrameIO *io, const uint32_t *cta_map, const int level,
                             const int fused, const __grid_constant__ BatchTileMaps maps)
{
	__shared__ LevelParams s_p;
	__shared__ PlaneInput s_in;
	__shared__ EncodeBuffers s_buf;
	int f, local;
	batch_item(cta_map, f, local);
	load_params(s_p, frames[f].lp[level]);
	load_params(s_in, io[f].in);
	load_params(s_buf, frames[f].eb);
	__syncthreads();
	const int ntiles = s_p.L.tiles_x * s_p.L.tiles_y;
	__shared__ DwtShared sh;
	dwt_forward_body<kThreads>(sh, s_p, s_in, s_buf, f < kBatchTileMapFrames ? &maps.frame[f] : nullptr, fused,
	                           local % ntiles, local / ntiles);
}

// Quantiser over a pyramid already in storage (the reference's
// Encoder::encode_pre_transformed, pyrowave_encoder.cpp:1138-1151, and the
// small levels of a frame). G 32x32 blocks per CTA, 128 * S threads each:
// blocks first + item * G + group, those below `end`. `tile` holds G band
// tiles of 32 x kBandPitch floats, `q` G reduction scratches.
template <int S, int G>
__device__ __forceinline__ void quant_blocks_body(const BlockParams &p, const EncodeBuffers &buf, const int first,
                                                  const int end, const int item, float (*tile)[32][kBandPitch],
                                                  QuantGroupShared *q)
{
	constexpr int kGroupThreads = 128 * S;
	pdl_trigger();
	const int grp = threadIdx.x / kGroupThreads, t = threadIdx.x % kGroupThreads;
	const int b = first + item * G + grp;
	const bool active = b < end;
	const int k = active ? find_band(p, b) : 0;
	const BandEntry &E = p.band[k];
	const LevelDesc &L = p.level[E.level];
	const int rel = b - E.block32_offset;
	const int by = rel / E.block32_stride, bx = rel - by * E.block32_stride;
	if (buf.tile_done)
	{
		// Tile dataflow: the block's transform tile is stored once its counter is complete.
		if (active && t == 0 && !wait_counter(buf.tile_done + E.done_index + rel, uint32_t(E.done_parts)))
			atomicOr(&buf.rc->error, kErrorLevelWait);
		__syncthreads();
	}
	else
		pdl_wait();
	if (active)
	{
		// The block's 32 rows as 8 vectors of 4 each, every load in flight at once.
		for (int i = t; i < 256; i += kGroupThreads)
		{
			const int r = i >> 3, c4 = (i & 7) * 4;
			const int64_t idx = E.offset + int64_t(by * 32 + r) * L.pitch + bx * 32 + c4;
			float4 f;
			if (L.fp16)
			{
				const uint2 hv = __ldcg(reinterpret_cast<const uint2 *>(buf.coef16 + idx));
				const float2 a = __half22float2(*reinterpret_cast<const __half2 *>(&hv.x));
				const float2 c = __half22float2(*reinterpret_cast<const __half2 *>(&hv.y));
				f = make_float4(a.x, a.y, c.x, c.y);
			}
			else
				f = __ldcg(reinterpret_cast<const float4 *>(buf.coef32 + idx));
			tile[grp][r][c4 + 0] = f.x;
			tile[grp][r][c4 + 1] = f.y;
			tile[grp][r][c4 + 2] = f.z;
			tile[grp][r][c4 + 3] = f.w;
		}
	}
	__syncthreads();
	BandParam B;
	B.offset = E.offset;
	B.block8_offset = E.block8_offset;
	B.block8_stride = E.block8_stride;
	B.block32_offset = E.block32_offset;
	B.block32_stride = E.block32_stride;
	B.quant_resolution = E.quant_resolution;
	B.rdo_scale = E.rdo_scale;
	B.quant_code = E.quant_code;
	quant_analyze_block<S>(&tile[grp][0][0], kBandPitch, active, t, q[grp], L, B, p.subdivision_shift, bx, by, buf);
}

// One 32x32 block per CTA: the launch follows the last small-level transform
// on the critical path, and one block per CTA is the shortest CTA lifetime
// (the blocks of a frame's small levels fit one wave).
template <int S>
__global__ void __launch_bounds__(128 * S) quant_pretransformed_kernel(const BlockParams p, const EncodeBuffers buf,
                                                                       const int nblocks)
{
	__shared__ float tile[1][32][kBandPitch];
	__shared__ QuantGroupShared q[1];
	quant_blocks_body<S, 1>(p, buf, 0, nblocks, int(blockIdx.x), tile, q);
}

// Batched form: one CTA per pair of blocks among each frame's small-level blocks.
template <int S>
__global__ void __launch_bounds__(256 * S) quant_blocks_batch_kernel(const BatchFrame *frames, const uint32_t *cta_map)
{
	__shared__ BlockParams s_p;
	__shared__ EncodeBuffers s_buf;
	__shared__ float tile[2][32][kBandPitch];
	__shared__ QuantGroupShared q[2];
	int f, local;
	batch_item(cta_map, f, local);
	load_params(s_p, frames[f].bp);
	load_params(s_buf, frames[f].eb);
	__syncthreads();
	quant_blocks_body<S, 2>(s_p, s_buf, 0, frames[f].small_blocks, local, tile, q);
}

// ---------------------------------------------------------------------------
// Block-wide exclusive scan (blockDim.x a multiple of 32, at most 1024);
// returns the exclusive prefix and the block total.
template <typename T> __device__ __forceinline__ T block_exclusive_scan(T v, T *warp_sums, T &total)
{
	const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5, nwarps = blockDim.x >> 5;
	T x = v;
#pragma unroll
	for (int off = 1; off < 32; off *= 2)
	{
		const T y = __shfl_up_sync(0xffffffffu, x, off);
		if (lane >= off)
			x += y;
	}
	if (lane == 31)
		warp_sums[warp] = x;
	__syncthreads();
	if (warp == 0)
	{
		T s = lane < nwarps ? warp_sums[lane] : T(0);
#pragma unroll
		for (int off = 1; off < 32; off *= 2)
		{
			const T y = __shfl_up_sync(0xffffffffu, s, off);
			if (lane >= off)
				s += y;
		}
		warp_sums[lane] = s;
	}
	__syncthreads();
	const T base = warp == 0 ? T(0) : warp_sums[warp - 1];
	total = warp_sums[nwarps - 1];
	__syncthreads();
	return base + x - v;
}

// The RD row of one 32x32 block as stored: 16 u16 word counts (quant 0..15)
// and 16 u8 buckets, 48 bytes in three 16-byte loads.
struct RawRD
{
	uint4 c0, c1, bb;
};

__device__ __forceinline__ RawRD load_raw_rd(const EncodeBuffers &buf, int blk)
{
	RawRD r;
	r.c0 = __ldcg(reinterpret_cast<const uint4 *>(buf.rd_cost + size_t(blk) * 16));
	r.c1 = __ldcg(reinterpret_cast<const uint4 *>(buf.rd_cost + size_t(blk) * 16) + 1);
	r.bb = __ldcg(reinterpret_cast<const uint4 *>(buf.rd_bucket + size_t(blk) * 16));
	return r;
}

__device__ __forceinline__ uint32_t u4_word(const uint4 &v, int i)
{
	return i == 0 ? v.x : (i == 1 ? v.y : (i == 2 ? v.z : v.w));
}

// Word count at quant l (l is a compile-time index after unrolling).
__device__ __forceinline__ uint32_t rd_cost_at(const RawRD &r, int l)
{
	const uint32_t w = l < 8 ? u4_word(r.c0, l >> 1) : u4_word(r.c1, (l - 8) >> 1);
	return (w >> (16 * (l & 1))) & 0xffffu;
}

__device__ __forceinline__ uint32_t rd_bucket_at(const RawRD &r, int l)
{
	return (u4_word(r.bb, l >> 2) >> (8 * (l & 3))) & 0xffu;
}

// Saving of the block's RD operation in bucket bk (0 if none). Buckets of one
// block strictly increase with the step, so at most one step matches.
__device__ __forceinline__ uint32_t op_saving_at_bucket(const RawRD &r, uint32_t bk)
{
	uint32_t sv = 0;
#pragma unroll
	for (int l = 1; l < 16; l++)
		if (rd_bucket_at(r, l) == bk)
			sv = rd_cost_at(r, l - 1) - rd_cost_at(r, l);
	return sv;
}

// Quant of a block: its largest applied RD step. Steps are applied when their
// (bucket, subdivision) slot precedes x*, or equals it and the block precedes the cut.
__device__ __forceinline__ uint32_t block_words(const RawRD &r, int blk, int sdiv, int xstar, uint32_t cut, int &q)
{
	q = 0;
	uint32_t words = rd_cost_at(r, 0);
#pragma unroll
	for (int l = 1; l < 16; l++)
	{
		const uint32_t cost = rd_cost_at(r, l);
		const uint32_t saving = rd_cost_at(r, l - 1) - cost;
		const int x = int(rd_bucket_at(r, l)) * kSubdivisions + sdiv;
		if (saving != 0 && (x < xstar || (x == xstar && uint32_t(blk) < cut)))
		{
			q = l;
			words = cost;
		}
	}
	return words;
}

// Exact-rate resolve (analyze_rate_control_finalize.comp + resolve_rate_control.comp).
//
// The reference walks all 2048 (bucket, subdivision) slots; for each slot with
// savings it applies RD operations in block order while the running saving
// stays below need - savings_of_earlier_slots. Every slot before the first slot
// x* whose inclusive prefix reaches `need` is applied in full, slots after x*
// not at all, and x* up to the first operation whose exclusive prefix reaches
// its requirement (the cut).
//
// The blocks are split into slices of consecutive blocks, one 1024-thread CTA
// each. Every CTA scans the histogram for x* itself; a CTA whose slice meets
// the x* subdivision also finds the cut (from the savings of that subdivision
// up to the end of its slice). It then gives its blocks their quant (the
// largest applied step), word counts and offsets: the slice's own scan plus
// the totals the preceding slices publish.
constexpr int kOwnBatch = 2;           // RD rows per thread with their loads in flight together
constexpr int kSliceWaitSpins = 1 << 20; // bounded wait for one preceding slice's total

// Calls f(blk, row) for blocks [b0, b1) in order, the first kOwnBatch rows from
// `first`, the rest loaded kOwnBatch at a time.
template <typename F>
__device__ __forceinline__ void for_rows(const EncodeBuffers &buf, int b0, int b1, const RawRD (&first)[kOwnBatch],
                                         F f)
{
#pragma unroll
	for (int i = 0; i < kOwnBatch; i++)
		if (b0 + i < b1)
			f(b0 + i, first[i]);
	for (int base = b0 + kOwnBatch; base < b1; base += kOwnBatch)
	{
		RawRD r[kOwnBatch];
#pragma unroll
		for (int i = 0; i < kOwnBatch; i++)
			if (base + i < b1)
				r[i] = load_raw_rd(buf, base + i);
#pragma unroll
		for (int i = 0; i < kOwnBatch; i++)
			if (base + i < b1)
				f(base + i, r[i]);
	}
}

__device__ __forceinline__ void load_rows(const EncodeBuffers &buf, int b0, int b1, RawRD (&r)[kOwnBatch])
{
#pragma unroll
	for (int i = 0; i < kOwnBatch; i++)
		if (b0 + i < b1)
			r[i] = load_raw_rd(buf, b0 + i);
}

// Tile dataflow: the forward levels with a fused quantiser may still run when
// the resolve starts (its wait covers only the launch before it); wait, bounded,
// until each has counted its quantiser finished. Called by every thread.
__device__ __forceinline__ void wait_fused_quantisers(const ResolveParams &p, RateControlState *rc)
{
	if (p.fused_ctas == 0)
		return;
	if (threadIdx.x == 0 && !wait_counter(&rc->fused_done, p.fused_ctas))
		atomicOr(&rc->error, kErrorLevelWait);
	__syncthreads();
}

__device__ __forceinline__ void resolve_body(const ResolveParams &p, const EncodeBuffers &buf, const int slice,
                                             const int nslices)
{
	__shared__ uint32_t scan[kHistSize];
	__shared__ uint32_t warp_sums[32];
	__shared__ unsigned long long warp_sums64[32];
	__shared__ int s_xstar;
	__shared__ uint32_t s_cut;
	__shared__ unsigned long long s_base;
	RateControlState *rc = buf.rc;
	const int t = threadIdx.x, nthreads = blockDim.x;
	const int nblocks = p.block_count_32x32;
	// Slices are rate-control subdivisions, or 1024-block parts of larger
	// ones: only the slices of the x* subdivision depend on the cut.
	const int slice_blocks = resolve_slice_blocks(nblocks, p.blocks_per_subdivision);
	const int s0 = min(slice * slice_blocks, nblocks), s1 = min(s0 + slice_blocks, nblocks);
	const int per = (s1 - s0 + nthreads - 1) / nthreads;
	const int b0 = min(s0 + t * per, s1), b1 = min(b0 + per, s1);
	// Every quantiser has finished once the wait returns (with the tile dataflow,
	// the fused ones once their count is complete). The packer is released only
	// then, because it reads their output before its own wait.
	pdl_wait();
	wait_fused_quantisers(p, rc);
	pdl_trigger();

	RawRD own[kOwnBatch];
	load_rows(buf, b0, b1, own);
	// The histogram: kHistSize / nthreads consecutive slots per thread.
	const int hper = kHistSize / nthreads, h0 = t * hper;
	uint32_t hv[kHistSize / 256];
	uint32_t hsum = 0;
#pragma unroll
	for (int i = 0; i < kHistSize / 256; i++)
		if (i < hper)
		{
			hv[i] = __ldcg(&rc->histogram[h0 + i]);
			hsum += hv[i];
		}
	const uint32_t consumed = __ldcg(&rc->consumed);
	if (t == 0)
	{
		s_xstar = -1;
		s_cut = 0xffffffffu;
	}
	uint32_t total;
	uint32_t run = block_exclusive_scan(hsum, warp_sums, total);
#pragma unroll
	for (int i = 0; i < kHistSize / 256; i++)
		if (i < hper)
		{
			run += hv[i];
			scan[h0 + i] = run;
		}
	__syncthreads();

	const int64_t need = int64_t(consumed) - int64_t(p.target_words);
	if (need > 0)
	{
		for (int x = h0; x < h0 + hper; x++)
			if (int64_t(scan[x]) >= need && (x == 0 || int64_t(scan[x - 1]) < need))
				s_xstar = x;
	}
	__syncthreads();
	const int xstar = s_xstar;

	const int start = xstar >= 0 ? (xstar & (kSubdivisions - 1)) * p.blocks_per_subdivision : 0;
	const int end = xstar >= 0 ? min(start + p.blocks_per_subdivision, nblocks) : 0;
	if (xstar >= 0 && s0 < end && s1 > start)
	{
		// The cut, as far as this slice needs it: scan the savings at bucket b*
		// of the x* subdivision's blocks up to the end of the slice.
		const int64_t required = need - (xstar > 0 ? int64_t(scan[xstar - 1]) : 0);
		const uint32_t bk = uint32_t(xstar >> 4);
		const int c1 = min(end, s1);
		const int cper = (c1 - start + nthreads - 1) / nthreads;
		const int c0 = min(start + t * cper, c1), c0e = min(c0 + cper, c1);
		RawRD r0[kOwnBatch];
		load_rows(buf, c0, c0e, r0);
		uint32_t local = 0;
		for_rows(buf, c0, c0e, r0, [&](int, const RawRD &r) { local += op_saving_at_bucket(r, bk); });
		uint32_t tot;
		uint32_t ex = block_exclusive_scan(local, warp_sums, tot);
		bool found = false;
		for_rows(buf, c0, c0e, r0, [&](int blk, const RawRD &r) {
			const uint32_t sv = op_saving_at_bucket(r, bk);
			if (!found && sv != 0 && int64_t(ex) >= required)
			{
				atomicMin(&s_cut, uint32_t(blk));
				found = true;
			}
			ex += sv;
		});
		__syncthreads();
	}
	const uint32_t cut = s_cut;

	// Word counts of this thread's run, the slice scan, then the slice's base
	// from the totals of the preceding slices.
	unsigned long long local = 0; // words << 32 | non-empty blocks << 1
	for_rows(buf, b0, b1, own, [&](int blk, const RawRD &r) {
		int q;
		const uint32_t w = block_words(r, blk, blk >> p.subdivision_shift, xstar, cut, q);
		local += (uint64_t(w) << 32) | (uint64_t(w != 0 ? 1 : 0) << 1);
	});
	unsigned long long slice_sum;
	const unsigned long long run_excl = block_exclusive_scan(local, warp_sums64, slice_sum);
	if (t == 0)
		st_release_u64(&rc->slice_total[slice], slice_sum | 1ull);
	unsigned long long pred = 0;
	if (t < slice)
	{
		// Every slice CTA is resident (the grid is at most kMaxResolveSlices
		// CTAs and the packer launches only after all of them started), so the
		// wait ends; it is bounded all the same.
		unsigned long long v;
		int spins = 0;
		while (((v = ld_acquire_u64(&rc->slice_total[t])) & 1ull) == 0ull)
		{
			if (++spins > kSliceWaitSpins)
			{
				atomicOr(&rc->error, kErrorSliceWait);
				v = 1ull;
				break;
			}
			__nanosleep(64);
		}
		pred = v & ~1ull;
	}
	unsigned long long base_total;
	(void)block_exclusive_scan(pred, warp_sums64, base_total);
	if (t == 0)
		s_base = base_total;
	__syncthreads();
	unsigned long long pos = s_base + run_excl;
	for_rows(buf, b0, b1, own, [&](int blk, const RawRD &r) {
		int q;
		const uint32_t w = block_words(r, blk, blk >> p.subdivision_shift, xstar, cut, q);
		buf.quant[blk] = q;
		*reinterpret_cast<uint2 *>(buf.block_meta + 2 * size_t(blk)) = make_uint2(uint32_t(pos >> 32), w);
		pos += uint64_t(w) << 32;
	});

	if (t == 0 && slice == nslices - 1)
	{
		const unsigned long long all = s_base + slice_sum;
		const uint32_t total_words = uint32_t(all >> 32);
		const uint32_t non_zero = uint32_t(all & 0xffffffffull) >> 1;
		rc->xstar = xstar;
		rc->sequence = p.sequence & 7u;
		rc->total_words = total_words;
		rc->non_zero_blocks = non_zero;
		if (2 + uint64_t(total_words) > buf.stream_capacity_words)
			atomicOr(&rc->error, kErrorStreamCapacity);
		// Start-of-frame sequence header (bitstream.md:250-265).
		buf.stream[0] = uint32_t(p.width - 1) | (uint32_t(p.height - 1) << 14) | ((p.sequence & 7u) << 28) | (1u << 31);
		buf.stream[1] = (non_zero & 0xffffffu) | (uint32_t(p.chroma444 ? 1 : 0) << 26);
	}
}

template <int kThreads>
__global__ void __launch_bounds__(kThreads) resolve_kernel(const ResolveParams p, const EncodeBuffers buf)
{
	resolve_body(p, buf, int(blockIdx.x), int(gridDim.x));
}

// The same resolve on one thread-block cluster of C CTAs (C a power of two up
// to 16), for frames of at most C * 1024 * R blocks: thread g = rank * 1024 + t
// owns the run of at most R consecutive blocks from g * R', R' = ceil(blocks /
// (C * 1024)), its RD rows loaded once into registers. Every CTA scans the
// whole histogram itself (8 KB), so all of them find x* and the requirement
// with no exchange. The cut and the offsets need prefixes across CTAs: each
// CTA writes its totals into the shared memory of every higher-ranked CTA
// (distributed shared memory) and a hardware cluster barrier publishes them:
// once for the offsets, and once for the cut unless the x* subdivision lies
// inside one CTA. An operation at the x* slot is applied when the exclusive
// prefix of the x* subdivision's savings before its block is below the
// requirement, which is the same set as the blocks before the cut. Results are
// those of resolve_body.
constexpr int kClusterResolveThreads = 1024;
constexpr int kMaxResolveCluster = 16;

template <int R>
__global__ void __launch_bounds__(kClusterResolveThreads, 1)
    resolve_cluster_kernel(const ResolveParams p, const EncodeBuffers buf)
{
	__shared__ uint32_t scan[kHistSize];
	__shared__ uint32_t warp_sums[32];
	__shared__ unsigned long long warp_sums64[32];
	__shared__ int s_xstar;
	__shared__ unsigned long long s_saving_totals[kMaxResolveCluster]; // [r]: savings total of rank r < this rank
	__shared__ unsigned long long s_word_totals[kMaxResolveCluster];   // [r]: words << 32 | non-empty << 1 of rank r
	// Peers write into this CTA's shared memory only after every CTA started.
	cluster_arrive_relaxed();
	RateControlState *rc = buf.rc;
	const int t = threadIdx.x;
	const uint32_t rank = cluster_rank(), ncta = cluster_size();
	const int n = p.block_count_32x32;
	const int per = (n + int(ncta) * kClusterResolveThreads - 1) / (int(ncta) * kClusterResolveThreads); // <= R
	const int b0 = min((int(rank) * kClusterResolveThreads + t) * per, n), b1 = min(b0 + per, n);
	pdl_wait();
	wait_fused_quantisers(p, rc);
	pdl_trigger();

	RawRD rows[R];
#pragma unroll
	for (int i = 0; i < R; i++)
		if (b0 + i < b1)
			rows[i] = load_raw_rd(buf, b0 + i);
	static_assert(kHistSize == 2 * kClusterResolveThreads, "two histogram slots per thread");
	const uint32_t h0 = __ldcg(&rc->histogram[2 * t]), h1 = __ldcg(&rc->histogram[2 * t + 1]);
	const uint32_t consumed = __ldcg(&rc->consumed);
	if (t == 0)
		s_xstar = -1;
	uint32_t total;
	const uint32_t run = block_exclusive_scan(h0 + h1, warp_sums, total);
	scan[2 * t] = run + h0;
	scan[2 * t + 1] = run + h0 + h1;
	__syncthreads();

	const int64_t need = int64_t(consumed) - int64_t(p.target_words);
	if (need > 0)
	{
		for (int x = 2 * t; x < 2 * t + 2; x++)
			if (int64_t(scan[x]) >= need && (x == 0 || int64_t(scan[x - 1]) < need))
				s_xstar = x;
	}
	__syncthreads();
	const int xstar = s_xstar; // the same in every CTA: each scanned the same histogram
	cluster_wait();

	// Which of this thread's blocks apply their operation at the x* slot.
	bool apply_x[R];
#pragma unroll
	for (int i = 0; i < R; i++)
		apply_x[i] = false;
	if (xstar >= 0)
	{
		const int start = (xstar & (kSubdivisions - 1)) * p.blocks_per_subdivision;
		const int end = min(start + p.blocks_per_subdivision, n);
		const int64_t required = need - (xstar > 0 ? int64_t(scan[xstar - 1]) : 0);
		const uint32_t bk = uint32_t(xstar >> 4);
		uint32_t sv[R];
		uint32_t local = 0;
#pragma unroll
		for (int i = 0; i < R; i++)
		{
			const int blk = b0 + i;
			sv[i] = (blk < b1 && blk >= start && blk < end) ? op_saving_at_bucket(rows[i], bk) : 0u;
			local += sv[i];
		}
		uint32_t cta_total;
		uint32_t ex = block_exclusive_scan(local, warp_sums, cta_total);
		// When the x* subdivision lies inside one CTA's blocks (every CTA sees
		// the same x*, so all take the same branch), the other CTAs hold none of
		// its savings and the prefix needs no exchange.
		const int cta_blocks = per * kClusterResolveThreads;
		uint64_t base = 0;
		if (start / cta_blocks != (end - 1) / cta_blocks)
		{
			if (t < int(ncta) && t > int(rank))
				st_cluster_u64(&s_saving_totals[rank], uint32_t(t), cta_total);
			cluster_sync();
			for (uint32_t r = 0; r < rank; r++)
				base += s_saving_totals[r];
		}
#pragma unroll
		for (int i = 0; i < R; i++)
		{
			apply_x[i] = sv[i] != 0 && int64_t(base + ex) < required;
			ex += sv[i];
		}
	}

	// Word counts, the cluster-wide scan of offsets, the per-block decisions.
	uint32_t w[R];
	int q[R];
	unsigned long long local = 0; // words << 32 | non-empty blocks << 1
#pragma unroll
	for (int i = 0; i < R; i++)
	{
		const int blk = b0 + i;
		w[i] = 0;
		q[i] = 0;
		if (blk < b1)
		{
			// Operations before the x* slot, plus the one at it where applied.
			w[i] = block_words(rows[i], blk, blk >> p.subdivision_shift, xstar, apply_x[i] ? 0xffffffffu : 0u, q[i]);
			local += (uint64_t(w[i]) << 32) | (uint64_t(w[i] != 0 ? 1 : 0) << 1);
		}
	}
	unsigned long long cta_words;
	unsigned long long pos = block_exclusive_scan(local, warp_sums64, cta_words);
	if (t < int(ncta) && t > int(rank))
		st_cluster_u64(&s_word_totals[rank], uint32_t(t), cta_words);
	cluster_sync();
	unsigned long long base = 0;
	for (uint32_t r = 0; r < rank; r++)
		base += s_word_totals[r];
	pos += base;
#pragma unroll
	for (int i = 0; i < R; i++)
	{
		const int blk = b0 + i;
		if (blk < b1)
		{
			buf.quant[blk] = q[i];
			*reinterpret_cast<uint2 *>(buf.block_meta + 2 * size_t(blk)) = make_uint2(uint32_t(pos >> 32), w[i]);
			pos += uint64_t(w[i]) << 32;
		}
	}
	if (t == 0 && rank == ncta - 1)
	{
		const unsigned long long all = base + cta_words;
		const uint32_t total_words = uint32_t(all >> 32);
		const uint32_t non_zero = uint32_t(all & 0xffffffffull) >> 1;
		rc->xstar = xstar;
		rc->sequence = p.sequence & 7u;
		rc->total_words = total_words;
		rc->non_zero_blocks = non_zero;
		if (2 + uint64_t(total_words) > buf.stream_capacity_words)
			atomicOr(&rc->error, kErrorStreamCapacity);
		// Start-of-frame sequence header (bitstream.md:250-265).
		buf.stream[0] = uint32_t(p.width - 1) | (uint32_t(p.height - 1) << 14) | ((p.sequence & 7u) << 28) | (1u << 31);
		buf.stream[1] = (non_zero & 0xffffffu) | (uint32_t(p.chroma444 ? 1 : 0) << 26);
	}
}

// Batched form: one CTA per (frame, slice).
__global__ void __launch_bounds__(kResolveBatchThreads) resolve_batch_kernel(const BatchFrame *frames, const BatchFrameIO *io,
                                                             const uint32_t *cta_map)
{
	__shared__ ResolveParams s_p;
	__shared__ EncodeBuffers s_buf;
	int f, local;
	batch_item(cta_map, f, local);
	load_params(s_p, io[f].rp);
	load_params(s_buf, frames[f].eb);
	__syncthreads();
	resolve_body(s_p, s_buf, local, frames[f].slices);
}

// ---------------------------------------------------------------------------
// Block packing: one 32x32 block per 128-thread CTA, assembled in shared
// memory and written as whole words at its prefix-scanned offset.
struct PackShared
{
	uint32_t pkt[kMaxBlockWords];
	uint32_t s_ballot[4];
	uint32_t s_bytes[16];
	uint32_t s_sig[4];
};

// One 32x32 block on a group of 128 / kSubs threads: with kSubs = 1 the group
// is threadIdx.x & 127, synchronised with hardware barrier `bar`; with kSubs =
// 2 the whole 64-thread CTA, each thread packing the sub-blocks of 8x8 rows ly
// and ly + 2.
template <int kSubs = 1>
__device__ __forceinline__ void pack_body(PackShared &sh, const BlockParams &p, const EncodeBuffers &buf, const int blk,
                                          const int bar)
{
	static_assert(kSubs == 1 || kSubs == 2, "one or two sub-blocks per thread");
	constexpr int kGroup = 128 / kSubs;
	constexpr int kRowStep = 4 / kSubs;
	uint32_t *const pkt = sh.pkt;
	uint32_t *const s_ballot = sh.s_ballot;
	uint32_t *const s_bytes = sh.s_bytes;
	uint32_t *const s_sig = sh.s_sig;
	pdl_trigger();
	const int k = find_band(p, blk);
	const BandEntry &B = p.band[k];
	const LevelDesc &L = p.level[B.level];
	const int rel = blk - B.block32_offset;
	const int by32 = rel / B.block32_stride, bx32 = rel - by32 * B.block32_stride;
	const int t = threadIdx.x & (kGroup - 1), lane = t & 31;
	const int sub = t & 7, lx = (t >> 3) & 3, ly0 = t >> 5;
	const int x8 = bx32 * 4 + lx;

	// The resolve kernel releases this grid only after every quantiser has
	// finished, so the quantised magnitudes and code words can be fetched before
	// the wait; only the rate-control decisions come from the resolve kernel itself.
	uint32_t cw0[kSubs];
	uint4 sm[kSubs];
#pragma unroll
	for (int h = 0; h < kSubs; h++)
	{
		const int ly = ly0 + h * kRowStep, y8 = by32 * 4 + ly;
		const bool in_range = x8 < L.blocks8_x && y8 < L.blocks8_y;
		cw0[h] = in_range ? __ldcg(&buf.code_words[B.block8_offset + y8 * B.block8_stride + x8]) : 0u;
		sm[h] = __ldcg(reinterpret_cast<const uint4 *>(buf.mag16 + int64_t(blk) * 1024 + 8 * (sub + 8 * lx + 32 * ly)));
	}
	pdl_wait();

	const uint2 meta = __ldcg(reinterpret_cast<const uint2 *>(buf.block_meta) + blk);
	const int quant = __ldcg(&buf.quant[blk]);
	const uint32_t words = meta.y;
	if (words == 0)
		return;
	const uint32_t offset = meta.x;

	// The thread's sub-blocks as the quantiser scaled them (sign-magnitude).
	uint32_t cw[kSubs], mag[kSubs][8], neg[kSubs], planes[kSubs], sig[kSubs];
	bool active[kSubs];
#pragma unroll
	for (int h = 0; h < kSubs; h++)
	{
		cw[h] = quantize_code_word(cw0[h], quant);
		active[h] = (cw[h] & 0xffffu) != 0;
		const uint32_t w[4] = {sm[h].x, sm[h].y, sm[h].z, sm[h].w};
		neg[h] = 0;
#pragma unroll
		for (int i = 0; i < 8; i++)
		{
			const uint32_t x = (w[i >> 1] >> (16 * (i & 1))) & 0xffffu;
			mag[h][i] = x & 0x7fffu;
			neg[h] |= (x >> 15) << i;
		}
		const uint32_t out_q = (cw[h] >> kQPlanesOffset) & 0xfu;
		planes[h] = active[h] ? ((cw[h] >> (2 * sub)) & 3u) + out_q : 0u;
		sig[h] = 0;
		if (planes[h] != 0)
		{
#pragma unroll
			for (int i = 0; i < 8; i++)
				if ((mag[h][i] >> quant) != 0)
					sig[h] |= 1u << i;
		}
	}

	// Per 8x8 row (one warp per row): the ballot of coded 8x8s, their plane
	// bytes, and the inclusive prefix of significant coefficients.
	uint32_t nsig[kSubs], inc[kSubs], sub_plane_offset[kSubs];
#pragma unroll
	for (int h = 0; h < kSubs; h++)
	{
		const int ly = ly0 + h * kRowStep, grp = ly * 4 + lx;
		const uint32_t wb = __ballot_sync(0xffffffffu, active[h] && sub == 0);
		if (lane == 0)
			s_ballot[ly] = ((wb >> 0) & 1u) | ((wb >> 7) & 2u) | ((wb >> 14) & 4u) | ((wb >> 21) & 8u);
		if (sub == 0)
			s_bytes[grp] = required_8x8_bytes(cw[h]);
		nsig[h] = uint32_t(__popc(sig[h]));
		inc[h] = nsig[h];
#pragma unroll
		for (int off = 1; off < 32; off *= 2)
		{
			const uint32_t y = __shfl_up_sync(0xffffffffu, inc[h], off);
			if (lane >= off)
				inc[h] += y;
		}
		if (lane == 31)
			s_sig[ly] = inc[h];
		// Exclusive prefix of plane bytes over the 8 sub-blocks of this 8x8.
		uint32_t pinc = planes[h];
#pragma unroll
		for (int off = 1; off < 8; off *= 2)
		{
			const uint32_t y = __shfl_up_sync(0xffffffffu, pinc, off);
			if (sub >= off)
				pinc += y;
		}
		sub_plane_offset[h] = pinc - planes[h];
	}
	for (int w = t; w < int(words) && w < kMaxBlockWords; w += kGroup)
		pkt[w] = 0u;
	block_sync<kSubs>(bar);

	const uint32_t ballot = s_ballot[0] | (s_ballot[1] << 4) | (s_ballot[2] << 8) | (s_ballot[3] << 12);
	const uint32_t n = uint32_t(__popc(ballot));
	// Plane bytes before each 8x8 and in total: a 16-lane inclusive scan in every warp.
	uint32_t scan_bytes = s_bytes[lane & 15];
#pragma unroll
	for (int off = 1; off < 16; off *= 2)
	{
		const uint32_t y = __shfl_up_sync(0xffffffffu, scan_bytes, off, 16);
		if ((lane & 15) >= off)
			scan_bytes += y;
	}
	const uint32_t total_bytes = __shfl_sync(0xffffffffu, scan_bytes, 15);
	const uint32_t total_sig = s_sig[0] + s_sig[1] + s_sig[2] + s_sig[3];

	uint8_t *bytes = reinterpret_cast<uint8_t *>(pkt);
	if (t == 0)
	{
		pkt[0] = (ballot & 0xffffu) | (words << 16) | ((__ldcg(&buf.rc->sequence) & 7u) << 28);
		pkt[1] = modify_quant_code(B.quant_code, quant) | (uint32_t(blk) << 8);
	}
	uint32_t sig_excl[kSubs];
#pragma unroll
	for (int h = 0; h < kSubs; h++)
	{
		const int ly = ly0 + h * kRowStep, grp = ly * 4 + lx;
		const uint32_t excl_bytes = __shfl_sync(0xffffffffu, scan_bytes, grp) - s_bytes[grp];
		uint32_t sig_base = 0;
		for (int w = 0; w < ly; w++)
			sig_base += s_sig[w];
		sig_excl[h] = sig_base + inc[h] - nsig[h];
		if (active[h] && sub == 0)
		{
			const uint32_t compact = uint32_t(__popc(ballot & ((1u << grp) - 1u)));
			bytes[8 + 2 * compact + 0] = uint8_t(cw[h]);
			bytes[8 + 2 * compact + 1] = uint8_t(cw[h] >> 8);
			bytes[8 + 2 * n + compact] = uint8_t(cw[h] >> 16);
		}
		const uint32_t plane_base = 8 + 3 * n + excl_bytes + sub_plane_offset[h];
		if (planes[h] != 0)
		{
			// Bit plane k of the 8 magnitudes is byte k of the transposed bit matrix
			// whose byte i holds the magnitude of coefficient i (low and high 8 bits).
			unsigned long long lo = 0, hi = 0;
#pragma unroll
			for (int i = 0; i < 8; i++)
			{
				lo |= (unsigned long long)(mag[h][i] & 0xffu) << (8 * i);
				hi |= (unsigned long long)((mag[h][i] >> 8) & 0xffu) << (8 * i);
			}
			lo = transpose8x8(lo);
			hi = transpose8x8(hi);
			for (uint32_t pl = 0; pl < planes[h]; pl++)
			{
				const uint32_t bit = uint32_t(quant) + planes[h] - 1u - pl; // most significant plane first
				const uint32_t by = bit < 8 ? uint32_t(lo >> (8 * bit)) : (bit < 16 ? uint32_t(hi >> (8 * (bit - 8))) : 0u);
				if (plane_base + pl < uint32_t(kMaxBlockWords) * 4)
					bytes[plane_base + pl] = uint8_t(by);
			}
		}
	}
	block_sync<kSubs>(bar);

	// Sign bits of significant coefficients, in coefficient order, after the planes.
	// A sub-block's sign bits are consecutive in the stream: gather them (sign
	// of each significant coefficient, in order) and OR them in with at most two
	// word updates.
#pragma unroll
	for (int h = 0; h < kSubs; h++)
	{
		const uint32_t bitpos = (8 + 3 * n + total_bytes) * 8 + sig_excl[h];
		uint32_t bits = 0;
		int kk = 0;
#pragma unroll
		for (int i = 0; i < 8; i++)
		{
			if ((sig[h] >> i) & 1u)
			{
				bits |= ((neg[h] >> i) & 1u) << kk;
				kk++;
			}
		}
		const uint32_t w = bitpos >> 5, shift = bitpos & 31u;
		if (bits != 0 && w < uint32_t(kMaxBlockWords))
		{
			atomicOr(&pkt[w], bits << shift);
			if (shift != 0 && (bits >> (32u - shift)) != 0 && w + 1 < uint32_t(kMaxBlockWords))
				atomicOr(&pkt[w + 1], bits >> (32u - shift));
		}
	}
	block_sync<kSubs>(bar);

	// The word count must match the rate-control estimate the offsets were built from.
	const uint32_t bits = 8 * (3 * n + total_bytes) + total_sig;
	const uint32_t expect = (bits + 31) / 32 + 2;
	const bool fits = words <= uint32_t(kMaxBlockWords) && 2 + offset + words <= buf.stream_capacity_words;
	if (t == 0 && (expect != words || !fits))
		atomicOr(&buf.rc->error, kErrorWordCount);
	if (!fits)
		return;
	uint32_t *dst = buf.stream + 2 + offset;
	for (int w = t; w < int(words); w += kGroup)
		dst[w] = pkt[w];
}

// One 32x32 block per 64-thread CTA, two sub-blocks per thread, registers
// bounded for 23 CTAs per SM: about twice the blocks resident per SM of
// 128-thread CTAs (a 1080p frame's 3261 blocks in one wave).
constexpr int kPackThreads = 64;
__global__ void __launch_bounds__(kPackThreads, 23) pack_kernel(const BlockParams p, const EncodeBuffers buf)
{
	__shared__ PackShared sh;
	pack_body<128 / kPackThreads>(sh, p, buf, int(blockIdx.x), 1);
}

// Batched form: one CTA per (frame, block).
__global__ void __launch_bounds__(128, 12) pack_batch_kernel(const BatchFrame *frames, const uint32_t *cta_map)
{
	__shared__ BlockParams s_p;
	__shared__ EncodeBuffers s_buf;
	int f, local;
	batch_item(cta_map, f, local);
	load_params(s_p, frames[f].bp);
	load_params(s_buf, frames[f].eb);
	__syncthreads();
	__shared__ PackShared sh;
	pack_body(sh, s_p, s_buf, local, 1);
}

// ---------------------------------------------------------------------------
// The batched form as one persistent launch. Each CTA loops: take the next
// work item from the ticket counter, wait (bounded) until every item of the
// frame's gating stage has finished, copy the stage's parameters of that frame
// into shared memory, run the stage's body on the item, and count the item as
// finished. Items are taken in ticket order, so a CTA only ever waits for items
// that running CTAs took before it: the waits end whether or not every CTA of
// the grid is resident. Every stage body is the one the single-frame kernels
// run (at 256 threads; the block-level stages run two blocks per item, one per
// 128-thread group), so each frame's results are those of the single-frame path.
constexpr uint32_t kBatchWaitSpins = 1u << 22;

struct BatchQuantShared
{
	float tile[2][32][kBandPitch];
	QuantGroupShared q[2];
};

struct BatchShared
{
	union
	{
		DwtShared dwt;
		IdwtShared idwt;
		PackShared pack[2];
		DequantShared deq[2];
		BatchQuantShared quant;
	} u;
	union
	{
		LevelParams lp;
		BlockParams bp;
		ResolveParams rp;
	} prm;
	EncodeBuffers eb;
	DecodeInput di;
	PlaneInput in;
	PlaneOutput out;
	int item;
};
static_assert(sizeof(BatchShared) <= 56 * 1024, "the persistent kernel's stage storage fits four CTAs per SM");

// The kernel's shared memory (dynamic: its stages' storage is a union larger
// than a static allocation may be).
extern __shared__ __align__(128) unsigned char batch_smem[];
__device__ __forceinline__ BatchShared &batch_shared() { return *reinterpret_cast<BatchShared *>(batch_smem); }

// Each stage body is its own function (not inlined into the loop), so that
// register allocation happens per stage, as in the single-frame kernels; each
// reaches the shared storage through the kernel's own symbol.
__device__ __noinline__ void batch_forward_item(int level, int small_level, int local)
{
	BatchShared &sh = batch_shared();
	const int per_comp = sh.prm.lp.L.tiles_x * sh.prm.lp.L.tiles_y;
	dwt_forward_body<kBatchPersistentThreads>(sh.u.dwt, sh.prm.lp, sh.in, sh.eb, nullptr, level < small_level ? 1 : 0,
	                                          local % per_comp, local / per_comp);
}

__device__ __noinline__ void batch_quant_item(int small_blocks, int local)
{
	BatchShared &sh = batch_shared();
	quant_blocks_body<1, 2>(sh.prm.bp, sh.eb, 0, small_blocks, local, sh.u.quant.tile, sh.u.quant.q);
}

__device__ __noinline__ void batch_resolve_item(int slice, int slices)
{
	BatchShared &sh = batch_shared();
	resolve_body(sh.prm.rp, sh.eb, slice, slices);
}

__device__ __noinline__ void batch_pack_item(int blk, int half)
{
	BatchShared &sh = batch_shared();
	pack_body(sh.u.pack[half], sh.prm.bp, sh.eb, blk, 1 + half);
}

__device__ __noinline__ void batch_dequant_item(int blk, int half)
{
	BatchShared &sh = batch_shared();
	dequant_body(sh.u.deq[half], sh.prm.bp, sh.di, blk, blk == 0, 1 + half);
}

__device__ __noinline__ void batch_inverse_item(int local)
{
	BatchShared &sh = batch_shared();
	const int per_comp = sh.prm.lp.L.tiles_x * sh.prm.lp.L.tiles_y;
	idwt_body<kBatchPersistentThreads>(sh.u.idwt, sh.prm.lp, sh.di, sh.out, nullptr, local % per_comp,
	                                   local / per_comp);
}

__global__ void __launch_bounds__(kBatchPersistentThreads, 4) batch_persistent_kernel(const BatchRunParams rp)
{
	BatchShared &sh = batch_shared();
	// Thread 0 holds the CTA's next ticket, taken while the current item runs,
	// so the ticket's round trip overlaps the work. Tickets are still processed
	// in increasing order by every CTA, and an item only waits for items with
	// smaller tickets, so every wait still ends.
	int next = 0;
	if (threadIdx.x == 0)
		next = int(atomicAdd(rp.ticket, 1u));
	for (;;)
	{
		if (threadIdx.x == 0)
			sh.item = next;
		__syncthreads();
		const int item = sh.item;
		if (item >= rp.nwork)
			return;
		if (threadIdx.x == 0)
			next = int(atomicAdd(rp.ticket, 1u));
		const uint32_t w = __ldg(rp.work + item);
		const int f = int(w >> 24), stage = int((w >> kBatchLocalBits) & 31u);
		const int local = int(w & ((1u << kBatchLocalBits) - 1u));
		const BatchFrame &fr = rp.frames[f];
		if (threadIdx.x == 0)
		{
			const uint32_t gate = __ldg(rp.gates + f * kBatchStages + stage);
			if (gate != kNoGate)
			{
				const uint32_t *count = rp.done + f * kBatchStages + (gate >> 24);
				const uint32_t target = gate & 0xffffffu;
				uint32_t spins = 0;
				while (ld_acquire_u32(count) < target)
				{
					if (++spins > kBatchWaitSpins)
					{
						atomicOr(&fr.eb.rc->error, kErrorLevelWait);
						break;
					}
					__nanosleep(64);
				}
			}
		}
		if (stage < kStageQuant)
		{
			load_params(sh.prm.lp, fr.lp[stage - kStageDwt0]);
			load_params(sh.in, rp.io[f].in);
			load_params(sh.eb, fr.eb);
		}
		else if (stage == kStageQuant || stage == kStagePack)
		{
			load_params(sh.prm.bp, fr.bp);
			load_params(sh.eb, fr.eb);
		}
		else if (stage == kStageResolve)
		{
			load_params(sh.prm.rp, rp.io[f].rp);
			load_params(sh.eb, fr.eb);
		}
		else if (stage == kStageDequant)
		{
			load_params(sh.prm.bp, fr.bp);
			load_params(sh.di, fr.di);
		}
		else
		{
			load_params(sh.prm.lp, fr.lp[kStageIdwt4 + 4 - stage]);
			load_params(sh.di, fr.di);
			load_params(sh.out, rp.io[f].out);
		}
		__syncthreads();
		const int half = int(threadIdx.x) >> 7;
		if (stage < kStageQuant)
			batch_forward_item(stage - kStageDwt0, rp.small_level, local);
		else if (stage == kStageQuant)
			batch_quant_item(fr.small_blocks, local);
		else if (stage == kStageResolve)
			batch_resolve_item(local, fr.slices);
		else if (stage == kStagePack)
		{
			const int blk = local * 2 + half;
			if (blk < fr.block_count)
				batch_pack_item(blk, half);
		}
		else if (stage == kStageDequant)
		{
			const int blk = local * 2 + half;
			if (blk < fr.block_count)
				batch_dequant_item(blk, half);
		}
		else
			batch_inverse_item(local);
		__syncthreads();
		if (threadIdx.x == 0)
		{
			__threadfence();
			atomicAdd(rp.done + f * kBatchStages + stage, 1u);
		}
	}
}

} // namespace

int batch_persistent_max_ctas_per_sm()
{
	static int cached = 0;
	if (!cached)
	{
		cudaFuncSetAttribute(batch_persistent_kernel, cudaFuncAttributeMaxDynamicSharedMemorySize,
		                     int(sizeof(BatchShared)));
		int n = 0;
		if (cudaOccupancyMaxActiveBlocksPerMultiprocessor(&n, batch_persistent_kernel, kBatchPersistentThreads,
		                                                  sizeof(BatchShared)) != cudaSuccess ||
		    n < 1)
		{
			(void)cudaGetLastError();
			n = 1;
		}
		cached = n;
	}
	return cached;
}

// The kernel's shared-memory attribute is set by batch_persistent_max_ctas_per_sm,
// which the batch calls before any launch (outside stream capture).
void launch_batch_persistent(const BatchRunParams &rp, int ctas, cudaStream_t stream)
{
	batch_persistent_kernel<<<ctas, kBatchPersistentThreads, sizeof(BatchShared), stream>>>(rp);
}

LaunchConfig::LaunchConfig(dim3 grid, dim3 block, cudaStream_t stream, bool programmatic)
{
	cfg = {};
	cfg.gridDim = grid;
	cfg.blockDim = block;
	cfg.dynamicSmemBytes = 0;
	cfg.stream = stream;
	attr.id = cudaLaunchAttributeProgrammaticStreamSerialization;
	attr.val.programmaticStreamSerializationAllowed = 1;
	cfg.attrs = programmatic ? &attr : nullptr;
	cfg.numAttrs = programmatic ? 1 : 0;
}

int forward_fused_mode(const LevelParams &p, bool fused_quant)
{
	if (!fused_quant)
		return 0;
	const int tiles = p.L.tiles_x * p.L.tiles_y * ((p.level == 0 && !p.chroma444) ? 1 : 3);
	return tiles < kSplitTailTiles ? kFusedSplitTail : 1;
}

void launch_dwt_forward_level(const LevelParams &p, const PlaneInput &in, const EncodeBuffers &buf,
                              const LevelTileMap *maps, bool fused_quant, bool programmatic, cudaStream_t stream)
{
	const dim3 grid(p.L.tiles_x * p.L.tiles_y, (p.level == 0 && !p.chroma444) ? 1 : 3);
	const int f = forward_fused_mode(p, fused_quant);
	LevelTileMap m = {};
	if (maps)
		m = *maps;
	if (int(grid.x * grid.y) < kSmallLevelTiles && f == 0)
	{
		LaunchConfig lc(dim3(grid.x * kDwtStripes, grid.y), dim3(kLargeLevelThreads), stream, programmatic);
		cudaLaunchKernelEx(&lc.cfg, dwt_stripes_kernel, p, in, buf, f, m);
	}
	else if (int(grid.x * grid.y) < kSmallLevelTiles)
	{
		LaunchConfig lc(grid, dim3(1024), stream, programmatic);
		cudaLaunchKernelEx(&lc.cfg, dwt_forward_kernel<1024>, p, in, buf, f, m);
	}
	else
	{
		LaunchConfig lc(grid, dim3(kLargeLevelThreads), stream, programmatic);
		cudaLaunchKernelEx(&lc.cfg, dwt_forward_kernel<kLargeLevelThreads>, p, in, buf, f, m);
	}
}

void launch_quant_pretransformed(const BlockParams &p, const EncodeBuffers &buf, int nblocks, bool programmatic,
                                 cudaStream_t stream)
{
	LaunchConfig lc(dim3(nblocks), dim3(256), stream, programmatic);
	cudaLaunchKernelEx(&lc.cfg, quant_pretransformed_kernel<2>, p, buf, nblocks);
}

int resolve_cluster_max()
{
	static int cached = 0;
	if (cached == 0)
	{
		// Clusters of 16 CTAs are opt-in; use them where the device can place one.
		int n = 0;
		if (cudaFuncSetAttribute(resolve_cluster_kernel<1>, cudaFuncAttributeNonPortableClusterSizeAllowed, 1) ==
		        cudaSuccess &&
		    cudaFuncSetAttribute(resolve_cluster_kernel<2>, cudaFuncAttributeNonPortableClusterSizeAllowed, 1) ==
		        cudaSuccess &&
		    cudaFuncSetAttribute(resolve_cluster_kernel<4>, cudaFuncAttributeNonPortableClusterSizeAllowed, 1) ==
		        cudaSuccess)
		{
			cudaLaunchConfig_t cfg = {};
			cudaLaunchAttribute attr = {};
			cfg.gridDim = dim3(kMaxResolveCluster);
			cfg.blockDim = dim3(kClusterResolveThreads);
			attr.id = cudaLaunchAttributeClusterDimension;
			attr.val.clusterDim.x = kMaxResolveCluster;
			attr.val.clusterDim.y = 1;
			attr.val.clusterDim.z = 1;
			cfg.attrs = &attr;
			cfg.numAttrs = 1;
			if (cudaOccupancyMaxActiveClusters(&n, resolve_cluster_kernel<4>, &cfg) != cudaSuccess)
				n = 0;
		}
		(void)cudaGetLastError();
		cached = n > 0 ? kMaxResolveCluster : 8;
	}
	return cached;
}

bool resolve_cluster_shape(int blocks, int &ctas, int &rows)
{
	const int cmax = resolve_cluster_max();
	int c = 1;
	while (c < cmax && c * kClusterResolveThreads < blocks)
		c *= 2;
	const int r = (blocks + c * kClusterResolveThreads - 1) / (c * kClusterResolveThreads);
	if (r > 4)
		return false;
	ctas = c;
	rows = r <= 1 ? 1 : (r <= 2 ? 2 : 4);
	return true;
}

void launch_resolve(const ResolveParams &p, const EncodeBuffers &buf, cudaStream_t stream)
{
	int ctas = 0, rows = 0;
	if (resolve_cluster_shape(p.block_count_32x32, ctas, rows))
	{
		cudaLaunchConfig_t cfg = {};
		cudaLaunchAttribute attrs[2] = {};
		cfg.gridDim = dim3(ctas);
		cfg.blockDim = dim3(kClusterResolveThreads);
		cfg.stream = stream;
		attrs[0].id = cudaLaunchAttributeProgrammaticStreamSerialization;
		attrs[0].val.programmaticStreamSerializationAllowed = 1;
		attrs[1].id = cudaLaunchAttributeClusterDimension;
		attrs[1].val.clusterDim.x = unsigned(ctas);
		attrs[1].val.clusterDim.y = 1;
		attrs[1].val.clusterDim.z = 1;
		cfg.attrs = attrs;
		cfg.numAttrs = 2;
		if (rows == 1)
			cudaLaunchKernelEx(&cfg, resolve_cluster_kernel<1>, p, buf);
		else if (rows == 2)
			cudaLaunchKernelEx(&cfg, resolve_cluster_kernel<2>, p, buf);
		else
			cudaLaunchKernelEx(&cfg, resolve_cluster_kernel<4>, p, buf);
		return;
	}
	const int slices = resolve_slices(p.block_count_32x32, p.blocks_per_subdivision);
	// One thread per block of a slice, 256 to 1024 per CTA.
	if (p.blocks_per_subdivision >= 1024)
	{
		LaunchConfig lc(dim3(slices), dim3(1024), stream, true);
		cudaLaunchKernelEx(&lc.cfg, resolve_kernel<1024>, p, buf);
	}
	else if (p.blocks_per_subdivision >= 512)
	{
		LaunchConfig lc(dim3(slices), dim3(512), stream, true);
		cudaLaunchKernelEx(&lc.cfg, resolve_kernel<512>, p, buf);
	}
	else
	{
		LaunchConfig lc(dim3(slices), dim3(256), stream, true);
		cudaLaunchKernelEx(&lc.cfg, resolve_kernel<256>, p, buf);
	}
}

void launch_pack(const BlockParams &p, const EncodeBuffers &buf, cudaStream_t stream)
{
	LaunchConfig lc(dim3(p.block_count_32x32), dim3(kPackThreads), stream, true);
	cudaLaunchKernelEx(&lc.cfg, pack_kernel, p, buf);
}

void launch_dwt_forward_batch(const BatchFrame *frames, const BatchFrameIO *io, const uint32_t *cta_map, int nctas,
                              int level, const BatchTileMaps *maps, bool fused_quant, bool large_ctas,
                              bool programmatic, cudaStream_t stream)
{
	const int f = fused_quant ? 1 : 0;
	static const BatchTileMaps none = {};
	const BatchTileMaps &m = maps ? *maps : none;
	if (large_ctas)
	{
		LaunchConfig lc(dim3(nctas), dim3(1024), stream, programmatic);
		cudaLaunchKernelEx(&lc.cfg, dwt_forward_batch_kernel<1024>, frames, io, cta_map, level, f, m);
	}
	else
	{
		LaunchConfig lc(dim3(nctas), dim3(kLargeLevelThreads), stream, programmatic);
		cudaLaunchKernelEx(&lc.cfg, dwt_forward_batch_kernel<kLargeLevelThreads>, frames, io, cta_map, level, f, m);
	}
}

void launch_quant_blocks_batch(const BatchFrame *frames, const uint32_t *cta_map, int nctas, bool programmatic,
                               cudaStream_t stream)
{
	LaunchConfig lc(dim3(nctas), dim3(512), stream, programmatic);
	cudaLaunchKernelEx(&lc.cfg, quant_blocks_batch_kernel<2>, frames, cta_map);
}

void launch_resolve_batch(const BatchFrame *frames, const BatchFrameIO *io, const uint32_t *cta_map, int nctas,
                          cudaStream_t stream)
{
	LaunchConfig lc(dim3(nctas), dim3(kResolveBatchThreads), stream, true);
	cudaLaunchKernelEx(&lc.cfg, resolve_batch_kernel, frames, io, cta_map);
}

void launch_pack_batch(const BatchFrame *frames, const uint32_t *cta_map, int nctas, cudaStream_t stream)
{
	LaunchConfig lc(dim3(nctas), dim3(128), stream, true);
	cudaLaunchKernelEx(&lc.cfg, pack_batch_kernel, frames, cta_map);
}

} // namespace pw
