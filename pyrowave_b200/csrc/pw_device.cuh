// Device helpers shared by the sm_100a kernels.
//
// Floating point conventions (mirrored by the CPU oracle, which is how the two
// are compared bit for bit): every FP32 operation is an IEEE round-to-nearest
// operation written out with explicit _rn intrinsics; the library is built with
// --fmad=false, so the only fused multiply-adds are the explicit ones (lifting
// updates and squared sums). Reductions use the xor-butterfly order, FP16
// rounding is round-to-nearest-even.
#pragma once

#include "pw_internal.h"

namespace pw
{
// CDF 9/7 lifting constants (T.800 F.4.8.2, the values used in the reference's
// dwt_common.h:37-42), as single-precision literals; 1/K is a float division.
constexpr float kAlpha = -1.586134342059924f;
constexpr float kBeta = -0.052980118572961f;
constexpr float kGamma = 0.882911075530934f;
constexpr float kDelta = 0.443506852043971f;
constexpr float kK = 1.230174104914001f;
constexpr float kInvK = 1.0f / 1.230174104914001f;

// Vulkan MIRRORED_REPEAT addressing over [0, n).
__device__ __forceinline__ int mirrored_repeat(int i, int n)
{
	int p = 2 * n;
	int t = i % p;
	if (t < 0)
		t += p;
	return t < n ? t : p - 1 - t;
}

// Forward transform input addressing (reference: dwt.comp:27-36 gather on a
// mirrored-repeat sampler, with the clamp-to-edge fold for the region between
// the real size and the aligned size). Resolved per sample; the coordinate
// adjustment is decided on the even sample of each pair.
__device__ __forceinline__ int fwd_index(int p, int resolution, int aligned)
{
	int x = p & ~1;
	int idx;
	if (x < 0)
		idx = p - 1;
	else if (x + 1 >= 2 * aligned - resolution)
		idx = p + 1 + 2 * (resolution - aligned);
	else
		idx = min(p, resolution);
	return mirrored_repeat(idx, resolution);
}

// Inverse transform band addressing (reference: idwt.comp:25-32): low-pass
// (even) and high-pass (odd) samples of a band of n samples.
__device__ __forceinline__ int inv_index_low(int p, int n) { return mirrored_repeat(p < 0 ? p - 1 : p, n); }
__device__ __forceinline__ int inv_index_high(int p, int n)
{
	int q = p & ~1;
	return mirrored_repeat(q + 1 >= n ? p + 1 : p, n);
}

// One lifting update v +/- c * (a + b): a rounded add, then one fused multiply-add.
__device__ __forceinline__ float lift_add(float v, float c, float a, float b)
{
	return __fmaf_rn(c, __fadd_rn(a, b), v);
}
__device__ __forceinline__ float lift_sub(float v, float c, float a, float b)
{
	return __fmaf_rn(-c, __fadd_rn(a, b), v);
}

// Forward lifting over a register window e[0..N); window position j has the
// same parity as the signal position it holds. Outputs e[4 .. N-4) are exact.
template <int N> __device__ __forceinline__ void lift_forward(float (&e)[N])
{
#pragma unroll
	for (int j = 1; j + 1 < N; j += 2)
		e[j] = lift_add(e[j], kAlpha, e[j - 1], e[j + 1]);
#pragma unroll
	for (int j = 2; j + 1 < N; j += 2)
		e[j] = lift_add(e[j], kBeta, e[j - 1], e[j + 1]);
#pragma unroll
	for (int j = 3; j + 1 < N; j += 2)
		e[j] = lift_add(e[j], kGamma, e[j - 1], e[j + 1]);
#pragma unroll
	for (int j = 4; j + 1 < N; j += 2)
		e[j] = lift_add(e[j], kDelta, e[j - 1], e[j + 1]);
}

template <int N> __device__ __forceinline__ void lift_inverse(float (&e)[N])
{
#pragma unroll
	for (int j = 2; j + 1 < N; j += 2)
		e[j] = lift_sub(e[j], kDelta, e[j - 1], e[j + 1]);
#pragma unroll
	for (int j = 3; j + 1 < N; j += 2)
		e[j] = lift_sub(e[j], kGamma, e[j - 1], e[j + 1]);
#pragma unroll
	for (int j = 4; j + 1 < N; j += 2)
		e[j] = lift_sub(e[j], kBeta, e[j - 1], e[j + 1]);
#pragma unroll
	for (int j = 5; j + 1 < N; j += 2)
		e[j] = lift_sub(e[j], kAlpha, e[j - 1], e[j + 1]);
}

__device__ __forceinline__ float round_to_half(float v) { return __half2float(__float2half_rn(v)); }

// Programmatic dependent launch (sm_90+ griddepcontrol): let the next kernel
// of the sequence start its prologue now / wait until the previous kernel of
// the sequence has completed and its writes are visible. Without a
// programmatic predecessor both are no-ops.
__device__ __forceinline__ void pdl_trigger() { asm volatile("griddepcontrol.launch_dependents;" ::: "memory"); }
__device__ __forceinline__ void pdl_wait() { asm volatile("griddepcontrol.wait;" ::: "memory"); }

// Tensor-memory-access (TMA) tile loads into shared memory, completed on an
// mbarrier. Plain CTA-local loads: no cluster multicast.
__device__ __forceinline__ uint32_t smem_addr(const void *p) { return uint32_t(__cvta_generic_to_shared(p)); }

__device__ __forceinline__ void mbarrier_init(uint64_t *bar, uint32_t count)
{
	asm volatile("mbarrier.init.shared::cta.b64 [%0], %1;" ::"r"(smem_addr(bar)), "r"(count) : "memory");
	asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
}

__device__ __forceinline__ void mbarrier_expect_tx(uint64_t *bar, uint32_t bytes)
{
	asm volatile("mbarrier.arrive.expect_tx.shared::cta.b64 _, [%0], %1;" ::"r"(smem_addr(bar)), "r"(bytes) : "memory");
}

// Waits for phase `parity` of the barrier to complete, at most `max_polls`
// polls (each a bounded hardware wait); false when it gave up.
__device__ __forceinline__ bool mbarrier_wait(uint64_t *bar, uint32_t parity, uint32_t max_polls)
{
	const uint32_t a = smem_addr(bar);
	for (uint32_t i = 0; i < max_polls; i++)
	{
		uint32_t done;
		asm volatile("{\n\t.reg .pred p;\n\t"
		             "mbarrier.try_wait.parity.shared::cta.b64 p, [%1], %2;\n\t"
		             "selp.u32 %0, 1, 0, p;\n\t}"
		             : "=r"(done)
		             : "r"(a), "r"(parity)
		             : "memory");
		if (done)
			return true;
	}
	return false;
}

__device__ __forceinline__ void prefetch_tensor_map(const void *tensor_map)
{
	asm volatile("prefetch.tensormap [%0];" ::"l"(tensor_map) : "memory");
}

// 2D tile load: the box of the tensor map at (x, y) (x * element size a
// multiple of 16 bytes) into shared memory at dst (16-byte aligned).
__device__ __forceinline__ void tma_load_2d(void *dst, const void *tensor_map, int x, int y, uint64_t *bar)
{
	asm volatile("cp.async.bulk.tensor.2d.shared::cluster.global.mbarrier::complete_tx::bytes [%0], [%1, {%2, %3}], [%4];"
	             ::"r"(smem_addr(dst)), "l"(tensor_map), "r"(x), "r"(y), "r"(smem_addr(bar))
	             : "memory");
}

// GPU-scope acquire load of a 32-bit counter (work items finished by other CTAs).
__device__ __forceinline__ uint32_t ld_acquire_u32(const uint32_t *p)
{
	uint32_t v;
	asm volatile("ld.acquire.gpu.global.u32 %0, [%1];" : "=r"(v) : "l"(p) : "memory");
	return v;
}

// Orders this thread's generic-proxy view of global memory (data other CTAs
// stored, observed through an acquire) before its later async-proxy (TMA) reads.
__device__ __forceinline__ void fence_proxy_async_global() { asm volatile("fence.proxy.async.global;" ::: "memory"); }

// Bounded wait until a counter reaches `target` (one thread). Returns false
// when it gave up after kDataflowWaitSpins polls.
__device__ __forceinline__ bool wait_counter(const uint32_t *c, uint32_t target)
{
	uint32_t spins = 0;
	while (ld_acquire_u32(c) < target)
	{
		if (++spins > kDataflowWaitSpins)
			return false;
		__nanosleep(64);
	}
	return true;
}

// Adds one to a counter once every thread of the CTA has stored its part
// (called by every thread; the barrier orders the CTA's stores before the
// fence of thread 0).
__device__ __forceinline__ void cta_count_done(uint32_t *c)
{
	__syncthreads();
	if (threadIdx.x == 0)
	{
		__threadfence();
		atomicAdd(c, 1u);
	}
}

// GPU-scope acquire load / release store of a 64-bit word (flags between CTAs).
__device__ __forceinline__ unsigned long long ld_acquire_u64(const unsigned long long *p)
{
	unsigned long long v;
	asm volatile("ld.acquire.gpu.global.u64 %0, [%1];" : "=l"(v) : "l"(p) : "memory");
	return v;
}
__device__ __forceinline__ void st_release_u64(unsigned long long *p, unsigned long long v)
{
	asm volatile("st.release.gpu.global.u64 [%0], %1;" ::"l"(p), "l"(v) : "memory");
}

// Packed pairs of FP32 values (sm_100 f32x2 arithmetic): each lane of the pair
// is rounded exactly as the scalar operation of the same name rounds it, so a
// computation written on pairs gives the scalar results bit for bit in half
// the instructions.
typedef unsigned long long f32x2;
__device__ __forceinline__ f32x2 f2_pack(float lo, float hi)
{
	f32x2 r;
	asm("mov.b64 %0, {%1, %2};" : "=l"(r) : "f"(lo), "f"(hi));
	return r;
}
__device__ __forceinline__ void f2_unpack(f32x2 v, float &lo, float &hi)
{
	asm("mov.b64 {%0, %1}, %2;" : "=f"(lo), "=f"(hi) : "l"(v));
}
__device__ __forceinline__ f32x2 f2_add_rz(f32x2 a, f32x2 b)
{
	f32x2 r;
	asm("add.rz.f32x2 %0, %1, %2;" : "=l"(r) : "l"(a), "l"(b));
	return r;
}
__device__ __forceinline__ f32x2 f2_add_rn(f32x2 a, f32x2 b)
{
	f32x2 r;
	asm("add.rn.f32x2 %0, %1, %2;" : "=l"(r) : "l"(a), "l"(b));
	return r;
}
__device__ __forceinline__ f32x2 f2_sub_rn(f32x2 a, f32x2 b)
{
	f32x2 r;
	asm("sub.rn.f32x2 %0, %1, %2;" : "=l"(r) : "l"(a), "l"(b));
	return r;
}
__device__ __forceinline__ f32x2 f2_mul_rn(f32x2 a, f32x2 b)
{
	f32x2 r;
	asm("mul.rn.f32x2 %0, %1, %2;" : "=l"(r) : "l"(a), "l"(b));
	return r;
}
__device__ __forceinline__ f32x2 f2_fma_rn(f32x2 a, f32x2 b, f32x2 c)
{
	f32x2 r;
	asm("fma.rn.f32x2 %0, %1, %2, %3;" : "=l"(r) : "l"(a), "l"(b), "l"(c));
	return r;
}

// Thread-block clusters: this CTA's rank, the cluster's CTA count, hardware
// cluster barriers (every thread of every CTA of the cluster takes part) and
// 64-bit stores into another CTA's shared memory (distributed shared memory).
__device__ __forceinline__ uint32_t cluster_rank()
{
	uint32_t r;
	asm volatile("mov.u32 %0, %%cluster_ctarank;" : "=r"(r));
	return r;
}
__device__ __forceinline__ uint32_t cluster_size()
{
	uint32_t n;
	asm volatile("mov.u32 %0, %%cluster_nctarank;" : "=r"(n));
	return n;
}
// Arrive early (relaxed: orders nothing) and wait before the first access to
// another CTA's shared memory: every CTA of the cluster has started by then.
__device__ __forceinline__ void cluster_arrive_relaxed() { asm volatile("barrier.cluster.arrive.relaxed.aligned;" ::: "memory"); }
__device__ __forceinline__ void cluster_wait() { asm volatile("barrier.cluster.wait.acquire.aligned;" ::: "memory"); }
// Full barrier: shared and global memory writes before it are visible to every
// thread of the cluster after it.
__device__ __forceinline__ void cluster_sync()
{
	asm volatile("barrier.cluster.arrive.release.aligned;" ::: "memory");
	asm volatile("barrier.cluster.wait.acquire.aligned;" ::: "memory");
}
__device__ __forceinline__ void st_cluster_u64(const void *local_smem, uint32_t rank, unsigned long long v)
{
	uint32_t remote;
	asm volatile("mapa.shared::cluster.u32 %0, %1, %2;" : "=r"(remote) : "r"(smem_addr(local_smem)), "r"(rank));
	asm volatile("st.shared::cluster.u64 [%0], %1;" ::"r"(remote), "l"(v) : "memory");
}

// 8x8 bit-matrix transpose: bit j of byte i of the input becomes bit i of byte
// j of the output (three swap stages of 1, 2 and 4 bit-square blocks).
__device__ __forceinline__ unsigned long long transpose8x8(unsigned long long x)
{
	unsigned long long t = (x ^ (x >> 7)) & 0x00AA00AA00AA00AAull;
	x = x ^ t ^ (t << 7);
	t = (x ^ (x >> 14)) & 0x0000CCCC0000CCCCull;
	x = x ^ t ^ (t << 14);
	t = (x ^ (x >> 28)) & 0x00000000F0F0F0F0ull;
	return x ^ t ^ (t << 28);
}

// The 8 coefficients of a 4x2 sub-block in the quantiser's order (i = 2 * column
// + row) as two 4-wide row vectors: idx is the element index of (row 0, column
// 0), a multiple of 4 (the sub-block starts on a 4-column boundary of a
// 32-aligned band row), pitch the row pitch in elements.
__device__ __forceinline__ void load_subblock(const float *c32, const __half *c16, bool fp16, int64_t idx, int pitch,
                                              float (&c)[8])
{
	float4 r0, r1;
	if (fp16)
	{
		const uint2 a = __ldcg(reinterpret_cast<const uint2 *>(c16 + idx));
		const uint2 b = __ldcg(reinterpret_cast<const uint2 *>(c16 + idx + pitch));
		const float2 a0 = __half22float2(*reinterpret_cast<const __half2 *>(&a.x));
		const float2 a1 = __half22float2(*reinterpret_cast<const __half2 *>(&a.y));
		const float2 b0 = __half22float2(*reinterpret_cast<const __half2 *>(&b.x));
		const float2 b1 = __half22float2(*reinterpret_cast<const __half2 *>(&b.y));
		r0 = make_float4(a0.x, a0.y, a1.x, a1.y);
		r1 = make_float4(b0.x, b0.y, b1.x, b1.y);
	}
	else
	{
		r0 = __ldcg(reinterpret_cast<const float4 *>(c32 + idx));
		r1 = __ldcg(reinterpret_cast<const float4 *>(c32 + idx + pitch));
	}
	c[0] = r0.x, c[2] = r0.y, c[4] = r0.z, c[6] = r0.w;
	c[1] = r1.x, c[3] = r1.y, c[5] = r1.z, c[7] = r1.w;
}

__device__ __forceinline__ void store_subblock(float *c32, __half *c16, bool fp16, int64_t idx, int pitch,
                                               const float (&c)[8])
{
	if (fp16)
	{
		const __half2 a0 = __floats2half2_rn(c[0], c[2]), a1 = __floats2half2_rn(c[4], c[6]);
		const __half2 b0 = __floats2half2_rn(c[1], c[3]), b1 = __floats2half2_rn(c[5], c[7]);
		*reinterpret_cast<uint2 *>(c16 + idx) =
		    make_uint2(*reinterpret_cast<const uint32_t *>(&a0), *reinterpret_cast<const uint32_t *>(&a1));
		*reinterpret_cast<uint2 *>(c16 + idx + pitch) =
		    make_uint2(*reinterpret_cast<const uint32_t *>(&b0), *reinterpret_cast<const uint32_t *>(&b1));
	}
	else
	{
		*reinterpret_cast<float4 *>(c32 + idx) = make_float4(c[0], c[2], c[4], c[6]);
		*reinterpret_cast<float4 *>(c32 + idx + pitch) = make_float4(c[1], c[3], c[5], c[7]);
	}
}

// Barrier of one 128-thread group of a CTA (hardware barrier `id`, 1 or 2):
// the block-level bodies (packing, dequantisation) run one 32x32 block per
// group, so a CTA of 256 threads can hold two independent blocks.
__device__ __forceinline__ void group_sync(int id) { asm volatile("bar.sync %0, 128;" ::"r"(id) : "memory"); }

// Cooperative copy of a parameter struct from global to shared memory (the
// caller synchronises before use).
template <typename T> __device__ __forceinline__ void load_params(T &dst, const T &src)
{
	static_assert(sizeof(T) % 4 == 0, "parameter structs are word multiples");
	const uint32_t *s = reinterpret_cast<const uint32_t *>(&src);
	uint32_t *d = reinterpret_cast<uint32_t *>(&dst);
	for (int i = int(threadIdx.x); i < int(sizeof(T) / 4); i += int(blockDim.x))
		d[i] = __ldg(s + i);
}

// Frame and work item of this CTA in a batched launch (batch_cta() words).
__device__ __forceinline__ void batch_item(const uint32_t *cta_map, int &frame, int &local)
{
	const uint32_t m = __ldg(cta_map + blockIdx.x);
	frame = int(m >> 24);
	local = int(m & 0xffffffu);
}

// Band of a 32x32 block (block index order): the last band whose first block
// is <= blk, then the block's position in it.
__device__ __forceinline__ int find_band(const BlockParams &p, int blk)
{
	int lo = 0, hi = p.nbands - 1;
	while (lo < hi)
	{
		const int mid = (lo + hi + 1) >> 1;
		if (p.band[mid].block32_offset <= blk)
			lo = mid;
		else
			hi = mid - 1;
	}
	return lo;
}

// One coefficient, read through L2 (other CTAs of the same launch may have written it).
__device__ __forceinline__ float load_coef(const float *c32, const __half *c16, bool fp16, int64_t idx)
{
	return fp16 ? __half2float(__ldcg(c16 + idx)) : __ldcg(c32 + idx);
}

// ---------------------------------------------------------------------------
// Quantiser helpers (reference: dwt_quant_scale.h, wavelet_quant.comp,
// block_packing.comp, pyrowave_common.hpp:124-145).
// code / 8 + 0.25 (the division by 8 is exact, so it is a multiplication).
__device__ __forceinline__ float decode_quant_scale(uint32_t code)
{
	return __fadd_rn(__fmul_rn(float(code), 0.125f), 0.25f);
}

// Custom FP quant code of the 32x32 header: (8+m) * 2^(20+e) / 2^23 with
// e = 4 - (code >> 3): an exact product with the power of two 2^(e-3)
// (e - 3 is within [-30, 1], a normal exponent).
__device__ __forceinline__ float decode_quant(uint32_t code)
{
	const int e = kMaxScaleExp - int(code >> 3);
	const int m = int(code & 7u);
	return __fmul_rn(float(8 + m), __int_as_float((127 + e - 3) << 23));
}

__device__ __forceinline__ int find_msb(uint32_t v) { return v ? 31 - __clz(v) : -1; }

// 8-bit quant scale per 8x8 block (wavelet_quant.comp:95-111).
__device__ __forceinline__ void compute_quant_scale(float max_wave, uint32_t &code, float &scale)
{
	if (max_wave < 1.0f)
	{
		code = 6u;
		scale = 1.0f;
	}
	else
	{
		int e;
		frexpf(__fsub_rn(max_wave, 0.25f), &e);
		float target_max = __fsub_rn(float(1 << e), 0.25f);
		float inv_scale = __fdiv_rn(max_wave, target_max);
		code = uint32_t(ceilf(__fmul_rn(__fsub_rn(inv_scale, 0.25f), 8.0f)));
		scale = __fdiv_rn(1.0f, decode_quant_scale(code));
	}
}

// Required plane bytes of an 8x8 block (block_packing.comp:97-105).
__device__ __forceinline__ uint32_t required_8x8_bytes(uint32_t cw)
{
	uint32_t q_bits = (cw >> kQPlanesOffset) & 0xfu;
	uint32_t lsbs = cw & 0x5555u;
	uint32_t msbs = cw & 0xaaaau;
	msbs |= msbs >> 1;
	return uint32_t(__popc(lsbs) + __popc(msbs)) + q_bits * 8u;
}

// Drop `quant` planes from a code word (block_packing.comp:107-142): first the
// Q planes, then max(code - rest, 0) per 4x2 sub-block.
__device__ __forceinline__ uint32_t quantize_code_word(uint32_t cw, int quant)
{
	if (quant != 0 && cw != 0)
	{
		int q_bits = int((cw >> kQPlanesOffset) & 0xfu);
		int sub = min(q_bits, quant);
		q_bits -= sub;
		quant -= sub;
		if (quant != 0)
		{
			quant = min(quant, 3);
			uint32_t p0 = cw & 0x5555u;
			uint32_t p1 = (cw & 0xaaaau) >> 1;
			uint32_t p2 = p0 & p1;
			for (int i = 0; i < quant; i++)
			{
				p0 = p1;
				p1 = p2;
				p2 = 0;
			}
			p0 &= ~p1;
			cw = (cw & ~0xffffu) | ((p0 | (p1 << 1)) & 0xffffu);
		}
		cw = (cw & ~(0xfu << kQPlanesOffset)) | (uint32_t(q_bits) << kQPlanesOffset);
	}
	return cw;
}

// block_packing.comp:161-167
__device__ __forceinline__ uint32_t modify_quant_code(uint32_t code, int quant)
{
	int e = int((code >> 3) & 31u);
	e = max(e - quant, 0);
	return (code & ~(31u << 3)) | (uint32_t(e) << 3);
}

// Rate-control bucket of a quant step (analyze_rate_control.comp:73-83):
// uint(max(60 + 2*log2(r) + 0.5, 0)), evaluated with the exact value of log2:
// for r = m * 2^e, m in [1,2), the result is 60 + 2e + [m >= 2^0.25] + [m >= 2^0.75].
// 0x1837f1 / 0x5744fd are the mantissas of the smallest floats >= 2^0.25 / 2^0.75.
__device__ __forceinline__ uint32_t bucket_index(float d, float cost, float d_base, float cost_base)
{
	if (cost == cost_base)
		return 0;
	float num = fmaxf(__fsub_rn(d, d_base), 0.0f);
	float den = __fsub_rn(cost_base, cost);
	float r = __fdiv_rn(num, den);
	if (!(r > 0.0f))
		return 0;
	uint32_t bits = __float_as_uint(r);
	uint32_t ef = bits >> 23;
	if (ef == 0)
		return 0;
	if (ef >= 255)
		return 255;
	int e = int(ef) - 127;
	uint32_t mant = bits & 0x7fffffu;
	int idx = 60 + 2 * e + (mant >= 0x1837f1u ? 1 : 0) + (mant >= 0x5744fdu ? 1 : 0);
	return idx < 0 ? 0u : uint32_t(idx);
}

// Origin of 4x2 sub-block s inside an 8x8 block (the reference's
// unswizzle8x8(s << 3)) and the pixel order inside it (bitstream.md:350-368).
__device__ __forceinline__ int sub_x(int s) { return (s >> 2) * 4; }
__device__ __forceinline__ int sub_y(int s) { return (s & 3) * 2; }
} // namespace pw
