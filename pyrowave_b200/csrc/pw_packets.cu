// Device-side packet assembly for the decoder: the packets of a frame, as
// received into device memory, are parsed and turned into the per-block
// table the dequantiser reads, with the sequence and first-copy rules of the
// reference's host parser (pyrowave_decoder.cpp:154-262, as restated by the
// host parser in pw_host.cpp), so nothing of the frame passes through the host.
//
// The parser's state is the sequence of the frame being assembled (none or
// 0..7). Pushing one packet maps a state to a state, so the state before every
// packet follows from a scan of the packets' state maps:
//   1. packet_tables_kernel  one CTA per packet: the packet's items are found
//      (below) and the packet is evaluated from each of the 9 possible states:
//      the state after it, the last restart (the reference's clear()) inside
//      it, the block total of the last accepted sequence header, and whether
//      the parser rejects it. The last CTA to finish scans the state maps of
//      all packets: the state before each packet, the last restart of the
//      whole list, the frame's sequence and block total; it also clears the
//      first-copy table.
//   2. packet_blocks_kernel  one CTA per packet from the last restart on:
//      every block the parser keeps proposes (packet, item, word offset) and
//      the smallest, the first copy pushed, wins by a 64-bit atomicMin; the
//      winners are counted. The dequantiser reads the winning keys directly.
#include "pw_device.cuh"

namespace pw
{
namespace
{
constexpr uint32_t kNoneState = 0;          // states: 0 = no sequence yet, 1 + s = sequence s
constexpr uint32_t kNoPos = 0xffffu;        // no restart inside the packet
constexpr uint32_t kNoTotal = 0xffffffffu;  // no sequence header accepted
constexpr uint32_t kMaxItems = 1u << 14;    // items (headers + blocks) per packet
constexpr unsigned long long kNoKey = ~0ull;

struct WalkResult
{
	uint32_t state;
	uint32_t restart; // item index of the last restart, kNoPos if none
	uint32_t total;   // blocks announced by the last header after the last restart
	bool error;       // the host parser returns false for this packet
};

// One pass of the host parser over one packet (push_packet). `word(i)` reads
// word i of the packet; `size` is the packet's size in bytes. on_block(block,
// word position, item index) is called for every block the parser keeps.
template <typename R, typename F>
__device__ WalkResult walk_packet(R word, uint32_t size, uint32_t state, const PacketParams &pp, F on_block)
{
	WalkResult res{state, kNoPos, kNoTotal, false};
	uint32_t pos = 0; // in words
	for (uint32_t item = 0; size >= 8; item++)
	{
		if (item >= kMaxItems)
		{
			res.error = true;
			return res;
		}
		const uint32_t w0 = word(pos), w1 = word(pos + 1);
		const uint32_t seq = (w0 >> 28) & 7u;
		const bool fresh = res.state == kNoneState;
		const uint32_t diff = fresh ? 0u : ((seq - (res.state - 1)) & 7u);
		if ((w0 >> 31) & 1u)
		{
			// Start-of-frame sequence header (bitstream.md:250-265).
			if (((w1 >> 26) & 1u) != uint32_t(pp.chroma444))
			{
				res.error = true;
				return res;
			}
			if (!fresh && diff > 3)
				return res; // an older sequence: the rest of the packet is ignored
			if (fresh || diff != 0)
			{
				res.state = 1 + seq;
				res.restart = item;
				res.total = kNoTotal;
			}
			if (((w1 >> 24) & 3u) != 0 || int(w0 & 0x3fffu) + 1 != pp.width ||
			    int((w0 >> 14) & 0x3fffu) + 1 != pp.height)
			{
				res.error = true;
				return res;
			}
			res.total = w1 & 0xffffffu;
			pos += 2;
			size -= 8;
			continue;
		}
		const uint32_t words = (w0 >> 16) & 0xfffu;
		if (words * 4u > size)
		{
			res.error = true;
			return res;
		}
		if (!fresh && diff > 3)
			return res;
		if (fresh || diff != 0)
		{
			res.state = 1 + seq;
			res.restart = item;
			res.total = kNoTotal;
		}
		const uint32_t block = (w1 >> 8) & 0xffffffu;
		// A block shorter than its own header makes the packet invalid; it is
		// left missing.
		if (block >= uint32_t(pp.block_count) || words < 2)
		{
			res.error = true;
			return res;
		}
		on_block(block, pos, item);
		pos += words;
		size -= words * 4u;
	}
	res.error = res.error || size != 0;
	return res;
}

// The packet's bytes, or why it cannot be read as words.
__device__ __forceinline__ bool packet_span(const PacketParams &pp, int p, uint32_t &first_word, uint32_t &size)
{
	const unsigned long long off = pp.packets[2 * p], sz = pp.packets[2 * p + 1];
	if ((off & 3u) != 0 || off > pp.data_bytes || sz > pp.data_bytes - off || sz > 0xffffffffull)
		return false;
	first_word = uint32_t(off >> 2);
	size = uint32_t(sz);
	return true;
}

// ---------------------------------------------------------------------------
// Item discovery. A packet is a chain of items (sequence headers of 2 words,
// blocks of their announced word count): item k + 1 starts where item k ends.
// Every word position p gets next(p) in parallel: the position after an item
// starting at p, or where the parser stops (an item it rejects, the end, fewer
// than 8 bytes left). Three doubling passes give next^8; one thread follows it
// from 0 (one shared-memory load per 8 items), the items between those anchors
// are filled in parallel, and every later step runs over the items in
// parallel. Packets whose items share one sequence number (every packet of a
// frame) need no walk at all: the parser's state change has a closed form.
// Other packets are walked item by item.
constexpr int kFastWords = 8192;  // packets up to 32 KiB take this path
constexpr uint32_t kDone = 0xffffffffu; // the item ends the packet exactly
constexpr uint32_t kStop = 0xfffffffeu; // the parser rejects the item
constexpr uint32_t kLeft = 0xfffffffdu; // fewer than 8 bytes left: not an item
constexpr int kPacketThreads = 1024;
constexpr uint16_t kJumpEnd = 0xffffu;
constexpr int kAnchorRounds = 3;                 // the chase follows next^8
constexpr int kAnchorStep = 1 << kAnchorRounds;

struct PacketSmem
{
	uint32_t words[kFastWords];
	uint32_t next[kFastWords];
	uint32_t items[kFastWords / 2 + 2]; // item start positions in push order
	uint16_t jump[2][kFastWords];        // next^(2^r), kJumpEnd where the chain stops first
	uint16_t anchors[kFastWords / 16 + 2]; // every kAnchorStep-th item
};
constexpr size_t kPacketSmemBytes = sizeof(PacketSmem);

struct ItemSummary // also the per-packet record in PacketParams::summaries (8 words)
{
	uint32_t nitems;
	uint32_t error;         // first rejected item << 2 | kind (1: before the sequence check, 2: after it); ~0u: none
	uint32_t trailing;      // 1: bytes left over after the last item (the parser's size != 0)
	uint32_t seq_min, seq_max;
	uint32_t fast;                  // 1: the items were listed (the packet fits kFastWords)
	unsigned long long last_header; // (item + 1) << 32 | announced blocks, of the last accepted header; 0: none
};
static_assert(sizeof(ItemSummary) == 32, "per-packet record");

// Classification of an item starting at word p (rem >= 8 bytes left).
struct ItemInfo
{
	bool header;
	uint32_t seq, words, block, total;
	uint32_t error; // 0, 1 (before the sequence check), 2 (after it)
};

__device__ __forceinline__ ItemInfo classify(const uint32_t *w, uint32_t p, uint32_t rem, const PacketParams &pp)
{
	ItemInfo it;
	const uint32_t w0 = w[p], w1 = w[p + 1];
	it.header = (w0 >> 31) & 1u;
	it.seq = (w0 >> 28) & 7u;
	it.total = w1 & 0xffffffu;
	it.block = (w1 >> 8) & 0xffffffu;
	it.error = 0;
	if (it.header)
	{
		it.words = 2;
		if (((w1 >> 26) & 1u) != uint32_t(pp.chroma444))
			it.error = 1;
		else if (((w1 >> 24) & 3u) != 0 || int(w0 & 0x3fffu) + 1 != pp.width || int((w0 >> 14) & 0x3fffu) + 1 != pp.height)
			it.error = 2;
	}
	else
	{
		it.words = (w0 >> 16) & 0xfffu;
		if (it.words * 4u > rem)
			it.error = 1;
		else if (it.block >= uint32_t(pp.block_count) || it.words < 2)
			it.error = 2;
	}
	return it;
}

// Stages the packet (nwords <= kFastWords), lists its items in sm.items and
// fills the item summary. Every thread of the CTA calls it.
__device__ void discover_items(PacketSmem &sm, ItemSummary &sum, const PacketParams &pp, uint32_t first,
                               uint32_t size, uint32_t nwords)
{
	const int t = threadIdx.x;
	// Stage: eight loads in flight per thread.
	for (uint32_t base = 0; base < nwords; base += 8 * kPacketThreads)
	{
		uint32_t v[8];
#pragma unroll
		for (int u = 0; u < 8; u++)
		{
			const uint32_t i = base + t + u * kPacketThreads;
			v[u] = i < nwords ? __ldg(pp.data + first + i) : 0u;
		}
#pragma unroll
		for (int u = 0; u < 8; u++)
		{
			const uint32_t i = base + t + u * kPacketThreads;
			if (i < nwords)
				sm.words[i] = v[u];
		}
	}
	if (t == 0)
	{
		sum.nitems = 0;
		sum.error = ~0u;
		sum.trailing = 0;
		sum.seq_min = 7;
		sum.seq_max = 0;
		sum.last_header = 0;
	}
	__syncthreads();
	for (uint32_t p = t; p < nwords; p += kPacketThreads)
	{
		const uint32_t rem = size - 4 * p;
		uint32_t nxt = kLeft;
		if (rem >= 8)
		{
			const ItemInfo it = classify(sm.words, p, rem, pp);
			nxt = it.error ? kStop : (p + it.words < nwords ? p + it.words : kDone);
		}
		sm.next[p] = nxt;
	}
	__syncthreads();
	// next^8 by three doubling passes; one thread then follows it from 0 (one
	// load per 8 items) and the items between anchors are filled in parallel.
	for (uint32_t p = t; p < nwords; p += kPacketThreads)
	{
		const uint32_t nx = sm.next[p];
		sm.jump[0][p] = nx < nwords ? uint16_t(nx) : kJumpEnd;
	}
	__syncthreads();
	int cur = 0;
	for (int r = 0; r < kAnchorRounds; r++)
	{
		for (uint32_t p = t; p < nwords; p += kPacketThreads)
		{
			const uint32_t j = sm.jump[cur][p];
			sm.jump[cur ^ 1][p] = j == kJumpEnd ? kJumpEnd : sm.jump[cur][j];
		}
		__syncthreads();
		cur ^= 1;
	}
	__shared__ uint32_t s_anchors;
	if (t == 0)
	{
		uint32_t m = 0, p = 0;
		while (nwords > 0)
		{
			sm.anchors[m++] = uint16_t(p);
			const uint32_t j = sm.jump[cur][p];
			if (j == kJumpEnd)
				break;
			p = j;
		}
		s_anchors = m;
	}
	__syncthreads();
	const uint32_t na = s_anchors;
	for (uint32_t a = t; a < na; a += kPacketThreads)
	{
		uint32_t q = sm.anchors[a];
		for (uint32_t i = 0; i < uint32_t(kAnchorStep); i++)
		{
			const uint32_t nx = sm.next[q];
			if (nx == kLeft)
			{
				sum.trailing = 1; // q is not an item: fewer than 8 bytes were left
				sum.nitems = a * kAnchorStep + i;
				break;
			}
			sm.items[a * kAnchorStep + i] = q;
			if (nx == kStop || nx == kDone)
			{
				sum.nitems = a * kAnchorStep + i + 1;
				break;
			}
			q = nx;
		}
	}
	__syncthreads();
	const uint32_t n = sum.nitems;
	for (uint32_t k = t; k < n; k += kPacketThreads)
	{
		const uint32_t p = sm.items[k];
		const ItemInfo it = classify(sm.words, p, size - 4 * p, pp);
		if (it.error)
			atomicMin(&sum.error, k << 2 | it.error); // only the last item can be rejected
	}
	__syncthreads();
	// Sequence range of the items whose sequence number the parser looks at,
	// and the last accepted header.
	const uint32_t err_item = sum.error == ~0u ? ~0u : sum.error >> 2;
	const uint32_t err_kind = sum.error == ~0u ? 0u : sum.error & 3u;
	uint32_t smin = 7, smax = 0;
	unsigned long long lh = 0;
	for (uint32_t k = t; k < n; k += kPacketThreads)
	{
		if (k == err_item && err_kind == 1)
			continue;
		const uint32_t p = sm.items[k];
		const ItemInfo it = classify(sm.words, p, size - 4 * p, pp);
		smin = min(smin, it.seq);
		smax = max(smax, it.seq);
		if (it.header && k != err_item)
			lh = max(lh, (unsigned long long)(k + 1) << 32 | it.total);
	}
	if (smin <= smax)
	{
		atomicMin(&sum.seq_min, smin);
		atomicMax(&sum.seq_max, smax);
	}
	if (lh)
		atomicMax(&sum.last_header, lh);
	__syncthreads();
}

// The parser's pass over a packet whose items share one sequence number, in
// closed form (see walk_packet for the item-by-item rules).
__device__ __forceinline__ WalkResult uniform_walk(const ItemSummary &sum, uint32_t state, bool &accepts_blocks)
{
	WalkResult r{state, kNoPos, kNoTotal, false};
	accepts_blocks = false;
	const uint32_t err_item = sum.error == ~0u ? ~0u : sum.error >> 2;
	const uint32_t err_kind = sum.error == ~0u ? 0u : sum.error & 3u;
	if (sum.nitems == 0)
	{
		r.error = sum.trailing != 0;
		return r;
	}
	if (err_item == 0 && err_kind == 1)
	{
		r.error = true; // rejected before its sequence number is looked at
		return r;
	}
	const uint32_t s = sum.seq_min;
	const bool fresh = state == kNoneState;
	const uint32_t diff = fresh ? 0u : ((s - (state - 1)) & 7u);
	if (!fresh && diff > 3)
		return r; // an older sequence: the packet is ignored
	if (fresh || diff != 0)
	{
		r.state = 1 + s;
		r.restart = 0;
	}
	if (sum.last_header)
		r.total = uint32_t(sum.last_header & 0xffffffffull);
	r.error = err_item != ~0u || sum.trailing != 0;
	accepts_blocks = true;
	return r;
}

// State maps as 9 nibbles: nibble x = state after the packet(s) from state x.
__device__ __forceinline__ uint32_t map_at(unsigned long long m, uint32_t x)
{
	return x < 8 ? (uint32_t(m) >> (4 * x)) & 0xfu : uint32_t(m >> 32) & 0xfu;
}

__device__ __forceinline__ unsigned long long compose(unsigned long long a, unsigned long long b)
{
	// a first, then b
	uint32_t lo = 0;
#pragma unroll
	for (int x = 0; x < 8; x++)
		lo |= map_at(b, map_at(a, x)) << (4 * x);
	return (unsigned long long)map_at(b, map_at(a, 8)) << 32 | lo;
}

constexpr unsigned long long kIdentityMap = 0x876543210ull; // nibble x = x

__device__ __forceinline__ unsigned long long packet_map(const PacketParams &pp, int p)
{
	unsigned long long m = 0;
	for (int x = 0; x < 9; x++)
		m |= (unsigned long long)(__ldcg(pp.tables + (size_t(p) * 9 + x) * 2) & 0xfu) << (4 * x);
	return m;
}

// Run by the last CTA of the table pass (1024 threads), once every packet's
// table is written.
__device__ void scan_packets(const PacketParams &pp)
{
	__shared__ unsigned long long s_warp[32];
	__shared__ unsigned long long s_last_restart, s_last_total;
	__shared__ uint32_t s_invalid;
	const int t = threadIdx.x, n = pp.count, lane = t & 31, warp = t >> 5;
	const int per = (n + 1023) / 1024;
	const int p0 = min(t * per, n), p1 = min(p0 + per, n);
	if (t == 0)
	{
		s_last_restart = 0;
		s_last_total = 0;
		s_invalid = 0;
	}
	// This thread's packets composed, then a scan over threads: within each
	// warp by shuffles, then over the warp totals. Warps past the last packet
	// hold the identity.
	const bool active = warp * 32 * per < n; // uniform over the warp
	unsigned long long incl = kIdentityMap;
	for (int p = p0; p < p1; p++)
		incl = compose(incl, packet_map(pp, p));
	if (active)
	{
#pragma unroll
		for (int off = 1; off < 32; off *= 2)
		{
			const unsigned long long other = __shfl_up_sync(0xffffffffu, incl, off);
			if (lane >= off)
				incl = compose(other, incl);
		}
	}
	if (lane == 31)
		s_warp[warp] = incl;
	__syncthreads();
	if (warp == 0)
	{
		unsigned long long w = s_warp[lane];
#pragma unroll
		for (int off = 1; off < 32; off *= 2)
		{
			const unsigned long long other = __shfl_up_sync(0xffffffffu, w, off);
			if (lane >= off)
				w = compose(other, w);
		}
		s_warp[lane] = w; // inclusive over warps
	}
	__syncthreads();
	unsigned long long excl = active ? __shfl_up_sync(0xffffffffu, incl, 1) : kIdentityMap;
	if (lane == 0)
		excl = kIdentityMap;
	const unsigned long long before = compose(warp == 0 ? kIdentityMap : s_warp[warp - 1], excl);
	// State before each of this thread's packets (the maps applied to "no
	// sequence"); the last restart and the last accepted header (ordered by
	// packet, then item: 1 + packet << 16 | item).
	uint32_t state = map_at(before, kNoneState);
	unsigned long long last_restart = 0, last_total = 0;
	uint32_t invalid = 0;
	for (int p = p0; p < p1; p++)
	{
		pp.state_before[p] = uint8_t(state);
		const uint32_t a = __ldcg(pp.tables + (size_t(p) * 9 + state) * 2);
		const uint32_t total = __ldcg(pp.tables + (size_t(p) * 9 + state) * 2 + 1);
		const uint32_t restart = a >> 8;
		if (restart != kNoPos)
			last_restart = 1ull + ((unsigned long long)p << 16 | restart);
		if (total != kNoTotal)
			last_total = 1ull + ((unsigned long long)p << 32 | total);
		invalid += (a >> 4) & 1u;
		state = a & 0xfu;
	}
	if (last_restart)
		atomicMax(&s_last_restart, last_restart);
	if (last_total)
		atomicMax(&s_last_total, last_total);
	if (invalid)
		atomicAdd(&s_invalid, invalid);
	for (int b = t; b < pp.block_count; b += 1024)
		pp.first[b] = kNoKey;
	__syncthreads();
	if (t == 0)
	{
		PacketStatus st = {};
		const uint32_t final_state = n > 0 ? map_at(s_warp[31], kNoneState) : kNoneState;
		st.sequence = final_state == kNoneState ? 0xffffffffu : final_state - 1;
		st.invalid_packets = s_invalid;
		const unsigned long long lr = s_last_restart;
		st.restart_packet = lr ? uint32_t((lr - 1) >> 16) : 0u;
		st.restart_item = lr ? uint32_t((lr - 1) & 0xffffu) : 0u;
		// The block total: the last header at or after the last restart, else
		// the frame's block count (clear() in the reference parser).
		const unsigned long long lt = s_last_total;
		const uint32_t total_packet = lt ? uint32_t((lt - 1) >> 32) : 0u;
		st.total_blocks = (lt && lr && total_packet >= st.restart_packet) ? uint32_t((lt - 1) & 0xffffffffu)
		                                                                  : uint32_t(pp.block_count);
		st.decoded_blocks = 0;
		*pp.status = st;
	}
}

__global__ void __launch_bounds__(kPacketThreads) packet_tables_kernel(const PacketParams pp)
{
	extern __shared__ __align__(16) unsigned char s_raw[];
	PacketSmem &sm = *reinterpret_cast<PacketSmem *>(s_raw);
	__shared__ ItemSummary sum;
	const int p = blockIdx.x;
	uint32_t first = 0, size = 0;
	const bool ok = packet_span(pp, p, first, size);
	const uint32_t nwords = (size + 3) / 4;
	const bool fast = ok && nwords <= uint32_t(kFastWords);
	pdl_trigger(); // the block pass may launch meanwhile
	if (fast)
	{
		discover_items(sm, sum, pp, first, size, nwords);
		// The item list goes to the packet's own word range of pp.items, for the block pass.
		for (uint32_t k = threadIdx.x; k < sum.nitems; k += kPacketThreads)
			pp.items[first + k] = sm.items[k];
	}
	if (threadIdx.x == 0)
	{
		ItemSummary rec = fast ? sum : ItemSummary{};
		rec.fast = fast ? 1u : 0u;
		reinterpret_cast<ItemSummary *>(pp.summaries)[p] = rec;
	}
	if (threadIdx.x < 9)
	{
	const uint32_t init = threadIdx.x;
	WalkResult r;
	bool acc;
	if (!ok)
		r = WalkResult{init, kNoPos, kNoTotal, true};
	else if (fast && sum.seq_min == sum.seq_max)
		r = uniform_walk(sum, init, acc);
	else if (fast)
		r = walk_packet([&](uint32_t i) { return i < nwords ? sm.words[i] : 0u; }, size, init, pp,
		                [](uint32_t, uint32_t, uint32_t) {});
	else
		r = walk_packet([&](uint32_t i) { return i < nwords ? __ldg(pp.data + first + i) : 0u; }, size, init, pp,
		                [](uint32_t, uint32_t, uint32_t) {});
	pp.tables[(size_t(p) * 9 + init) * 2 + 0] = r.state | (r.error ? 16u : 0u) | (r.restart << 8);
	pp.tables[(size_t(p) * 9 + init) * 2 + 1] = r.total;
	}
	// The last CTA to finish scans every packet's table (threadfence reduction:
	// no CTA waits for another).
	__shared__ uint32_t s_ticket;
	__threadfence();
	__syncthreads();
	if (threadIdx.x == 0)
		s_ticket = atomicAdd(pp.counter, 1u);
	__syncthreads();
	if (s_ticket != uint32_t(pp.count) - 1)
		return;
	__threadfence();
	if (threadIdx.x == 0)
		*pp.counter = 0; // ready for the next call
	scan_packets(pp);
}


__global__ void __launch_bounds__(256) packet_blocks_kernel(const PacketParams pp)
{
	const int p = blockIdx.x;
	uint32_t first = 0, size = 0;
	const bool ok = packet_span(pp, p, first, size);
	const uint32_t nwords = (size + 3) / 4;
	pdl_wait();
	const uint32_t rp = __ldcg(&pp.status->restart_packet), ri = __ldcg(&pp.status->restart_item);
	const uint32_t seq = __ldcg(&pp.status->sequence);
	if (!ok || seq == 0xffffffffu || uint32_t(p) < rp)
		return; // uniform over the CTA
	const uint32_t state = pp.state_before[p];
	const ItemSummary sum = reinterpret_cast<const ItemSummary *>(pp.summaries)[p];
	__shared__ uint32_t s_new;
	if (threadIdx.x == 0)
		s_new = 0;
	__syncthreads();
	uint32_t fresh = 0; // blocks this thread saw first
	auto keep = [&](uint32_t block, uint32_t pos, uint32_t item) {
		if (uint32_t(p) == rp && item < ri)
			return; // before the last restart: cleared
		const unsigned long long key = (unsigned long long)p << 44 | (unsigned long long)item << 30 | (first + pos);
		if (atomicMin(pp.first + block, key) == kNoKey)
			fresh++;
	};
	if (sum.fast && sum.seq_min == sum.seq_max)
	{
		bool accepts;
		(void)uniform_walk(sum, state, accepts);
		const uint32_t err_item = sum.error == ~0u ? ~0u : sum.error >> 2;
		const uint32_t n = accepts ? min(sum.nitems, err_item) : 0u;
		for (uint32_t k = threadIdx.x; k < n; k += blockDim.x)
		{
			const uint32_t q = __ldcg(pp.items + first + k);
			if (q + 1 >= nwords)
				continue;
			const uint32_t w0 = __ldg(pp.data + first + q), w1 = __ldg(pp.data + first + q + 1);
			const uint32_t block = (w1 >> 8) & 0xffffffu;
			if (((w0 >> 31) & 1u) || block >= uint32_t(pp.block_count))
				continue; // a sequence header
			keep(block, q, k);
		}
	}
	else if (threadIdx.x == 0)
		walk_packet([&](uint32_t i) { return i < nwords ? __ldg(pp.data + first + i) : 0u; }, size, state, pp, keep);
	if (fresh)
		atomicAdd(&s_new, fresh);
	__syncthreads();
	if (threadIdx.x == 0 && s_new)
		atomicAdd(&pp.status->decoded_blocks, s_new);
}

} // namespace

void launch_packet_assembly(const PacketParams &pp, cudaStream_t stream)
{
	cudaFuncSetAttribute(packet_tables_kernel, cudaFuncAttributeMaxDynamicSharedMemorySize, int(kPacketSmemBytes));
	{
		LaunchConfig lc(dim3(pp.count), dim3(kPacketThreads), stream, false);
		lc.cfg.dynamicSmemBytes = kPacketSmemBytes;
		cudaLaunchKernelEx(&lc.cfg, packet_tables_kernel, pp);
	}
	{
		LaunchConfig lc(dim3(pp.count), dim3(256), stream, true);
		cudaLaunchKernelEx(&lc.cfg, packet_blocks_kernel, pp);
	}
}
} // namespace pw
