// Serving loop: continuous batching of encode + decode requests from many
// video streams on one GPU, built on the library's own C API.
//
// Each stream's device state is a working set: a pyrowave_encoder and a
// pyrowave_decoder with their device buffers and captured graphs. It stays
// resident between the stream's frames. Requests wait in per-stream FIFO
// queues and are admitted by memory: a request whose stream has no working set
// starts only when the pool has room for one, after releasing the working sets
// of idle streams, least recently used first, if needed; otherwise it waits
// until a running request completes. A dispatcher thread starts the head
// request of every idle stream as soon as one of the server's CUDA streams is
// free and admission allows, and completes requests by polling one event per
// CUDA stream, so requests that arrive while others run are admitted at once
// and their kernels overlap on the device.
#include "pw_internal.h"

#include "pyrowave.h"
#include "pyrowave_cuda.h"

#include <algorithm>
#include <atomic>
#include <chrono>
#include <condition_variable>
#include <cstring>
#include <deque>
#include <map>
#include <memory>
#include <mutex>
#include <new>
#include <thread>
#include <vector>

using namespace pw;

namespace
{
using Clock = std::chrono::steady_clock;

// Device bytes an encoder and a decoder of this frame hold once allocated
// (the allocations of the encoder and decoder objects).
size_t stream_state_bytes(const Geometry &g, size_t capacity_words)
{
	const size_t n8 = size_t(g.block_count_8x8), n32 = size_t(g.block_count_32x32);
	const size_t coef = size_t(g.storage_elems32) * 4 + size_t(g.storage_elems16) * 2;
	const size_t enc = coef + n8 * 4 + n32 * (1024 * 2 + 16 * 2 + 16 + 16 * 4 + 4 + 8 + 4 + 4) + sizeof(RateControlState) +
	                   capacity_words * 4;
	const size_t dec = coef + n32 * 8;
	return enc + dec;
}

struct Request
{
	uint64_t id = 0;
	uint32_t stream = 0;
	pyrowave_cuda_planes input = {}, output = {};
	bool decode = false;
	size_t budget = 0;
	Clock::time_point submitted;
};

struct VideoStream
{
	uint32_t id = 0;
	int width = 0, height = 0;
	pyrowave_chroma_subsampling chroma = PYROWAVE_CHROMA_SUBSAMPLING_420;
	// Working set (null while released); `bytes` is what it takes from the pool.
	pyrowave_encoder encoder = nullptr;
	pyrowave_decoder decoder = nullptr;
	size_t bytes = 0;
	uint32_t frames = 0;    // frames encoded (mod 8): carried over when the working set is re-created
	uint64_t last_use = 0;  // admission tick of the last frame (least recently used release order)
	std::deque<Request> queue;
	bool busy = false;    // a frame of this stream is on the GPU
	bool closing = false; // free once the queue drains
};

struct Slot
{
	cudaStream_t stream = nullptr;
	cudaEvent_t done = nullptr;
	bool busy = false;
	Request req;
};
} // namespace

struct pyrowave_cuda_server_opaque
{
	pyrowave_device device = nullptr;
	size_t pool = 0, used = 0;
	std::vector<Slot> slots;
	std::map<uint32_t, std::unique_ptr<VideoStream>> streams;
	uint32_t next_stream = 1;
	uint64_t next_request = 1;
	uint64_t tick = 0;
	size_t peak_used = 0;
	uint64_t releases = 0; // working sets released to admit another stream's request
	std::deque<pyrowave_cuda_server_completion> completed;
	// Finished requests not yet polled plus requests not yet finished: submit
	// refuses new requests beyond this, so a caller that never polls cannot grow
	// the completion queue without bound.
	static constexpr size_t kMaxOutstanding = size_t(1) << 20;
	// Latencies since the last stats reset: the most recent kLatencySamples in a
	// ring, so a server that never resets its statistics stays bounded.
	static constexpr size_t kLatencySamples = size_t(1) << 20;
	std::vector<double> latencies;
	size_t latency_next = 0;     // ring position once the ring is full
	uint64_t finished_since_reset = 0;
	std::mutex lock;
	std::condition_variable wake, done_cv;
	std::atomic<bool> stop{false};
	size_t pending = 0; // queued + in flight
	std::thread dispatcher;

	// Releases a stream's working set (its encoder and decoder) back to the pool.
	void release_working_set(VideoStream &vs)
	{
		if (!vs.encoder && !vs.decoder)
			return;
		vs.frames = encoder_frames(vs.encoder);
		if (vs.encoder)
			pyrowave_encoder_destroy(vs.encoder);
		if (vs.decoder)
			pyrowave_decoder_destroy(vs.decoder);
		vs.encoder = nullptr;
		vs.decoder = nullptr;
		used -= vs.bytes;
	}

	// Admission by memory (called with the lock held): gives the stream a
	// working set if it has none, releasing idle streams' working sets (least
	// recently used first) while the pool lacks room. False: the request waits.
	bool admit(VideoStream &vs)
	{
		if (vs.encoder)
			return true;
		while (used + vs.bytes > pool)
		{
			VideoStream *victim = nullptr;
			for (auto &kv : streams)
			{
				VideoStream &o = *kv.second;
				if (&o != &vs && o.encoder && !o.busy && (!victim || o.last_use < victim->last_use))
					victim = &o;
			}
			if (!victim)
				return false;
			release_working_set(*victim);
			releases++;
		}
		pyrowave_encoder_create_info ei = {device, vs.width, vs.height, vs.chroma};
		pyrowave_decoder_create_info di = {};
		di.device = device;
		di.width = vs.width;
		di.height = vs.height;
		di.chroma = vs.chroma;
		if (pyrowave_encoder_create(&ei, &vs.encoder) != PYROWAVE_SUCCESS ||
		    pyrowave_decoder_create(&di, &vs.decoder) != PYROWAVE_SUCCESS)
		{
			if (vs.encoder)
				pyrowave_encoder_destroy(vs.encoder);
			vs.encoder = nullptr;
			vs.decoder = nullptr;
			return false;
		}
		encoder_set_frames(vs.encoder, vs.frames);
		used += vs.bytes;
		peak_used = std::max(peak_used, used);
		return true;
	}

	// Start a request on a free slot (called with the lock held, after admit()).
	void start(Slot &slot, VideoStream &vs)
	{
		vs.last_use = ++tick;
		Request r = vs.queue.front();
		vs.queue.pop_front();
		vs.busy = true;
		slot.busy = true;
		slot.req = r;
		pyrowave_rate_control rc = {r.budget};
		const pyrowave_cuda_stream s = reinterpret_cast<pyrowave_cuda_stream>(slot.stream);
		pyrowave_result res = pyrowave_cuda_encoder_encode(vs.encoder, &r.input, &rc, s);
		if (res == PYROWAVE_SUCCESS && r.decode)
		{
			const uint32_t *words = nullptr, *meta = nullptr;
			size_t cap = 0;
			res = pyrowave_cuda_encoder_get_device_bitstream(vs.encoder, &words, &meta, &cap);
			if (res == PYROWAVE_SUCCESS)
				res = pyrowave_cuda_decoder_decode_blocks(vs.decoder, meta, words + 2, cap - 2, &r.output, s);
		}
		if (res != PYROWAVE_SUCCESS)
			finish(slot, vs, res);
		else
			cudaEventRecord(slot.done, slot.stream);
	}

	// Complete the slot's request (called with the lock held).
	void finish(Slot &slot, VideoStream &vs, pyrowave_result res)
	{
		pyrowave_cuda_server_completion c = {};
		c.request_id = slot.req.id;
		c.stream_id = vs.id;
		c.result = res;
		if (res == PYROWAVE_SUCCESS)
		{
			size_t bytes = 0;
			c.result = pyrowave_cuda_encoder_get_size(vs.encoder, &bytes);
			c.bytes = bytes;
			// The decode's own outcome (its event completed with the slot's).
			if (c.result == PYROWAVE_SUCCESS && slot.req.decode)
				c.result = pyrowave_cuda_decoder_get_error(vs.decoder, nullptr);
		}
		c.latency_us = std::chrono::duration<double, std::micro>(Clock::now() - slot.req.submitted).count();
		completed.push_back(c);
		if (latencies.size() < kLatencySamples)
			latencies.push_back(c.latency_us);
		else
		{
			latencies[latency_next] = c.latency_us;
			latency_next = (latency_next + 1) % kLatencySamples;
		}
		finished_since_reset++;
		slot.busy = false;
		vs.busy = false;
		pending--;
		done_cv.notify_all();
	}

	void run()
	{
		// This thread starts with device 0 current; the slots' streams, the
		// encoders and their buffers belong to the server's device.
		cudaSetDevice(device_ordinal(device));
		std::unique_lock<std::mutex> g(lock);
		size_t rr = 0; // round-robin start among streams
		while (!stop.load() || pending > 0)
		{
			bool progress = false;
			for (Slot &slot : slots)
			{
				if (!slot.busy)
					continue;
				const cudaError_t q = cudaEventQuery(slot.done);
				if (q == cudaErrorNotReady)
					continue;
				auto it = streams.find(slot.req.stream);
				finish(slot, *it->second, q == cudaSuccess ? PYROWAVE_SUCCESS : PYROWAVE_ERROR_GENERIC);
				(void)cudaGetLastError();
				progress = true;
			}
			// Streams that are closing and drained release their memory.
			for (auto it = streams.begin(); it != streams.end();)
			{
				VideoStream &vs = *it->second;
				if (vs.closing && !vs.busy && vs.queue.empty())
				{
					release_working_set(vs);
					it = streams.erase(it);
					progress = true;
				}
				else
					++it;
			}
			// Admit the head request of idle streams onto free slots.
			if (!streams.empty())
			{
				std::vector<VideoStream *> order;
				order.reserve(streams.size());
				for (auto &kv : streams)
					order.push_back(kv.second.get());
				const size_t n = order.size();
				for (size_t k = 0; k < n; k++)
				{
					VideoStream &vs = *order[(rr + k) % n];
					if (vs.busy || vs.queue.empty())
						continue;
					auto free_slot = std::find_if(slots.begin(), slots.end(), [](const Slot &s) { return !s.busy; });
					if (free_slot == slots.end())
						break;
					if (!admit(vs))
						continue; // no memory until a running request completes
					start(*free_slot, vs);
					progress = true;
				}
				rr++;
			}
			if (!progress)
			{
				// Nothing to do right now: sleep briefly, or until a submission.
				const bool any_busy = std::any_of(slots.begin(), slots.end(), [](const Slot &s) { return s.busy; });
				wake.wait_for(g, std::chrono::microseconds(any_busy ? 10 : 1000));
			}
		}
	}
};

extern "C" {

pyrowave_result pyrowave_cuda_server_create(pyrowave_device device, const pyrowave_cuda_server_info *info,
                                            pyrowave_cuda_server *server)
{
	if (!device || !info || !server || info->max_in_flight == 0 || info->max_in_flight > 64)
		return PYROWAVE_ERROR_INVALID_ARGUMENT;
	auto *sv = new (std::nothrow) pyrowave_cuda_server_opaque;
	if (!sv)
		return PYROWAVE_ERROR_OUT_OF_HOST_MEMORY;
	sv->device = device;
	sv->pool = info->memory_pool_bytes;
	sv->slots.resize(info->max_in_flight);
	int least = 0, greatest = 0;
	cudaDeviceGetStreamPriorityRange(&least, &greatest);
	for (Slot &s : sv->slots)
	{
		if (cudaStreamCreateWithPriority(&s.stream, cudaStreamNonBlocking, greatest) != cudaSuccess ||
		    cudaEventCreateWithFlags(&s.done, cudaEventDisableTiming) != cudaSuccess)
		{
			(void)cudaGetLastError();
			for (Slot &t : sv->slots)
			{
				if (t.stream)
					cudaStreamDestroy(t.stream);
				if (t.done)
					cudaEventDestroy(t.done);
			}
			delete sv;
			return PYROWAVE_ERROR_GENERIC;
		}
	}
	sv->dispatcher = std::thread([sv] { sv->run(); });
	*server = sv;
	return PYROWAVE_SUCCESS;
}

void pyrowave_cuda_server_destroy(pyrowave_cuda_server server)
{
	if (!server)
		return;
	{
		std::lock_guard<std::mutex> g(server->lock);
		server->stop.store(true);
		server->wake.notify_all();
	}
	server->dispatcher.join();
	for (auto &kv : server->streams)
		server->release_working_set(*kv.second);
	for (Slot &s : server->slots)
	{
		cudaStreamDestroy(s.stream);
		cudaEventDestroy(s.done);
	}
	delete server;
}

pyrowave_result pyrowave_cuda_server_open_stream(pyrowave_cuda_server server, int width, int height,
                                                 pyrowave_chroma_subsampling chroma, size_t maximum_bitstream_size,
                                                 uint32_t *stream_id)
{
	if (!server || !stream_id)
		return PYROWAVE_ERROR_INVALID_ARGUMENT;
	const uint64_t target = uint64_t(maximum_bitstream_size) & ~uint64_t(3);
	if (target == 0 || target > 0xffffffffull)
		return PYROWAVE_ERROR_INVALID_ARGUMENT;
	Geometry g;
	if (width <= 0 || height <= 0 ||
	    (chroma != PYROWAVE_CHROMA_SUBSAMPLING_420 && chroma != PYROWAVE_CHROMA_SUBSAMPLING_444) ||
	    (chroma == PYROWAVE_CHROMA_SUBSAMPLING_420 && ((width & 1) || (height & 1))) ||
	    !make_geometry(g, width, height, chroma == PYROWAVE_CHROMA_SUBSAMPLING_444, 0))
		return PYROWAVE_ERROR_INVALID_ARGUMENT;
	const size_t bytes = stream_state_bytes(g, size_t((target >= 8 ? target - 8 : target) / 4) + 2);
	std::lock_guard<std::mutex> guard(server->lock);
	// A stream whose working set can never fit the pool is refused; any other
	// is opened, and its requests are admitted as memory allows.
	if (bytes > server->pool)
		return PYROWAVE_ERROR_OUT_OF_DEVICE_MEMORY;
	auto vs = std::make_unique<VideoStream>();
	vs->width = width;
	vs->height = height;
	vs->chroma = chroma;
	vs->id = server->next_stream++;
	vs->bytes = bytes;
	*stream_id = vs->id;
	server->streams[vs->id] = std::move(vs);
	return PYROWAVE_SUCCESS;
}

pyrowave_result pyrowave_cuda_server_close_stream(pyrowave_cuda_server server, uint32_t stream_id)
{
	if (!server)
		return PYROWAVE_ERROR_INVALID_ARGUMENT;
	std::lock_guard<std::mutex> g(server->lock);
	auto it = server->streams.find(stream_id);
	if (it == server->streams.end() || it->second->closing)
		return PYROWAVE_ERROR_INVALID_ARGUMENT;
	it->second->closing = true;
	server->wake.notify_all();
	return PYROWAVE_SUCCESS;
}

pyrowave_result pyrowave_cuda_server_submit(pyrowave_cuda_server server, uint32_t stream_id,
                                            const pyrowave_cuda_planes *input, size_t budget,
                                            const pyrowave_cuda_planes *output, uint64_t *request_id)
{
	if (!server || !input || budget == 0)
		return PYROWAVE_ERROR_INVALID_ARGUMENT;
	Request r;
	r.stream = stream_id;
	r.input = *input;
	r.decode = output != nullptr;
	if (output)
		r.output = *output;
	r.budget = budget;
	r.submitted = Clock::now();
	std::lock_guard<std::mutex> g(server->lock);
	auto it = server->streams.find(stream_id);
	if (it == server->streams.end() || it->second->closing)
		return PYROWAVE_ERROR_INVALID_ARGUMENT;
	if (server->pending + server->completed.size() >= pyrowave_cuda_server_opaque::kMaxOutstanding)
		return PYROWAVE_ERROR_OUT_OF_HOST_MEMORY; // poll the finished requests first
	r.id = server->next_request++;
	it->second->queue.push_back(r);
	server->pending++;
	if (request_id)
		*request_id = r.id;
	server->wake.notify_all();
	return PYROWAVE_SUCCESS;
}

pyrowave_result pyrowave_cuda_server_poll(pyrowave_cuda_server server, pyrowave_cuda_server_completion *completions,
                                          uint32_t capacity, uint32_t *count, uint32_t timeout_us)
{
	if (!server || !count || (capacity && !completions))
		return PYROWAVE_ERROR_INVALID_ARGUMENT;
	std::unique_lock<std::mutex> g(server->lock);
	if (server->completed.empty() && timeout_us)
		server->done_cv.wait_for(g, std::chrono::microseconds(timeout_us),
		                         [server] { return !server->completed.empty(); });
	uint32_t n = 0;
	while (n < capacity && !server->completed.empty())
	{
		completions[n++] = server->completed.front();
		server->completed.pop_front();
	}
	*count = n;
	return PYROWAVE_SUCCESS;
}

pyrowave_result pyrowave_cuda_server_get_memory(pyrowave_cuda_server server, size_t *used_bytes,
                                                size_t *peak_bytes, uint64_t *releases)
{
	if (!server)
		return PYROWAVE_ERROR_INVALID_ARGUMENT;
	std::lock_guard<std::mutex> g(server->lock);
	if (used_bytes)
		*used_bytes = server->used;
	if (peak_bytes)
		*peak_bytes = server->peak_used;
	if (releases)
		*releases = server->releases;
	return PYROWAVE_SUCCESS;
}

pyrowave_result pyrowave_cuda_server_stats(pyrowave_cuda_server server, double *p50_us, double *p99_us,
                                           uint64_t *frames, bool reset)
{
	if (!server)
		return PYROWAVE_ERROR_INVALID_ARGUMENT;
	std::vector<double> lat;
	uint64_t finished = 0;
	{
		std::lock_guard<std::mutex> g(server->lock);
		lat = server->latencies;
		finished = server->finished_since_reset;
		if (reset)
		{
			server->latencies.clear();
			server->latency_next = 0;
			server->finished_since_reset = 0;
		}
	}
	std::sort(lat.begin(), lat.end());
	auto pct = [&](double p) {
		if (lat.empty())
			return 0.0;
		size_t i = size_t(p * double(lat.size() - 1) + 0.5);
		return lat[std::min(i, lat.size() - 1)];
	};
	if (p50_us)
		*p50_us = pct(0.50);
	if (p99_us)
		*p99_us = pct(0.99);
	if (frames)
		*frames = finished;
	return PYROWAVE_SUCCESS;
}
}
