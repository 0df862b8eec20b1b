// pyrowave-encode <input.y4m> <output.pyrowave> <bytes_per_frame>
//
// The reference's encoder tool (encode.cpp:128-261) over this library's C API:
// every frame of a 4:2:0 or 4:4:4 YUV4MPEG2 stream, 8-bit or 10- to 16-bit
// (coded from 16-bit planes, encode.cpp:152), is encoded at the given byte
// budget and written to the .pyrowave container as one packet.
// Messages go to stderr; the exit status is 0 on success and 1 on any error
// (the reference prints the error and exits 0).
#include <stdint.h>
#include <stdio.h>
#include <stdlib.h>

#include <string>
#include <vector>

#include "pyrowave.h"
#include "pyrowave_cuda.h"
#include "wave_container.hpp"
#include "y4m.hpp"

using namespace pwcli;

namespace
{
int fail(const std::string &msg)
{
	fprintf(stderr, "pyrowave-encode: %s\n", msg.c_str());
	return 1;
}

struct Session
{
	pyrowave_device device = nullptr;
	pyrowave_encoder encoder = nullptr;
	FILE *out = nullptr;
	~Session()
	{
		if (out)
			fclose(out);
		pyrowave_encoder_destroy(encoder);
		pyrowave_device_destroy(device);
	}
};
} // namespace

int main(int argc, char **argv)
{
	if (argc != 4)
	{
		fprintf(stderr, "Usage: pyrowave-encode <input.y4m> <output.pyrowave> <bytes_per_frame>\n");
		return 1;
	}
	char *end = nullptr;
	const unsigned long long budget = strtoull(argv[3], &end, 0);
	if (!end || *end != '\0' || budget < 8 || budget > 0xffffffffull)
		return fail("bytes_per_frame must be an integer from 8 to 4294967295");

	Y4mReader input;
	std::string error;
	if (!input.open(argv[1], error))
		return fail(error);
	const Y4mInfo &info = input.info();
	const bool wide = format_is_16bit(info.format);
	const bool c420 = format_is_420(info.format);
	if (c420 && ((info.width | info.height) & 1))
		return fail("4:2:0 input needs an even width and height");

	Session s;
	if (pyrowave_create_default_device(&s.device) != PYROWAVE_SUCCESS)
		return fail("no CUDA device");
	pyrowave_encoder_create_info ci = {};
	ci.device = s.device;
	ci.width = info.width;
	ci.height = info.height;
	ci.chroma = c420 ? PYROWAVE_CHROMA_SUBSAMPLING_420 : PYROWAVE_CHROMA_SUBSAMPLING_444;
	if (pyrowave_encoder_create(&ci, &s.encoder) != PYROWAVE_SUCCESS)
		return fail("cannot create an encoder for this frame size");

	s.out = fopen(argv[2], "wb");
	if (!s.out)
		return fail(std::string("cannot create ") + argv[2]);
	WaveHeader wh;
	wh.width = info.width;
	wh.height = info.height;
	// 10- to 14-bit streams were up-converted to 16 bits, so the container
	// records the 16-bit format of the same chroma (as the reference does).
	wh.format = info.format;
	wh.chroma = c420 ? 0 : 1;
	wh.full_range = info.full_range;
	wh.frame_rate_num = info.frame_rate_num;
	wh.frame_rate_den = info.frame_rate_den;
	if (!write_wave_header(s.out, wh))
		return fail(std::string("cannot write ") + argv[2]);

	std::vector<uint8_t> planes[3];
	std::vector<uint8_t> bitstream(size_t(budget) + 64);
	const pyrowave_rate_control rc = {size_t(budget)};
	// A boundary past the budget: the whole frame is one packet (the reference
	// packetizes with its payload buffer's size, encode.cpp:108-116).
	const size_t boundary = bitstream.size();
	size_t frames = 0, total_bytes = 0;
	for (;;)
	{
		if (!input.read_frame(planes, error))
		{
			if (!error.empty())
				return fail(error + " (after " + std::to_string(frames) + " frames)");
			break;
		}
		pyrowave_cpu_buffer buf = {};
		for (int p = 0; p < 3; p++)
		{
			int w, h;
			plane_dims(info, p, w, h);
			buf.data[p] = planes[p].data();
			buf.row_stride_in_bytes[p] = size_t(w) * (wide ? 2 : 1);
			buf.plane_size_in_bytes[p] = planes[p].size();
		}
		buf.width = info.width;
		buf.height = info.height;
		if (wide)
			buf.format = c420 ? PYROWAVE_CPU_BUFFER_FORMAT_YUV420P16 : PYROWAVE_CPU_BUFFER_FORMAT_YUV444P16;
		else
			buf.format = c420 ? PYROWAVE_CPU_BUFFER_FORMAT_YUV420P : PYROWAVE_CPU_BUFFER_FORMAT_YUV444P;
		if (pyrowave_encoder_encode_cpu_synchronous(s.encoder, &buf, &rc) != PYROWAVE_SUCCESS)
			return fail("encode failed at frame " + std::to_string(frames));
		size_t num_packets = 0, got = 0;
		if (pyrowave_encoder_compute_num_packets(s.encoder, boundary, &num_packets) != PYROWAVE_SUCCESS ||
		    num_packets != 1)
			return fail("packet count failed at frame " + std::to_string(frames));
		pyrowave_packet packet = {};
		if (pyrowave_encoder_packetize(s.encoder, &packet, boundary, &got, bitstream.data(), bitstream.size()) !=
		        PYROWAVE_SUCCESS ||
		    got != 1 || packet.offset + packet.size > bitstream.size())
			return fail("packetize failed at frame " + std::to_string(frames));
		if (!write_wave_packet(s.out, bitstream.data() + packet.offset, uint32_t(packet.size)))
			return fail(std::string("cannot write ") + argv[2]);
		frames++;
		total_bytes += packet.size;
	}
	if (fclose(s.out) != 0)
	{
		s.out = nullptr;
		return fail(std::string("cannot write ") + argv[2]);
	}
	s.out = nullptr;
	fprintf(stderr, "pyrowave-encode: %zu frames, %.1f bytes per frame\n", frames,
	        frames ? double(total_bytes) / double(frames) : 0.0);
	return 0;
}
