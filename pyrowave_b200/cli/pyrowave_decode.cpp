// pyrowave-decode <input.pyrowave> <output.y4m>
//
// The reference's decoder tool (decode.cpp:162-287) over this library's C API:
// packets of the .pyrowave container go to the decoder's parser until a frame
// is complete; each complete frame is decoded and appended to the YUV4MPEG2
// output. A frame that the file ends inside is dropped, as in the reference; a
// packet cut short by the end of the file is an error, reported after the
// complete frames before it are written. Messages go to stderr; the exit status
// is 0 on success and 1 on any error (the reference prints the error and exits
// 0). The output header carries the reference decoder's tags
// (decode.cpp:196-197) after a single "YUV4MPEG2 " magic (the reference writes
// the magic twice; readers take either).
#include <stdint.h>
#include <stdio.h>

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
	fprintf(stderr, "pyrowave-decode: %s\n", msg.c_str());
	return 1;
}

struct Session
{
	pyrowave_device device = nullptr;
	pyrowave_decoder decoder = nullptr;
	FILE *in = nullptr;
	~Session()
	{
		if (in)
			fclose(in);
		pyrowave_decoder_destroy(decoder);
		pyrowave_device_destroy(device);
	}
};
} // namespace

int main(int argc, char **argv)
{
	if (argc != 3)
	{
		fprintf(stderr, "Usage: pyrowave-decode <input.pyrowave> <output.y4m>\n");
		return 1;
	}
	Session s;
	s.in = fopen(argv[1], "rb");
	if (!s.in)
		return fail(std::string("cannot open ") + argv[1]);
	WaveHeader wh;
	std::string error;
	if (!read_wave_header(s.in, wh, error))
		return fail(error);
	const bool wide = format_is_16bit(wh.format);
	if (wh.chroma == 0 && ((wh.width | wh.height) & 1))
		return fail("4:2:0 streams need an even width and height");

	if (pyrowave_create_default_device(&s.device) != PYROWAVE_SUCCESS)
		return fail("no CUDA device");
	pyrowave_decoder_create_info ci = {};
	ci.device = s.device;
	ci.width = wh.width;
	ci.height = wh.height;
	ci.chroma = wh.chroma == 0 ? PYROWAVE_CHROMA_SUBSAMPLING_420 : PYROWAVE_CHROMA_SUBSAMPLING_444;
	ci.fragment_path = false;
	if (pyrowave_decoder_create(&ci, &s.decoder) != PYROWAVE_SUCCESS)
		return fail("cannot create a decoder for this frame size");

	Y4mInfo info;
	info.width = wh.width;
	info.height = wh.height;
	info.format = wh.format;
	info.bit_depth = wide ? 16 : 8;
	info.full_range = wh.full_range;
	info.frame_rate_num = wh.frame_rate_num;
	info.frame_rate_den = wh.frame_rate_den;
	Y4mWriter output;
	if (!output.open(argv[2], info, error))
		return fail(error);

	std::vector<uint8_t> planes[3];
	for (int p = 0; p < 3; p++)
	{
		int w, h;
		plane_dims(info, p, w, h);
		planes[p].assign(size_t(w) * size_t(h) * (wide ? 2 : 1), 0);
	}
	std::vector<uint8_t> packet;
	size_t frames = 0, packets = 0;
	for (;;)
	{
		if (!read_wave_packet(s.in, packet, error))
		{
			if (!error.empty())
			{
				output.close(); // the complete frames before the damage stay in the output
				return fail(error + " after " + std::to_string(frames) + " frames");
			}
			break;
		}
		packets++;
		if (pyrowave_decoder_push_packet(s.decoder, packet.data(), packet.size()) != PYROWAVE_SUCCESS)
			return fail("malformed packet " + std::to_string(packets - 1));
		if (!pyrowave_decoder_decode_is_ready(s.decoder, false))
			continue;
		pyrowave_cpu_buffer buf = {};
		for (int p = 0; p < 3; p++)
		{
			int w, h;
			plane_dims(info, p, w, h);
			buf.data[p] = planes[p].data();
			buf.row_stride_in_bytes[p] = size_t(w) * (wide ? 2 : 1);
			buf.plane_size_in_bytes[p] = planes[p].size();
		}
		buf.width = wh.width;
		buf.height = wh.height;
		if (wide)
			buf.format = wh.chroma == 0 ? PYROWAVE_CPU_BUFFER_FORMAT_YUV420P16 : PYROWAVE_CPU_BUFFER_FORMAT_YUV444P16;
		else
			buf.format = wh.chroma == 0 ? PYROWAVE_CPU_BUFFER_FORMAT_YUV420P : PYROWAVE_CPU_BUFFER_FORMAT_YUV444P;
		if (pyrowave_decoder_decode_cpu_buffer_synchronous(s.decoder, &buf) != PYROWAVE_SUCCESS)
			return fail("decode failed at frame " + std::to_string(frames));
		if (!output.write_frame(planes))
			return fail(std::string("cannot write ") + argv[2]);
		frames++;
	}
	if (!output.close())
		return fail(std::string("cannot write ") + argv[2]);
	fprintf(stderr, "pyrowave-decode: %zu frames from %zu packets\n", frames, packets);
	return 0;
}
