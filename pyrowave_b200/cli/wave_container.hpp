// The .pyrowave file the reference's command-line tools write and read
// (encode.cpp:144-165,117-125; decode.cpp:124-145,162-190):
//
//   "PYROWAVE"                        8-byte magic
//   int32 params[8]                   width, height, YUV4MPEG2 format (Y4mFormat),
//                                     chroma (0 = 4:2:0, 1 = 4:4:4), full range (0/1),
//                                     frame rate numerator, denominator, 0 (reserved:
//                                     chroma siting)
//   per packet: uint32 size, then `size` bytes of one packetized frame or part
//
// All integers are little-endian. The encoder writes each frame as one packet
// (the whole packetized frame); the decoder accepts frames split over several
// packets, feeding packets to the parser until a frame is complete.
#pragma once

#include <stdint.h>
#include <stdio.h>

#include <string>
#include <vector>

#include "y4m.hpp"

namespace pwcli
{
struct WaveHeader
{
	int32_t width = 0;
	int32_t height = 0;
	Y4mFormat format = Y4mFormat::YUV420P;
	int32_t chroma = 0; // 0 = 4:2:0, 1 = 4:4:4
	bool full_range = false;
	int32_t frame_rate_num = 60;
	int32_t frame_rate_den = 1;
};

bool write_wave_header(FILE *f, const WaveHeader &h);
// False with a message on a bad magic, a short header or invalid fields.
bool read_wave_header(FILE *f, WaveHeader &h, std::string &error);
bool write_wave_packet(FILE *f, const void *data, uint32_t size);
// Returns false at the end of the file (`error` empty) or on a truncated
// packet (`error` set).
bool read_wave_packet(FILE *f, std::vector<uint8_t> &data, std::string &error);
} // namespace pwcli
