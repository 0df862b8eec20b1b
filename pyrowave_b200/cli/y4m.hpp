// YUV4MPEG2 streams for the command-line tools: the reader and writer that the
// reference's pyrowave-encode / pyrowave-decode use (yuv4mpeg.hpp,
// yuv4mpeg.cpp), restated for this library's 8-bit planar input and output.
//
// Header: "YUV4MPEG2 " then space-separated tags up to '\n'. W and H are
// required; F<num>:<den> defaults to 60:1; C420* (jpeg, paldv, mpeg2 or none)
// selects 4:2:0 and C444 4:4:4, no C tag means 4:2:0; XCOLORRANGE=FULL or
// LIMITED sets the range flag (limited by default). A tag of "jpeg" marks
// centred chroma. Frames: a "FRAME" line (optionally with tags), then Y, Cb, Cr.
//
// 10- to 16-bit streams (C420p10 ... C444p16; little-endian 16-bit samples)
// are up-converted to full-range 16-bit planes on reading, min(1, v / max) *
// 65535 rounded, max being the stream's largest code (yuv4mpeg.cpp:101-141,
// 191-213), and written back at 16 bits (C420p16 / C444p16, as the reference's
// decoder writes them). The reference up-converts only 4:2:0 streams and reads
// 4:4:4 ones raw; here both are converted. Other chroma tags (C422, Cmono,
// C444alpha), which the reference reads as 4:2:0 or 4:4:4 planes of the wrong
// size, are rejected.
#pragma once

#include <stdint.h>
#include <stdio.h>

#include <string>
#include <vector>

namespace pwcli
{
// Stream formats, with the values the .pyrowave container stores
// (the reference's YUV4MPEGFile::Format, yuv4mpeg.hpp:24-30).
enum class Y4mFormat : int32_t
{
	YUV420P = 0,
	YUV444P = 1,
	YUV420P16 = 2,
	YUV444P16 = 3
};

struct Y4mInfo
{
	int width = 0;
	int height = 0;
	Y4mFormat format = Y4mFormat::YUV420P;
	bool full_range = false;
	bool center_chroma = false;
	int frame_rate_num = 60;
	int frame_rate_den = 1;
	int bit_depth = 8; // 8, or 10 / 12 / 14 / 16 for the 16-bit formats
};

bool format_is_16bit(Y4mFormat f);
bool format_is_420(Y4mFormat f);

// Plane sizes in samples (4:2:0 chroma rounds up, as YUV4MPEG2 does); 16-bit
// formats take two bytes per sample.
void plane_dims(const Y4mInfo &info, int plane, int &w, int &h);
size_t frame_bytes(const Y4mInfo &info);

// Parses a header parameter string (everything after "YUV4MPEG2 "). False with
// a message on a missing or invalid W / H / F or an unsupported chroma tag.
bool parse_params(const std::string &params, Y4mInfo &info, std::string &error);

class Y4mReader
{
public:
	~Y4mReader();
	bool open(const char *path, std::string &error);
	const Y4mInfo &info() const { return info_; }
	// Reads the next frame into planes[3] (resized as needed; 16-bit formats as
	// little-endian 16-bit samples, up-converted to 16 bits). Returns false at
	// the end of the stream; `error` is empty there, and holds a message when
	// the stream is malformed or ends inside a frame.
	bool read_frame(std::vector<uint8_t> (&planes)[3], std::string &error);

private:
	FILE *file_ = nullptr;
	Y4mInfo info_;
};

class Y4mWriter
{
public:
	~Y4mWriter();
	// Writes "YUV4MPEG2 W.. H.. F..:.. Ip A1:1 XCOLORRANGE=.. C420|C444".
	bool open(const char *path, const Y4mInfo &info, std::string &error);
	bool write_frame(const std::vector<uint8_t> (&planes)[3]);
	bool close();

private:
	FILE *file_ = nullptr;
};
} // namespace pwcli
