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
// The reference up-converts 10- to 16-bit streams (C420p10 ... C444p16) to 16-bit
// planes; this library codes 8-bit planes only, so those streams are reported as
// unsupported. Other chroma tags (C422, Cmono, C444alpha), which the reference
// reads as 4:2:0 or 4:4:4 planes of the wrong size, are rejected.
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
};

bool format_is_16bit(Y4mFormat f);
bool format_is_420(Y4mFormat f);

// Plane sizes of one 8-bit frame (4:2:0 chroma rounds up, as YUV4MPEG2 does).
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
	// Reads the next frame into planes[3] (resized as needed). Returns false at
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
