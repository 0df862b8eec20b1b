// YUV4MPEG2 reader and writer (reference yuv4mpeg.cpp:45-245).
#include "y4m.hpp"

#include <stdlib.h>
#include <string.h>

namespace pwcli
{
namespace
{
constexpr size_t kMaxLine = 4096; // header and FRAME lines longer than this are rejected

// Reads up to '\n' (not stored). False at end of file before any character;
// `too_long` is set when no '\n' came within kMaxLine characters.
bool read_line(FILE *f, std::string &line, bool &too_long)
{
	line.clear();
	too_long = false;
	int c;
	bool any = false;
	while ((c = fgetc(f)) != EOF)
	{
		any = true;
		if (c == '\n')
			return true;
		if (line.size() >= kMaxLine)
		{
			too_long = true;
			return true;
		}
		line += char(c);
	}
	return any;
}

bool parse_int(const std::string &s, int &out)
{
	if (s.empty())
		return false;
	char *end = nullptr;
	const long v = strtol(s.c_str(), &end, 10);
	if (*end != '\0' || v <= 0 || v > 1 << 20)
		return false;
	out = int(v);
	return true;
}
} // namespace

bool format_is_16bit(Y4mFormat f) { return f == Y4mFormat::YUV420P16 || f == Y4mFormat::YUV444P16; }
bool format_is_420(Y4mFormat f) { return f == Y4mFormat::YUV420P || f == Y4mFormat::YUV420P16; }

void plane_dims(const Y4mInfo &info, int plane, int &w, int &h)
{
	w = info.width;
	h = info.height;
	if (plane > 0 && format_is_420(info.format))
	{
		w = (w + 1) / 2;
		h = (h + 1) / 2;
	}
}

size_t frame_bytes(const Y4mInfo &info)
{
	size_t n = 0;
	for (int p = 0; p < 3; p++)
	{
		int w, h;
		plane_dims(info, p, w, h);
		n += size_t(w) * size_t(h) * (format_is_16bit(info.format) ? 2 : 1);
	}
	return n;
}

bool parse_params(const std::string &params, Y4mInfo &info, std::string &error)
{
	info = Y4mInfo{};
	bool have_w = false, have_h = false;
	size_t pos = 0;
	while (pos < params.size())
	{
		const size_t end = std::min(params.find(' ', pos), params.size());
		const std::string tok = params.substr(pos, end - pos);
		pos = end + 1;
		if (tok.empty())
			continue;
		const std::string val = tok.substr(1);
		switch (tok[0])
		{
		case 'W':
			if (!parse_int(val, info.width))
			{
				error = "invalid width tag '" + tok + "'";
				return false;
			}
			have_w = true;
			break;
		case 'H':
			if (!parse_int(val, info.height))
			{
				error = "invalid height tag '" + tok + "'";
				return false;
			}
			have_h = true;
			break;
		case 'F':
		{
			const size_t colon = val.find(':');
			if (colon == std::string::npos || !parse_int(val.substr(0, colon), info.frame_rate_num) ||
			    !parse_int(val.substr(colon + 1), info.frame_rate_den))
			{
				error = "invalid frame rate tag '" + tok + "'";
				return false;
			}
			break;
		}
		case 'C':
			if (val == "420" || val == "420jpeg" || val == "420paldv" || val == "420mpeg2")
				info.format = Y4mFormat::YUV420P;
			else if (val == "444")
				info.format = Y4mFormat::YUV444P;
			else if (val == "420p10" || val == "420p12" || val == "420p14" || val == "420p16")
			{
				info.format = Y4mFormat::YUV420P16;
				info.bit_depth = atoi(val.c_str() + 4);
			}
			else if (val == "444p10" || val == "444p12" || val == "444p14" || val == "444p16")
			{
				info.format = Y4mFormat::YUV444P16;
				info.bit_depth = atoi(val.c_str() + 4);
			}
			else
			{
				error = "unsupported chroma format '" + tok + "' (4:2:0 and 4:4:4 only)";
				return false;
			}
			break;
		case 'X':
			if (tok == "XCOLORRANGE=FULL")
				info.full_range = true;
			else if (tok == "XCOLORRANGE=LIMITED")
				info.full_range = false;
			break;
		default:
			break; // interlacing, aspect ratio and other tags do not change the planes
		}
	}
	info.center_chroma = params.find("jpeg") != std::string::npos || params.find("JPEG") != std::string::npos;
	if (!have_w || !have_h)
	{
		error = "header has no W or H tag";
		return false;
	}
	return true;
}

Y4mReader::~Y4mReader()
{
	if (file_)
		fclose(file_);
}

bool Y4mReader::open(const char *path, std::string &error)
{
	file_ = fopen(path, "rb");
	if (!file_)
	{
		error = std::string("cannot open ") + path;
		return false;
	}
	char magic[10];
	if (fread(magic, 1, sizeof(magic), file_) != sizeof(magic) || memcmp(magic, "YUV4MPEG2 ", sizeof(magic)) != 0)
	{
		error = std::string(path) + " is not a YUV4MPEG2 stream";
		return false;
	}
	std::string params;
	bool too_long;
	if (!read_line(file_, params, too_long) || too_long)
	{
		error = "unterminated or overlong YUV4MPEG2 header";
		return false;
	}
	return parse_params(params, info_, error);
}

bool Y4mReader::read_frame(std::vector<uint8_t> (&planes)[3], std::string &error)
{
	error.clear();
	std::string line;
	bool too_long;
	if (!read_line(file_, line, too_long))
		return false; // end of stream
	if (too_long || !(line == "FRAME" || line.compare(0, 6, "FRAME ") == 0))
	{
		error = "expected a FRAME line";
		return false;
	}
	const size_t bpc = format_is_16bit(info_.format) ? 2 : 1;
	for (int p = 0; p < 3; p++)
	{
		int w, h;
		plane_dims(info_, p, w, h);
		planes[p].resize(size_t(w) * size_t(h) * bpc);
		if (fread(planes[p].data(), 1, planes[p].size(), file_) != planes[p].size())
		{
			error = "stream ends inside a frame";
			return false;
		}
		if (bpc == 2 && info_.bit_depth < 16)
		{
			// Up-convert to 16 bits (yuv4mpeg.cpp:191-213): min(1, v / max) * 65535, rounded.
			const float max_code = float((1 << info_.bit_depth) - 1);
			for (size_t i = 0; i + 1 < planes[p].size(); i += 2)
			{
				const uint32_t v = uint32_t(planes[p][i]) | (uint32_t(planes[p][i + 1]) << 8);
				const float f = float(v) / max_code;
				const uint32_t u = uint32_t((f < 1.0f ? f : 1.0f) * 65535.0f + 0.5f);
				planes[p][i] = uint8_t(u);
				planes[p][i + 1] = uint8_t(u >> 8);
			}
		}
	}
	return true;
}

Y4mWriter::~Y4mWriter() { close(); }

bool Y4mWriter::open(const char *path, const Y4mInfo &info, std::string &error)
{
	file_ = fopen(path, "wb");
	if (!file_)
	{
		error = std::string("cannot create ") + path;
		return false;
	}
	const char *chroma = info.format == Y4mFormat::YUV444P     ? "C444"
	                     : info.format == Y4mFormat::YUV420P16 ? "C420p16"
	                     : info.format == Y4mFormat::YUV444P16 ? "C444p16"
	                                                           : "C420";
	// The tags the reference's decoder writes (decode.cpp:196-197).
	if (fprintf(file_, "YUV4MPEG2 W%d H%d F%d:%d Ip A1:1 XCOLORRANGE=%s %s\n", info.width, info.height,
	            info.frame_rate_num, info.frame_rate_den, info.full_range ? "FULL" : "LIMITED", chroma) < 0)
	{
		error = std::string("cannot write ") + path;
		return false;
	}
	return true;
}

bool Y4mWriter::write_frame(const std::vector<uint8_t> (&planes)[3])
{
	if (!file_ || fwrite("FRAME\n", 1, 6, file_) != 6)
		return false;
	for (const auto &p : planes)
		if (fwrite(p.data(), 1, p.size(), file_) != p.size())
			return false;
	return true;
}

bool Y4mWriter::close()
{
	if (!file_)
		return true;
	const bool ok = fclose(file_) == 0;
	file_ = nullptr;
	return ok;
}
} // namespace pwcli
