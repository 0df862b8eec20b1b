// .pyrowave container (reference encode.cpp:117-165, decode.cpp:124-190).
#include "wave_container.hpp"

#include <string.h>

#include <algorithm>

namespace pwcli
{
namespace
{
void put_le32(uint8_t *p, uint32_t v)
{
	for (int i = 0; i < 4; i++)
		p[i] = uint8_t(v >> (8 * i));
}

uint32_t get_le32(const uint8_t *p)
{
	return uint32_t(p[0]) | (uint32_t(p[1]) << 8) | (uint32_t(p[2]) << 16) | (uint32_t(p[3]) << 24);
}
} // namespace

bool write_wave_header(FILE *f, const WaveHeader &h)
{
	uint8_t buf[8 + 32];
	memcpy(buf, "PYROWAVE", 8);
	const int32_t params[8] = {h.width, h.height, int32_t(h.format), h.chroma, h.full_range ? 1 : 0,
	                           h.frame_rate_num, h.frame_rate_den, 0};
	for (int i = 0; i < 8; i++)
		put_le32(buf + 8 + 4 * i, uint32_t(params[i]));
	return fwrite(buf, 1, sizeof(buf), f) == sizeof(buf);
}

bool read_wave_header(FILE *f, WaveHeader &h, std::string &error)
{
	uint8_t buf[8 + 32];
	if (fread(buf, 1, sizeof(buf), f) != sizeof(buf))
	{
		error = "file is shorter than a .pyrowave header";
		return false;
	}
	if (memcmp(buf, "PYROWAVE", 8) != 0)
	{
		error = "not a .pyrowave file (bad magic)";
		return false;
	}
	int32_t p[8];
	for (int i = 0; i < 8; i++)
		p[i] = int32_t(get_le32(buf + 8 + 4 * i));
	h.width = p[0];
	h.height = p[1];
	h.chroma = p[3];
	h.full_range = p[4] != 0;
	h.frame_rate_num = p[5];
	h.frame_rate_den = p[6];
	if (h.width <= 0 || h.height <= 0 || h.width > 16384 || h.height > 16384)
	{
		error = "invalid frame size in the header";
		return false;
	}
	if (p[2] < 0 || p[2] > 3)
	{
		error = "invalid YUV4MPEG2 format in the header";
		return false;
	}
	h.format = Y4mFormat(p[2]);
	if (h.chroma != 0 && h.chroma != 1)
	{
		error = "invalid chroma subsampling in the header";
		return false;
	}
	if ((h.chroma == 0) != format_is_420(h.format))
	{
		error = "header chroma subsampling and format disagree";
		return false;
	}
	return true;
}

bool write_wave_packet(FILE *f, const void *data, uint32_t size)
{
	uint8_t len[4];
	put_le32(len, size);
	return fwrite(len, 1, 4, f) == 4 && fwrite(data, 1, size, f) == size;
}

bool read_wave_packet(FILE *f, std::vector<uint8_t> &data, std::string &error)
{
	error.clear();
	uint8_t len[4];
	const size_t got = fread(len, 1, 4, f);
	if (got == 0)
		return false; // end of file
	if (got != 4)
	{
		error = "truncated packet size";
		return false;
	}
	const uint32_t size = get_le32(len);
	// Read in pieces so that a corrupt size fails at the end of the file
	// instead of allocating it up front.
	constexpr size_t kPiece = size_t(1) << 20;
	data.clear();
	size_t done = 0;
	while (done < size)
	{
		const size_t n = std::min<size_t>(kPiece, size - done);
		data.resize(done + n);
		if (fread(data.data() + done, 1, n, f) != n)
		{
			error = "truncated packet";
			return false;
		}
		done += n;
	}
	return true;
}
} // namespace pwcli
