// Test infrastructure only: the pyrowave.h calls that pyrowave-encode and
// pyrowave-decode make, implemented over the CPU oracle (oracle/liboracle.so),
// so that tests/test_cli.py can run the tools' own sources end to end on a
// machine without a GPU. The argument checks are the library's
// (pyrowave_c.cpp:1058-1088 and :1346-1374 of the reference); the codec is the
// oracle at FP32, which the CUDA library matches bit for bit. Never part of the
// product: the shipped tools link libpyrowave-shared.so.0.
#include <string.h>

#include <vector>

#include "pyrowave.h"
#include "pyrowave_cuda.h"
#include "pyrowave_oracle.h"

struct pyrowave_device_opaque
{
	int unused;
};

struct pyrowave_encoder_opaque
{
	oracle_codec *codec = nullptr;
	int width = 0, height = 0;
	bool c444 = false;
	uint32_t sequence = 0;
	bool encoded = false;
};

struct pyrowave_decoder_opaque
{
	oracle_codec *codec = nullptr;
	oracle_parser *parser = nullptr;
	int width = 0, height = 0;
	bool c444 = false;
};

namespace
{
void plane_dims(bool c444, int w, int h, int p, int &pw, int &ph)
{
	pw = (p == 0 || c444) ? w : w / 2;
	ph = (p == 0 || c444) ? h : h / 2;
}

// Planar 8-bit or 16-bit buffers only; `wide` is set for the 16-bit formats.
bool planes_ok(const pyrowave_cpu_buffer *b, bool c444, int w, int h, bool &wide)
{
	if (!b || b->width != w || b->height != h)
		return false;
	wide = b->format == (c444 ? PYROWAVE_CPU_BUFFER_FORMAT_YUV444P16 : PYROWAVE_CPU_BUFFER_FORMAT_YUV420P16);
	if (!wide && b->format != (c444 ? PYROWAVE_CPU_BUFFER_FORMAT_YUV444P : PYROWAVE_CPU_BUFFER_FORMAT_YUV420P))
		return false;
	for (int p = 0; p < 3; p++)
	{
		int pw, ph;
		plane_dims(c444, w, h, p, pw, ph);
		if (!b->data[p] || b->row_stride_in_bytes[p] < size_t(pw) * (wide ? 2 : 1) ||
		    b->row_stride_in_bytes[p] > b->plane_size_in_bytes[p] / size_t(ph))
			return false;
	}
	return true;
}
} // namespace

extern "C" {

void pyrowave_get_api_version(uint32_t *major, uint32_t *minor, uint32_t *patch)
{
	*major = PYROWAVE_API_VERSION_MAJOR;
	*minor = PYROWAVE_API_VERSION_MINOR;
	*patch = PYROWAVE_API_VERSION_PATCH;
}

pyrowave_result pyrowave_create_default_device(pyrowave_device *device)
{
	if (!device)
		return PYROWAVE_ERROR_INVALID_ARGUMENT;
	*device = new pyrowave_device_opaque();
	return PYROWAVE_SUCCESS;
}

void pyrowave_device_destroy(pyrowave_device device) { delete device; }

pyrowave_result pyrowave_encoder_create(const pyrowave_encoder_create_info *info, pyrowave_encoder *encoder)
{
	if (!info || !encoder || !info->device || info->width <= 0 || info->height <= 0)
		return PYROWAVE_ERROR_INVALID_ARGUMENT;
	const bool c444 = info->chroma == PYROWAVE_CHROMA_SUBSAMPLING_444;
	if (!c444 && ((info->width | info->height) & 1))
		return PYROWAVE_ERROR_INVALID_ARGUMENT;
	auto *e = new pyrowave_encoder_opaque();
	e->codec = oracle_create(info->width, info->height, c444 ? 1 : 0, 0);
	e->width = info->width;
	e->height = info->height;
	e->c444 = c444;
	*encoder = e;
	return PYROWAVE_SUCCESS;
}

pyrowave_result pyrowave_encoder_encode_cpu_synchronous(pyrowave_encoder e, const pyrowave_cpu_buffer *buffers,
                                                        const pyrowave_rate_control *rc)
{
	bool wide = false;
	if (!e || !planes_ok(buffers, e->c444, e->width, e->height, wide) || !rc)
		return PYROWAVE_ERROR_INVALID_ARGUMENT;
	const uint64_t target = uint64_t(rc->maximum_bitstream_size) & ~uint64_t(3);
	if (target == 0 || target > 0xffffffffull)
		return PYROWAVE_ERROR_INVALID_ARGUMENT;
	std::vector<float> pyramid(oracle_pyramid_size(e->codec));
	int strides[3];
	int rc_dwt;
	if (wide)
	{
		const uint16_t *planes[3];
		for (int p = 0; p < 3; p++)
		{
			planes[p] = static_cast<const uint16_t *>(buffers->data[p]);
			strides[p] = int(buffers->row_stride_in_bytes[p] / 2);
		}
		rc_dwt = oracle_dwt16(e->codec, planes, strides, ORACLE_MODE_F32, pyramid.data());
	}
	else
	{
		const uint8_t *planes[3];
		for (int p = 0; p < 3; p++)
		{
			planes[p] = static_cast<const uint8_t *>(buffers->data[p]);
			strides[p] = int(buffers->row_stride_in_bytes[p]);
		}
		rc_dwt = oracle_dwt(e->codec, planes, strides, ORACLE_MODE_F32, pyramid.data());
	}
	if (rc_dwt != 0)
		return PYROWAVE_ERROR_GENERIC;
	e->sequence = (e->sequence + 1) & 7u;
	if (oracle_encode_pyramid(e->codec, pyramid.data(), rc->maximum_bitstream_size, e->sequence, -1.0f) != 0)
		return PYROWAVE_ERROR_GENERIC;
	e->encoded = true;
	return PYROWAVE_SUCCESS;
}

pyrowave_result pyrowave_encoder_compute_num_packets(pyrowave_encoder e, size_t boundary, size_t *num_packets)
{
	if (!e || !num_packets)
		return PYROWAVE_ERROR_INVALID_ARGUMENT;
	if (!e->encoded)
		return PYROWAVE_ERROR_GENERIC;
	*num_packets = oracle_compute_num_packets(e->codec, boundary);
	return PYROWAVE_SUCCESS;
}

pyrowave_result pyrowave_encoder_packetize(pyrowave_encoder e, pyrowave_packet *packets, size_t boundary,
                                           size_t *out_packets, void *bitstream, size_t size)
{
	if (!e || !packets || !out_packets || !bitstream)
		return PYROWAVE_ERROR_INVALID_ARGUMENT;
	if (!e->encoded)
		return PYROWAVE_ERROR_GENERIC;
	std::vector<uint64_t> pairs(2 * (oracle_compute_num_packets(e->codec, boundary) + 1));
	const size_t n = oracle_packetize(e->codec, pairs.data(), boundary, static_cast<uint8_t *>(bitstream), size);
	for (size_t i = 0; i < n; i++)
	{
		packets[i].offset = size_t(pairs[2 * i]);
		packets[i].size = size_t(pairs[2 * i + 1]);
	}
	*out_packets = n;
	return PYROWAVE_SUCCESS;
}

void pyrowave_encoder_destroy(pyrowave_encoder e)
{
	if (!e)
		return;
	oracle_destroy(e->codec);
	delete e;
}

pyrowave_result pyrowave_decoder_create(const pyrowave_decoder_create_info *info, pyrowave_decoder *decoder)
{
	if (!info || !decoder || !info->device || info->width <= 0 || info->height <= 0)
		return PYROWAVE_ERROR_INVALID_ARGUMENT;
	const bool c444 = info->chroma == PYROWAVE_CHROMA_SUBSAMPLING_444;
	if (!c444 && ((info->width | info->height) & 1))
		return PYROWAVE_ERROR_INVALID_ARGUMENT;
	auto *d = new pyrowave_decoder_opaque();
	d->codec = oracle_create(info->width, info->height, c444 ? 1 : 0, 0);
	d->parser = oracle_parser_create(d->codec);
	d->width = info->width;
	d->height = info->height;
	d->c444 = c444;
	*decoder = d;
	return PYROWAVE_SUCCESS;
}

pyrowave_result pyrowave_decoder_push_packet(pyrowave_decoder d, const void *data, size_t size)
{
	if (!d || (!data && size))
		return PYROWAVE_ERROR_INVALID_ARGUMENT;
	return oracle_parser_push_packet(d->parser, data, size) == 0 ? PYROWAVE_SUCCESS : PYROWAVE_ERROR_INVALID_ARGUMENT;
}

bool pyrowave_decoder_decode_is_ready(pyrowave_decoder d, bool allow_partial_frame)
{
	return d && oracle_parser_decode_is_ready(d->parser, allow_partial_frame ? 1 : 0) != 0;
}

pyrowave_result pyrowave_decoder_decode_cpu_buffer_synchronous(pyrowave_decoder d, const pyrowave_cpu_buffer *buffers)
{
	bool wide = false;
	if (!d || !planes_ok(buffers, d->c444, d->width, d->height, wide))
		return PYROWAVE_ERROR_INVALID_ARGUMENT;
	std::vector<uint32_t> offsets(size_t(oracle_block_count_32x32(d->codec)));
	const size_t nwords = oracle_parser_payload_words(d->parser);
	std::vector<uint32_t> payload(nwords + 1);
	oracle_parser_get(d->parser, offsets.data(), payload.data());
	std::vector<float> pyramid(oracle_pyramid_size(d->codec));
	if (oracle_dequant(d->codec, offsets.data(), payload.data(), nwords, ORACLE_MODE_F32, pyramid.data()) != 0)
		return PYROWAVE_ERROR_GENERIC;
	int strides[3];
	int rc_idwt;
	if (wide)
	{
		uint16_t *planes[3];
		for (int p = 0; p < 3; p++)
		{
			planes[p] = static_cast<uint16_t *>(buffers->data[p]);
			strides[p] = int(buffers->row_stride_in_bytes[p] / 2);
		}
		rc_idwt = oracle_idwt16(d->codec, pyramid.data(), ORACLE_MODE_F32, planes, strides);
	}
	else
	{
		uint8_t *planes[3];
		for (int p = 0; p < 3; p++)
		{
			planes[p] = static_cast<uint8_t *>(buffers->data[p]);
			strides[p] = int(buffers->row_stride_in_bytes[p]);
		}
		rc_idwt = oracle_idwt(d->codec, pyramid.data(), ORACLE_MODE_F32, planes, strides);
	}
	if (rc_idwt != 0)
		return PYROWAVE_ERROR_GENERIC;
	oracle_parser_mark_decoded(d->parser);
	return PYROWAVE_SUCCESS;
}

void pyrowave_decoder_destroy(pyrowave_decoder d)
{
	if (!d)
		return;
	oracle_parser_destroy(d->parser);
	oracle_destroy(d->codec);
	delete d;
}
}
