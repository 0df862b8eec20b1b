// C ABI over the reference's own Granite-free bitstream code
// (metal/pyrowave_bitstream.{hpp,cpp} in the reference tree, compiled in place by
// oracle/Makefile into oracle/_ref/). TEST INFRASTRUCTURE ONLY: it pins the
// oracle's block layout, packetize and packet parser against the reference.
#include "pyrowave_bitstream.hpp"

#include <stdint.h>
#include <string.h>

using namespace PyroWave;

extern "C" {

void *ref_layout_create(int width, int height, int chroma444)
{
	auto *layout = new BlockLayout;
	if (!layout->init(width, height, chroma444 ? ChromaSubsampling::Chroma444 : ChromaSubsampling::Chroma420))
	{
		delete layout;
		return nullptr;
	}
	return layout;
}

void ref_layout_destroy(void *layout) { delete static_cast<BlockLayout *>(layout); }

void ref_layout_counts(const void *layout_, int32_t *out)
{
	auto *layout = static_cast<const BlockLayout *>(layout_);
	out[0] = layout->block_count_8x8;
	out[1] = layout->block_count_32x32;
	out[2] = layout->aligned_width;
	out[3] = layout->aligned_height;
}

// Same packing as oracle_block_info: [comp][level][band][4]; bands that the
// layout never assigns keep the zero-initialised entry, reported as -1.
void ref_layout_block_info(const void *layout_, int32_t *out)
{
	auto *layout = static_cast<const BlockLayout *>(layout_);
	for (int c = 0; c < 3; c++)
		for (int l = 0; l < 5; l++)
			for (int b = 0; b < 4; b++)
			{
				bool present = !(l == 0 && c != 0 && layout->chroma == ChromaSubsampling::Chroma420) &&
				               !(b == 0 && l != 4);
				const auto &info = layout->block_meta[c][l][b];
				int32_t *o = out + ((c * 5 + l) * 4 + b) * 4;
				o[0] = present ? info.block_offset_8x8 : -1;
				o[1] = present ? info.block_stride_8x8 : -1;
				o[2] = present ? info.block_offset_32x32 : -1;
				o[3] = present ? info.block_stride_32x32 : -1;
			}
}

void ref_layout_block_mapping(const void *layout_, int32_t *out)
{
	auto *layout = static_cast<const BlockLayout *>(layout_);
	for (size_t i = 0; i < layout->block_32x32_to_8x8_mapping.size(); i++)
	{
		const auto &m = layout->block_32x32_to_8x8_mapping[i];
		out[4 * i + 0] = m.block_offset_8x8;
		out[4 * i + 1] = m.block_stride_8x8;
		out[4 * i + 2] = m.block_width_8x8;
		out[4 * i + 3] = m.block_height_8x8;
	}
}

int ref_block_count_per_subdivision(int num_blocks) { return compute_block_count_per_subdivision(num_blocks); }

size_t ref_compute_num_packets(const void *layout_, const uint32_t *meta, size_t packet_boundary)
{
	return compute_num_packets(*static_cast<const BlockLayout *>(layout_), meta, packet_boundary);
}

size_t ref_packetize(const void *layout_, uint64_t *packets, size_t max_packets, size_t packet_boundary, uint8_t *out,
                     size_t size, const uint32_t *meta, const uint32_t *bitstream)
{
	std::vector<Packet> tmp(max_packets + 1);
	size_t n = packetize(*static_cast<const BlockLayout *>(layout_), tmp.data(), packet_boundary, out, size, meta,
	                     bitstream);
	for (size_t i = 0; i < n && i < max_packets; i++)
	{
		packets[2 * i + 0] = tmp[i].offset;
		packets[2 * i + 1] = tmp[i].size;
	}
	return n;
}

float ref_decode_quant(uint32_t code) { return decode_quant(uint8_t(code)); }
uint32_t ref_encode_quant(float v) { return encode_quant(v); }

void *ref_parser_create(const void *layout_)
{
	auto *p = new BitstreamParser;
	p->init(static_cast<const BlockLayout *>(layout_));
	return p;
}

void ref_parser_destroy(void *p) { delete static_cast<BitstreamParser *>(p); }
void ref_parser_clear(void *p) { static_cast<BitstreamParser *>(p)->clear(); }
int ref_parser_push_packet(void *p, const void *data, size_t size)
{
	return static_cast<BitstreamParser *>(p)->push_packet(data, size) ? 0 : -1;
}
int ref_parser_decode_is_ready(const void *p, int allow_partial)
{
	return static_cast<const BitstreamParser *>(p)->decode_is_ready(allow_partial != 0);
}
void ref_parser_mark_decoded(void *p) { static_cast<BitstreamParser *>(p)->mark_frame_decoded(); }
size_t ref_parser_payload_words(const void *p) { return static_cast<const BitstreamParser *>(p)->payload().size(); }
void ref_parser_get(const void *p_, uint32_t *offsets, uint32_t *payload)
{
	auto *p = static_cast<const BitstreamParser *>(p_);
	memcpy(offsets, p->dequant_offsets().data(), p->dequant_offsets().size() * 4);
	if (!p->payload().empty())
		memcpy(payload, p->payload().data(), p->payload().size() * 4);
}
int ref_parser_decoded_blocks(const void *p) { return static_cast<const BitstreamParser *>(p)->get_decoded_blocks(); }
int ref_parser_total_blocks(const void *p)
{
	return static_cast<const BitstreamParser *>(p)->get_total_blocks_in_sequence();
}
}
