/*
 * PyroWave CPU oracle: C ABI.
 *
 * TEST INFRASTRUCTURE ONLY. This library is the checker that the CUDA
 * implementation in pyrowave_b200/ is compared against. Only tests/, the
 * smoke() check in __graft_entry__.py and the cpu_baseline leg of bench.py may
 * load it; the product never does.
 *
 * It restates the reference's algorithm for the encode/decode path (file:line
 * citations are in pyrowave_oracle.cpp next to each function):
 *   - geometry and block tables        pyrowave_common.cpp:191-241, bitstream.md:99-152,472-511
 *   - CDF 9/7 forward DWT              shaders/dwt.comp, shaders/dwt_common.h
 *   - quantiser + RD statistics        shaders/wavelet_quant.comp
 *   - rate-control analyze/finalize    shaders/analyze_rate_control*.comp
 *   - rate-control resolve             shaders/resolve_rate_control.comp
 *   - block packing                    shaders/block_packing.comp
 *   - packetize / compute_num_packets  pyrowave_encoder.cpp:596-623,1048-1115
 *   - packet parser                    pyrowave_decoder.cpp:126-262,780-794,832-840
 *   - dequantiser                      shaders/wavelet_dequant.comp (STORAGE_MODE 0)
 *   - inverse DWT                      shaders/idwt.comp, pyrowave_decoder.cpp:699-778
 *
 * Parity pinning: the bitstream layer (block layout, packetize, parser) is
 * checked against the reference's own Granite-free C++
 * (metal/pyrowave_bitstream.cpp, built into oracle/_ref/ by oracle/Makefile);
 * the arithmetic stages follow the GLSL line by line and are pinned by the
 * reference's known-answer tests (pyrowave_c_test.cpp). The GLSL itself cannot
 * run on this machine (no Vulkan device), so the arithmetic is "restated, not
 * executed": bit-exact agreement of the CUDA kernels with this restatement is
 * what the GPU tests check.
 */
#ifndef PYROWAVE_ORACLE_H_
#define PYROWAVE_ORACLE_H_

#include <stddef.h>
#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

/* Transform arithmetic modes. */
enum
{
	ORACLE_MODE_F32 = 0,   /* FP32 lifting, non-fused ops, storage rounding per level mask */
	ORACLE_MODE_REF16 = 1, /* the reference's default precision 1: FP32 math, FP16 shared staging */
	ORACLE_MODE_F64 = 2    /* FP64 math oracle (outputs through the *_f64 entry points) */
};

typedef struct oracle_codec oracle_codec;

/* fp16_level_mask: bit L set = level L coefficients are stored as FP16. */
oracle_codec *oracle_create(int width, int height, int chroma444, unsigned fp16_level_mask);
void oracle_destroy(oracle_codec *codec);

int oracle_aligned_width(const oracle_codec *codec);
int oracle_aligned_height(const oracle_codec *codec);
int oracle_block_count_8x8(const oracle_codec *codec);
int oracle_block_count_32x32(const oracle_codec *codec);
/* Number of coefficients in the canonical pyramid layout (all transmitted bands, in block-index band order). */
size_t oracle_pyramid_size(const oracle_codec *codec);
/* out[((c * 5 + level) * 4 + band) * 4 + {0..3}] = {offset_8x8, stride_8x8, offset_32x32, stride_32x32}; -1 if absent. */
void oracle_block_info(const oracle_codec *codec, int32_t *out);
/* out[b * 4 + {0..3}] = {offset_8x8, stride_8x8, width_8x8, height_8x8} for every 32x32 block b. */
void oracle_block_mapping(const oracle_codec *codec, int32_t *out);
/* out[((c * 5 + level) * 4 + band)] = canonical pyramid offset of that band, -1 if absent. */
void oracle_band_offsets(const oracle_codec *codec, int64_t *out);

/* Quantiser tables (host side of pyrowave_encoder.cpp:107-172). out has 3*5*4 entries. */
void oracle_quant_tables(const oracle_codec *codec, float *quant_resolution, float *rdo_distortion_scale);

/* Forward DWT of 8-bit planes into the canonical pyramid.
 * planes/strides: Y, Cb, Cr (4:2:0 chroma planes are width/2 x height/2). */
int oracle_dwt(oracle_codec *codec, const uint8_t *const planes[3], const int strides[3], int mode, float *out_pyramid);
int oracle_dwt_f64(oracle_codec *codec, const uint8_t *const planes[3], const int strides[3], double *out_pyramid);
/* 16-bit (R16_UNORM) planes, strides in samples. */
int oracle_dwt16(oracle_codec *codec, const uint16_t *const planes[3], const int strides[3], int mode, float *out_pyramid);

/* Encodes a canonical pyramid (the reference's Encoder::encode_pre_transformed when
 * quant_scale >= 0, otherwise the default per-band resolutions). Results are kept
 * in the codec and read back with the getters below. Returns 0 on success. */
int oracle_encode_pyramid(oracle_codec *codec, const float *pyramid, uint64_t maximum_bitstream_size,
                          uint32_t sequence, float quant_scale);

void oracle_get_code_words(const oracle_codec *codec, uint32_t *out);   /* block_count_8x8 */
void oracle_get_block_stats(const oracle_codec *codec, uint32_t *out);  /* block_count_8x8 * 17 words: num_planes + 16 x {fp16 error, cost bits} */
void oracle_get_rd(const oracle_codec *codec, uint32_t *rate_cost, float *distortion, uint32_t *bucket); /* blocks32 * 16 each */
void oracle_get_histogram(const oracle_codec *codec, uint32_t *scan2048, uint32_t *consumed);
void oracle_get_quant(const oracle_codec *codec, int32_t *out);          /* block_count_32x32 */
void oracle_get_meta(const oracle_codec *codec, uint32_t *out);          /* block_count_32x32 * {offset_u32, num_words} */
size_t oracle_get_bitstream_words(const oracle_codec *codec);
void oracle_get_bitstream(const oracle_codec *codec, uint32_t *out);

/* Packetization of the last encode (pyrowave_encoder.cpp:596-623,1048-1115).
 * packets: pairs of {offset, size}. */
void oracle_set_encoded(oracle_codec *codec, const uint32_t *meta, const uint32_t *words, size_t nwords,
                        uint32_t sequence);
size_t oracle_compute_num_packets(const oracle_codec *codec, size_t packet_boundary);
size_t oracle_packetize(const oracle_codec *codec, uint64_t *packets, size_t packet_boundary, uint8_t *out, size_t size);

/* Decoder side. */
typedef struct oracle_parser oracle_parser;
oracle_parser *oracle_parser_create(const oracle_codec *codec);
void oracle_parser_destroy(oracle_parser *parser);
void oracle_parser_clear(oracle_parser *parser);
int oracle_parser_push_packet(oracle_parser *parser, const void *data, size_t size); /* 0 = ok, -1 = invalid */
int oracle_parser_decode_is_ready(const oracle_parser *parser, int allow_partial_frame);
void oracle_parser_mark_decoded(oracle_parser *parser);
size_t oracle_parser_payload_words(const oracle_parser *parser);
void oracle_parser_get(const oracle_parser *parser, uint32_t *offsets, uint32_t *payload);
int oracle_parser_decoded_blocks(const oracle_parser *parser);
int oracle_parser_total_blocks(const oracle_parser *parser);

/* Dequantise (offsets + concatenated payload words) into a canonical pyramid.
 * mode selects the storage rounding (F32 uses the level mask, REF16 rounds levels 0-1). */
int oracle_dequant(const oracle_codec *codec, const uint32_t *offsets, const uint32_t *payload, size_t payload_words,
                   int mode, float *out_pyramid);

/* Inverse DWT of a canonical pyramid into 8-bit planes. */
int oracle_idwt(oracle_codec *codec, const float *pyramid, int mode, uint8_t *const planes[3], const int strides[3]);
int oracle_idwt_f64(oracle_codec *codec, const double *pyramid, uint8_t *const planes[3], const int strides[3]);
int oracle_idwt16(oracle_codec *codec, const float *pyramid, int mode, uint16_t *const planes[3], const int strides[3]);

/* PSNR-HVS-M (shaders/psnr_hvs_m.comp, psnr.cpp:25-28,126-224,245-320 of the
 * reference): adds, per height factor 1 + i/8 (i = 0..15), the fixed-point
 * (2^-24) error sum of every 8x8 window at a stride of 4 of the luma planes
 * into errors[16]. Tables: 16 x {csf, mask, inv_mask} x 64 floats. */
void oracle_psnr_hvs_m(const uint8_t *ref, int ref_stride, const uint8_t *dist, int dist_stride, int width,
                       int height, uint64_t *errors);
void oracle_psnr_hvs_m_tables(int height, float *out);
uint64_t oracle_psnr_hvs_m_pixels(int width, int height);
void oracle_hvs_dct8(const float *in, float *out);

/* Packing analysis of a decoded frame (the reference's disabled statistics pass,
 * pyrowave_encoder.cpp:625-958, for the current block format), from the
 * parser's offsets and payload: layout_bytes[5] = estimated bytes of 32x32
 * packets with 2x2, 4x2 and 2x4 sub-blocks, 64x32 with 4x4 and 64x64 with 8x4;
 * band_bytes[(c * 5 + level) * 4 + band] = coded bytes; significant = nonzero
 * coefficients; hist[16 * 256] = plane bytes by position in their sub-block's
 * run of planes (0: most significant). */
int oracle_analyze_packing(const oracle_codec *codec, const uint32_t *offsets, const uint32_t *payload,
                           size_t payload_words, uint64_t *layout_bytes, uint64_t *band_bytes, uint64_t *significant,
                           uint32_t *hist);

/* Helpers exposed for unit tests. */
uint16_t oracle_float_to_half(float v);
float oracle_half_to_float(uint16_t h);
uint32_t oracle_bucket_index(float d, float cost, float d_base, float cost_base);

#ifdef __cplusplus
}
#endif

#endif
