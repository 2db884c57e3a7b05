/*
 * mans_oracle.h -- CPU restatement of the MANS hot path (TEST INFRASTRUCTURE).
 *
 * This is the parity checker for the CUDA library in mans_b200/. Only the
 * tests, the smoke check and the CPU-baseline leg of bench.py load it. The
 * product path never calls into it.
 *
 * Parity pin: checked against outputs of the reference's own code run on the
 * same seeded inputs (CPU ADM mapping built from mapping/cpu/mappingcpuV2.cpp,
 * GPU ADM mapping mapping/nv/mappingV15_fused_uint16.cu and the GPU rANS codec
 * in include/ans, built with nvcc), recorded as fixtures under tests/golden/.
 */
#ifndef MANS_ORACLE_H
#define MANS_ORACLE_H

#include <stddef.h>
#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

/* ---- ADM uint16 (unary bit-signal format, merged layout of V15) ---- */
uint64_t mo_adm_u16_merged_size(const uint16_t* in, uint64_t n);
/* Returns bytes written, or -1 if cap is too small. */
int64_t mo_adm_u16_map(const uint16_t* in, uint64_t n, uint8_t* out, uint64_t cap);
/* Returns 0 on success, <0 on a malformed merged buffer. */
int mo_adm_u16_unmap(const uint8_t* m, uint64_t msize, uint64_t n, uint16_t* out);
/* Compatibility layouts of the uint16 merged buffer (see mans_oracle.c). */
#define MO_LAYOUT_V15 0
#define MO_LAYOUT_V12 1
#define MO_LAYOUT_CPUV2 2
uint64_t mo_adm_u16_header_bytes(uint64_t n, int layout);
int64_t mo_adm_u16_map_layout(const uint16_t* in, uint64_t n, int layout, uint8_t* out,
                              uint64_t cap);
int mo_adm_u16_unmap_layout(const uint8_t* m, uint64_t msize, uint64_t n, int layout,
                            uint16_t* out);

/* ---- ADM uint32 (escape-byte format of V9, self-describing merged layout) ---- */
uint64_t mo_adm_u32_max_merged_size(uint64_t n);
int64_t mo_adm_u32_map(const uint32_t* in, uint64_t n, uint8_t* out, uint64_t cap);
int mo_adm_u32_unmap(const uint8_t* m, uint64_t msize, uint64_t n, uint32_t* out);

/* ---- byte rANS (include/ans stream format) ---- */
void mo_ans_histogram(const uint8_t* in, uint64_t n, uint32_t hist[256]);
/* Quantise a histogram to a 2^prob_bits pdf exactly as the reference normaliser. */
int mo_ans_normalize(const uint32_t hist[256], uint32_t total, int prob_bits,
                     uint32_t pdf[256], uint32_t cdf[256]);
uint64_t mo_ans_max_compressed_size(uint64_t n);
/* Returns the stream size, or -1 (bad precision), -2 (cap too small). */
int64_t mo_ans_encode(int prob_bits, const uint8_t* in, uint64_t n, uint8_t* out, uint64_t cap);
/* Same, with per-block word counts reported (for sizing checks). */
int64_t mo_ans_encode_ex(int prob_bits, const uint8_t* in, uint64_t n, uint8_t* out,
                         uint64_t cap, uint32_t* block_words);
/* Returns 0 on success; *out_n receives the decoded size. */
int mo_ans_decode(const uint8_t* in, uint64_t in_size, uint8_t* out, uint64_t out_cap,
                  uint64_t* out_n);
/* Read the decoded size recorded in a stream header (0 if the header is bad). */
uint64_t mo_ans_stream_uncompressed_size(const uint8_t* in, uint64_t in_size);
/* Zero the bytes the reference encoder leaves uninitialised (header options
 * bits 4..31, checksum, unused words, the odd-count block-word pad, per-block
 * word padding, and the pdf of an empty stream). */
void mo_ans_mask(uint8_t* stream, uint64_t size);

/* ---- MANS end to end: ANS(ADM(x)) ---- */
int64_t mo_mans_compress_u16(int prob_bits, const uint16_t* in, uint64_t n, uint8_t* out,
                             uint64_t cap);
int mo_mans_decompress_u16(const uint8_t* in, uint64_t in_size, uint64_t n, uint16_t* out);
int64_t mo_mans_compress_u32(int prob_bits, const uint32_t* in, uint64_t n, uint8_t* out,
                             uint64_t cap);
int mo_mans_decompress_u32(const uint8_t* in, uint64_t in_size, uint64_t n, uint32_t* out);

/* ---- OpenMP variants (same bytes), used as the timed CPU baseline ---- */
void mo_set_threads(int n); /* threads of the variants below */
void mo_ans_histogram_par(const uint8_t* in, uint64_t n, uint32_t hist[256]);
uint64_t mo_ans_par_scratch_words(uint64_t n);
int64_t mo_ans_encode_par(int prob_bits, const uint8_t* in, uint64_t n, uint8_t* out,
                          uint64_t cap, uint16_t* scratch, uint32_t* scratch_states,
                          uint32_t* scratch_nw);
int mo_ans_decode_par(const uint8_t* in, uint64_t in_size, uint8_t* out, uint64_t out_cap);
int64_t mo_adm_u16_map_layout_par(const uint16_t* in, uint64_t n, int layout, uint8_t* out,
                                  uint64_t cap);
int64_t mo_adm_u32_map_par(const uint32_t* in, uint64_t n, uint8_t* out, uint64_t cap);
int mo_adm_u32_unmap_par(const uint8_t* m, uint64_t msize, uint64_t n, uint32_t* out);

#ifdef __cplusplus
}
#endif
#endif
