/*
 * mans_oracle.c -- CPU restatement of the MANS hot path (TEST INFRASTRUCTURE).
 *
 * The parity checker for the CUDA library. Only tests/, the smoke check and
 * the CPU-baseline leg of bench.py may load it; the product path never does.
 * Plain C99, written for clarity rather than speed; the OpenMP variants at
 * the end of the file (used as the timed CPU baseline) produce the same bytes.
 *
 * Every function cites the reference code it restates (paths are relative to
 * the hpdps-group/MANS tree). Where the reference is undefined or wrong the
 * defined behaviour chosen here is stated beside the code.
 */
#include "mans_oracle.h"

#include <stdlib.h>
#include <string.h>

/* ------------------------------------------------------------------------ */
/* ADM constants: mapping/nv/mappingV15_fused_uint16.cu:16-20,               */
/* mapping/cpu/mappingcpuV2.cpp:14-18                                        */
/* ------------------------------------------------------------------------ */
#define ADM_LANES 32        /* cmp_tblock_size */
#define ADM_CHUNK 16        /* cmp_chunk: elements per lane */
#define ADM_GROUP 512       /* elements per group (one warp) */
#define ADM_STEP 126        /* residue range of one code byte */
/* Longest unary stream of one lane: 16 elements x ceil(65535/126)=521 bits. */
#define ADM_U16_MAX_LANE_BYTES ((ADM_CHUNK * 521 + 7) / 8)

static inline uint64_t div_up(uint64_t a, uint64_t b) { return (a + b - 1) / b; }

static inline void wr32(uint8_t* p, uint32_t v) { memcpy(p, &v, 4); }
static inline void wr16(uint8_t* p, uint16_t v) { memcpy(p, &v, 2); }
static inline uint32_t rd32(const uint8_t* p) { uint32_t v; memcpy(&v, p, 4); return v; }
static inline uint16_t rd16(const uint8_t* p) { uint16_t v; memcpy(&v, p, 2); return v; }

/* Group center: truncated mean of the group's elements.
 * mappingcpuV2.cpp:52-64 (uint64 sum); V15 :152-174 (uint32 sum, which
 * cannot overflow for 512 uint16 values, so both agree). */
static uint32_t adm_center_u16(const uint16_t* in, uint64_t start, uint64_t end) {
  uint64_t s = 0;
  for (uint64_t i = start; i < end; ++i) s += in[i];
  return end > start ? (uint32_t)(s / (end - start)) : 0;
}

/* Per-element mapping shared by the uint16 and uint32 formats:
 * k = 1 for the center, else ceil(diff/126); code = 1 for the center, else
 * 2r (above) or 2r+1 (below) with r = diff - 126(k-1) in [1,126].
 * mappingcpuV2.cpp:84-89; V15 :191-202; V9 :523-533. */
static inline void adm_map_elem(uint64_t v, uint64_t c, uint64_t* k, uint8_t* code) {
  if (v == c) {
    *k = 1;
    *code = 1;
    return;
  }
  uint64_t d = v > c ? v - c : c - v;
  uint64_t kk = (d + ADM_STEP - 1) / ADM_STEP;
  uint64_t r = d - ADM_STEP * (kk - 1);
  *k = kk;
  *code = (uint8_t)(2 * r + (v > c ? 0 : 1));
}

/* Encode one lane's unary bit stream (MSB first within a byte): a 1 bit per
 * element followed by k-1 zero bits. Returns the number of bits.
 * mappingcpuV2.cpp:81-94; V15 :204-207. */
static uint32_t adm_lane_bits_u16(const uint16_t* in, uint64_t start, uint64_t end, uint32_t c,
                                  uint8_t* bits, uint8_t* codes) {
  uint32_t off = 0;
  for (uint64_t i = start; i < end; ++i) {
    uint64_t k;
    uint8_t code;
    adm_map_elem(in[i], c, &k, &code);
    if (codes) codes[i - start] = code;
    if (bits) bits[off >> 3] |= (uint8_t)(1u << (7 - (off & 7)));
    off += (uint32_t)k;
  }
  return off;
}

/* Lane element range [s, e) of group grp, lane l (may be empty). */
static inline void lane_range(uint64_t n, uint64_t grp, int l, uint64_t* s, uint64_t* e) {
  uint64_t a = grp * ADM_GROUP + (uint64_t)l * ADM_CHUNK;
  uint64_t b = a + ADM_CHUNK;
  if (a > n) a = n;
  if (b > n) b = n;
  *s = a;
  *e = b;
}

/* Group signal length in bytes: max over lanes of ceil(bits/8).
 * mappingcpuV2.cpp:96-98; V15 :331-336. */
static uint32_t adm_group_len_u16(const uint16_t* in, uint64_t n, uint64_t grp, uint32_t* c_out) {
  uint64_t gs = grp * ADM_GROUP, ge = gs + ADM_GROUP;
  if (ge > n) ge = n;
  uint32_t c = adm_center_u16(in, gs, ge);
  uint32_t mx = 0;
  for (int l = 0; l < ADM_LANES; ++l) {
    uint64_t s, e;
    lane_range(n, grp, l, &s, &e);
    uint32_t b = adm_lane_bits_u16(in, s, e, c, NULL, NULL);
    uint32_t by = (b + 7) / 8;
    if (by > mx) mx = by;
  }
  if (c_out) *c_out = c;
  return mx;
}

uint64_t mo_adm_u16_merged_size(const uint16_t* in, uint64_t n) {
  uint64_t g = div_up(n, ADM_GROUP);
  uint64_t tot = 0;
  for (uint64_t grp = 0; grp < g; ++grp) tot += adm_group_len_u16(in, n, grp, NULL);
  return 6 * g + n + 32 * tot;
}

/* Merged uint16 layout (V15 main :933-957):
 *   [i32 exclusive signal-length prefix x g][u16 center x g][u8 code x n]
 *   [bits: for each group, for each lane, len[g] bytes]
 * The lane tail: when a lane's stream is shorter than the group length, the
 * byte holding its end gets its remaining low bits set to 1 (0xFF when the
 * end is byte aligned); later bytes stay 0. mappingcpuV2.cpp:102-114;
 * V15 :345-350. Ragged n (n % 8 != 0) follows the CPU mapping (only valid
 * elements are coded); the reference GPU kernel reads past n there.
 *
 * Compatibility layouts (same codes and bits):
 *   MO_LAYOUT_V12:   [u16 signal length x g][u16 center x g][codes][bits]
 *                    (mappingV12_bit-adm-thrust-prefixsum.cu :606-634). Its
 *                    concat kernel (:405-428) copies only lanes that hold an
 *                    element into a buffer filled with 255 (:504), so a lane
 *                    past n is 0xFF in all of its len[g] bytes.
 *   MO_LAYOUT_CPUV2: [i32 signal-length prefix x (g + 1), the last = total]
 *                    [u16 center x g][codes][bits] (mappingcpuV2.cpp:117-121,
 *                    271-285). */
uint64_t mo_adm_u16_header_bytes(uint64_t n, int layout) {
  uint64_t g = div_up(n, ADM_GROUP);
  if (layout == MO_LAYOUT_V12) return 4 * g;
  if (layout == MO_LAYOUT_CPUV2) return 6 * g + 4;
  return 6 * g;
}

int64_t mo_adm_u16_map_layout(const uint16_t* in, uint64_t n, int layout, uint8_t* out,
                              uint64_t cap) {
  uint64_t g = div_up(n, ADM_GROUP);
  if (layout < 0 || layout > 2) return -2;
  uint32_t* len = (uint32_t*)calloc(g ? g : 1, sizeof(uint32_t));
  uint32_t* ctr = (uint32_t*)calloc(g ? g : 1, sizeof(uint32_t));
  uint64_t tot = 0;
  for (uint64_t grp = 0; grp < g; ++grp) {
    len[grp] = adm_group_len_u16(in, n, grp, &ctr[grp]);
    tot += len[grp];
  }
  const uint64_t hdr = mo_adm_u16_header_bytes(n, layout);
  uint64_t msize = hdr + n + 32 * tot;
  if (msize > cap) {
    free(len);
    free(ctr);
    return -1;
  }
  const uint64_t pre = hdr - 2 * g;  /* bytes before the centers */
  uint8_t* p_len = out;
  uint8_t* p_ctr = out + pre;
  uint8_t* p_code = out + hdr;
  uint8_t* p_bits = out + hdr + n;
  memset(p_bits, 0, 32 * tot);
  uint64_t excl = 0;
  uint8_t* lanebuf = (uint8_t*)malloc(ADM_U16_MAX_LANE_BYTES + 8);
  for (uint64_t grp = 0; grp < g; ++grp) {
    if (layout == MO_LAYOUT_V12) wr16(p_len + 2 * grp, (uint16_t)len[grp]);
    else wr32(p_len + 4 * grp, (uint32_t)excl);
    wr16(p_ctr + 2 * grp, (uint16_t)ctr[grp]);
    uint32_t L = len[grp];
    for (int l = 0; l < ADM_LANES; ++l) {
      uint64_t s, e;
      lane_range(n, grp, l, &s, &e);
      memset(lanebuf, 0, ADM_U16_MAX_LANE_BYTES + 8);
      if (layout == MO_LAYOUT_V12 && s >= e) {
        memset(lanebuf, 0xFF, L);
      } else {
        uint32_t b = adm_lane_bits_u16(in, s, e, ctr[grp], lanebuf, p_code + s);
        if (b < L * 8) lanebuf[b >> 3] |= (uint8_t)(0xFFu >> (b & 7));
      }
      memcpy(p_bits + 32 * excl + (uint64_t)l * L, lanebuf, L);
    }
    excl += L;
  }
  if (layout == MO_LAYOUT_CPUV2) wr32(p_len + 4 * g, (uint32_t)excl);
  free(lanebuf);
  free(len);
  free(ctr);
  return (int64_t)msize;
}

int64_t mo_adm_u16_map(const uint16_t* in, uint64_t n, uint8_t* out, uint64_t cap) {
  return mo_adm_u16_map_layout(in, n, MO_LAYOUT_V15, out, cap);
}

/* Inverse mapping. Signal restore follows mappingcpuV2.cpp:161-197 (scan the
 * lane's bytes MSB first; a 1 starts the next element, a 0 adds one to the
 * current element's signal count, stop after the 17th one); value restore
 * follows :202-224 (odd code: center - diff, even: center + diff, with
 * diff = code/2 + 126*signal). Signal counts are kept as int here; the
 * reference stores them in uint8_t, which wraps for k > 256. */
int mo_adm_u16_unmap_layout(const uint8_t* m, uint64_t msize, uint64_t n, int layout,
                            uint16_t* out) {
  uint64_t g = div_up(n, ADM_GROUP);
  if (layout < 0 || layout > 2) return -6;
  const uint64_t hdr = mo_adm_u16_header_bytes(n, layout);
  if (msize < hdr + n) return -1;
  uint64_t bits_bytes = msize - hdr - n;
  if (bits_bytes % 32) return -2;
  uint64_t tot = bits_bytes / 32;
  const uint8_t* p_len = m;
  const uint8_t* p_ctr = m + hdr - 2 * g;
  const uint8_t* p_code = m + hdr;
  const uint8_t* p_bits = m + hdr + n;
  if (layout == MO_LAYOUT_CPUV2 && rd32(p_len + 4 * g) != tot) return -3;
  uint64_t run = 0;  /* V12: the prefix is recomputed from the lengths */
  for (uint64_t grp = 0; grp < g; ++grp) {
    uint64_t ex, nx;
    if (layout == MO_LAYOUT_V12) {
      ex = run;
      nx = ex + rd16(p_len + 2 * grp);
      run = nx;
    } else {
      ex = rd32(p_len + 4 * grp);
      nx = grp + 1 < g ? rd32(p_len + 4 * (grp + 1)) : tot;
    }
    if (nx < ex || nx > tot) return -3;
    uint64_t L = nx - ex;
    uint32_t c = rd16(p_ctr + 2 * grp);
    for (int l = 0; l < ADM_LANES; ++l) {
      uint64_t s, e;
      lane_range(n, grp, l, &s, &e);
      if (s >= e) continue;
      const uint8_t* lb = p_bits + 32 * ex + (uint64_t)l * L;
      int cnt = (int)(e - s);
      int sig[ADM_CHUNK];
      memset(sig, 0, sizeof(sig));
      int idx = -1;
      for (uint64_t by = 0; by < L && idx < ADM_CHUNK; ++by) {
        for (int bit = 7; bit >= 0 && idx < ADM_CHUNK; --bit) {
          if ((lb[by] >> bit) & 1) {
            ++idx;
          } else {
            if (idx < 0) return -4;
            if (idx < ADM_CHUNK) sig[idx]++;
          }
        }
      }
      if (idx < cnt - 1) return -5;
      for (int i = 0; i < cnt; ++i) {
        uint8_t code = p_code[s + i];
        uint32_t d = (code & 1) ? (uint32_t)(code - 1) / 2 : (uint32_t)code / 2;
        d += (uint32_t)ADM_STEP * (uint32_t)sig[i];
        out[s + i] = (uint16_t)((code & 1) ? c - d : c + d);
      }
    }
  }
  if (layout == MO_LAYOUT_V12 && run != tot) return -3;
  return 0;
}

int mo_adm_u16_unmap(const uint8_t* m, uint64_t msize, uint64_t n, uint16_t* out) {
  return mo_adm_u16_unmap_layout(m, msize, n, MO_LAYOUT_V15, out);
}

/* ------------------------------------------------------------------------ */
/* ADM uint32: escape-byte format of mapping/nv/mappingV9_fuse.cu:458-651.   */
/* Per lane record: for each element with k <= 8, k-1 zero bytes then the   */
/* code byte (:530-540); otherwise 254 followed by the value big-endian      */
/* (:541-548); the record is padded with 255 to a multiple of 8 bytes       */
/* (:634-639). Records are concatenated in group-major, lane-major order     */
/* (thread order of the exclusive scan, :875, and coalescing, :654-676).    */
/* The reference persists only the records (:998); this layout adds what a  */
/* decoder needs:                                                           */
/*   [i32 exclusive record-byte offset per group x g][u32 center x g]       */
/*   [u8 record length / 8 per lane x 32g][records]                         */
/* Centers use a 64-bit sum (the reference's uint32 sum overflows once the  */
/* group sum reaches 2^32; below that both agree) and diffs are computed in */
/* 64-bit (the reference's int diff is undefined for values >= 2^31).       */
/* ------------------------------------------------------------------------ */
#define ADM_U32_MAX_K 8

static uint32_t adm_center_u32(const uint32_t* in, uint64_t start, uint64_t end) {
  uint64_t s = 0;
  for (uint64_t i = start; i < end; ++i) s += in[i];
  return end > start ? (uint32_t)(s / (end - start)) : 0;
}

static uint32_t adm_lane_record_u32(const uint32_t* in, uint64_t s, uint64_t e, uint32_t c,
                                    uint8_t* rec) {
  uint32_t pos = 0;
  for (uint64_t i = s; i < e; ++i) {
    uint64_t k;
    uint8_t code;
    adm_map_elem(in[i], c, &k, &code);
    if (k <= ADM_U32_MAX_K) {
      if (rec) {
        memset(rec + pos, 0, k - 1);
        rec[pos + k - 1] = code;
      }
      pos += (uint32_t)k;
    } else {
      uint32_t v = in[i];
      if (rec) {
        rec[pos] = 254;
        rec[pos + 1] = (uint8_t)(v >> 24);
        rec[pos + 2] = (uint8_t)(v >> 16);
        rec[pos + 3] = (uint8_t)(v >> 8);
        rec[pos + 4] = (uint8_t)v;
      }
      pos += 5;
    }
  }
  uint32_t padded = (pos + 7) / 8 * 8;
  if (rec) memset(rec + pos, 255, padded - pos);
  return padded;
}

uint64_t mo_adm_u32_max_merged_size(uint64_t n) {
  uint64_t g = div_up(n, ADM_GROUP);
  return 40 * g + 8 * n;
}

int64_t mo_adm_u32_map(const uint32_t* in, uint64_t n, uint8_t* out, uint64_t cap) {
  uint64_t g = div_up(n, ADM_GROUP);
  uint64_t hdr = 40 * g;
  if (cap < hdr) return -1;
  uint8_t rec[ADM_CHUNK * ADM_U32_MAX_K + 8];
  uint64_t pos = hdr;
  for (uint64_t grp = 0; grp < g; ++grp) {
    uint64_t gs = grp * ADM_GROUP, ge = gs + ADM_GROUP;
    if (ge > n) ge = n;
    uint32_t c = adm_center_u32(in, gs, ge);
    wr32(out + 4 * grp, (uint32_t)(pos - hdr));
    wr32(out + 4 * g + 4 * grp, c);
    for (int l = 0; l < ADM_LANES; ++l) {
      uint64_t s, e;
      lane_range(n, grp, l, &s, &e);
      uint32_t len = adm_lane_record_u32(in, s, e, c, rec);
      out[8 * g + 32 * grp + l] = (uint8_t)(len / 8);
      if (pos + len > cap) return -1;
      memcpy(out + pos, rec, len);
      pos += len;
    }
  }
  return (int64_t)pos;
}

/* Record decode follows mappingV9_fuse.cu:126-157: a byte below 254 starts
 * an element (count leading zero bytes, then the code byte), 254 starts a
 * 4-byte big-endian literal, 255 is padding to the next 8-byte boundary. */
static int adm_u32_unmap_group(const uint8_t* m, uint64_t g, uint64_t grp, uint64_t rec_bytes,
                               uint64_t n, uint32_t* out) {
  const uint8_t* recs = m + 40 * g;
  uint64_t off = rd32(m + 4 * grp);
  uint32_t c = rd32(m + 4 * g + 4 * grp);
  for (int l = 0; l < ADM_LANES; ++l) {
    uint64_t len = 8ull * m[8 * g + 32 * grp + l];
    uint64_t s, e;
    lane_range(n, grp, l, &s, &e);
    if (off + len > rec_bytes) return -2;
    const uint8_t* r = recs + off;
    uint64_t rp = 0, o = s;
    while (rp < len && o < e) {
      uint8_t b = r[rp];
      if (b == 255) {
        rp = (rp + 8) / 8 * 8;
      } else if (b == 254) {
        if (rp + 5 > len) return -3;
        out[o++] = ((uint32_t)r[rp + 1] << 24) | ((uint32_t)r[rp + 2] << 16) |
                   ((uint32_t)r[rp + 3] << 8) | (uint32_t)r[rp + 4];
        rp += 5;
      } else {
        uint32_t z = 0;
        while (z < ADM_U32_MAX_K - 1 && rp + z < len && r[rp + z] == 0) ++z;
        if (rp + z >= len) return -4;
        uint8_t code = r[rp + z];
        uint32_t d = (code & 1) ? (uint32_t)(code - 1) / 2 : (uint32_t)code / 2;
        d += (uint32_t)ADM_STEP * z;
        out[o++] = (code & 1) ? c - d : c + d;
        rp += z + 1;
      }
    }
    if (o != e) return -5;
    off += len;
  }
  return 0;
}

int mo_adm_u32_unmap(const uint8_t* m, uint64_t msize, uint64_t n, uint32_t* out) {
  uint64_t g = div_up(n, ADM_GROUP);
  if (msize < 40 * g) return -1;
  for (uint64_t grp = 0; grp < g; ++grp) {
    int rc = adm_u32_unmap_group(m, g, grp, msize - 40 * g, n, out);
    if (rc) return rc;
  }
  return 0;
}

/* ------------------------------------------------------------------------ */
/* rANS: include/ans/GpuANSCodec.h constants                                 */
/* ------------------------------------------------------------------------ */
#define ANS_SYMS 256
#define ANS_BLOCK 4096u                 /* kDefaultBlockSize, :38 */
#define ANS_STATE_BITS 31               /* kANSStateBits, :42 */
#define ANS_ENC_BITS 16                 /* kANSEncodedBits, :43 */
#define ANS_START_STATE (1u << 15)      /* kANSStartState / kANSMinState, :47-50 */
#define ANS_MAGIC 0xd00du               /* :53 */
#define ANS_VERSION 0x0001u             /* :56 */
#define ANS_HDR 32u                     /* sizeof(ANSCoalescedHeader) */

/* GpuANSCodec.h:70-83: header + pdf + warp states + roundUp(nb,2) uint2. */
static uint64_t ans_overhead(uint64_t nb) {
  return ANS_HDR + 2 * ANS_SYMS + 128 * nb + 8 * ((nb + 1) / 2 * 2);
}

/* Histogram of the byte buffer. GpuANSStatistics.h:24-136. */
void mo_ans_histogram(const uint8_t* in, uint64_t n, uint32_t hist[256]) {
  memset(hist, 0, 256 * sizeof(uint32_t));
  for (uint64_t i = 0; i < n; ++i) hist[in[i]]++;
}

/* Probability normalisation, GpuANSStatistics.h:187-385.
 *  1. q = (uint32)((float)2^p * ((float)count / (float)total)), IEEE single
 *     precision, truncated (:225); q = 1 if the symbol is present and q == 0
 *     (:228).
 *  2. Rank symbols by the key (q << 16 | symbol), descending (:239-262).
 *  3. diff = 2^p - sum(q). If positive, repeatedly add 1 to every symbol whose
 *     symbol id (not rank) is below min(diff, 256) (:268-283) -- absent
 *     symbols included. If negative, repeatedly count the entries with q > 1,
 *     and subtract 1 from the ranks [count - min(-diff, count), count)
 *     (:284-326).
 *  4. cdf = exclusive prefix sum of pdf over symbol ids (:347-352).
 * An all-zero histogram leaves pdf/cdf zero (the reference writes nothing). */
int mo_ans_normalize(const uint32_t hist[256], uint32_t total, int prob_bits, uint32_t pdf[256],
                     uint32_t cdf[256]) {
  memset(pdf, 0, 256 * sizeof(uint32_t));
  memset(cdf, 0, 256 * sizeof(uint32_t));
  if (total == 0) return 0;
  uint32_t weight = 1u << prob_bits;
  uint32_t q[256];
  int64_t sum = 0;
  for (int s = 0; s < 256; ++s) {
    volatile float ratio = (float)hist[s] / (float)total;
    volatile float scaled = (float)weight * ratio;
    uint32_t v = (uint32_t)scaled;
    if (hist[s] > 0 && v == 0) v = 1;
    q[s] = v;
    sum += v;
  }
  /* rank order: rank r holds symbol order[r] */
  int order[256];
  for (int s = 0; s < 256; ++s) {
    uint32_t key = (q[s] << 16) | (uint32_t)s;
    int rank = 0;
    for (int t = 0; t < 256; ++t) {
      uint32_t kt = (q[t] << 16) | (uint32_t)t;
      if (kt > key) ++rank;
    }
    order[rank] = s;
  }
  int64_t diff = (int64_t)weight - sum;
  if (diff > 0) {
    while (diff > 0) {
      int64_t it = diff < 256 ? diff : 256;
      for (int s = 0; s < it; ++s) q[s] += 1;
      diff -= it;
    }
  } else if (diff < 0) {
    diff = -diff;
    while (diff > 0) {
      int64_t gt1 = 0;
      for (int r = 0; r < 256; ++r) gt1 += q[order[r]] > 1;
      if (gt1 == 0) return -1; /* unreachable: 2^p >= 512 > 256 symbols */
      int64_t it = diff < gt1 ? diff : gt1;
      int64_t start = gt1 - it;
      for (int64_t r = start; r < gt1; ++r) q[order[r]] -= 1;
      diff -= it;
    }
  }
  uint32_t run = 0;
  for (int s = 0; s < 256; ++s) {
    pdf[s] = q[s];
    cdf[s] = run;
    run += q[s];
  }
  return 0;
}

/* True worst case: a 4 KiB block of symbols whose pdf is 1 at p = 11 costs
 * 11 bits each, 88 words per lane plus one for the start state. The
 * reference's getMaxCompressedSize (GpuANSCodec.h:237-246) assumes 1.25x and
 * can be exceeded by adversarial inputs. */
uint64_t mo_ans_max_compressed_size(uint64_t n) {
  uint64_t nb = div_up(n, ANS_BLOCK);
  uint64_t per_block_words = 32 * (128 * 11 / 16 + 2);
  per_block_words = (per_block_words + 7) / 8 * 8;
  return ans_overhead(nb) + nb * per_block_words * 2;
}

/* rANS encode of one 4 KiB block, GpuANSEncode.h:25-164. Lane l encodes
 * bytes l, l+32, ... in order; each step first renormalises (emit the low 16
 * bits when state >= pdf << (31-p), lanes in ascending order, :40-52), then
 * state = (state / pdf) << p + state % pdf + cdf (:54-69). */
static uint32_t ans_encode_block(int p, const uint8_t* in, uint32_t bs, const uint32_t* pdf,
                                 const uint32_t* cdf, uint32_t state_out[32], uint16_t* words) {
  uint32_t st[32];
  for (int l = 0; l < 32; ++l) st[l] = ANS_START_STATE;
  uint32_t nw = 0;
  uint32_t steps = (bs + 31) / 32;
  for (uint32_t j = 0; j < steps; ++j) {
    for (int l = 0; l < 32; ++l) {
      uint32_t idx = j * 32 + (uint32_t)l;
      if (idx >= bs) continue;
      uint32_t f = pdf[in[idx]];
      if (st[l] >= (f << (ANS_STATE_BITS - p))) {
        words[nw++] = (uint16_t)(st[l] & 0xffff);
        st[l] >>= ANS_ENC_BITS;
      }
    }
    for (int l = 0; l < 32; ++l) {
      uint32_t idx = j * 32 + (uint32_t)l;
      if (idx >= bs) continue;
      uint32_t sym = in[idx];
      uint32_t f = pdf[sym];
      st[l] = ((st[l] / f) << p) + st[l] % f + cdf[sym];
    }
  }
  memcpy(state_out, st, sizeof(st));
  return nw;
}

/* Coalesced stream, GpuANSCodec.h:68-209 and GpuANSEncode.h:181-284:
 *   header{magic<<16|version, numBlocks, uncompressed bytes, compressed words,
 *          options(p in bits 0-3), checksum, unused0, unused1}
 *   u16 pdf[256]; u32 states[nb][32];
 *   uint2 blockWords[roundUp(nb,2)] = {(blockBytes << 16) | words, wordPrefix}
 *   u16 data: each block's words padded to a multiple of 8 words.
 * Bytes the reference leaves uninitialised are written as zero here. */
int64_t mo_ans_encode_ex(int p, const uint8_t* in, uint64_t n, uint8_t* out, uint64_t cap,
                         uint32_t* block_words) {
  if (p < 9 || p > 11) return -1;
  if (n > 0xffffffffull) return -3;
  uint64_t nb = div_up(n, ANS_BLOCK);
  uint32_t hist[256], pdf[256], cdf[256];
  mo_ans_histogram(in, n, hist);
  mo_ans_normalize(hist, (uint32_t)n, p, pdf, cdf);
  uint64_t over = ans_overhead(nb);
  if (cap < over) return -2;
  memset(out, 0, over);
  uint16_t* words = (uint16_t*)malloc(sizeof(uint16_t) * 4096 + 64);
  uint8_t* states = out + ANS_HDR + 512;
  uint8_t* bw = states + 128 * nb;
  uint8_t* data = out + over;
  uint64_t prefix = 0;
  for (uint64_t b = 0; b < nb; ++b) {
    uint32_t bs = (uint32_t)((n - b * ANS_BLOCK) < ANS_BLOCK ? (n - b * ANS_BLOCK) : ANS_BLOCK);
    uint32_t st[32];
    uint32_t nw = ans_encode_block(p, in + b * ANS_BLOCK, bs, pdf, cdf, st, words);
    if (block_words) block_words[b] = nw;
    uint32_t padded = (nw + 7) / 8 * 8;
    if (over + 2 * (prefix + padded) > cap) {
      free(words);
      return -2;
    }
    memcpy(states + 128 * b, st, 128);
    wr32(bw + 8 * b, (bs << 16) | nw);
    wr32(bw + 8 * b + 4, (uint32_t)prefix);
    memcpy(data + 2 * prefix, words, 2 * nw);
    memset(data + 2 * (prefix + nw), 0, 2 * (padded - nw));
    prefix += padded;
  }
  free(words);
  wr32(out + 0, (ANS_MAGIC << 16) | ANS_VERSION);
  wr32(out + 4, (uint32_t)nb);
  wr32(out + 8, (uint32_t)n);
  wr32(out + 12, (uint32_t)prefix);
  wr32(out + 16, (uint32_t)p);
  for (int s = 0; s < 256; ++s) wr16(out + ANS_HDR + 2 * s, (uint16_t)pdf[s]);
  return (int64_t)(over + 2 * prefix);
}

int64_t mo_ans_encode(int p, const uint8_t* in, uint64_t n, uint8_t* out, uint64_t cap) {
  return mo_ans_encode_ex(p, in, n, out, cap, NULL);
}

uint64_t mo_ans_stream_uncompressed_size(const uint8_t* in, uint64_t in_size) {
  if (in_size < ANS_HDR) return 0;
  if ((rd32(in) >> 16) != ANS_MAGIC || (rd32(in) & 0xffff) != ANS_VERSION) return 0;
  return rd32(in + 8);
}

/* Decode, GpuANSDecode.h:27-302 (lookup table :307-377). The table maps a
 * slot s in [0, 2^p) to (symbol, pdf, s - cdf). A block is decoded from its
 * last step to its first; a partial last step (bytes % 32) is handled first
 * (:157-183). Per step: s = state & (2^p-1); state = pdf*(state >> p) + s-cdf;
 * lanes with state < 2^15 then read one word each walking backwards from the
 * block's end, highest lane first (:78-92). The reference validates the
 * header with device asserts; here a bad header returns an error. */
int mo_ans_decode(const uint8_t* in, uint64_t in_size, uint8_t* out, uint64_t out_cap,
                  uint64_t* out_n) {
  if (in_size < ANS_HDR + 512) return -1;
  uint32_t mv = rd32(in);
  if ((mv >> 16) != ANS_MAGIC || (mv & 0xffff) != ANS_VERSION) return -2;
  uint32_t nb = rd32(in + 4);
  uint32_t n = rd32(in + 8);
  uint32_t cw = rd32(in + 12);
  int p = (int)(rd32(in + 16) & 0xf);
  if (p < 9 || p > 11) return -3;
  if (div_up(n, ANS_BLOCK) != nb) return -4;
  uint64_t over = ans_overhead(nb);
  if (in_size < over + 2ull * cw) return -5;
  if (out_cap < n) return -6;
  if (out_n) *out_n = n;
  if (n == 0) return 0;
  uint32_t pdf[256], cdf[256], run = 0;
  for (int s = 0; s < 256; ++s) {
    pdf[s] = rd16(in + ANS_HDR + 2 * s);
    cdf[s] = run;
    run += pdf[s];
  }
  if (run != (1u << p)) return -7;
  uint32_t* lut = (uint32_t*)malloc(sizeof(uint32_t) << p);
  for (int s = 0; s < 256; ++s)
    for (uint32_t j = 0; j < pdf[s]; ++j) lut[cdf[s] + j] = ((j) << 20) | (pdf[s] << 8) | (uint32_t)s;
  const uint8_t* states = in + ANS_HDR + 512;
  const uint8_t* bw = states + 128ull * nb;
  const uint16_t* data = (const uint16_t*)(in + over);
  uint32_t mask = (1u << p) - 1;
  int rc = 0;
  for (uint32_t b = 0; b < nb && rc == 0; ++b) {
    uint32_t st[32];
    memcpy(st, states + 128ull * b, 128);
    uint32_t w0 = rd32(bw + 8ull * b), pre = rd32(bw + 8ull * b + 4);
    uint32_t bs = w0 >> 16, nw = w0 & 0xffff;
    uint32_t expect = (b + 1 == nb) ? n - b * ANS_BLOCK : ANS_BLOCK;
    if (bs != expect || (uint64_t)pre + nw > cw) {
      rc = -8;
      break;
    }
    int64_t ptr = (int64_t)pre + nw; /* one past the last unread word */
    uint8_t* ob = out + (uint64_t)b * ANS_BLOCK;
    uint32_t rem = bs % 32;
    int64_t steps = (int64_t)(bs + 31) / 32;
    for (int64_t j = steps - 1; j >= 0; --j) {
      uint32_t valid = (j == steps - 1 && rem) ? rem : 32;
      int rd[32];
      for (uint32_t l = 0; l < 32; ++l) {
        rd[l] = 0;
        if (l >= valid) continue;
        uint32_t e = lut[st[l] & mask];
        uint32_t sym = e & 0xff, f = (e >> 8) & 0xfff, sc = e >> 20;
        ob[j * 32 + l] = (uint8_t)sym;
        st[l] = f * (st[l] >> p) + sc;
        rd[l] = st[l] < ANS_START_STATE;
      }
      for (int l = 31; l >= 0; --l) {
        if (!rd[l]) continue;
        if (ptr <= (int64_t)pre) {
          rc = -9;
          break;
        }
        --ptr;
        st[l] = (st[l] << 16) + data[ptr];
      }
      if (rc) break;
    }
    if (rc == 0 && ptr != (int64_t)pre) rc = -10;
    for (int l = 0; l < 32 && rc == 0; ++l)
      if (st[l] != ANS_START_STATE) rc = -11;
  }
  free(lut);
  return rc;
}

void mo_ans_mask(uint8_t* s, uint64_t size) {
  if (size < ANS_HDR + 512) return;
  uint32_t opt = rd32(s + 16) & 0xf;
  wr32(s + 16, opt);
  wr32(s + 20, 0);
  wr32(s + 24, 0);
  wr32(s + 28, 0);
  uint32_t nb = rd32(s + 4);
  uint32_t n = rd32(s + 8);
  if (n == 0) memset(s + ANS_HDR, 0, 512);
  uint64_t over = ans_overhead(nb);
  if (over > size) return;
  uint8_t* bw = s + ANS_HDR + 512 + 128ull * nb;
  if (nb & 1) memset(bw + 8ull * nb, 0, 8);
  uint8_t* data = s + over;
  for (uint32_t b = 0; b < nb; ++b) {
    uint32_t nw = rd32(bw + 8ull * b) & 0xffff;
    uint32_t pre = rd32(bw + 8ull * b + 4);
    uint32_t padded = (nw + 7) / 8 * 8;
    if (over + 2ull * (pre + padded) > size) return;
    memset(data + 2ull * (pre + nw), 0, 2ull * (padded - nw));
  }
}

/* ---- end to end ---- */
int64_t mo_mans_compress_u16(int p, const uint16_t* in, uint64_t n, uint8_t* out, uint64_t cap) {
  uint64_t ms = mo_adm_u16_merged_size(in, n);
  uint8_t* m = (uint8_t*)malloc(ms ? ms : 1);
  int64_t r = mo_adm_u16_map(in, n, m, ms);
  if (r < 0) {
    free(m);
    return -4;
  }
  r = mo_ans_encode(p, m, ms, out, cap);
  free(m);
  return r;
}

int mo_mans_decompress_u16(const uint8_t* in, uint64_t in_size, uint64_t n, uint16_t* out) {
  uint64_t ms = mo_ans_stream_uncompressed_size(in, in_size);
  uint8_t* m = (uint8_t*)malloc(ms ? ms : 1);
  uint64_t got = 0;
  int rc = mo_ans_decode(in, in_size, m, ms, &got);
  if (rc == 0) rc = mo_adm_u16_unmap(m, got, n, out) ? -20 : 0;
  free(m);
  return rc;
}

int64_t mo_mans_compress_u32(int p, const uint32_t* in, uint64_t n, uint8_t* out, uint64_t cap) {
  uint64_t ms = mo_adm_u32_max_merged_size(n);
  uint8_t* m = (uint8_t*)malloc(ms ? ms : 1);
  int64_t r = mo_adm_u32_map(in, n, m, ms);
  if (r < 0) {
    free(m);
    return -4;
  }
  r = mo_ans_encode(p, m, (uint64_t)r, out, cap);
  free(m);
  return r;
}

int mo_mans_decompress_u32(const uint8_t* in, uint64_t in_size, uint64_t n, uint32_t* out) {
  uint64_t ms = mo_ans_stream_uncompressed_size(in, in_size);
  uint8_t* m = (uint8_t*)malloc(ms ? ms : 1);
  uint64_t got = 0;
  int rc = mo_ans_decode(in, in_size, m, ms, &got);
  if (rc == 0) rc = mo_adm_u32_unmap(m, got, n, out) ? -20 : 0;
  free(m);
  return rc;
}

/* ------------------------------------------------------------------------ */
/* Multi-threaded variants (OpenMP) of the same functions, used as the timed */
/* CPU baseline. Output is byte-identical to the single-threaded versions.   */
/* ------------------------------------------------------------------------ */
#ifdef _OPENMP
#include <omp.h>
#endif

void mo_set_threads(int n) {
#ifdef _OPENMP
  omp_set_num_threads(n > 0 ? n : 1);
#else
  (void)n;
#endif
}

void mo_ans_histogram_par(const uint8_t* in, uint64_t n, uint32_t hist[256]) {
  memset(hist, 0, 256 * sizeof(uint32_t));
#pragma omp parallel
  {
    uint32_t h[256];
    memset(h, 0, sizeof(h));
#pragma omp for schedule(static)
    for (int64_t i = 0; i < (int64_t)n; ++i) h[in[i]]++;
#pragma omp critical
    for (int s = 0; s < 256; ++s) hist[s] += h[s];
  }
}

/* Encode with blocks distributed over threads: pass 1 encodes every block
 * into a per-block slot of `scratch` (nb * MO_SLOT_WORDS words), pass 2 lays
 * the blocks out at their prefix offsets. */
#define MO_SLOT_WORDS 2880u
uint64_t mo_ans_par_scratch_words(uint64_t n) { return div_up(n, ANS_BLOCK) * MO_SLOT_WORDS; }

int64_t mo_ans_encode_par(int p, const uint8_t* in, uint64_t n, uint8_t* out, uint64_t cap,
                          uint16_t* scratch, uint32_t* scratch_states, uint32_t* scratch_nw) {
  if (p < 9 || p > 11) return -1;
  if (n > 0xffffffffull) return -3;
  uint64_t nb = div_up(n, ANS_BLOCK);
  uint32_t hist[256], pdf[256], cdf[256];
  mo_ans_histogram_par(in, n, hist);
  mo_ans_normalize(hist, (uint32_t)n, p, pdf, cdf);
  uint64_t over = ans_overhead(nb);
  if (cap < over) return -2;
#pragma omp parallel for schedule(dynamic, 16)
  for (int64_t b = 0; b < (int64_t)nb; ++b) {
    uint64_t left = n - (uint64_t)b * ANS_BLOCK;
    uint32_t bs = (uint32_t)(left < ANS_BLOCK ? left : ANS_BLOCK);
    scratch_nw[b] = ans_encode_block(p, in + (uint64_t)b * ANS_BLOCK, bs, pdf, cdf,
                                     scratch_states + 32 * b, scratch + (uint64_t)b * MO_SLOT_WORDS);
  }
  uint64_t prefix = 0;
  uint32_t* pre = (uint32_t*)malloc(sizeof(uint32_t) * (nb ? nb : 1));
  for (uint64_t b = 0; b < nb; ++b) {
    pre[b] = (uint32_t)prefix;
    prefix += (scratch_nw[b] + 7) / 8 * 8;
  }
  if (over + 2 * prefix > cap) {
    free(pre);
    return -2;
  }
  memset(out, 0, ANS_HDR);
  wr32(out + 0, (ANS_MAGIC << 16) | ANS_VERSION);
  wr32(out + 4, (uint32_t)nb);
  wr32(out + 8, (uint32_t)n);
  wr32(out + 12, (uint32_t)prefix);
  wr32(out + 16, (uint32_t)p);
  for (int s = 0; s < 256; ++s) wr16(out + ANS_HDR + 2 * s, (uint16_t)pdf[s]);
  uint8_t* states = out + ANS_HDR + 512;
  uint8_t* bw = states + 128 * nb;
  uint8_t* data = out + over;
  if (nb & 1) memset(bw + 8 * nb, 0, 8);
#pragma omp parallel for schedule(static)
  for (int64_t b = 0; b < (int64_t)nb; ++b) {
    uint64_t left = n - (uint64_t)b * ANS_BLOCK;
    uint32_t bs = (uint32_t)(left < ANS_BLOCK ? left : ANS_BLOCK);
    uint32_t nw = scratch_nw[b];
    memcpy(states + 128 * b, scratch_states + 32 * b, 128);
    wr32(bw + 8 * b, (bs << 16) | nw);
    wr32(bw + 8 * b + 4, pre[b]);
    memcpy(data + 2ull * pre[b], scratch + (uint64_t)b * MO_SLOT_WORDS, 2ull * nw);
    memset(data + 2ull * (pre[b] + nw), 0, 2ull * ((nw + 7) / 8 * 8 - nw));
  }
  free(pre);
  return (int64_t)(over + 2 * prefix);
}

/* Block-parallel decode; no error checks beyond the header (the baseline
 * only decodes streams it produced). */
int mo_ans_decode_par(const uint8_t* in, uint64_t in_size, uint8_t* out, uint64_t out_cap) {
  if (in_size < ANS_HDR + 512) return -1;
  uint32_t nb = rd32(in + 4);
  uint32_t n = rd32(in + 8);
  int p = (int)(rd32(in + 16) & 0xf);
  if (p < 9 || p > 11 || out_cap < n) return -3;
  uint32_t pdf[256], cdf[256], run = 0;
  for (int s = 0; s < 256; ++s) {
    pdf[s] = rd16(in + ANS_HDR + 2 * s);
    cdf[s] = run;
    run += pdf[s];
  }
  if (n && run != (1u << p)) return -7;
  uint32_t* lut = (uint32_t*)malloc(sizeof(uint32_t) << p);
  for (int s = 0; s < 256; ++s)
    for (uint32_t j = 0; j < pdf[s]; ++j) lut[cdf[s] + j] = (j << 20) | (pdf[s] << 8) | (uint32_t)s;
  uint64_t over = ans_overhead(nb);
  const uint8_t* states = in + ANS_HDR + 512;
  const uint8_t* bw = states + 128ull * nb;
  const uint16_t* data = (const uint16_t*)(in + over);
  uint32_t mask = (1u << p) - 1;
#pragma omp parallel for schedule(dynamic, 16)
  for (int64_t b = 0; b < (int64_t)nb; ++b) {
    uint32_t st[32];
    memcpy(st, states + 128 * b, 128);
    uint32_t w0 = rd32(bw + 8 * b), pre = rd32(bw + 8 * b + 4);
    uint32_t bs = w0 >> 16, nw = w0 & 0xffff;
    int64_t ptr = (int64_t)pre + nw;
    uint8_t* ob = out + (uint64_t)b * ANS_BLOCK;
    uint32_t rem = bs % 32;
    int64_t steps = (int64_t)(bs + 31) / 32;
    for (int64_t j = steps - 1; j >= 0; --j) {
      uint32_t valid = (j == steps - 1 && rem) ? rem : 32;
      uint32_t rdm = 0;
      for (uint32_t l = 0; l < valid; ++l) {
        uint32_t e = lut[st[l] & mask];
        ob[j * 32 + l] = (uint8_t)(e & 0xff);
        st[l] = ((e >> 8) & 0xfff) * (st[l] >> p) + (e >> 20);
        rdm |= (uint32_t)(st[l] < ANS_START_STATE) << l;
      }
      for (int l = 31; l >= 0; --l)
        if ((rdm >> l) & 1) st[l] = (st[l] << 16) + data[--ptr];
    }
  }
  free(lut);
  return 0;
}

/* Group-parallel uint16 mapping (same bytes as mo_adm_u16_map_layout): pass 1
 * computes every group's center and signal length, a serial scan gives the
 * offsets, pass 2 writes each group's codes and lane streams. out == NULL
 * returns the mapped size only. */
int64_t mo_adm_u16_map_layout_par(const uint16_t* in, uint64_t n, int layout, uint8_t* out,
                                  uint64_t cap) {
  uint64_t g = div_up(n, ADM_GROUP);
  if (layout < 0 || layout > 2) return -2;
  uint32_t* len = (uint32_t*)calloc(g ? g : 1, sizeof(uint32_t));
  uint32_t* ctr = (uint32_t*)calloc(g ? g : 1, sizeof(uint32_t));
  uint64_t* excl = (uint64_t*)calloc(g ? g : 1, sizeof(uint64_t));
#pragma omp parallel for schedule(static)
  for (int64_t grp = 0; grp < (int64_t)g; ++grp)
    len[grp] = adm_group_len_u16(in, n, (uint64_t)grp, &ctr[grp]);
  uint64_t tot = 0;
  for (uint64_t grp = 0; grp < g; ++grp) {
    excl[grp] = tot;
    tot += len[grp];
  }
  const uint64_t hdr = mo_adm_u16_header_bytes(n, layout);
  const uint64_t msize = hdr + n + 32 * tot;
  if (!out || msize > cap) {  /* out == NULL: size query */
    free(len);
    free(ctr);
    free(excl);
    return out ? -1 : (int64_t)msize;
  }
  const uint64_t pre = hdr - 2 * g;
  uint8_t* p_len = out;
  uint8_t* p_ctr = out + pre;
  uint8_t* p_code = out + hdr;
  uint8_t* p_bits = out + hdr + n;
#pragma omp parallel
  {
    uint8_t lanebuf[ADM_U16_MAX_LANE_BYTES + 8];
#pragma omp for schedule(static)
    for (int64_t gi = 0; gi < (int64_t)g; ++gi) {
      const uint64_t grp = (uint64_t)gi;
      if (layout == MO_LAYOUT_V12) wr16(p_len + 2 * grp, (uint16_t)len[grp]);
      else wr32(p_len + 4 * grp, (uint32_t)excl[grp]);
      wr16(p_ctr + 2 * grp, (uint16_t)ctr[grp]);
      const uint32_t L = len[grp];
      for (int l = 0; l < ADM_LANES; ++l) {
        uint64_t s, e;
        lane_range(n, grp, l, &s, &e);
        memset(lanebuf, 0, sizeof(lanebuf));
        if (layout == MO_LAYOUT_V12 && s >= e) {
          memset(lanebuf, 0xFF, L);
        } else {
          uint32_t b = adm_lane_bits_u16(in, s, e, ctr[grp], lanebuf, p_code + s);
          if (b < L * 8) lanebuf[b >> 3] |= (uint8_t)(0xFFu >> (b & 7));
        }
        memcpy(p_bits + 32 * excl[grp] + (uint64_t)l * L, lanebuf, L);
      }
    }
  }
  if (layout == MO_LAYOUT_CPUV2) wr32(p_len + 4 * g, (uint32_t)tot);
  free(len);
  free(ctr);
  free(excl);
  return (int64_t)msize;
}

/* Group-parallel uint32 mapping: pass 1 sizes every group's records, a
 * serial scan gives offsets, pass 2 writes. */
int64_t mo_adm_u32_map_par(const uint32_t* in, uint64_t n, uint8_t* out, uint64_t cap) {
  uint64_t g = div_up(n, ADM_GROUP);
  uint64_t hdr = 40 * g;
  if (cap < hdr) return -1;
  uint32_t* glen = (uint32_t*)malloc(sizeof(uint32_t) * (g ? g : 1));
#pragma omp parallel for schedule(static)
  for (int64_t grp = 0; grp < (int64_t)g; ++grp) {
    uint64_t gs = (uint64_t)grp * ADM_GROUP, ge = gs + ADM_GROUP;
    if (ge > n) ge = n;
    uint32_t c = adm_center_u32(in, gs, ge);
    wr32(out + 4 * g + 4 * grp, c);
    uint32_t tot = 0;
    for (int l = 0; l < ADM_LANES; ++l) {
      uint64_t s, e;
      lane_range(n, (uint64_t)grp, l, &s, &e);
      uint32_t len = adm_lane_record_u32(in, s, e, c, NULL);
      out[8 * g + 32 * grp + l] = (uint8_t)(len / 8);
      tot += len;
    }
    glen[grp] = tot;
  }
  uint64_t pos = 0;
  for (uint64_t grp = 0; grp < g; ++grp) {
    wr32(out + 4 * grp, (uint32_t)pos);
    pos += glen[grp];
  }
  free(glen);
  if (hdr + pos > cap) return -1;
#pragma omp parallel for schedule(static)
  for (int64_t grp = 0; grp < (int64_t)g; ++grp) {
    uint64_t off = hdr + rd32(out + 4 * grp);
    uint32_t c = rd32(out + 4 * g + 4 * grp);
    for (int l = 0; l < ADM_LANES; ++l) {
      uint64_t s, e;
      lane_range(n, (uint64_t)grp, l, &s, &e);
      off += adm_lane_record_u32(in, s, e, c, out + off);
    }
  }
  return (int64_t)(hdr + pos);
}

int mo_adm_u32_unmap_par(const uint8_t* m, uint64_t msize, uint64_t n, uint32_t* out) {
  uint64_t g = div_up(n, ADM_GROUP);
  if (msize < 40 * g) return -1;
  int bad = 0;
#pragma omp parallel for schedule(static) reduction(| : bad)
  for (int64_t grp = 0; grp < (int64_t)g; ++grp)
    bad |= adm_u32_unmap_group(m, g, (uint64_t)grp, msize - 40 * g, n, out) != 0;
  return bad ? -1 : 0;
}
