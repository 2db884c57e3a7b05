// adm_u16.cuh -- ADM byte mapping of uint16 arrays (unary bit-signal format)
// for sm_100a: the per-group work of the map (fused with the group-length scan
// and the rANS histogram) and of the unmap, shared by the single-buffer and
// batched kernels.
//
// Format: mapping/nv/mappingV15_fused_uint16.cu (map :124-373 / :400-730,
// merged layout :933-957), identical in its bytes to
// mapping/cpu/mappingcpuV2.cpp:35-143. Per group of 512 elements (32 lanes x
// 16 consecutive elements):
//   center = truncated mean; code = 1 (center), 2r (above), 2r+1 (below) with
//   r = d - 126(k-1), k = ceil(d/126); each element appends "1" then k-1 "0"s
//   to its lane's bit stream (MSB first); the group length L is the longest
//   lane in bytes; a shorter lane's final partial byte is filled with 1s.
// Merged: [i32 exclusive L prefix x g][u16 center x g][u8 code x n][bits].
// Compatibility layouts (same codes and bits) replace the length header:
//   kLayoutV12   [u16 L x g] (mappingV12_bit-adm-thrust-prefixsum.cu
//                :606-634; a lane holding no element is 0xFF in all its L
//                bytes, since V12's concat (:405-428) skips it in a buffer
//                filled with 255 (:504));
//   kLayoutCpuV2 [i32 L prefix x (g + 1), the last = total]
//                (mapping/cpu/mappingcpuV2.cpp:117-121, 271-285).
//
// B200 organisation: each warp maps one group at a time, groups handed out
// in order by an atomic counter. The group-length prefix is a single-pass
// decoupled look-back over per-group flags (the reference V15 uses a thrust
// scan plus a concat kernel above 1,024 groups, and an unbounded look-back
// below), so bits are written once, directly at their final offset. Every
// byte written is counted in a per-warp shared histogram, which gives the
// rANS histogram of the merged buffer without reading it again.
#pragma once

#include "ans_table.cuh"

namespace mans {

constexpr int kLayoutV15 = 0, kLayoutV12 = 1, kLayoutCpuV2 = 2;

// Bytes before the centers and before the codes, for g groups.
__host__ __device__ constexpr uint64_t u16_len_bytes(int layout, uint64_t g) {
  return layout == kLayoutV12 ? 2 * g : layout == kLayoutCpuV2 ? 4 * g + 4 : 4 * g;
}
__host__ __device__ constexpr uint64_t u16_header_bytes(int layout, uint64_t g) {
  return u16_len_bytes(layout, g) + 2 * g;
}

constexpr int kMapWarps = kAdmGroupsPerTile;  // 8
constexpr int kMapThreads = kMapWarps * 32;   // 256

// floor(a / 126) for a < 89,240: (a * ceil(2^23/126)) >> 23.
__device__ __forceinline__ uint32_t div126(uint32_t a) {
  return __umulhi(a << 9, 66577u);
}

// k = max(1, ceil(d/126)), code = 2r + (v <= c), r = d + 126 - 126k, i.e.
// code = 2d + 252 + (v <= c) - 252k; (d + 125) << 9 is one multiply-add.
__device__ __forceinline__ void adm_elem_u16(uint32_t v, uint32_t c, uint32_t& k, uint32_t& code) {
  const int s = (int)v - (int)c;
  const uint32_t d = (uint32_t)abs(s);
  k = max(1u, __umulhi(d * 512u + 64000u, 66577u));
  code = d + d + (s <= 0 ? 253u : 252u) - 252u * k;
}

__device__ __forceinline__ uint32_t elem16(const uint32_t (&w)[8], int i) {
  return (w[i >> 1] >> ((i & 1) * 16)) & 0xffffu;
}

// Bits [63-(pos|7), 63-pos] set: the rest of the byte holding stream bit pos.
__device__ __forceinline__ uint64_t tail_fill_mask(uint32_t pos) {
  const uint64_t hi = (pos == 0) ? ~0ull : ((1ull << (64 - pos)) - 1);
  const uint32_t lo_bits = 63 - (pos | 7);
  const uint64_t lo = (1ull << lo_bits) - 1;
  return hi & ~lo;
}

// Lane's 16 elements of group grp as 8 packed words (zeros past n).
__device__ __forceinline__ void load_lane_u16(const uint16_t* __restrict__ in, uint64_t n,
                                              uint64_t grp, int lane, uint32_t (&w)[8]) {
  const uint64_t ls = grp * kAdmGroup + (uint64_t)lane * kAdmChunk;
  if (ls + 16 <= n) {
    const uint4* src = reinterpret_cast<const uint4*>(in + ls);
    const uint4 a = __ldcs(src), b = __ldcs(src + 1);
    w[0] = a.x; w[1] = a.y; w[2] = a.z; w[3] = a.w;
    w[4] = b.x; w[5] = b.y; w[6] = b.z; w[7] = b.w;
  } else {
#pragma unroll
    for (int i = 0; i < 8; ++i) {
      const uint32_t lo = (ls + 2 * i < n) ? in[ls + 2 * i] : 0u;
      const uint32_t hi = (ls + 2 * i + 1 < n) ? in[ls + 2 * i + 1] : 0u;
      w[i] = lo | (hi << 16);
    }
  }
}

// One lane's share of a mapped group between the two halves of the map.
struct Map16Lane {
  uint64_t acc;   // the lane's first 64 stream bits (tail-filled when shorter)
  uint32_t pos;   // the lane's stream bits
  uint32_t L;     // the group's lane length in bytes (the longest lane)
  uint32_t c;     // the group's center
  int cnt;        // valid elements of the lane
};

// x << s with the PTX rule for s >= 64 (the result is 0).
__device__ __forceinline__ uint64_t shl_b64(uint64_t x, uint32_t s) {
  uint64_t r;
  asm("shl.b64 %0, %1, %2;" : "=l"(r) : "l"(x), "r"(s));
  return r;
}

// Codes and unary stream of a lane's elements (kFull: all 16 valid, no
// per-element branch): code bytes packed into codes, each counted in hist;
// the stream's first 64 bits in acc (left-aligned; meaningful when the
// stream is shorter than 64 bits), its length in pos. Each element appends
// "1" and k - 1 zeros at the bottom of acc, which is aligned once at the end.
template <bool kFull>
__device__ __forceinline__ void map16_elems(const uint32_t (&w)[8], uint32_t c, int cnt,
                                            uint32_t* hist, uint32_t (&codes)[4], uint64_t& acc,
                                            uint32_t& pos) {
  uint32_t cb[16];
#pragma unroll
  for (int i = 0; i < 16; ++i) {
    cb[i] = 0;
    if (kFull || i < cnt) {
      uint32_t k, code;
      adm_elem_u16(elem16(w, i), c, k, code);
      cb[i] = code;
      atomicAdd(&hist[code], 1u);
      acc = shl_b64((acc << 1) | 1ull, k - 1);  // k - 1 >= 64 only in a long lane
      pos += k;
    }
    if ((i & 3) == 3)  // four code bytes per word
      codes[i >> 2] = __byte_perm(__byte_perm(cb[i - 3], cb[i - 2], 0x1140u),
                                  __byte_perm(cb[i - 1], cb[i], 0x1140u), 0x5410u);
  }
  acc = (pos - 1u) < 63u ? acc << (64u - pos) : 0ull;
}

// First half of mapping group `grp` (one warp): everything that does not
// depend on the group's offset -- center, codes (stored), the lane bit
// streams' first 64 bits, the group length and the histogram of the codes
// and of a short lane's bit bytes. hist: the warp's shared histogram.
template <int kLayout = kLayoutV15>
__device__ __forceinline__ void map16_front(const uint16_t* __restrict__ in, uint64_t n,
                                            uint8_t* __restrict__ M, uint32_t grp,
                                            uint32_t* hist, int lane, Map16Lane& a) {
  const uint64_t g = div_up_u64(n, kAdmGroup);
  uint8_t* p_code = M + u16_header_bytes(kLayout, g);
  uint32_t w[8];
  load_lane_u16(in, n, grp, lane, w);

  const uint64_t gs = (uint64_t)grp * kAdmGroup;
  const uint64_t ls = gs + (uint64_t)lane * kAdmChunk;
  a.cnt = ls >= n ? 0 : (int)min_u64(16, n - ls);

  // ---- center: truncated mean (u32 sum of at most 512 uint16 values)
  // sum of the 16 halves: S = sum of the words (mod 2^32) counts each high
  // half 65536 times, so the halves sum to S - 65535 * (sum of high halves)
  uint32_t wsum = 0, hsum = 0;
#pragma unroll
  for (int i = 0; i < 8; ++i) {
    wsum += w[i];
    hsum += w[i] >> 16;
  }
  const uint32_t lsum = wsum - 65535u * hsum;
  const uint32_t gsum = __reduce_add_sync(0xffffffffu, lsum);
  const uint32_t gcnt = (uint32_t)min_u64(kAdmGroup, n - gs);
  a.c = gcnt == kAdmGroup ? (gsum >> 9) : gsum / gcnt;

  // ---- map: codes, unary bits (first 64 bits in a register), lane length
  uint32_t codes[4] = {0, 0, 0, 0};
  uint64_t acc = 0;
  uint32_t pos = 0;
  if (a.cnt == 16) map16_elems<true>(w, a.c, 16, hist, codes, acc, pos);
  else map16_elems<false>(w, a.c, a.cnt, hist, codes, acc, pos);
  a.L = __reduce_max_sync(0xffffffffu, (pos + 7) >> 3);
  a.pos = pos;

  // codes: 16-byte aligned (the codes section is aligned by the caller)
  if (a.cnt == 16) {
    *reinterpret_cast<uint4*>(p_code + ls) = make_uint4(codes[0], codes[1], codes[2], codes[3]);
  } else {
#pragma unroll
    for (int i = 0; i < 16; ++i)
      if (i < a.cnt) p_code[ls + i] = (uint8_t)(codes[i >> 2] >> ((i & 3) * 8));
  }
  // bit bytes of a short lane (< 64 bits): tail fill and histogram now. In
  // the V12 layout a lane without elements is all 0xFF.
  const bool v12_empty = kLayout == kLayoutV12 && a.cnt == 0;
  if (pos < 64) {
    if (v12_empty) acc = ~0ull;
    else if (pos < 8 * a.L) acc |= tail_fill_mask(pos);
    const uint32_t hi = (uint32_t)(acc >> 32), lo = (uint32_t)acc;
#pragma unroll
    for (uint32_t b = 0; b < 8; ++b) {
      const uint32_t byte = (b < 4 ? hi >> (24 - 8 * b) : lo >> (56 - 8 * b)) & 0xffu;
      if (b < a.L) atomicAdd(&hist[byte], 1u);
    }
    if (a.L > 8) atomicAdd(&hist[v12_empty ? 0xffu : 0u], a.L - 8);
  }
  a.acc = acc;
}

// A long lane's bit bytes (64 stream bits or more), regenerated byte by byte
// from its elements and counted in hist. Out of line: rare, and its code
// would otherwise crowd the instruction cache of the map loop.
static __device__ __noinline__ void map16_long_lane(const uint16_t* __restrict__ in, uint64_t n,
                                             uint32_t grp, int lane, int cnt, uint32_t c,
                                             uint32_t pos, uint32_t L, uint8_t* dst,
                                             uint32_t* hist) {
  uint32_t w[8];
  load_lane_u16(in, n, grp, lane, w);
  uint32_t cur = 0, bi = 0, bp = 0;
#pragma unroll
  for (int i = 0; i < 16; ++i) {
    if (i < cnt) {
      uint32_t k, code;
      adm_elem_u16(elem16(w, i), c, k, code);
      while ((bp >> 3) > bi) {
        dst[bi++] = (uint8_t)cur;
        atomicAdd(&hist[cur], 1u);
        cur = 0;
      }
      cur |= 0x80u >> (bp & 7);
      bp += k;
    }
  }
  while ((pos >> 3) > bi) {
    dst[bi++] = (uint8_t)cur;
    atomicAdd(&hist[cur], 1u);
    cur = 0;
  }
  if (bi < L) {
    if (pos < 8 * L) cur |= 0xffu >> (pos & 7);
    dst[bi++] = (uint8_t)cur;
    atomicAdd(&hist[cur], 1u);
  }
  for (; bi < L; ++bi) {
    dst[bi] = 0;
    atomicAdd(&hist[0], 1u);
  }
}

// Second half, once the group's bit offset gexcl (in units of 32 bytes) is
// known: the merged size (last group), the group's length (or prefix) and
// center fields with their histogram counts, and the lanes' bit bytes. A
// long lane (64 bits or more) reloads its elements and regenerates its
// stream byte by byte.
template <int kLayout = kLayoutV15>
__device__ __forceinline__ void map16_back(const uint16_t* __restrict__ in, uint64_t n,
                                           uint8_t* __restrict__ M, uint64_t m_cap,
                                           unsigned long long* msize_out, uint32_t grp,
                                           uint32_t gexcl, const Map16Lane& a, const Sink& sink,
                                           uint32_t* hist, int lane) {
  const uint64_t g = div_up_u64(n, kAdmGroup);
  const uint64_t hdr = u16_header_bytes(kLayout, g);
  uint8_t* p_len = M;
  uint8_t* p_ctr = M + u16_len_bytes(kLayout, g);
  uint8_t* p_bits = M + hdr + n;
  const uint64_t bits_base = hdr + n;  // offset of the bits section in M
  const uint32_t L = a.L, c = a.c, pos = a.pos;
  if (lane == 0 && (uint64_t)grp + 1 == g) {
    const unsigned long long msize = bits_base + 32ull * (gexcl + L);
    *msize_out = msize;
    if (msize > m_cap) report(sink, MANS_ERR_WORKSPACE_OVERFLOW, msize);
  }

  // lengths (i32 written as two u16: M is only 2-byte aligned here, or u16 L)
  // and center, one store and one histogram byte per lane
  {
    constexpr uint32_t nlen = kLayout == kLayoutV12 ? 2 : 4;  // length field bytes
    const uint32_t lenv = kLayout == kLayoutV12 ? L : gexcl;
    if ((uint32_t)lane < nlen) atomicAdd(&hist[(lenv >> (8 * lane)) & 0xffu], 1u);
    else if ((uint32_t)lane < nlen + 2) atomicAdd(&hist[(c >> (8 * (lane - nlen))) & 0xffu], 1u);
    if ((uint32_t)lane < nlen / 2)
      reinterpret_cast<uint16_t*>(p_len + (uint64_t)nlen * grp)[lane] =
          (uint16_t)(lenv >> (16 * lane));
    else if ((uint32_t)lane == nlen / 2)
      reinterpret_cast<uint16_t*>(p_ctr + 2ull * grp)[0] = (uint16_t)c;
    if (kLayout == kLayoutCpuV2 && (uint64_t)grp + 1 == g && lane == 0) {
      const uint32_t tot = gexcl + L;  // the CPU layout's extra final prefix word
      reinterpret_cast<uint16_t*>(p_len + 4ull * g)[0] = (uint16_t)(tot & 0xffffu);
      reinterpret_cast<uint16_t*>(p_len + 4ull * g)[1] = (uint16_t)(tot >> 16);
      atomicAdd(&hist[tot & 0xff], 1u);
      atomicAdd(&hist[(tot >> 8) & 0xff], 1u);
      atomicAdd(&hist[(tot >> 16) & 0xff], 1u);
      atomicAdd(&hist[tot >> 24], 1u);
    }
  }
  // bits: lane region [32*gexcl + lane*L, +L) of the bits section
  const uint64_t gend = bits_base + 32ull * ((uint64_t)gexcl + L);
  if (gend <= m_cap) {
    uint8_t* dst = p_bits + 32ull * gexcl + (uint64_t)lane * L;
    if (pos < 64) {
      const uint32_t hi = (uint32_t)(a.acc >> 32), lo = (uint32_t)a.acc;
#pragma unroll
      for (uint32_t b = 0; b < 8; ++b)
        if (b < L) dst[b] = (uint8_t)(b < 4 ? hi >> (24 - 8 * b) : lo >> (56 - 8 * b));
      if (L > 8) {
        const uint8_t rest = (kLayout == kLayoutV12 && a.cnt == 0) ? 0xffu : 0u;
        for (uint32_t b = 8; b < L; ++b) dst[b] = rest;
      }
    } else {
      map16_long_lane(in, n, grp, lane, a.cnt, c, pos, L, dst, hist);
    }
  }
}

// Map group `grp` of one buffer (one warp) with a per-group look-back.
// flags: the buffer's per-group look-back flags; msize_out: written by the
// buffer's last group; hist: the warp's shared histogram. The group length is
// published as soon as it is known; the prefix is read after the work that
// does not depend on it.
template <int kLayout = kLayoutV15>
__device__ __forceinline__ void map16_group(const uint16_t* __restrict__ in, uint64_t n,
                                            uint8_t* __restrict__ M, uint64_t m_cap,
                                            unsigned long long* flags,
                                            unsigned long long* msize_out, uint32_t grp,
                                            uint32_t epoch, const Sink& sink, uint32_t* hist,
                                            int lane) {
  Map16Lane a;
  map16_front<kLayout>(in, n, M, grp, hist, lane, a);
  if (lane == 0) st_flag(&flags[grp], make_flag(grp == 0 ? kFlagIncl : kFlagAgg, epoch, a.L));
  uint32_t gexcl = 0;
  if (grp > 0) {
    gexcl = lookback_exclusive(flags, grp, epoch, sink);
    if (lane == 0) st_flag(&flags[grp], make_flag(kFlagIncl, epoch, gexcl + a.L));
  }
  map16_back<kLayout>(in, n, M, m_cap, msize_out, grp, gexcl, a, sink, hist, lane);
}

// ------------------------------------------------------------------------
// Unmap: restore the lane signals (mappingcpuV2.cpp:161-197, V15 :39-86) and
// values (mappingcpuV2.cpp:202-224, V15 :101-112). One warp per group.
// ------------------------------------------------------------------------
constexpr int kUnmapThreads = 256;

__device__ __forceinline__ uint32_t rd_u32_2aligned(const uint8_t* p) {
  const uint16_t* q = reinterpret_cast<const uint16_t*>(p);
  return (uint32_t)q[0] | ((uint32_t)q[1] << 16);
}

__device__ __forceinline__ uint32_t shl_w(uint32_t x, uint32_t s) {  // 0 for s >= 32
  uint32_t r;
  asm("shl.b32 %0, %1, %2;" : "=r"(r) : "r"(x), "r"(s));
  return r;
}
__device__ __forceinline__ uint64_t shl_w(uint64_t x, uint32_t s) { return shl_b64(x, s); }
__device__ __forceinline__ int clz_w(uint32_t x) { return __clz(x); }
__device__ __forceinline__ int clz_w(uint64_t x) { return __clzll(x); }

// The signal counts of a lane's unary stream held left-aligned in acc (a
// 32-bit word when the group's lanes take at most 4 bytes, else 64 bits;
// nbits = 8L): per element, the zeros after its leading 1. Element i starts
// at bit s (s = 0 for the first); its signal is the distance to the next 1
// bit, at most to the lane's end, and the next element starts there. The
// stream is malformed when it does not start with a 1 or an element starts
// at or past the lane's end (s only grows, so the last element's start
// decides). Returns true when malformed. kFull: all 16 elements are valid
// (no per-element branch).
template <bool kFull, typename W>
__device__ __forceinline__ bool unary_signals(W acc, int nbits, int cnt, uint32_t (&sig)[16]) {
  constexpr int kTop = 8 * (int)sizeof(W) - 1;
  bool bad = (kFull || cnt > 0) && !(acc >> kTop);
  int s = 0;
#pragma unroll
  for (int i = 0; i < 16; ++i) {
    sig[i] = 0;
    if (kFull || i < cnt) {
      if (!kFull || i == 15) bad |= s >= nbits;
      const int t = s + 1;
      const int z = clz_w(shl_w(acc, (uint32_t)t));
      const int g = min(z, max(nbits - t, 0));
      sig[i] = (uint32_t)g;
      s = t + g;
    }
  }
  return bad;
}

// Restore group `grp` of one buffer (one warp). tot: bit bytes / 32
// (validated by the caller). V12 layout: v12_excl holds the exclusive prefix
// of its u16 lengths (computed by the caller).
template <int kLayout = kLayoutV15>
__device__ __forceinline__ void unmap16_group(const uint8_t* __restrict__ M, uint64_t n,
                                              uint64_t tot, uint16_t* __restrict__ out,
                                              uint64_t grp, const Sink& sink, int lane,
                                              const uint32_t* v12_excl = nullptr) {
  const uint64_t g = div_up_u64(n, kAdmGroup);
  const uint64_t bits_base = u16_header_bytes(kLayout, g) + n;
  const uint8_t* p_len = M;
  const uint8_t* p_ctr = M + u16_len_bytes(kLayout, g);
  const uint8_t* p_code = M + u16_header_bytes(kLayout, g);
  const uint8_t* p_bits = M + bits_base;
  uint64_t ex, nx;
  if constexpr (kLayout == kLayoutV12) {
    ex = __ldg(v12_excl + grp);
    nx = ex + reinterpret_cast<const uint16_t*>(p_len)[grp];
  } else {
    ex = rd_u32_2aligned(p_len + 4 * grp);
    nx = grp + 1 < g ? rd_u32_2aligned(p_len + 4 * (grp + 1)) : tot;
  }
  // the layouts that record the total must agree with the decoded size
  const bool last = grp + 1 == g;
  if ((kLayout == kLayoutV12 && last && nx != tot) ||
      (kLayout == kLayoutCpuV2 && last && rd_u32_2aligned(p_len + 4 * g) != tot)) {
    if (lane == 0) report(sink, MANS_ERR_CORRUPT, grp);
    return;
  }
  if (ex > nx || nx > tot) {
    if (lane == 0) report(sink, MANS_ERR_CORRUPT, grp);
    return;
  }
  const uint32_t L = (uint32_t)(nx - ex);
  const uint32_t c = reinterpret_cast<const uint16_t*>(p_ctr)[grp];
  const uint64_t ls = grp * kAdmGroup + (uint64_t)lane * kAdmChunk;
  const int cnt = ls >= n ? 0 : (int)min_u64(16, n - ls);
  uint32_t codes[4] = {0, 0, 0, 0};
  if (cnt == 16) {
    const uint4 v = __ldcs(reinterpret_cast<const uint4*>(p_code + ls));
    codes[0] = v.x; codes[1] = v.y; codes[2] = v.z; codes[3] = v.w;
  } else {
#pragma unroll
    for (int i = 0; i < 16; ++i)
      if (i < cnt) codes[i >> 2] |= (uint32_t)p_code[ls + i] << ((i & 3) * 8);
  }
  const uint8_t* src = p_bits + 32ull * ex + (uint64_t)lane * L;
  uint32_t sig[16];
  bool bad = false;
  if (L <= 8) {
    uint64_t acc = 0;
#pragma unroll
    for (uint32_t b = 0; b < 8; ++b)  // all loads in flight at once
      if (b < L) acc |= (uint64_t)__ldg(src + b) << (56 - 8 * b);
    if (L <= 4) {
      const uint32_t a32 = (uint32_t)(acc >> 32);
      if (cnt == 16) bad = unary_signals<true>(a32, (int)(8 * L), 16, sig);
      else bad = unary_signals<false>(a32, (int)(8 * L), cnt, sig);
    } else {
      if (cnt == 16) bad = unary_signals<true>(acc, (int)(8 * L), 16, sig);
      else bad = unary_signals<false>(acc, (int)(8 * L), cnt, sig);
    }
  } else {
    // Long lanes: scan byte by byte like the reference.
    int idx = -1;
#pragma unroll
    for (int i = 0; i < 16; ++i) sig[i] = 0;
    for (uint32_t b = 0; b < L && idx < 16; ++b) {
      const uint32_t byte = src[b];
      for (int bit = 7; bit >= 0 && idx < 16; --bit) {
        if ((byte >> bit) & 1u) {
          ++idx;
        } else if (idx < 0) {
          bad = true;
        } else {
#pragma unroll
          for (int i = 0; i < 16; ++i) sig[i] += (i == idx) ? 1u : 0u;
        }
      }
    }
    if (idx < cnt - 1) bad = true;
  }
  if (__any_sync(0xffffffffu, bad) && lane == 0) report(sink, MANS_ERR_CORRUPT, grp);
  uint32_t vals[8];
#pragma unroll
  for (int i = 0; i < 16; i += 2) {
    uint32_t r[2];
#pragma unroll
    for (int h = 0; h < 2; ++h) {
      const uint32_t code = __byte_perm(codes[(i + h) >> 2], 0u, 0x4440u | ((i + h) & 3));
      const uint32_t d = (code >> 1) + 126u * sig[i + h];
      r[h] = (code & 1u) ? c - d : c + d;
    }
    vals[i >> 1] = __byte_perm(r[0], r[1], 0x5410u);  // low halves of both
  }
  if (cnt == 16) {
    uint4* o = reinterpret_cast<uint4*>(out + ls);
    o[0] = make_uint4(vals[0], vals[1], vals[2], vals[3]);
    o[1] = make_uint4(vals[4], vals[5], vals[6], vals[7]);
  } else {
#pragma unroll
    for (int i = 0; i < 16; ++i)
      if (i < cnt) out[ls + i] = (uint16_t)(vals[i >> 1] >> ((i & 1) * 16));
  }
}

}  // namespace mans
