// adm_u32.cuh -- ADM byte mapping of uint32 arrays (escape-byte format) for
// sm_100a: the per-group work of the map (fused with the record-offset scan
// and the rANS histogram) and of the unmap, shared by the single-buffer and
// batched kernels.
//
// Element format: mapping/nv/mappingV9_fuse.cu:458-651. Per lane of 16
// consecutive elements, with the group center c (truncated mean):
//   k = 1 (v == c) or ceil(|v-c|/126); k <= 8: k-1 zero bytes then the code
//   byte (1, 2r, 2r+1 as in the uint16 format, :530-540); k > 8: 254 and the
//   value big-endian (:541-548); the record is padded with 255 to a multiple
//   of 8 bytes (:634-639). Records are concatenated in group-major,
//   lane-major order (exclusive scan :875, coalescing :654-676).
// The reference persists only the records (:998) and so cannot be decoded
// from its file. The merged layout here adds what a decoder needs:
//   [i32 exclusive record offset per group x g][u32 center x g]
//   [u8 record length / 8 per lane x 32g][records]
// Defined where the reference is not: the center uses a 64-bit sum (the
// reference's uint32 sum wraps once a group's sum reaches 2^32) and |v-c| is
// computed without overflow (the reference's int diff is undefined for
// values >= 2^31). Where the reference is defined the records are identical.
#pragma once

#include "ans_table.cuh"
#include "smem_io.cuh"

namespace mans {


constexpr int kMap32Warps = kAdmGroupsPerTile;  // 8
constexpr int kMap32Threads = kMap32Warps * 32;
constexpr uint32_t kRecMax = kAdmChunk * 8;    // longest lane record: 128 bytes
constexpr uint32_t kGroupRecMax = 32 * kRecMax;  // 4096

__device__ __forceinline__ uint32_t div126_u32(uint32_t a) {  // a < 89,240
  return __umulhi(a << 9, 66577u);
}

// Per-element record bytes: k (k <= 8) or 5 (escape).
__device__ __forceinline__ void adm_elem_u32(uint32_t v, uint32_t c, uint32_t& nbytes,
                                             uint32_t& code, bool& esc) {
  const uint32_t d = v > c ? v - c : c - v;
  if (d > 8u * kAdmStep) {
    esc = true;
    nbytes = 5;
    code = 0;
    return;
  }
  esc = false;
  const uint32_t k = max(1u, div126_u32(d + 125u));
  const uint32_t r = d + 126u - 126u * k;
  nbytes = k;
  code = 2u * r + (v <= c ? 1u : 0u);
}

struct Map32Smem {
  alignas(16) uint8_t stage[kMap32Warps][kGroupRecMax + 16];
};

// Lane's 16 elements of group grp (zeros past n).
__device__ __forceinline__ void load_lane_u32(const uint32_t* __restrict__ in, uint64_t n,
                                              uint64_t grp, int lane, uint32_t (&v)[16]) {
  const uint64_t ls = grp * kAdmGroup + (uint64_t)lane * kAdmChunk;
  if (ls + 16 <= n) {
    const uint4* src = reinterpret_cast<const uint4*>(in + ls);
#pragma unroll
    for (int q = 0; q < 4; ++q) {
      const uint4 a = __ldcs(src + q);
      v[4 * q] = a.x; v[4 * q + 1] = a.y; v[4 * q + 2] = a.z; v[4 * q + 3] = a.w;
    }
  } else {
#pragma unroll
    for (int i = 0; i < 16; ++i) v[i] = ls + i < n ? in[ls + i] : 0u;
  }
}

// Stage a lane's record at phase 0 as whole 8-byte words: bytes are
// appended to a 16-byte accumulator (lo, hi) and each completed word is
// stored once; the last word is padded with 255. Record starts are
// multiples of 8, so every store is an aligned 8-byte store. kFull: all 16
// elements are valid (no per-element branch on the byte count).
template <bool kFull>
__device__ __forceinline__ void map32_stage(const uint32_t* __restrict__ in, uint64_t ls,
                                            const uint32_t (&nbp)[2], const uint32_t (&codes)[4],
                                            uint32_t escm, uint32_t* hist, uint8_t* rec) {
  uint64_t lo = 0, hi = 0;
  uint32_t fill = 0, wpos = 0;
#pragma unroll
  for (int i = 0; i < 16; ++i) {
    const uint32_t nb = (nbp[i >> 3] >> ((i & 7) * 4)) & 0xfu;
    if (kFull || nb != 0) {
      if ((escm >> i) & 1u) {
        const uint32_t x = __ldg(in + ls + i);  // re-read: keeps v[] out of the live range
        // 254 then the value big-endian
        const uint64_t e = 254ull | ((uint64_t)__byte_perm(x, 0, 0x0123) << 8);
        lo |= e << (8 * fill);
        hi |= fill ? e >> (64 - 8 * fill) : 0ull;
        atomicAdd(&hist[254], 1u);
        atomicAdd(&hist[x >> 24], 1u);
        atomicAdd(&hist[(x >> 16) & 0xff], 1u);
        atomicAdd(&hist[(x >> 8) & 0xff], 1u);
        atomicAdd(&hist[x & 0xff], 1u);
      } else {
        // nb - 1 zero bytes, then the code byte
        const uint32_t code = (codes[i >> 2] >> ((i & 3) * 8)) & 0xffu;
        const uint32_t at = fill + nb - 1;  // < 15
        if (at < 8) lo |= (uint64_t)code << (8 * at);
        else hi |= (uint64_t)code << (8 * (at - 8));
        atomicAdd(&hist[code], 1u);
      }
      fill += nb;
      if (fill >= 8) {
        *reinterpret_cast<uint64_t*>(rec + wpos) = lo;
        wpos += 8;
        lo = hi;
        hi = 0;
        fill -= 8;
      }
    }
  }
  if (fill) *reinterpret_cast<uint64_t*>(rec + wpos) = lo | (~0ull << (8 * fill));
}

// Map group `grp` of one buffer (one warp). flags: the buffer's per-group
// look-back flags; msize_out: written by the buffer's last group; hist: the
// warp's shared histogram; stage: the warp's kGroupRecMax + 16 byte stage.
__device__ __forceinline__ void map32_group(const uint32_t* __restrict__ in, uint64_t n,
                                            uint8_t* __restrict__ M, uint64_t m_cap,
                                            unsigned long long* flags,
                                            unsigned long long* msize_out, uint32_t grp,
                                            uint32_t epoch, const Sink& sink, uint32_t* hist,
                                            uint8_t* stage, int lane) {
  const uint64_t g = div_up_u64(n, kAdmGroup);
  const uint64_t rec_base = 40 * g;
  uint32_t v[16];
  load_lane_u32(in, n, grp, lane, v);

  const uint64_t gs = (uint64_t)grp * kAdmGroup;
  const uint64_t ls = gs + (uint64_t)lane * kAdmChunk;
  const int cnt = ls >= n ? 0 : (int)min_u64(16, n - ls);
  // center: 64-bit sum
  unsigned long long lsum = 0;
#pragma unroll
  for (int i = 0; i < 16; ++i) lsum += v[i];
#pragma unroll
  for (int o = 16; o > 0; o >>= 1) lsum += __shfl_xor_sync(0xffffffffu, lsum, o);
  const uint32_t gcnt = (uint32_t)min_u64(kAdmGroup, n - gs);
  const uint32_t c = (uint32_t)(gcnt == kAdmGroup ? (lsum >> 9) : lsum / gcnt);

  // each element once: bytes (k or 5), code byte, escape flag
  uint32_t nbp[2] = {0, 0};      // 4-bit byte counts
  uint32_t codes[4] = {0, 0, 0, 0};
  uint32_t escm = 0, rlen = 0;
#pragma unroll
  for (int i = 0; i < 16; ++i) {
    uint32_t nb, code;
    bool esc;
    adm_elem_u32(v[i], c, nb, code, esc);
    nb = i < cnt ? nb : 0u;
    nbp[i >> 3] |= nb << ((i & 7) * 4);
    codes[i >> 2] |= code << ((i & 3) * 8);
    escm |= (esc && i < cnt) ? (1u << i) : 0u;
    rlen += nb;
  }
  const uint32_t padded = (rlen + 7) & ~7u;
  uint32_t incl = padded;
#pragma unroll
  for (int o = 1; o < 32; o <<= 1) {
    const uint32_t y = __shfl_up_sync(0xffffffffu, incl, o);
    if (lane >= o) incl += y;
  }
  const uint32_t loff = incl - padded;
  const uint32_t gtot = __shfl_sync(0xffffffffu, incl, 31);

  // publish the group's aggregate now; the prefix is read after staging
  if (lane == 0) st_flag(&flags[grp], make_flag(grp == 0 ? kFlagIncl : kFlagAgg, epoch, gtot));

  if (cnt == 16) map32_stage<true>(in, ls, nbp, codes, escm, hist, stage + loff);
  else map32_stage<false>(in, ls, nbp, codes, escm, hist, stage + loff);
  {
    // zero bytes: all bytes that are not codes, escapes or padding
    const uint32_t nesc = __popc(escm);
    const uint32_t ncode = (uint32_t)cnt - nesc;
    const uint32_t zeros = rlen - ncode - 5 * nesc;
    if (zeros) atomicAdd(&hist[0], zeros);
    if (padded > rlen) atomicAdd(&hist[255], padded - rlen);
  }
  M[8 * g + 32ull * grp + lane] = (uint8_t)(padded >> 3);
  atomicAdd(&hist[padded >> 3], 1u);

  // group record offset (predecessors have had the staging time to finish)
  uint32_t goff = 0;
  if (grp > 0) {
    goff = lookback_exclusive(flags, grp, epoch, sink);
    if (lane == 0) st_flag(&flags[grp], make_flag(kFlagIncl, epoch, goff + gtot));
  }
  if (lane == 0) {
    if ((uint64_t)grp + 1 == g) {
      const unsigned long long msize = rec_base + (unsigned long long)goff + gtot;
      *msize_out = msize;
      if (msize > m_cap) report(sink, MANS_ERR_WORKSPACE_OVERFLOW, msize);
    }
    reinterpret_cast<uint32_t*>(M)[grp] = goff;
    reinterpret_cast<uint32_t*>(M + 4 * g)[grp] = c;
    atomicAdd(&hist[goff & 0xff], 1u);
    atomicAdd(&hist[(goff >> 8) & 0xff], 1u);
    atomicAdd(&hist[(goff >> 16) & 0xff], 1u);
    atomicAdd(&hist[goff >> 24], 1u);
    atomicAdd(&hist[c & 0xff], 1u);
    atomicAdd(&hist[(c >> 8) & 0xff], 1u);
    atomicAdd(&hist[(c >> 16) & 0xff], 1u);
    atomicAdd(&hist[c >> 24], 1u);
  }
  __syncwarp();
  // store: M + rec_base is 16-byte aligned and goff a multiple of 8
  if (rec_base + (uint64_t)goff + gtot <= m_cap) {
    uint2* dst = reinterpret_cast<uint2*>(M + rec_base + goff);
    const uint2* src = reinterpret_cast<const uint2*>(stage);
    for (uint32_t i = lane; i < gtot / 8; i += 32) dst[i] = src[i];
  }
  __syncwarp();
}

// ------------------------------------------------------------------------
// Unmap (record decode of mappingV9_fuse.cu:126-157). One warp per group;
// the group's records are staged in shared memory with coalesced loads, then
// each lane walks its record with an 8-byte window: three aligned 32-bit
// shared loads and two byte permutes give the bytes at the cursor, the
// leading zero bytes are counted with one bit scan, and a 254 marker takes
// the next four bytes as a big-endian literal.
// ------------------------------------------------------------------------
constexpr int kUnmap32Warps = 8;
constexpr int kUnmap32Threads = kUnmap32Warps * 32;

struct Unmap32Smem {
  alignas(16) uint8_t stage[kUnmap32Warps][kGroupRecMax + 48];
};

// One lane's record (nw 8-byte words at rw) back to its values; returns the
// bytes consumed. kFull: all 16 elements are valid (no per-element branch on
// the count).
template <bool kFull>
__device__ __forceinline__ uint32_t unmap32_lane(const uint64_t* rw, uint32_t nw, uint32_t c,
                                                 int cnt, uint32_t (&vals)[16], bool& bad) {
  uint64_t A = nw > 0 ? rw[0] : 0ull, B = nw > 1 ? rw[1] : 0ull;
  uint32_t blk = 0, cur = 0;
#pragma unroll
  for (int i = 0; i < 16; ++i) {
    vals[i] = 0;
    if (kFull || i < cnt) {
      const uint32_t sh = 8u * (cur & 7u);
      uint64_t bsh;  // B << (64 - sh), 0 for sh == 0 (PTX clamps the shift)
      asm("shl.b64 %0, %1, %2;" : "=l"(bsh) : "l"(B), "r"(64u - sh));
      const uint64_t win = (A >> sh) | bsh;
      const uint32_t lo = (uint32_t)win, hi = (uint32_t)(win >> 32);
      uint32_t used;
      if ((lo & 0xffu) == 254u) {
        vals[i] = __byte_perm(lo, hi, 0x1234);  // big-endian literal, bytes 1..4
        used = 5;
      } else {
        // leading zero bytes (at most 7), then the code byte
        // (a window of eight zero bytes only occurs in a corrupt record)
        const uint32_t z = min(7u, lo ? (uint32_t)(__ffs(lo) - 1) >> 3
                                      : 4u + ((uint32_t)(__ffs(hi) - 1) >> 3));
        const uint32_t code = __byte_perm(lo, hi, z) & 0xffu;  // byte z of the window
        bad |= code - 1u >= 253u;  // 0 (an all-zero window), 254 or 255
        const uint32_t d = (code >> 1) + 126u * z;
        vals[i] = (code & 1u) ? c - d : c + d;
        used = z + 1;
      }
      cur += used;
      if ((cur >> 3) != blk) {  // crossed into the next word
        ++blk;
        A = B;
        B = blk + 1 < nw ? rw[blk + 1] : 0ull;
      }
    }
  }
  return cur;
}

// Restore group `grp` of one buffer (one warp). rec_bytes: record bytes of
// the merged buffer (validated by the caller); stage: the warp's
// kGroupRecMax + 48 byte stage.
__device__ __forceinline__ void unmap32_group(const uint8_t* __restrict__ M, uint64_t n,
                                              uint64_t rec_bytes, uint32_t* __restrict__ out,
                                              uint64_t grp, const Sink& sink, uint8_t* stage,
                                              int lane) {
  const uint64_t g = div_up_u64(n, kAdmGroup);
  const uint64_t rec_base = 40 * g;
  const uint32_t goff = reinterpret_cast<const uint32_t*>(M)[grp];
  const uint32_t c = reinterpret_cast<const uint32_t*>(M + 4 * g)[grp];
  const uint32_t len = 8u * M[8 * g + 32 * grp + lane];
  uint32_t incl = len;
#pragma unroll
  for (int o = 1; o < 32; o <<= 1) {
    const uint32_t y = __shfl_up_sync(0xffffffffu, incl, o);
    if (lane >= o) incl += y;
  }
  const uint32_t loff = incl - len;
  const uint32_t gtot = __shfl_sync(0xffffffffu, incl, 31);
  const uint64_t ls = grp * kAdmGroup + (uint64_t)lane * kAdmChunk;
  const int cnt = ls >= n ? 0 : (int)min_u64(16, n - ls);
  if ((uint64_t)goff + gtot > rec_bytes || gtot > kGroupRecMax || (goff & 7)) {
    if (lane == 0) report(sink, MANS_ERR_CORRUPT, grp);
    return;
  }
  const uint8_t* src = M + rec_base + goff;
  __syncwarp();
  warp_load_phase(stage, src, gtot, lane);
  __syncwarp();
  // The lane's record, 8-byte aligned in shared memory (phase 0 or 8, loff %
  // 8 == 0), is read as a stream of 8-byte words: A and B hold words blk and
  // blk + 1, the cursor's bytes are a funnel shift of the two, and a word is
  // loaded only when the cursor crosses into the next one (at most once per
  // element, since an element takes at most 8 bytes). Words past the record
  // read as zeros, so a corrupt record never reads outside it.
  const uint64_t* rw = reinterpret_cast<const uint64_t*>(stage + phase16(src) + loff);
  const uint32_t nw = len >> 3;
  uint32_t vals[16];
  bool bad = false;
  uint32_t cur;
  if (cnt == 16) cur = unmap32_lane<true>(rw, nw, c, 16, vals, bad);
  else cur = unmap32_lane<false>(rw, nw, c, cnt, vals, bad);
  bad |= cur > len;
  if (__any_sync(0xffffffffu, bad) && lane == 0) report(sink, MANS_ERR_CORRUPT, grp);
  if (cnt == 16) {
    uint4* dst = reinterpret_cast<uint4*>(out + ls);
#pragma unroll
    for (int q = 0; q < 4; ++q)
      dst[q] = make_uint4(vals[4 * q], vals[4 * q + 1], vals[4 * q + 2], vals[4 * q + 3]);
  } else {
#pragma unroll
    for (int i = 0; i < 16; ++i)
      if (i < cnt) out[ls + i] = vals[i];
  }
}

}  // namespace mans
