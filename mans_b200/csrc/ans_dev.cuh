// ans_dev.cuh -- per-block work of the byte rANS codec for sm_100a (encode
// with in-place output compaction, decode), shared by the single-buffer and
// batched kernels.
//
// Arithmetic and layout: include/ans/GpuANSEncode.h:25-164 and :181-284,
// include/ans/GpuANSDecode.h:27-302 (see ans_codec.cu for the organisation).
#pragma once

#include "ans_table.cuh"
#include "smem_io.cuh"

namespace mans {

constexpr int kEncWarps = 8;
constexpr int kEncThreads = kEncWarps * 32;
constexpr uint32_t kEncOutWords = kAnsMaxBlockWords + 8;
// A block's words compacted in global memory: slots of whole 128-byte lines.
constexpr uint32_t kEncSlotBytes = (kEncOutWords * 2 + 127) / 128 * 128;

constexpr uint32_t kEncStageBytes = kAnsBlock + 16;  // a block plus its 16-byte phase

// The encoder's per-symbol entry in shared memory, expanded from the packed
// table (make_enc_entry) so that a step needs almost no field extraction:
// {reciprocal, renormalisation threshold pdf << (31 - p), bias,
//  shift | cmpl << 5}. The quotient's shift is taken from the low five bits
// of the last word by a wrapping funnel shift.
struct alignas(16) EncEntry4 {
  uint32_t rcp, thr, bias, cs;
};
__device__ __forceinline__ EncEntry4 expand_enc_entry(uint2 e, int p) {
  const uint32_t cmpl = e.y >> 20;
  return EncEntry4{e.x, ((1u << p) - cmpl) << (kAnsStateBits - p), (e.y >> 5) & 0x1fffu,
                   (e.y & 31u) | (cmpl << 5)};
}

struct EncSmemSlots {  // words go to global slots
  union {
    EncEntry4 table4[kAnsSyms];  // expanded entries
    uint2 table2[kAnsSyms];      // packed entries
  };
  alignas(16) uint8_t in[kEncWarps][kEncStageBytes];
  uint64_t bar[kEncWarps];
};
struct EncSmem {  // words compacted in shared memory
  union {
    EncEntry4 table4[kAnsSyms];
    uint2 table2[kAnsSyms];
  };
  alignas(16) uint8_t in[kEncWarps][kEncStageBytes];
  uint64_t bar[kEncWarps];
  alignas(16) uint16_t out[kEncWarps][kEncOutWords];
};

// The coding step's symbol arithmetic for precision kP:
// x' = (xr / pdf << p) + xr % pdf + cdf = xr + bias + q * cmpl, q = xr / pdf.
template <int kP>
__device__ __forceinline__ uint32_t enc_code(uint32_t xr, const uint2& e) {
  const uint32_t q = __funnelshift_r(__umulhi(xr, e.x), 0u, e.y);  // shift = y & 31
  return xr + ((e.y >> 5) & 0x1fffu) + q * (e.y >> 20);
}
template <int kP>
__device__ __forceinline__ uint32_t enc_code(uint32_t xr, const EncEntry4& e) {
  const uint32_t q = __funnelshift_r(__umulhi(xr, e.rcp), 0u, e.cs);  // shift = cs & 31
  return xr + e.bias + q * (e.cs >> 5);
}
template <int kP>
__device__ __forceinline__ uint32_t enc_threshold(const uint2& e) {
  return ((1u << kP) - (e.y >> 20)) << (kAnsStateBits - kP);
}
template <int kP>
__device__ __forceinline__ uint32_t enc_threshold(const EncEntry4& e) {
  return e.thr;
}

// One interleaved step: renormalise (emit 16 bits, lanes in ascending order
// into the compacted word buffer), then code the symbol.
// kGuard: drop words past the buffer (see encode_words).
template <int kP, bool kGuard, bool kShared, typename TabT>
__device__ __forceinline__ void enc_step(bool valid, uint32_t& x, uint32_t sym,
                                         const TabT* __restrict__ tab, uint16_t* __restrict__ out,
                                         uint32_t& nw, uint32_t ltmask) {
  const TabT e = tab[sym];
  const bool wr = valid && x >= enc_threshold<kP>(e);
  const uint32_t vote = __ballot_sync(0xffffffffu, wr);
  const uint32_t idx = nw + __popc(vote & ltmask);
  const bool st = wr && (!kGuard || idx < kEncOutWords);
  if constexpr (kShared) {
    asm volatile("{\n .reg .pred q;\n setp.ne.u32 q, %2, 0;\n @q st.shared.u16 [%0], %1;\n}\n"
                 ::"r"((uint32_t)__cvta_generic_to_shared(out + idx)), "h"((uint16_t)x),
                 "r"((uint32_t)st)
                 : "memory");
  } else {
    asm volatile("{\n .reg .pred q;\n setp.ne.u32 q, %2, 0;\n @q st.global.u16 [%0], %1;\n}\n"
                 ::"l"(out + idx), "h"((uint16_t)x), "r"((uint32_t)st)
                 : "memory");
  }
  nw += __popc(vote);
  const uint32_t xr = wr ? (x >> 16) : x;
  x = valid ? enc_code<kP>(xr, e) : xr;
}

__device__ __forceinline__ void discard_l2_line(const void* p) {
  asm volatile("discard.global.L2 [%0], 128;" ::"l"(p) : "memory");
}

// The coding of one staged block (syms: the lane's first symbol in the stage,
// bs bytes) at precision kP. kShared: sout is in shared memory (else a
// global slot). Returns the word count; x receives the lane's final state.
template <int kP, bool kShared, typename TabT>
__device__ __forceinline__ uint32_t encode_staged(const uint8_t* syms, uint32_t bs,
                                                  const TabT* table, uint16_t* sout, int lane,
                                                  uint32_t& x) {
  const uint32_t ltmask = lanemask_lt();
  x = kAnsStartState;
  uint32_t nw = 0;
  const uint32_t full = bs >> 5;
  uint32_t j = 0;
  // Each step adds at most 32 words, and nw is the same in every lane: while
  // nw <= kRoom the next eight steps fit in the buffer without a check. The
  // eight symbol loads of a round do not depend on the state, so they issue
  // ahead of the round's coding chain.
  constexpr uint32_t kRoom = kEncOutWords - 8 * 32;
  for (; j + 8 <= full && nw <= kRoom; j += 8) {
#pragma unroll
    for (int u = 0; u < 8; ++u)
      enc_step<kP, false, kShared>(true, x, syms[(j + u) * 32], table, sout, nw, ltmask);
  }
  const bool tail_valid = (uint32_t)lane < (bs & 31);
  if (nw <= kRoom) {  // at most seven more steps and the partial one
    for (; j < full; ++j)
      enc_step<kP, false, kShared>(true, x, syms[j * 32], table, sout, nw, ltmask);
    if (bs & 31)
      enc_step<kP, false, kShared>(tail_valid, x, tail_valid ? syms[j * 32] : 0u, table, sout, nw,
                                   ltmask);
  } else {
    for (; j < full; ++j)
      enc_step<kP, true, kShared>(true, x, syms[j * 32], table, sout, nw, ltmask);
    if (bs & 31)
      enc_step<kP, true, kShared>(tail_valid, x, tail_valid ? syms[j * 32] : 0u, table, sout, nw,
                                  ltmask);
  }
  return nw;
}

// Encode block b of one buffer (one warp) into the warp's word buffer sout
// (kSharedOut: in shared memory, else a per-warp slot in global memory,
// which stays in L2): one bulk copy of the block into the warp's stage, then the
// interleaved coding; the word count is padded to a 16-byte multiple with
// zeros (GpuANSEncode.h:275). Returns the number of words; x receives the
// lane's final state.
template <bool kSharedOut, typename TabT>
__device__ __forceinline__ uint32_t encode_words(const uint8_t* __restrict__ in, uint64_t n,
                                                 uint32_t b, const TabT* table, uint8_t* stage,
                                                 uint64_t* bar, uint32_t& parity, uint16_t* sout,
                                                 int p, const Sink& sink, int lane, uint32_t& x) {
  const uint64_t start = (uint64_t)b * kAnsBlock;
  const uint32_t bs = (uint32_t)min_u64(kAnsBlock, n - start);
  // one bulk copy of the block (rounded out to 16-byte boundaries) into this
  // warp's stage; the previous block's reads of the stage are complete
  __syncwarp();
  if (lane == 0) {
    const uintptr_t a0 = reinterpret_cast<uintptr_t>(in + start) & ~uintptr_t(15);
    const uintptr_t a1 = (reinterpret_cast<uintptr_t>(in + start) + bs + 15) & ~uintptr_t(15);
    bulk_load(stage, reinterpret_cast<const void*>(a0), (uint32_t)(a1 - a0), bar);
  }
  if (!mbar_wait(bar, parity) && lane == 0) report(sink, MANS_ERR_TIMEOUT, b);
  parity ^= 1u;
  const uint8_t* syms = stage + phase16(in + start) + lane;
  uint32_t nw;
  switch (p) {
    case 9: nw = encode_staged<9, kSharedOut>(syms, bs, table, sout, lane, x); break;
    case 10: nw = encode_staged<10, kSharedOut>(syms, bs, table, sout, lane, x); break;
    default: nw = encode_staged<11, kSharedOut>(syms, bs, table, sout, lane, x); break;
  }
  // A table that fits the block's bytes keeps each lane within its bound of
  // words (kAnsMaxBlockWords / 32); only a table built from other bytes (two
  // calls racing on one scratch area) can exceed it. Word writes past the
  // buffer are dropped above, and the block is reported.
  if (nw > kAnsMaxBlockWords) {
    if (lane == 0) report(sink, MANS_ERR_CORRUPT, b);
    nw = kAnsMaxBlockWords;
  }
  const uint32_t padded = (nw + 7) & ~7u;
  if ((uint32_t)lane < padded - nw) sout[nw + lane] = 0;
  return nw;
}

// Store block b, whose nw words (padded to padded) start at word `prefix` of
// the stream's data section: lane states, block word entry, the words, and
// for the buffer's last block the header, pdf and size. Then the slot's
// lines are dropped from L2 without write-back.
template <bool kSlots>
__device__ __forceinline__ void encode_store(uint8_t* __restrict__ out, uint64_t out_cap,
                                             uint64_t n, int p, const uint32_t* __restrict__ pdf,
                                             unsigned long long* out_size64, uint32_t* out_size32,
                                             const Sink& sink, uint32_t b, uint32_t nw,
                                             uint32_t prefix, uint32_t x, const uint16_t* sout,
                                             int lane) {
  const uint64_t nb = div_up_u64(n, kAnsBlock);
  const uint64_t over = ans_overhead(nb);
  const uint32_t bs = (uint32_t)min_u64(kAnsBlock, n - (uint64_t)b * kAnsBlock);
  const uint32_t padded = (nw + 7) & ~7u;
  const uint64_t end = over + 2ull * ((uint64_t)prefix + padded);
  const bool last = (uint64_t)b + 1 == nb;
  if (last && end > out_cap && lane == 0) report(sink, MANS_ERR_OUTPUT_OVERFLOW, end);
  if (end <= out_cap) {
    uint32_t* states = reinterpret_cast<uint32_t*>(out + kAnsHeaderBytes + 2 * kAnsSyms);
    states[(uint64_t)b * 32 + lane] = x;
    uint2* bw = reinterpret_cast<uint2*>(out + kAnsHeaderBytes + 2 * kAnsSyms + 128 * nb);
    if (lane == 0) bw[b] = make_uint2((bs << 16) | nw, prefix);
    uint4* dst = reinterpret_cast<uint4*>(out + over + 2ull * prefix);
    const uint4* src = reinterpret_cast<const uint4*>(sout);
    for (uint32_t i = lane; i < padded / 8; i += 32) {
      if (kSlots) dst[i] = __ldcg(src + i);
      else dst[i] = src[i];
    }
    if (last) {
      if (lane < 8) {
        const uint32_t hv = lane == 0 ? kAnsMagicVersion
                          : lane == 1 ? (uint32_t)nb
                          : lane == 2 ? (uint32_t)n
                          : lane == 3 ? prefix + padded
                          : lane == 4 ? (uint32_t)p : 0u;
        reinterpret_cast<uint32_t*>(out)[lane] = hv;
      }
      for (int i = lane; i < kAnsSyms; i += 32)
        reinterpret_cast<uint16_t*>(out + kAnsHeaderBytes)[i] = (uint16_t)pdf[i];
      if (lane == 0 && (nb & 1)) bw[nb] = make_uint2(0, 0);
      if (lane == 0) {
        if (out_size64) *out_size64 = end;
        if (out_size32) *out_size32 = (uint32_t)end;
      }
    }
  }
  __syncwarp();
  if (kSlots) {
    // the slot's lines are consumed: drop them from L2 without write-back
    const uint32_t lines = (2 * padded + 127) / 128;
    if ((uint32_t)lane < lines) discard_l2_line(reinterpret_cast<const uint8_t*>(sout) + 128 * lane);
    if ((uint32_t)lane + 32 < lines)
      discard_l2_line(reinterpret_cast<const uint8_t*>(sout) + 128 * (lane + 32));
    __syncwarp();
  }
}

// A block whose words wait in their slot for the block's stream offset.
struct EncPending {
  uint32_t b;      // block index (0xffffffff: none)
  uint32_t nw;     // its words
  uint32_t x;      // the lane's final state
  uint16_t* sout;  // its word slot
};

// The second half of a block: the exclusive word prefix from the decoupled
// look-back, the block's inclusive prefix, and the store.
template <bool kSlots>
__device__ __forceinline__ void encode_finish(
    uint8_t* __restrict__ out, uint64_t out_cap, uint64_t n, unsigned long long* out_size64,
    uint32_t* out_size32, const uint32_t* __restrict__ pdf, unsigned long long* flags,
    uint32_t epoch, int p, const Sink& sink, const EncPending& pb, int lane) {
  const uint32_t padded = (pb.nw + 7) & ~7u;
  uint32_t prefix = 0;
  if (pb.b > 0) {
    prefix = lookback_exclusive(flags, pb.b, epoch, sink);
    if (lane == 0) st_flag(&flags[pb.b], make_flag(kFlagIncl, epoch, prefix + padded));
  }
  __syncwarp();
  encode_store<kSlots>(out, out_cap, n, p, pdf, out_size64, out_size32, sink, pb.b, pb.nw, prefix,
                       pb.x, pb.sout, lane);
}

// One block as the unit of the single-pass prefix (flags per block): encode,
// publish the aggregate, look back, store.
template <bool kSlots, typename TabT>
__device__ __forceinline__ void encode_block(
    const uint8_t* __restrict__ in, uint64_t n, uint8_t* __restrict__ out, uint64_t out_cap,
    unsigned long long* out_size64, uint32_t* out_size32, const uint32_t* __restrict__ pdf,
    unsigned long long* flags, uint32_t epoch, int p, const Sink& sink, const TabT* table,
    uint8_t* stage, uint64_t* bar, uint32_t& parity, uint16_t* sout, uint32_t b, int lane) {
  uint32_t x;
  const uint32_t nw =
      encode_words<!kSlots>(in, n, b, table, stage, bar, parity, sout, p, sink, lane, x);
  const uint32_t padded = (nw + 7) & ~7u;
  if (lane == 0) st_flag(&flags[b], make_flag(b == 0 ? kFlagIncl : kFlagAgg, epoch, padded));
  encode_finish<kSlots>(out, out_cap, n, out_size64, out_size32, pdf, flags, epoch, p, sink,
                        EncPending{b, nw, x, sout}, lane);
}

constexpr int kDecWarps = 8;
constexpr int kDecThreads = kDecWarps * 32;
constexpr int kMaxProbBits = 11;

// Build the slot table of a stream's pdf in shared memory (one CTA of 256
// threads, thread t owns symbol t): lut[s] = pdf << 20 | (s - cdf) << 8 |
// symbol (GpuANSDecode.h:307-377 packs the same fields in one word, in
// another order). Returns false when the pdf does not sum to 2^p.
__device__ __forceinline__ bool build_decode_tables(const uint8_t* __restrict__ in, int p,
                                                    uint32_t* lut, uint32_t* s_scan) {
  const int t = threadIdx.x, warp = t >> 5, lane = t & 31;
  const uint16_t* probs = reinterpret_cast<const uint16_t*>(in + kAnsHeaderBytes);
  const uint32_t pdf = __ldg(probs + t);
  uint32_t incl = pdf;
#pragma unroll
  for (int o = 1; o < 32; o <<= 1) {
    const uint32_t v = __shfl_up_sync(0xffffffffu, incl, o);
    if (lane >= o) incl += v;
  }
  __syncthreads();
  if (lane == 31) s_scan[warp] = incl;
  __syncthreads();
  uint32_t base = 0, total = 0;
  for (int w = 0; w < kDecWarps; ++w) {
    if (w < warp) base += s_scan[w];
    total += s_scan[w];
  }
  const uint32_t cdf = base + incl - pdf;
  if (total != (1u << p)) return false;
  for (uint32_t j = 0; j < pdf; ++j) {
    lut[cdf + j] = (pdf << 20) | (j << 8) | (uint32_t)t;
  }
  return true;
}

// ---- decode ----
// Words staged in shared memory per warp (5 KiB): every block whose padded
// word count fits -- all blocks but those of bytes that the coding expands by
// a quarter or more -- decodes from shared memory; a block with more words
// reads its words from global memory instead.
constexpr uint32_t kDecStageWords = 2560;
// Decoded bytes leave through a per-warp 512-byte stage, 16 steps at a time,
// as one 16-byte store per lane.
constexpr int kDecChunkSteps = 16;
constexpr uint32_t kDecChunkBytes = kDecChunkSteps * 32;

struct DecWarpSmem {
  alignas(16) uint16_t words[kDecStageWords];
  alignas(16) uint8_t out[kDecChunkBytes + 16];  // a chunk at its destination's phase
};

__device__ __forceinline__ uint32_t ld_shared_u16(uint32_t addr) {
  uint16_t v;
  asm volatile("ld.shared.u16 %0, [%1];" : "=h"(v) : "r"(addr));
  return v;
}
__device__ __forceinline__ uint32_t ld_shared_u32(uint32_t addr) {
  uint32_t v;
  asm volatile("ld.shared.u32 %0, [%1];" : "=r"(v) : "r"(addr));
  return v;
}

// Store one decoded 512-byte chunk from the warp's stage, where it sits at
// offset ph = g & 15 (the destination's phase), to g: 16-byte stores for the
// whole 16-byte units and byte stores for a partial first and last unit (the
// mapped buffer that a MANS decode writes starts at any phase).
__device__ __forceinline__ void dec_flush_chunk(uint8_t* __restrict__ g, const uint8_t* ostage,
                                                uint32_t ph, int lane) {
  if (ph == 0) {
    reinterpret_cast<uint4*>(g)[lane] = reinterpret_cast<const uint4*>(ostage)[lane];
    return;
  }
  uint8_t* g0 = g - ph;  // 16-byte aligned; stage unit u <-> g0 + 16 u
  if (lane >= 1) reinterpret_cast<uint4*>(g0)[lane] = reinterpret_cast<const uint4*>(ostage)[lane];
  if (lane < 16) {
    if ((uint32_t)lane >= ph) g0[lane] = ostage[lane];                  // unit 0
    else g0[kDecChunkBytes + lane] = ostage[kDecChunkBytes + lane];      // unit 32
  }
}

// The 128 steps of a full block whose words are staged in shared memory, for
// precision kP. State x per lane; wa: shared byte address one past the next
// word to read (words are read backwards, the highest reading lane first,
// GpuANSDecode.h:78-92); lut: shared address of the slot table. Each step:
// slot -> table entry {pdf:12, slot - cdf:12, symbol:8}; x = pdf * (x >> p) +
// (slot - cdf); lanes whose state fell below 2^15 read one word each.
// A corrupt stream can move wa below the warp's words, by at most 128 steps x
// 32 words = 8 KiB; the slot table (8 KiB) lies below every warp's words in
// the CTA's shared memory, so such reads stay inside it, and the final
// position check reports the block. Returns false when the block does not
// end exactly at its first word in the start state.
template <int kP>
__device__ __forceinline__ bool decode_full_smem(uint32_t x, uint32_t wa, uint32_t wa_end,
                                                 uint32_t lut, uint8_t* __restrict__ dst,
                                                 uint8_t* ostage, int lane) {
  constexpr uint32_t kMask = (1u << kP) - 1u;
  const uint32_t ltmask = lanemask_lt();
  const uint32_t ph = phase16(dst);  // dst + 512 c has the same phase
  uint8_t* st = ostage + ph + lane;
#pragma unroll 1
  for (int c = kAnsStepsPerBlock / kDecChunkSteps - 1; c >= 0; --c) {
#pragma unroll
    for (int i = kDecChunkSteps - 1; i >= 0; --i) {
      const uint32_t e = ld_shared_u32(lut + ((x & kMask) << 2));
      st[i * 32] = (uint8_t)e;
      x = (e >> 20) * (x >> kP) + ((e >> 8) & 0xfffu);
      const bool rd = x < kAnsStartState;
      const uint32_t vote = __ballot_sync(0xffffffffu, rd);
      wa -= 2u * __popc(vote);
      if (rd) x = (x << 16) | ld_shared_u16(wa + 2u * __popc(vote & ltmask));
    }
    __syncwarp();
    dec_flush_chunk(dst + kDecChunkBytes * c, ostage, ph, lane);
    __syncwarp();
  }
  return wa == wa_end && x == kAnsStartState;
}

// Any block (partial last block, or words in global memory): the same steps
// with byte stores and a clamped word index. words: the block's first word
// (shared or global); ptr: its word count.
__device__ __forceinline__ bool decode_any(uint32_t x, const uint16_t* words, int ptr, uint32_t bs,
                                           int p, const uint32_t* lut, uint8_t* __restrict__ dst,
                                           int lane) {
  const uint32_t mask = (1u << p) - 1u;
  const uint32_t gemask = lanemask_ge();
  const uint32_t rem = bs & 31;
  int j = (int)((bs + 31) >> 5) - 1;
  for (; j >= 0; --j) {
    const bool valid = rem == 0 || j < (int)(bs >> 5) || (uint32_t)lane < rem;
    if (valid) {
      const uint32_t e = lut[x & mask];
      dst[j * 32 + lane] = (uint8_t)e;
      x = (e >> 20) * (x >> p) + ((e >> 8) & 0xfffu);
    }
    const bool rd = valid && x < kAnsStartState;
    const uint32_t vote = __ballot_sync(0xffffffffu, rd);
    // a read below the block's first word only happens in a corrupt stream;
    // it is clamped here and caught by the final position check
    if (rd) x = x * 65536u + words[max(ptr - __popc(vote & gemask), 0)];
    ptr -= __popc(vote);
  }
  return ptr == 0 && x == kAnsStartState;
}

// Decode block b of one stream (one warp) into out + 4096 b. in: the stream
// (header validated by the caller: nb blocks, n bytes, cw words, precision
// p); lut: the slot table in shared memory (2^11 words, placed below every
// warp's stage); ws / bar / parity: the warp's stage and its mbarrier.
__device__ __forceinline__ void decode_block(const uint8_t* __restrict__ in, uint32_t nb,
                                             uint32_t n, uint32_t cw, int p,
                                             uint8_t* __restrict__ out, const uint32_t* lut,
                                             DecWarpSmem* ws, uint64_t* bar, uint32_t& parity,
                                             const Sink& sink, uint32_t b, int lane) {
  const uint64_t over = ans_overhead(nb);
  const uint32_t* states = reinterpret_cast<const uint32_t*>(in + kAnsHeaderBytes + 2 * kAnsSyms);
  const uint2* bwords = reinterpret_cast<const uint2*>(in + kAnsHeaderBytes + 2 * kAnsSyms + 128ull * nb);
  const uint16_t* data = reinterpret_cast<const uint16_t*>(in + over);
  const uint32_t x = __ldg(states + (uint64_t)b * 32 + lane);
  const uint2 bw = __ldg(bwords + b);
  const uint32_t bs = bw.x >> 16, nw = bw.x & 0xffffu, pre = bw.y;
  const uint32_t expect = (b + 1 == nb) ? n - b * kAnsBlock : kAnsBlock;
  const uint32_t padded = (nw + 7) & ~7u;
  if (bs != expect || (uint64_t)pre + padded > cw || padded > kEncOutWords || (pre & 7)) {
    if (lane == 0) report(sink, MANS_ERR_CORRUPT, b);
    return;
  }
  uint8_t* dst = out + (uint64_t)b * kAnsBlock;
  bool ok;
  if (padded <= kDecStageWords) {
    // stage the block's words with one bulk copy (16-byte aligned: over % 16
    // == 0, pre % 8 == 0); the previous block's reads of the stage are done
    __syncwarp();
    if (padded) {
      if (lane == 0) bulk_load(ws->words, data + pre, 2 * padded, bar);
      if (!mbar_wait(bar, parity) && lane == 0) report(sink, MANS_ERR_TIMEOUT, b);
      parity ^= 1u;
    }
    if (bs == kAnsBlock) {
      const uint32_t w0 = smem_addr(ws->words), l0 = smem_addr(lut);
      switch (p) {
        case 9: ok = decode_full_smem<9>(x, w0 + 2 * nw, w0, l0, dst, ws->out, lane); break;
        case 10: ok = decode_full_smem<10>(x, w0 + 2 * nw, w0, l0, dst, ws->out, lane); break;
        default: ok = decode_full_smem<11>(x, w0 + 2 * nw, w0, l0, dst, ws->out, lane); break;
      }
    } else {
      ok = decode_any(x, ws->words, (int)nw, bs, p, lut, dst, lane);
    }
  } else {
    ok = decode_any(x, data + pre, (int)nw, bs, p, lut, dst, lane);
  }
  if (__any_sync(0xffffffffu, !ok) && lane == 0) report(sink, MANS_ERR_CORRUPT, b);
}

}  // namespace mans
