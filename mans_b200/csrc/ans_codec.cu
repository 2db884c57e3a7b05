// ans_codec.cu -- byte rANS over 4 KiB blocks for sm_100a: histogram,
// encode (with single-pass output compaction) and decode.
//
// Stream layout and arithmetic are those of include/ans (GpuANSCodec.h,
// GpuANSEncode.h, GpuANSDecode.h); the kernels are organised differently:
//  * encode writes the final coalesced stream directly: each warp stages its
//    block's words in shared memory, learns its word offset through a
//    decoupled look-back over per-block flags, and stores 16-byte vectors.
//    The reference instead writes an uncoalesced scratch (5,248-byte stride),
//    scans with up to three kernels and copies with a fourth.
//  * the table is normalised by the last CTA of the histogram kernel, not by
//    a separate launch;
//  * decode validates the header on the device and reports a status instead
//    of device asserts, and checks that every block consumes exactly its
//    words and returns to the start state.
#include "ans_table.cuh"
#include "mans_internal.h"
#include "smem_io.cuh"

namespace mans {

// ------------------------------------------------------------------------
// Histogram of a raw byte buffer (GpuANSStatistics.h:24-151), with per-warp
// shared-memory bins merged into the global histogram once per CTA.
// ------------------------------------------------------------------------
constexpr int kHistThreads = 256;

__device__ __forceinline__ void hist_word(uint32_t* h, uint32_t w) {
  atomicAdd(&h[w & 0xff], 1u);
  atomicAdd(&h[(w >> 8) & 0xff], 1u);
  atomicAdd(&h[(w >> 16) & 0xff], 1u);
  atomicAdd(&h[w >> 24], 1u);
}

__global__ __launch_bounds__(kHistThreads) void hist_bytes_kernel(const uint8_t* __restrict__ in,
                                                                  uint64_t n, Ctrl* ctrl,
                                                                  int prob_bits) {
  __shared__ uint32_t s_h[kHistThreads / 32][kAnsSyms];
  const int t = threadIdx.x, warp = t >> 5;
  for (int i = t; i < (kHistThreads / 32) * kAnsSyms; i += kHistThreads) (&s_h[0][0])[i] = 0;
  __syncthreads();
  uint32_t* h = s_h[warp];
  const uint64_t n16 = n >> 4;
  const uint4* in4 = reinterpret_cast<const uint4*>(in);
  for (uint64_t i = (uint64_t)blockIdx.x * kHistThreads + t; i < n16;
       i += (uint64_t)gridDim.x * kHistThreads) {
    uint4 v = __ldcs(in4 + i);
    hist_word(h, v.x);
    hist_word(h, v.y);
    hist_word(h, v.z);
    hist_word(h, v.w);
  }
  if (blockIdx.x == 0) {
    uint64_t i = (n16 << 4) + t;
    if (i < n) atomicAdd(&h[in[i]], 1u);
  }
  hist_merge_and_normalize(s_h, kHistThreads / 32, ctrl, n, 0, prob_bits);
}

// ------------------------------------------------------------------------
// Encode (GpuANSEncode.h:25-164 arithmetic, :181-284 layout).
//
// One warp encodes one 4 KiB block: lane l codes bytes l, l+32, ... The
// block arrives in the warp's shared stage with one bulk (TMA) copy from L2,
// where it was prefetched one grid of warps earlier; symbols are read eight
// steps ahead of use. Output words are compacted in a per-warp shared buffer (the
// only shared staging), then stored as 16-byte vectors once the block's word
// offset is known.
// ------------------------------------------------------------------------
constexpr int kEncWarps = 8;
constexpr int kEncThreads = kEncWarps * 32;
constexpr uint32_t kEncOutWords = kAnsMaxBlockWords + 8;
// A block's words compacted in global memory: slots of whole 128-byte lines.
constexpr uint32_t kEncSlotBytes = (kEncOutWords * 2 + 127) / 128 * 128;

constexpr uint32_t kEncStageBytes = kAnsBlock + 16;  // a block plus its 16-byte phase

struct EncSmemSlots {  // words go to global slots
  uint2 table[kAnsSyms];
  alignas(16) uint8_t in[kEncWarps][kEncStageBytes];
  uint64_t bar[kEncWarps];
};
struct EncSmem {  // words compacted in shared memory
  uint2 table[kAnsSyms];
  alignas(16) uint8_t in[kEncWarps][kEncStageBytes];
  uint64_t bar[kEncWarps];
  alignas(16) uint16_t out[kEncWarps][kEncOutWords];
};

// One interleaved step: renormalise (emit 16 bits, lanes in ascending order
// into the compacted word buffer), then x = (x/pdf << p) + x%pdf + cdf.
__device__ __forceinline__ void enc_step(bool valid, uint32_t& x, uint32_t sym,
                                         const uint2* __restrict__ tab, uint16_t* __restrict__ out,
                                         uint32_t& nw, uint32_t mp, uint32_t sh, uint32_t ltmask) {
  const uint2 e = tab[sym];
  const uint32_t cmpl = (e.y >> 13) & 0xfffu;
  const uint32_t thr = (mp - cmpl) << sh;
  const bool wr = valid && x >= thr;
  const uint32_t vote = __ballot_sync(0xffffffffu, wr);
  if (wr) out[nw + __popc(vote & ltmask)] = (uint16_t)(x & 0xffffu);
  nw += __popc(vote);
  const uint32_t xr = wr ? (x >> 16) : x;
  if (valid) {
    const uint32_t q = __umulhi(xr, e.x) >> (e.y >> 25);
    x = xr + (e.y & 0x1fffu) + q * cmpl;
  } else {
    x = xr;
  }
}

__device__ __forceinline__ uint32_t claim(uint32_t* counter, int lane) {
  uint32_t b = 0;
  if (lane == 0) b = atomicAdd(counter, 1u);
  return __shfl_sync(0xffffffffu, b, 0);
}

__device__ __forceinline__ void discard_l2_line(const void* p) {
  asm volatile("discard.global.L2 [%0], 128;" ::"l"(p) : "memory");
}

// kSlots: the block's words are compacted in a per-warp slot of `slots`
// (global memory, stays in L2 and is discarded after the final copy), so
// shared memory holds only the coding table. Otherwise they are compacted in
// shared memory.
template <bool kSlots>
__global__ __launch_bounds__(kEncThreads) void ans_encode_kernel(
    const uint8_t* __restrict__ in, uint8_t* __restrict__ out, uint64_t out_cap,
    unsigned long long* out_size64, uint32_t* out_size32, Ctrl* ctrl,
    unsigned long long* flags, uint32_t epoch, int p, uint8_t* __restrict__ slots) {
  extern __shared__ __align__(16) uint8_t smem_raw[];
  EncSmemSlots& ss = *reinterpret_cast<EncSmemSlots*>(smem_raw);  // common prefix of both layouts
  uint2* table = ss.table;
  __shared__ int s_last;
  const int t = threadIdx.x, warp = t >> 5, lane = t & 31;
  const uint32_t ltmask = lanemask_lt();
  const uint32_t mp = 1u << p, sh = kAnsStateBits - p;
  uint8_t* stage = ss.in[warp];
  uint64_t* bar = &ss.bar[warp];
  if (lane == 0) mbar_init(bar);
  uint32_t parity = 0;

  const bool failed = *((volatile uint32_t*)&ctrl->status) != 0;
  const uint64_t n = __ldcg(&ctrl->merged_size);
  const uint64_t nb = div_up_u64(n, kAnsBlock);
  const uint64_t over = ans_overhead(nb);

  if (!failed) {
    for (int i = t; i < kAnsSyms; i += kEncThreads) table[i] = ctrl->enc_table[i];
  }
  __syncthreads();

  if (!failed && nb == 0 && blockIdx.x == 0 && warp == 0) {
    // Empty input: header and a zero pdf only (GpuANSEncode.h:201-237).
    if (over > out_cap) {
      if (lane == 0) report_error(ctrl, MANS_ERR_OUTPUT_OVERFLOW, over);
    } else {
      if (lane < 8) {
        const uint32_t hv = lane == 0 ? kAnsMagicVersion : (lane == 4 ? (uint32_t)p : 0u);
        reinterpret_cast<uint32_t*>(out)[lane] = hv;
      }
      for (int i = lane; i < kAnsSyms; i += 32)
        reinterpret_cast<uint16_t*>(out + kAnsHeaderBytes)[i] = (uint16_t)ctrl->pdf[i];
      if (lane == 0) {
        if (out_size64) *out_size64 = over;
        if (out_size32) *out_size32 = (uint32_t)over;
      }
    }
  }

  uint16_t* sout;
  if constexpr (kSlots) {
    sout = reinterpret_cast<uint16_t*>(slots + ((uint64_t)blockIdx.x * kEncWarps + warp) * kEncSlotBytes);
  } else {
    sout = reinterpret_cast<EncSmem*>(smem_raw)->out[warp];
  }
  // Blocks are claimed one at a time (a claim held while another block is
  // encoded would stall every later block's look-back); the block one grid
  // of warps ahead is prefetched into L2 for whichever warp claims it.
  const uint32_t ahead = gridDim.x * kEncWarps;
  while (!failed) {
    const uint32_t b = claim(&ctrl->tile_counter[1], lane);
    if (b >= nb) break;
    if (lane == 0 && (uint64_t)b + ahead < nb) {
      const uint64_t s1 = ((uint64_t)b + ahead) * kAnsBlock;
      prefetch_l2(in + s1, (uint32_t)min_u64(kAnsBlock, n - s1));
    }
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
    if (!mbar_wait(bar, parity) && lane == 0) report_error(ctrl, MANS_ERR_TIMEOUT, b);
    parity ^= 1u;
    const uint8_t* syms = stage + phase16(in + start) + lane;

    uint32_t x = kAnsStartState, nw = 0;
    const uint32_t full = bs >> 5;
    uint32_t j = 0;
    if (full >= 8) {
      uint32_t cur[8];
#pragma unroll
      for (int u = 0; u < 8; ++u) cur[u] = syms[u * 32];
      for (; j + 16 <= full; j += 8) {
        uint32_t nx[8];
#pragma unroll
        for (int u = 0; u < 8; ++u) nx[u] = syms[(j + 8 + u) * 32];
#pragma unroll
        for (int u = 0; u < 8; ++u) enc_step(true, x, cur[u], table, sout, nw, mp, sh, ltmask);
#pragma unroll
        for (int u = 0; u < 8; ++u) cur[u] = nx[u];
      }
#pragma unroll
      for (int u = 0; u < 8; ++u) enc_step(true, x, cur[u], table, sout, nw, mp, sh, ltmask);
      j += 8;
    }
    for (; j < full; ++j) enc_step(true, x, syms[j * 32], table, sout, nw, mp, sh, ltmask);
    if (bs & 31) {
      const bool valid = (uint32_t)lane < (bs & 31);
      enc_step(valid, x, valid ? syms[j * 32] : 0u, table, sout, nw, mp, sh, ltmask);
    }

    // Pad the word count to a 16-byte multiple with zeros (GpuANSEncode.h:275).
    const uint32_t padded = (nw + 7) & ~7u;
    if ((uint32_t)lane < padded - nw) sout[nw + lane] = 0;

    // Single-pass prefix over padded word counts.
    if (lane == 0) st_flag(&flags[b], make_flag(b == 0 ? kFlagIncl : kFlagAgg, epoch, padded));
    uint32_t prefix = 0;
    if (b > 0) {
      prefix = lookback_exclusive(flags, b, epoch, ctrl);
      if (lane == 0) st_flag(&flags[b], make_flag(kFlagIncl, epoch, prefix + padded));
    }
    __syncwarp();

    const uint64_t end = over + 2ull * ((uint64_t)prefix + padded);
    const bool last = (uint64_t)b + 1 == nb;
    if (last && end > out_cap && lane == 0) report_error(ctrl, MANS_ERR_OUTPUT_OVERFLOW, end);
    if (end <= out_cap) {
      uint32_t* states = reinterpret_cast<uint32_t*>(out + kAnsHeaderBytes + 2 * kAnsSyms);
      states[(uint64_t)b * 32 + lane] = x;
      uint2* bw = reinterpret_cast<uint2*>(out + kAnsHeaderBytes + 2 * kAnsSyms + 128 * nb);
      if (lane == 0) bw[b] = make_uint2((bs << 16) | nw, prefix);
      uint4* dst = reinterpret_cast<uint4*>(out + over + 2ull * prefix);
      const uint4* src = reinterpret_cast<const uint4*>(sout);
      for (uint32_t i = lane; i < padded / 8; i += 32) {
        if constexpr (kSlots) dst[i] = __ldcg(src + i);
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
          reinterpret_cast<uint16_t*>(out + kAnsHeaderBytes)[i] = (uint16_t)ctrl->pdf[i];
        if (lane == 0 && (nb & 1)) bw[nb] = make_uint2(0, 0);
        if (lane == 0) {
          if (out_size64) *out_size64 = end;
          if (out_size32) *out_size32 = (uint32_t)end;
        }
      }
    }
    __syncwarp();
    if constexpr (kSlots) {
      // the slot's lines are consumed: drop them from L2 without write-back
      const uint32_t lines = (2 * padded + 127) / 128;
      if ((uint32_t)lane < lines) discard_l2_line(reinterpret_cast<const uint8_t*>(sout) + 128 * lane);
      if ((uint32_t)lane + 32 < lines)
        discard_l2_line(reinterpret_cast<const uint8_t*>(sout) + 128 * (lane + 32));
      __syncwarp();
    }
  }

  __syncthreads();
  if (t == 0) {
    __threadfence();
    s_last = atomicAdd(&ctrl->done_counter[1], 1u) == gridDim.x - 1;
  }
  __syncthreads();
  if (s_last && t == 0) {
    ctrl->tile_counter[1] = 0;
    ctrl->done_counter[1] = 0;
  }
}

// ------------------------------------------------------------------------
// Decode (GpuANSDecode.h:27-302; lookup table :307-377).
//
// One warp decodes one block from its last step to its first. The block's
// words are staged in shared memory (read backwards, data-dependently, every
// step); decoded bytes go straight to global memory, 32 consecutive bytes per
// step. The next block is claimed early and its words prefetched into L2.
// ------------------------------------------------------------------------
constexpr int kDecWarps = 8;
constexpr int kDecThreads = kDecWarps * 32;
constexpr int kMaxProbBits = 11;

// Decode table per slot s = state & (2^p - 1): pdf << 16 | (s - cdf) and the
// symbol (GpuANSDecode.h:27-34 packs the same three fields in one word).
struct DecSmem {
  uint32_t lut[1 << kMaxProbBits];
  uint8_t sym[1 << kMaxProbBits];
  alignas(16) uint16_t in[kDecWarps][kEncOutWords];
  uint64_t bar[kDecWarps];
};

__global__ __launch_bounds__(kDecThreads) void ans_decode_kernel(
    const uint8_t* __restrict__ in, uint64_t in_size, uint8_t* __restrict__ out, uint64_t out_cap,
    Ctrl* ctrl, int expect_p, int record) {
  extern __shared__ __align__(16) uint8_t smem_raw[];
  DecSmem& sm = *reinterpret_cast<DecSmem*>(smem_raw);
  __shared__ uint32_t s_scan[kDecWarps];
  __shared__ int s_ok, s_last;
  const int t = threadIdx.x, warp = t >> 5, lane = t & 31;
  uint64_t* bar = &sm.bar[warp];
  if (lane == 0) mbar_init(bar);
  uint32_t parity = 0;

  // ---- header validation (GpuANSCodec.h:106-113 asserts, GpuANSDecode.h:220-227)
  uint32_t h[5] = {0, 0, 0, 0, 0};
  bool ok = in_size >= kAnsHeaderBytes + 2 * kAnsSyms;
  if (ok) {
#pragma unroll
    for (int i = 0; i < 5; ++i) h[i] = __ldg(reinterpret_cast<const uint32_t*>(in) + i);
  }
  const uint32_t nb = h[1], n = h[2], cw = h[3];
  const int p = (int)(h[4] & 0xfu);
  ok = ok && h[0] == kAnsMagicVersion && p >= 9 && p <= kMaxProbBits &&
       (expect_p < 0 || p == expect_p) && (uint64_t)nb == div_up_u64(n, kAnsBlock) &&
       ans_overhead(nb) + 2ull * cw <= in_size && (uint64_t)n <= out_cap;
  const bool failed_before = *((volatile uint32_t*)&ctrl->status) != 0;
  if (t == 0) s_ok = ok && !failed_before;
  if (!ok && blockIdx.x == 0 && t == 0 && !failed_before)
    report_error(ctrl, MANS_ERR_BAD_STREAM, 0);
  if (record && ok && blockIdx.x == 0 && t == 0) ctrl->merged_size = n;
  __syncthreads();

  if (s_ok && n > 0) {
    // ---- slot -> (cdf_in_bucket, pdf, symbol) table; thread t owns symbol t
    const uint16_t* probs = reinterpret_cast<const uint16_t*>(in + kAnsHeaderBytes);
    const uint32_t pdf = __ldg(probs + t);
    uint32_t incl = pdf;
#pragma unroll
    for (int o = 1; o < 32; o <<= 1) {
      const uint32_t v = __shfl_up_sync(0xffffffffu, incl, o);
      if (lane >= o) incl += v;
    }
    if (lane == 31) s_scan[warp] = incl;
    __syncthreads();
    uint32_t base = 0, total = 0;
    for (int w = 0; w < kDecWarps; ++w) {
      if (w < warp) base += s_scan[w];
      total += s_scan[w];
    }
    const uint32_t cdf = base + incl - pdf;
    if (total != (1u << p)) {
      if (t == 0) {
        s_ok = 0;
        if (blockIdx.x == 0) report_error(ctrl, MANS_ERR_BAD_STREAM, 1);
      }
    } else {
      for (uint32_t j = 0; j < pdf; ++j) {
        sm.lut[cdf + j] = (pdf << 16) | j;
        sm.sym[cdf + j] = (uint8_t)t;
      }
    }
  }
  __syncthreads();

  if (s_ok && n > 0) {
    const uint64_t over = ans_overhead(nb);
    const uint32_t* states = reinterpret_cast<const uint32_t*>(in + kAnsHeaderBytes + 2 * kAnsSyms);
    const uint2* bwords = reinterpret_cast<const uint2*>(in + kAnsHeaderBytes + 2 * kAnsSyms + 128ull * nb);
    const uint8_t* data = in + over;
    const uint32_t mask = (1u << p) - 1u;
    const uint32_t gemask = lanemask_ge();
    uint16_t* sin = sm.in[warp];
    uint32_t b = claim(&ctrl->tile_counter[2], lane);
    while (b < nb) {
      const uint32_t nxt = claim(&ctrl->tile_counter[2], lane);
      uint32_t x = __ldg(states + (uint64_t)b * 32 + lane);
      const uint2 bw = __ldg(bwords + b);
      if (nxt < nb && lane == 0) {
        const uint2 bn = __ldg(bwords + nxt);
        const uint32_t wn = ((bn.x & 0xffffu) + 7) & ~7u;
        if ((uint64_t)bn.y + wn <= cw) prefetch_l2(data + 2ull * bn.y, 2 * wn);
      }
      const uint32_t bs = bw.x >> 16, nw = bw.x & 0xffffu, pre = bw.y;
      const uint32_t expect = (b + 1 == nb) ? n - b * kAnsBlock : kAnsBlock;
      const uint32_t padded = (nw + 7) & ~7u;
      if (bs != expect || (uint64_t)pre + padded > cw || padded > kEncOutWords || (pre & 7)) {
        if (lane == 0) report_error(ctrl, MANS_ERR_CORRUPT, b);
        b = nxt;
        continue;
      }
      // stage the block's words with one bulk copy (16-byte aligned: over % 16
      // == 0, pre % 8 == 0); the previous block's reads of the stage are done
      __syncwarp();
      if (padded) {
        if (lane == 0) bulk_load(sin, data + 2ull * pre, 2 * padded, bar);
        if (!mbar_wait(bar, parity) && lane == 0) report_error(ctrl, MANS_ERR_TIMEOUT, b);
        parity ^= 1u;
      }
      uint8_t* dst = out + (uint64_t)b * kAnsBlock + lane;
      int ptr = (int)nw;
      bool bad;
      const uint32_t rem = bs & 31;
      int j = (int)((bs + 31) >> 5) - 1;
      if (rem) {
        const bool valid = (uint32_t)lane < rem;
        if (valid) {
          const uint32_t s0 = x & mask;
          const uint32_t e = sm.lut[s0];
          dst[j * 32] = sm.sym[s0];
          x = (e >> 16) * (x >> p) + (e & 0xffffu);
        }
        const bool rd = valid && x < kAnsStartState;
        const uint32_t vote = __ballot_sync(0xffffffffu, rd);
        if (rd) x = x * 65536u + sin[max(ptr - __popc(vote & gemask), 0)];
        ptr -= __popc(vote);
        --j;
      }
#pragma unroll 4
      for (; j >= 0; --j) {
        const uint32_t s0 = x & mask;
        const uint32_t e = sm.lut[s0];
        dst[j * 32] = sm.sym[s0];
        x = (e >> 16) * (x >> p) + (e & 0xffffu);
        const bool rd = x < kAnsStartState;
        const uint32_t vote = __ballot_sync(0xffffffffu, rd);
        // A read below the block's first word only happens in a corrupt
        // stream; it is clamped here and caught by the final ptr check.
        if (rd) x = x * 65536u + sin[max(ptr - __popc(vote & gemask), 0)];
        ptr -= __popc(vote);
      }
      bad = ptr != 0 || x != kAnsStartState;
      if (__any_sync(0xffffffffu, bad) && lane == 0) report_error(ctrl, MANS_ERR_CORRUPT, b);
      b = nxt;
    }
  }

  __syncthreads();
  if (t == 0) {
    __threadfence();
    s_last = atomicAdd(&ctrl->done_counter[2], 1u) == gridDim.x - 1;
  }
  __syncthreads();
  if (s_last && t == 0) {
    ctrl->tile_counter[2] = 0;
    ctrl->done_counter[2] = 0;
  }
}

// ------------------------------------------------------------------------
// Host launchers
// ------------------------------------------------------------------------
static int occupancy(const void* fn, int threads, size_t smem) {
  int n = 0;
  if (cudaOccupancyMaxActiveBlocksPerMultiprocessor(&n, fn, threads, smem) != cudaSuccess) n = 1;
  return n > 0 ? n : 1;
}

void init_ans_launch_cfg(LaunchCfg& cfg) {
  cudaFuncSetAttribute(ans_encode_kernel<false>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                       (int)sizeof(EncSmem));
  cudaFuncSetAttribute(ans_decode_kernel, cudaFuncAttributeMaxDynamicSharedMemorySize,
                       (int)sizeof(DecSmem));
  cfg.enc_ctas = occupancy((const void*)ans_encode_kernel<false>, kEncThreads, sizeof(EncSmem));
  cudaFuncSetAttribute(ans_encode_kernel<true>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                       (int)sizeof(EncSmemSlots));
  cfg.enc_slot_ctas = occupancy((const void*)ans_encode_kernel<true>, kEncThreads,
                                sizeof(EncSmemSlots));
  cfg.dec_ctas = occupancy((const void*)ans_decode_kernel, kDecThreads, sizeof(DecSmem));
  cfg.hist_ctas = occupancy((const void*)hist_bytes_kernel, kHistThreads, 0);
}

cudaError_t launch_hist_bytes(const uint8_t* in, uint64_t n, Ctrl* ctrl, int prob_bits,
                              const LaunchCfg& cfg, cudaStream_t s) {
  uint64_t want = div_up_u64(n >> 4, kHistThreads);
  uint64_t cap = (uint64_t)cfg.sms * cfg.hist_ctas;
  unsigned grid = (unsigned)(want < 1 ? 1 : (want < cap ? want : cap));
  hist_bytes_kernel<<<grid, kHistThreads, 0, s>>>(in, n, ctrl, prob_bits);
  return cudaGetLastError();
}

uint64_t ans_encode_slot_bytes(const LaunchCfg& cfg) {
  return (uint64_t)cfg.sms * cfg.enc_slot_ctas * kEncWarps * kEncSlotBytes;
}

cudaError_t launch_ans_encode(const uint8_t* in, uint8_t* out, uint64_t out_cap,
                              unsigned long long* out_size64, uint32_t* out_size32, Ctrl* ctrl,
                              unsigned long long* flags, uint32_t epoch, int prob_bits,
                              uint64_t max_blocks, const LaunchCfg& cfg, cudaStream_t s,
                              uint8_t* slots) {
  const uint64_t want = div_up_u64(max_blocks, kEncWarps);
  if (slots) {
    const uint64_t cap = (uint64_t)cfg.sms * cfg.enc_slot_ctas;
    const unsigned grid = (unsigned)(want < 1 ? 1 : (want < cap ? want : cap));
    ans_encode_kernel<true><<<grid, kEncThreads, sizeof(EncSmemSlots), s>>>(
        in, out, out_cap, out_size64, out_size32, ctrl, flags, epoch, prob_bits, slots);
  } else {
    const uint64_t cap = (uint64_t)cfg.sms * cfg.enc_ctas;
    const unsigned grid = (unsigned)(want < 1 ? 1 : (want < cap ? want : cap));
    ans_encode_kernel<false><<<grid, kEncThreads, sizeof(EncSmem), s>>>(
        in, out, out_cap, out_size64, out_size32, ctrl, flags, epoch, prob_bits, nullptr);
  }
  return cudaGetLastError();
}

cudaError_t launch_ans_decode(const uint8_t* in, uint64_t in_size, uint8_t* out, uint64_t out_cap,
                              Ctrl* ctrl, int expect_p, int record, uint64_t max_blocks,
                              const LaunchCfg& cfg, cudaStream_t s) {
  uint64_t want = div_up_u64(max_blocks, kDecWarps);
  uint64_t cap = (uint64_t)cfg.sms * cfg.dec_ctas;
  unsigned grid = (unsigned)(want < 1 ? 1 : (want < cap ? want : cap));
  ans_decode_kernel<<<grid, kDecThreads, sizeof(DecSmem), s>>>(in, in_size, out, out_cap, ctrl,
                                                                expect_p, record);
  return cudaGetLastError();
}

}  // namespace mans
