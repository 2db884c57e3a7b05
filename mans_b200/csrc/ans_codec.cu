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
#include "ans_dev.cuh"
#include "mans_internal.h"

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
// Encode: one warp per 4 KiB block. The block arrives in the warp's shared
// stage with one bulk (TMA) copy from L2, where it was prefetched one grid of
// warps earlier; symbols are read eight steps ahead of use. Blocks are
// claimed one at a time (a claim held while another block is encoded would
// stall every later block's look-back).
// ------------------------------------------------------------------------
// Four CTAs of eight warps per SM (32 warps, 64 registers a thread): with
// five the register cap spills the pending block's state, which costs more
// than the extra warps gain (0.695 vs 0.720 ms on 1 GiB of detector frames).
constexpr int kEncMinCtas = 4;

template <bool kSlots, bool kWide>
__global__ __launch_bounds__(kEncThreads, kEncMinCtas) void ans_encode_kernel(
    const uint8_t* __restrict__ in, uint8_t* __restrict__ out, uint64_t out_cap,
    unsigned long long* out_size64, uint32_t* out_size32, Ctrl* ctrl,
    unsigned long long* flags, int p, uint8_t* __restrict__ slots) {
  extern __shared__ __align__(16) uint8_t smem_raw[];
  EncSmemSlots& ss = *reinterpret_cast<EncSmemSlots*>(smem_raw);  // common prefix of both layouts
  __shared__ int s_last;
  const int t = threadIdx.x, warp = t >> 5, lane = t & 31;
  uint64_t* bar = &ss.bar[warp];
  if (lane == 0) mbar_init(bar);
  uint32_t parity = 0;
  const Sink sink = sink_of(ctrl);
  const bool failed = sink_failed(sink);
  const uint32_t epoch = *((volatile uint32_t*)&ctrl->epoch);
  const uint64_t n = __ldcg(&ctrl->merged_size);
  const uint64_t nb = div_up_u64(n, kAnsBlock);
  const uint64_t over = ans_overhead(nb);
  // Table layout: with a concentrated symbol distribution most lanes of a
  // step look up the same few entries, and the expanded 16-byte entries save
  // integer work; with a flat one the lanes spread over many entries, and
  // the packed 8-byte entries cost fewer shared-memory wavefronts. The
  // effective number of symbols 2^(2p) / sum(pdf^2) decides (<= 16:
  // expanded). Both variants are launched; the one that does not match the
  // table returns at once, before touching any counter. Either layout
  // yields the same bytes.
  __shared__ uint32_t s_sq[kEncWarps];
  {
    const uint32_t q = ctrl->pdf[t];
    const uint32_t sq = __reduce_add_sync(0xffffffffu, q * q);
    if (lane == 0) s_sq[warp] = sq;
  }
  __syncthreads();
  uint64_t tot = 0;
  for (int w = 0; w < kEncWarps; ++w) tot += s_sq[w];
  if ((tot * 16ull >= (1ull << (2 * p))) != kWide) return;
  if (!failed) {
    if constexpr (kWide) ss.table4[t] = expand_enc_entry(ctrl->enc_table[t], p);
    else ss.table2[t] = ctrl->enc_table[t];
  }
  __syncthreads();

  if (!failed && nb == 0 && blockIdx.x == 0 && warp == 0) {
    // Empty input: header and a zero pdf only (GpuANSEncode.h:201-237).
    if (over > out_cap) {
      if (lane == 0) report(sink, MANS_ERR_OUTPUT_OVERFLOW, over);
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

  const uint32_t ahead = gridDim.x * kEncWarps;
  if constexpr (kSlots) {
    // Two word slots per warp. A block's words wait in one slot for its
    // stream offset while the warp encodes its next block into the other;
    // the look-back of the waiting block then runs after that next block's
    // aggregate is published, when its predecessors have usually finished,
    // instead of stalling the warp. Every claimed block publishes its
    // aggregate as soon as it is encoded, before any wait, so the deferred
    // look-backs always complete.
    uint16_t* const slot0 = reinterpret_cast<uint16_t*>(
        slots + ((uint64_t)blockIdx.x * kEncWarps + warp) * 2 * kEncSlotBytes);
    EncPending pend{0xffffffffu, 0, 0, nullptr};
    uint32_t cur = 0;
    while (!failed) {
      const uint32_t b = warp_claim(&ctrl->tile_counter[1], lane);
      if (b >= nb) break;
      if (lane == 0 && (uint64_t)b + ahead < nb) {
        const uint64_t s1 = ((uint64_t)b + ahead) * kAnsBlock;
        prefetch_l2(in + s1, (uint32_t)min_u64(kAnsBlock, n - s1));
      }
      uint16_t* const sout = slot0 + cur * (kEncSlotBytes / 2);
      uint32_t x;
      uint32_t nw;
      if constexpr (kWide)
        nw = encode_words<false>(in, n, b, ss.table4, ss.in[warp], bar, parity, sout, p, sink,
                                 lane, x);
      else
        nw = encode_words<false>(in, n, b, ss.table2, ss.in[warp], bar, parity, sout, p, sink,
                                 lane, x);
      if (lane == 0)
        st_flag(&flags[b], make_flag(b == 0 ? kFlagIncl : kFlagAgg, epoch, (nw + 7) & ~7u));
      if (pend.b != 0xffffffffu)
        encode_finish<true>(out, out_cap, n, out_size64, out_size32, ctrl->pdf, flags, epoch, p,
                            sink, pend, lane);
      pend = EncPending{b, nw, x, sout};
      cur ^= 1u;
    }
    if (pend.b != 0xffffffffu)
      encode_finish<true>(out, out_cap, n, out_size64, out_size32, ctrl->pdf, flags, epoch, p,
                          sink, pend, lane);
  } else {
    uint16_t* sout = reinterpret_cast<EncSmem*>(smem_raw)->out[warp];
    while (!failed) {
      const uint32_t b = warp_claim(&ctrl->tile_counter[1], lane);
      if (b >= nb) break;
      if (lane == 0 && (uint64_t)b + ahead < nb) {
        const uint64_t s1 = ((uint64_t)b + ahead) * kAnsBlock;
        prefetch_l2(in + s1, (uint32_t)min_u64(kAnsBlock, n - s1));
      }
      if constexpr (kWide)
        encode_block<false>(in, n, out, out_cap, out_size64, out_size32, ctrl->pdf, flags, epoch,
                            p, sink, ss.table4, ss.in[warp], bar, parity, sout, b, lane);
      else
        encode_block<false>(in, n, out, out_cap, out_size64, out_size32, ctrl->pdf, flags, epoch,
                            p, sink, ss.table2, ss.in[warp], bar, parity, sout, b, lane);
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
    ctrl->epoch = (epoch + 1) & 0x3fffffffu;  // the call's flags are now stale
  }
}

// ------------------------------------------------------------------------
// Decode: one warp per block, decoded from its last step to its first. The
// block's words are staged in shared memory with one bulk copy (read
// backwards, data-dependently, every step); decoded bytes collect in a
// 512-byte per-warp stage and leave as 16-byte stores every 16 steps. The
// next block is claimed early and its words prefetched into L2 (no
// look-back: claiming ahead costs nothing here).
// ------------------------------------------------------------------------
struct DecSmem {
  uint32_t lut[1 << kMaxProbBits];  // below every warp's stage (see decode_full_smem)
  DecWarpSmem warp[kDecWarps];
  uint64_t bar[kDecWarps];
};
// Four CTAs of eight warps per SM (32 warps): 50 KiB of shared memory each,
// with word stages of 2,560 words, so that blocks of poorly compressible
// bytes (about 2,048 words) also decode from shared memory (5 CTAs with
// 2,048-word stages: 1 GiB of gradient data decoded in 1.30 ms, here 0.59).
constexpr int kDecMinCtas = 4;

__global__ __launch_bounds__(kDecThreads, kDecMinCtas) void ans_decode_kernel(
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
  const Sink sink = sink_of(ctrl);

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
  const bool failed_before = sink_failed(sink);
  if (t == 0) s_ok = ok && !failed_before;
  if (!ok && blockIdx.x == 0 && t == 0 && !failed_before) report(sink, MANS_ERR_BAD_STREAM, 0);
  if (record && ok && blockIdx.x == 0 && t == 0) ctrl->merged_size = n;
  __syncthreads();

  if (s_ok && n > 0) {
    const bool tables_ok = build_decode_tables(in, p, sm.lut, s_scan);
    if (!tables_ok && t == 0) {
      s_ok = 0;
      if (blockIdx.x == 0) report(sink, MANS_ERR_BAD_STREAM, 1);
    }
  }
  __syncthreads();

  if (s_ok && n > 0) {
    const uint64_t over = ans_overhead(nb);
    const uint2* bwords = reinterpret_cast<const uint2*>(in + kAnsHeaderBytes + 2 * kAnsSyms + 128ull * nb);
    uint32_t b = warp_claim(&ctrl->tile_counter[2], lane);
    while (b < nb) {
      const uint32_t nxt = warp_claim(&ctrl->tile_counter[2], lane);
      if (nxt < nb && lane == 0) {
        const uint2 bn = __ldg(bwords + nxt);
        const uint32_t wn = ((bn.x & 0xffffu) + 7) & ~7u;
        if ((uint64_t)bn.y + wn <= cw) prefetch_l2(in + over + 2ull * bn.y, 2 * wn);
      }
      decode_block(in, nb, n, cw, p, out, sm.lut, &sm.warp[warp], bar, parity, sink, b, lane);
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
  cudaFuncSetAttribute(ans_encode_kernel<false, false>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                       (int)sizeof(EncSmem));
  cudaFuncSetAttribute(ans_encode_kernel<false, true>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                       (int)sizeof(EncSmem));
  cudaFuncSetAttribute(ans_decode_kernel, cudaFuncAttributeMaxDynamicSharedMemorySize,
                       (int)sizeof(DecSmem));
  cfg.enc_ctas = max(occupancy((const void*)ans_encode_kernel<false, false>, kEncThreads, sizeof(EncSmem)),
                     occupancy((const void*)ans_encode_kernel<false, true>, kEncThreads, sizeof(EncSmem)));
  cudaFuncSetAttribute(ans_encode_kernel<true, false>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                       (int)sizeof(EncSmemSlots));
  cudaFuncSetAttribute(ans_encode_kernel<true, true>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                       (int)sizeof(EncSmemSlots));
  cfg.enc_slot_ctas = max(occupancy((const void*)ans_encode_kernel<true, false>, kEncThreads,
                                    sizeof(EncSmemSlots)),
                          occupancy((const void*)ans_encode_kernel<true, true>, kEncThreads,
                                    sizeof(EncSmemSlots)));
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
  return (uint64_t)cfg.sms * cfg.enc_slot_ctas * kEncWarps * 2 * kEncSlotBytes;  // two per warp
}

cudaError_t launch_ans_encode(const uint8_t* in, uint8_t* out, uint64_t out_cap,
                              unsigned long long* out_size64, uint32_t* out_size32, Ctrl* ctrl,
                              unsigned long long* flags, int prob_bits, uint64_t max_blocks,
                              const LaunchCfg& cfg, cudaStream_t s, uint8_t* slots) {
  // Both table-layout variants are launched; each decides from the pdf on
  // the device and the one that does not match returns at once.
  const uint64_t want = div_up_u64(max_blocks, kEncWarps);
  if (slots) {
    const uint64_t cap = (uint64_t)cfg.sms * cfg.enc_slot_ctas;
    const unsigned grid = (unsigned)(want < 1 ? 1 : (want < cap ? want : cap));
    ans_encode_kernel<true, false><<<grid, kEncThreads, sizeof(EncSmemSlots), s>>>(
        in, out, out_cap, out_size64, out_size32, ctrl, flags, prob_bits, slots);
    ans_encode_kernel<true, true><<<grid, kEncThreads, sizeof(EncSmemSlots), s>>>(
        in, out, out_cap, out_size64, out_size32, ctrl, flags, prob_bits, slots);
  } else {
    const uint64_t cap = (uint64_t)cfg.sms * cfg.enc_ctas;
    const unsigned grid = (unsigned)(want < 1 ? 1 : (want < cap ? want : cap));
    ans_encode_kernel<false, false><<<grid, kEncThreads, sizeof(EncSmem), s>>>(
        in, out, out_cap, out_size64, out_size32, ctrl, flags, prob_bits, nullptr);
    ans_encode_kernel<false, true><<<grid, kEncThreads, sizeof(EncSmem), s>>>(
        in, out, out_cap, out_size64, out_size32, ctrl, flags, prob_bits, nullptr);
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
