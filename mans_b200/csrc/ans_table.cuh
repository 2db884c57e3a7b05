// ans_table.cuh -- probability normalisation and coding tables (device side).
#pragma once

#include "mans_device.cuh"

namespace mans {

// Encoder table entry for one symbol:
//   x = rcp   : ceil(2^(31+l) / pdf) with l = ceil(log2 pdf) (0xffffffff for pdf 1)
//   y = shift | bias << 5 | cmpl << 20
//       bias  = cdf (cdf + 2^p - 1 for pdf 1), cmpl = 2^p - pdf, shift = l - 1
//       (shift in the low five bits: a wrapping funnel shift applies it as
//       it stands)
// so that for a state x < 2^31:
//   q  = umulhi(x, rcp) >> shift          == x / pdf        (exact, below)
//   x' = x + bias + q * cmpl              == (x/pdf << p) + x%pdf + cdf
// The quotient is the Granlund-Montgomery round-up method for 31-bit
// numerators (Granlund & Montgomery, PLDI 1994, Thm 4.2: m*d - 2^(31+l) <= 2^l
// holds for m = ceil(2^(31+l)/d)); the pdf == 1 case uses rcp = 2^32-1 and a
// bias that absorbs the off-by-one (q = x - 1). Only the resulting state
// enters the stream, so any exact division gives the reference's bytes
// (include/ans/GpuANSEncode.h:54-69 uses a different exact reciprocal).
__host__ __device__ inline uint2 make_enc_entry(uint32_t pdf, uint32_t cdf, int p) {
  uint32_t cmpl = (1u << p) - pdf;
  if (pdf <= 1) {
    // pdf == 0 (absent symbol) is never encoded; keep a harmless entry.
    uint32_t bias = cdf + (1u << p) - 1;
    return make_uint2(0xffffffffu, 0u | (bias << 5) | ((cmpl & 0xfffu) << 20));
  }
  uint32_t l = 0;
  while ((1u << l) < pdf) ++l;
  uint64_t rcp = ((1ull << (31 + l)) + pdf - 1) / pdf;
  return make_uint2((uint32_t)rcp, (l - 1) | (cdf << 5) | (cmpl << 20));
}

// Probability normalisation of one histogram, executed by one CTA of exactly
// 256 threads (thread t owns symbol t). Restates
// include/ans/GpuANSStatistics.h:187-385 step for step:
//  1. q = (u32)((float)2^p * ((float)count / (float)total)) with IEEE single
//     precision round-to-nearest division and multiply, truncated (:225);
//     q = 1 when the symbol is present and q == 0 (:228).
//  2. rank symbols by the unique key (q << 16 | symbol), descending
//     (cub::BlockRadixSort in the reference, :239-262; here each thread counts
//     the keys above its own, which yields the same permutation).
//  3. diff = 2^p - sum(q). diff > 0: add 1 to every symbol whose id is below
//     min(diff, 256), repeatedly (:268-283). diff < 0: count entries with
//     q > 1, subtract 1 from the ranks [count - min(-diff, count), count),
//     repeatedly (:284-326).
//  4. cdf = exclusive prefix sum over symbol ids (:347-352).
// Writes pdf[256] and the encoder table enc[256]. total == 0 gives all zeros.
__device__ inline void normalize_cta(const uint32_t* __restrict__ hist, uint32_t total, int p,
                                     uint32_t* __restrict__ pdf_out, uint2* __restrict__ enc_out) {
  __shared__ uint32_t s_key[kAnsSyms];
  __shared__ uint32_t s_q[kAnsSyms];
  __shared__ int s_order[kAnsSyms];
  __shared__ int s_red[8];
  const int t = threadIdx.x;
  const int lane = t & 31, warp = t >> 5;

  uint32_t count = hist[t];
  uint32_t q = 0;
  if (total > 0) {
    float ratio = __fdiv_rn(__uint2float_rn(count), __uint2float_rn(total));
    float scaled = __fmul_rn(__uint2float_rn(1u << p), ratio);
    q = __float2uint_rz(scaled);
    if (count > 0 && q == 0) q = 1;
  }
  // block sum of q
  int v = __reduce_add_sync(0xffffffffu, (int)q);
  if (lane == 0) s_red[warp] = v;
  s_key[t] = (q << 16) | (uint32_t)t;
  __syncthreads();
  int sum = 0;
#pragma unroll
  for (int w = 0; w < 8; ++w) sum += s_red[w];
  uint32_t key = (q << 16) | (uint32_t)t;
  int rank = 0;
  for (int u = 0; u < kAnsSyms; ++u) rank += s_key[u] > key;
  s_order[rank] = t;
  s_q[t] = q;
  __syncthreads();

  int diff = (int)(1u << p) - sum;
  if (total > 0 && diff > 0) {
    while (diff > 0) {
      int it = diff < kAnsSyms ? diff : kAnsSyms;
      if (t < it) s_q[t] += 1;
      diff -= it;
    }
    __syncthreads();
  } else if (total > 0 && diff < 0) {
    diff = -diff;
    // thread t now owns rank t
    int sym = s_order[t];
    uint32_t qr = s_q[sym];
    while (diff > 0) {
      __syncthreads();
      int gt = __reduce_add_sync(0xffffffffu, (int)(qr > 1));
      if (lane == 0) s_red[warp] = gt;
      __syncthreads();
      int gt1 = 0;
#pragma unroll
      for (int w = 0; w < 8; ++w) gt1 += s_red[w];
      if (gt1 == 0) break;  // unreachable: 2^p >= 512 exceeds the 256 symbols
      int it = diff < gt1 ? diff : gt1;
      int start = gt1 - it;
      if (t >= start && t < gt1) qr -= 1;
      diff -= it;
    }
    s_q[sym] = qr;
    __syncthreads();
  }
  uint32_t pdf = s_q[t];
  // exclusive scan over symbol ids
  uint32_t incl = pdf;
#pragma unroll
  for (int o = 1; o < 32; o <<= 1) {
    uint32_t n = __shfl_up_sync(0xffffffffu, incl, o);
    if (lane >= o) incl += n;
  }
  if (lane == 31) s_red[warp] = (int)incl;
  __syncthreads();
  uint32_t base = 0;
  for (int w = 0; w < warp; ++w) base += (uint32_t)s_red[w];
  uint32_t cdf = base + incl - pdf;
  pdf_out[t] = pdf;
  enc_out[t] = make_enc_entry(pdf, cdf, p);
}

// Shared epilogue of every histogram producer (CTAs of exactly 256 threads):
// merge the CTA's bins into ctrl->hist; the last CTA to finish normalises,
// records the merged size and clears the histogram and its counters for the
// next call. merged_size_if_known == ~0 reads the size from ctrl.
__device__ inline void hist_merge_and_normalize(uint32_t (*s_h)[kAnsSyms], int nwarps, Ctrl* ctrl,
                                         unsigned long long merged_size_if_known,
                                         int counter_slot, int prob_bits) {
  __shared__ int s_last;
  __shared__ uint32_t s_hist[kAnsSyms];
  __syncthreads();
  const int t = threadIdx.x;
  if (t < kAnsSyms) {
    uint32_t v = 0;
    for (int w = 0; w < nwarps; ++w) v += s_h[w][t];
    if (v) atomicAdd(&ctrl->hist[t], v);
  }
  __threadfence();
  __syncthreads();
  if (t == 0) s_last = atomicAdd(&ctrl->done_counter[counter_slot], 1u) == gridDim.x - 1;
  __syncthreads();
  if (!s_last) return;
  __threadfence();
  if (t < kAnsSyms) s_hist[t] = __ldcg(&ctrl->hist[t]);
  unsigned long long msize = merged_size_if_known;
  if (msize == ~0ull) msize = __ldcg(&ctrl->merged_size);
  __syncthreads();
  normalize_cta(s_hist, (uint32_t)msize, prob_bits, ctrl->pdf, ctrl->enc_table);
  ctrl->hist[t] = 0;
  if (t == 0) {
    ctrl->merged_size = msize;
    ctrl->tile_counter[counter_slot] = 0;
    ctrl->done_counter[counter_slot] = 0;
  }
}

}  // namespace mans
