// batch.cu -- batched MANS compress / decompress for sm_100a: thousands of
// buffers of uneven size and element type go through one persistent launch
// per stage, fed by a device work queue.
//
// The work queue is the concatenation of every buffer's units (mapping
// groups, rANS blocks, decode chunks): warps (or CTAs) claim global unit
// indices in order from an atomic counter and find the unit's buffer by
// scanning the descriptor table forward from the last buffer they worked on
// (claims only increase, so the scan is amortised O(1)). Each buffer keeps
// its own look-back flags (slices of shared arrays), histogram, coding table
// and status, so one buffer's error does not disturb the others, and the
// bytes produced for a buffer are exactly those of the single-buffer path.
//
// Stages. Compress: begin (reset statuses) -> map (ADM mapping + histogram
// per buffer; raw-byte buffers are only histogrammed) -> plan (one CTA per
// buffer: normalise, scan of block counts across buffers, header of empty
// buffers) -> encode. Decompress: begin -> plan (validate headers, scan of
// decode chunks) -> decode (a CTA takes a chunk of up to 8 blocks of one
// buffer and keeps that buffer's decode table in shared memory) -> unmap.
// Every stage reads its bounds from device memory, and the look-back epoch is
// device-resident, so a whole batch can be captured in a CUDA graph.
#include "adm_u16.cuh"
#include "adm_u32.cuh"
#include "ans_dev.cuh"
#include "batch_internal.h"
#include "mans_internal.h"

namespace mans {

constexpr int kBWarps = 8;
constexpr int kBThreads = kBWarps * 32;
constexpr uint32_t kRawChunk = 4096;  // histogram unit of a raw-byte buffer

__device__ __forceinline__ Sink item_sink(Ctrl* ctrl, BatchState* st) {
  return Sink{&ctrl->status, &ctrl->detail, &st->status, &st->detail};
}

// Forward scan: the item owning global unit u, starting from `it`.
template <typename BaseFn>
__device__ __forceinline__ uint32_t find_item(uint32_t it, uint32_t count, uint64_t u, BaseFn base) {
  while (it + 1 < count && u >= base(it + 1)) ++it;
  return it;
}

// ------------------------------------------------------------------------
__global__ void batch_begin_kernel(BatchState* states, uint32_t count, Ctrl* ctrl) {
  for (uint32_t i = blockIdx.x * blockDim.x + threadIdx.x; i < count; i += gridDim.x * blockDim.x) {
    states[i].status = 0;
    states[i].detail = 0;
  }
  if (blockIdx.x == 0 && threadIdx.x == 0) {
    ctrl->status = 0;
    ctrl->detail = 0;
  }
}

// ------------------------------------------------------------------------
// Compress stage 1: mapping over the global group space.
// ------------------------------------------------------------------------
struct BatchMapSmem {
  alignas(16) uint8_t stage[kBWarps][kGroupRecMax + 16];
};

__device__ __forceinline__ void flush_hist(uint32_t* h, uint32_t* dst, int lane) {
  __syncwarp();
  for (int i = lane; i < kAnsSyms; i += 32) {
    const uint32_t v = h[i];
    if (v) {
      atomicAdd(&dst[i], v);
      h[i] = 0;
    }
  }
  __syncwarp();
}

__global__ __launch_bounds__(kBThreads) void batch_map_kernel(const BatchItem* __restrict__ items,
                                                              BatchState* states, uint32_t count,
                                                              uint64_t total_units, Ctrl* ctrl,
                                                              unsigned long long* flags) {
  extern __shared__ __align__(16) uint8_t smem_raw[];
  BatchMapSmem& sm = *reinterpret_cast<BatchMapSmem*>(smem_raw);
  __shared__ uint32_t s_h[kBWarps][kAnsSyms];
  const int t = threadIdx.x, warp = t >> 5, lane = t & 31;
  for (int i = t; i < kBWarps * kAnsSyms; i += kBThreads) (&s_h[0][0])[i] = 0;
  __syncthreads();
  const uint32_t epoch = *((volatile uint32_t*)&ctrl->epoch);
  uint32_t it = 0, cur_item = 0xffffffffu;
  auto base = [&](uint32_t i) { return items[i].group_base; };
  while (true) {
    const uint32_t u = warp_claim(&ctrl->tile_counter[0], lane);
    if (u >= total_units) break;
    it = find_item(it, count, u, base);
    if (it != cur_item) {
      if (cur_item != 0xffffffffu) flush_hist(s_h[warp], states[cur_item].hist, lane);
      cur_item = it;
    }
    const BatchItem& b = items[it];
    BatchState* st = &states[it];
    const Sink sink = item_sink(ctrl, st);
    const uint32_t grp = (uint32_t)(u - b.group_base);
    if (b.dtype == MANS_U16) {
      map16_group(reinterpret_cast<const uint16_t*>(b.in), b.n, b.m, b.m_cap, flags + b.group_base,
                  &st->msize, grp, epoch, sink, s_h[warp], lane);
    } else if (b.dtype == MANS_U32) {
      map32_group(reinterpret_cast<const uint32_t*>(b.in), b.n, b.m, b.m_cap,
                  flags + b.group_base, &st->msize, grp, epoch, sink, s_h[warp], sm.stage[warp],
                  lane);
    } else {
      // raw bytes: histogram one 4 KiB chunk
      const uint64_t s0 = (uint64_t)grp * kRawChunk;
      const uint32_t len = (uint32_t)min_u64(kRawChunk, b.n - s0);
      const uint8_t* p = b.in + s0;
      uint32_t* h = s_h[warp];
      if (len == kRawChunk) {
        const uint4* p4 = reinterpret_cast<const uint4*>(p);
#pragma unroll
        for (int q = 0; q < 8; ++q) {
          const uint4 v = __ldcs(p4 + q * 32 + lane);
          const uint32_t w[4] = {v.x, v.y, v.z, v.w};
#pragma unroll
          for (int k = 0; k < 4; ++k) {
            atomicAdd(&h[w[k] & 0xff], 1u);
            atomicAdd(&h[(w[k] >> 8) & 0xff], 1u);
            atomicAdd(&h[(w[k] >> 16) & 0xff], 1u);
            atomicAdd(&h[w[k] >> 24], 1u);
          }
        }
      } else {
        for (uint32_t i = lane; i < len; i += 32) atomicAdd(&h[p[i]], 1u);
      }
    }
  }
  if (cur_item != 0xffffffffu) flush_hist(s_h[warp], states[cur_item].hist, lane);

  __shared__ int s_last;
  __syncthreads();
  if (t == 0) {
    __threadfence();
    s_last = atomicAdd(&ctrl->done_counter[0], 1u) == gridDim.x - 1;
  }
  __syncthreads();
  if (s_last && t == 0) {
    ctrl->tile_counter[0] = 0;
    ctrl->done_counter[0] = 0;
  }
}

// ------------------------------------------------------------------------
// Compress stage 2: per buffer (one CTA of 256 threads each, claimed in
// order): normalise the histogram, scan the block counts across buffers,
// write the header of an empty stream.
// ------------------------------------------------------------------------
__global__ __launch_bounds__(256) void batch_plan_encode_kernel(const BatchItem* __restrict__ items,
                                                                BatchState* states, uint32_t count,
                                                                Ctrl* ctrl,
                                                                unsigned long long* item_flags) {
  __shared__ uint32_t s_item;
  __shared__ uint32_t s_hist[kAnsSyms];
  __shared__ int s_last;
  const int t = threadIdx.x, lane = t & 31;
  const uint32_t epoch = *((volatile uint32_t*)&ctrl->epoch);
  while (true) {
    if (t == 0) s_item = atomicAdd(&ctrl->tile_counter[1], 1u);
    __syncthreads();
    const uint32_t i = s_item;
    if (i >= count) break;
    const BatchItem& b = items[i];
    BatchState* st = &states[i];
    const bool ok = *((volatile uint32_t*)&st->status) == 0;
    unsigned long long msize = b.dtype == MANS_U8 ? b.n : (b.n == 0 ? 0ull : __ldcg(&st->msize));
    s_hist[t] = __ldcg(&st->hist[t]);
    __syncthreads();
    normalize_cta(s_hist, (uint32_t)(ok ? msize : 0), (int)b.prob_bits, st->pdf, st->enc);
    st->hist[t] = 0;
    const uint32_t nb = ok ? (uint32_t)div_up_u64(msize, kAnsBlock) : 0u;
    if (t < 32) {
      if (lane == 0) st_flag(&item_flags[i], make_flag(i == 0 ? kFlagIncl : kFlagAgg, epoch, nb));
      uint32_t excl = 0;
      if (i > 0) {
        excl = lookback_exclusive(item_flags, i, epoch, item_sink(ctrl, st));
        if (lane == 0) st_flag(&item_flags[i], make_flag(kFlagIncl, epoch, excl + nb));
      }
      if (lane == 0) {
        st->msize = msize;
        st->nb = nb;
        st->unit_base = excl;
        if (i + 1 == count) ctrl->merged_size = excl + nb;  // total blocks of the batch
      }
      // an empty stream is its header and a zero pdf (GpuANSEncode.h:201-237)
      if (ok && msize == 0) {
        const uint64_t over = ans_overhead(0);
        if (over > b.out_cap) {
          if (lane == 0) report(item_sink(ctrl, st), MANS_ERR_OUTPUT_OVERFLOW, over);
        } else {
          if (lane < 8) {
            const uint32_t hv = lane == 0 ? kAnsMagicVersion : (lane == 4 ? b.prob_bits : 0u);
            reinterpret_cast<uint32_t*>(b.out)[lane] = hv;
          }
          for (int k = lane; k < kAnsSyms; k += 32)
            reinterpret_cast<uint16_t*>(b.out + kAnsHeaderBytes)[k] = 0;
          if (lane == 0 && b.out_size) *b.out_size = over;
        }
      }
    }
    __syncthreads();
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
// Compress stage 3: encode over the global block space.
// ------------------------------------------------------------------------
struct BatchEncSmem {
  uint2 table[kBWarps][kAnsSyms];
  alignas(16) uint8_t in[kBWarps][kEncStageBytes];
  uint64_t bar[kBWarps];
};

__global__ __launch_bounds__(kBThreads) void batch_encode_kernel(const BatchItem* __restrict__ items,
                                                                 BatchState* states, uint32_t count,
                                                                 Ctrl* ctrl,
                                                                 unsigned long long* flags,
                                                                 uint8_t* __restrict__ slots) {
  extern __shared__ __align__(16) uint8_t smem_raw[];
  BatchEncSmem& sm = *reinterpret_cast<BatchEncSmem*>(smem_raw);
  __shared__ int s_last;
  const int t = threadIdx.x, warp = t >> 5, lane = t & 31;
  uint64_t* bar = &sm.bar[warp];
  if (lane == 0) mbar_init(bar);
  uint32_t parity = 0;
  __syncthreads();
  const uint32_t epoch = *((volatile uint32_t*)&ctrl->epoch);
  const uint64_t total = __ldcg(&ctrl->merged_size);
  uint16_t* sout =
      reinterpret_cast<uint16_t*>(slots + ((uint64_t)blockIdx.x * kBWarps + warp) * kEncSlotBytes);
  uint32_t it = 0, cur_item = 0xffffffffu;
  auto base = [&](uint32_t i) { return (uint64_t)states[i].unit_base; };
  while (true) {
    const uint32_t u = warp_claim(&ctrl->tile_counter[2], lane);
    if (u >= total) break;
    it = find_item(it, count, u, base);
    const BatchItem& b = items[it];
    BatchState* st = &states[it];
    if (it != cur_item) {
      __syncwarp();
      for (int k = lane; k < kAnsSyms; k += 32) sm.table[warp][k] = st->enc[k];
      __syncwarp();
      cur_item = it;
    }
    const uint32_t blk = u - st->unit_base;
    const uint8_t* src = b.dtype == MANS_U8 ? b.in : b.m;
    encode_block<true>(src, st->msize, b.out, b.out_cap, b.out_size, nullptr, st->pdf,
                       flags + st->unit_base, epoch, (int)b.prob_bits, item_sink(ctrl, st),
                       sm.table[warp], sm.in[warp], bar, parity, sout, blk, lane);
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
    ctrl->epoch = (epoch + 1) & 0x3fffffffu;
  }
}

// ------------------------------------------------------------------------
// Decompress stage 1: per buffer, validate the header and scan the decode
// chunks (8 blocks each) across buffers.
// ------------------------------------------------------------------------
constexpr uint32_t kChunkBlocks = kBWarps;

__global__ __launch_bounds__(32) void batch_plan_decode_kernel(const BatchItem* __restrict__ items,
                                                               BatchState* states, uint32_t count,
                                                               Ctrl* ctrl,
                                                               unsigned long long* item_flags) {
  const int lane = threadIdx.x;
  const uint32_t epoch = *((volatile uint32_t*)&ctrl->epoch);
  while (true) {
    const uint32_t i = warp_claim(&ctrl->tile_counter[0], lane);
    if (i >= count) break;
    const BatchItem& b = items[i];
    BatchState* st = &states[i];
    const Sink sink = item_sink(ctrl, st);
    uint32_t h[5] = {0, 0, 0, 0, 0};
    bool ok = b.in_bytes >= kAnsHeaderBytes + 2 * kAnsSyms;
    if (ok) {
#pragma unroll
      for (int k = 0; k < 5; ++k) h[k] = __ldg(reinterpret_cast<const uint32_t*>(b.in) + k);
    }
    const uint32_t nb = h[1], n = h[2], cw = h[3];
    const int p = (int)(h[4] & 0xfu);
    const uint64_t cap = b.dtype == MANS_U8 ? b.n : b.m_cap;
    ok = ok && h[0] == kAnsMagicVersion && p >= 9 && p <= kMaxProbBits &&
         (uint64_t)nb == div_up_u64(n, kAnsBlock) && ans_overhead(nb) + 2ull * cw <= b.in_bytes &&
         (b.dtype != MANS_U8 || (uint64_t)n == b.n);
    if (!ok && lane == 0) report(sink, MANS_ERR_BAD_STREAM, i);
    if (ok && (uint64_t)n > cap) {  // mapped bytes beyond this buffer's room
      if (lane == 0) report(sink, MANS_ERR_WORKSPACE_OVERFLOW, n);
      ok = false;
    }
    const uint32_t chunks = ok ? (nb + kChunkBlocks - 1) / kChunkBlocks : 0u;
    if (lane == 0) st_flag(&item_flags[i], make_flag(i == 0 ? kFlagIncl : kFlagAgg, epoch, chunks));
    uint32_t excl = 0;
    if (i > 0) {
      excl = lookback_exclusive(item_flags, i, epoch, sink);
      if (lane == 0) st_flag(&item_flags[i], make_flag(kFlagIncl, epoch, excl + chunks));
    }
    if (lane == 0) {
      st->nb = ok ? nb : 0u;
      st->n_hdr = n;
      st->cw = cw;
      st->p = (uint32_t)p;
      st->msize = ok ? n : 0ull;
      st->unit_base = excl;
      if (i + 1 == count) ctrl->merged_size = excl + chunks;  // total chunks
    }
  }
  __shared__ int s_last;
  __syncthreads();
  if (lane == 0) {
    __threadfence();
    s_last = atomicAdd(&ctrl->done_counter[0], 1u) == gridDim.x - 1;
  }
  __syncthreads();
  if (s_last && lane == 0) {
    ctrl->tile_counter[0] = 0;
    ctrl->done_counter[0] = 0;
    ctrl->epoch = (epoch + 1) & 0x3fffffffu;
  }
}

// ------------------------------------------------------------------------
// Decompress stage 2: a CTA claims a chunk of up to 8 blocks of one buffer;
// warp w decodes block 8c + w. The decode tables of the CTA's current
// buffer stay in shared memory until the CTA moves to another buffer.
// ------------------------------------------------------------------------
struct BatchDecSmem {
  uint32_t lut[1 << kMaxProbBits];
  uint8_t sym[1 << kMaxProbBits];
  alignas(16) uint16_t in[kBWarps][kEncOutWords];
  uint64_t bar[kBWarps];
};

__global__ __launch_bounds__(kBThreads) void batch_decode_kernel(const BatchItem* __restrict__ items,
                                                                 BatchState* states, uint32_t count,
                                                                 Ctrl* ctrl) {
  extern __shared__ __align__(16) uint8_t smem_raw[];
  BatchDecSmem& sm = *reinterpret_cast<BatchDecSmem*>(smem_raw);
  __shared__ uint32_t s_scan[kBWarps];
  __shared__ uint32_t s_chunk;
  __shared__ int s_last, s_tables;
  const int t = threadIdx.x, warp = t >> 5, lane = t & 31;
  uint64_t* bar = &sm.bar[warp];
  if (lane == 0) mbar_init(bar);
  uint32_t parity = 0;
  const uint64_t total = __ldcg(&ctrl->merged_size);
  uint32_t it = 0, cur_item = 0xffffffffu;
  auto base = [&](uint32_t i) { return (uint64_t)states[i].unit_base; };
  while (true) {
    __syncthreads();
    if (t == 0) s_chunk = atomicAdd(&ctrl->tile_counter[1], 1u);
    __syncthreads();
    const uint32_t c = s_chunk;
    if (c >= total) break;
    it = find_item(it, count, c, base);  // uniform across the CTA
    const BatchItem& b = items[it];
    BatchState* st = &states[it];
    const uint32_t p = st->p;
    if (it != cur_item) {
      const bool ok = build_decode_tables(b.in, (int)p, sm.lut, sm.sym, s_scan);
      if (t == 0) s_tables = ok;
      __syncthreads();
      if (!s_tables && t == 0) report(item_sink(ctrl, st), MANS_ERR_BAD_STREAM, it);
      cur_item = it;
    }
    if (!s_tables) continue;
    const uint32_t blk = (c - st->unit_base) * kChunkBlocks + warp;
    if (blk < st->nb) {
      uint8_t* dst = b.dtype == MANS_U8 ? b.out : b.m;
      decode_block(b.in, st->nb, st->n_hdr, st->cw, (int)p, dst, sm.lut, sm.sym, sm.in[warp], bar,
                   parity, item_sink(ctrl, st), blk, lane);
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
// Decompress stage 3: inverse mapping over the global group space.
// ------------------------------------------------------------------------
struct BatchUnmapSmem {
  alignas(16) uint8_t stage[kBWarps][kGroupRecMax + 48];
};

__global__ __launch_bounds__(kBThreads) void batch_unmap_kernel(const BatchItem* __restrict__ items,
                                                                BatchState* states, uint32_t count,
                                                                uint64_t total_units, Ctrl* ctrl) {
  extern __shared__ __align__(16) uint8_t smem_raw[];
  BatchUnmapSmem& sm = *reinterpret_cast<BatchUnmapSmem*>(smem_raw);
  __shared__ int s_last;
  const int t = threadIdx.x, warp = t >> 5, lane = t & 31;
  uint32_t it = 0;
  auto base = [&](uint32_t i) { return items[i].group_base; };
  while (true) {
    const uint32_t u = warp_claim(&ctrl->tile_counter[2], lane);
    if (u >= total_units) break;
    it = find_item(it, count, u, base);
    const BatchItem& b = items[it];
    BatchState* st = &states[it];
    if (*((volatile uint32_t*)&st->status) != 0) continue;
    const Sink sink = item_sink(ctrl, st);
    const uint64_t grp = u - b.group_base;
    const uint64_t g = div_up_u64(b.n, kAdmGroup);
    const uint64_t msize = st->msize;
    if (b.dtype == MANS_U16) {
      const uint64_t bits_base = 6 * g + b.n;
      if (msize < bits_base || ((msize - bits_base) & 31)) {
        if (lane == 0) report(sink, MANS_ERR_CORRUPT, msize);
        continue;
      }
      unmap16_group(b.m, b.n, (msize - bits_base) >> 5, reinterpret_cast<uint16_t*>(b.out), grp,
                    sink, lane);
    } else {
      const uint64_t rec_base = 40 * g;
      if (msize < rec_base) {
        if (lane == 0) report(sink, MANS_ERR_CORRUPT, msize);
        continue;
      }
      unmap32_group(b.m, b.n, msize - rec_base, reinterpret_cast<uint32_t*>(b.out), grp, sink,
                    sm.stage[warp], lane);
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
static int occ(const void* fn, int threads, size_t smem) {
  int n = 0;
  if (cudaOccupancyMaxActiveBlocksPerMultiprocessor(&n, fn, threads, smem) != cudaSuccess) n = 1;
  return n > 0 ? n : 1;
}

void init_batch_cfg(BatchCfg& c, const LaunchCfg& base) {
  cudaFuncSetAttribute(batch_map_kernel, cudaFuncAttributeMaxDynamicSharedMemorySize,
                       (int)sizeof(BatchMapSmem));
  cudaFuncSetAttribute(batch_encode_kernel, cudaFuncAttributeMaxDynamicSharedMemorySize,
                       (int)sizeof(BatchEncSmem));
  cudaFuncSetAttribute(batch_decode_kernel, cudaFuncAttributeMaxDynamicSharedMemorySize,
                       (int)sizeof(BatchDecSmem));
  cudaFuncSetAttribute(batch_unmap_kernel, cudaFuncAttributeMaxDynamicSharedMemorySize,
                       (int)sizeof(BatchUnmapSmem));
  c.sms = base.sms;
  c.occ[kStageMap] = occ((const void*)batch_map_kernel, kBThreads, sizeof(BatchMapSmem));
  c.occ[kStagePlanEnc] = occ((const void*)batch_plan_encode_kernel, 256, 0);
  c.occ[kStageEncode] = occ((const void*)batch_encode_kernel, kBThreads, sizeof(BatchEncSmem));
  c.occ[kStagePlanDec] = occ((const void*)batch_plan_decode_kernel, 32, 0);
  c.occ[kStageDecode] = occ((const void*)batch_decode_kernel, kBThreads, sizeof(BatchDecSmem));
  c.occ[kStageUnmap] = occ((const void*)batch_unmap_kernel, kBThreads, sizeof(BatchUnmapSmem));
  for (int s = 0; s < kStages; ++s) c.ctas_per_sm[s] = c.occ[s];
}

uint64_t batch_slot_bytes(const BatchCfg& c) {
  return (uint64_t)c.sms * c.occ[kStageEncode] * kBWarps * kEncSlotBytes;
}

static unsigned grid_of(const BatchCfg& c, int stage, uint64_t want) {
  const uint64_t cap = (uint64_t)c.sms * (uint64_t)c.ctas_per_sm[stage];
  return (unsigned)(want < 1 ? 1 : (want < cap ? want : cap));
}

cudaError_t launch_batch_compress(const BatchDev& d, uint32_t count, uint64_t total_groups,
                                  uint64_t max_blocks, const BatchCfg& c, cudaStream_t s) {
  batch_begin_kernel<<<(count + 255) / 256 + 1, 256, 0, s>>>(d.states, count, d.ctrl);
  batch_map_kernel<<<grid_of(c, kStageMap, div_up_u64(total_groups, kBWarps)), kBThreads,
                     sizeof(BatchMapSmem), s>>>(d.items, d.states, count, total_groups, d.ctrl,
                                                d.group_flags);
  batch_plan_encode_kernel<<<grid_of(c, kStagePlanEnc, count), 256, 0, s>>>(
      d.items, d.states, count, d.ctrl, d.item_flags);
  batch_encode_kernel<<<grid_of(c, kStageEncode, div_up_u64(max_blocks, kBWarps)), kBThreads,
                        sizeof(BatchEncSmem), s>>>(d.items, d.states, count, d.ctrl,
                                                   d.block_flags, d.slots);
  return cudaGetLastError();
}

cudaError_t launch_batch_decompress(const BatchDev& d, uint32_t count, uint64_t total_groups,
                                    uint64_t max_chunks, const BatchCfg& c, cudaStream_t s) {
  batch_begin_kernel<<<(count + 255) / 256 + 1, 256, 0, s>>>(d.states, count, d.ctrl);
  batch_plan_decode_kernel<<<grid_of(c, kStagePlanDec, count), 32, 0, s>>>(
      d.items, d.states, count, d.ctrl, d.item_flags);
  batch_decode_kernel<<<grid_of(c, kStageDecode, max_chunks), kBThreads, sizeof(BatchDecSmem),
                        s>>>(d.items, d.states, count, d.ctrl);
  batch_unmap_kernel<<<grid_of(c, kStageUnmap, div_up_u64(total_groups, kBWarps)), kBThreads,
                       sizeof(BatchUnmapSmem), s>>>(d.items, d.states, count, total_groups, d.ctrl);
  return cudaGetLastError();
}

}  // namespace mans
