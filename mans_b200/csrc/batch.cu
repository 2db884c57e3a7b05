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
// decode chunks) -> decode (a CTA takes a chunk of up to 32 blocks of one
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
// Compress stage 1: mapping, one launch per dtype over that dtype's unit
// space (units of other dtypes' buffers are empty), so each launch carries
// only its own code path, registers and shared memory. As in the
// single-buffer mappers, units are claimed one at a time and the unit one
// grid of warps ahead is prefetched into L2 (a second forward cursor finds
// its buffer).
// ------------------------------------------------------------------------
struct BatchMapSmem {
  alignas(16) uint8_t stage[kBWarps][kGroupRecMax + 16];
};
// dynamic shared memory of the uint32 map for CTAs of `warps` warps (the
// stages of the warps present)
inline size_t map32_smem(int warps) { return (size_t)warps * (kGroupRecMax + 16); }

// Histogram merging. Every warp counts into its own shared histogram. When
// it leaves a buffer, it adds those counts into a CTA-level slot for that
// buffer (shared by the CTA's warps on the same buffer, reference counted);
// the last warp to leave a slot adds it into the buffer's global histogram.
// So a buffer that the whole GPU works on at once is merged into global
// memory about once per CTA instead of once per warp. A warp that finds its
// slot taken by another buffer merges straight into global memory.
constexpr int kCtaSlots = 4;
struct MapHist {
  uint32_t warp[kBWarps][kAnsSyms];
  uint32_t slot[kCtaSlots][kAnsSyms];
  uint32_t state[kCtaSlots];  // 0 free; else (buffer + 1) << 12 | warps inside
};

__device__ __forceinline__ uint32_t* item_hist(uint32_t* hists, uint32_t hist_items, uint32_t item) {
  return hists + ((uint64_t)(blockIdx.x % kHistCopies) * hist_items + item) * kAnsSyms;
}

// Enter buffer `item`: the slot index, or -1 when its slot is busy.
__device__ __forceinline__ int hist_enter(MapHist& mh, uint32_t item, int lane) {
  int k = -1;
  if (lane == 0) {
    const int s = (int)(item % kCtaSlots);
    const uint32_t tag = (item + 1) << 12;
    uint32_t old = *((volatile uint32_t*)&mh.state[s]);
    for (int tries = 0; tries < 8; ++tries) {
      uint32_t nv;
      if (old == 0) nv = tag | 1u;
      else if ((old & ~0xfffu) == tag && (old & 0xfffu) != 0) nv = old + 1;
      else break;  // another buffer, or this one being merged out
      const uint32_t prev = atomicCAS(&mh.state[s], old, nv);
      if (prev == old) {
        k = s;
        break;
      }
      old = prev;
    }
  }
  return __shfl_sync(0xffffffffu, k, 0);
}

__device__ __forceinline__ void hist_leave(MapHist& mh, int slot, uint32_t* wh, uint32_t* gh,
                                           int lane) {
  __syncwarp();
  if (slot < 0) {
    for (int i = lane; i < kAnsSyms; i += 32) {
      const uint32_t v = wh[i];
      if (v) {
        atomicAdd(&gh[i], v);
        wh[i] = 0;
      }
    }
    __syncwarp();
    return;
  }
  uint32_t* sh = mh.slot[slot];
  for (int i = lane; i < kAnsSyms; i += 32) {
    const uint32_t v = wh[i];
    if (v) {
      atomicAdd(&sh[i], v);
      wh[i] = 0;
    }
  }
  __threadfence_block();
  __syncwarp();
  uint32_t last = 0;
  if (lane == 0) last = (atomicSub(&mh.state[slot], 1u) & 0xfffu) == 1u;
  last = __shfl_sync(0xffffffffu, last, 0);
  if (last) {
    // no warp can add to the slot now (entering needs a nonzero count)
    __threadfence_block();
    for (int i = lane; i < kAnsSyms; i += 32) {
      const uint32_t v = sh[i];
      if (v) {
        atomicAdd(&gh[i], v);
        sh[i] = 0;
      }
    }
    __threadfence_block();
    __syncwarp();
    if (lane == 0) atomicExch(&mh.state[slot], 0u);
  }
  __syncwarp();
}

// Bytes of unit u of a buffer of this dtype (for the L2 prefetch).
template <uint32_t kDtype>
__device__ __forceinline__ void unit_span(const BatchItem& b, uint64_t u, const uint8_t*& p,
                                          uint32_t& bytes) {
  constexpr uint32_t eb = kDtype == MANS_U8 ? 1 : kDtype == MANS_U16 ? 2 : 4;
  constexpr uint32_t per = kDtype == MANS_U8    ? kRawChunk
                           : kDtype == MANS_U16 ? kU16MapUnit * kAdmGroup
                                                : kAdmGroup;
  const uint64_t s0 = u * per;
  p = b.in + s0 * eb;
  bytes = (uint32_t)(min_u64(per, b.n - s0) * eb);
}

template <uint32_t kDtype>
__global__ __launch_bounds__(kBThreads, kDtype == MANS_U32 ? 3 : kDtype == MANS_U16 ? 4 : 5) void batch_map_kernel(const BatchItem* __restrict__ items,
                                                              BatchState* states, uint32_t count,
                                                              uint64_t total_units, Ctrl* ctrl,
                                                              unsigned long long* flags,
                                                              uint32_t* hists, uint32_t hist_items,
                                                              uint32_t prefetch_grids) {
  extern __shared__ __align__(16) uint8_t smem_raw[];
  __shared__ MapHist mh;
  constexpr int kSlot = 3 + (kDtype == MANS_U8 ? 0 : kDtype == MANS_U16 ? 1 : 2);
  const int t = threadIdx.x, warp = t >> 5, lane = t & 31;
  for (int i = t; i < (int)(sizeof(MapHist) / 4); i += blockDim.x) reinterpret_cast<uint32_t*>(&mh)[i] = 0;
  __syncthreads();
  uint32_t* wh = mh.warp[warp];
  int hslot = -1;
  const uint32_t epoch = *((volatile uint32_t*)&ctrl->epoch);
  // the unit prefetch_grids grids of warps ahead is prefetched into L2
  const uint64_t ahead = (uint64_t)prefetch_grids * gridDim.x * (blockDim.x >> 5);
  uint32_t it = 0, pit = 0, cur_item = 0xffffffffu;
  auto base = [&](uint32_t i) {
    const BatchItem& x = items[i];
    return x.dtype == kDtype ? x.group_base : ~0ull;  // other dtypes: empty, skipped below
  };
  // Forward scan in this dtype's unit space: buffers of other dtypes hold no
  // units, so the owner of u is the last buffer of this dtype with base <= u.
  auto owner = [&](uint32_t from, uint64_t u) {
    uint32_t k = from;
    for (uint32_t j = from + 1; j < count; ++j) {
      const uint64_t bj = base(j);
      if (bj == ~0ull) continue;
      if (bj > u) break;
      k = j;
    }
    return k;
  };
  // uint16: a unit waits in registers (its groups' front halves) for its
  // offset while the warp maps the front of its next unit, whose length is
  // published first; its look-back then finds its predecessors' lengths
  // published instead of stalling on a predecessor that started at the same
  // time. A pending unit is finished before the warp moves to another buffer,
  // so that its histogram counts stay with its own buffer.
  Map16Lane P[kU16MapUnit];
  uint32_t p_grp = 0xffffffffu, p_len = 0, p_it = 0;
  auto finish16 = [&]() {
    const BatchItem& pb = items[p_it];
    BatchState* pst = &states[p_it];
    const Sink psink = item_sink(ctrl, pst);
    const uint16_t* in16 = reinterpret_cast<const uint16_t*>(pb.in);
    const uint64_t g = div_up_u64(pb.n, kAdmGroup);
    unsigned long long* fl = flags + pb.flag_base;
    uint32_t off = 0;
    if (p_grp > 0) {
      off = lookback_exclusive(fl, p_grp, epoch, psink);
      if (lane == 0) st_flag(&fl[p_grp], make_flag(kFlagIncl, epoch, off + p_len));
    }
#pragma unroll
    for (uint32_t q = 0; q < kU16MapUnit; ++q) {
      if ((uint64_t)p_grp * kU16MapUnit + q < g)
        map16_back(in16, pb.n, pb.m, pb.m_cap, &pst->msize, p_grp * kU16MapUnit + q, off, P[q],
                   psink, wh, lane);
      off += P[q].L;
    }
    p_grp = 0xffffffffu;
  };
  while (true) {
    const uint32_t u = warp_claim(&ctrl->tile_counter[kSlot], lane);
    if (u >= total_units) break;
    if (lane == 0 && ahead && (uint64_t)u + ahead < total_units) {
      pit = owner(pit, (uint64_t)u + ahead);
      const BatchItem& pb = items[pit];
      const uint8_t* pp;
      uint32_t pbytes;
      unit_span<kDtype>(pb, (uint64_t)u + ahead - pb.group_base, pp, pbytes);
      prefetch_l2(pp, pbytes);
    }
    it = owner(it, u);
    if (it != cur_item) {
      if constexpr (kDtype == MANS_U16) {
        if (p_grp != 0xffffffffu) finish16();
      }
      if (cur_item != 0xffffffffu)
        hist_leave(mh, hslot, wh, item_hist(hists, hist_items, cur_item), lane);
      cur_item = it;
      hslot = hist_enter(mh, it, lane);
    }
    const BatchItem& b = items[it];
    BatchState* st = &states[it];
    const Sink sink = item_sink(ctrl, st);
    const uint32_t grp = (uint32_t)(u - b.group_base);
    if constexpr (kDtype == MANS_U16) {
      // unit grp: groups kU16MapUnit * grp + q of the buffer, one look-back
      const uint16_t* in16 = reinterpret_cast<const uint16_t*>(b.in);
      const uint64_t g = div_up_u64(b.n, kAdmGroup);
      unsigned long long* fl = flags + b.flag_base;
      Map16Lane S[kU16MapUnit];
      uint32_t len = 0;
#pragma unroll
      for (uint32_t q = 0; q < kU16MapUnit; ++q) {
        S[q].L = 0;
        if ((uint64_t)grp * kU16MapUnit + q < g) {
          map16_front(in16, b.n, b.m, grp * kU16MapUnit + q, wh, lane, S[q]);
          len += S[q].L;
        }
      }
      if (lane == 0) st_flag(&fl[grp], make_flag(grp == 0 ? kFlagIncl : kFlagAgg, epoch, len));
      if (p_grp != 0xffffffffu) finish16();
#pragma unroll
      for (uint32_t q = 0; q < kU16MapUnit; ++q) P[q] = S[q];
      p_grp = grp;
      p_len = len;
      p_it = it;
    } else if constexpr (kDtype == MANS_U32) {
      BatchMapSmem& sm = *reinterpret_cast<BatchMapSmem*>(smem_raw);
      map32_group(reinterpret_cast<const uint32_t*>(b.in), b.n, b.m, b.m_cap, flags + b.flag_base,
                  &st->msize, grp, epoch, sink, wh, sm.stage[warp], lane);
    } else {
      // raw bytes: histogram one 4 KiB chunk
      const uint64_t s0 = (uint64_t)grp * kRawChunk;
      const uint32_t len = (uint32_t)min_u64(kRawChunk, b.n - s0);
      const uint8_t* p = b.in + s0;
      uint32_t* h = wh;
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
  if constexpr (kDtype == MANS_U16) {
    if (p_grp != 0xffffffffu) finish16();
  }
  if (cur_item != 0xffffffffu)
    hist_leave(mh, hslot, wh, item_hist(hists, hist_items, cur_item), lane);

  __shared__ int s_last;
  __syncthreads();
  if (t == 0) {
    __threadfence();
    s_last = atomicAdd(&ctrl->done_counter[kSlot], 1u) == gridDim.x - 1;
  }
  __syncthreads();
  if (s_last && t == 0) {
    ctrl->tile_counter[kSlot] = 0;
    ctrl->done_counter[kSlot] = 0;
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
                                                                unsigned long long* item_flags,
                                                                uint32_t* hists,
                                                                uint32_t hist_items) {
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
    uint32_t hv = 0;
#pragma unroll
    for (int c = 0; c < kHistCopies; ++c) {
      uint32_t* h = hists + ((uint64_t)c * hist_items + i) * kAnsSyms + t;
      hv += __ldcg(h);
      *h = 0;
    }
    s_hist[t] = hv;
    __syncthreads();
    normalize_cta(s_hist, (uint32_t)(ok ? msize : 0), (int)b.prob_bits, st->pdf, st->enc);
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

__global__ __launch_bounds__(kBThreads, 4) void batch_encode_kernel(const BatchItem* __restrict__ items,
                                                                 BatchState* states, uint32_t count,
                                                                 Ctrl* ctrl,
                                                                 unsigned long long* flags,
                                                                 uint8_t* __restrict__ slots,
                                                                 uint32_t prefetch_grids) {
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
  // Two word slots per warp: a block's words wait in one for its stream
  // offset while the warp encodes its next block into the other (the
  // single-buffer encoder does the same; every claimed block publishes its
  // aggregate before any wait, so the deferred look-backs complete).
  uint16_t* const slot0 = reinterpret_cast<uint16_t*>(
      slots + ((uint64_t)blockIdx.x * kBWarps + warp) * 2 * kEncSlotBytes);
  uint32_t cur = 0;
  EncPending pend{0xffffffffu, 0, 0, nullptr};
  uint32_t pend_item = 0;
  auto finish = [&](const EncPending& pb, uint32_t i) {
    const BatchItem& bi = items[i];
    BatchState* si = &states[i];
    encode_finish<true>(bi.out, bi.out_cap, si->msize, bi.out_size, nullptr, si->pdf,
                        flags + si->unit_base, epoch, (int)bi.prob_bits, item_sink(ctrl, si), pb,
                        lane);
  };
  uint32_t it = 0, pit = 0, cur_item = 0xffffffffu;
  auto base = [&](uint32_t i) { return (uint64_t)states[i].unit_base; };
  // the block prefetch_grids grids of warps ahead is prefetched into L2 (a
  // second forward cursor finds its buffer)
  const uint64_t ahead = (uint64_t)prefetch_grids * gridDim.x * kBWarps;
  while (true) {
    const uint32_t u = warp_claim(&ctrl->tile_counter[2], lane);
    if (u >= total) break;
    if (ahead && (uint64_t)u + ahead < total) {
      pit = find_item(pit, count, (uint32_t)(u + ahead), base);
      if (lane == 0) {
        const BatchItem& pb = items[pit];
        const BatchState* ps = &states[pit];
        const uint64_t s0 = (uint64_t)(u + ahead - ps->unit_base) * kAnsBlock;
        if (s0 < ps->msize)
          prefetch_l2((pb.dtype == MANS_U8 ? pb.in : pb.m) + s0,
                      (uint32_t)min_u64(kAnsBlock, ps->msize - s0));
      }
    }
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
    uint16_t* const sout = slot0 + cur * (kEncSlotBytes / 2);
    uint32_t x;
    const uint32_t nw = encode_words<false>(src, st->msize, blk, sm.table[warp], sm.in[warp], bar,
                                            parity, sout, (int)b.prob_bits, item_sink(ctrl, st),
                                            lane, x);
    if (lane == 0)
      st_flag(&flags[st->unit_base + blk],
              make_flag(blk == 0 ? kFlagIncl : kFlagAgg, epoch, (nw + 7) & ~7u));
    if (pend.b != 0xffffffffu) finish(pend, pend_item);
    pend = EncPending{blk, nw, x, sout};
    pend_item = it;
    cur ^= 1u;
  }
  if (pend.b != 0xffffffffu) finish(pend, pend_item);
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
// chunks (32 blocks each) across buffers.
// ------------------------------------------------------------------------
// Four blocks per warp per chunk: the CTA's barriers between chunks wait for
// its slowest warp, and longer chunks even the warps out (4,096 mixed
// buffers: decode stage 21.5 ms with one block per warp, 20.4 with four).
constexpr uint32_t kChunkBlocks = 4 * kBWarps;

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
// Decompress stage 2: a CTA claims a chunk of up to 32 blocks of one buffer;
// warp w decodes blocks 32c + w + 8k, k = 0..3. The decode tables of the CTA's current
// buffer stay in shared memory until the CTA moves to another buffer.
// ------------------------------------------------------------------------
struct BatchDecSmem {
  uint32_t lut[1 << kMaxProbBits];  // below every warp's stage (see decode_full_smem)
  DecWarpSmem warp[kBWarps];
  uint64_t bar[kBWarps];
};

__global__ __launch_bounds__(kBThreads) void batch_decode_kernel(const BatchItem* __restrict__ items,
                                                                 BatchState* states, uint32_t count,
                                                                 Ctrl* ctrl) {
  extern __shared__ __align__(16) uint8_t smem_raw[];
  BatchDecSmem& sm = *reinterpret_cast<BatchDecSmem*>(smem_raw);
  __shared__ uint32_t s_scan[kBWarps];
  __shared__ uint32_t s_claim[2];
  __shared__ int s_last, s_tables;
  const int t = threadIdx.x, warp = t >> 5, lane = t & 31;
  uint64_t* bar = &sm.bar[warp];
  if (lane == 0) mbar_init(bar);
  uint32_t parity = 0;
  const uint64_t total = __ldcg(&ctrl->merged_size);
  uint32_t it = 0, pit = 0, cur_item = 0xffffffffu;
  auto base = [&](uint32_t i) { return (uint64_t)states[i].unit_base; };
  // Chunks are claimed two ahead: while chunk c is decoded, thread 0 claims
  // the chunk after next (its atomic's latency is hidden) and every warp
  // prefetches into L2 the words of its block of the next chunk.
  // Every barrier in the loop below is reached by all threads: c and nxt are
  // read from shared memory between two barriers, so they are the same in
  // every thread, and thread 0 writes a claim only after all have read.
  if (t == 0) {
    s_claim[0] = atomicAdd(&ctrl->tile_counter[1], 1u);
    s_claim[1] = atomicAdd(&ctrl->tile_counter[1], 1u);
  }
  __syncthreads();
  uint32_t c = s_claim[0], nxt = s_claim[1];
  __syncthreads();  // all have read both claims before thread 0 writes the next
  while (c < total) {
    if (t == 0) s_claim[0] = atomicAdd(&ctrl->tile_counter[1], 1u);  // read after the barrier below
    if (nxt < total && lane == 0) {
      pit = find_item(pit, count, nxt, base);
      const BatchState* ps = &states[pit];
      for (uint32_t k = 0; k < kChunkBlocks / kBWarps; ++k) {
        const uint32_t pblk = (nxt - ps->unit_base) * kChunkBlocks + warp + k * kBWarps;
        if (pblk < ps->nb) {
          const uint8_t* pin = items[pit].in;
          const uint2 bw = __ldg(reinterpret_cast<const uint2*>(
                                     pin + kAnsHeaderBytes + 2 * kAnsSyms + 128ull * ps->nb) +
                                 pblk);
          const uint32_t wn = ((bw.x & 0xffffu) + 7) & ~7u;
          if ((uint64_t)bw.y + wn <= ps->cw)
            prefetch_l2(pin + ans_overhead(ps->nb) + 2ull * bw.y, 2 * wn);
        }
      }
    }
    it = find_item(it, count, c, base);  // uniform across the CTA
    const BatchItem& b = items[it];
    BatchState* st = &states[it];
    const uint32_t p = st->p;
    if (it != cur_item) {
      const bool ok = build_decode_tables(b.in, (int)p, sm.lut, s_scan);
      if (t == 0) s_tables = ok;
      __syncthreads();
      if (!s_tables && t == 0) report(item_sink(ctrl, st), MANS_ERR_BAD_STREAM, it);
      cur_item = it;
    }
    if (s_tables) {
      for (uint32_t k = 0; k < kChunkBlocks / kBWarps; ++k) {
        const uint32_t blk = (c - st->unit_base) * kChunkBlocks + warp + k * kBWarps;
        if (blk < st->nb) {
          uint8_t* dst = b.dtype == MANS_U8 ? b.out : b.m;
          decode_block(b.in, st->nb, st->n_hdr, st->cw, (int)p, dst, sm.lut, &sm.warp[warp], bar,
                       parity, item_sink(ctrl, st), blk, lane);
        }
      }
    }
    __syncthreads();  // the chunk is done (the table may be rebuilt); s_claim[0] is set
    c = nxt;
    nxt = s_claim[0];
    __syncthreads();  // everyone has read s_claim[0] before thread 0 overwrites it
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
// Decompress stage 3: inverse mapping, one launch per dtype (MANS_U16,
// MANS_U32) over that dtype's unit space.
// ------------------------------------------------------------------------
struct BatchUnmapSmem {
  alignas(16) uint8_t stage[kBWarps][kGroupRecMax + 48];
};

// uint16: 3 CTAs per SM (68 registers): at 64 the unary-stream decoding and
// the batch's per-unit state leave the loads no room to run ahead (28.1 vs
// 24.5 ms on 4,096 mixed buffers); uint32: 5 CTAs.
template <uint32_t kDtype>
__global__ __launch_bounds__(kBThreads, kDtype == MANS_U16 ? 3 : 5) void batch_unmap_kernel(const BatchItem* __restrict__ items,
                                                                BatchState* states, uint32_t count,
                                                                uint64_t total_units, Ctrl* ctrl) {
  extern __shared__ __align__(16) uint8_t smem_raw[];
  __shared__ int s_last;
  constexpr int kSlot = kDtype == MANS_U16 ? 2 : 6;
  const int t = threadIdx.x, warp = t >> 5, lane = t & 31;
  uint32_t it = 0;
  // Units do not depend on one another here (no look-back), so the next
  // unit is claimed while this one is restored: the claim's round trip to
  // L2 leaves the unit's dependency chain.
  uint32_t u = warp_claim(&ctrl->tile_counter[kSlot], lane);
  while (u < total_units) {
    uint32_t nxt = 0;
    if (lane == 0) nxt = atomicAdd(&ctrl->tile_counter[kSlot], 1u);
    for (uint32_t j = it + 1; j < count; ++j) {
      const BatchItem& x = items[j];
      if (x.dtype != kDtype) continue;
      if (x.group_base > u) break;
      it = j;
    }
    do {  // one unit; a skipped unit leaves by break
      const BatchItem& b = items[it];
      BatchState* st = &states[it];
      if (*((volatile uint32_t*)&st->status) != 0) break;
      const Sink sink = item_sink(ctrl, st);
      const uint64_t grp = u - b.group_base;
      const uint64_t g = div_up_u64(b.n, kAdmGroup);
      const uint64_t msize = st->msize;
      if constexpr (kDtype == MANS_U16) {
        const uint64_t bits_base = 6 * g + b.n;
        if (msize < bits_base || ((msize - bits_base) & 31)) {
          if (lane == 0) report(sink, MANS_ERR_CORRUPT, msize);
          break;
        }
        unmap16_group(b.m, b.n, (msize - bits_base) >> 5, reinterpret_cast<uint16_t*>(b.out),
                      grp, sink, lane);
      } else {
        BatchUnmapSmem& sm = *reinterpret_cast<BatchUnmapSmem*>(smem_raw);
        const uint64_t rec_base = 40 * g;
        if (msize < rec_base) {
          if (lane == 0) report(sink, MANS_ERR_CORRUPT, msize);
          break;
        }
        unmap32_group(b.m, b.n, msize - rec_base, reinterpret_cast<uint32_t*>(b.out), grp, sink,
                      sm.stage[warp], lane);
      }
    } while (false);
    u = __shfl_sync(0xffffffffu, nxt, 0);
  }
  __syncthreads();
  if (t == 0) {
    __threadfence();
    s_last = atomicAdd(&ctrl->done_counter[kSlot], 1u) == gridDim.x - 1;
  }
  __syncthreads();
  if (s_last && t == 0) {
    ctrl->tile_counter[kSlot] = 0;
    ctrl->done_counter[kSlot] = 0;
  }
}

// ------------------------------------------------------------------------
// Gather every buffer's status and detail into compact arrays (for an
// asynchronous copy to the host).
// ------------------------------------------------------------------------
__global__ void batch_gather_status_kernel(const BatchState* states, uint32_t count,
                                           uint32_t* status, unsigned long long* detail) {
  for (uint32_t i = blockIdx.x * blockDim.x + threadIdx.x; i < count; i += gridDim.x * blockDim.x) {
    status[i] = states[i].status;
    detail[i] = states[i].detail;
  }
}

cudaError_t launch_batch_gather_status(const BatchDev& d, uint32_t count, uint32_t* status,
                                       unsigned long long* detail, cudaStream_t s) {
  const unsigned grid = (unsigned)((count + 255) / 256 > 0 ? (count + 255) / 256 : 1);
  batch_gather_status_kernel<<<grid, 256, 0, s>>>(d.states, count, status, detail);
  return cudaGetLastError();
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
  cudaFuncSetAttribute(batch_map_kernel<MANS_U32>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                       (int)sizeof(BatchMapSmem));
  cudaFuncSetAttribute(batch_encode_kernel, cudaFuncAttributeMaxDynamicSharedMemorySize,
                       (int)sizeof(BatchEncSmem));
  cudaFuncSetAttribute(batch_decode_kernel, cudaFuncAttributeMaxDynamicSharedMemorySize,
                       (int)sizeof(BatchDecSmem));
  cudaFuncSetAttribute(batch_unmap_kernel<MANS_U32>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                       (int)sizeof(BatchUnmapSmem));
  c.sms = base.sms;
  // the map and unmap stages report the occupancy of their heaviest variant
  c.occ[kStageMap] = min(occ((const void*)batch_map_kernel<MANS_U16>, kBThreads, 0),
                         occ((const void*)batch_map_kernel<MANS_U32>, kBThreads, map32_smem(kBWarps)));
  c.occ[kStagePlanEnc] = occ((const void*)batch_plan_encode_kernel, 256, 0);
  c.occ[kStageEncode] = occ((const void*)batch_encode_kernel, kBThreads, sizeof(BatchEncSmem));
  c.occ[kStagePlanDec] = occ((const void*)batch_plan_decode_kernel, 32, 0);
  c.occ[kStageDecode] = occ((const void*)batch_decode_kernel, kBThreads, sizeof(BatchDecSmem));
  c.occ[kStageUnmap] = min(occ((const void*)batch_unmap_kernel<MANS_U16>, kBThreads, 0),
                           occ((const void*)batch_unmap_kernel<MANS_U32>, kBThreads,
                               sizeof(BatchUnmapSmem)));
  for (int s = 0; s < kStages; ++s) c.ctas_per_sm[s] = c.occ[s];
  c.occ_u16_map = occ((const void*)batch_map_kernel<MANS_U16>, kBThreads, 0);
  c.occ_u8_map = occ((const void*)batch_map_kernel<MANS_U8>, kBThreads, 0);
  c.occ_u16_unmap = occ((const void*)batch_unmap_kernel<MANS_U16>, kBThreads, 0);
  c.occ_map4[0] = occ((const void*)batch_map_kernel<MANS_U8>, 128, 0);
  c.occ_map4[1] = occ((const void*)batch_map_kernel<MANS_U16>, 128, 0);
  c.occ_map4[2] = occ((const void*)batch_map_kernel<MANS_U32>, 128, map32_smem(4));
}

uint64_t batch_slot_bytes(const BatchCfg& c) {
  return (uint64_t)c.sms * c.occ[kStageEncode] * kBWarps * 2 * kEncSlotBytes;  // two per warp
}

// Map stage of dtype kind k: grid for the schedule's warps per CTA (the
// schedule counts CTAs of 8 warps; 4-warp CTAs keep the warps per SM).
static unsigned map_grid(const BatchCfg& c, int kind, uint64_t units, int extra_occ) {
  int per_sm = c.ctas_per_sm[kStageMap];
  if (extra_occ > c.occ[kStageMap]) per_sm = per_sm * extra_occ / c.occ[kStageMap];
  const int w = c.warps[kStageMap];
  if (w != kBWarps) {
    per_sm = per_sm * kBWarps / w;
    if (per_sm > c.occ_map4[kind]) per_sm = c.occ_map4[kind];
  }
  const uint64_t want = div_up_u64(units, (uint64_t)w);
  const uint64_t cap = (uint64_t)c.sms * (uint64_t)(per_sm > 0 ? per_sm : 1);
  return (unsigned)(want < 1 ? 1 : (want < cap ? want : cap));
}

static unsigned grid_of(const BatchCfg& c, int stage, uint64_t want, int extra_occ = 0) {
  // the stage's schedule, scaled for a lighter variant that fits more CTAs
  int per_sm = c.ctas_per_sm[stage];
  if (extra_occ > c.occ[stage]) per_sm = per_sm * extra_occ / c.occ[stage];
  const uint64_t cap = (uint64_t)c.sms * (uint64_t)(per_sm > 0 ? per_sm : 1);
  return (unsigned)(want < 1 ? 1 : (want < cap ? want : cap));
}

cudaError_t launch_batch_compress(const BatchDev& d, uint32_t count, const uint64_t groups[3],
                                  uint64_t max_blocks, const BatchCfg& c, cudaStream_t s,
                                  cudaEvent_t* marks) {
  if (marks) cudaEventRecord(marks[0], s);
  batch_begin_kernel<<<(count + 255) / 256 + 1, 256, 0, s>>>(d.states, count, d.ctrl);
  const int mw = c.warps[kStageMap];
  const uint32_t mpf = (uint32_t)c.prefetch[kStageMap];
  if (groups[1])
    batch_map_kernel<MANS_U16><<<map_grid(c, 1, groups[1], c.occ_u16_map), 32 * mw, 0, s>>>(
        d.items, d.states, count, groups[1], d.ctrl, d.group_flags, d.hists, d.hist_items, mpf);
  if (groups[2])
    batch_map_kernel<MANS_U32><<<map_grid(c, 2, groups[2], 0), 32 * mw, map32_smem(mw), s>>>(
        d.items, d.states, count, groups[2], d.ctrl, d.group_flags, d.hists, d.hist_items, mpf);
  if (groups[0])
    batch_map_kernel<MANS_U8><<<map_grid(c, 0, groups[0], c.occ_u8_map), 32 * mw, 0, s>>>(
        d.items, d.states, count, groups[0], d.ctrl, d.group_flags, d.hists, d.hist_items, mpf);
  if (marks) cudaEventRecord(marks[1], s);
  batch_plan_encode_kernel<<<grid_of(c, kStagePlanEnc, count), 256, 0, s>>>(
      d.items, d.states, count, d.ctrl, d.item_flags, d.hists, d.hist_items);
  if (marks) cudaEventRecord(marks[2], s);
  batch_encode_kernel<<<grid_of(c, kStageEncode, div_up_u64(max_blocks, kBWarps)), kBThreads,
                        sizeof(BatchEncSmem), s>>>(d.items, d.states, count, d.ctrl,
                                                   d.block_flags, d.slots,
                                                   (uint32_t)c.prefetch[kStageEncode]);
  if (marks) cudaEventRecord(marks[3], s);
  return cudaGetLastError();
}

cudaError_t launch_batch_decompress(const BatchDev& d, uint32_t count, const uint64_t groups[3],
                                    uint64_t max_chunks, const BatchCfg& c, cudaStream_t s,
                                    cudaEvent_t* marks) {
  if (marks) cudaEventRecord(marks[0], s);
  batch_begin_kernel<<<(count + 255) / 256 + 1, 256, 0, s>>>(d.states, count, d.ctrl);
  batch_plan_decode_kernel<<<grid_of(c, kStagePlanDec, count), 32, 0, s>>>(
      d.items, d.states, count, d.ctrl, d.item_flags);
  if (marks) cudaEventRecord(marks[1], s);
  batch_decode_kernel<<<grid_of(c, kStageDecode, max_chunks), kBThreads, sizeof(BatchDecSmem),
                        s>>>(d.items, d.states, count, d.ctrl);
  if (marks) cudaEventRecord(marks[2], s);
  if (groups[1])
    batch_unmap_kernel<MANS_U16><<<grid_of(c, kStageUnmap, div_up_u64(groups[1], kBWarps),
                                           c.occ_u16_unmap),
                                   kBThreads, 0, s>>>(d.items, d.states, count, groups[1], d.ctrl);
  if (groups[2])
    batch_unmap_kernel<MANS_U32><<<grid_of(c, kStageUnmap, div_up_u64(groups[2], kBWarps)),
                                   kBThreads, sizeof(BatchUnmapSmem), s>>>(d.items, d.states, count,
                                                                          groups[2], d.ctrl);
  if (marks) cudaEventRecord(marks[3], s);
  return cudaGetLastError();
}

}  // namespace mans
