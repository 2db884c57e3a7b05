// adm_u16.cu -- single-buffer kernels of the uint16 ADM mapping (per-group
// work in adm_u16.cuh).
#include "adm_u16.cuh"
#include "mans_internal.h"

namespace mans {

// One warp maps a unit of kMapUnit consecutive groups at a time, and the unit
// is the decoupled look-back's unit: the warp maps the front of each group
// (everything that does not depend on its offset), publishes the unit's
// length, reads the unit's offset and writes each group at it. A uint16 group
// is only 1 KiB of input, so per-group claims and look-backs cost a fifth of
// the kernel; units of two groups halve them (1 GiB: 1.88 -> 1.40 ms). Units
// are claimed in order, one at a time (a claim held while another unit is
// mapped would stall every later unit's look-back), and the unit one grid of
// warps ahead is prefetched into L2 for whichever warp claims it. Each
// unit's look-back is deferred until the warp has published its next unit
// (below): two units' fronts in registers (64 registers, 4 CTAs per SM;
// 2 GiB volume frames 2.44 -> 2.02 ms).
constexpr uint32_t kMapUnit = kU16MapUnit;

template <int kLayout>
__global__ __launch_bounds__(kMapThreads, 4) void adm_u16_map_kernel(
    const uint16_t* __restrict__ in, uint64_t n, uint8_t* __restrict__ M, uint64_t m_cap,
    Ctrl* ctrl, unsigned long long* flags, int prob_bits) {
  __shared__ uint32_t s_h[kMapWarps][kAnsSyms];
  const int t = threadIdx.x, warp = t >> 5, lane = t & 31;
  for (int i = t; i < kMapWarps * kAnsSyms; i += kMapThreads) (&s_h[0][0])[i] = 0;
  __syncthreads();
  const uint64_t g = div_up_u64(n, kAdmGroup);
  const Sink sink = sink_of(ctrl);
  const bool failed = sink_failed(sink);
  const uint32_t epoch = *((volatile uint32_t*)&ctrl->epoch);
  const uint64_t units = div_up_u64(g, kMapUnit);
  const uint32_t ahead = gridDim.x * kMapWarps;
  // The offset-dependent half of a unit: look-back, inclusive prefix, and
  // the groups' fields and bit bytes.
  auto finish = [&](uint32_t u, const Map16Lane (&S)[kMapUnit], uint32_t len) {
    uint32_t off = 0;
    if (u > 0) {
      off = lookback_exclusive(flags, u, epoch, sink);
      if (lane == 0) st_flag(&flags[u], make_flag(kFlagIncl, epoch, off + len));
    }
#pragma unroll
    for (uint32_t q = 0; q < kMapUnit; ++q) {
      if ((uint64_t)u * kMapUnit + q < g)
        map16_back<kLayout>(in, n, M, m_cap, &ctrl->merged_size, u * kMapUnit + q, off, S[q],
                            sink, s_h[warp], lane);
      off += S[q].L;
    }
  };
  // A unit waits in registers (its groups' front halves) for its offset
  // while the warp maps the front of its next unit; its look-back then runs
  // after that unit's length is published, when its predecessors have
  // published theirs, instead of stalling the warp on a predecessor that
  // started at the same time. Every claimed unit publishes its length before
  // any wait, so the deferred look-backs always complete.
  Map16Lane P[kMapUnit];
  uint32_t pu = 0xffffffffu, plen = 0;
  while (!failed) {
    const uint32_t u = warp_claim(&ctrl->tile_counter[0], lane);
    if (u >= units) break;
    if (lane == 0 && (uint64_t)u + ahead < units) {
      const uint64_t ns = ((uint64_t)u + ahead) * kMapUnit * kAdmGroup;
      prefetch_l2(in + ns, (uint32_t)(2 * min_u64(kMapUnit * kAdmGroup, n - ns)));
    }
    Map16Lane S[kMapUnit];
    uint32_t len = 0;  // the unit's length in 32-byte units
#pragma unroll
    for (uint32_t q = 0; q < kMapUnit; ++q) {
      S[q].L = 0;
      if ((uint64_t)u * kMapUnit + q < g) {
        map16_front<kLayout>(in, n, M, u * kMapUnit + q, s_h[warp], lane, S[q]);
        len += S[q].L;
      }
    }
    if (lane == 0) st_flag(&flags[u], make_flag(u == 0 ? kFlagIncl : kFlagAgg, epoch, len));
    if (pu != 0xffffffffu) finish(pu, P, plen);
#pragma unroll
    for (uint32_t q = 0; q < kMapUnit; ++q) P[q] = S[q];
    pu = u;
    plen = len;
  }
  if (pu != 0xffffffffu) finish(pu, P, plen);
  // An empty input maps to nothing, except in the CPU layout, whose g + 1
  // prefix words are then the single word 0 (mappingcpuV2.cpp:117-121).
  unsigned long long empty_size = 0;
  if (kLayout == kLayoutCpuV2 && g == 0) {
    empty_size = 4;
    if (blockIdx.x == 0 && t == 0) {
      reinterpret_cast<uint16_t*>(M)[0] = 0;
      reinterpret_cast<uint16_t*>(M)[1] = 0;
      s_h[0][0] += 4;
    }
  }
  hist_merge_and_normalize(s_h, kMapWarps, ctrl, g == 0 ? empty_size : ~0ull, 0, prob_bits);
}

template <int kLayout>
__global__ __launch_bounds__(kUnmapThreads, 4) void adm_u16_unmap_kernel(
    const uint8_t* __restrict__ M, uint64_t n, uint16_t* __restrict__ out, Ctrl* ctrl,
    const uint32_t* __restrict__ v12_excl) {
  const Sink sink = sink_of(ctrl);
  if (sink_failed(sink)) return;
  const int lane = threadIdx.x & 31;
  const uint64_t g = div_up_u64(n, kAdmGroup);
  const uint64_t msize = __ldcg(&ctrl->merged_size);
  const uint64_t bits_base = u16_header_bytes(kLayout, g) + n;
  if (msize < bits_base || ((msize - bits_base) & 31)) {
    if (blockIdx.x == 0 && threadIdx.x == 0) report(sink, MANS_ERR_CORRUPT, msize);
    return;
  }
  const uint64_t tot = (msize - bits_base) >> 5;
  const uint64_t warps = (uint64_t)gridDim.x * (kUnmapThreads / 32);
  for (uint64_t grp = (uint64_t)blockIdx.x * (kUnmapThreads / 32) + (threadIdx.x >> 5); grp < g;
       grp += warps)
    unmap16_group<kLayout>(M, n, tot, out, grp, sink, lane, v12_excl);
}

// V12 layout: exclusive prefix of the u16 group lengths into excl (tiles of
// 2,048 groups, one per CTA of 256 threads, claimed in order; single-pass
// look-back over per-tile flags). The last CTA advances the epoch, because
// the flags are shared with the rANS encoder.
constexpr int kScanThreads = 256, kScanPer = 8, kScanTile = kScanThreads * kScanPer;

__global__ __launch_bounds__(kScanThreads) void adm_u16_v12_scan_kernel(
    const uint8_t* __restrict__ M, uint64_t n, uint32_t* __restrict__ excl, Ctrl* ctrl,
    unsigned long long* flags) {
  __shared__ uint32_t s_tile, s_warp[kScanThreads / 32], s_prefix;
  __shared__ int s_last;
  const int t = threadIdx.x, warp = t >> 5, lane = t & 31;
  const uint64_t g = div_up_u64(n, kAdmGroup);
  const uint16_t* len = reinterpret_cast<const uint16_t*>(M);
  const uint32_t epoch = *((volatile uint32_t*)&ctrl->epoch);
  const Sink sink = sink_of(ctrl);
  while (true) {
    __syncthreads();
    if (t == 0) s_tile = atomicAdd(&ctrl->tile_counter[6], 1u);
    __syncthreads();
    const uint32_t tile = s_tile;
    const uint64_t base = (uint64_t)tile * kScanTile;
    if (base >= g) break;
    uint32_t v[kScanPer], sum = 0;
#pragma unroll
    for (int i = 0; i < kScanPer; ++i) {
      const uint64_t k = base + (uint64_t)t * kScanPer + i;
      v[i] = k < g ? len[k] : 0u;
      sum += v[i];
    }
    uint32_t incl = sum;
#pragma unroll
    for (int o = 1; o < 32; o <<= 1) {
      const uint32_t y = __shfl_up_sync(0xffffffffu, incl, o);
      if (lane >= o) incl += y;
    }
    if (lane == 31) s_warp[warp] = incl;
    __syncthreads();
    uint32_t wbase = 0, total = 0;
    for (int w = 0; w < kScanThreads / 32; ++w) {
      if (w < warp) wbase += s_warp[w];
      total += s_warp[w];
    }
    if (warp == 0) {
      if (lane == 0) st_flag(&flags[tile], make_flag(tile == 0 ? kFlagIncl : kFlagAgg, epoch, total));
      uint32_t pre = 0;
      if (tile > 0) {
        pre = lookback_exclusive(flags, tile, epoch, sink);
        if (lane == 0) st_flag(&flags[tile], make_flag(kFlagIncl, epoch, pre + total));
      }
      if (lane == 0) s_prefix = pre;
    }
    __syncthreads();
    uint32_t run = s_prefix + wbase + incl - sum;
#pragma unroll
    for (int i = 0; i < kScanPer; ++i) {
      const uint64_t k = base + (uint64_t)t * kScanPer + i;
      if (k < g) excl[k] = run;
      run += v[i];
    }
  }
  __syncthreads();
  if (t == 0) {
    __threadfence();
    s_last = atomicAdd(&ctrl->done_counter[6], 1u) == gridDim.x - 1;
  }
  __syncthreads();
  if (s_last && t == 0) {
    ctrl->tile_counter[6] = 0;
    ctrl->done_counter[6] = 0;
    ctrl->epoch = (epoch + 1) & 0x3fffffffu;
  }
}

// ------------------------------------------------------------------------
void init_adm_u16_launch_cfg(LaunchCfg& cfg) {
  int nmap = 0;
  cudaOccupancyMaxActiveBlocksPerMultiprocessor(&nmap, adm_u16_map_kernel<kLayoutV15>, kMapThreads,
                                                0);
  cfg.map_ctas = nmap > 0 ? nmap : 1;
}

cudaError_t launch_adm_u16_map(const uint16_t* in, uint64_t n, uint8_t* m, uint64_t m_cap,
                               Ctrl* ctrl, unsigned long long* flags, int prob_bits,
                               const LaunchCfg& cfg, cudaStream_t s, int layout) {
  const uint64_t ctas = div_up_u64(div_up_u64(div_up_u64(n, kAdmGroup), kMapUnit), kMapWarps);
  const uint64_t cap = (uint64_t)cfg.sms * cfg.map_ctas;
  const unsigned grid = (unsigned)(ctas < 1 ? 1 : (ctas < cap ? ctas : cap));
  if (layout == kLayoutV12)
    adm_u16_map_kernel<kLayoutV12><<<grid, kMapThreads, 0, s>>>(in, n, m, m_cap, ctrl, flags, prob_bits);
  else if (layout == kLayoutCpuV2)
    adm_u16_map_kernel<kLayoutCpuV2><<<grid, kMapThreads, 0, s>>>(in, n, m, m_cap, ctrl, flags, prob_bits);
  else
    adm_u16_map_kernel<kLayoutV15><<<grid, kMapThreads, 0, s>>>(in, n, m, m_cap, ctrl, flags, prob_bits);
  return cudaGetLastError();
}

cudaError_t launch_adm_u16_unmap(const uint8_t* m, uint64_t n, uint16_t* out, Ctrl* ctrl,
                                 const LaunchCfg& cfg, cudaStream_t s, int layout,
                                 uint32_t* v12_excl, unsigned long long* scan_flags) {
  const uint64_t groups = div_up_u64(n, kAdmGroup);
  const uint64_t want = div_up_u64(groups, kUnmapThreads / 32);
  const uint64_t cap = (uint64_t)cfg.sms * 8;
  const unsigned grid = (unsigned)(want < 1 ? 1 : (want < cap ? want : cap));
  if (layout == kLayoutV12) {
    const uint64_t tiles = div_up_u64(groups, kScanTile);
    const unsigned sgrid = (unsigned)(tiles < 1 ? 1 : (tiles < (uint64_t)cfg.sms * 4 ? tiles : cfg.sms * 4));
    adm_u16_v12_scan_kernel<<<sgrid, kScanThreads, 0, s>>>(m, n, v12_excl, ctrl, scan_flags);
    adm_u16_unmap_kernel<kLayoutV12><<<grid, kUnmapThreads, 0, s>>>(m, n, out, ctrl, v12_excl);
  } else if (layout == kLayoutCpuV2) {
    adm_u16_unmap_kernel<kLayoutCpuV2><<<grid, kUnmapThreads, 0, s>>>(m, n, out, ctrl, nullptr);
  } else {
    adm_u16_unmap_kernel<kLayoutV15><<<grid, kUnmapThreads, 0, s>>>(m, n, out, ctrl, nullptr);
  }
  return cudaGetLastError();
}

}  // namespace mans
