// adm_u16.cu -- single-buffer kernels of the uint16 ADM mapping (per-group
// work in adm_u16.cuh).
#include "adm_u16.cuh"
#include "mans_internal.h"

namespace mans {

// One warp maps one group at a time; groups are claimed in order, one at a
// time (a claim held while another group is mapped would stall every later
// group's look-back), and the group one grid of warps ahead is prefetched
// into L2 for whichever warp claims it. The group's bit offset comes from a
// decoupled look-back over per-group flags.
__global__ __launch_bounds__(kMapThreads) void adm_u16_map_kernel(
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
  const uint32_t ahead = gridDim.x * kMapWarps;
  while (!failed) {
    const uint32_t grp = warp_claim(&ctrl->tile_counter[0], lane);
    if (grp >= g) break;
    if (lane == 0 && (uint64_t)grp + ahead < g) {
      const uint64_t ns = ((uint64_t)grp + ahead) * kAdmGroup;
      prefetch_l2(in + ns, (uint32_t)(2 * min_u64(kAdmGroup, n - ns)));
    }
    map16_group(in, n, M, m_cap, flags, &ctrl->merged_size, grp, epoch, sink, s_h[warp], lane);
  }
  hist_merge_and_normalize(s_h, kMapWarps, ctrl, g == 0 ? 0ull : ~0ull, 0, prob_bits);
}

__global__ __launch_bounds__(kUnmapThreads, 4) void adm_u16_unmap_kernel(
    const uint8_t* __restrict__ M, uint64_t n, uint16_t* __restrict__ out, Ctrl* ctrl) {
  const Sink sink = sink_of(ctrl);
  if (sink_failed(sink)) return;
  const int lane = threadIdx.x & 31;
  const uint64_t g = div_up_u64(n, kAdmGroup);
  const uint64_t msize = __ldcg(&ctrl->merged_size);
  const uint64_t bits_base = 6 * g + n;
  if (msize < bits_base || ((msize - bits_base) & 31)) {
    if (blockIdx.x == 0 && threadIdx.x == 0) report(sink, MANS_ERR_CORRUPT, msize);
    return;
  }
  const uint64_t tot = (msize - bits_base) >> 5;
  const uint64_t warps = (uint64_t)gridDim.x * (kUnmapThreads / 32);
  for (uint64_t grp = (uint64_t)blockIdx.x * (kUnmapThreads / 32) + (threadIdx.x >> 5); grp < g;
       grp += warps)
    unmap16_group(M, n, tot, out, grp, sink, lane);
}

// ------------------------------------------------------------------------
void init_adm_u16_launch_cfg(LaunchCfg& cfg) {
  int nmap = 0;
  cudaOccupancyMaxActiveBlocksPerMultiprocessor(&nmap, adm_u16_map_kernel, kMapThreads, 0);
  cfg.map_ctas = nmap > 0 ? nmap : 1;
}

cudaError_t launch_adm_u16_map(const uint16_t* in, uint64_t n, uint8_t* m, uint64_t m_cap,
                               Ctrl* ctrl, unsigned long long* flags, int prob_bits,
                               const LaunchCfg& cfg, cudaStream_t s) {
  const uint64_t ctas = div_up_u64(div_up_u64(n, kAdmGroup), kMapWarps);
  const uint64_t cap = (uint64_t)cfg.sms * cfg.map_ctas;
  const unsigned grid = (unsigned)(ctas < 1 ? 1 : (ctas < cap ? ctas : cap));
  adm_u16_map_kernel<<<grid, kMapThreads, 0, s>>>(in, n, m, m_cap, ctrl, flags, prob_bits);
  return cudaGetLastError();
}

cudaError_t launch_adm_u16_unmap(const uint8_t* m, uint64_t n, uint16_t* out, Ctrl* ctrl,
                                 const LaunchCfg& cfg, cudaStream_t s) {
  const uint64_t groups = div_up_u64(n, kAdmGroup);
  const uint64_t want = div_up_u64(groups, kUnmapThreads / 32);
  const uint64_t cap = (uint64_t)cfg.sms * 8;
  const unsigned grid = (unsigned)(want < 1 ? 1 : (want < cap ? want : cap));
  adm_u16_unmap_kernel<<<grid, kUnmapThreads, 0, s>>>(m, n, out, ctrl);
  return cudaGetLastError();
}

}  // namespace mans
