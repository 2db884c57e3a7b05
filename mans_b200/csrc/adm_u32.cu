// adm_u32.cu -- single-buffer kernels of the uint32 ADM mapping (per-group
// work in adm_u32.cuh).
#include "adm_u32.cuh"
#include "mans_internal.h"

namespace mans {

// One warp maps one group at a time. Groups are claimed in order, one at a
// time (a claim held while another group is mapped would stall every later
// group's look-back), and the group one grid of warps ahead is prefetched
// into L2 for whichever warp claims it. The warp publishes its group's record
// bytes as soon as they are counted, builds the records in shared memory
// while its predecessors finish, and only then reads its offset from the
// decoupled look-back and stores the records (8-byte aligned) to M.
__global__ __launch_bounds__(kMap32Threads) void adm_u32_map_kernel(
    const uint32_t* __restrict__ in, uint64_t n, uint8_t* __restrict__ M, uint64_t m_cap,
    Ctrl* ctrl, unsigned long long* flags, int prob_bits) {
  extern __shared__ __align__(16) uint8_t smem_raw[];
  Map32Smem& sm = *reinterpret_cast<Map32Smem*>(smem_raw);
  __shared__ uint32_t s_h[kMap32Warps][kAnsSyms];
  const int t = threadIdx.x, warp = t >> 5, lane = t & 31;
  for (int i = t; i < kMap32Warps * kAnsSyms; i += kMap32Threads) (&s_h[0][0])[i] = 0;
  __syncthreads();
  const uint64_t g = div_up_u64(n, kAdmGroup);
  const Sink sink = sink_of(ctrl);
  const bool failed = sink_failed(sink);
  const uint32_t epoch = *((volatile uint32_t*)&ctrl->epoch);
  const uint32_t ahead = gridDim.x * kMap32Warps;
  while (!failed) {
    const uint32_t grp = warp_claim(&ctrl->tile_counter[0], lane);
    if (grp >= g) break;
    if (lane == 0 && (uint64_t)grp + ahead < g) {
      const uint64_t ns = ((uint64_t)grp + ahead) * kAdmGroup;
      prefetch_l2(in + ns, (uint32_t)(4 * min_u64(kAdmGroup, n - ns)));
    }
    map32_group(in, n, M, m_cap, flags, &ctrl->merged_size, grp, epoch, sink, s_h[warp],
                sm.stage[warp], lane);
  }
  hist_merge_and_normalize(s_h, kMap32Warps, ctrl, g == 0 ? 0ull : ~0ull, 0, prob_bits);
}

__global__ __launch_bounds__(kUnmap32Threads) void adm_u32_unmap_kernel(
    const uint8_t* __restrict__ M, uint64_t n, uint32_t* __restrict__ out, Ctrl* ctrl) {
  extern __shared__ __align__(16) uint8_t smem_raw[];
  Unmap32Smem& sm = *reinterpret_cast<Unmap32Smem*>(smem_raw);
  const Sink sink = sink_of(ctrl);
  if (sink_failed(sink)) return;
  const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
  const uint64_t g = div_up_u64(n, kAdmGroup);
  const uint64_t msize = __ldcg(&ctrl->merged_size);
  const uint64_t rec_base = 40 * g;
  if (msize < rec_base) {
    if (blockIdx.x == 0 && threadIdx.x == 0) report(sink, MANS_ERR_CORRUPT, msize);
    return;
  }
  const uint64_t warps = (uint64_t)gridDim.x * kUnmap32Warps;
  for (uint64_t grp = (uint64_t)blockIdx.x * kUnmap32Warps + warp; grp < g; grp += warps)
    unmap32_group(M, n, msize - rec_base, out, grp, sink, sm.stage[warp], lane);
}

// ------------------------------------------------------------------------
static int occupancy32(const void* fn, int threads, size_t smem) {
  int n = 0;
  if (cudaOccupancyMaxActiveBlocksPerMultiprocessor(&n, fn, threads, smem) != cudaSuccess) {
    cudaGetLastError();
    n = 1;
  }
  return n > 0 ? n : 1;
}

// Called once per device (with the device current) by init_launch_cfg; the
// results live in the caller's LaunchCfg, so launches on several devices or
// from several host threads read no shared mutable state.
void init_adm_u32_launch_cfg(LaunchCfg& cfg) {
  cudaFuncSetAttribute(adm_u32_map_kernel, cudaFuncAttributeMaxDynamicSharedMemorySize,
                       (int)sizeof(Map32Smem));
  cudaFuncSetAttribute(adm_u32_unmap_kernel, cudaFuncAttributeMaxDynamicSharedMemorySize,
                       (int)sizeof(Unmap32Smem));
  cfg.map32_ctas = occupancy32((const void*)adm_u32_map_kernel, kMap32Threads, sizeof(Map32Smem));
  cfg.unmap32_ctas =
      occupancy32((const void*)adm_u32_unmap_kernel, kUnmap32Threads, sizeof(Unmap32Smem));
}

static unsigned grid_for(uint64_t want, uint64_t cap) {
  return (unsigned)(want < 1 ? 1 : (want < cap ? want : cap));
}

cudaError_t launch_adm_u32_map(const uint32_t* in, uint64_t n, uint8_t* m, uint64_t m_cap,
                               Ctrl* ctrl, unsigned long long* flags, int prob_bits,
                               const LaunchCfg& cfg, cudaStream_t s) {
  const int occ = cfg.map32_ctas > 0 ? cfg.map32_ctas : 1;
  const uint64_t ctas = div_up_u64(div_up_u64(n, kAdmGroup), kMap32Warps);
  adm_u32_map_kernel<<<grid_for(ctas, (uint64_t)cfg.sms * occ), kMap32Threads, sizeof(Map32Smem),
                       s>>>(in, n, m, m_cap, ctrl, flags, prob_bits);
  return cudaGetLastError();
}

cudaError_t launch_adm_u32_unmap(const uint8_t* m, uint64_t n, uint32_t* out, Ctrl* ctrl,
                                 const LaunchCfg& cfg, cudaStream_t s) {
  const int occ = cfg.unmap32_ctas > 0 ? cfg.unmap32_ctas : 1;
  const uint64_t groups = div_up_u64(n, kAdmGroup);
  adm_u32_unmap_kernel<<<grid_for(div_up_u64(groups, kUnmap32Warps), (uint64_t)cfg.sms * occ),
                         kUnmap32Threads, sizeof(Unmap32Smem), s>>>(m, n, out, ctrl);
  return cudaGetLastError();
}

}  // namespace mans
