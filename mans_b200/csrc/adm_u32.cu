// adm_u32.cu -- ADM byte mapping of uint32 arrays (escape-byte format) for
// sm_100a: map (fused with the record-offset scan and the rANS histogram) and
// unmap.
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
#include "ans_table.cuh"
#include "mans_internal.h"
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

__global__ __launch_bounds__(kMap32Threads) void adm_u32_map_kernel(
    const uint32_t* __restrict__ in, uint64_t n, uint8_t* __restrict__ M, uint64_t m_cap,
    Ctrl* ctrl, unsigned long long* flags, uint32_t epoch, int prob_bits) {
  extern __shared__ __align__(16) uint8_t smem_raw[];
  Map32Smem& sm = *reinterpret_cast<Map32Smem*>(smem_raw);
  __shared__ uint32_t s_h[kMap32Warps][kAnsSyms];
  __shared__ uint32_t s_tile;
  __shared__ uint32_t s_len[kMap32Warps];
  __shared__ uint32_t s_excl;
  const int t = threadIdx.x, warp = t >> 5, lane = t & 31;
  for (int i = t; i < kMap32Warps * kAnsSyms; i += kMap32Threads) (&s_h[0][0])[i] = 0;

  const uint64_t g = div_up_u64(n, kAdmGroup);
  const uint64_t ntiles = div_up_u64(g, kMap32Warps);
  const uint64_t rec_base = 40 * g;
  uint32_t* hist = s_h[warp];
  const bool failed = *((volatile uint32_t*)&ctrl->status) != 0;
  __syncthreads();

  while (!failed) {
    if (t == 0) s_tile = atomicAdd(&ctrl->tile_counter[0], 1u);
    __syncthreads();
    const uint64_t tile = s_tile;
    if (tile >= ntiles) break;
    const uint64_t grp = tile * kMap32Warps + warp;
    const bool gvalid = grp < g;
    const uint64_t gs = grp * kAdmGroup;
    const uint64_t ls = gs + (uint64_t)lane * kAdmChunk;
    const int cnt = (!gvalid || ls >= n) ? 0 : (int)min_u64(16, n - ls);

    uint32_t v[16];
    if (cnt == 16) {
      const uint4* src = reinterpret_cast<const uint4*>(in + ls);
#pragma unroll
      for (int q = 0; q < 4; ++q) {
        const uint4 a = __ldcs(src + q);
        v[4 * q] = a.x; v[4 * q + 1] = a.y; v[4 * q + 2] = a.z; v[4 * q + 3] = a.w;
      }
    } else {
#pragma unroll
      for (int i = 0; i < 16; ++i) v[i] = i < cnt ? in[ls + i] : 0u;
    }
    // center: 64-bit sum
    unsigned long long lsum = 0;
#pragma unroll
    for (int i = 0; i < 16; ++i) lsum += v[i];
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) lsum += __shfl_xor_sync(0xffffffffu, lsum, o);
    const uint32_t gcnt = gvalid ? (uint32_t)min_u64(kAdmGroup, n - gs) : 1u;
    const uint32_t c = (uint32_t)(gcnt == kAdmGroup ? (lsum >> 9) : lsum / gcnt);

    // pass 1: record length
    uint32_t rlen = 0;
#pragma unroll
    for (int i = 0; i < 16; ++i) {
      if (i < cnt) {
        uint32_t nb, code;
        bool esc;
        adm_elem_u32(v[i], c, nb, code, esc);
        rlen += nb;
      }
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
    if (lane == 0) s_len[warp] = gvalid ? gtot : 0u;

    // pass 2: build the group's records in shared memory (zero-filled first)
    uint8_t* stage = sm.stage[warp];
    {
      uint4* z = reinterpret_cast<uint4*>(stage);
      for (int i = lane; i < (int)((kGroupRecMax + 16) / 16); i += 32) z[i] = make_uint4(0, 0, 0, 0);
    }
    __syncthreads();  // also publishes s_len

    if (warp == 0) {
      const uint32_t my = lane < kMap32Warps ? s_len[lane] : 0u;
      const uint32_t agg = __reduce_add_sync(0xffffffffu, my);
      if (lane == 0)
        st_release_u64(&flags[tile], make_flag(tile == 0 ? kFlagIncl : kFlagAgg, epoch, agg));
      uint32_t excl = 0;
      if (tile > 0) {
        excl = lookback_exclusive(flags, (uint32_t)tile, epoch, ctrl);
        if (lane == 0) st_release_u64(&flags[tile], make_flag(kFlagIncl, epoch, excl + agg));
      }
      if (lane == 0) {
        s_excl = excl;
        if (tile + 1 == ntiles) {
          const unsigned long long msize = rec_base + (unsigned long long)excl + agg;
          ctrl->merged_size = msize;
          if (msize > m_cap) report_error(ctrl, MANS_ERR_WORKSPACE_OVERFLOW, msize);
        }
      }
    }
    __syncthreads();
    uint32_t goff = s_excl;
#pragma unroll
    for (int i = 0; i < kMap32Warps; ++i) goff += (i < warp) ? s_len[i] : 0u;

    if (gvalid) {
      uint8_t* dst = M + rec_base + goff;
      const uint32_t ph = phase16(dst);
      uint8_t* rec = stage + ph + loff;
      uint32_t pos = 0, zeros = 0;
#pragma unroll
      for (int i = 0; i < 16; ++i) {
        if (i < cnt) {
          uint32_t nb, code;
          bool esc;
          adm_elem_u32(v[i], c, nb, code, esc);
          if (esc) {
            rec[pos] = 254;
            rec[pos + 1] = (uint8_t)(v[i] >> 24);
            rec[pos + 2] = (uint8_t)(v[i] >> 16);
            rec[pos + 3] = (uint8_t)(v[i] >> 8);
            rec[pos + 4] = (uint8_t)v[i];
            atomicAdd(&hist[254], 1u);
            atomicAdd(&hist[v[i] >> 24], 1u);
            atomicAdd(&hist[(v[i] >> 16) & 0xff], 1u);
            atomicAdd(&hist[(v[i] >> 8) & 0xff], 1u);
            atomicAdd(&hist[v[i] & 0xff], 1u);
          } else {
            rec[pos + nb - 1] = (uint8_t)code;
            zeros += nb - 1;
            atomicAdd(&hist[code], 1u);
          }
          pos += nb;
        }
      }
      for (uint32_t i = pos; i < padded; ++i) rec[i] = 255;
      if (zeros) atomicAdd(&hist[0], zeros);
      if (padded > pos) atomicAdd(&hist[255], padded - pos);
      // header fields: group offset, center, lane record length / 8
      if (lane == 0) {
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
      M[8 * g + 32 * grp + lane] = (uint8_t)(padded >> 3);
      atomicAdd(&hist[padded >> 3], 1u);
      __syncwarp();
      if (rec_base + (uint64_t)goff + gtot <= m_cap) warp_store_phase(dst, stage, gtot, lane);
    }
    __syncthreads();
  }
  hist_merge_and_normalize(s_h, kMap32Warps, ctrl, ntiles == 0 ? 0ull : ~0ull, 0, prob_bits);
}

// ------------------------------------------------------------------------
// Unmap (record decode of mappingV9_fuse.cu:126-157). One warp per group;
// the group's records are staged in shared memory with coalesced loads.
// ------------------------------------------------------------------------
constexpr int kUnmap32Warps = 8;
constexpr int kUnmap32Threads = kUnmap32Warps * 32;

struct Unmap32Smem {
  alignas(16) uint8_t stage[kUnmap32Warps][kGroupRecMax + 32];
};

__global__ __launch_bounds__(kUnmap32Threads) void adm_u32_unmap_kernel(
    const uint8_t* __restrict__ M, uint64_t n, uint32_t* __restrict__ out, Ctrl* ctrl) {
  extern __shared__ __align__(16) uint8_t smem_raw[];
  Unmap32Smem& sm = *reinterpret_cast<Unmap32Smem*>(smem_raw);
  if (*((volatile uint32_t*)&ctrl->status) != 0) return;
  const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
  const uint64_t g = div_up_u64(n, kAdmGroup);
  const uint64_t msize = __ldcg(&ctrl->merged_size);
  const uint64_t rec_base = 40 * g;
  if (msize < rec_base) {
    if (blockIdx.x == 0 && threadIdx.x == 0) report_error(ctrl, MANS_ERR_CORRUPT, msize);
    return;
  }
  const uint64_t rec_bytes = msize - rec_base;
  uint8_t* stage = sm.stage[warp];
  const uint64_t warps = (uint64_t)gridDim.x * kUnmap32Warps;
  for (uint64_t grp = (uint64_t)blockIdx.x * kUnmap32Warps + warp; grp < g; grp += warps) {
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
    if ((uint64_t)goff + gtot > rec_bytes || gtot > kGroupRecMax) {
      if (lane == 0) report_error(ctrl, MANS_ERR_CORRUPT, grp);
      continue;
    }
    const uint8_t* src = M + rec_base + goff;
    __syncwarp();
    warp_load_phase(stage, src, gtot, lane);
    __syncwarp();
    const uint8_t* r = stage + phase16(src) + loff;
    uint32_t vals[16];
    uint32_t rp = 0;
    int o = 0;
    bool bad = false;
#pragma unroll
    for (int i = 0; i < 16; ++i) {
      vals[i] = 0;
      if (i < cnt) {
        if (rp >= len) {
          bad = true;
          continue;
        }
        const uint32_t b = r[rp];
        if (b == 254u) {
          if (rp + 5 > len) {
            bad = true;
            continue;
          }
          vals[i] = ((uint32_t)r[rp + 1] << 24) | ((uint32_t)r[rp + 2] << 16) |
                    ((uint32_t)r[rp + 3] << 8) | (uint32_t)r[rp + 4];
          rp += 5;
        } else if (b == 255u) {
          bad = true;  // padding before all elements were decoded
          continue;
        } else {
          uint32_t z = 0;
          while (z < 7 && rp + z < len && r[rp + z] == 0) ++z;
          if (rp + z >= len) {
            bad = true;
            continue;
          }
          const uint32_t code = r[rp + z];
          const uint32_t d = (code >> 1) + 126u * z;
          vals[i] = (code & 1u) ? c - d : c + d;
          rp += z + 1;
        }
        ++o;
      }
    }
    if (__any_sync(0xffffffffu, bad) && lane == 0) report_error(ctrl, MANS_ERR_CORRUPT, grp);
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
    (void)o;
  }
}

// ------------------------------------------------------------------------
void init_adm_u32_launch_cfg(LaunchCfg& cfg) {
  cudaFuncSetAttribute(adm_u32_map_kernel, cudaFuncAttributeMaxDynamicSharedMemorySize,
                       (int)sizeof(Map32Smem));
  cudaFuncSetAttribute(adm_u32_unmap_kernel, cudaFuncAttributeMaxDynamicSharedMemorySize,
                       (int)sizeof(Unmap32Smem));
}

static unsigned grid_for(uint64_t want, uint64_t cap) {
  return (unsigned)(want < 1 ? 1 : (want < cap ? want : cap));
}

cudaError_t launch_adm_u32_map(const uint32_t* in, uint64_t n, uint8_t* m, uint64_t m_cap,
                               Ctrl* ctrl, unsigned long long* flags, uint32_t epoch,
                               int prob_bits, const LaunchCfg& cfg, cudaStream_t s) {
  static int occ = 0;
  if (occ == 0) {
    cudaOccupancyMaxActiveBlocksPerMultiprocessor(&occ, adm_u32_map_kernel, kMap32Threads,
                                                  sizeof(Map32Smem));
    if (occ < 1) occ = 1;
  }
  const uint64_t ntiles = div_up_u64(div_up_u64(n, kAdmGroup), kMap32Warps);
  adm_u32_map_kernel<<<grid_for(ntiles, (uint64_t)cfg.sms * occ), kMap32Threads, sizeof(Map32Smem),
                       s>>>(in, n, m, m_cap, ctrl, flags, epoch, prob_bits);
  return cudaGetLastError();
}

cudaError_t launch_adm_u32_unmap(const uint8_t* m, uint64_t n, uint32_t* out, Ctrl* ctrl,
                                 const LaunchCfg& cfg, cudaStream_t s) {
  static int occ = 0;
  if (occ == 0) {
    cudaOccupancyMaxActiveBlocksPerMultiprocessor(&occ, adm_u32_unmap_kernel, kUnmap32Threads,
                                                  sizeof(Unmap32Smem));
    if (occ < 1) occ = 1;
  }
  const uint64_t groups = div_up_u64(n, kAdmGroup);
  adm_u32_unmap_kernel<<<grid_for(div_up_u64(groups, kUnmap32Warps), (uint64_t)cfg.sms * occ),
                         kUnmap32Threads, sizeof(Unmap32Smem), s>>>(m, n, out, ctrl);
  return cudaGetLastError();
}

}  // namespace mans
