// smem_io.cuh -- warp-cooperative copies between global memory at arbitrary
// byte alignment and shared-memory staging buffers.
//
// A staging buffer holds byte i of a global range [g, g+n) at
// stage[(g & 15) + i]: global and shared addresses then share their phase
// modulo 16, so the interior moves as aligned 16-byte vectors and only the
// head and tail are moved as bytes. Staging buffers are 16-byte aligned and
// hold n + 16 bytes.
#pragma once

#include <cstdint>

namespace mans {

__device__ __forceinline__ uint32_t phase16(const void* p) {
  return (uint32_t)(reinterpret_cast<uintptr_t>(p) & 15u);
}

// Load global bytes [src, src+n) into stage (phase-matched). Reads the whole
// 16-byte aligned chunks that overlap the range (never crossing a page, so
// never faulting on a valid buffer). Caller synchronises the warp afterwards.
__device__ __forceinline__ void warp_load_phase(uint8_t* __restrict__ stage,
                                                const uint8_t* __restrict__ src, uint32_t n,
                                                int lane) {
  if (n == 0) return;
  const uintptr_t a0 = reinterpret_cast<uintptr_t>(src) & ~uintptr_t(15);
  const uintptr_t a1 = (reinterpret_cast<uintptr_t>(src) + n + 15) & ~uintptr_t(15);
  const uint32_t chunks = (uint32_t)((a1 - a0) >> 4);
  const uint4* g = reinterpret_cast<const uint4*>(a0);
  uint4* s = reinterpret_cast<uint4*>(stage);
  for (uint32_t i = lane; i < chunks; i += 32) s[i] = __ldg(g + i);
}

// Store stage bytes (phase-matched) to global [dst, dst+n). Bytes outside
// the range are never written, so neighbouring ranges owned by other warps
// are safe.
__device__ __forceinline__ void warp_store_phase(uint8_t* __restrict__ dst,
                                                 const uint8_t* __restrict__ stage, uint32_t n,
                                                 int lane) {
  if (n == 0) return;
  const uint32_t ph = phase16(dst);
  uint32_t head = (16u - ph) & 15u;
  if (head > n) head = n;
  if ((uint32_t)lane < head) dst[lane] = stage[ph + lane];
  const uint32_t body = (n - head) >> 4;
  uint4* gd = reinterpret_cast<uint4*>(dst + head);
  const uint4* sd = reinterpret_cast<const uint4*>(stage + ph + head);
  for (uint32_t i = lane; i < body; i += 32) gd[i] = sd[i];
  const uint32_t tail0 = head + (body << 4);
  const uint32_t tail = n - tail0;
  if ((uint32_t)lane < tail) dst[tail0 + lane] = stage[ph + tail0 + lane];
}

}  // namespace mans
