// mans_device.cuh -- format constants and device helpers shared by the MANS
// kernels (sm_100a).
//
// Format constants restate include/ans/GpuANSCodec.h:18-61 (rANS stream) and
// mapping/nv/mappingV15_fused_uint16.cu:16-20 (ADM groups); they are fixed by
// the stream layout and may not change.
#pragma once

#include <cstdint>
#include <cuda_runtime.h>

#include "../../include/mans.h"

namespace mans {

// ---- rANS stream (GpuANSCodec.h) ----
constexpr int kWarp = 32;
constexpr uint32_t kAnsBlock = 4096;          // kDefaultBlockSize
constexpr int kAnsSyms = 256;                 // kNumSymbols
constexpr int kAnsStateBits = 31;             // kANSStateBits
constexpr uint32_t kAnsStartState = 1u << 15; // kANSStartState == kANSMinState
constexpr uint32_t kAnsMagicVersion = (0xd00du << 16) | 0x0001u;
constexpr uint32_t kAnsHeaderBytes = 32;      // sizeof(ANSCoalescedHeader)
constexpr uint32_t kAnsStepsPerBlock = kAnsBlock / kWarp;  // 128
// Worst case words of one block: 32 lanes x (128 symbols x 11 bits / 16 + 1).
constexpr uint32_t kAnsMaxBlockWords = 32 * 90;

__host__ __device__ constexpr uint64_t ans_overhead(uint64_t nb) {
  return kAnsHeaderBytes + 2 * kAnsSyms + 128 * nb + 8 * ((nb + 1) / 2 * 2);
}

// ---- ADM groups (mappingV15_fused_uint16.cu, mappingV9_fuse.cu) ----
constexpr int kAdmChunk = 16;     // elements per lane
constexpr int kAdmGroup = 512;    // elements per group (one warp)
constexpr uint32_t kAdmStep = 126;
// Longest uint16 lane stream in bytes: 16 elements of at most
// ceil(65535 / 126) = 521 bits each.
constexpr uint64_t kU16MaxLaneBytes = (kAdmChunk * 521 + 7) / 8;  // 1,042
constexpr int kAdmGroupsPerTile = 8;  // warps (groups in flight) per CTA of the mappers
// uint16 groups per unit of the map's claims and look-back (a uint16 group is
// 1 KiB of input; two halve the per-byte cost of claims and look-backs).
constexpr uint32_t kU16MapUnit = 2;

// ---- device status (first error wins) ----
struct Ctrl {
  uint32_t status;        // mans_status of the first device-side error
  uint32_t pad0;
  unsigned long long detail;  // e.g. bytes needed
  uint32_t tile_counter[8];   // dynamic work counters, reset by the last CTA
  uint32_t done_counter[8];   // CTA completion counters, reset by the last CTA
  uint32_t hist[kAnsSyms];    // histogram of the merged bytes
  uint2 enc_table[kAnsSyms];  // {reciprocal, shift | bias << 5 | cmpl << 20}
  uint32_t pdf[kAnsSyms];
  unsigned long long merged_size;  // merged bytes of the current call
  uint32_t total_words;
  // Look-back epoch of the current call: read by every kernel of a compress,
  // advanced by the last CTA of its final kernel, so a call needs no host
  // bookkeeping and a captured CUDA graph stays correct across replays.
  uint32_t epoch;
};

__device__ __forceinline__ void report_error(Ctrl* c, uint32_t code, unsigned long long detail) {
  if (atomicCAS(&c->status, 0u, code) == 0u) c->detail = detail;
}

// Where device-side errors of one unit of work go: the call's control block
// and, in a batch, the buffer's own status (first error wins in each).
struct Sink {
  uint32_t* status;
  unsigned long long* detail;
  uint32_t* item_status;
  unsigned long long* item_detail;
};
__device__ __forceinline__ Sink sink_of(Ctrl* c) {
  return Sink{&c->status, &c->detail, nullptr, nullptr};
}
__device__ __forceinline__ void report(const Sink& s, uint32_t code, unsigned long long detail) {
  if (atomicCAS(s.status, 0u, code) == 0u) *s.detail = detail;
  if (s.item_status && atomicCAS(s.item_status, 0u, code) == 0u) *s.item_detail = detail;
}
__device__ __forceinline__ bool sink_failed(const Sink& s) {
  return *((volatile uint32_t*)s.status) != 0;
}

__device__ __forceinline__ int lane_id() {
  int l;
  asm("mov.u32 %0, %%laneid;" : "=r"(l));
  return l;
}
__device__ __forceinline__ uint32_t lanemask_lt() {
  uint32_t m;
  asm("mov.u32 %0, %%lanemask_lt;" : "=r"(m));
  return m;
}
__device__ __forceinline__ uint32_t lanemask_ge() {
  uint32_t m;
  asm("mov.u32 %0, %%lanemask_ge;" : "=r"(m));
  return m;
}

// Look-back flags carry their own value, so they need coherence but no
// ordering with other memory: relaxed GPU-scope accesses, no fences.
__device__ __forceinline__ unsigned long long ld_flag(const unsigned long long* p) {
  unsigned long long v;
  asm volatile("ld.relaxed.gpu.global.u64 %0, [%1];" : "=l"(v) : "l"(p) : "memory");
  return v;
}
__device__ __forceinline__ void st_flag(unsigned long long* p, unsigned long long v) {
  asm volatile("st.relaxed.gpu.global.u64 [%0], %1;" ::"l"(p), "l"(v) : "memory");
}

// Prefetch one 128-byte line into L1.
__device__ __forceinline__ void prefetch_l1(const void* p) {
  asm volatile("prefetch.global.L1 [%0];" ::"l"(p));
}

// Prefetch [p, p+bytes) into L2 with one bulk request (p and bytes are
// rounded out to 16-byte boundaries; the range must lie in one allocation).
__device__ __forceinline__ void prefetch_l2(const void* p, uint32_t bytes) {
  const uintptr_t a0 = reinterpret_cast<uintptr_t>(p) & ~uintptr_t(15);
  const uintptr_t a1 = (reinterpret_cast<uintptr_t>(p) + bytes + 15) & ~uintptr_t(15);
  if (a1 > a0)
    asm volatile("cp.async.bulk.prefetch.L2.global [%0], %1;" ::"l"(a0), "r"((uint32_t)(a1 - a0))
                 : "memory");
}

// ---- bulk (TMA) copies global -> shared with mbarrier completion ----
// One mbarrier per warp-owned staging buffer, arrival count 1 (the issuing
// lane). No multicast: each copy lands in the issuing CTA only.
__device__ __forceinline__ uint32_t smem_addr(const void* p) {
  return (uint32_t)__cvta_generic_to_shared(p);
}
__device__ __forceinline__ void mbar_init(uint64_t* bar) {
  asm volatile("mbarrier.init.shared::cta.b64 [%0], 1;" ::"r"(smem_addr(bar)) : "memory");
  asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
}
// Issued by one lane: copy `bytes` (multiple of 16; both addresses 16-byte
// aligned) and arm the barrier's transaction count.
__device__ __forceinline__ void bulk_load(void* smem_dst, const void* gmem_src, uint32_t bytes,
                                          uint64_t* bar) {
  asm volatile("fence.proxy.async.shared::cta;" ::: "memory");
  asm volatile("mbarrier.arrive.expect_tx.shared::cta.b64 _, [%0], %1;" ::"r"(smem_addr(bar)),
               "r"(bytes)
               : "memory");
  asm volatile(
      "cp.async.bulk.shared::cluster.global.mbarrier::complete_tx::bytes [%0], [%1], %2, [%3];" ::"r"(
          smem_addr(smem_dst)),
      "l"(gmem_src), "r"(bytes), "r"(smem_addr(bar))
      : "memory");
}
// Bounded wait for the phase with the given parity to complete. Returns false
// after 2^20 polls (each try_wait may suspend briefly; about a second at
// most) and the caller records MANS_ERR_TIMEOUT.
__device__ __forceinline__ bool mbar_wait(uint64_t* bar, uint32_t parity) {
  const uint32_t a = smem_addr(bar);
  for (uint32_t i = 0; i < (1u << 20); ++i) {
    uint32_t done;
    asm volatile(
        "{\n .reg .pred p;\n mbarrier.try_wait.parity.shared::cta.b64 p, [%1], %2;\n"
        " selp.u32 %0, 1, 0, p;\n}\n"
        : "=r"(done)
        : "r"(a), "r"(parity)
        : "memory");
    if (done) return true;
  }
  return false;
}

// ---- single-pass decoupled look-back (epoch tagged, bounded waits) ----
// A flag word packs {value:32}{epoch:30}{state:2}; state 1 = aggregate
// published, 2 = inclusive prefix published. Flags from an older call carry
// an older epoch and read as "not ready", so the arrays never need clearing.
constexpr uint32_t kFlagAgg = 1, kFlagIncl = 2;
__device__ __forceinline__ unsigned long long make_flag(uint32_t state, uint32_t epoch,
                                                        uint32_t value) {
  return ((unsigned long long)value << 32) | ((unsigned long long)(epoch & 0x3fffffffu) << 2) |
         state;
}
// Bounded spin: about one second at most (2^22 polls x ~0.25 us backoff).
constexpr uint32_t kSpinLimit = 1u << 22;

// Warp-cooperative exclusive prefix of `tile` over flags[0..tile). Every lane
// returns the same value. On timeout reports MANS_ERR_TIMEOUT and returns the
// partial sum (the call's output is then invalid, but the kernel finishes).
__device__ __forceinline__ uint32_t lookback_exclusive(unsigned long long* flags, uint32_t tile,
                                                       uint32_t epoch, const Sink& sink) {
  const int lane = lane_id();
  uint32_t excl = 0;
  int64_t base = (int64_t)tile - 1;
  const uint32_t ep = epoch & 0x3fffffffu;
  while (base >= 0) {
    int64_t idx = base - lane;
    unsigned long long w = 0;
    uint32_t st = kFlagIncl, val = 0;
    if (idx >= 0) {
      uint32_t spins = 0, ns = 32;
      while (true) {
        w = ld_flag(&flags[idx]);
        st = (uint32_t)(w & 3u);
        uint32_t wep = (uint32_t)((w >> 2) & 0x3fffffffu);
        if (st != 0 && wep == ep) break;
        ++spins;
        // Give up after the bound, or at once when another waiter already
        // recorded an error (so one expired wait does not multiply).
        if (spins > kSpinLimit ||
            ((spins & 63u) == 0 && *((volatile uint32_t*)sink.status) == MANS_ERR_TIMEOUT)) {
          report(sink, MANS_ERR_TIMEOUT, tile);
          st = kFlagIncl;
          w = 0;
          break;
        }
        __nanosleep(ns);
        if (ns < 256) ns <<= 1;
      }
      val = (uint32_t)(w >> 32);
    }
    uint32_t incl_mask = __ballot_sync(0xffffffffu, st == kFlagIncl);
    if (incl_mask) {
      int first = __ffs(incl_mask) - 1;  // nearest predecessor with a full prefix
      uint32_t v = lane <= first ? val : 0u;
      excl += __reduce_add_sync(0xffffffffu, v);
      break;
    }
    excl += __reduce_add_sync(0xffffffffu, val);
    base -= kWarp;
  }
  return excl;
}

__device__ __forceinline__ uint32_t warp_claim(uint32_t* counter, int lane) {
  uint32_t v = 0;
  if (lane == 0) v = atomicAdd(counter, 1u);
  return __shfl_sync(0xffffffffu, v, 0);
}

__host__ __device__ inline uint64_t div_up_u64(uint64_t a, uint64_t b) { return (a + b - 1) / b; }
__host__ __device__ inline uint64_t min_u64(uint64_t a, uint64_t b) { return a < b ? a : b; }

}  // namespace mans
