// mans_internal.h -- host-side launch interface between the C-ABI layer and
// the kernel translation units. Not part of the public API.
#pragma once

#include <cstdint>
#include <cuda_runtime.h>

#include <nvtx3/nvToolsExt.h>

namespace mans {

struct Ctrl;

// NVTX range over a host call (free when no tool is attached), so a trace
// shows each codec call beside the kernels it enqueued.
struct NvtxRange {
  explicit NvtxRange(const char* name) { nvtxRangePushA(name); }
  ~NvtxRange() { nvtxRangePop(); }
  NvtxRange(const NvtxRange&) = delete;
  NvtxRange& operator=(const NvtxRange&) = delete;
};

struct LaunchCfg {
  int sms = 148;        // multiprocessors of the device
  int enc_ctas = 0;     // resident CTAs per SM of the encode kernel (shared-memory staging)
  int enc_slot_ctas = 0;  // resident CTAs per SM of the encode kernel (global slots)
  int dec_ctas = 0;     // resident CTAs per SM of the decode kernel
  int map_ctas = 0;     // resident CTAs per SM of the ADM map kernels
  int map32_ctas = 0;   // resident CTAs per SM of the uint32 ADM map kernel
  int unmap32_ctas = 0; // resident CTAs per SM of the uint32 ADM unmap kernel
  int hist_ctas = 0;    // resident CTAs per SM of the byte histogram kernel
};

// Query occupancy once per device.
void init_launch_cfg(LaunchCfg& cfg, int device);

// ---- rANS over bytes (ans_codec.cu) ----
// Histogram of n raw bytes + normalisation into ctrl (table, pdf, merged_size = n).
cudaError_t launch_hist_bytes(const uint8_t* in, uint64_t n, Ctrl* ctrl, int prob_bits,
                              const LaunchCfg& cfg, cudaStream_t s);
// Encode ctrl->merged_size bytes at `in` (table from ctrl) into the coalesced
// stream at `out`. max_blocks bounds the number of 4 KiB blocks (grid size).
// slots: ans_encode_slot_bytes(cfg) bytes of global scratch for the words of
// blocks in flight, or nullptr to compact them in shared memory instead.
cudaError_t launch_ans_encode(const uint8_t* in, uint8_t* out, uint64_t out_cap,
                              unsigned long long* out_size64, uint32_t* out_size32, Ctrl* ctrl,
                              unsigned long long* flags, int prob_bits, uint64_t max_blocks,
                              const LaunchCfg& cfg, cudaStream_t s, uint8_t* slots);
uint64_t ans_encode_slot_bytes(const LaunchCfg& cfg);
// Decode the stream at `in` into `out` (at most out_cap bytes). expect_p < 0
// accepts any valid precision. record != 0 stores the decoded size in ctrl.
cudaError_t launch_ans_decode(const uint8_t* in, uint64_t in_size, uint8_t* out, uint64_t out_cap,
                              Ctrl* ctrl, int expect_p, int record, uint64_t max_blocks,
                              const LaunchCfg& cfg, cudaStream_t s);

// ---- ADM uint16 (adm_u16.cu) ----
// Map n values into the merged buffer M (16-byte aligned codes section),
// histogram it and normalise (ctrl). flags: >= ceil(n/4096) entries.
// layout: 0 V15 (canonical), 1 V12, 2 CPU-V2 (see adm_u16.cuh).
cudaError_t launch_adm_u16_map(const uint16_t* in, uint64_t n, uint8_t* m, uint64_t m_cap,
                               Ctrl* ctrl, unsigned long long* flags, int prob_bits,
                               const LaunchCfg& cfg, cudaStream_t s, int layout = 0);
// V12: v12_excl (>= ceil(n/512) u32) receives the group offsets and
// scan_flags (>= ceil(n/2^20) + 1 entries) serves the scan's look-back.
cudaError_t launch_adm_u16_unmap(const uint8_t* m, uint64_t n, uint16_t* out, Ctrl* ctrl,
                                 const LaunchCfg& cfg, cudaStream_t s, int layout = 0,
                                 uint32_t* v12_excl = nullptr,
                                 unsigned long long* scan_flags = nullptr);

// ---- ADM uint32 (adm_u32.cu) ----
cudaError_t launch_adm_u32_map(const uint32_t* in, uint64_t n, uint8_t* m, uint64_t m_cap,
                               Ctrl* ctrl, unsigned long long* flags, int prob_bits,
                               const LaunchCfg& cfg, cudaStream_t s);
cudaError_t launch_adm_u32_unmap(const uint8_t* m, uint64_t n, uint32_t* out, Ctrl* ctrl,
                                 const LaunchCfg& cfg, cudaStream_t s);

// Byte offset of the merged buffer inside its 16-byte aligned region so that
// the per-element section (codes / records) is 16-byte aligned.
inline uint64_t merged_pad(uint64_t header_bytes) { return (16 - (header_bytes & 15)) & 15; }
inline uint64_t adm_u16_header_bytes(uint64_t n, int layout = 0) {
  const uint64_t g = (n + 511) / 512;
  return layout == 1 ? 4 * g : layout == 2 ? 6 * g + 4 : 6 * g;
}
inline uint64_t adm_u32_header_bytes(uint64_t n) { return 40 * ((n + 511) / 512); }

}  // namespace mans
