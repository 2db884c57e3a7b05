// batch_internal.h -- device descriptors and launch interface of the batched
// codec (batch.cu). Not part of the public API.
#pragma once

#include <cstdint>
#include <cuda_runtime.h>

#include "mans_internal.h"
#include "../../include/mans.h"

namespace mans {

struct Ctrl;

// One buffer of a batch, built by the host for every call.
struct BatchItem {
  const uint8_t* in;             // compress: values; decompress: stream
  uint8_t* out;                  // compress: stream; decompress: values
  unsigned long long* out_size;  // compress: stream bytes (device, may be null)
  uint64_t n;                    // elements
  uint64_t in_bytes;             // decompress: stream bytes available
  uint64_t out_cap;              // compress: stream capacity
  uint8_t* m;                    // mapped bytes (per-element section 16-byte aligned)
  uint64_t m_cap;
  uint64_t group_base;           // first mapping unit of this buffer in its dtype's unit space
  uint64_t flag_base;            // first look-back flag of this buffer's groups
  uint32_t dtype;                // MANS_U8 / MANS_U16 / MANS_U32
  uint32_t prob_bits;
};

// Per-buffer device state (kept in the batch workspace).
struct BatchState {
  uint2 enc[256];
  uint32_t pdf[256];
  unsigned long long msize;   // mapped bytes (compress) / decoded bytes (decompress)
  unsigned long long detail;  // detail of the buffer's first error
  uint32_t status;            // the buffer's first error (mans_status)
  uint32_t nb;                // rANS blocks
  uint32_t unit_base;         // first global block (compress) / decode chunk (decompress)
  uint32_t n_hdr, cw, p;      // decompress: header fields
};

// Each buffer's histogram is kept in kHistCopies copies (CTA b adds into copy
// b % kHistCopies), which spreads the merge atomics over more L2 slices; the
// plan stage sums them. Copy c of buffer i: hists + (c * hist_items + i) * 256.
constexpr int kHistCopies = 4;

struct BatchDev {
  Ctrl* ctrl;
  BatchItem* items;
  BatchState* states;
  uint32_t* hists;
  uint32_t hist_items;
  unsigned long long* item_flags;
  unsigned long long* group_flags;
  unsigned long long* block_flags;
  uint8_t* slots;
};

enum BatchStage {
  kStageMap = 0,
  kStagePlanEnc,
  kStageEncode,
  kStagePlanDec,
  kStageDecode,
  kStageUnmap,
  kStages
};

// Schedule of the batched kernels. The bytes produced do not depend on it.
//   ctas_per_sm: resident CTAs per SM of each stage (<= occ); for the map
//     stage counted in CTAs of 8 warps, whatever its warps per CTA.
//   warps: warps per CTA (the map stage takes 4 or 8; the others 8).
//   prefetch: L2 prefetch distance of the map and encode stages, in grids of
//     units ahead (0: none; at most kMaxPrefetch).
struct BatchCfg {
  int sms = 148;
  int occ[kStages] = {1, 1, 1, 1, 1, 1};
  int ctas_per_sm[kStages] = {1, 1, 1, 1, 1, 1};
  int warps[kStages] = {8, 8, 8, 8, 8, 8};
  int prefetch[kStages] = {0, 0, 0, 0, 0, 0};
  // occupancy of the lighter map / unmap variants (grids scale with it)
  int occ_u16_map = 1, occ_u8_map = 1, occ_u16_unmap = 1;
  // occupancy of the 4-warp map variants, by dtype kind (u8, u16, u32)
  int occ_map4[3] = {1, 1, 1};
};
constexpr int kMaxPrefetch = 2;

void init_batch_cfg(BatchCfg& c, const LaunchCfg& base);
uint64_t batch_slot_bytes(const BatchCfg& c);
// marks (optional): four events recorded before the first kernel and after
// each stage (compress: map, plan, encode; decompress: plan, decode, unmap).
// groups[k]: mapping units of the buffers of dtype kind k (0: MANS_U8
// histogram chunks, 1: MANS_U16 groups, 2: MANS_U32 groups); each kind has
// its own unit space and its own launch of the map (unmap) stage.
cudaError_t launch_batch_compress(const BatchDev& d, uint32_t count, const uint64_t groups[3],
                                  uint64_t max_blocks, const BatchCfg& c, cudaStream_t s,
                                  cudaEvent_t* marks = nullptr);
cudaError_t launch_batch_decompress(const BatchDev& d, uint32_t count, const uint64_t groups[3],
                                    uint64_t max_chunks, const BatchCfg& c, cudaStream_t s,
                                    cudaEvent_t* marks = nullptr);
cudaError_t launch_batch_gather_status(const BatchDev& d, uint32_t count, uint32_t* status,
                                       unsigned long long* detail, cudaStream_t s);
inline int dtype_kind(uint32_t dtype) { return dtype == 1 ? 0 : dtype == 2 ? 1 : 2; }

}  // namespace mans

namespace mans {
// Enqueue on s: copy the first `count` buffers' statuses and details of the
// batch's last call into host (pinned) arrays. For the serving loop.
mans_status batch_enqueue_status(mans_batch* b, uint32_t count, uint32_t* host_status,
                                 uint64_t* host_detail, cudaStream_t s);
// The same for a single-buffer workspace (one call); also clears its status.
mans_status workspace_enqueue_status(mans_workspace* ws, uint32_t* host_status,
                                     uint64_t* host_detail, cudaStream_t s);
// Worst-case rANS stream bytes of n input bytes.
uint64_t ans_stream_bound(uint64_t n);
}  // namespace mans
