// mans_capi.cu -- the C ABI of libmans_b200.so (declared in include/mans.h):
// workspaces, argument checks, kernel dispatch and the reference-compatible
// rANS entry points.
#include <cstring>
#include <map>
#include <memory>
#include <mutex>
#include <new>
#include <utility>

#include "ans_table.cuh"
#include "mans_device.cuh"
#include "mans_internal.h"

namespace mans {
void init_ans_launch_cfg(LaunchCfg& cfg);
void init_adm_u16_launch_cfg(LaunchCfg& cfg);
void init_adm_u32_launch_cfg(LaunchCfg& cfg);

void init_launch_cfg(LaunchCfg& cfg, int device) {
  int sms = 0;
  cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, device);
  cfg.sms = sms > 0 ? sms : 148;
  init_ans_launch_cfg(cfg);
  init_adm_u16_launch_cfg(cfg);
  init_adm_u32_launch_cfg(cfg);
}
}  // namespace mans

using namespace mans;

struct mans_workspace {
  int device = 0;
  uint64_t max_input_bytes = 0;
  uint64_t merged_cap = 0;
  uint8_t* base = nullptr;
  uint64_t bytes = 0;
  Ctrl* ctrl = nullptr;
  unsigned long long* adm_flags = nullptr;
  uint64_t adm_flags_n = 0;
  unsigned long long* ans_flags = nullptr;
  uint64_t ans_flags_n = 0;
  uint8_t* merged = nullptr;  // 16-byte aligned region of merged_cap + slack bytes
  uint8_t* enc_slots = nullptr;  // per-warp word slots of the encode kernel
  uint32_t* v12_excl = nullptr;  // group offsets of the V12 layout's unmap
  LaunchCfg cfg;
  // Opt-in kernel timing: a ring of event triples per recorded call
  // (compress: start, after mapping, after encode; decompress: start, after
  // decode, after unmapping), read and cleared by mans_workspace_kernel_times.
  static constexpr int kRing = 128;
  bool timing = false;
  cudaEvent_t ev_c[kRing][3] = {};
  cudaEvent_t ev_d[kRing][3] = {};
  int nc = 0, nd = 0;  // recorded calls since the last read
};

namespace {

// i: 0..2 compress marks, 3..5 decompress marks. A call is recorded only
// while its ring has room (the slot is claimed at the call's first mark).
inline void mark(mans_workspace* ws, int i, cudaStream_t s) {
  if (!ws->timing) return;
  if (i < 3) {
    if (i == 0) {
      if (ws->nc >= mans_workspace::kRing) return;
      ++ws->nc;
    } else if (ws->nc == 0) {
      return;
    }
    cudaEventRecord(ws->ev_c[ws->nc - 1][i], s);
  } else {
    if (i == 3) {
      if (ws->nd >= mans_workspace::kRing) return;
      ++ws->nd;
    } else if (ws->nd == 0) {
      return;
    }
    cudaEventRecord(ws->ev_d[ws->nd - 1][i - 3], s);
  }
}

constexpr uint64_t kMaxMerged = 0xfffffff0ull;  // rANS header counts are u32
constexpr uint64_t kSlack = 256;

inline bool aligned16(const void* p) { return (reinterpret_cast<uintptr_t>(p) & 15u) == 0; }
inline uint64_t align_up(uint64_t v, uint64_t a) { return (v + a - 1) / a * a; }

uint64_t elem_bytes(mans_dtype d) {
  switch (d) {
    case MANS_U8: return 1;
    case MANS_U16: return 2;
    case MANS_U32: return 4;
  }
  return 0;
}

bool valid_precision(int p) { return p >= 9 && p <= 11; }

// Worst-case rANS stream for n bytes: 32 lanes x 90 words per 4 KiB block.
uint64_t ans_bound(uint64_t n) {
  const uint64_t nb = div_up_u64(n, kAnsBlock);
  return ans_overhead(nb) + nb * (uint64_t)kAnsMaxBlockWords * 2;
}

}  // namespace

namespace mans {
// Enqueue on s: copy the workspace's device status and detail into host
// (pinned) memory, then clear them for the next call. For the serving loop.
mans_status workspace_enqueue_status(mans_workspace* ws, uint32_t* host_status,
                                     uint64_t* host_detail, cudaStream_t s) {
  if (!ws) return MANS_ERR_INVALID_ARG;
  if (cudaMemcpyAsync(host_status, &ws->ctrl->status, 4, cudaMemcpyDeviceToHost, s) != cudaSuccess ||
      cudaMemcpyAsync(host_detail, &ws->ctrl->detail, 8, cudaMemcpyDeviceToHost, s) != cudaSuccess ||
      cudaMemsetAsync(&ws->ctrl->status, 0, 4, s) != cudaSuccess ||
      cudaMemsetAsync(&ws->ctrl->detail, 0, 8, s) != cudaSuccess)
    return MANS_ERR_CUDA;
  return MANS_OK;
}
uint64_t ans_stream_bound(uint64_t n) { return ans_bound(n); }
}  // namespace mans

namespace {

// Copy the mapped bytes (size in ctrl) out of the workspace, with a capacity
// check; thread 0 stores the size. It ends a map-only call, so it also
// advances the look-back epoch (in a compress the encoder does), which the
// mapping kernels before it have read: the next call's flags then never
// match this call's.
__global__ void export_merged_kernel(const uint8_t* __restrict__ src, uint8_t* __restrict__ dst,
                                     uint64_t cap, Ctrl* ctrl, unsigned long long* out_size) {
  if (blockIdx.x == 0 && threadIdx.x == 0) ctrl->epoch = (ctrl->epoch + 1) & 0x3fffffffu;
  if (*((volatile uint32_t*)&ctrl->status) != 0) return;
  const uint64_t n = __ldcg(&ctrl->merged_size);
  if (n > cap) {
    if (blockIdx.x == 0 && threadIdx.x == 0) report_error(ctrl, MANS_ERR_OUTPUT_OVERFLOW, n);
    return;
  }
  for (uint64_t i = (uint64_t)blockIdx.x * blockDim.x + threadIdx.x; i < n;
       i += (uint64_t)gridDim.x * blockDim.x)
    dst[i] = src[i];
  if (blockIdx.x == 0 && threadIdx.x == 0 && out_size) *out_size = n;
}

// Copy caller-supplied mapped bytes into the workspace and record their size.
__global__ void import_merged_kernel(const uint8_t* __restrict__ src, uint8_t* __restrict__ dst,
                                     uint64_t n, Ctrl* ctrl) {
  for (uint64_t i = (uint64_t)blockIdx.x * blockDim.x + threadIdx.x; i < n;
       i += (uint64_t)gridDim.x * blockDim.x)
    dst[i] = src[i];
  if (blockIdx.x == 0 && threadIdx.x == 0) ctrl->merged_size = n;
}

// One warp waits for the prefix of unit 4 over flags that nothing
// publishes: the bounded wait must run out and record MANS_ERR_TIMEOUT.
__global__ void debug_wait_kernel(unsigned long long* flags, Ctrl* ctrl) {
  lookback_exclusive(flags, 4, 1u, sink_of(ctrl));
}

unsigned copy_grid(const LaunchCfg& cfg, uint64_t n) {
  const uint64_t want = div_up_u64(n, 256 * 16);
  const uint64_t cap = (uint64_t)cfg.sms * 8;
  return (unsigned)(want < 1 ? 1 : (want < cap ? want : cap));
}

bool valid_layout(mans_dtype dtype, mans_layout layout) {
  if (layout == MANS_LAYOUT_NATIVE) return true;
  return dtype == MANS_U16 && (layout == MANS_LAYOUT_V12 || layout == MANS_LAYOUT_CPUV2);
}

mans_status compress_impl(mans_workspace* ws, mans_dtype dtype, mans_layout layout,
                          const void* d_in, uint64_t n_elems, void* d_out, uint64_t out_capacity,
                          uint64_t* d_out_size, int precision, mans_stream_t stream,
                          bool map_only) {
  NvtxRange range(map_only ? "mans_adm_map" : "mans_compress");
  if (!ws || !d_out || !d_out_size || (!d_in && n_elems)) return MANS_ERR_INVALID_ARG;
  const uint64_t eb = elem_bytes(dtype);
  if (eb == 0 || !valid_layout(dtype, layout)) return MANS_ERR_INVALID_ARG;
  if (!valid_precision(precision)) return MANS_ERR_UNSUPPORTED_PRECISION;
  if ((d_in && !aligned16(d_in)) || !aligned16(d_out)) return MANS_ERR_ALIGNMENT;
  const uint64_t in_bytes = n_elems * eb;
  if (in_bytes > ws->max_input_bytes) return MANS_ERR_TOO_LARGE;
  cudaStream_t s = reinterpret_cast<cudaStream_t>(stream);
  unsigned long long* osz = reinterpret_cast<unsigned long long*>(d_out_size);
  cudaError_t e = cudaSuccess;
  if (dtype == MANS_U8 && in_bytes > kMaxMerged) return MANS_ERR_TOO_LARGE;
  uint8_t* m = nullptr;
  mark(ws, 0, s);
  if (dtype == MANS_U8) {
    e = launch_hist_bytes((const uint8_t*)d_in, in_bytes, ws->ctrl, precision, ws->cfg, s);
    mark(ws, 1, s);
    if (e == cudaSuccess)
      e = launch_ans_encode((const uint8_t*)d_in, (uint8_t*)d_out, out_capacity, osz, nullptr,
                            ws->ctrl, ws->ans_flags, precision,
                            div_up_u64(in_bytes, kAnsBlock), ws->cfg, s, ws->enc_slots);
    mark(ws, 2, s);
    return e == cudaSuccess ? MANS_OK : MANS_ERR_CUDA;
  }
  if (dtype == MANS_U16) {
    const uint64_t hdr = adm_u16_header_bytes(n_elems, (int)layout);
    const uint64_t g = div_up_u64(n_elems, kAdmGroup);
    if (hdr + n_elems + 32 * g > ws->merged_cap) return MANS_ERR_TOO_LARGE;
    m = ws->merged + merged_pad(hdr);
    e = launch_adm_u16_map((const uint16_t*)d_in, n_elems, m, ws->merged_cap, ws->ctrl,
                           ws->adm_flags, precision, ws->cfg, s, (int)layout);
  } else {
    const uint64_t hdr = adm_u32_header_bytes(n_elems);
    if (hdr + n_elems > ws->merged_cap) return MANS_ERR_TOO_LARGE;
    m = ws->merged + merged_pad(hdr);
    e = launch_adm_u32_map((const uint32_t*)d_in, n_elems, m, ws->merged_cap, ws->ctrl,
                           ws->adm_flags, precision, ws->cfg, s);
  }
  mark(ws, 1, s);
  if (e == cudaSuccess) {
    if (map_only) {
      export_merged_kernel<<<copy_grid(ws->cfg, ws->merged_cap), 256, 0, s>>>(
          m, (uint8_t*)d_out, out_capacity, ws->ctrl, osz);
      e = cudaGetLastError();
    } else {
      e = launch_ans_encode(m, (uint8_t*)d_out, out_capacity, osz, nullptr, ws->ctrl,
                            ws->ans_flags, precision, div_up_u64(ws->merged_cap, kAnsBlock),
                            ws->cfg, s, ws->enc_slots);
    }
  }
  mark(ws, 2, s);
  return e == cudaSuccess ? MANS_OK : MANS_ERR_CUDA;
}

mans_status decompress_impl(mans_workspace* ws, mans_dtype dtype, mans_layout layout,
                            const void* d_in, uint64_t in_size, void* d_out, uint64_t n_elems,
                            mans_stream_t stream, bool unmap_only) {
  NvtxRange range(unmap_only ? "mans_adm_unmap" : "mans_decompress");
  // an empty mapped buffer (n = 0) may come without a pointer
  if (!ws || (!d_in && !(unmap_only && in_size == 0)) || (!d_out && n_elems))
    return MANS_ERR_INVALID_ARG;
  const uint64_t eb = elem_bytes(dtype);
  if (eb == 0 || !valid_layout(dtype, layout)) return MANS_ERR_INVALID_ARG;
  if ((d_in && !aligned16(d_in)) || (d_out && !aligned16(d_out))) return MANS_ERR_ALIGNMENT;
  const uint64_t out_bytes = n_elems * eb;
  if (out_bytes > ws->max_input_bytes) return MANS_ERR_TOO_LARGE;
  cudaStream_t s = reinterpret_cast<cudaStream_t>(stream);
  cudaError_t e = cudaSuccess;
  mark(ws, 3, s);
  if (dtype == MANS_U8) {
    e = launch_ans_decode((const uint8_t*)d_in, in_size, (uint8_t*)d_out, out_bytes, ws->ctrl, -1,
                          0, div_up_u64(out_bytes, kAnsBlock), ws->cfg, s);
    mark(ws, 4, s);
    mark(ws, 5, s);
    return e == cudaSuccess ? MANS_OK : MANS_ERR_CUDA;
  }
  const uint64_t hdr = dtype == MANS_U16 ? adm_u16_header_bytes(n_elems, (int)layout)
                                         : adm_u32_header_bytes(n_elems);
  uint8_t* m = ws->merged + merged_pad(hdr);
  if (unmap_only) {
    if (in_size > ws->merged_cap) return MANS_ERR_TOO_LARGE;
    import_merged_kernel<<<copy_grid(ws->cfg, in_size), 256, 0, s>>>((const uint8_t*)d_in, m,
                                                                      in_size, ws->ctrl);
    e = cudaGetLastError();
  } else {
    e = launch_ans_decode((const uint8_t*)d_in, in_size, m, ws->merged_cap, ws->ctrl, -1, 1,
                          div_up_u64(ws->merged_cap, kAnsBlock), ws->cfg, s);
  }
  mark(ws, 4, s);
  if (e == cudaSuccess) {
    if (dtype == MANS_U16)
      e = launch_adm_u16_unmap(m, n_elems, (uint16_t*)d_out, ws->ctrl, ws->cfg, s, (int)layout,
                               ws->v12_excl, ws->ans_flags);
    else
      e = launch_adm_u32_unmap(m, n_elems, (uint32_t*)d_out, ws->ctrl, ws->cfg, s);
  }
  mark(ws, 5, s);
  return e == cudaSuccess ? MANS_OK : MANS_ERR_CUDA;
}

}  // namespace

extern "C" {

const char* mans_version(void) { return "mans_b200 0.1.0 (sm_100a)"; }

mans_status mans_workspace_create(mans_workspace** out, uint64_t max_input_bytes,
                                  uint64_t merged_capacity) {
  if (!out) return MANS_ERR_INVALID_ARG;
  *out = nullptr;
  if (merged_capacity == 0) merged_capacity = max_input_bytes / 10 * 21 + 4096;
  if (merged_capacity > kMaxMerged) merged_capacity = kMaxMerged;
  auto* ws = new (std::nothrow) mans_workspace();
  if (!ws) return MANS_ERR_OUT_OF_MEMORY;
  if (cudaGetDevice(&ws->device) != cudaSuccess) {
    delete ws;
    return MANS_ERR_CUDA;
  }
  ws->max_input_bytes = max_input_bytes;
  ws->merged_cap = merged_capacity;
  // one flag per ADM group (512 elements, >= 1 KiB of input) and per 4 KiB rANS block
  ws->adm_flags_n = max_input_bytes / 1024 + 2;
  uint64_t ans_src = merged_capacity > max_input_bytes ? merged_capacity : max_input_bytes;
  ws->ans_flags_n = div_up_u64(ans_src, kAnsBlock) + 2;
  init_launch_cfg(ws->cfg, ws->device);
  const uint64_t off_ctrl = 0;
  const uint64_t off_adm = align_up(sizeof(Ctrl), 256);
  const uint64_t off_ans = align_up(off_adm + 8 * ws->adm_flags_n, 256);
  const uint64_t off_slots = align_up(off_ans + 8 * ws->ans_flags_n, 256);
  const uint64_t off_v12 = align_up(off_slots + ans_encode_slot_bytes(ws->cfg), 256);
  const uint64_t off_m = align_up(off_v12 + 4 * ws->adm_flags_n, 256);
  ws->bytes = align_up(off_m + merged_capacity + kSlack, 256);
  if (cudaMalloc(&ws->base, ws->bytes) != cudaSuccess) {
    cudaGetLastError();
    delete ws;
    return MANS_ERR_OUT_OF_MEMORY;
  }
  if (cudaMemset(ws->base, 0, off_slots) != cudaSuccess) {
    cudaFree(ws->base);
    delete ws;
    return MANS_ERR_CUDA;
  }
  ws->ctrl = reinterpret_cast<Ctrl*>(ws->base + off_ctrl);
  ws->adm_flags = reinterpret_cast<unsigned long long*>(ws->base + off_adm);
  ws->ans_flags = reinterpret_cast<unsigned long long*>(ws->base + off_ans);
  ws->enc_slots = ws->base + off_slots;
  ws->v12_excl = reinterpret_cast<uint32_t*>(ws->base + off_v12);
  ws->merged = ws->base + off_m;
  *out = ws;
  return MANS_OK;
}

mans_status mans_workspace_destroy(mans_workspace* ws) {
  if (!ws) return MANS_ERR_INVALID_ARG;
  int prev = 0;
  cudaGetDevice(&prev);
  cudaSetDevice(ws->device);
  for (auto& row : ws->ev_c)
    for (auto& ev : row)
      if (ev) cudaEventDestroy(ev);
  for (auto& row : ws->ev_d)
    for (auto& ev : row)
      if (ev) cudaEventDestroy(ev);
  cudaError_t e = cudaFree(ws->base);
  cudaSetDevice(prev);
  delete ws;
  return e == cudaSuccess ? MANS_OK : MANS_ERR_CUDA;
}

uint64_t mans_workspace_device_bytes(const mans_workspace* ws) { return ws ? ws->bytes : 0; }

mans_status mans_workspace_status(mans_workspace* ws, mans_stream_t stream, uint64_t* detail) {
  if (!ws) return MANS_ERR_INVALID_ARG;
  cudaStream_t s = reinterpret_cast<cudaStream_t>(stream);
  if (cudaStreamSynchronize(s) != cudaSuccess) return MANS_ERR_CUDA;
  struct {
    uint32_t status, pad;
    unsigned long long detail;
  } h = {0, 0, 0};
  if (cudaMemcpy(&h, ws->ctrl, sizeof(h), cudaMemcpyDeviceToHost) != cudaSuccess)
    return MANS_ERR_CUDA;
  if (detail) *detail = h.detail;
  if (h.status != 0) {
    decltype(h) z = {0, 0, 0};
    if (cudaMemcpy(ws->ctrl, &z, sizeof(z), cudaMemcpyHostToDevice) != cudaSuccess)
      return MANS_ERR_CUDA;
  }
  return (mans_status)h.status;
}

uint64_t mans_max_mapped_size(mans_dtype dtype, uint64_t n_elems) {
  // Beyond 2^40 elements every sum below could wrap; no such buffer exists.
  if (elem_bytes(dtype) == 0 || n_elems > (1ull << 40)) return 0;
  const uint64_t g = div_up_u64(n_elems, kAdmGroup);
  switch (dtype) {
    case MANS_U8: return n_elems;
    case MANS_U16:
      // lanes of at most 16 x 521 bits = 1,042 bytes, 32 lanes per group;
      // codes; the largest header (CPU-V2: 6 bytes per group + 4)
      return g * (32ull * kU16MaxLaneBytes + 6) + 4 + n_elems;
    case MANS_U32:
      // at most 8 record bytes per element; 40 header bytes per group
      return 40 * g + 8 * n_elems;
  }
  return 0;
}

uint64_t mans_stream_bound(uint64_t mapped_bytes) { return ans_bound(mapped_bytes); }

uint64_t mans_max_compressed_size(mans_dtype dtype, uint64_t n_elems) {
  const uint64_t eb = elem_bytes(dtype);
  if (eb == 0) return 0;
  if (dtype == MANS_U8) return ans_bound(n_elems);
  const uint64_t merged = mans_max_mapped_size(dtype, n_elems);
  return ans_bound(merged < kMaxMerged ? merged : kMaxMerged);
}

mans_status mans_compress(mans_workspace* ws, mans_dtype dtype, const void* d_in,
                          uint64_t n_elems, void* d_out, uint64_t out_capacity,
                          uint64_t* d_out_size, int precision, mans_stream_t stream) {
  return compress_impl(ws, dtype, MANS_LAYOUT_NATIVE, d_in, n_elems, d_out, out_capacity,
                       d_out_size, precision, stream, false);
}

mans_status mans_compress_ex(mans_workspace* ws, mans_dtype dtype, mans_layout layout,
                             const void* d_in, uint64_t n_elems, void* d_out,
                             uint64_t out_capacity, uint64_t* d_out_size, int precision,
                             mans_stream_t stream) {
  return compress_impl(ws, dtype, layout, d_in, n_elems, d_out, out_capacity, d_out_size,
                       precision, stream, false);
}

mans_status mans_adm_map(mans_workspace* ws, mans_dtype dtype, mans_layout layout,
                         const void* d_in, uint64_t n_elems, void* d_out, uint64_t out_capacity,
                         uint64_t* d_out_size, mans_stream_t stream) {
  if (dtype == MANS_U8) return MANS_ERR_INVALID_ARG;
  return compress_impl(ws, dtype, layout, d_in, n_elems, d_out, out_capacity, d_out_size, 10,
                       stream, true);
}

mans_status mans_decompress(mans_workspace* ws, mans_dtype dtype, const void* d_in,
                            uint64_t in_size, void* d_out, uint64_t n_elems,
                            mans_stream_t stream) {
  return decompress_impl(ws, dtype, MANS_LAYOUT_NATIVE, d_in, in_size, d_out, n_elems, stream,
                         false);
}

mans_status mans_decompress_ex(mans_workspace* ws, mans_dtype dtype, mans_layout layout,
                               const void* d_in, uint64_t in_size, void* d_out, uint64_t n_elems,
                               mans_stream_t stream) {
  return decompress_impl(ws, dtype, layout, d_in, in_size, d_out, n_elems, stream, false);
}

mans_status mans_adm_unmap(mans_workspace* ws, mans_dtype dtype, mans_layout layout,
                           const void* d_in, uint64_t in_size, void* d_out, uint64_t n_elems,
                           mans_stream_t stream) {
  if (dtype == MANS_U8) return MANS_ERR_INVALID_ARG;
  return decompress_impl(ws, dtype, layout, d_in, in_size, d_out, n_elems, stream, true);
}

mans_status mans_workspace_set_timing(mans_workspace* ws, int enable) {
  if (!ws) return MANS_ERR_INVALID_ARG;
  if (enable) {
    for (auto& row : ws->ev_c)
      for (auto& ev : row)
        if (!ev && cudaEventCreate(&ev) != cudaSuccess) return MANS_ERR_CUDA;
    for (auto& row : ws->ev_d)
      for (auto& ev : row)
        if (!ev && cudaEventCreate(&ev) != cudaSuccess) return MANS_ERR_CUDA;
  }
  ws->timing = enable != 0;
  ws->nc = ws->nd = 0;
  return MANS_OK;
}

mans_status mans_workspace_kernel_times(mans_workspace* ws, float ms[4], int calls[2]) {
  if (!ws || !ms) return MANS_ERR_INVALID_ARG;
  for (int i = 0; i < 4; ++i) ms[i] = 0.f;
  for (int c = 0; c < ws->nc; ++c) {
    if (cudaEventSynchronize(ws->ev_c[c][2]) != cudaSuccess) return MANS_ERR_CUDA;
    float a = 0, b = 0;
    if (cudaEventElapsedTime(&a, ws->ev_c[c][0], ws->ev_c[c][1]) != cudaSuccess ||
        cudaEventElapsedTime(&b, ws->ev_c[c][1], ws->ev_c[c][2]) != cudaSuccess)
      return MANS_ERR_CUDA;
    ms[0] += a;
    ms[1] += b;
  }
  for (int c = 0; c < ws->nd; ++c) {
    if (cudaEventSynchronize(ws->ev_d[c][2]) != cudaSuccess) return MANS_ERR_CUDA;
    float a = 0, b = 0;
    if (cudaEventElapsedTime(&a, ws->ev_d[c][0], ws->ev_d[c][1]) != cudaSuccess ||
        cudaEventElapsedTime(&b, ws->ev_d[c][1], ws->ev_d[c][2]) != cudaSuccess)
      return MANS_ERR_CUDA;
    ms[2] += a;
    ms[3] += b;
  }
  if (calls) {
    calls[0] = ws->nc;
    calls[1] = ws->nd;
  }
  ws->nc = ws->nd = 0;
  return MANS_OK;
}

}  // extern "C"

// ------------------------------------------------------------------------
// Reference-compatible entry points on a library-owned workspace per
// (device, stream). The reference allocates scratch on every call and never
// frees it (GpuANSEncode.h:298-327, GpuANSDecode.h:386-387); here a call
// allocates only when the workspace has to grow.
// ------------------------------------------------------------------------
namespace {
// A workspace replaced by a larger one is destroyed when its last user
// drops it, after the work queued on its stream has finished, so a call on
// another host thread that still holds it never sees its memory freed.
struct WsRelease {
  cudaStream_t s;
  void operator()(mans_workspace* ws) const {
    cudaStreamSynchronize(s);
    mans_workspace_destroy(ws);
  }
};
using WsRef = std::shared_ptr<mans_workspace>;
std::mutex g_mu;
std::map<std::pair<int, cudaStream_t>, WsRef> g_ws;

// The caller holds g_mu until its launches are enqueued: the calls of
// several host threads on one stream share that stream's workspace, so one
// call's launches (histogram, then encode) must stay adjacent in stream
// order.
WsRef default_ws(cudaStream_t s, uint64_t need_bytes, mans_status* st) {
  int dev = 0;
  if (cudaGetDevice(&dev) != cudaSuccess) {
    *st = MANS_ERR_CUDA;
    return nullptr;
  }
  auto key = std::make_pair(dev, s);
  auto it = g_ws.find(key);
  if (it != g_ws.end() && it->second->max_input_bytes >= need_bytes) {
    *st = MANS_OK;
    return it->second;
  }
  uint64_t cap = 1ull << 20;
  if (it != g_ws.end()) {
    cap = it->second->max_input_bytes * 2;
    g_ws.erase(it);
  }
  while (cap < need_bytes) cap *= 2;
  mans_workspace* ws = nullptr;
  *st = mans_workspace_create(&ws, cap, 0);
  if (*st != MANS_OK) return nullptr;
  WsRef ref(ws, WsRelease{s});
  g_ws[key] = ref;
  return ref;
}
}  // namespace

extern "C" {

uint32_t mans_ans_max_compressed_size(uint32_t in_size) {
  const uint64_t b = ans_bound(in_size);
  return b > 0xffffffffull ? 0xffffffffu : (uint32_t)b;
}

mans_status mans_ans_encode(int precision, const uint8_t* d_in, uint32_t in_size,
                            uint8_t* d_out, uint32_t* d_out_size, mans_stream_t stream) {
  if (!d_out || !d_out_size || (!d_in && in_size)) return MANS_ERR_INVALID_ARG;
  if (!valid_precision(precision)) return MANS_ERR_UNSUPPORTED_PRECISION;
  if ((d_in && !aligned16(d_in)) || !aligned16(d_out)) return MANS_ERR_ALIGNMENT;
  cudaStream_t s = reinterpret_cast<cudaStream_t>(stream);
  mans_status st = MANS_OK;
  std::lock_guard<std::mutex> lock(g_mu);
  const WsRef ws = default_ws(s, in_size, &st);
  if (!ws) return st;
  cudaError_t e = launch_hist_bytes(d_in, in_size, ws->ctrl, precision, ws->cfg, s);
  if (e == cudaSuccess)
    e = launch_ans_encode(d_in, d_out, ans_bound(in_size), nullptr, d_out_size, ws->ctrl,
                          ws->ans_flags, precision, div_up_u64(in_size, kAnsBlock),
                          ws->cfg, s, ws->enc_slots);
  return e == cudaSuccess ? MANS_OK : MANS_ERR_CUDA;
}

mans_status mans_ans_decode(int precision, const uint8_t* d_in, uint8_t* d_out,
                            mans_stream_t stream) {
  if (!d_in || !d_out) return MANS_ERR_INVALID_ARG;
  if (!valid_precision(precision)) return MANS_ERR_UNSUPPORTED_PRECISION;
  if (!aligned16(d_in) || !aligned16(d_out)) return MANS_ERR_ALIGNMENT;
  cudaStream_t s = reinterpret_cast<cudaStream_t>(stream);
  mans_status st = MANS_OK;
  std::lock_guard<std::mutex> lock(g_mu);
  const WsRef ws = default_ws(s, 0, &st);
  if (!ws) return st;
  // Sizes come from the stream header on the device (as in the reference):
  // the grid is one resident wave and the caller sized d_out from the header.
  const uint64_t wave = (uint64_t)ws->cfg.sms * ws->cfg.dec_ctas * 4;
  cudaError_t e = launch_ans_decode(d_in, ~0ull, d_out, ~0ull, ws->ctrl, precision, 0, wave,
                                    ws->cfg, s);
  return e == cudaSuccess ? MANS_OK : MANS_ERR_CUDA;
}

mans_status mans_ans_encode_batch(int precision, const uint8_t* d_in, uint32_t in_size,
                                  uint8_t* d_out, uint32_t* d_out_size, mans_stream_t stream) {
  return mans_ans_encode(precision, d_in, in_size, d_out, d_out_size, stream);
}

mans_status mans_ans_decode_batch(int precision, const uint8_t* d_in, uint8_t* d_out,
                                  mans_stream_t stream) {
  return mans_ans_decode(precision, d_in, d_out, stream);
}

mans_status mans_ans_last_status(mans_stream_t stream, uint64_t* detail) {
  cudaStream_t s = reinterpret_cast<cudaStream_t>(stream);
  int dev = 0;
  if (cudaGetDevice(&dev) != cudaSuccess) return MANS_ERR_CUDA;
  WsRef ws;
  {
    std::lock_guard<std::mutex> lock(g_mu);
    auto it = g_ws.find(std::make_pair(dev, s));
    if (it == g_ws.end()) {
      if (detail) *detail = 0;
      return MANS_OK;
    }
    ws = it->second;
  }
  return mans_workspace_status(ws.get(), stream, detail);
}

// Diagnostic: the encoder's division table entry for (pdf, cdf, p).
mans_status mans_debug_bounded_wait(uint32_t* status, float* elapsed_ms) {
  NvtxRange range("mans_debug_bounded_wait");
  if (!status) return MANS_ERR_INVALID_ARG;
  uint8_t* mem = nullptr;
  const size_t flags_off = (sizeof(Ctrl) + 255) / 256 * 256;
  const size_t bytes = flags_off + 64 * sizeof(unsigned long long);
  if (cudaMalloc(&mem, bytes) != cudaSuccess) {
    cudaGetLastError();
    return MANS_ERR_OUT_OF_MEMORY;
  }
  cudaEvent_t e0, e1;
  cudaEventCreate(&e0);
  cudaEventCreate(&e1);
  cudaError_t e = cudaMemset(mem, 0, bytes);
  Ctrl* ctrl = reinterpret_cast<Ctrl*>(mem);
  cudaEventRecord(e0, 0);
  if (e == cudaSuccess) {
    debug_wait_kernel<<<1, 32>>>(reinterpret_cast<unsigned long long*>(mem + flags_off), ctrl);
    e = cudaGetLastError();
  }
  cudaEventRecord(e1, 0);
  if (e == cudaSuccess) e = cudaEventSynchronize(e1);
  uint32_t st = 0;
  if (e == cudaSuccess) e = cudaMemcpy(&st, &ctrl->status, sizeof(st), cudaMemcpyDeviceToHost);
  float ms = 0.f;
  if (e == cudaSuccess) cudaEventElapsedTime(&ms, e0, e1);
  cudaEventDestroy(e0);
  cudaEventDestroy(e1);
  cudaFree(mem);
  if (e != cudaSuccess) return MANS_ERR_CUDA;
  *status = st;
  if (elapsed_ms) *elapsed_ms = ms;
  return MANS_OK;
}

void mans_debug_enc_entry(uint32_t pdf, uint32_t cdf, int p, uint32_t out[2]) {
  const uint2 e = make_enc_entry(pdf, cdf, p);
  out[0] = e.x;
  out[1] = e.y;
}

}  // extern "C"
