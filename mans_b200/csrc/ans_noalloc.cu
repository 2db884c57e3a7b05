// ans_noalloc.cu -- rANS encode (the reference's ansEncode) that allocates no
// device memory, for callers that cannot call cudaMalloc on their call path:
// for example a real-time acquisition loop that cannot absorb cudaMalloc's
// latency or the device synchronisation cudaMalloc/cudaFree may imply, or a
// process whose device memory is entirely reserved up front by another
// allocator. mans_ans_encode instead creates (and may grow) a workspace on
// the first call on each stream.
//
// The scratch the kernels need -- the control block (status, work counters,
// histogram, coding table) and the per-block look-back flags -- lives in the
// file-scope array below, of fixed size, which every GPU that loads the
// library holds until the process exits. All calls on a device share it:
// calls that overlap on the GPU (e.g. on two streams) race and must not be
// issued; calls ordered on one stream are fine. Each call clears the part of
// the array that must start at zero (status, counters, histogram); the flags
// need no clearing because each call tags them with the epoch kept in the
// control block, which the call's last kernel advances.
#include <cstddef>
#include <mutex>

#include "ans_table.cuh"
#include "mans_internal.h"

namespace mans {
namespace {

// Largest input accepted (bytes); larger inputs are rejected.
constexpr uint32_t kNoAllocMaxBytes = 64u << 20;
constexpr uint32_t kNoAllocMaxBlocks = kNoAllocMaxBytes / kAnsBlock;  // 16,384
constexpr size_t kCtrlBytes = (sizeof(Ctrl) + 255) / 256 * 256;
constexpr size_t kScratchBytes = kCtrlBytes + sizeof(unsigned long long) * (kNoAllocMaxBlocks + 2);

// About 132 KiB per device: control block + look-back flags.
static __device__ __align__(256) unsigned char g_noalloc_scratch[kScratchBytes];

struct DeviceState {
  bool ready = false;
  unsigned char* scratch = nullptr;  // device address of g_noalloc_scratch
  LaunchCfg cfg;
};
constexpr int kMaxDevices = 64;
std::mutex g_mu;
DeviceState g_state[kMaxDevices];

uint64_t ans_bound_bytes(uint64_t n) {
  const uint64_t nb = div_up_u64(n, kAnsBlock);
  return ans_overhead(nb) + nb * (uint64_t)kAnsMaxBlockWords * 2;
}

}  // namespace
}  // namespace mans

using namespace mans;

extern "C" mans_status mans_ans_encode_noalloc(int precision, const uint8_t* d_in,
                                               uint32_t in_size, uint8_t* d_out,
                                               uint32_t* d_out_size, mans_stream_t stream) {
  if (!d_out || !d_out_size || (!d_in && in_size)) return MANS_ERR_INVALID_ARG;
  if (precision < 9 || precision > 11) return MANS_ERR_UNSUPPORTED_PRECISION;
  if ((d_in && (reinterpret_cast<uintptr_t>(d_in) & 15u)) ||
      (reinterpret_cast<uintptr_t>(d_out) & 15u))
    return MANS_ERR_ALIGNMENT;
  if (in_size > kNoAllocMaxBytes) return MANS_ERR_TOO_LARGE;
  int dev = 0;
  if (cudaGetDevice(&dev) != cudaSuccess) return MANS_ERR_CUDA;
  if (dev < 0 || dev >= kMaxDevices) return MANS_ERR_INVALID_ARG;

  unsigned char* scratch = nullptr;
  LaunchCfg cfg;
  {
    std::lock_guard<std::mutex> lock(g_mu);
    DeviceState& st = g_state[dev];
    if (!st.ready) {
      // One-time set-up on this device (the device is current): the device
      // address of the scratch array and the launch configuration.
      if (cudaGetSymbolAddress(reinterpret_cast<void**>(&st.scratch), g_noalloc_scratch) !=
          cudaSuccess) {
        cudaGetLastError();
        return MANS_ERR_CUDA;
      }
      init_launch_cfg(st.cfg, dev);
      st.ready = true;
    }
    scratch = st.scratch;
    cfg = st.cfg;
  }
  Ctrl* ctrl = reinterpret_cast<Ctrl*>(scratch);
  unsigned long long* flags = reinterpret_cast<unsigned long long*>(scratch + kCtrlBytes);
  cudaStream_t s = reinterpret_cast<cudaStream_t>(stream);
  // status, detail, work counters and histogram start at zero
  if (cudaMemsetAsync(ctrl, 0, offsetof(Ctrl, enc_table), s) != cudaSuccess) return MANS_ERR_CUDA;
  cudaError_t e = launch_hist_bytes(d_in, in_size, ctrl, precision, cfg, s);
  if (e == cudaSuccess)
    e = launch_ans_encode(d_in, d_out, ans_bound_bytes(in_size), nullptr, d_out_size, ctrl, flags,
                          precision, div_up_u64(in_size, kAnsBlock), cfg, s, nullptr);
  return e == cudaSuccess ? MANS_OK : MANS_ERR_CUDA;
}

// Device-side errors of the last call (an expired bounded wait, a block past
// its word bound) land in the control block at the start of the fixed array;
// this copies them out with a synchronous copy into caller stack memory, so it
// allocates nothing either. The next encode call's memset clears them.
extern "C" mans_status mans_ans_noalloc_status(mans_stream_t stream, uint64_t* detail) {
  int dev = 0;
  if (cudaGetDevice(&dev) != cudaSuccess) return MANS_ERR_CUDA;
  if (dev < 0 || dev >= kMaxDevices) return MANS_ERR_INVALID_ARG;
  unsigned char* scratch = nullptr;
  {
    std::lock_guard<std::mutex> lock(g_mu);
    if (g_state[dev].ready) scratch = g_state[dev].scratch;
  }
  if (detail) *detail = 0;
  if (!scratch) return MANS_OK;  // no call has been made on this device
  if (cudaStreamSynchronize(reinterpret_cast<cudaStream_t>(stream)) != cudaSuccess)
    return MANS_ERR_CUDA;
  struct {
    uint32_t status, pad;
    unsigned long long detail;
  } h = {0, 0, 0};
  static_assert(offsetof(Ctrl, status) == 0 && offsetof(Ctrl, detail) == 8,
                "status and detail lead the control block");
  if (cudaMemcpy(&h, scratch, sizeof(h), cudaMemcpyDeviceToHost) != cudaSuccess)
    return MANS_ERR_CUDA;
  if (detail) *detail = h.detail;
  return (mans_status)h.status;
}
