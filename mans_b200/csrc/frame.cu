// frame.cu -- the self-describing MANS frame (include/mans.h, "frames"): a
// 64-byte header in front of a MANS stream that records what the reference
// leaves out of band (element type, element count, mapping layout,
// precision) and the sizes a reader needs to check the stream, so a frame can
// be decoded with nothing else. For uint32 data the stream's mapped bytes
// already carry the group centers and record lengths that mappingV9_fuse.cu
// (:998) never writes; the frame adds the element count and type.
//
// Header (little endian):
//   0  u32 magic 'MANS' (0x534e414d)     4  u16 version (1)
//   6  u8  dtype (1, 2, 4)               7  u8  layout (0, 1, 2)
//   8  u8  precision (9..11)             9  u8  flags (0)
//  10  u16 header bytes (64)            12  u32 reserved (0)
//  16  u64 element count                24  u64 mapped bytes (the rANS input)
//  32  u64 stream bytes                 40  24 bytes reserved (0)
// The stream's own integrity checks (every block must consume exactly its
// words and end in the start state) guard the body.
#include <cstring>

#include "mans_device.cuh"
#include "mans_internal.h"

using namespace mans;

namespace {

constexpr uint32_t kFrameMagic = 0x534e414du;  // "MANS"
constexpr uint16_t kFrameVersion = 1;
constexpr uint32_t kFrameBytes = 64;

inline bool aligned16(const void* p) { return (reinterpret_cast<uintptr_t>(p) & 15u) == 0; }
inline uint64_t elem_bytes(uint32_t d) { return d == 1 ? 1 : d == 2 ? 2 : d == 4 ? 4 : 0; }

// Writes the header once the stream is complete (its size comes from the
// compress call's device-side output size). A size above the capacity means
// the compress call failed; the header then records no stream.
__global__ void frame_header_kernel(uint8_t* frame, uint64_t cap, uint32_t dtype, uint32_t layout,
                                    uint32_t precision, uint64_t n,
                                    unsigned long long* size_io) {
  const unsigned long long sz = *size_io;
  const bool ok = sz <= cap;
  const uint32_t mapped = ok && sz >= 32 ? reinterpret_cast<const uint32_t*>(frame + kFrameBytes)[2] : 0u;
  uint32_t* w = reinterpret_cast<uint32_t*>(frame);
  w[0] = kFrameMagic;
  w[1] = (uint32_t)kFrameVersion | (dtype << 16) | (layout << 24);
  w[2] = precision | (kFrameBytes << 16);
  w[3] = 0;
  unsigned long long* q = reinterpret_cast<unsigned long long*>(frame);
  q[2] = n;
  q[3] = mapped;
  q[4] = ok ? sz : 0ull;
  q[5] = q[6] = q[7] = 0;
  *size_io = kFrameBytes + (ok ? sz : 0ull);
}

}  // namespace

extern "C" {

mans_status mans_frame_parse(const void* header, uint64_t avail, mans_frame_info* info) {
  if (!header || !info) return MANS_ERR_INVALID_ARG;
  if (avail < kFrameBytes) return MANS_ERR_BAD_STREAM;
  const uint8_t* h = static_cast<const uint8_t*>(header);
  uint32_t magic;
  uint16_t ver, hb;
  std::memcpy(&magic, h, 4);
  std::memcpy(&ver, h + 4, 2);
  std::memcpy(&hb, h + 10, 2);
  if (magic != kFrameMagic || ver != kFrameVersion || hb != kFrameBytes) return MANS_ERR_BAD_STREAM;
  mans_frame_info f{};
  f.dtype = (mans_dtype)h[6];
  f.layout = (mans_layout)h[7];
  f.precision = h[8];
  std::memcpy(&f.n_elems, h + 16, 8);
  std::memcpy(&f.mapped_bytes, h + 24, 8);
  std::memcpy(&f.stream_bytes, h + 32, 8);
  f.header_bytes = kFrameBytes;
  const uint64_t eb = elem_bytes(f.dtype);
  if (eb == 0 || (uint32_t)f.layout > 2 || (f.layout != MANS_LAYOUT_NATIVE && f.dtype != MANS_U16) ||
      f.precision < 9 || f.precision > 11 || f.n_elems > (~0ull) / eb)
    return MANS_ERR_BAD_STREAM;
  if (f.dtype == MANS_U8 && f.mapped_bytes != f.n_elems) return MANS_ERR_BAD_STREAM;
  // The mapped bytes cannot exceed the worst case for the element count (nor
  // the rANS header's u32 count), and the stream cannot exceed the worst case
  // for the mapped bytes: this bounds every size handed to the decoder even
  // when the frame's available size is unknown.
  if (f.mapped_bytes > mans_max_mapped_size(f.dtype, f.n_elems) || f.mapped_bytes > 0xffffffffull)
    return MANS_ERR_BAD_STREAM;
  if (f.stream_bytes < 544) return MANS_ERR_BAD_STREAM;  // header + pdf of an empty stream
  if (f.stream_bytes > mans_stream_bound(f.mapped_bytes)) return MANS_ERR_BAD_STREAM;
  // compared without an addition that could wrap
  if (avail != ~0ull && f.stream_bytes > avail - kFrameBytes) return MANS_ERR_BAD_STREAM;
  *info = f;
  return MANS_OK;
}

uint64_t mans_frame_max_size(mans_dtype dtype, uint64_t n_elems) {
  const uint64_t s = mans_max_compressed_size(dtype, n_elems);
  return s ? s + kFrameBytes : 0;
}

mans_status mans_frame_compress(mans_workspace* ws, mans_dtype dtype, mans_layout layout,
                                const void* d_in, uint64_t n_elems, void* d_out,
                                uint64_t out_capacity, uint64_t* d_out_size, int precision,
                                mans_stream_t stream) {
  if (!d_out || !d_out_size) return MANS_ERR_INVALID_ARG;
  if (!aligned16(d_out)) return MANS_ERR_ALIGNMENT;
  if (out_capacity < kFrameBytes) return MANS_ERR_INVALID_ARG;
  uint8_t* body = static_cast<uint8_t*>(d_out) + kFrameBytes;
  cudaStream_t s = reinterpret_cast<cudaStream_t>(stream);
  // *d_out_size first receives the stream size (set to "none" beforehand,
  // in case the call fails on the device), then the frame size
  if (cudaMemsetAsync(d_out_size, 0xff, sizeof(uint64_t), s) != cudaSuccess) return MANS_ERR_CUDA;
  mans_status st = mans_compress_ex(ws, dtype, layout, d_in, n_elems, body,
                                    out_capacity - kFrameBytes, d_out_size, precision, stream);
  if (st != MANS_OK) return st;
  frame_header_kernel<<<1, 1, 0, s>>>(static_cast<uint8_t*>(d_out), out_capacity - kFrameBytes,
                                      (uint32_t)dtype, (uint32_t)layout, (uint32_t)precision,
                                      n_elems, reinterpret_cast<unsigned long long*>(d_out_size));
  return cudaGetLastError() == cudaSuccess ? MANS_OK : MANS_ERR_CUDA;
}

mans_status mans_frame_decompress(mans_workspace* ws, const mans_frame_info* info,
                                  const void* d_frame, void* d_out, uint64_t out_capacity,
                                  mans_stream_t stream) {
  if (!ws || !info || !d_frame) return MANS_ERR_INVALID_ARG;
  const uint64_t eb = elem_bytes(info->dtype);
  if (eb == 0) return MANS_ERR_BAD_STREAM;
  if (info->n_elems * eb > out_capacity) return MANS_ERR_OUTPUT_OVERFLOW;
  const uint8_t* body = static_cast<const uint8_t*>(d_frame) + kFrameBytes;
  return mans_decompress_ex(ws, info->dtype, info->layout, body, info->stream_bytes, d_out,
                            info->n_elems, stream);
}

}  // extern "C"
