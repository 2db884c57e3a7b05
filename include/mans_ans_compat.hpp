// mans_ans_compat.hpp -- source-compatible replacement for the reference's
// codec entry points (namespace multibyte_ans, include/ans/*.h), forwarding
// to the C ABI of libmans_b200.so. A caller of the reference switches by
// including this header instead of ans/GpuANSEncode.h + ans/GpuANSDecode.h
// and linking -lmans_b200.
//
// Differences from the reference (all additions): the functions return a
// mans_status instead of void (the reference printed and continued), and
// getMaxCompressedSize() is a true upper bound.
#pragma once

#include <cstdint>
#include <cuda_runtime.h>

#include "mans.h"

namespace multibyte_ans {

// include/ans/GpuANSEncode.h:286
inline mans_status ansEncode(int precision, uint8_t* in, uint32_t inSize, uint8_t* out,
                             uint32_t* outSize, cudaStream_t stream) {
  return mans_ans_encode(precision, in, inSize, out, outSize,
                         reinterpret_cast<mans_stream_t>(stream));
}

// include/ans/GpuANSDecode.h:379
inline mans_status ansDecode(int precision, uint8_t* in, uint8_t* out, cudaStream_t stream) {
  return mans_ans_decode(precision, in, out, reinterpret_cast<mans_stream_t>(stream));
}

// src/GpuANS.cu:16
inline mans_status ansEncodeBatch(int precision, uint8_t* in, uint32_t inSize, uint8_t* out,
                                  uint32_t* outSize, cudaStream_t stream) {
  return mans_ans_encode_batch(precision, in, inSize, out, outSize,
                               reinterpret_cast<mans_stream_t>(stream));
}

// src/GpuANS.cu:33
inline mans_status ansDecodeBatch(int precision, uint8_t* in, uint8_t* out, cudaStream_t stream) {
  return mans_ans_decode_batch(precision, in, out, reinterpret_cast<mans_stream_t>(stream));
}

// include/ans/GpuANSCodec.h:237
inline uint32_t getMaxCompressedSize(uint32_t uncompressedBytes) {
  return mans_ans_max_compressed_size(uncompressedBytes);
}

}  // namespace multibyte_ans
