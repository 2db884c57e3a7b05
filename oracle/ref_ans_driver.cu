// ref_ans_driver.cu -- runs the reference's own GPU rANS codec on a file
// (TEST INFRASTRUCTURE, golden-vector generation only).
//
// Compiled by oracle/Makefile with the reference's include/ directory on the
// include path (the reference headers are compiled where they lie, never
// copied). Usage: ref_ans_driver <precision> <input.bin> <stream.ans> <decoded.bin>
// Calls multibyte_ans::ansEncode (include/ans/GpuANSEncode.h:286) and
// multibyte_ans::ansDecode (include/ans/GpuANSDecode.h:379) exactly as
// examples/compress.cu:48-55,105-110 does, with the precision as an argument.
#include <cstdio>
#include <cstdlib>
#include <vector>

#include "ans/GpuANSDecode.h"
#include "ans/GpuANSEncode.h"

static std::vector<uint8_t> read_file(const char* path) {
  std::vector<uint8_t> v;
  FILE* f = std::fopen(path, "rb");
  if (!f) return v;
  std::fseek(f, 0, SEEK_END);
  long sz = std::ftell(f);
  std::fseek(f, 0, SEEK_SET);
  v.resize(sz);
  if (sz > 0 && std::fread(v.data(), 1, sz, f) != (size_t)sz) v.clear();
  std::fclose(f);
  return v;
}

static int write_file(const char* path, const uint8_t* p, size_t n) {
  FILE* f = std::fopen(path, "wb");
  if (!f) return 1;
  size_t w = n ? std::fwrite(p, 1, n, f) : 0;
  std::fclose(f);
  return w == n ? 0 : 1;
}

int main(int argc, char** argv) {
  if (argc < 5) {
    std::fprintf(stderr, "usage: %s <precision> <in> <stream> <decoded>\n", argv[0]);
    return 2;
  }
  int precision = std::atoi(argv[1]);
  std::vector<uint8_t> in = read_file(argv[2]);
  uint32_t n = (uint32_t)in.size();
  uint8_t* d_in = nullptr;
  uint8_t* d_out = nullptr;
  uint8_t* d_dec = nullptr;
  uint32_t* d_size = nullptr;
  uint32_t cap = multibyte_ans::getMaxCompressedSize(n);
  if (cudaMalloc(&d_in, n ? n : 16) || cudaMalloc(&d_out, cap) || cudaMalloc(&d_dec, n ? n : 16) ||
      cudaMalloc(&d_size, 4)) {
    std::fprintf(stderr, "cudaMalloc failed\n");
    return 3;
  }
  if (n) cudaMemcpy(d_in, in.data(), n, cudaMemcpyHostToDevice);
  multibyte_ans::ansEncode(precision, d_in, n, d_out, d_size, 0);
  if (cudaDeviceSynchronize() != cudaSuccess) {
    std::fprintf(stderr, "encode failed\n");
    return 4;
  }
  uint32_t out_size = 0;
  cudaMemcpy(&out_size, d_size, 4, cudaMemcpyDeviceToHost);
  std::vector<uint8_t> stream(out_size);
  cudaMemcpy(stream.data(), d_out, out_size, cudaMemcpyDeviceToHost);
  if (write_file(argv[3], stream.data(), out_size)) return 5;
  if (n) {
    multibyte_ans::ansDecode(precision, d_out, d_dec, 0);
    if (cudaDeviceSynchronize() != cudaSuccess) {
      std::fprintf(stderr, "decode failed\n");
      return 6;
    }
  }
  std::vector<uint8_t> dec(n);
  if (n) cudaMemcpy(dec.data(), d_dec, n, cudaMemcpyDeviceToHost);
  if (write_file(argv[4], dec.data(), n)) return 7;
  std::printf("ref_ans_driver: n=%u stream=%u roundtrip=%s\n", n, out_size,
              dec == in ? "ok" : "MISMATCH");
  return dec == in ? 0 : 8;
}
