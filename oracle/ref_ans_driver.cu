// ref_ans_driver.cu -- runs the reference's own GPU rANS codec on a file
// (TEST INFRASTRUCTURE: golden-vector generation, and the timed comparison
// with the reference's GPU path).
//
// Compiled by oracle/Makefile with the reference's include/ directory on the
// include path (the reference headers are compiled where they lie, never
// copied). Usage: ref_ans_driver <precision> <input.bin> <stream.ans> <decoded.bin>
// Calls multibyte_ans::ansEncode (include/ans/GpuANSEncode.h:286) and
// multibyte_ans::ansDecode (include/ans/GpuANSDecode.h:379) exactly as
// examples/compress.cu:48-55,105-110 does, with the precision as an argument.
#include <chrono>
#include <cstdio>
#include <cstdlib>
#include <string>
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

// Timing mode (reference-GPU comparison in bench.py): ref_ans_driver time
// <precision> <in> <reps>. Warm-up calls first (the reference allocates its
// scratch inside every call, GpuANSEncode.h:298-327, and never frees it, so
// reps stays small), then reps encodes and reps decodes, each timed with CUDA
// events around the call plus a stream synchronisation, and with a host clock
// around the same span as examples/compress.cu:45-63 does.
static int time_mode(int precision, const char* path, int reps) {
  std::vector<uint8_t> in = read_file(path);
  uint32_t n = (uint32_t)in.size();
  if (n == 0) return 2;
  uint8_t *d_in = nullptr, *d_out = nullptr, *d_dec = nullptr;
  uint32_t* d_size = nullptr;
  uint32_t cap = multibyte_ans::getMaxCompressedSize(n);
  if (cudaMalloc(&d_in, n) || cudaMalloc(&d_out, cap) || cudaMalloc(&d_dec, n) ||
      cudaMalloc(&d_size, 4))
    return 3;
  cudaMemcpy(d_in, in.data(), n, cudaMemcpyHostToDevice);
  cudaEvent_t e0, e1;
  cudaEventCreate(&e0);
  cudaEventCreate(&e1);
  for (int w = 0; w < 2; ++w) {
    multibyte_ans::ansEncode(precision, d_in, n, d_out, d_size, 0);
    multibyte_ans::ansDecode(precision, d_out, d_dec, 0);
  }
  if (cudaDeviceSynchronize() != cudaSuccess) return 4;
  double enc_ev = 0, dec_ev = 0, enc_wall = 0, dec_wall = 0;
  for (int r = 0; r < reps; ++r) {
    auto t0 = std::chrono::steady_clock::now();
    cudaEventRecord(e0, 0);
    multibyte_ans::ansEncode(precision, d_in, n, d_out, d_size, 0);
    cudaEventRecord(e1, 0);
    cudaStreamSynchronize(0);
    auto t1 = std::chrono::steady_clock::now();
    float ms = 0;
    cudaEventElapsedTime(&ms, e0, e1);
    enc_ev += ms;
    enc_wall += std::chrono::duration<double, std::milli>(t1 - t0).count();
  }
  for (int r = 0; r < reps; ++r) {
    auto t0 = std::chrono::steady_clock::now();
    cudaEventRecord(e0, 0);
    multibyte_ans::ansDecode(precision, d_out, d_dec, 0);
    cudaEventRecord(e1, 0);
    cudaStreamSynchronize(0);
    auto t1 = std::chrono::steady_clock::now();
    float ms = 0;
    cudaEventElapsedTime(&ms, e0, e1);
    dec_ev += ms;
    dec_wall += std::chrono::duration<double, std::milli>(t1 - t0).count();
  }
  if (cudaDeviceSynchronize() != cudaSuccess) return 4;
  uint32_t out_size = 0;
  cudaMemcpy(&out_size, d_size, 4, cudaMemcpyDeviceToHost);
  std::vector<uint8_t> dec(n);
  cudaMemcpy(dec.data(), d_dec, n, cudaMemcpyDeviceToHost);
  std::printf("REFTIME n=%u stream=%u reps=%d encode_event_ms=%.4f encode_wall_ms=%.4f "
              "decode_event_ms=%.4f decode_wall_ms=%.4f roundtrip=%s\n",
              n, out_size, reps, enc_ev / reps, enc_wall / reps, dec_ev / reps, dec_wall / reps,
              dec == in ? "ok" : "MISMATCH");
  return dec == in ? 0 : 8;
}

int main(int argc, char** argv) {
  if (argc >= 5 && std::string(argv[1]) == "time")
    return time_mode(std::atoi(argv[2]), argv[3], std::atoi(argv[4]));
  if (argc < 5) {
    std::fprintf(stderr, "usage: %s <precision> <in> <stream> <decoded>\n"
                         "       %s time <precision> <in> <reps>\n", argv[0], argv[0]);
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
