// mans_cli -- command-line driver with the argv shape of the reference's
// examples/compress.cu: compress <input> into <temp>, decompress <temp> into
// <output>, print times, bandwidth and the compression ratio.
//
//   mans_cli <input.img> <temp.ans> <output.img> [--dtype u8|u16|u32]
//            [--precision 9|10|11] [--layout native|v12|cpuv2]
//   mans_cli --compress <input> <output.mans> [--dtype ...] [--precision ...] [--layout ...]
//   mans_cli --decompress <input.mans> <output>
//
// The last two forms write and read self-describing frames (a 64-byte header
// with the element type, count, layout and precision before the stream), so
// compression and decompression can run separately.
//
// --dtype u8 (the default) is exactly the reference example: byte rANS of the
// file (multibyte_ans::ansEncode / ansDecode). u16 / u32 add the ADM mapping.
// The stream file holds the stream only; the element count travels out of
// band as in the reference (examples/compress.cu:79-97), so one run does both
// directions. Exit status 0 only if the round trip is byte-identical.
#include <chrono>
#include <cstdio>
#include <cstdlib>
#include <cstring>
#include <fstream>
#include <string>
#include <vector>

#include <cuda_runtime.h>

#include "mans.h"

namespace {

bool read_file(const char* path, std::vector<uint8_t>& out) {
  std::ifstream f(path, std::ios::binary | std::ios::ate);
  if (!f) return false;
  const std::streamsize n = f.tellg();
  out.resize((size_t)n);
  f.seekg(0);
  return (bool)f.read(reinterpret_cast<char*>(out.data()), n) || n == 0;
}

bool write_file(const char* path, const uint8_t* p, size_t n) {
  std::ofstream f(path, std::ios::binary);
  return f && (bool)f.write(reinterpret_cast<const char*>(p), (std::streamsize)n);
}

int usage(const char* argv0) {
  std::fprintf(stderr,
               "Usage: %s <input.img> <temp.ans> <output.img> [--dtype u8|u16|u32] "
               "[--precision 9|10|11] [--layout native|v12|cpuv2]\n"
               "       %s --compress <input> <output.mans> [--dtype ...] [--precision ...] "
               "[--layout ...]\n"
               "       %s --decompress <input.mans> <output>\n",
               argv0, argv0, argv0);
  return 1;
}

#define CK(x)                                                                   \
  do {                                                                          \
    cudaError_t e_ = (x);                                                       \
    if (e_ != cudaSuccess) {                                                    \
      std::fprintf(stderr, "CUDA error %s at %s:%d\n", cudaGetErrorString(e_),  \
                   __FILE__, __LINE__);                                         \
      return 2;                                                                 \
    }                                                                           \
  } while (0)
#define MK(x)                                                                   \
  do {                                                                          \
    mans_status s_ = (x);                                                       \
    if (s_ != MANS_OK) {                                                        \
      std::fprintf(stderr, "mans error %d at %s:%d\n", (int)s_, __FILE__,       \
                   __LINE__);                                                   \
      return 3;                                                                 \
    }                                                                           \
  } while (0)

int frame_compress_file(const char* src, const char* dst, mans_dtype dtype, mans_layout layout,
                        int precision) {
  std::vector<uint8_t> in;
  if (!read_file(src, in)) {
    std::fprintf(stderr, "cannot read %s\n", src);
    return 1;
  }
  const uint64_t eb = dtype == MANS_U8 ? 1 : dtype == MANS_U16 ? 2 : 4;
  const uint64_t n = in.size() / eb, bytes = n * eb;
  mans_workspace* ws = nullptr;
  MK(mans_workspace_create(&ws, bytes ? bytes : 1, 0));
  const uint64_t cap = mans_frame_max_size(dtype, n);
  uint8_t *d_in = nullptr, *d_f = nullptr;
  uint64_t* d_size = nullptr;
  CK(cudaMalloc(&d_in, bytes ? bytes : 16));
  CK(cudaMalloc(&d_f, cap));
  CK(cudaMalloc(&d_size, 8));
  CK(cudaMemcpy(d_in, in.data(), bytes, cudaMemcpyHostToDevice));
  auto t0 = std::chrono::high_resolution_clock::now();
  MK(mans_frame_compress(ws, dtype, layout, bytes ? d_in : nullptr, n, d_f, cap, d_size, precision,
                         nullptr));
  uint64_t detail = 0;
  MK(mans_workspace_status(ws, nullptr, &detail));
  auto t1 = std::chrono::high_resolution_clock::now();
  uint64_t fsize = 0;
  CK(cudaMemcpy(&fsize, d_size, 8, cudaMemcpyDeviceToHost));
  std::vector<uint8_t> f(fsize);
  CK(cudaMemcpy(f.data(), d_f, fsize, cudaMemcpyDeviceToHost));
  if (!write_file(dst, f.data(), fsize)) return 1;
  const double ms = std::chrono::duration<double, std::milli>(t1 - t0).count();
  std::printf("comp   time %.3f ms B/W %.1f GB/s\ncompress ratio: %f\n", ms,
              bytes / 1e9 / (ms * 1e-3), fsize ? 1.0 * bytes / fsize : 0.0);
  cudaFree(d_in);
  cudaFree(d_f);
  cudaFree(d_size);
  mans_workspace_destroy(ws);
  return 0;
}

int frame_decompress_file(const char* src, const char* dst) {
  std::vector<uint8_t> f;
  if (!read_file(src, f)) {
    std::fprintf(stderr, "cannot read %s\n", src);
    return 1;
  }
  mans_frame_info info;
  MK(mans_frame_parse(f.data(), f.size(), &info));
  const uint64_t eb = info.dtype == MANS_U8 ? 1 : info.dtype == MANS_U16 ? 2 : 4;
  const uint64_t bytes = info.n_elems * eb;
  mans_workspace* ws = nullptr;
  MK(mans_workspace_create(&ws, bytes ? bytes : 1, 0));
  uint8_t *d_f = nullptr, *d_out = nullptr;
  CK(cudaMalloc(&d_f, f.size()));
  CK(cudaMalloc(&d_out, bytes ? bytes : 16));
  CK(cudaMemcpy(d_f, f.data(), f.size(), cudaMemcpyHostToDevice));
  auto t0 = std::chrono::high_resolution_clock::now();
  MK(mans_frame_decompress(ws, &info, d_f, bytes ? d_out : nullptr, bytes, nullptr));
  uint64_t detail = 0;
  MK(mans_workspace_status(ws, nullptr, &detail));
  auto t1 = std::chrono::high_resolution_clock::now();
  std::vector<uint8_t> out(bytes);
  CK(cudaMemcpy(out.data(), d_out, bytes, cudaMemcpyDeviceToHost));
  if (!write_file(dst, out.data(), bytes)) return 1;
  const double ms = std::chrono::duration<double, std::milli>(t1 - t0).count();
  std::printf("decomp time %.3f ms B/W %.1f GB/s\n", ms, f.size() / 1e9 / (ms * 1e-3));
  cudaFree(d_f);
  cudaFree(d_out);
  mans_workspace_destroy(ws);
  return 0;
}

}  // namespace

int main(int argc, char** argv) {
  std::vector<const char*> pos;
  int mode = 0;  // 0 round trip (reference argv), 1 frame compress, 2 frame decompress
  mans_dtype dtype = MANS_U8;
  mans_layout layout = MANS_LAYOUT_NATIVE;
  int precision = 10;
  for (int i = 1; i < argc; ++i) {
    const std::string a = argv[i];
    if (a == "-h" || a == "--help") {
      usage(argv[0]);
      return 0;
    } else if (a == "--compress") {
      mode = 1;
    } else if (a == "--decompress") {
      mode = 2;
    } else if (a == "--dtype" && i + 1 < argc) {
      const std::string v = argv[++i];
      dtype = v == "u16" ? MANS_U16 : v == "u32" ? MANS_U32 : v == "u8" ? MANS_U8 : (mans_dtype)0;
      if (dtype == 0) return usage(argv[0]);
    } else if (a == "--precision" && i + 1 < argc) {
      precision = std::atoi(argv[++i]);
    } else if (a == "--layout" && i + 1 < argc) {
      const std::string v = argv[++i];
      layout = v == "v12" ? MANS_LAYOUT_V12 : v == "cpuv2" ? MANS_LAYOUT_CPUV2 : MANS_LAYOUT_NATIVE;
      if (v != "v12" && v != "cpuv2" && v != "native") return usage(argv[0]);
    } else {
      pos.push_back(argv[i]);
    }
  }
  if (mode == 1 || mode == 2) {
    if (pos.size() != 2) return usage(argv[0]);
    return mode == 1 ? frame_compress_file(pos[0], pos[1], dtype, layout, precision)
                     : frame_decompress_file(pos[0], pos[1]);
  }
  if (pos.size() != 3) return usage(argv[0]);

  std::vector<uint8_t> in;
  if (!read_file(pos[0], in)) {
    std::fprintf(stderr, "cannot read %s\n", pos[0]);
    return 1;
  }
  const uint64_t eb = dtype == MANS_U8 ? 1 : dtype == MANS_U16 ? 2 : 4;
  const uint64_t n = in.size() / eb;  // a trailing partial element is not coded
  const uint64_t bytes = n * eb;

  cudaStream_t stream;
  CK(cudaStreamCreate(&stream));
  mans_workspace* ws = nullptr;
  MK(mans_workspace_create(&ws, bytes ? bytes : 1, 0));
  const uint64_t cap = mans_max_compressed_size(dtype, n);
  uint8_t *d_in = nullptr, *d_s = nullptr, *d_out = nullptr;
  uint64_t* d_size = nullptr;
  CK(cudaMalloc(&d_in, bytes ? bytes : 16));
  CK(cudaMalloc(&d_s, cap));
  CK(cudaMalloc(&d_out, bytes ? bytes : 16));
  CK(cudaMalloc(&d_size, sizeof(uint64_t)));
  CK(cudaMemcpy(d_in, in.data(), bytes, cudaMemcpyHostToDevice));

  std::printf("encode start!\n");
  auto t0 = std::chrono::high_resolution_clock::now();
  MK(mans_compress_ex(ws, dtype, layout, bytes ? d_in : nullptr, n, d_s, cap, d_size, precision,
                      reinterpret_cast<mans_stream_t>(stream)));
  CK(cudaStreamSynchronize(stream));
  auto t1 = std::chrono::high_resolution_clock::now();
  uint64_t detail = 0;
  MK(mans_workspace_status(ws, reinterpret_cast<mans_stream_t>(stream), &detail));
  const double comp_ms = std::chrono::duration<double, std::milli>(t1 - t0).count();
  std::printf("comp   time %.3f ms B/W %.1f GB/s\n", comp_ms, bytes / 1e9 / (comp_ms * 1e-3));
  uint64_t csize = 0;
  CK(cudaMemcpy(&csize, d_size, sizeof(csize), cudaMemcpyDeviceToHost));
  std::vector<uint8_t> stream_bytes(csize);
  CK(cudaMemcpy(stream_bytes.data(), d_s, csize, cudaMemcpyDeviceToHost));
  if (!write_file(pos[1], stream_bytes.data(), csize)) {
    std::fprintf(stderr, "cannot write %s\n", pos[1]);
    return 1;
  }
  std::printf("compress ratio: %f\n", csize ? 1.0 * bytes / csize : 0.0);

  // decompress from the file, as the reference does
  std::vector<uint8_t> s2;
  if (!read_file(pos[1], s2)) return 1;
  CK(cudaMemcpy(d_s, s2.data(), s2.size(), cudaMemcpyHostToDevice));
  std::printf("decode start!\n");
  t0 = std::chrono::high_resolution_clock::now();
  MK(mans_decompress_ex(ws, dtype, layout, d_s, s2.size(), bytes ? d_out : nullptr, n,
                        reinterpret_cast<mans_stream_t>(stream)));
  CK(cudaStreamSynchronize(stream));
  t1 = std::chrono::high_resolution_clock::now();
  MK(mans_workspace_status(ws, reinterpret_cast<mans_stream_t>(stream), &detail));
  const double dec_ms = std::chrono::duration<double, std::milli>(t1 - t0).count();
  std::printf("decomp time %.3f ms B/W %.1f GB/s\n", dec_ms, s2.size() / 1e9 / (dec_ms * 1e-3));
  std::vector<uint8_t> out(bytes);
  CK(cudaMemcpy(out.data(), d_out, bytes, cudaMemcpyDeviceToHost));
  if (!write_file(pos[2], out.data(), bytes)) {
    std::fprintf(stderr, "cannot write %s\n", pos[2]);
    return 1;
  }
  const bool same = std::memcmp(out.data(), in.data(), bytes) == 0;
  cudaFree(d_in);
  cudaFree(d_s);
  cudaFree(d_out);
  cudaFree(d_size);
  mans_workspace_destroy(ws);
  cudaStreamDestroy(stream);
  if (!same) {
    std::printf("round trip mismatch\n");
    return 4;
  }
  std::printf("Compression completed successfully.\n");
  return 0;
}
