// ref_adm_shim.cpp -- C entry points over the reference's own CPU ADM mapping
// (TEST INFRASTRUCTURE).
//
// Linked together with mapping/cpu/mappingcpuV2.cpp, compiled where it lies
// in the reference tree (its main() renamed on the command line), into
// oracle/_ref/libref_adm_cpu.so by oracle/Makefile. Used to pin the oracle's
// uint16 mapping against the reference and as the timed CPU baseline.
#include <omp.h>

#include <cstdint>
#include <cstring>
#include <vector>

// Signatures of mappingcpuV2.cpp:35-41 and :146-152.
void compress(const std::vector<uint16_t>& input_data, std::vector<int>& output_lengths,
              std::vector<uint16_t>& centers, std::vector<uint8_t>& codes,
              std::vector<uint8_t>& bit_signals);
void decompress(const std::vector<int>& output_lengths, const std::vector<uint16_t>& centers,
                const std::vector<uint8_t>& codes, const std::vector<uint8_t>& bit_signals,
                std::vector<uint16_t>& output_data);

namespace {
struct RefState {
  std::vector<uint16_t> input;
  std::vector<int> lengths;  // g + 1 entries after compress()
  std::vector<uint16_t> centers;
  std::vector<uint8_t> codes;
  std::vector<uint8_t> bits;
  std::vector<uint16_t> recovered;
};
}  // namespace

extern "C" {

// OpenMP threads used by the reference mapping. With more than one thread the
// reference's per-group length update (mappingcpuV2.cpp:98) is a data race
// whenever one group's lanes fall in different OpenMP chunks.
void ref_adm_cpu_set_threads(int n) { omp_set_num_threads(n); }
int ref_adm_cpu_get_threads(void) { return omp_get_max_threads(); }

void* ref_adm_cpu_create(const uint16_t* in, uint64_t n) {
  auto* s = new RefState();
  s->input.assign(in, in + n);
  return s;
}

void ref_adm_cpu_destroy(void* h) { delete static_cast<RefState*>(h); }

// One call of the reference compress() on the held input.
void ref_adm_cpu_compress(void* h) {
  auto* s = static_cast<RefState*>(h);
  compress(s->input, s->lengths, s->centers, s->codes, s->bits);
}

// One call of the reference decompress() on the held compressed arrays.
void ref_adm_cpu_decompress(void* h) {
  auto* s = static_cast<RefState*>(h);
  decompress(s->lengths, s->centers, s->codes, s->bits, s->recovered);
}

// Size of the merged buffer. v15_layout=1 drops the CPU mapping's extra
// trailing length entry so the layout matches the GPU mapping
// (mappingV15_fused_uint16.cu:933-957); v15_layout=0 keeps the CPU layout
// (mappingcpuV2.cpp:271-283).
uint64_t ref_adm_cpu_merged_size(void* h, int v15_layout) {
  auto* s = static_cast<RefState*>(h);
  uint64_t nl = s->lengths.size() - (v15_layout && !s->lengths.empty() ? 1 : 0);
  return nl * 4 + s->centers.size() * 2 + s->codes.size() + s->bits.size();
}

uint64_t ref_adm_cpu_merged(void* h, int v15_layout, uint8_t* out) {
  auto* s = static_cast<RefState*>(h);
  uint64_t nl = s->lengths.size() - (v15_layout && !s->lengths.empty() ? 1 : 0);
  uint64_t o = 0;
  std::memcpy(out + o, s->lengths.data(), nl * 4);
  o += nl * 4;
  std::memcpy(out + o, s->centers.data(), s->centers.size() * 2);
  o += s->centers.size() * 2;
  std::memcpy(out + o, s->codes.data(), s->codes.size());
  o += s->codes.size();
  std::memcpy(out + o, s->bits.data(), s->bits.size());
  o += s->bits.size();
  return o;
}

uint64_t ref_adm_cpu_recovered(void* h, uint16_t* out) {
  auto* s = static_cast<RefState*>(h);
  std::memcpy(out, s->recovered.data(), s->recovered.size() * 2);
  return s->recovered.size();
}

}  // extern "C"
