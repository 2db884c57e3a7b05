// serve.cu -- the serving loop (include/mans.h, "serving"): a scheduler
// thread admits queued compress / decompress requests against an HBM budget
// and folds whatever is queued into the next batched launch.
//
// Device memory is fixed at creation and never exceeds the budget: per lane
// a batch workspace (or, in plain mode, a single-buffer workspace), and an
// output arena for results the caller does not place itself. A request is
// admitted when its lane has room and its worst-case output fits in the
// arena; a compress result is shrunk to its real size when it completes and
// returned to the arena when the caller releases it.
//
// Continuous batching: there are several lanes per direction, each with its
// own stream, so a batch is formed and launched from the requests that
// arrived while earlier batches are still on the GPU; nothing waits for a
// batch to fill. Completion is signalled by a host function enqueued after
// each batch, and the scheduler collects the per-request statuses that were
// copied to pinned memory behind it.
#include <atomic>
#include <chrono>
#include <condition_variable>
#include <cstring>
#include <deque>
#include <map>
#include <mutex>
#include <new>
#include <thread>
#include <unordered_map>
#include <vector>

#include "batch_internal.h"
#include "mans_device.cuh"

using namespace mans;

namespace {

inline uint64_t now_ns() {
  return (uint64_t)std::chrono::duration_cast<std::chrono::nanoseconds>(
             std::chrono::steady_clock::now().time_since_epoch())
      .count();
}
inline uint64_t align256(uint64_t v) { return (v + 255) / 256 * 256; }
inline uint64_t elem_bytes(uint32_t d) { return d == MANS_U8 ? 1 : d == MANS_U16 ? 2 : d == MANS_U32 ? 4 : 0; }
inline bool aligned16(const void* p) { return (reinterpret_cast<uintptr_t>(p) & 15u) == 0; }

// First-fit allocator over [0, size) in 256-byte granules, with coalescing.
class Arena {
 public:
  void reset(uint64_t size) {
    free_.clear();
    if (size) free_[0] = size;
    size_ = size;
    used_ = peak_ = 0;
  }
  bool alloc(uint64_t bytes, uint64_t* off) {
    bytes = align256(bytes ? bytes : 256);
    for (auto it = free_.begin(); it != free_.end(); ++it) {
      if (it->second >= bytes) {
        *off = it->first;
        const uint64_t rest = it->second - bytes, at = it->first + bytes;
        free_.erase(it);
        if (rest) free_[at] = rest;
        used_ += bytes;
        if (used_ > peak_) peak_ = used_;
        return true;
      }
    }
    return false;
  }
  void release(uint64_t off, uint64_t bytes) {
    bytes = align256(bytes ? bytes : 256);
    used_ -= bytes;
    auto it = free_.emplace(off, bytes).first;
    auto nx = std::next(it);
    if (nx != free_.end() && it->first + it->second == nx->first) {
      it->second += nx->second;
      free_.erase(nx);
    }
    if (it != free_.begin()) {
      auto pv = std::prev(it);
      if (pv->first + pv->second == it->first) {
        pv->second += it->second;
        free_.erase(it);
      }
    }
  }
  // Keep the first new_bytes of an allocation and free the rest.
  void shrink(uint64_t off, uint64_t old_bytes, uint64_t new_bytes) {
    old_bytes = align256(old_bytes ? old_bytes : 256);
    new_bytes = align256(new_bytes ? new_bytes : 256);
    if (new_bytes < old_bytes) release(off + new_bytes, old_bytes - new_bytes);
  }
  uint64_t size() const { return size_; }
  uint64_t used() const { return used_; }
  uint64_t peak() const { return peak_; }

 private:
  std::map<uint64_t, uint64_t> free_;
  uint64_t size_ = 0, used_ = 0, peak_ = 0;
};

struct Req {
  uint64_t ticket = 0;
  mans_request r{};
  uint64_t t_arrive = 0, t_launch = 0;
  bool in_arena = false;
  uint64_t arena_off = 0, arena_bytes = 0;
  uint8_t* out = nullptr;
  uint64_t out_cap = 0;
};

struct Lane {
  int op = 0;
  mans_batch* batch = nullptr;     // batched mode
  mans_workspace* ws = nullptr;    // plain mode
  cudaStream_t stream = nullptr;
  cudaEvent_t done = nullptr;
  bool busy = false;
  std::vector<Req> reqs;
  uint32_t* h_status = nullptr;    // pinned, per request of the launch
  uint64_t* h_detail = nullptr;
  uint64_t* h_sizes = nullptr;
  uint64_t* d_sizes = nullptr;     // device compress sizes
};

}  // namespace

struct mans_server {
  int device = 0;
  mans_server_config cfg{};
  uint32_t max_items = 0;
  std::vector<Lane> lanes;
  uint8_t* arena_base = nullptr;
  Arena arena;
  std::mutex mu;
  std::condition_variable cv;       // scheduler wake-up
  std::condition_variable done_cv;  // poll wake-up
  std::deque<Req> queue[2];
  std::deque<mans_completion> completed;
  std::unordered_map<uint64_t, std::pair<uint64_t, uint64_t>> held;  // ticket -> arena block
  uint64_t next_ticket = 1;
  bool stop = false;
  std::thread sched;
  mans_server_stats stats{};
};

namespace {

void CUDART_CB notify_host(void* p) {
  // runs on a CUDA callback thread: no CUDA calls, only a wake-up
  static_cast<mans_server*>(p)->cv.notify_one();
}

// Worst-case output bytes of a request.
uint64_t output_need(const mans_server* s, const mans_request& r) {
  const uint64_t bytes = r.n_elems * elem_bytes((uint32_t)r.dtype);
  if (r.op == MANS_OP_DECOMPRESS) return bytes;
  if (r.dtype == MANS_U8) return ans_stream_bound(bytes);
  const uint32_t pct = s->cfg.merged_ratio_pct ? s->cfg.merged_ratio_pct : 210;
  uint64_t m = bytes / 100 * pct + (bytes % 100) * pct / 100 + 4096;
  if (s->cfg.plain) m = bytes / 10 * 21 + 4096;  // the single-buffer workspace's room
  if (m > 0xfffffff0ull) m = 0xfffffff0ull;
  return ans_stream_bound(m);
}

// Admit queued requests of the lane's direction; returns true if any.
bool admit(mans_server* s, Lane& L) {
  auto& q = s->queue[L.op];
  uint64_t bytes = 0;
  const uint32_t cap_items = s->cfg.plain ? 1u : s->max_items;
  while (!q.empty() && L.reqs.size() < cap_items) {
    Req& r = q.front();
    const uint64_t b = r.r.n_elems * elem_bytes((uint32_t)r.r.dtype);
    if (!L.reqs.empty() && bytes + b > s->cfg.max_batch_bytes) break;
    if (!r.r.d_out) {
      const uint64_t need = output_need(s, r.r);
      uint64_t off = 0;
      if (!s->arena.alloc(need, &off)) break;  // wait for memory (FIFO, no overtaking)
      r.in_arena = true;
      r.arena_off = off;
      r.arena_bytes = need;
      r.out = s->arena_base + off;
      r.out_cap = need;
    } else {
      r.out = static_cast<uint8_t*>(r.r.d_out);
      r.out_cap = r.r.out_capacity;
    }
    bytes += b;
    L.reqs.push_back(r);
    q.pop_front();
  }
  return !L.reqs.empty();
}

void fail_all(mans_server* s, Lane& L, mans_status st);

void launch(mans_server* s, Lane& L) {
  NvtxRange range(L.op == MANS_OP_COMPRESS ? "mans_server_launch_compress"
                                           : "mans_server_launch_decompress");
  const uint32_t n = (uint32_t)L.reqs.size();
  const uint64_t t = now_ns();
  for (auto& r : L.reqs) r.t_launch = t;
  mans_status st = MANS_OK;
  if (s->cfg.plain) {
    const Req& r = L.reqs[0];
    if (L.op == MANS_OP_COMPRESS)
      st = mans_compress(L.ws, r.r.dtype, r.r.d_in, r.r.n_elems, r.out, r.out_cap, L.d_sizes,
                         r.r.precision, reinterpret_cast<mans_stream_t>(L.stream));
    else
      st = mans_decompress(L.ws, r.r.dtype, r.r.d_in, r.r.in_bytes, r.out, r.r.n_elems,
                           reinterpret_cast<mans_stream_t>(L.stream));
    if (st == MANS_OK) st = workspace_enqueue_status(L.ws, L.h_status, L.h_detail, L.stream);
  } else {
    std::vector<mans_batch_item> items(n);
    for (uint32_t i = 0; i < n; ++i) {
      const Req& r = L.reqs[i];
      mans_batch_item& it = items[i];
      it.dtype = r.r.dtype;
      it.precision = r.r.precision;
      it.n_elems = r.r.n_elems;
      it.d_in = r.r.d_in;
      it.d_out = r.out;
      it.d_out_size = L.op == MANS_OP_COMPRESS ? L.d_sizes + i : nullptr;
      it.in_bytes = r.r.in_bytes;
      it.out_capacity = r.out_cap;
    }
    st = L.op == MANS_OP_COMPRESS
             ? mans_batch_compress(L.batch, items.data(), n, reinterpret_cast<mans_stream_t>(L.stream))
             : mans_batch_decompress(L.batch, items.data(), n, reinterpret_cast<mans_stream_t>(L.stream));
    if (st == MANS_OK) st = batch_enqueue_status(L.batch, n, L.h_status, L.h_detail, L.stream);
  }
  if (st == MANS_OK && L.op == MANS_OP_COMPRESS &&
      cudaMemcpyAsync(L.h_sizes, L.d_sizes, 8ull * n, cudaMemcpyDeviceToHost, L.stream) != cudaSuccess)
    st = MANS_ERR_CUDA;
  if (st == MANS_OK && cudaEventRecord(L.done, L.stream) != cudaSuccess) st = MANS_ERR_CUDA;
  if (st == MANS_OK && cudaLaunchHostFunc(L.stream, notify_host, s) != cudaSuccess) st = MANS_ERR_CUDA;
  if (st != MANS_OK) {
    fail_all(s, L, st);
    return;
  }
  L.busy = true;
  s->stats.launches++;
  s->stats.in_flight += n;
}

void complete_one(mans_server* s, Req& r, mans_status st, uint64_t detail, uint64_t out_bytes,
                  uint32_t batch_items) {
  mans_completion c{};
  c.ticket = r.ticket;
  c.tag = r.r.tag;
  c.status = st;
  c.detail = detail;
  c.d_out = r.out;
  c.out_bytes = st == MANS_OK ? out_bytes : 0;
  const uint64_t t = now_ns();
  c.queued_ns = r.t_launch > r.t_arrive ? r.t_launch - r.t_arrive : 0;
  c.latency_ns = t > r.t_arrive ? t - r.t_arrive : 0;
  c.batch_items = batch_items;
  if (r.in_arena) {
    if (st != MANS_OK) {
      s->arena.release(r.arena_off, r.arena_bytes);
      c.d_out = nullptr;
    } else {
      if (r.r.op == MANS_OP_COMPRESS) {
        s->arena.shrink(r.arena_off, r.arena_bytes, out_bytes);
        r.arena_bytes = out_bytes;
      }
      s->held[r.ticket] = {r.arena_off, r.arena_bytes};
    }
  }
  s->completed.push_back(c);
  s->stats.completed++;
}

void fail_all(mans_server* s, Lane& L, mans_status st) {
  for (auto& r : L.reqs) complete_one(s, r, st, 0, 0, (uint32_t)L.reqs.size());
  L.reqs.clear();
  s->done_cv.notify_all();
}

void finish(mans_server* s, Lane& L) {
  const uint32_t n = (uint32_t)L.reqs.size();
  const cudaError_t e = cudaEventSynchronize(L.done);  // already complete: returns at once
  for (uint32_t i = 0; i < n; ++i) {
    Req& r = L.reqs[i];
    mans_status st = e == cudaSuccess ? (mans_status)L.h_status[i] : MANS_ERR_CUDA;
    const uint64_t out_bytes = r.r.op == MANS_OP_COMPRESS
                                   ? L.h_sizes[i]
                                   : r.r.n_elems * elem_bytes((uint32_t)r.r.dtype);
    complete_one(s, r, st, e == cudaSuccess ? L.h_detail[i] : 0, out_bytes, n);
  }
  s->stats.in_flight -= n;
  L.reqs.clear();
  L.busy = false;
  s->done_cv.notify_all();
}

void scheduler(mans_server* s) {
  cudaSetDevice(s->device);
  std::unique_lock<std::mutex> lk(s->mu);
  while (true) {
    bool progress = false;
    for (auto& L : s->lanes) {
      if (L.busy && cudaEventQuery(L.done) != cudaErrorNotReady) {
        finish(s, L);
        progress = true;
      }
    }
    for (auto& L : s->lanes) {
      if (!L.busy && admit(s, L)) {
        launch(s, L);
        progress = true;
      }
    }
    bool idle = s->queue[0].empty() && s->queue[1].empty();
    for (auto& L : s->lanes) idle = idle && !L.busy;
    if (s->stop && idle) break;
    if (!progress) s->cv.wait_for(lk, std::chrono::microseconds(200));
  }
}

void destroy_lanes(mans_server* s) {
  for (auto& L : s->lanes) {
    if (L.stream) cudaStreamSynchronize(L.stream);
    if (L.batch) mans_batch_destroy(L.batch);
    if (L.ws) mans_workspace_destroy(L.ws);
    if (L.done) cudaEventDestroy(L.done);
    if (L.stream) cudaStreamDestroy(L.stream);
    if (L.h_status) cudaFreeHost(L.h_status);
    if (L.h_detail) cudaFreeHost(L.h_detail);
    if (L.h_sizes) cudaFreeHost(L.h_sizes);
    if (L.d_sizes) cudaFree(L.d_sizes);
  }
  s->lanes.clear();
}

}  // namespace

extern "C" {

uint64_t mans_clock_ns(void) { return now_ns(); }

mans_status mans_server_create(mans_server** out, const mans_server_config* cfg) {
  if (!out || !cfg || cfg->hbm_budget_bytes == 0) return MANS_ERR_INVALID_ARG;
  *out = nullptr;
  auto* s = new (std::nothrow) mans_server();
  if (!s) return MANS_ERR_OUT_OF_MEMORY;
  if (cudaGetDevice(&s->device) != cudaSuccess) {
    delete s;
    return MANS_ERR_CUDA;
  }
  s->cfg = *cfg;
  if (s->cfg.max_batch_bytes == 0) s->cfg.max_batch_bytes = cfg->hbm_budget_bytes / 8;
  if (s->cfg.max_batch_items == 0) s->cfg.max_batch_items = 1024;
  if (s->cfg.lanes == 0) s->cfg.lanes = s->cfg.plain ? 1 : 2;
  s->max_items = s->cfg.plain ? 1 : s->cfg.max_batch_items;
  uint64_t used = 0;
  mans_status st = MANS_OK;
  s->lanes.resize(2 * s->cfg.lanes);
  for (uint32_t k = 0; k < s->lanes.size() && st == MANS_OK; ++k) {
    Lane& L = s->lanes[k];
    L.op = (int)(k % 2);
    if (s->cfg.plain) {
      st = mans_workspace_create(&L.ws, s->cfg.max_batch_bytes, 0);
      if (st == MANS_OK) used += mans_workspace_device_bytes(L.ws);
    } else {
      st = mans_batch_create(&L.batch, s->max_items, s->cfg.max_batch_bytes, s->cfg.merged_ratio_pct);
      if (st == MANS_OK) used += mans_batch_device_bytes(L.batch);
    }
    if (st != MANS_OK) break;
    if (cudaStreamCreateWithFlags(&L.stream, cudaStreamNonBlocking) != cudaSuccess ||
        cudaEventCreateWithFlags(&L.done, cudaEventDisableTiming) != cudaSuccess ||
        cudaMallocHost(&L.h_status, 4ull * s->max_items) != cudaSuccess ||
        cudaMallocHost(&L.h_detail, 8ull * s->max_items) != cudaSuccess ||
        cudaMallocHost(&L.h_sizes, 8ull * s->max_items) != cudaSuccess ||
        cudaMalloc(&L.d_sizes, 8ull * s->max_items) != cudaSuccess) {
      st = MANS_ERR_OUT_OF_MEMORY;
      break;
    }
    used += 8ull * s->max_items;
  }
  if (st == MANS_OK && used + (64ull << 20) > cfg->hbm_budget_bytes) st = MANS_ERR_TOO_LARGE;
  if (st == MANS_OK) {
    const uint64_t arena = (cfg->hbm_budget_bytes - used) / 256 * 256;
    if (cudaMalloc(&s->arena_base, arena) != cudaSuccess) {
      cudaGetLastError();
      st = MANS_ERR_OUT_OF_MEMORY;
    } else {
      s->arena.reset(arena);
    }
  }
  if (st != MANS_OK) {
    destroy_lanes(s);
    if (s->arena_base) cudaFree(s->arena_base);
    delete s;
    return st;
  }
  s->stats.arena_bytes = s->arena.size();
  s->stats.device_bytes = used + s->arena.size();
  s->sched = std::thread(scheduler, s);
  *out = s;
  return MANS_OK;
}

mans_status mans_server_destroy(mans_server* s) {
  if (!s) return MANS_ERR_INVALID_ARG;
  {
    std::lock_guard<std::mutex> lk(s->mu);
    s->stop = true;
  }
  s->cv.notify_all();
  if (s->sched.joinable()) s->sched.join();
  int prev = 0;
  cudaGetDevice(&prev);
  cudaSetDevice(s->device);
  destroy_lanes(s);
  if (s->arena_base) cudaFree(s->arena_base);
  cudaSetDevice(prev);
  delete s;
  return MANS_OK;
}

mans_status mans_server_submit(mans_server* s, const mans_request* r, uint64_t* ticket) {
  if (!s || !r) return MANS_ERR_INVALID_ARG;
  if (r->op != MANS_OP_COMPRESS && r->op != MANS_OP_DECOMPRESS) return MANS_ERR_INVALID_ARG;
  const uint64_t eb = elem_bytes((uint32_t)r->dtype);
  if (eb == 0) return MANS_ERR_INVALID_ARG;
  const uint64_t bytes = r->n_elems * eb;
  if (r->op == MANS_OP_COMPRESS && (r->precision < 9 || r->precision > 11))
    return MANS_ERR_UNSUPPORTED_PRECISION;
  if ((!r->d_in && (bytes || r->op == MANS_OP_DECOMPRESS)) || (r->d_out && !r->out_capacity && bytes))
    return MANS_ERR_INVALID_ARG;
  if ((r->d_in && !aligned16(r->d_in)) || (r->d_out && !aligned16(r->d_out))) return MANS_ERR_ALIGNMENT;
  if (bytes > s->cfg.max_batch_bytes) return MANS_ERR_TOO_LARGE;
  if (!r->d_out && align256(output_need(s, *r)) > s->arena.size()) return MANS_ERR_TOO_LARGE;
  Req q;
  q.r = *r;
  q.t_arrive = r->arrival_ns ? r->arrival_ns : now_ns();
  {
    std::lock_guard<std::mutex> lk(s->mu);
    if (s->stop) return MANS_ERR_INVALID_ARG;
    q.ticket = s->next_ticket++;
    s->queue[r->op].push_back(q);
    s->stats.submitted++;
  }
  s->cv.notify_one();
  if (ticket) *ticket = q.ticket;
  return MANS_OK;
}

mans_status mans_server_poll(mans_server* s, mans_completion* out, uint32_t max, uint32_t* n,
                             uint32_t timeout_us) {
  if (!s || !n || (!out && max)) return MANS_ERR_INVALID_ARG;
  std::unique_lock<std::mutex> lk(s->mu);
  if (s->completed.empty() && timeout_us)
    s->done_cv.wait_for(lk, std::chrono::microseconds(timeout_us),
                        [s] { return !s->completed.empty(); });
  uint32_t k = 0;
  while (k < max && !s->completed.empty()) {
    out[k++] = s->completed.front();
    s->completed.pop_front();
  }
  *n = k;
  return MANS_OK;
}

mans_status mans_server_release(mans_server* s, uint64_t ticket) {
  if (!s) return MANS_ERR_INVALID_ARG;
  {
    std::lock_guard<std::mutex> lk(s->mu);
    auto it = s->held.find(ticket);
    if (it == s->held.end()) return MANS_ERR_INVALID_ARG;
    s->arena.release(it->second.first, it->second.second);
    s->held.erase(it);
  }
  s->cv.notify_one();
  return MANS_OK;
}

mans_status mans_server_get_stats(mans_server* s, mans_server_stats* out) {
  if (!s || !out) return MANS_ERR_INVALID_ARG;
  std::lock_guard<std::mutex> lk(s->mu);
  *out = s->stats;
  out->queued = s->queue[0].size() + s->queue[1].size();
  out->arena_used = s->arena.used();
  out->arena_peak = s->arena.peak();
  return MANS_OK;
}

// Diagnostic: run a sequence of arena operations on a host-only arena (no
// device memory): ops[i] = {kind, a, b} with kind 0 alloc(a) -> result
// offset or ~0, 1 release(a = offset, b = bytes), 2 shrink(a = offset, b =
// new bytes of the block allocated at a, whose size is taken from the
// matching alloc). Returns the used bytes after the sequence.
uint64_t mans_debug_arena(uint64_t size, const uint64_t* ops, uint32_t n_ops, uint64_t* results) {
  Arena a;
  a.reset(size);
  std::map<uint64_t, uint64_t> sizes;
  for (uint32_t i = 0; i < n_ops; ++i) {
    const uint64_t kind = ops[3 * i], x = ops[3 * i + 1], y = ops[3 * i + 2];
    uint64_t r = 0;
    if (kind == 0) {
      uint64_t off = 0;
      if (a.alloc(x, &off)) {
        r = off;
        sizes[off] = x;
      } else {
        r = ~0ull;
      }
    } else if (kind == 1) {
      a.release(x, y);
      sizes.erase(x);
    } else {
      a.shrink(x, sizes[x], y);
      sizes[x] = y;
    }
    if (results) results[i] = r;
  }
  return a.used();
}

}  // extern "C"
