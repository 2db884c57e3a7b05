/*
 * mans.h -- C ABI of the B200-native MANS codec (libmans_b200.so).
 *
 * MANS compresses 16/32-bit integer arrays in two stages: the ADM byte
 * mapping (a per-group center, one code byte per element and a unary
 * bit-signal plane, with a prefix-sum compaction), then a warp-interleaved
 * byte rANS over the mapped bytes. The streams are byte-for-byte those of the
 * reference implementation (hpdps-group/MANS): the rANS stream is the
 * coalesced layout of include/ans/GpuANSCodec.h and the uint16 mapping is the
 * merged layout written by mapping/nv/mappingV15_fused_uint16.cu:933-957.
 *
 * All pointers named d_* are device pointers on the calling thread's current
 * device; all work is enqueued on `stream` and returns without synchronising.
 * Device buffers passed as inputs or outputs must be 16-byte aligned.
 * Functions return a mans_status for errors detectable on the host; errors
 * that depend on the data (an output or workspace that turns out too small, a
 * corrupt stream, an expired wait) are recorded in the workspace and read
 * with mans_workspace_status() after the stream has been synchronised.
 */
#ifndef MANS_H
#define MANS_H

#include <stddef.h>
#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

typedef struct CUstream_st* mans_stream_t; /* binary-compatible with cudaStream_t */

typedef enum mans_status {
  MANS_OK = 0,
  MANS_ERR_INVALID_ARG = 1,          /* null pointer, bad dtype, size out of range */
  MANS_ERR_UNSUPPORTED_PRECISION = 2,/* precision not in {9,10,11} */
  MANS_ERR_ALIGNMENT = 3,            /* device pointer not 16-byte aligned */
  MANS_ERR_TOO_LARGE = 4,            /* input exceeds the workspace capacity */
  MANS_ERR_CUDA = 5,                 /* a CUDA runtime call failed */
  MANS_ERR_OUT_OF_MEMORY = 6,        /* workspace allocation failed */
  MANS_ERR_BAD_STREAM = 7,           /* magic, version, precision or sizes invalid */
  MANS_ERR_OUTPUT_OVERFLOW = 8,      /* compressed stream exceeds out_capacity */
  MANS_ERR_WORKSPACE_OVERFLOW = 9,   /* mapped bytes exceed the workspace */
  MANS_ERR_CORRUPT = 10,             /* decode consistency check failed */
  MANS_ERR_TIMEOUT = 11              /* a bounded device wait expired */
} mans_status;

typedef enum mans_dtype {
  MANS_U8 = 1,  /* raw bytes: rANS only (the include/ans codec) */
  MANS_U16 = 2, /* uint16: ADM unary-signal mapping + rANS */
  MANS_U32 = 4  /* uint32: ADM escape-byte mapping + rANS */
} mans_dtype;

typedef struct mans_workspace mans_workspace;

/* ------------------------------------------------------------------------
 * Workspace: device scratch reused across calls, so a call allocates
 * nothing. max_input_bytes bounds the uncompressed size of one call;
 * merged_capacity bounds the mapped (ADM) bytes (0 = 2.1 x max_input_bytes,
 * which always suffices for MANS_U32 and MANS_U8, and for MANS_U16 data whose
 * values stay within a few thousand of their 512-element group's mean; pass
 * mans_max_mapped_size(MANS_U16, n) to accept any uint16 input). A workspace
 * serves one stream at a time.
 * ---------------------------------------------------------------------- */
mans_status mans_workspace_create(mans_workspace** ws, uint64_t max_input_bytes,
                                  uint64_t merged_capacity);
mans_status mans_workspace_destroy(mans_workspace* ws);
/* Device bytes held by the workspace. */
uint64_t mans_workspace_device_bytes(const mans_workspace* ws);
/* Synchronise `stream`, then return (and clear) the first device-side error
 * recorded since the last call; *detail receives e.g. the bytes needed. */
mans_status mans_workspace_status(mans_workspace* ws, mans_stream_t stream, uint64_t* detail);

/* Opt-in per-kernel timing: when enabled, CUDA events are recorded on the
 * call's stream around every kernel of up to 128 compress and 128 decompress
 * calls (no synchronisation is added). */
mans_status mans_workspace_set_timing(mans_workspace* ws, int enable);
/* Summed milliseconds, over the calls recorded since the last read, of the
 * compress kernels (ms[0] mapping or histogram, ms[1] rANS encode) and the
 * decompress kernels (ms[2] rANS decode, ms[3] inverse mapping); calls[0..1]
 * (optional) receive the numbers of compress and decompress calls. Waits for
 * the recorded events, then clears the record. */
mans_status mans_workspace_kernel_times(mans_workspace* ws, float ms[4], int calls[2]);

/* Worst-case mapped (ADM) bytes of n elements of dtype, in any layout, for
 * any values. uint16: a lane's unary stream holds at most 16 x 521 bits
 * (k <= ceil(65535/126)), so a 512-element group maps to at most 32 x 1,042
 * bit bytes plus one code byte per element and its header fields -- about 33
 * bytes per input byte for pathological data, against ~1.2 for smooth data.
 * uint32: at most 8 record bytes per element plus 40 header bytes per group
 * (~2.02 x the input). MANS_U8: n. Pass it as the workspace's
 * merged_capacity to accept any uint16 input. */
uint64_t mans_max_mapped_size(mans_dtype dtype, uint64_t n_elems);
/* Worst-case rANS stream bytes for mapped_bytes of rANS input (32 lanes x 90
 * words per 4 KiB block plus the header, pdf, states and block words). */
uint64_t mans_stream_bound(uint64_t mapped_bytes);
/* Upper bound of the compressed size for n elements of dtype, for any values:
 * mans_stream_bound(min(mans_max_mapped_size(dtype, n), 0xfffffff0)). Mapped
 * buffers beyond 0xfffffff0 bytes (the rANS header's u32 counts) are
 * rejected, so the clamp keeps the bound valid for every stream that can
 * exist. The data must also fit the workspace's merged_capacity (see
 * mans_workspace_create) or the call reports MANS_ERR_WORKSPACE_OVERFLOW. */
uint64_t mans_max_compressed_size(mans_dtype dtype, uint64_t n_elems);

/* ------------------------------------------------------------------------
 * MANS compress: d_out receives the rANS stream of the mapped bytes and
 * *d_out_size (device, u64) its length. For MANS_U8 this is exactly
 * multibyte_ans::ansEncode (include/ans/GpuANSEncode.h:286); for MANS_U16 it
 * is ansEncode applied to the V15 merged buffer of the input.
 * ---------------------------------------------------------------------- */
mans_status mans_compress(mans_workspace* ws, mans_dtype dtype, const void* d_in,
                          uint64_t n_elems, void* d_out, uint64_t out_capacity,
                          uint64_t* d_out_size, int precision, mans_stream_t stream);

/* MANS decompress of a stream produced by mans_compress. n_elems travels out
 * of band, as in the reference (examples/compress.cu:79-97). For MANS_U8 this
 * is multibyte_ans::ansDecode (include/ans/GpuANSDecode.h:379). */
mans_status mans_decompress(mans_workspace* ws, mans_dtype dtype, const void* d_in,
                            uint64_t in_size, void* d_out, uint64_t n_elems,
                            mans_stream_t stream);

/* ------------------------------------------------------------------------
 * On-disk compatibility layouts of the uint16 mapped buffer. NATIVE is the
 * V15 merged layout for MANS_U16 (mapping/nv/mappingV15_fused_uint16.cu
 * :933-957) and the decodable record layout for MANS_U32. V12 replaces the
 * i32 prefix header by u16 group lengths (mappingV12_bit-adm-thrust-prefixsum.cu
 * :606-634; lanes past n are 0xFF); CPUV2 writes g + 1 prefix words, the last
 * one the total (mapping/cpu/mappingcpuV2.cpp:117-121, 271-285). The layout
 * changes the mapped bytes and so the stream; decode with the same layout.
 * ---------------------------------------------------------------------- */
typedef enum mans_layout {
  MANS_LAYOUT_NATIVE = 0,
  MANS_LAYOUT_V12 = 1,   /* MANS_U16 only */
  MANS_LAYOUT_CPUV2 = 2  /* MANS_U16 only */
} mans_layout;

mans_status mans_compress_ex(mans_workspace* ws, mans_dtype dtype, mans_layout layout,
                             const void* d_in, uint64_t n_elems, void* d_out,
                             uint64_t out_capacity, uint64_t* d_out_size, int precision,
                             mans_stream_t stream);
mans_status mans_decompress_ex(mans_workspace* ws, mans_dtype dtype, mans_layout layout,
                               const void* d_in, uint64_t in_size, void* d_out, uint64_t n_elems,
                               mans_stream_t stream);
/* The mapping alone: d_out receives the mapped buffer exactly as the
 * reference's mapping programs write it to disk (for MANS_U32 the record
 * layout, whose records section is mappingV9_fuse.cu's output), and
 * *d_out_size (device, u64) its size. MANS_U16 / MANS_U32 only. */
mans_status mans_adm_map(mans_workspace* ws, mans_dtype dtype, mans_layout layout,
                         const void* d_in, uint64_t n_elems, void* d_out, uint64_t out_capacity,
                         uint64_t* d_out_size, mans_stream_t stream);
/* Inverse of mans_adm_map: in_size mapped bytes at d_in back to n_elems values. */
mans_status mans_adm_unmap(mans_workspace* ws, mans_dtype dtype, mans_layout layout,
                           const void* d_in, uint64_t in_size, void* d_out, uint64_t n_elems,
                           mans_stream_t stream);

/* ------------------------------------------------------------------------
 * Reference-compatible rANS entry points (include/ans, src/GpuANS.cu). Same
 * arguments and meaning as the reference; they run on a library-owned
 * workspace per (device, stream) that is created on first use, so the first
 * call on a stream allocates. Errors the reference could only print are
 * returned as a status. They may be called from several host threads, on one
 * stream or on several: each call enqueues its launches under a lock, so the
 * launches of one call stay adjacent in stream order, and a workspace that
 * grows is freed only after the work queued on it has finished.
 * ---------------------------------------------------------------------- */
/* multibyte_ans::ansEncode, include/ans/GpuANSEncode.h:286. d_out must hold
 * mans_ans_max_compressed_size(in_size) bytes; *d_out_size is a device u32. */
mans_status mans_ans_encode(int precision, const uint8_t* d_in, uint32_t in_size,
                            uint8_t* d_out, uint32_t* d_out_size, mans_stream_t stream);
/* multibyte_ans::ansDecode, include/ans/GpuANSDecode.h:379. d_out must hold
 * the uncompressed size recorded in the stream. */
mans_status mans_ans_decode(int precision, const uint8_t* d_in, uint8_t* d_out,
                            mans_stream_t stream);
/* multibyte_ans::ansEncodeBatch / ansDecodeBatch, src/GpuANS.cu:16,33. */
mans_status mans_ans_encode_batch(int precision, const uint8_t* d_in, uint32_t in_size,
                                  uint8_t* d_out, uint32_t* d_out_size, mans_stream_t stream);
mans_status mans_ans_decode_batch(int precision, const uint8_t* d_in, uint8_t* d_out,
                                  mans_stream_t stream);
/* multibyte_ans::getMaxCompressedSize, include/ans/GpuANSCodec.h:237. Unlike
 * the reference's 1.25x estimate this is a true upper bound. */
uint32_t mans_ans_max_compressed_size(uint32_t in_size);
/* First device-side error of the library-owned workspace of `stream`. */
mans_status mans_ans_last_status(mans_stream_t stream, uint64_t* detail);

/* rANS encode that allocates nothing, for callers that cannot call
 * cudaMalloc on their call path (e.g. a real-time loop that cannot absorb
 * cudaMalloc's latency or implicit synchronisation, or a process whose device
 * memory is reserved up front by another allocator). No counterpart in the
 * reference; same arguments and output as mans_ans_encode. Its scratch is a
 * fixed ~132 KiB device array inside the library, held on every GPU that
 * loads the library until exit; inputs above 64 MiB are rejected with
 * MANS_ERR_TOO_LARGE. The first call on a device looks up that array's
 * address (make it before any stream capture). All calls share the array:
 * calls that overlap on the GPU race, so issue them on one stream. */
mans_status mans_ans_encode_noalloc(int precision, const uint8_t* d_in, uint32_t in_size,
                                    uint8_t* d_out, uint32_t* d_out_size, mans_stream_t stream);
/* The device-side status of the last mans_ans_encode_noalloc call on the
 * current device (an expired bounded wait, a stream past its bound): waits
 * for `stream`, then copies the status and *detail out of the fixed scratch
 * array, allocating nothing. The next mans_ans_encode_noalloc call clears it,
 * so read it before issuing the next call. MANS_OK when no call was made. */
mans_status mans_ans_noalloc_status(mans_stream_t stream, uint64_t* detail);

/* ------------------------------------------------------------------------
 * Self-describing frames: a 64-byte header in front of a MANS stream, so
 * a frame decodes with nothing kept out of band. Header, little endian:
 *   0 u32 magic 0x534e414d ("MANS")   4 u16 version (1)
 *   6 u8 dtype (1, 2, 4)              7 u8 layout (0, 1, 2)
 *   8 u8 precision (9..11)            9 u8 flags (0)
 *  10 u16 header bytes (64)          12 u32 reserved (0)
 *  16 u64 element count              24 u64 mapped bytes (the rANS input)
 *  32 u64 stream bytes               40 24 reserved bytes (0)
 * The reference keeps the
 * element count and type outside the stream (examples/compress.cu:79-97) and,
 * for uint32, writes no centers or lengths at all (mappingV9_fuse.cu:998);
 * the frame plus the record layout's header carry both.
 * ---------------------------------------------------------------------- */
typedef struct mans_frame_info {
  mans_dtype dtype;
  mans_layout layout;
  int precision;
  uint32_t header_bytes;   /* 64 */
  uint64_t n_elems;
  uint64_t mapped_bytes;   /* ADM output = rANS input */
  uint64_t stream_bytes;   /* MANS stream after the header */
} mans_frame_info;

/* Upper bound of a frame's size. */
uint64_t mans_frame_max_size(mans_dtype dtype, uint64_t n_elems);
/* Compress into a frame at d_out (16-byte aligned); *d_out_size (device u64)
 * receives the frame size. */
mans_status mans_frame_compress(mans_workspace* ws, mans_dtype dtype, mans_layout layout,
                                const void* d_in, uint64_t n_elems, void* d_out,
                                uint64_t out_capacity, uint64_t* d_out_size, int precision,
                                mans_stream_t stream);
/* Parse and check a frame header held in HOST memory (no GPU needed); avail =
 * bytes of the frame available (~0 when unknown), checked against its size. */
mans_status mans_frame_parse(const void* header, uint64_t avail, mans_frame_info* info);
/* Decompress the frame at d_frame (device) described by info (from
 * mans_frame_parse) into d_out (out_capacity bytes). */
mans_status mans_frame_decompress(mans_workspace* ws, const mans_frame_info* info,
                                  const void* d_frame, void* d_out, uint64_t out_capacity,
                                  mans_stream_t stream);

/* ------------------------------------------------------------------------
 * Batched MANS: many buffers of uneven size and element type in one
 * persistent launch per stage (a device work queue over every buffer's
 * mapping groups and rANS blocks). Each buffer's stream is byte-identical to
 * mans_compress of that buffer alone; errors are kept per buffer. The
 * reference codes one buffer per call (examples/compress.cu:55-97 loops over
 * files, src/GpuANS.cu:16-48 over whole inputs). Calls on one batch workspace
 * must be ordered (one stream). Every call's bounds live on the device, so a
 * call can be captured in a CUDA graph and replayed: each capture keeps its
 * descriptors in the next of four host buffers, so the graphs of a
 * workspace's last four captures may be replayed.
 * ---------------------------------------------------------------------- */
typedef struct mans_batch mans_batch;

typedef struct mans_batch_item {
  mans_dtype dtype;
  int precision;          /* compress: probability bits, 9..11 */
  uint64_t n_elems;       /* elements of the uncompressed buffer */
  const void* d_in;       /* compress: values; decompress: stream (16-byte aligned) */
  void* d_out;            /* compress: stream; decompress: values (16-byte aligned) */
  uint64_t* d_out_size;   /* compress: device u64 receiving the stream size (may be NULL) */
  uint64_t in_bytes;      /* decompress: stream bytes available at d_in */
  uint64_t out_capacity;  /* compress: bytes available at d_out */
} mans_batch_item;

/* Workspace for batches of up to max_items buffers totalling at most
 * max_total_bytes uncompressed bytes (on the current device). Each MANS_U16 /
 * MANS_U32 buffer gets room for merged_ratio_pct percent of its bytes of
 * mapped data, plus 4 KiB (0 = 210, the single-buffer default, enough for
 * any MANS_U32 input); a buffer whose mapping needs more fails alone with
 * MANS_ERR_WORKSPACE_OVERFLOW. */
mans_status mans_batch_create(mans_batch** b, uint32_t max_items, uint64_t max_total_bytes,
                              uint32_t merged_ratio_pct);
mans_status mans_batch_destroy(mans_batch* b);
uint64_t mans_batch_device_bytes(const mans_batch* b);
/* Enqueue on `stream`; host-side argument errors are returned at once. */
mans_status mans_batch_compress(mans_batch* b, const mans_batch_item* items, uint32_t count,
                                mans_stream_t stream);
mans_status mans_batch_decompress(mans_batch* b, const mans_batch_item* items, uint32_t count,
                                  mans_stream_t stream);
/* Synchronise `stream`; return the batch's first device-side error and fill
 * the first `count` buffers' statuses and details (either may be NULL). */
mans_status mans_batch_status(mans_batch* b, mans_stream_t stream, uint32_t* item_status,
                              uint64_t* item_detail, uint32_t count);
/* Opt-in stage timing: when enabled, CUDA events are recorded around the
 * stages of up to 64 compress and 64 decompress calls that are not being
 * captured (no synchronisation is added). */
mans_status mans_batch_set_timing(mans_batch* b, int enable);
/* Summed milliseconds of the recorded calls' stages (ms[0..2] compress: map
 * with histogram, plan, encode; ms[3..5] decompress: plan, decode, unmap) and
 * the numbers of recorded calls; waits for the events, then clears them. */
mans_status mans_batch_stage_times(mans_batch* b, float ms[6], int calls[2]);
/* Schedule: resident CTAs per SM of each stage (map, plan, encode,
 * decode plan, decode, unmap); never changes the bytes produced. */
mans_status mans_batch_get_schedule(const mans_batch* b, int ctas_per_sm[6],
                                    int max_ctas_per_sm[6]);
mans_status mans_batch_set_schedule(mans_batch* b, const int ctas_per_sm[6]);
/* The full schedule, per stage (same order): resident CTAs per SM (the map
 * stage counts CTAs of 8 warps), warps per CTA (4 or 8 for the map stage, 8
 * for the others) and the L2 prefetch distance in grids of units ahead (0 to
 * 2 for the map and encode stages, 0 for the others). Never changes the bytes
 * produced. limits (may be NULL) receives the largest accepted values. */
typedef struct mans_batch_schedule {
  int ctas_per_sm[6];
  int warps_per_cta[6];
  int prefetch_grids[6];
} mans_batch_schedule;
mans_status mans_batch_get_schedule_ex(const mans_batch* b, mans_batch_schedule* sch,
                                       mans_batch_schedule* limits);
mans_status mans_batch_set_schedule_ex(mans_batch* b, const mans_batch_schedule* sch);
/* Time candidate schedules on this batch (it is compressed several times):
 * coordinate descent over the map stage's CTAs per SM, warps per CTA and
 * prefetch distance, then the encode stage's CTAs per SM and prefetch
 * distance. Keeps the fastest schedule whose streams match the starting
 * schedule's checksum, and reports its time. */
mans_status mans_batch_autotune(mans_batch* b, const mans_batch_item* items, uint32_t count,
                                mans_stream_t stream, float* best_ms);

/* ------------------------------------------------------------------------
 * Serving loop: a scheduler thread inside the library admits mixed compress
 * and decompress requests against an HBM budget and folds whatever is queued
 * into the next batched launch (continuous batching: several launches per
 * direction are in flight on their own streams, and requests that arrive
 * meanwhile form the next ones). All device memory the server holds -- batch
 * workspaces and an arena for results -- is allocated at creation within the
 * budget. The reference has no serving form; each result is byte-identical to
 * mans_compress / mans_decompress of that request alone.
 * ---------------------------------------------------------------------- */
typedef struct mans_server mans_server;

typedef enum mans_op { MANS_OP_COMPRESS = 0, MANS_OP_DECOMPRESS = 1 } mans_op;

typedef struct mans_server_config {
  uint64_t hbm_budget_bytes;  /* device memory the server may hold */
  uint64_t max_batch_bytes;   /* uncompressed bytes of one launch, and of one request
                                 (0 = budget / 8) */
  uint32_t max_batch_items;   /* requests of one launch (0 = 1024) */
  uint32_t lanes;             /* launches in flight per direction (0 = 2; plain: 1) */
  uint32_t merged_ratio_pct;  /* mapped-byte room per buffer, see mans_batch_create */
  int plain;                  /* 1: one request per launch through mans_compress /
                                 mans_decompress (the per-request baseline) */
} mans_server_config;

typedef struct mans_request {
  mans_op op;
  mans_dtype dtype;
  int precision;          /* compress: 9..11 */
  uint32_t pad;
  uint64_t n_elems;       /* uncompressed elements */
  const void* d_in;       /* device; compress: values, decompress: stream (16-byte aligned) */
  uint64_t in_bytes;      /* decompress: stream bytes */
  void* d_out;            /* caller-owned device output, or NULL for one from the arena */
  uint64_t out_capacity;  /* bytes at d_out */
  uint64_t tag;           /* returned in the completion */
  uint64_t arrival_ns;    /* arrival time on mans_clock_ns() (0 = at submission) */
} mans_request;

typedef struct mans_completion {
  uint64_t ticket;
  uint64_t tag;
  mans_status status;     /* this request's own status */
  uint32_t batch_items;   /* requests in the launch that served it */
  uint64_t detail;
  void* d_out;            /* the result (device); arena results stay valid until released */
  uint64_t out_bytes;     /* stream bytes (compress) or value bytes (decompress) */
  uint64_t queued_ns;     /* arrival -> launch */
  uint64_t latency_ns;    /* arrival -> completion seen by the scheduler */
} mans_completion;

typedef struct mans_server_stats {
  uint64_t submitted, completed, launches, in_flight, queued;
  uint64_t arena_bytes, arena_used, arena_peak, device_bytes;
} mans_server_stats;

/* Monotonic clock of the server (ns), for arrival_ns. */
uint64_t mans_clock_ns(void);
mans_status mans_server_create(mans_server** s, const mans_server_config* cfg);
/* Finishes every submitted request, then frees everything. */
mans_status mans_server_destroy(mans_server* s);
/* Validates and queues a request (MANS_ERR_TOO_LARGE when it can never fit). */
mans_status mans_server_submit(mans_server* s, const mans_request* r, uint64_t* ticket);
/* Up to max completions; waits up to timeout_us for the first (0 = no wait). */
mans_status mans_server_poll(mans_server* s, mans_completion* out, uint32_t max, uint32_t* n,
                             uint32_t timeout_us);
/* Returns an arena result's memory to the server. */
mans_status mans_server_release(mans_server* s, uint64_t ticket);
mans_status mans_server_get_stats(mans_server* s, mans_server_stats* out);
/* Diagnostic: the server's arena allocator on the host (no device memory). */
uint64_t mans_debug_arena(uint64_t size, const uint64_t* ops, uint32_t n_ops, uint64_t* results);

/* Library version string. */
const char* mans_version(void);

/* Diagnostic of the failure path: runs one bounded device wait that nothing
 * ever satisfies (a look-back over flags no unit publishes) on the current
 * device and returns the status the kernel recorded -- MANS_ERR_TIMEOUT after
 * about a second or a few -- and the elapsed time. No fault, trap or hang:
 * the context stays usable. Allocates and frees its own scratch. */
mans_status mans_debug_bounded_wait(uint32_t* status, float* elapsed_ms);

/* Diagnostic: the encoder's division-table entry {reciprocal, packed} for a
 * symbol of probability pdf / 2^p and cumulative frequency cdf; packed =
 * shift | bias << 5 | (2^p - pdf) << 20, with x / pdf = umulhi(x, rcp) >>
 * shift for every state the encoder holds. */
void mans_debug_enc_entry(uint32_t pdf, uint32_t cdf, int p, uint32_t out[2]);

#ifdef __cplusplus
}
#endif
#endif /* MANS_H */
