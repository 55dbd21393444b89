/*
 * orot_b200.h -- C ABI of the B200 DEFLATE compression engine (liborot_b200.so).
 *
 * The first block of entry points has exactly the signatures, enum values and
 * error conventions of orot's public DEFLATE compress API, so a program (or a
 * cgo / ctypes / JNI binding) that calls orot for compression can link this
 * library instead.  Each declaration cites the reference interface it
 * replaces (include/orot/deflate.h in daramkun/orot).  All buffers are host
 * memory owned by the caller; device memory is managed inside the library.
 *
 * The second block is this engine's own extension: batches of buffers kept
 * on the device, compressed by one pass of kernels (optionally replayed from
 * a CUDA graph), and a continuous-batching server.
 */
#ifndef OROT_B200_H
#define OROT_B200_H

#include <stddef.h>
#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

/* deflate_result -- include/orot/deflate.h:15-25 (same values) */
typedef enum deflate_result {
  DEFLATE_OK = 0,
  DEFLATE_STREAM_END = 1,
  DEFLATE_NEED_INPUT = 2,
  DEFLATE_NEED_OUTPUT = 3,
  DEFLATE_DATA_ERROR = -1,
  DEFLATE_MEM_ERROR = -2,
  DEFLATE_BUF_ERROR = -3,
  DEFLATE_VERSION_ERROR = -4,
  DEFLATE_PARAM_ERROR = -5
} deflate_result;

/* deflate_format -- include/orot/deflate.h:28-32 (same values) */
typedef enum deflate_format {
  DEFLATE_FORMAT_RAW = 0,  /* RFC 1951 */
  DEFLATE_FORMAT_ZLIB = 1, /* RFC 1950, Adler-32 trailer */
  DEFLATE_FORMAT_GZIP = 2  /* RFC 1952, CRC-32 trailer */
} deflate_format;

/* levels -- include/orot/deflate.h:35-39; values outside 0..12 are clamped
 * exactly as src/deflate/lz77.cpp:33-34 does. */
#define DEFLATE_LEVEL_STORE 0
#define DEFLATE_LEVEL_FAST 1
#define DEFLATE_LEVEL_DEFAULT 6
#define DEFLATE_LEVEL_BETTER 9
#define DEFLATE_LEVEL_MAX 12

/* deflate_allocator -- include/orot/deflate.h:50-54 */
typedef struct deflate_allocator {
  void* (*alloc)(void* opaque, size_t size, size_t alignment);
  void (*free)(void* opaque, void* ptr);
  void* opaque;
} deflate_allocator;

/* Replaces deflate_set_allocator, include/orot/deflate.h:61.  Stored and
 * otherwise unused, as in the reference (src/api/deflate_api.cpp:75-77):
 * device memory never comes from a host allocator. */
void deflate_set_allocator(const deflate_allocator* alloc);

/* Replaces deflate_compress_bound, include/orot/deflate.h:66.
 * n + n/4096 + n/16384 + n/2^25 + 13, plus 6 (zlib) or 18 (gzip). */
size_t deflate_compress_bound(size_t in_size, deflate_format format);

/* Replaces deflate_compress, include/orot/deflate.h:72-77.  One DEFLATE
 * block for the whole input; levels 1-3 give byte-identical output to the
 * reference.  Returns the compressed size, or 0 if out_capacity is below
 * deflate_compress_bound() or on any device error.  Positions inside one
 * block are 32-bit on the device: an input above 4 GiB - 64 KiB returns 0
 * ("segment larger than 4 GiB"); deflate_parallel_compress, whose chunks are
 * independent, takes inputs of any size. */
size_t deflate_compress(const void* in, size_t in_size, void* out, size_t out_capacity, int level,
                        deflate_format format);

/* Replaces the parallel API, include/orot/deflate.h:122-145.  num_threads is
 * accepted and ignored (the chunks run on the GPU); block_size 0 selects
 * 128 KiB / 512 KiB / 1 MiB by level as src/parallel/parallel_compressor.cpp:16-20.
 * deflate_parallel_compress returns 0 for a NULL context, or when the stream
 * does not fit out_capacity. */
typedef struct deflate_parallel_ctx deflate_parallel_ctx;
deflate_parallel_ctx* deflate_parallel_new(int level, deflate_format format, int num_threads, size_t block_size);
void deflate_parallel_free(deflate_parallel_ctx* ctx);
size_t deflate_parallel_compress(deflate_parallel_ctx* ctx, const void* in, size_t in_size, void* out,
                                 size_t out_capacity);

/* Replace deflate_adler32 / deflate_crc32, include/orot/deflate.h:149-150.
 * CRC-32 is the IEEE polynomial (the reference's scalar and ARM paths,
 * src/simd/simd_detect.cpp:33-50). */
uint32_t deflate_adler32(uint32_t initial, const void* data, size_t len);
uint32_t deflate_crc32(uint32_t initial, const void* data, size_t len);

/* deflate_flush -- include/orot/deflate.h:42-47 (same values) */
typedef enum deflate_flush {
  DEFLATE_NO_FLUSH = 0,
  DEFLATE_SYNC_FLUSH = 1,
  DEFLATE_FULL_FLUSH = 2,
  DEFLATE_FINISH = 3
} deflate_flush;

/* Replaces the streaming compressor, include/orot/deflate.h:92-108
 * (src/api/stream_api.cpp:134-247).  Input is compressed on the GPU in 1 MiB
 * chunks, each an independent part of the stream that ends on a byte
 * boundary; SYNC and FULL flush compress the partial chunk (all input so far
 * becomes decodable), FINISH writes the last part and the zlib / gzip trailer
 * and then returns DEFLATE_STREAM_END.  Returns DEFLATE_OK when the input is
 * consumed and no output is pending, DEFLATE_NEED_OUTPUT when *avail_out ran
 * out first (call again with more room), DEFLATE_PARAM_ERROR for bad
 * arguments or input after the end, DEFLATE_MEM_ERROR on a device failure. */
typedef struct deflate_stream deflate_stream;
deflate_stream* deflate_stream_new(int level, deflate_format format);
void deflate_stream_free(deflate_stream* s);
deflate_result deflate_stream_compress(deflate_stream* s, const uint8_t** next_in, size_t* avail_in,
                                       uint8_t** next_out, size_t* avail_out, deflate_flush flush);

/* Replaces deflate_decompress, include/orot/deflate.h:79-89 (whole buffer,
 * src/api/deflate_api.cpp:138-219), decoded on the GPU: raw, zlib (header
 * rules and Adler-32 trailer checked) or gzip (header flags skipped, CRC-32
 * and ISIZE checked).  Returns DEFLATE_OK with *actual_out_size set;
 * DEFLATE_DATA_ERROR for corrupt input, truncated input or an output buffer
 * that is too small (as the reference); DEFLATE_PARAM_ERROR for bad
 * arguments. */
deflate_result deflate_decompress(const void* in, size_t in_size, void* out, size_t out_capacity,
                                  size_t* actual_out_size, deflate_format format);

/* ------------------------------------------------------------------------
 * Extension: device-resident batches (no counterpart in the reference, whose
 * only multi-buffer path is one deflate_compress call per buffer).
 * ---------------------------------------------------------------------- */

typedef struct deflate_gpu_batch deflate_gpu_batch;

/* A batch owns device arenas and a CUDA stream on the current device. */
deflate_gpu_batch* deflate_gpu_batch_new(void);
void deflate_gpu_batch_free(deflate_gpu_batch* b);

/* Copies `count` buffers (concatenated in host memory, sizes[i] bytes each)
 * into device memory and plans them: each buffer becomes one independent
 * stream with deflate_compress semantics (parallel = 0) or pigz chunking
 * (parallel = 1, block_size as deflate_parallel_new).  Returns 0 on success. */
int deflate_gpu_batch_load(deflate_gpu_batch* b, const void* host_concat, const size_t* sizes, size_t count, int level,
                           deflate_format format, int parallel, size_t block_size);

/* Runs the kernels on `cuda_stream` (a cudaStream_t, NULL = the batch's own
 * stream) without host synchronisation.  use_graph != 0 replays a CUDA graph
 * captured on first use.  Returns 0 on success. */
int deflate_gpu_batch_run(deflate_gpu_batch* b, void* cuda_stream, int use_graph);

/* Waits for the batch and copies the compressed sizes (0 = failed stream). */
int deflate_gpu_batch_sizes(deflate_gpu_batch* b, size_t* out_sizes);

/* Copies compressed stream i to host memory; returns its size or 0. */
size_t deflate_gpu_batch_output(deflate_gpu_batch* b, size_t i, void* dst, size_t capacity);

/* Number of kernel launches issued by the last deflate_gpu_batch_run. */
int deflate_gpu_batch_launches(const deflate_gpu_batch* b);

/* Per-phase timing: with profiling on, each run records CUDA events between
 * kernel phases (graph replay is disabled while on).  phase_ms fills
 * ms[0..n) with the milliseconds of each phase of the last run and returns
 * n (needs max >= n); deflate_gpu_phase_name(i) names phase i. */
int deflate_gpu_batch_profile(deflate_gpu_batch* b, int enable);
int deflate_gpu_batch_phase_ms(deflate_gpu_batch* b, float* ms, int max);
const char* deflate_gpu_phase_name(int i);

/* End-to-end batch from host buffers: copies in, compresses, copies every
 * output back (deflate_compress semantics per buffer).  out_sizes[i] = 0
 * marks a buffer whose output did not fit out_caps[i].  Returns the number of
 * buffers compressed. */
size_t deflate_gpu_compress_batch(const void* const* in, const size_t* in_sizes, void* const* out,
                                  const size_t* out_caps, size_t* out_sizes, size_t count, int level,
                                  deflate_format format);

/* End-to-end batch from one concatenated host buffer (sizes[i] bytes each,
 * back to back): one host-to-device copy (DMA straight from in_concat when it
 * is pinned), one pass of kernels, outputs packed on the device at 16-byte
 * aligned offsets and copied back with one transfer into out_packed.
 * out_offsets needs count + 1 entries (the last is the packed total);
 * out_sizes[i] = 0 marks a failed stream.  Returns the packed byte count, or
 * 0 on error (including out_capacity below the packed total; size it with
 * deflate_gpu_packed_bound). */
size_t deflate_gpu_compress_packed(const void* in_concat, const size_t* in_sizes, size_t count, int level,
                                   deflate_format format, void* out_packed, size_t out_capacity, uint64_t* out_offsets,
                                   size_t* out_sizes);
size_t deflate_gpu_packed_bound(const size_t* in_sizes, size_t count, deflate_format format);

/* Pipelined host-to-host batch (no counterpart in the reference): as
 * deflate_gpu_compress_packed, but the buffers are split into groups of about
 * group_bytes (0 = 256 MiB) and `lanes` passes (0 = 6) are kept in flight, so
 * the copies of one group overlap the kernels of another.  Group g's outputs
 * start at the sum of the packed bounds of groups before it; out_offsets[i]
 * are absolute, out_offsets[count] is the end of the last output.  Returns
 * that end, or 0 on error. */
size_t deflate_gpu_compress_pipelined(const void* in_concat, const size_t* in_sizes, size_t count, int level,
                                      deflate_format format, void* out_packed, size_t out_capacity,
                                      uint64_t* out_offsets, size_t* out_sizes, size_t group_bytes, int lanes);

/* Continuous-batching server (no counterpart in the reference).  A server
 * thread keeps up to `lanes` passes (0 = 3) on the GPU; whenever one
 * finishes, every pending request that fits the device-memory budget
 * (0 = 16 GiB) is admitted into the next pass, so requests that arrive while
 * others run join the next pass and passes overlap on the device.  Each
 * request has deflate_compress semantics at its own level and format, so its
 * bytes do not depend on its batch.
 *   submit: `in` and `out` must stay valid until wait returns; returns a
 *           ticket (0 on error, also for a request above 2 GiB: larger
 *           inputs go through deflate_compress or the batch calls).  An
 *           `out_capacity` below
 *           deflate_compress_bound() is accepted and makes that request fail
 *           alone if its output does not fit.
 *   wait:   0 done (*out_size, *latency_s = submit to completion), -2 failed,
 *           1 timed out (ticket still valid), -1 unknown ticket.
 *   stats:  passes issued and the most passes seen in flight at once. */
typedef struct deflate_gpu_server deflate_gpu_server;
deflate_gpu_server* deflate_gpu_server_new(size_t device_budget, int lanes);
void deflate_gpu_server_free(deflate_gpu_server* s);
uint64_t deflate_gpu_server_submit(deflate_gpu_server* s, const void* in, size_t in_size, void* out, size_t out_capacity,
                                   int level, deflate_format format);
int deflate_gpu_server_wait(deflate_gpu_server* s, uint64_t ticket, size_t* out_size, double* latency_s,
                            double timeout_s);
int deflate_gpu_server_stats(deflate_gpu_server* s, uint64_t* passes, uint64_t* max_in_flight);

/* gzip files of independent members (no counterpart in the reference's
 * compress API; the form pigz --independent writes): the input is cut into
 * members of member_size bytes, each a complete gzip stream at `level`, all
 * compressed in one pass.  Every gzip reader reads the concatenation as one
 * file; deflate_decompress decodes its members in parallel (the reference's
 * parallel gzip path, src/decompress/parallel_decompress.cpp:64-150).  Returns
 * the byte count, or 0 when out_capacity is below
 * deflate_gzip_members_bound() or on a device error. */
size_t deflate_gzip_members_bound(size_t in_size, size_t member_size);
size_t deflate_gpu_compress_gzip_members(const void* in, size_t in_size, int level, size_t member_size, void* out,
                                         size_t out_capacity);

/* On-device verification of the last run of a batch (no counterpart in the
 * reference): every stream is decoded on the GPU (one warp per stream),
 * compared byte for byte with its input, and its framing and trailer are
 * checked.  ok[i] = 1 for a stream that round-trips.  Returns the number of
 * streams that failed, or -1. */
int deflate_gpu_batch_verify(deflate_gpu_batch* b, int* ok);

/* One pigz-style stream compressed by several GPUs (no counterpart in the
 * reference; the unit it shards is the chunk of deflate_parallel_compress,
 * src/parallel/parallel_compressor.cpp:36-150).  The input is split into
 * contiguous ranges of whole block_size chunks, one per rank; each rank
 * compresses its range into a bare part: raw DEFLATE with no header or
 * trailer, ending with an empty stored block (sync point) unless it is the
 * final part, which carries BFINAL.  The stream is the header of `format`,
 * the parts in rank order and the trailer built from the combined checksum
 * and the total length.  *checksum receives the range's Adler-32 (zlib),
 * CRC-32 (gzip) or 0 (raw).  A rank with no chunks passes in_size 0 and
 * final_part 0 and gets an empty part.  Returns 0, -1 bad argument,
 * -2 device failure, -3 out_capacity too small (deflate_compress_bound() of
 * the range always suffices). */
int deflate_gpu_parallel_shard(const void* in, size_t in_size, int level, deflate_format format, size_t block_size,
                               int final_part, void* out, size_t out_capacity, size_t* out_size, uint32_t* checksum);
/* crc32(A||B) from crc32(A), crc32(B) and |B| (zlib's crc32_combine). */
uint32_t deflate_crc32_combine(uint32_t crc1, uint32_t crc2, uint64_t len2);
/* adler32(A||B) from adler32(A), adler32(B) and |B| (zlib's adler32_combine). */
uint32_t deflate_adler32_combine(uint32_t adler1, uint32_t adler2, uint64_t len2);

/* No-allocation variant (no counterpart in the reference).  For callers that
 * own every byte of device memory and cannot let a library call cudaMalloc
 * (a host framework's pool allocator, a fixed device-memory budget): inputs,
 * output and the output size are the caller's device pointers, and the only
 * working memory is a static device array of about 2.4 MB that every GPU
 * loading this library keeps until exit.  deflate_compress semantics for
 * levels 0-3 (same bytes); inputs up to DEFLATE_GPU_NOALLOC_MAX_INPUT bytes;
 * out_capacity must be at least deflate_compress_bound().  Asynchronous on
 * cuda_stream (NULL = legacy default stream); *d_out_size receives the
 * compressed size.  The first call on a device looks up the array's device
 * address, so make it before any stream capture.  Calls share the array:
 * calls that overlap on the GPU race and must be ordered by the caller.
 * Returns 0 when the work was enqueued; -1 bad pointer or format, -2 input
 * too large, -3 level above 3, -4 capacity below the bound, -5 device
 * set-up failed, -6 launch failed (orot_b200_last_error() says which). */
#define DEFLATE_GPU_NOALLOC_MAX_INPUT (1u << 20)
int deflate_gpu_compress_noalloc(const void* d_in, size_t in_size, void* d_out, size_t out_capacity, int level,
                                 deflate_format format, unsigned long long* d_out_size, void* cuda_stream);

/* Last error message of the calling thread ("" if none). */
const char* orot_b200_last_error(void);

/* Where the pass geometry (tile bytes, lazy-level run lengths per pass size)
 * compiled into this library came from: the autotuner's device and date, or
 * the hand-set rules it starts from (no counterpart in the reference). */
const char* orot_b200_geometry_source(void);

/* Tile bytes the planner uses at levels 1-3 (hash_bits 12: level 1; 14:
 * levels 2-3) for a pass of `pass_bytes` input bytes on a device of `sms`
 * SMs, from the compiled geometry table (no counterpart in the reference;
 * needs no GPU).  OROT_B200_TILE, when set, overrides it in a pass. */
uint32_t orot_b200_geometry_tile(uint64_t pass_bytes, int sms, int hash_bits);

#ifdef __cplusplus
}
#endif
#endif /* OROT_B200_H */
