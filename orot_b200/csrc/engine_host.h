// engine_host.h -- host-side engine object shared by the C ABI, the batch API
// and the server.
#pragma once
#include <cuda_runtime.h>
#include <cstdint>
#include <mutex>
#include <string>
#include <vector>
#include "engine.cuh"
#include "kernels.cuh"
#include "geometry_table.h"

namespace orotb {

void set_error(const std::string& e);
size_t raw_bound(size_t n);
size_t framed_bound(size_t n, int fmt);
size_t default_block(int level);
size_t parallel_bound(size_t n, int fmt, int level, size_t block);
int clamp_level(int l);

// A device arena that grows on demand.  With `pool` set, it grows by
// stream-ordered allocation on `st` (the only stream that uses it), which
// does not synchronise the device; otherwise by cudaMalloc / cudaFree, which
// waits for all work on the device (used where another stream may still be
// reading the old arena, e.g. a batch run on a caller's stream).
struct DevBuf {
  void* p = nullptr;
  size_t cap = 0;
  cudaMemPool_t pool = nullptr;
  cudaStream_t st = nullptr;
  bool ensure(size_t n);
  void release();
};
struct HostBuf {
  void* p = nullptr;
  size_t cap = 0;
  bool ensure(size_t n);
  void release();
};

// One output stream to produce.
struct Job {
  uint64_t in_off;      // in the input arena (16-byte aligned)
  uint64_t in_len;
  uint64_t out_off;     // in the output arena (16-byte aligned)
  uint64_t out_cap;
  int level;
  int fmt;
  bool parallel;        // pigz chunking instead of one block per buffer
  uint64_t block_size;  // chunk size for parallel (0 = by level)
  uint32_t mode = 0;    // kStreamBare | kStreamOpen
};

enum ListId {
  kLast12, kMulti12, kWalk12,
  kLast14, kMulti14, kWalk14,
  kLazyTiles, kLazySegs, kLazyRuns,
  kNumLists
};

class Engine {
 public:
  Engine();
  ~Engine();
  Engine(const Engine&) = delete;
  Engine& operator=(const Engine&) = delete;

  bool ensure_io(uint64_t in_bytes, uint64_t out_bytes);
  bool plan(const std::vector<Job>& jobs);
  bool launch(cudaStream_t st);
  Work work() const;
  // One stream from host memory to host memory; `mode` takes kStreamBare /
  // kStreamOpen and `result` (optional) receives the stream's table entry.
  size_t compress_host(const void* in, size_t n, void* out, size_t cap, int level, int fmt, bool parallel, size_t block,
                       uint32_t mode = 0, Stream* result = nullptr);
  uint32_t checksum_host(uint32_t init, const void* data, size_t n, bool adler);
  // Checksum of n bytes already on the device (d_data 16-byte aligned, with
  // readable padding after the last byte).
  uint32_t checksum_device(uint32_t init, const uint8_t* d_data, size_t n, bool adler);
  // Makes the arenas grow by stream-ordered allocation on the engine's own
  // stream (for engines whose work runs on that stream only).
  void use_stream_ordered_arenas();
  uint32_t pick_tile(uint64_t total_bytes, int hash_bits) const;
  const GeometryRow& geometry(uint64_t total_bytes) const;

  int device = 0, sms = 148;
  bool ok = false;  // the stream and the device's constant tables are set up
  cudaStream_t stream = nullptr;
  DevBuf d_in, d_out, d_scratch, d_tables, d_pack;
  HostBuf h_tables, h_stage;
  cudaGraphExec_t graph_exec = nullptr;
  uint32_t tile_override = 0;
  uint32_t lazy_run_override = 0;

  // planned tables (host copies)
  std::vector<Stream> streams;
  std::vector<Segment> segs;
  std::vector<Tile> tiles;
  std::vector<CkBlock> cks;
  std::vector<uint32_t> lists[kNumLists];
  uint32_t n_pieces = 0;
  uint64_t scratch_bytes = 0, upload_bytes = 0;
  uint64_t max_out_cap = 0;  // largest output slot of the planned pass
  uint64_t off_streams = 0, off_segs = 0, off_tiles = 0, off_ck = 0, off_pieces = 0, off_counters = 0;
  uint64_t off_ready = 0;  // per fast-level tile: candidates done (zeroed by every upload)
  uint64_t off_lists[kNumLists] = {};
  int launches = 0;
  Marks marks;
  bool made_events = false;
  cudaEvent_t stage_ev[8] = {};  // pieces of an output copied back (compress_host)
  bool made_stage_events = false;
  void phase_ms(float* ms) const;
};

std::mutex& global_mutex();

// The one-call entry points (deflate_compress, deflate_parallel_compress,
// deflate_crc32/adler32, deflate_decompress, the shard call) run on engines
// of the calling thread's current CUDA device.  A lease takes an idle engine
// of that device, creating one when none is idle (at most kMaxEngines per
// device; beyond that the caller waits for one), so calls from different
// host threads run at the same time, each on its own stream and arenas.
// Engines are kept for reuse, most recently used first, so a single-threaded
// caller keeps reusing one engine and its grown arenas.
constexpr int kMaxEngines = 32;
constexpr int kMaxDevices = 64;
class EngineLease {
 public:
  EngineLease();
  ~EngineLease();
  EngineLease(const EngineLease&) = delete;
  EngineLease& operator=(const EngineLease&) = delete;
  explicit operator bool() const { return e_ != nullptr; }
  Engine& operator*() const { return *e_; }
  Engine* operator->() const { return e_; }

 private:
  Engine* e_ = nullptr;
  int dev_ = -1;
};

// Makes `dev` the calling thread's current device for the scope and restores
// the caller's device afterwards: objects bound to a device (a batch, a lane)
// may be used from threads whose current device is another one.
class DeviceScope {
 public:
  explicit DeviceScope(int dev) {
    if (cudaGetDevice(&prev_) == cudaSuccess && prev_ != dev) changed_ = cudaSetDevice(dev) == cudaSuccess;
    cudaGetLastError();
  }
  ~DeviceScope() {
    if (changed_) cudaSetDevice(prev_);
  }
  DeviceScope(const DeviceScope&) = delete;
  DeviceScope& operator=(const DeviceScope&) = delete;

 private:
  int prev_ = -1;
  bool changed_ = false;
};

// The calling thread's current device, or -1 (with the error recorded) when
// it has none or its index is beyond kMaxDevices.
int current_device();

// Packs every stream's output of the last pass at 16-byte aligned offsets
// (d_off: count + 1 entries, the last the total) and optionally writes the
// sizes (0 = failed stream).  Defined in batch.cu.
void launch_pack(const Work& w, uint64_t* d_off, uint64_t* d_sizes, uint8_t* d_packed, cudaStream_t st);

}  // namespace orotb
