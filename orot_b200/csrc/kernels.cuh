// kernels.cuh -- launch interface between the host engine and the kernels.
#pragma once
#include <cuda_runtime.h>
#include <atomic>
#include <cstdint>
#include "engine.cuh"
#include "deflate_device.cuh"

namespace orotb {

// Index of the calling thread's current device for per-device launch caches
// (kernel attributes and occupancy are properties of a device and never
// change, so they are set and queried on a device's first launch only).
inline int device_slot() {
  int d = 0;
  if (cudaGetDevice(&d) != cudaSuccess || d < 0 || d >= 64) d = 0;
  return d;
}

// Device pointers of one compression pass.
struct Work {
  const uint8_t* in;     // input arena (16-byte aligned, 64 bytes of padding)
  uint8_t* out;          // output arena
  uint8_t* scratch;      // per-tile bit buffers, records, carried hash tables
  Stream* streams;
  Segment* segs;
  Tile* tiles;
  Piece* pieces;
  CkBlock* ck;
  uint32_t nstreams, nsegs, ntiles, npieces, nck;
  uint32_t pad;
};

// Index lists for the fast-level (1-3) pipeline of one hash width.
struct FastLists {
  const uint32_t* lastocc;   // tiles that publish a last-occurrence table
  uint32_t n_lastocc;
  const uint32_t* multi;     // segments with more than one tile
  uint32_t n_multi;
  const uint32_t* walk;      // tiles to walk
  uint32_t n_walk;
  uint32_t* counter;         // zeroed work counters
  uint32_t* ready;           // zeroed, one flag per tile of `walk` (candidates done)
};

// Index lists for the lazy-level (4-12) pipeline.
struct LazyLists {
  const uint32_t* runs;      // (first tile, tile count) of every run, count <= kLazyRun
  uint32_t n_runs;
  const uint32_t* tiles;     // tiles to encode
  uint32_t n_tiles;
  const uint32_t* segs;      // segments needing Huffman tables
  uint32_t n_segs;
  uint32_t* counter;
};

// Optional per-phase CUDA events: mark(id) records an event after phase id.
enum Phase { kPhPre = 0, kPhCand, kPhWalk, kPhFix, kPhLazyLz, kPhLazyHuff, kPhLazyEnc, kPhPlan, kPhJoin, kPhCheck, kPhFrame,
             kNumPhases };
struct Marks {
  cudaEvent_t ev[kNumPhases + 1];
  int id[kNumPhases + 1];
  int n = 0;
  bool on = false;
  void mark(int phase, cudaStream_t st) {
    if (!on || n > kNumPhases) return;
    cudaEventRecord(ev[n], st);
    id[n++] = phase;
  }
};

void launch_fast(const Work& wk, const FastLists& L, int hash_bits, cudaStream_t st, int sms, Marks* mk);
// Whether launch_fast runs the candidate pass and the parse as one kernel.
bool fast_launches_fused();
int launch_lazy(const Work& wk, const LazyLists& L, cudaStream_t st, int sms, Marks* mk);
void launch_plan(const Work& wk, uint64_t max_out, cudaStream_t st);  // max_out: largest stream bound
void launch_checksums(const Work& wk, cudaStream_t st);
void launch_ck_single(const CkBlock* ck, uint32_t nck, uint64_t total, uint32_t init, int adler, uint32_t* res,
                      const Work& wk, cudaStream_t st);
CrcPowers host_crc_powers();
void launch_join(const Work& wk, uint32_t* counter, cudaStream_t st, int sms);
void launch_frame(const Work& wk, cudaStream_t st);
bool upload_crc_tables();  // once per device; false on a device error

// One DEFLATE stream to decode (raw data, framing stripped by the host).
struct InflateJob {
  uint64_t in_off;   // raw DEFLATE bytes, relative to the input base
  uint64_t in_len;
  uint64_t out_off;  // output slot, relative to the output base
  uint64_t out_cap;
  uint64_t out_len;  // result: bytes written
  uint64_t in_used;  // result: bytes of input the stream occupied
  int32_t status;    // result: kInf*
  uint32_t pad;
};
constexpr int32_t kInfOk = 0, kInfData = 1, kInfOutput = 2, kInfInput = 3, kInfMismatch = 4;
// Decodes jobs[order[0..n)] (one warp per stream; the input and output
// buffers carry at least 8 bytes of padding); `counter` is a device word.
void launch_inflate(const uint8_t* in, uint8_t* out, InflateJob* jobs, const uint32_t* order, uint32_t njobs,
                    uint32_t* counter, int sms, cudaStream_t st);
// Marks kInfMismatch on streams whose framing or trailer is wrong (job i is stream i).
void launch_frame_check(const uint8_t* out, const Stream* streams, InflateJob* jobs, uint32_t n, cudaStream_t st);
// Marks kInfMismatch on jobs whose decoded bytes differ from ref[ref_off[j], + ref_len[j]).
void launch_inflate_compare(const uint8_t* decoded, const uint8_t* ref, InflateJob* jobs, const uint64_t* ref_off,
                            const uint64_t* ref_len, uint32_t njobs, cudaStream_t st);

}  // namespace orotb
