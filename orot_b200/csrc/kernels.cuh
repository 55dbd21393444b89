// kernels.cuh -- launch interface between the host engine and the kernels.
#pragma once
#include <cuda_runtime.h>
#include <cstdint>
#include "engine.cuh"
#include "deflate_device.cuh"

namespace orotb {

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
  uint32_t* counter;         // zeroed work counter for k_walk
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
enum Phase { kPhPre = 0, kPhWalk, kPhFix, kPhLazyLz, kPhLazyHuff, kPhLazyEnc, kPhPlan, kPhJoin, kPhCheck, kPhFrame,
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
int launch_lazy(const Work& wk, const LazyLists& L, cudaStream_t st, int sms, Marks* mk);
void launch_plan(const Work& wk, cudaStream_t st);
void launch_checksums(const Work& wk, cudaStream_t st);
void launch_ck_single(const CkBlock* ck, uint32_t nck, uint64_t total, uint32_t init, int adler, uint32_t* res,
                      const Work& wk, cudaStream_t st);
CrcPowers host_crc_powers();
void launch_join(const Work& wk, uint32_t* counter, cudaStream_t st, int sms);
void launch_frame(const Work& wk, cudaStream_t st);
void upload_crc_tables();

}  // namespace orotb
