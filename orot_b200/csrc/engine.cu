// engine.cu -- host side of the engine: planning, device arenas, launches,
// and the C ABI declared in include/orot_b200.h.
//
// A compression pass takes a list of jobs (one per output stream), lays out
// the Stream / Segment / Tile / Piece / CkBlock tables in one host buffer,
// uploads it with a single copy and launches:
//   fast-level LZ77 (kernels_fast.cu) and lazy-level LZ77 + Huffman
//   (kernels_lazy.cu), block planning and zeroing, bit join, checksums and
//   framing (kernels_common.cu).
#include <cuda_runtime.h>
#include <algorithm>
#include <cstdint>
#include <cstdio>
#include <cstdlib>
#include <cstring>
#include <condition_variable>
#include <mutex>
#include <new>
#include <string>
#include <vector>
#include "engine.cuh"
#include "kernels.cuh"
#include "engine_host.h"
#include "geometry_table.h"
#include "host_copy.h"
#include "../../include/orot_b200.h"

namespace orotb {

thread_local std::string g_err;
void set_error(const std::string& e) { g_err = e; }

#define CK(x)                                                                      \
  do {                                                                             \
    cudaError_t e_ = (x);                                                          \
    if (e_ != cudaSuccess) {                                                       \
      set_error(std::string(#x) + ": " + cudaGetErrorString(e_));                  \
      return false;                                                                \
    }                                                                              \
  } while (0)

size_t raw_bound(size_t n) { return n + (n >> 12) + (n >> 14) + (n >> 25) + 13; }
size_t framed_bound(size_t n, int fmt) { return raw_bound(n) + (fmt == kFmtZlib ? 6 : fmt == kFmtGzip ? 18 : 0); }
size_t default_block(int level) { return level <= 3 ? 131072 : level <= 6 ? 524288 : 1048576; }
int clamp_level(int l) { return l < 0 ? 0 : l > 12 ? 12 : l; }

bool DevBuf::ensure(size_t n) {
  if (n <= cap) return true;
  size_t want = std::max(n, cap + cap / 2);  // grow geometrically
  if (pool) {
    // pool arenas double (at least 1 MiB): mapping new memory into the pool
    // is the slow part of an allocation, so it should happen rarely
    want = std::max({n, 2 * cap, size_t(1) << 20});
    if (p) cudaFreeAsync(p, st);
    p = nullptr;
    cap = 0;
    if (cudaMallocFromPoolAsync(&p, want, pool, st) != cudaSuccess) {
      cudaGetLastError();
      if (cudaMallocFromPoolAsync(&p, n, pool, st) != cudaSuccess) {
        cudaGetLastError();
        p = nullptr;
        set_error("device arena allocation failed");
        return false;
      }
      want = n;
    }
    cap = want;
    return true;
  }
  if (p) cudaFree(p);  // synchronises the device
  p = nullptr;
  cap = 0;
  if (cudaMalloc(&p, want) != cudaSuccess) {
    cudaGetLastError();
    if (cudaMalloc(&p, n) != cudaSuccess) { cudaGetLastError(); p = nullptr; set_error("cudaMalloc failed"); return false; }
    want = n;
  }
  cap = want;
  return true;
}
void DevBuf::release() {
  if (p) {
    if (pool) cudaFreeAsync(p, st);
    else cudaFree(p);
  }
  p = nullptr;
  cap = 0;
}

// The arena memory pool of a device (the calling thread's current one): a
// pool of this library's own that keeps freed memory for reuse instead of
// returning it at every synchronisation; nullptr when the device has none.
static cudaMemPool_t arena_pool(int dev) {
  static std::mutex mu;
  static cudaMemPool_t pools[64] = {};
  static bool tried[64] = {};
  if (dev < 0 || dev >= 64) return nullptr;
  std::lock_guard<std::mutex> lk(mu);
  if (!tried[dev]) {
    tried[dev] = true;
    cudaMemPoolProps props{};
    props.allocType = cudaMemAllocationTypePinned;
    props.location.type = cudaMemLocationTypeDevice;
    props.location.id = dev;
    cudaMemPool_t pl = nullptr;
    if (cudaMemPoolCreate(&pl, &props) == cudaSuccess) {
      uint64_t keep = ~uint64_t(0);
      cudaMemPoolSetAttribute(pl, cudaMemPoolAttrReleaseThreshold, &keep);
      pools[dev] = pl;
    } else {
      cudaGetLastError();
    }
  }
  return pools[dev];
}

void Engine::use_stream_ordered_arenas() {
  cudaMemPool_t pl = arena_pool(device);
  if (!pl) return;
  for (DevBuf* b : {&d_in, &d_out, &d_scratch, &d_tables, &d_pack}) {
    if (b->p) continue;  // only arenas not yet allocated change mode
    b->pool = pl;
    b->st = stream;
  }
}

bool HostBuf::ensure(size_t n) {
  if (n <= cap) return true;
  size_t want = std::max(n, cap + cap / 2);
  if (p) cudaFreeHost(p);
  p = nullptr;
  cap = 0;
  if (cudaMallocHost(&p, want) != cudaSuccess) {
    cudaGetLastError();
    if (cudaMallocHost(&p, n) != cudaSuccess) { cudaGetLastError(); p = nullptr; set_error("cudaMallocHost failed"); return false; }
    want = n;
  }
  cap = want;
  return true;
}
void HostBuf::release() { if (p) cudaFreeHost(p); p = nullptr; cap = 0; }

Engine::Engine() {
  ok = cudaGetDevice(&device) == cudaSuccess &&
       cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, device) == cudaSuccess &&
       cudaStreamCreateWithFlags(&stream, cudaStreamNonBlocking) == cudaSuccess && upload_crc_tables();
  if (!ok) {
    cudaGetLastError();
    set_error("engine set-up failed (no usable CUDA device)");
  }
  // Tile size override (bytes, multiple of 32, at most 64 KiB) for tests.
  if (const char* v = std::getenv("OROT_B200_TILE")) {
    const long t = std::strtol(v, nullptr, 10);
    if (t >= 32 && t <= 65536 && t % 32 == 0) tile_override = uint32_t(t);
  }
  // Lazy-level run length override (tiles per CTA, 1..kLazyRun) for tests.
  if (const char* v = std::getenv("OROT_B200_LAZY_RUN")) {
    const long r = std::strtol(v, nullptr, 10);
    if (r >= 1 && r <= long(kLazyRun)) lazy_run_override = uint32_t(r);
  }
}
Engine::~Engine() {
  if (graph_exec) cudaGraphExecDestroy(graph_exec);
  if (made_stage_events)
    for (cudaEvent_t ev : stage_ev) cudaEventDestroy(ev);
  for (DevBuf* b : {&d_in, &d_out, &d_scratch, &d_tables, &d_pack}) b->release();
  if (stream) cudaStreamSynchronize(stream);
  h_tables.release();
  h_stage.release();
  if (stream) cudaStreamDestroy(stream);
}

// Pass geometry comes from the table the autotuner writes (geometry_table.h):
// the row of the largest pass-size class the pass reaches.  Classes are
// measured on 148 SMs; a device with fewer SMs reaches the same work per SM
// with proportionally less input.  Small tiles let more warps walk a small
// pass at once; large tiles carry fewer head tables (4 B per entry: 16 KB
// at 12 hash bits, 64 KB at 14) and fix up fewer boundaries.
// The table row of a pass of `total_bytes` on a device of `sms` SMs: sizes
// are scaled to a 148-SM device (multiplied first, so that a pass of exactly
// a class boundary belongs to that class).
static const GeometryRow& geometry_row(uint64_t total_bytes, int sms) {
  const uint64_t scaled = total_bytes * 148u / uint64_t(std::max(sms, 1));
  size_t k = 0;
  for (size_t i = 0; i < sizeof(kGeometry) / sizeof(kGeometry[0]); ++i)
    if (scaled >= kGeometry[i].min_bytes) k = i;
  return kGeometry[k];
}

const GeometryRow& Engine::geometry(uint64_t total_bytes) const { return geometry_row(total_bytes, sms); }

uint32_t Engine::pick_tile(uint64_t total_bytes, int hash_bits) const {
  if (tile_override) return tile_override;
  const GeometryRow& g = geometry(total_bytes);
  return hash_bits <= 12 ? g.tile12 : g.tile14;
}

template <class T>
static uint64_t put_table(std::vector<uint8_t>& buf, const std::vector<T>& v) {
  const uint64_t off = align_up(buf.size(), 256);
  buf.resize(off + v.size() * sizeof(T));
  if (!v.empty()) std::memcpy(buf.data() + off, v.data(), v.size() * sizeof(T));
  return off;
}

bool Engine::plan(const std::vector<Job>& jobs) {
  streams.clear(); segs.clear(); tiles.clear(); cks.clear();
  for (auto& l : lists) l.clear();
  uint64_t total = 0;
  max_out_cap = 0;
  for (const Job& j : jobs) {
    total += j.in_len;
    max_out_cap = std::max<uint64_t>(max_out_cap, j.out_cap);
  }
  const uint32_t T12 = pick_tile(total, 12), T14 = pick_tile(total, 14);
  uint64_t scratch = 0;
  uint32_t npieces = 0;
  for (size_t ji = 0; ji < jobs.size(); ++ji) {
    const Job& j = jobs[ji];
    Stream s{};
    s.in_off = j.in_off;
    s.in_len = j.in_len;
    s.out_off = j.out_off;
    s.out_cap = j.out_cap;
    s.level = j.level;
    s.fmt = uint32_t(j.fmt);
    s.parallel = j.parallel ? 1 : 0;
    s.mode = j.mode;
    s.seg_first = uint32_t(segs.size());
    s.piece_first = npieces;
    const int lv = clamp_level(j.level);
    const uint64_t blk = j.parallel ? (j.block_size ? j.block_size : default_block(j.level)) : std::max<uint64_t>(j.in_len, 1);
    const uint64_t nseg = j.in_len ? (j.in_len + blk - 1) / blk : 1;
    for (uint64_t k = 0; k < nseg; ++k) {
      Segment g{};
      const uint64_t off = k * blk;
      const uint64_t len = j.in_len ? std::min(blk, j.in_len - off) : 0;
      if (len > 0xFFFFFFFFull - 65536) { set_error("segment larger than 4 GiB"); return false; }
      g.in_off = j.in_off + off;
      g.len = uint32_t(len);
      g.stream = uint32_t(ji);
      g.level = lv;
      g.flags = (k + 1 == nseg && !(j.mode & kStreamOpen) ? kSegLast : 0) | (j.parallel ? 0 : kSegWholeBuf);
      g.tile_first = uint32_t(tiles.size());
      const int hb = lv <= 0 ? 0 : lv == 1 ? 12 : lv <= 3 ? 14 : 0;
      const uint32_t H = hb ? (1u << hb) : 0;
      if (lv > 0 && lv <= 3) {
        const uint32_t T = hb == 12 ? T12 : T14;
        const uint32_t nt = len ? uint32_t((len + T - 1) / T) : 1;
        g.tile_count = nt;
        const uint32_t seg_index = uint32_t(segs.size());
        if (nt > 1) lists[hb == 12 ? kMulti12 : kMulti14].push_back(seg_index);
        for (uint32_t t = 0; t < nt; ++t) {
          Tile tl{};
          tl.seg = seg_index;
          tl.start = t * T;
          tl.len = uint32_t(std::min<uint64_t>(T, len - std::min<uint64_t>(len, uint64_t(t) * T)));
          tl.index = t;
          const uint64_t sb = tile_stream_bytes(tl.len);
          tl.scratch = scratch;
          scratch += 2 * sb;  // speculative + fix-up bit buffers
          // window records and candidate distances (every tile: the parse
          // kernel reads them; the fix-up reads those of tiles after the first)
          tl.rec = scratch;
          scratch += align_up(uint64_t((tl.len + 31) / 32) * sizeof(WinRec), 256);
          tl.cand = scratch;
          scratch += align_up(uint64_t(tl.len) * 2 + 64, 256);
          if (t > 0) tl.carry = tiles.back().slot;
          if (t + 1 < nt) {
            tl.slot = scratch;
            scratch += uint64_t(H) * 4;
          }
          const uint32_t ti = uint32_t(tiles.size());
          lists[hb == 12 ? kWalk12 : kWalk14].push_back(ti);
          if (t + 1 < nt) lists[hb == 12 ? kLast12 : kLast14].push_back(ti);
          tiles.push_back(tl);
        }
      } else if (lv >= 4) {
        // independent 4 KiB tiles, each with its own token words and histogram
        const uint32_t LT = kLazyTile;
        const uint32_t nt = len ? uint32_t((len + LT - 1) / LT) : 1;
        g.tile_count = nt;
        const uint32_t seg_index = uint32_t(segs.size());
        lists[kLazySegs].push_back(seg_index);
        for (uint32_t t = 0; t < nt; ++t) {
          Tile tl{};
          tl.seg = seg_index;
          tl.start = t * LT;
          tl.len = uint32_t(std::min<uint64_t>(LT, len - std::min<uint64_t>(len, uint64_t(t) * LT)));
          tl.index = t;
          tl.scratch = scratch;
          scratch += lazy_stream_bytes(tl.len);
          tl.tok = scratch;
          scratch += align_up(uint64_t(tl.len) * 4 + 4, 256);
          tl.hist = scratch;
          scratch += 320 * 4;
          lists[kLazyTiles].push_back(uint32_t(tiles.size()));
          tiles.push_back(tl);
        }
        g.codes = scratch;
        scratch += 320 * 4;
        g.hdr_off = scratch;
        scratch += 1024;
      }
      const uint32_t stored_pieces = std::max<uint32_t>(1, uint32_t((len + 65534) / 65535));
      g.piece_off = npieces - s.piece_first;
      npieces += 1 + 2 * g.tile_count + 2 + 3 * stored_pieces;
      segs.push_back(g);
    }
    s.seg_count = uint32_t(segs.size()) - s.seg_first;
    if (j.mode & kStreamOpen) npieces += 2;  // the closing sync point
    s.piece_count = npieces - s.piece_first;
    s.ck_first = uint32_t(cks.size());
    if (j.fmt != kFmtRaw) {
      for (uint64_t o = 0; o < j.in_len; o += 65536) {
        CkBlock c{};
        c.in_off = j.in_off + o;
        c.len = uint32_t(std::min<uint64_t>(65536, j.in_len - o));
        c.stream = uint32_t(ji);
        c.what = j.fmt == kFmtGzip ? kCkCrc : kCkAdler;
        cks.push_back(c);
      }
    }
    s.ck_count = uint32_t(cks.size()) - s.ck_first;
    streams.push_back(s);
  }
  // Walkers take tiles longest first: full tiles, then the last (partial)
  // tiles of the segments by decreasing length, so that a walker which picks
  // up a tile near the end of the pass finishes soon after the others (one
  // warp needs about 3 ms for a full 64 KiB tile).  The order does not change
  // the output: tiles are walked independently and fixed up afterwards.
  for (const int li : {kWalk12, kWalk14}) {
    std::vector<uint32_t>& v = lists[li];
    std::vector<uint32_t> part;
    size_t nfull = 0;
    const uint32_t T = li == kWalk12 ? T12 : T14;
    for (const uint32_t x : v) {
      if (tiles[x].len == T) v[nfull++] = x;
      else part.push_back(x);
    }
    std::stable_sort(part.begin(), part.end(), [&](uint32_t a, uint32_t b) { return tiles[a].len > tiles[b].len; });
    std::copy(part.begin(), part.end(), v.begin() + nfull);
  }
  n_pieces = npieces;
  scratch_bytes = align_up(scratch + 256, 256);

  // one host buffer, one upload
  std::vector<uint8_t> buf;
  off_streams = put_table(buf, streams);
  off_segs = put_table(buf, segs);
  off_tiles = put_table(buf, tiles);
  off_ck = put_table(buf, cks);
  // Lazy tiles go to CTAs in runs of consecutive tiles of one segment (the
  // window slides from tile to tile, and every run first builds the links of
  // its whole window).  Short runs give small passes enough CTAs for every
  // SM; long runs build fewer windows.  The run length per level group and
  // pass size is the autotuner's (geometry_table.h).
  if (!lists[kLazySegs].empty()) {
    const GeometryRow& geo = geometry(total);
    for (uint32_t si : lists[kLazySegs]) {
      const Segment& g = segs[si];
      const int grp = g.level <= 6 ? 0 : g.level <= 9 ? 1 : 2;
      const uint32_t R = std::min(kLazyRun, std::max(1u, lazy_run_override ? lazy_run_override : geo.lazy_run[grp]));
      for (uint32_t t = 0; t < g.tile_count; t += R) {
        lists[kLazyRuns].push_back(g.tile_first + t);
        lists[kLazyRuns].push_back(std::min(R, g.tile_count - t));
      }
    }
  }
  for (int i = 0; i < kNumLists; ++i) off_lists[i] = put_table(buf, lists[i]);
  off_counters = align_up(buf.size(), 256);
  buf.resize(off_counters + 256, 0);
  off_ready = align_up(buf.size(), 256);
  buf.resize(off_ready + 4 * (lists[kWalk12].size() + lists[kWalk14].size()), 0);
  off_pieces = align_up(buf.size(), 256);
  const uint64_t table_bytes = off_pieces + uint64_t(npieces) * sizeof(Piece) + 256;
  if (!d_tables.ensure(table_bytes) || !h_tables.ensure(buf.size())) return false;
  std::memcpy(h_tables.p, buf.data(), buf.size());
  upload_bytes = buf.size();
  if (!d_scratch.ensure(scratch_bytes)) return false;
  return true;
}

Work Engine::work() const {
  Work w{};
  uint8_t* t = static_cast<uint8_t*>(d_tables.p);
  w.in = static_cast<const uint8_t*>(d_in.p);
  w.out = static_cast<uint8_t*>(d_out.p);
  w.scratch = static_cast<uint8_t*>(d_scratch.p);
  w.streams = reinterpret_cast<Stream*>(t + off_streams);
  w.segs = reinterpret_cast<Segment*>(t + off_segs);
  w.tiles = reinterpret_cast<Tile*>(t + off_tiles);
  w.pieces = reinterpret_cast<Piece*>(t + off_pieces);
  w.ck = reinterpret_cast<CkBlock*>(t + off_ck);
  w.nstreams = uint32_t(streams.size());
  w.nsegs = uint32_t(segs.size());
  w.ntiles = uint32_t(tiles.size());
  w.npieces = n_pieces;
  w.nck = uint32_t(cks.size());
  return w;
}

// Uploads the planned tables and launches every kernel of the pass on st.
bool Engine::launch(cudaStream_t st) {
  launches = 0;
  uint8_t* t = static_cast<uint8_t*>(d_tables.p);
  marks.n = 0;
  if (marks.on && !made_events) {
    for (auto& e : marks.ev) cudaEventCreate(&e);
    made_events = true;
  }
  CK(cudaMemcpyAsync(t, h_tables.p, upload_bytes, cudaMemcpyHostToDevice, st));
  marks.mark(-1, st);
  const Work w = work();
  uint32_t* counters = reinterpret_cast<uint32_t*>(t + off_counters);
  auto list = [&](int i) { return reinterpret_cast<const uint32_t*>(t + off_lists[i]); };
  const int hbs[2] = {12, 14};
  for (int g = 0; g < 2; ++g) {
    FastLists L{};
    L.lastocc = list(g ? kLast14 : kLast12);
    L.n_lastocc = uint32_t(lists[g ? kLast14 : kLast12].size());
    L.multi = list(g ? kMulti14 : kMulti12);
    L.n_multi = uint32_t(lists[g ? kMulti14 : kMulti12].size());
    L.walk = list(g ? kWalk14 : kWalk12);
    L.n_walk = uint32_t(lists[g ? kWalk14 : kWalk12].size());
    L.counter = counters + g;  // candidates: 0/1; fix-up round 1: 4/5 (+ 4); parse: 6/7 (+ 6); abort: 12/13 (+ 12)
    L.ready = reinterpret_cast<uint32_t*>(t + off_ready) + (g ? lists[kWalk12].size() : 0);
    if (L.n_walk) {
      launch_fast(w, L, hbs[g], st, sms, &marks);
      // k_lastocc; k_carry_scan, k_fix1, k_fix2 for multi-tile segments;
      // k_cand_parse (or k_cand and k_parse)
      launches += (L.n_lastocc ? 1 : 0) + (L.n_multi ? 3 : 0) + (fast_launches_fused() ? 1 : 2);
    }
  }
  if (!lists[kLazyTiles].empty()) {
    LazyLists L{};
    L.runs = list(kLazyRuns);
    L.n_runs = uint32_t(lists[kLazyRuns].size() / 2);
    L.tiles = list(kLazyTiles);
    L.n_tiles = uint32_t(lists[kLazyTiles].size());
    L.segs = list(kLazySegs);
    L.n_segs = uint32_t(lists[kLazySegs].size());
    L.counter = counters + 2;
    launches += launch_lazy(w, L, st, sms, &marks);
  }
  launch_plan(w, max_out_cap, st);
  marks.mark(kPhPlan, st);
  launches += 4;  // k_plan_seg, k_plan_stream, k_plan_pieces, k_zero
  launch_join(w, counters + 3, st, sms);
  marks.mark(kPhJoin, st);
  launches += w.npieces ? 1 : 0;
  bool framed = false;
  for (const Stream& s : streams) framed |= s.fmt != kFmtRaw;
  if (framed) {
    launch_checksums(w, st);
    launches += (w.nck ? 1 : 0) + 1;
  }
  marks.mark(kPhCheck, st);
  launch_frame(w, st);
  marks.mark(kPhFrame, st);
  launches += 1;
  CK(cudaGetLastError());
  return true;
}

// Milliseconds per phase of the last launch (after the stream completed).
void Engine::phase_ms(float* ms) const {
  for (int i = 0; i < kNumPhases; ++i) ms[i] = 0.f;
  for (int i = 1; i < marks.n; ++i) {
    float x = 0.f;
    if (cudaEventElapsedTime(&x, marks.ev[i - 1], marks.ev[i]) == cudaSuccess && marks.id[i] >= 0)
      ms[marks.id[i]] += x;
  }
}

bool Engine::ensure_io(uint64_t in_bytes, uint64_t out_bytes) {
  // 256 bytes of padding: kernels read whole words (and a staged window of
  // 64 bytes) past the last byte of a buffer, never using those bytes.
  return d_in.ensure(in_bytes + 256) && d_out.ensure(out_bytes + 256);
}

// Whole-buffer or pigz-style compression of one host buffer.
// Worst case of a pigz stream: every chunk stored (5 bytes per 65535-byte
// piece) plus up to one byte of padding before each stored block.
size_t parallel_bound(size_t n, int fmt, int level, size_t block) {
  const size_t blk = block ? block : default_block(level);
  const size_t nchunk = n ? (n + blk - 1) / blk : 1;
  const size_t pieces = (blk + 65534) / 65535;
  return std::max(framed_bound(n, fmt), n + nchunk * (5 * pieces + 1) + 32);
}

void host_copy(void* dst, const void* src, size_t n) {
  if (n < (size_t(4) << 20)) {
    std::memcpy(dst, src, n);
    return;
  }
  static std::once_flag once;
  static CopyPool* pool = nullptr;  // lives until the process exits
  static std::mutex busy;
  std::call_once(once, [] {
    const unsigned hw = std::thread::hardware_concurrency();
    pool = new CopyPool(int(std::min(8u, std::max(1u, hw / 2))));
  });
  std::unique_lock<std::mutex> lk(busy, std::try_to_lock);
  if (!lk.owns_lock()) {  // another thread's large copy has the copy threads
    std::memcpy(dst, src, n);
    return;
  }
  pool->run({Copy{static_cast<uint8_t*>(dst), static_cast<const uint8_t*>(src), n}});
}

// Calls above this many bytes move their input and output in pieces of at
// least kPieceMin bytes (so that each is copied by the copy threads), at most
// kStagePieces of them: the host copy of one piece overlaps the DMA of another.
constexpr size_t kPieceStage = size_t(8) << 20;
constexpr size_t kPieceMin = size_t(4) << 20;
constexpr int kStagePieces = 8;
static size_t stage_piece(size_t n) {
  return n < kPieceStage ? n : std::max(kPieceMin, align_up((n + kStagePieces - 1) / kStagePieces, 4096));
}

// Pinned staging of a one-call entry point is sized at least this much, so
// that the first calls do not each grow it (pinning memory is slow).
constexpr size_t kStageMin = size_t(4) << 20;
// Below this output bound, the result record and the whole output slot come
// back in one device-to-host round trip (one wait instead of two).
constexpr size_t kOneTripBound = size_t(1) << 20;

size_t Engine::compress_host(const void* in, size_t n, void* out, size_t cap, int level, int fmt, bool parallel,
                             size_t block, uint32_t mode, Stream* result) {
  const size_t bound = parallel ? parallel_bound(n, fmt, level, block) : framed_bound(n, fmt);
  if (!ensure_io(align_up(n, 16), align_up(bound, 16))) return 0;
  if (!h_stage.ensure(std::max({n, bound + 64, kStageMin}))) return 0;
  uint8_t* stage = static_cast<uint8_t*>(h_stage.p);
  const uint8_t* src = static_cast<const uint8_t*>(in);
  if (n) {
    // in pieces: the copy of piece k + 1 into staging overlaps the DMA of piece k
    const size_t piece = stage_piece(n);
    for (size_t o = 0; o < n; o += piece) {
      const size_t len = std::min(piece, n - o);
      host_copy(stage + o, src + o, len);
      if (cudaMemcpyAsync(static_cast<uint8_t*>(d_in.p) + o, stage + o, len, cudaMemcpyHostToDevice, stream) !=
          cudaSuccess) {
        set_error("H2D failed");
        return 0;
      }
    }
  }
  std::vector<Job> jobs(1);
  jobs[0] = Job{0, n, 0, parallel ? std::min<uint64_t>(cap, bound) : bound, level, fmt, parallel, block, mode};
  if (!plan(jobs) || !launch(stream)) return 0;
  const bool one_trip = bound <= kOneTripBound;
  Stream s{};
  if (cudaMemcpyAsync(&s, static_cast<uint8_t*>(d_tables.p) + off_streams, sizeof s, cudaMemcpyDeviceToHost, stream) != cudaSuccess ||
      (one_trip && cudaMemcpyAsync(stage, d_out.p, bound, cudaMemcpyDeviceToHost, stream) != cudaSuccess) ||
      cudaStreamSynchronize(stream) != cudaSuccess) {
    set_error(std::string("device error: ") + cudaGetErrorString(cudaGetLastError()));
    return 0;
  }
  if (result) *result = s;
  if (s.error || s.out_size == 0 || s.out_size > cap) return 0;
  uint8_t* dst = static_cast<uint8_t*>(out);
  if (one_trip) {
    std::memcpy(dst, stage + s.out_off, s.out_size);
    return s.out_size;
  }
  // in pieces: the copy out of piece k overlaps the DMA of piece k + 1
  const size_t m = s.out_size;
  const size_t piece = stage_piece(m);
  if (!made_stage_events) {
    for (cudaEvent_t& ev : stage_ev) cudaEventCreateWithFlags(&ev, cudaEventDisableTiming);
    made_stage_events = true;
  }
  int k = 0;
  for (size_t o = 0; o < m; o += piece, ++k) {
    const size_t len = std::min(piece, m - o);
    if (cudaMemcpyAsync(stage + o, static_cast<uint8_t*>(d_out.p) + s.out_off + o, len, cudaMemcpyDeviceToHost,
                        stream) != cudaSuccess ||
        cudaEventRecord(stage_ev[k], stream) != cudaSuccess) {
      set_error("D2H failed");
      return 0;
    }
  }
  k = 0;
  for (size_t o = 0; o < m; o += piece, ++k) {
    if (cudaEventSynchronize(stage_ev[k]) != cudaSuccess) {
      set_error("D2H failed");
      return 0;
    }
    host_copy(dst + o, stage + o, std::min(piece, m - o));
  }
  return s.out_size;
}

uint32_t Engine::checksum_host(uint32_t init, const void* data, size_t n, bool adler) {
  if (n == 0) return init;
  if (!ensure_io(align_up(n, 16), 64) || !h_stage.ensure(std::max(n, kStageMin))) return init;
  host_copy(h_stage.p, data, n);
  if (cudaMemcpyAsync(d_in.p, h_stage.p, n, cudaMemcpyHostToDevice, stream) != cudaSuccess) {
    set_error("H2D failed");
    return init;
  }
  return checksum_device(init, static_cast<const uint8_t*>(d_in.p), n, adler);
}

uint32_t Engine::checksum_device(uint32_t init, const uint8_t* d_data, size_t n, bool adler) {
  if (n == 0) return init;
  // checksum blocks of the whole buffer
  cks.clear();
  for (uint64_t o = 0; o < n; o += 65536) {
    CkBlock c{};
    c.in_off = o;
    c.len = uint32_t(std::min<uint64_t>(65536, n - o));
    c.what = adler ? kCkAdler : kCkCrc;
    cks.push_back(c);
  }
  const size_t ck_bytes = cks.size() * sizeof(CkBlock);
  if (!d_tables.ensure(ck_bytes + 256)) return init;
  uint32_t* d_res = reinterpret_cast<uint32_t*>(static_cast<uint8_t*>(d_tables.p) + align_up(ck_bytes, 256));
  Work w{};
  w.in = d_data;
  w.ck = static_cast<CkBlock*>(d_tables.p);
  w.nck = uint32_t(cks.size());
  uint32_t res = init;
  if (cudaMemcpyAsync(d_tables.p, cks.data(), ck_bytes, cudaMemcpyHostToDevice, stream) != cudaSuccess) {
    set_error("H2D failed");
    return init;
  }
  launch_ck_single(w.ck, w.nck, n, init, adler ? 1 : 0, d_res, w, stream);
  if (cudaMemcpyAsync(&res, d_res, 4, cudaMemcpyDeviceToHost, stream) != cudaSuccess ||
      cudaStreamSynchronize(stream) != cudaSuccess) {
    set_error("checksum failed");
    return init;
  }
  return res;
}

std::mutex& global_mutex() { static std::mutex m; return m; }
deflate_allocator g_allocator{};  // set by deflate_set_allocator, never used to allocate

int current_device() {
  int dev = -1;
  if (cudaGetDevice(&dev) != cudaSuccess) {
    cudaGetLastError();
    set_error("no CUDA device");
    return -1;
  }
  if (dev < 0 || dev >= kMaxDevices) {
    set_error("CUDA device index above 63");
    return -1;
  }
  return dev;
}

namespace {
struct EnginePool {
  std::mutex mu;
  std::condition_variable cv;
  std::vector<Engine*> idle;  // most recently returned last
  int created = 0;
};
EnginePool& pool_of(int dev) {
  static EnginePool pools[kMaxDevices];
  return pools[dev];
}
}  // namespace

EngineLease::EngineLease() {
  dev_ = current_device();
  if (dev_ < 0) return;
  EnginePool& P = pool_of(dev_);
  std::unique_lock<std::mutex> lk(P.mu);
  P.cv.wait(lk, [&] { return !P.idle.empty() || P.created < kMaxEngines; });
  if (!P.idle.empty()) {
    e_ = P.idle.back();
    P.idle.pop_back();
    return;
  }
  ++P.created;
  lk.unlock();
  Engine* e = new (std::nothrow) Engine();  // binds to this thread's current device, dev_
  if (e && e->ok) {
    e->use_stream_ordered_arenas();  // its work runs on its own stream only
    e_ = e;
    return;
  }
  delete e;
  lk.lock();
  --P.created;
  P.cv.notify_one();
}

EngineLease::~EngineLease() {
  if (!e_) return;
  EnginePool& P = pool_of(dev_);
  {
    std::lock_guard<std::mutex> lk(P.mu);
    P.idle.push_back(e_);
  }
  P.cv.notify_one();
}

}  // namespace orotb

// ====================================================================== C ABI
using namespace orotb;

struct deflate_parallel_ctx {
  int level;
  int fmt;
  size_t block;
};

extern "C" {

// Kept for ABI compatibility: like the reference (src/api/deflate_api.cpp:75-77)
// the allocator is stored and nothing allocates through it (device memory
// never comes from a host allocator).
void deflate_set_allocator(const deflate_allocator* a) {
  std::lock_guard<std::mutex> lk(global_mutex());
  g_allocator = a ? *a : deflate_allocator{};
}

size_t deflate_compress_bound(size_t n, deflate_format f) { return framed_bound(n, int(f)); }

size_t deflate_compress(const void* in, size_t n, void* out, size_t cap, int level, deflate_format f) {
  const int fmt = int(f);
  if (fmt < 0 || fmt > 2) return 0;
  if (cap < framed_bound(n, fmt)) return 0;
  if ((n && !in) || !out) return 0;
  EngineLease e;
  return e ? e->compress_host(in, n, out, cap, level, fmt, false, 0) : 0;
}

deflate_parallel_ctx* deflate_parallel_new(int level, deflate_format f, int, size_t block) {
  if (int(f) < 0 || int(f) > 2) return nullptr;
  return new (std::nothrow) deflate_parallel_ctx{level, int(f), block};
}
void deflate_parallel_free(deflate_parallel_ctx* c) { delete c; }

size_t deflate_parallel_compress(deflate_parallel_ctx* c, const void* in, size_t n, void* out, size_t cap) {
  if (!c || (n && !in) || !out) return 0;
  EngineLease e;
  return e ? e->compress_host(in, n, out, cap, c->level, c->fmt, true, c->block) : 0;
}

uint32_t deflate_crc32(uint32_t init, const void* data, size_t len) {
  if (!data || !len) return init;
  EngineLease e;
  return e ? e->checksum_host(init, data, len, false) : init;
}
uint32_t deflate_adler32(uint32_t init, const void* data, size_t len) {
  if (!data || !len) return init;
  EngineLease e;
  return e ? e->checksum_host(init, data, len, true) : init;
}

const char* orot_b200_last_error(void) { return g_err.c_str(); }
const char* orot_b200_geometry_source(void) { return kGeometrySource; }

uint32_t orot_b200_geometry_tile(uint64_t pass_bytes, int sms, int hash_bits) {
  const GeometryRow& g = geometry_row(pass_bytes, sms);
  return hash_bits <= 12 ? g.tile12 : g.tile14;
}

}  // extern "C"
