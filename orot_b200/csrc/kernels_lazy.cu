// kernels_lazy.cu -- LZ77 with hash chains and lazy evaluation (levels 4-12)
// and dynamic Huffman blocks, on sm_100a.
//
// Search semantics follow the reference's standard path
// (src/deflate/lz77.cpp:66-156, 435-495): chains of earlier positions with the
// same 16-bit hash, newest first; up to max_chain members examined, a 4-byte
// mismatch counts as a miss and miss_limit consecutive misses end the walk,
// the longest match wins (ties keep the nearest), nice_len ends the walk;
// the lazy step moves to pos+1 when the match there is two bytes longer.
// GPU-native differences, all keeping the stream valid:
//   * a chain ends at the 32 KiB window edge (the reference keeps walking
//     with distances taken mod 32768);
//   * every position is searched once with the full chain, and the lazy
//     step uses that match (the reference searches pos+1 again with half the
//     chain, skipping the candidate at distance 1);
//   * the input is cut into independent 4 KiB tiles (16 x 258 bytes): each
//     tile parses from its own first byte and matches do not run past its
//     end, while still referencing up to 32 KiB before the tile;
//   * levels 10-12 use the same chains with 1024/2048/4096 steps instead of
//     the reference's binary tree, and an optimal parse: costs from the
//     histogram of a lazy parse, then a backward pass over the tile picks the
//     cheapest literal / match (the found match shortened by up to 31 bytes)
//     at every position;
//   * code lengths come from an optimal two-queue Huffman construction with
//     the ITU-T T.81 Annex K.3 length limiter, and the block type is chosen
//     on exact sizes (the reference uses a flat header estimate).
//
//   k_lz     one CTA per run of consecutive tiles, sliding the staged window,
//            the links and the hash table from tile to tile: links built in
//            parallel chunks plus one ordered table pass, the match searched
//            at every position (lanes take new positions as their chains
//            end), the lazy parse split
//            across lanes with a convergence fix-up, then a block-wide
//            max-scan marks covered bytes and fills the histogram.
//   k_huff   one warp per segment: code lengths, canonical codes, block type,
//            RLE code-length header (deflate_block.cpp:196-290 rules).
//   k_enc    one warp per tile: resolves tokens 32 positions at a time and
//            packs the codes into the tile's bit buffer.
#include <cuda_runtime.h>
#include <cstdint>
#include "engine.cuh"
#include "deflate_device.cuh"
#include "kernels.cuh"

namespace orotb {

namespace {

constexpr uint32_t kAll = 0xFFFFFFFFu;
constexpr uint32_t T = kLazyTile, W = kLazyWindow;
constexpr uint32_t kRegion = W + T;                            // positions with links
constexpr uint32_t kDataBytes = (W + T + 48 + 127) / 128 * 128;  // + align + over-read tail
constexpr uint32_t kLinkBytes = (kRegion * 2 + 127) / 128 * 128;  // u16 per position
constexpr uint32_t kTblBytes = 65536;                          // u16 per 15-bit hash, kept across a run
constexpr uint32_t kFBytes = T * 4;                            // F[T]; link marks before the search
constexpr uint32_t kTokBytes = T * 4;
constexpr uint32_t kFmWords = T / 32;
constexpr uint32_t kOptBytes = T * 2 + 320 * 2 + 260 * 2;      // optimal parse: choice[T], symbol and length costs
constexpr uint32_t kSmemLz = kDataBytes + kLinkBytes + kTblBytes + kFBytes + kTokBytes + kFmWords * 4 + 320 * 4 +
                             64 * 4 + kOptBytes;
static_assert(T % 32 == 0, "tiles are whole windows of 32 positions");
static_assert(kSmemLz <= 227 * 1024, "one CTA per SM");
static_assert((T & 1) == 0 && (W & 1) == 0, "window shifts move whole u32 words of links");
static_assert((kRegion + 31) / 32 * 8 <= kFBytes, "first/last marks of every link chunk fit F");

constexpr uint32_t kSerialParse = 128;  // at most this many match positions: serial parse
constexpr int kStepsPerRound = 8;       // chain steps a searching lane takes between re-balancing rounds

// chain, nice, lazy depth, miss limit, optimal parse (levels 10-12)
struct LazyCfg { int chain, nice, lazy, miss, opt; };
__constant__ LazyCfg c_lazy[13] = {
    {0, 0, 0, 5, 0},       {0, 0, 0, 5, 0},       {0, 0, 0, 5, 0},       {0, 0, 0, 5, 0},
    {64, 128, 1, 5, 0},    {128, 128, 1, 5, 0},   {128, 258, 1, 5, 0},   {256, 258, 2, 6, 0},
    {512, 258, 2, 6, 0},   {768, 258, 3, 6, 0},   {1024, 258, 3, 8, 1},  {2048, 258, 3, 8, 1},
    {4096, 258, 3, 8, 1}};

struct SmemBytes {
  const uint32_t* w;  // 16-byte aligned shared words
  uint32_t boff;      // byte offset of region position 0
  __device__ __forceinline__ uint32_t load4(uint32_t r) const {
    const uint32_t i = r + boff;
    return __funnelshift_r(w[i >> 2], w[(i >> 2) + 1], (i & 3) * 8);
  }
  __device__ __forceinline__ uint32_t byte(uint32_t r) const {
    const uint32_t i = r + boff;
    return (w[i >> 2] >> ((i & 3) * 8)) & 0xFFu;
  }
};

__device__ __forceinline__ uint32_t hash16(uint32_t v) { return (v * 0x9E3779B1u) >> 16; }
__device__ __forceinline__ uint32_t hash15(uint32_t v) { return (v * 0x9E3779B1u) >> 17; }

// The longest match at region position r, walking the chain newest first
// with the reference's rules (src/deflate/lz77.cpp:66-156): candidates of the
// same 15-bit bucket but another 16-bit hash are skipped, `chain` candidates
// with the same 16-bit hash are examined, miss_limit consecutive 4-byte
// mismatches end the walk, the quick reject at byte `best` skips candidates
// that cannot be longer, ties keep the nearest, nice length ends the walk.
// The walk advances one candidate per lz_step call so that a lane can start
// its next position as soon as its chain ends.
struct LzState {
  uint32_t r, v4p, h16p, q, maxm, best, bd;
  uint32_t pqr;  // the 4 bytes of r ending at byte `best` (the quick reject's p side), once best >= 4
  uint32_t nl;   // link of the current candidate (loaded with it, so the next step does not wait for it)
  int steps, miss, bud;
};

__device__ __forceinline__ void lz_begin(LzState& s, const SmemBytes& sd, const uint16_t* __restrict__ link, uint32_t r,
                                         uint32_t maxm, int chain) {
  s.r = r;
  s.q = r;
  s.nl = link[r];
  s.v4p = sd.load4(r);
  s.h16p = hash16(s.v4p);
  s.maxm = maxm;
  s.best = 2;
  s.bd = 0;
  s.pqr = 0;
  s.steps = chain;
  s.miss = 0;
  s.bud = 2 * chain + 64;  // bounds the filtered candidates too
}

// One candidate; returns true once the search has ended.
__device__ __forceinline__ bool lz_step(LzState& s, const SmemBytes& sd, const uint16_t* __restrict__ link, int nice,
                                        int miss_limit) {
  if (s.bud-- <= 0) return true;
  const uint32_t l = s.nl;
  if (!l) return true;
  s.q -= l;
  const uint32_t q = s.q, r = s.r;
  if (r - q > 32767u) return true;
  s.nl = link[q];
  const uint32_t v = sd.load4(q);
  if (v != s.v4p && hash16(v) != s.h16p) return false;  // same 15-bit bucket, other 16-bit chain
  if (s.steps-- == 0) return true;
  if (v != s.v4p) return ++s.miss >= miss_limit;
  s.miss = 0;
  // quick reject (src/deflate/lz77.cpp:137-142), on the 4 bytes ending at
  // byte `best`: a longer match needs all of them
  const uint32_t maxm = s.maxm, mb = s.best;
  if (mb >= 4 && mb < maxm && sd.load4(q + mb - 3) != s.pqr) return false;
  // the comparison from byte 4: aligned words on both sides, each loaded once
  uint32_t len = 4;
  {
    const uint32_t pi = r + 4 + sd.boff, qi = q + 4 + sd.boff;
    const uint32_t ps = (pi & 3) * 8, qs = (qi & 3) * 8;
    const uint32_t* pw = sd.w + (pi >> 2);
    const uint32_t* qw = sd.w + (qi >> 2);
    uint32_t plo = pw[0], qlo = qw[0];
    for (uint32_t k = 1; len < maxm; ++k) {
      const uint32_t phi = pw[k], qhi = qw[k];
      const uint32_t x = __funnelshift_r(plo, phi, ps) ^ __funnelshift_r(qlo, qhi, qs);
      if (x) { len += (__ffs(x) - 1) >> 3; break; }
      len += 4;
      plo = phi;
      qlo = qhi;
    }
  }
  if (len > maxm) len = maxm;
  if (len > s.best) {
    s.best = len;
    s.bd = r - q;
    if (int(len) >= nice || len >= maxm) return true;
    if (len >= 4) s.pqr = sd.load4(r + len - 3);
  }
  return false;
}

// First position >= i where a match starts (a set bit of fm), or tl.
__device__ __forceinline__ uint32_t next_head(const uint32_t* fm, uint32_t i, uint32_t tl) {
  if (i >= tl) return tl;
  uint32_t w = i >> 5;
  uint32_t bits = fm[w] & (kAll << (i & 31));
  while (!bits && ++w < (tl + 31) / 32) bits = fm[w];
  return bits ? min(w * 32 + __ffs(bits) - 1, tl) : tl;
}

// One step of the lazy parse from head i (F[i] != 0): up to `lazy` moves to
// i + 1 while the match there is longer by two or more (the reference's lazy
// rule, lz77.cpp:449-493; the match at i + 1 is the full search of i + 1,
// where the reference searches again with half the chain).  Returns
// {match position, len << 16 | dist}.
__device__ __forceinline__ uint2 lazy_step(const uint32_t* F, uint32_t i, uint32_t tl, int lazy) {
  uint32_t m = F[i];
  int k = lazy;
  while (k > 0 && i + (m >> 16) + 1 < tl && i + 4 <= tl) {
    const uint32_t g = F[i + 1];
    if ((g >> 16) > (m >> 16) + 1) {
      ++i;
      m = g;
      --k;
    } else {
      break;
    }
  }
  return make_uint2(i, m);
}

// Clears the bits of positions [lo, hi).
__device__ __forceinline__ void clear_bits(uint32_t* bm, uint32_t lo, uint32_t hi) {
  while (lo < hi) {
    const uint32_t w = lo >> 5, b0 = lo & 31, n = min(32u - b0, hi - lo);
    const uint32_t mask = (n == 32 ? kAll : ((1u << n) - 1)) << b0;
    bm[w] &= ~mask;
    lo += n;
  }
}

__device__ __forceinline__ uint32_t block_max_excl(uint32_t v, uint32_t* scan) {
  const uint32_t lane = threadIdx.x & 31, wid = threadIdx.x >> 5;
  uint32_t inc = v;
#pragma unroll
  for (int o = 1; o < 32; o <<= 1) {
    const uint32_t t = __shfl_up_sync(kAll, inc, o);
    if (lane >= uint32_t(o)) inc = max(inc, t);
  }
  if (lane == 31) scan[wid] = inc;
  __syncthreads();
  if (wid == 0) {
    uint32_t x = lane < (blockDim.x >> 5) ? scan[lane] : 0;
#pragma unroll
    for (int o = 1; o < 32; o <<= 1) {
      const uint32_t t = __shfl_up_sync(kAll, x, o);
      if (lane >= uint32_t(o)) x = max(x, t);
    }
    scan[32 + lane] = x;  // inclusive over warps
  }
  __syncthreads();
  const uint32_t before_warp = wid ? scan[32 + wid - 1] : 0;
  const uint32_t excl_lane = __shfl_up_sync(kAll, inc, 1);
  return max(before_warp, lane ? excl_lane : 0u);
}

__device__ __forceinline__ uint32_t len_sym(uint32_t len) {
  uint32_t li, ne, ev;
  length_code(len, li, ne, ev);
  return li;
}
__device__ __forceinline__ uint32_t dist_sym(uint32_t d) {
  uint32_t dc, ne, ev;
  dist_code(d, dc, ne, ev);
  return dc;
}

// Literal/length and distance histogram of a tile's tokens (all threads):
// a block-wide max-scan of match ends marks the bytes matches cover, every
// other byte is a literal.
__device__ void tile_histogram(const uint32_t* tok_s, uint32_t tl, const SmemBytes& sd, uint32_t off, uint32_t* hist,
                               uint32_t* scan) {
  const uint32_t per = (T + blockDim.x - 1) / blockDim.x;
  const uint32_t i0 = threadIdx.x * per;
  uint32_t me = 0;
  for (uint32_t j = 0; j < per; ++j) {
    const uint32_t i = i0 + j;
    const uint32_t tk = i < tl ? tok_s[i] : 0;
    if (tk) me = max(me, i + ((tk >> 16) & 0x1FFu));
  }
  uint32_t run = block_max_excl(me, scan);
  for (uint32_t j = 0; j < per; ++j) {
    const uint32_t i = i0 + j;
    if (i >= tl) break;
    const uint32_t tk = tok_s[i];
    if (tk) {
      const uint32_t len = (tk >> 16) & 0x1FFu;
      atomicAdd(&hist[257 + len_sym(len)], 1u);
      atomicAdd(&hist[288 + dist_sym(tk & 0xFFFFu)], 1u);
      run = max(run, i + len);
    } else if (run <= i) {
      atomicAdd(&hist[sd.byte(off + i)], 1u);
    }
  }
  __syncthreads();
}

// Bit cost (1/16 bit) of a token with `count` in a histogram of `total`
// symbols: log2(total / count), 1..15 bits; unseen symbols cost 2 bits more
// than the rarest possible.
__device__ __forceinline__ uint16_t sym_cost(uint32_t count, uint32_t total) {
  const float b = count ? __log2f(float(total) / float(count)) : __log2f(float(total)) + 2.0f;
  return uint16_t(16.0f * fminf(fmaxf(b, 1.0f), 15.0f) + 0.5f);
}

// -- staging by the bulk-copy engine (TMA, untiled; the source is this GPU's
// own input arena, no multicast): one thread starts the copy of a tile's
// window into shared memory and the CTA waits on an mbarrier for its bytes.
__device__ __forceinline__ uint32_t smem_u32(const void* p) {
  return static_cast<uint32_t>(__cvta_generic_to_shared(p));
}
__device__ __forceinline__ void mbar_init(uint64_t* bar, uint32_t count) {
  asm volatile("mbarrier.init.shared::cta.b64 [%0], %1;" ::"r"(smem_u32(bar)), "r"(count) : "memory");
  asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
}
// Orders this thread's earlier generic-proxy accesses to shared memory before
// later bulk-copy writes (every thread that touched the staged bytes runs it
// before the barrier that precedes the next copy).
__device__ __forceinline__ void fence_proxy_async_smem() { asm volatile("fence.proxy.async.shared::cta;" ::: "memory"); }
__device__ __forceinline__ void bulk_stage(void* dst, const void* src, uint32_t bytes, uint64_t* bar) {
  asm volatile("mbarrier.arrive.expect_tx.shared::cta.b64 _, [%0], %1;" ::"r"(smem_u32(bar)), "r"(bytes) : "memory");
  asm volatile("cp.async.bulk.shared::cluster.global.mbarrier::complete_tx::bytes [%0], [%1], %2, [%3];" ::"r"(
                   smem_u32(dst)),
               "l"(src), "r"(bytes), "r"(smem_u32(bar))
               : "memory");
}
__device__ __forceinline__ bool mbar_try_wait(uint64_t* bar, uint32_t phase) {
  uint32_t ok;
  asm volatile(
      "{\n .reg .pred p;\n mbarrier.try_wait.parity.shared::cta.b64 p, [%1], %2;\n selp.u32 %0, 1, 0, p;\n}"
      : "=r"(ok)
      : "r"(smem_u32(bar)), "r"(phase)
      : "memory");
  return ok != 0;
}
__device__ __forceinline__ uint64_t global_ns() {
  uint64_t t;
  asm volatile("mov.u64 %0, %%globaltimer;" : "=l"(t));
  return t;
}
// Waits for the mbarrier's phase; gives up (false) after `limit_ns`.
__device__ __forceinline__ bool mbar_wait(uint64_t* bar, uint32_t phase, uint64_t limit_ns) {
  if (mbar_try_wait(bar, phase)) return true;
  const uint64_t t0 = global_ns();
  while (!mbar_try_wait(bar, phase))
    if (global_ns() - t0 > limit_ns) return false;
  return true;
}
constexpr uint64_t kStageWaitNs = 1000000000ull;  // a copy of 37 KB that takes a second has failed

}  // namespace

// ---------------------------------------------------------------- k_lz
// One CTA per run of up to kLazyRun consecutive tiles of a segment.  The
// links of the window and the hash table carry from one tile to the next
// (shifted down by the tile length), so each position is linked once.
__global__ void __launch_bounds__(1024, 1) k_lz(Work wk, const uint32_t* __restrict__ runs, uint32_t nruns) {
  extern __shared__ __align__(16) uint8_t sm[];
  uint32_t* sdata = reinterpret_cast<uint32_t*>(sm);
  uint16_t* link = reinterpret_cast<uint16_t*>(sm + kDataBytes);
  uint16_t* tbl = reinterpret_cast<uint16_t*>(sm + kDataBytes + kLinkBytes);
  uint8_t* fgb = sm + kDataBytes + kLinkBytes + kTblBytes;
  uint32_t* F = reinterpret_cast<uint32_t*>(fgb);
  uint32_t* tok_s = reinterpret_cast<uint32_t*>(fgb + kFBytes);
  uint32_t* fm = tok_s + T;
  uint32_t* hist = fm + kFmWords;
  uint32_t* scan = hist + 320;
  uint16_t* choice = reinterpret_cast<uint16_t*>(scan + 64);  // optimal parse: token length at each position
  uint16_t* scost = choice + T;                              // symbol costs, 1/16 bit: 0-255 literals, 257+ lengths, 288+ distances
  uint16_t* lcost = scost + 320;                             // cost of a match length 0..258 (code + extra bits)
  const uint32_t tid = threadIdx.x, lane = tid & 31, wid = tid >> 5;

  if (blockIdx.x >= nruns) return;
  __shared__ __align__(8) uint64_t stage_bar;  // completion of the bulk copy of a tile's window
  if (tid == 0) mbar_init(&stage_bar, 1);
  __syncthreads();
  uint32_t stage_phase = 0;
  const uint32_t first = runs[2 * blockIdx.x];
  const uint32_t last = first + runs[2 * blockIdx.x + 1];
  const Segment sg = wk.segs[wk.tiles[first].seg];
  const LazyCfg cfg = c_lazy[sg.level];
  uint32_t prev_rs = 0, prev_nreg = 0;

  for (uint32_t ti = first; ti < last; ++ti) {
    Tile* tp = wk.tiles + ti;
    const Tile t = *tp;
    const uint32_t ts = t.start, tl = t.len, tend = ts + tl;
    const uint32_t rs = ts > W ? ts - W : 0;           // region start (segment-relative)
    const uint32_t nreg = tend - rs;                    // positions with links
    const uint32_t copy_end = min(sg.len, tend + 8);    // bytes staged
    // -- stage bytes [rs, copy_end) at 16-byte granularity
    const uint64_t g0 = (sg.in_off + rs) & ~uint64_t(15);
    const uint32_t boff = uint32_t(sg.in_off + rs - g0);
    const uint32_t n16 = (boff + (copy_end - rs) + 15) / 16;
    // one thread starts the bulk copy; meanwhile the CTA clears the tail (the
    // bytes past the copy that whole-word reads may touch) and slides the
    // links and the table, which do not depend on the new bytes
    uint4* dst = reinterpret_cast<uint4*>(sm);
    if (tid == 0) bulk_stage(dst, wk.in + g0, n16 * 16, &stage_bar);
    for (uint32_t i = n16 + tid; i < kDataBytes / 16; i += blockDim.x) dst[i] = make_uint4(0, 0, 0, 0);
    for (uint32_t i = tid; i < 320; i += blockDim.x) hist[i] = 0;
    // -- carry links and table from the previous tile, or start empty
    uint32_t lstart = 0;
    if (ti == first) {
      for (uint32_t i = tid; i < kTblBytes / 4; i += blockDim.x) reinterpret_cast<uint32_t*>(tbl)[i] = kAll;
    } else {
      const uint32_t shift = rs - prev_rs;  // even: tiles and the window are even
      const uint32_t keep = prev_nreg - shift;
      uint32_t* lw = reinterpret_cast<uint32_t*>(link);
      constexpr uint32_t kMaxWords = (kRegion / 2 + 1023) / 1024;
      uint32_t tmp[kMaxWords];
#pragma unroll
      for (uint32_t k = 0; k < kMaxWords; ++k) {
        const uint32_t wi = tid + k * 1024;
        tmp[k] = wi * 2 < keep ? lw[wi + shift / 2] : 0u;
      }
      __syncthreads();
#pragma unroll
      for (uint32_t k = 0; k < kMaxWords; ++k) {
        const uint32_t wi = tid + k * 1024;
        if (wi * 2 < keep) {
          // a link that now points before the region start is dropped
          uint32_t lo = tmp[k] & 0xFFFFu, hi = tmp[k] >> 16;
          if (lo > wi * 2) lo = 0;
          if (hi > wi * 2 + 1) hi = 0;
          lw[wi] = lo | (hi << 16);
        }
      }
      for (uint32_t i = tid; i < 32768; i += blockDim.x) {
        const uint32_t e = tbl[i];
        tbl[i] = (e != 0xFFFFu && e >= shift) ? uint16_t(e - shift) : uint16_t(0xFFFFu);
      }
      lstart = keep;
    }
    const bool staged = mbar_wait(&stage_bar, stage_phase, kStageWaitNs);
    stage_phase ^= 1u;
    if (!__syncthreads_and(staged)) {
      // the copy did not complete: mark the stream failed, give the copy
      // another bounded wait so that no copy is left in flight, and stop
      if (tid == 0) atomicOr(&wk.segs[t.seg].flags, kSegFault);
      mbar_wait(&stage_bar, stage_phase ^ 1u, kStageWaitNs);
      return;
    }
    const SmemBytes sd{sdata, boff};

    // -- links of the new positions [lstart, nreg): the previous position
    // with the same 15-bit hash.  (1) All warps, 32-position chunks: the
    // nearest earlier lane with the same hash is the link inside the chunk;
    // the first lane of every hash is marked and, until step (2), holds in
    // its link the offset to the hash's last lane in the chunk.  (2) Warp 0,
    // chunk after chunk: each first lane reads the table's position (its
    // link) and writes its hash's last position in the chunk.  Only step (2)
    // is sequential: one table read and write per distinct hash, by one lane,
    // and one warp barrier per chunk (the next chunk's reads come after).
    {
      const uint32_t nch = (nreg - lstart + 31) / 32;
      uint32_t* fbits = F;  // F is free until the searches
      const uint32_t lt = (1u << lane) - 1;
      for (uint32_t c = wid; c < nch; c += blockDim.x >> 5) {
        const uint32_t x = lstart + c * 32 + lane;
        const bool valid = x < nreg && rs + x + 4 <= sg.len;
        const uint32_t h = valid ? hash15(sd.load4(x)) : 0x10000u + lane;  // invalid lanes match nobody
        const uint32_t peers = __match_any_sync(kAll, h);
        const uint32_t before = peers & lt;
        const bool is_first = valid && !before;
        if (x < nreg)
          link[x] = before ? uint16_t(__clz(before) - (31 - lane))
                           : is_first ? uint16_t((31 - __clz(peers)) - lane) : uint16_t(0);
        const uint32_t first = __ballot_sync(kAll, is_first);
        if (lane == 0) fbits[c] = first;
      }
      __syncthreads();
      if (wid == 0) {
        // eight chunks per round: their marks, hashes and last positions are
        // loaded first, then the table reads and writes go in chunk order
        // without waiting for each other's results
        constexpr uint32_t U = 8;
        for (uint32_t c0 = 0; c0 < nch; c0 += U) {
          uint32_t fb[U], h[U], p[U], lastp[U];
#pragma unroll
          for (uint32_t u = 0; u < U; ++u) fb[u] = c0 + u < nch ? (fbits[c0 + u] >> lane) & 1u : 0u;
#pragma unroll
          for (uint32_t u = 0; u < U; ++u) {
            const uint32_t x = lstart + (c0 + u) * 32 + lane;
            h[u] = fb[u] ? hash15(sd.load4(x)) : 0u;
            lastp[u] = fb[u] ? x + link[x] : 0u;
          }
#pragma unroll
          for (uint32_t u = 0; u < U; ++u) {
            p[u] = 0xFFFFu;
            if (fb[u]) {
              p[u] = tbl[h[u]];
              tbl[h[u]] = uint16_t(lastp[u]);
            }
            __syncwarp();
          }
#pragma unroll
          for (uint32_t u = 0; u < U; ++u) {
            const uint32_t x = lstart + (c0 + u) * 32 + lane;
            if (fb[u]) link[x] = p[u] == 0xFFFFu ? uint16_t(0) : uint16_t(x - p[u]);
          }
        }
      }
    }
    if (tid == 0) scan[62] = 0;
    __syncthreads();

    // -- searches at every tile position.  Warps take 32-position chunks; a
    // lane whose chain has ended takes the next position of its warp's chunk
    // at once, so lanes stay busy across chains of very different lengths.
    {
      const uint32_t nsearch = tl >= 4 ? tl - 3 : 0;
      const uint32_t nch = (nsearch + 31) / 32;
      for (uint32_t i = nsearch + tid; i < kFmWords * 32; i += blockDim.x) F[i] = 0;
      const uint32_t lt = (1u << lane) - 1;
      uint32_t pool = 0, avail = 0;  // warp-uniform: next position of the chunk, positions left
      bool more = true;
      uint32_t i = kAll;             // this lane's position
      LzState st;
      for (;;) {
        uint32_t idle = __ballot_sync(kAll, i == kAll);
        while (idle && (avail || more)) {
          if (!avail) {
            uint32_t c = 0;
            if (lane == 0) c = atomicAdd(&scan[62], 1u);
            c = __shfl_sync(kAll, c, 0);
            if (c >= nch) {
              more = false;
              break;
            }
            pool = c * 32;
            avail = min(32u, nsearch - pool);
          }
          const uint32_t take = min(uint32_t(__popc(idle)), avail);
          if (i == kAll && __popc(idle & lt) < take) {
            i = pool + __popc(idle & lt);
            lz_begin(st, sd, link, ts - rs + i, min(258u, tl - i), cfg.chain);
          }
          pool += take;
          avail -= take;
          idle = __ballot_sync(kAll, i == kAll);
        }
        if (idle == kAll) break;
        // a few chain steps per round: the warp re-balances (ballot, new
        // positions for lanes whose chain ended) once per kStepsPerRound steps
        if (i != kAll) {
#pragma unroll 1
          for (int k = 0; k < kStepsPerRound; ++k) {
            if (lz_step(st, sd, link, cfg.nice, cfg.miss)) {
              F[i] = st.best >= 3 ? (st.best << 16) | st.bd : 0u;
              i = kAll;
              break;
            }
          }
        }
      }
    }
    __syncthreads();
    for (uint32_t c = wid; c < kFmWords; c += blockDim.x >> 5) {
      const uint32_t b = __ballot_sync(kAll, F[c * 32 + lane] != 0);
      if (lane == 0) fm[c] = b;
    }
    for (uint32_t i = tid; i < T; i += blockDim.x) tok_s[i] = 0;
    __syncthreads();

    // -- parse (reference lazy rule, lz77.cpp:449-493, with n = tile end).
    // A parse step depends only on its start position (the head), so the
    // heads are found in parallel: (1) each lane of warp 0 parses one 1/32 of
    // the tile from its start; (2) lane 0 follows the true parse into every
    // segment until it meets a head of that segment's parse, after which the
    // two are the same; (3) every thread emits the matches of its heads.
    {
      uint32_t* hd = hist;  // heads, a bit per position (hist is zero until the histogram)
      uint32_t* sx = scan;  // where each segment's parse leaves it
      const uint32_t S = (tl + 31) / 32;
      uint32_t nf = 0;  // positions with a match: few -> one lane parses alone
      if (wid == 0) {
        for (uint32_t w = lane; w < kFmWords; w += 32) nf += __popc(fm[w]);
        nf = __reduce_add_sync(kAll, nf);
      }
      if (wid == 0 && nf <= kSerialParse) {
        if (lane == 0) {
          uint32_t i = 0;
          while ((i = next_head(fm, i, tl)) < tl) {
            hd[i >> 5] |= 1u << (i & 31);
            const uint2 m = lazy_step(F, i, tl, cfg.lazy);
            i = (m.x & 0xFFFFu) + (m.y >> 16);
          }
        }
      } else if (wid == 0) {
        const uint32_t a = min(lane * S, tl), b = min(a + S, tl);
        uint32_t i = a;
        while (i < b) {
          i = next_head(fm, i, tl);
          if (i >= b) break;
          atomicOr(&hd[i >> 5], 1u << (i & 31));
          const uint2 m = lazy_step(F, i, tl, cfg.lazy);
          i = (m.x & 0xFFFFu) + (m.y >> 16);
        }
        sx[lane] = i;
        __syncwarp();
        if (lane == 0) {
          uint32_t e = sx[0];
          for (uint32_t sgi = 1; sgi < 32; ++sgi) {
            const uint32_t a2 = min(sgi * S, tl), b2 = min(a2 + S, tl);
            if (a2 >= b2) break;
            clear_bits(hd, a2, min(e, b2));
            if (e >= b2) continue;
            uint32_t i2 = e;
            for (;;) {
              const uint32_t h = next_head(fm, i2, tl);
              if (h >= b2) {
                e = h;
                break;
              }
              if ((hd[h >> 5] >> (h & 31)) & 1u) {
                e = sx[sgi];
                break;
              }
              hd[h >> 5] |= 1u << (h & 31);
              const uint2 m = lazy_step(F, h, tl, cfg.lazy);
              i2 = (m.x & 0xFFFFu) + (m.y >> 16);
              clear_bits(hd, h + 1, min(i2, b2));
              if (i2 >= b2) {
                e = i2;
                break;
              }
            }
          }
        }
      }
      __syncthreads();
      for (uint32_t i = tid; i < tl; i += blockDim.x) {
        if ((hd[i >> 5] >> (i & 31)) & 1u) {
          const uint2 m = lazy_step(F, i, tl, cfg.lazy);
          tok_s[m.x & 0xFFFFu] = 0x80000000u | m.y;
        }
      }
      __syncthreads();
      if (wid == 0) {
        uint32_t nm = 0;
        for (uint32_t w = lane; w < kFmWords; w += 32) {
          nm += __popc(hd[w]);
          hd[w] = 0;
        }
        nm = __reduce_add_sync(kAll, nm);
        if (lane == 0) scan[63] = nm;
      }
    }
    __syncthreads();

    // -- levels 10-12: optimal parse.  Costs come from the histogram of the
    // lazy parse above; a backward pass finds, for every position, the
    // cheapest way to the tile end (a literal, or the match found there
    // shortened by up to 31 bytes), then the path from position 0 is read.
    if (cfg.opt) {
      tile_histogram(tok_s, tl, sd, ts - rs, hist, scan);
      {
        uint32_t lt = 1, dt = 0;  // totals (EOB counts once)
        for (uint32_t k = 0; k < 286; ++k) lt += hist[k];
        for (uint32_t k = 288; k < 318; ++k) dt += hist[k];
        for (uint32_t k = tid; k < 320; k += blockDim.x)
          scost[k] = k < 288 ? sym_cost(hist[k], lt) : sym_cost(hist[k], dt > 0 ? dt : 1);
      }
      __syncthreads();
      for (uint32_t k = tid; k < 320; k += blockDim.x) hist[k] = 0;
      for (uint32_t k = tid; k < 259; k += blockDim.x) {
        uint32_t li = 0, lne = 0, lev;
        if (k >= 3) length_code(k, li, lne, lev);
        lcost[k] = k >= 3 ? uint16_t(scost[257 + li] + 16 * lne) : uint16_t(0);
      }
      // per position, before the backward pass: cost[i] = literal cost,
      // choice[i] = cost of the distance of the match found at i
      uint32_t* cost = tok_s;  // cost to the tile end, per position (tokens are rebuilt below)
      for (uint32_t i = tid; i < tl; i += blockDim.x) {
        cost[i] = scost[sd.byte(ts - rs + i)];
        uint32_t dc = 0, dne = 0, dev;
        if (F[i]) dist_code(F[i] & 0xFFFFu, dc, dne, dev);
        choice[i] = F[i] ? uint16_t(scost[288 + dc] + 16 * dne) : uint16_t(0);
      }
      __syncthreads();
      if (wid == 0) {
        uint32_t next = 0;  // cost[i + 1]
        for (int i = int(tl) - 1; i >= 0; --i) {
          const uint32_t f = F[i];
          uint32_t best = ((cost[i] + next) << 9) | 1u;
          if (f) {
            const uint32_t flen = f >> 16, dcost = choice[i];
            const uint32_t L = flen - lane;
            uint32_t key = kAll;
            if (lane + 3 <= flen) key = ((lcost[L] + dcost + (i + L < tl ? cost[i + L] : 0u)) << 9) | L;
            best = __reduce_min_sync(kAll, lane == 0 ? min(key, best) : key);
          }
          next = best >> 9;
          __syncwarp();
          if (lane == 0) {
            cost[i] = next;
            choice[i] = uint16_t(best & 511u);
          }
          __syncwarp();
        }
      }
      __syncthreads();
      for (uint32_t i = tid; i < T; i += blockDim.x) tok_s[i] = 0;
      __syncthreads();
      if (tid == 0) {
        uint32_t i = 0, nm = 0;
        while (i < tl) {
          const uint32_t c = choice[i];
          if (c >= 3) {
            tok_s[i] = 0x80000000u | (c << 16) | (F[i] & 0xFFFFu);
            ++nm;
            i += c;
          } else {
            ++i;
          }
        }
        scan[63] = nm;
      }
      __syncthreads();
    }

    // -- covered bytes (max-scan of match ends) and the histogram
    const uint32_t nm = scan[63];
    __syncthreads();
    tile_histogram(tok_s, tl, sd, ts - rs, hist, scan);
    uint32_t* gh = reinterpret_cast<uint32_t*>(wk.scratch + t.hist);
    for (uint32_t i = tid; i < 320; i += blockDim.x) gh[i] = hist[i];
    uint32_t* gt = reinterpret_cast<uint32_t*>(wk.scratch + t.tok);
    for (uint32_t i = tid; i < tl; i += blockDim.x) gt[i] = tok_s[i];
    if (tid == 0) {
      tp->fin_matches = nm;
      tp->fix_bits = 0;
      tp->splice_bit = 0;
    }
    prev_rs = rs;
    prev_nreg = nreg;
    fence_proxy_async_smem();  // this tile's reads and writes of the staged bytes, before the next copy
    __syncthreads();
  }
}

// ---------------------------------------------------------------- Huffman
// Code lengths for one alphabet.  Symbols with non-zero frequency are sorted
// by (frequency, symbol) (by the warp, huff_sort); on one thread the two-queue construction
// (leaves in sorted order, internal nodes in creation order, a leaf wins a
// tie) builds an optimal tree; if it is deeper than `limit` the per-length
// counts are adjusted as in ITU-T T.81 Annex K.3 and lengths are handed out
// longest-first to the least frequent symbols.
struct HuffScratch {
  uint16_t sym[288];
  uint32_t w[288];      // internal node weights
  uint16_t par[576];    // parent of leaf i (0..m-1) and node k (m+k)
  uint8_t dep[576];
  uint32_t cnt[64];
};

// Sorts the used symbols (non-zero frequency) by (frequency, symbol) into
// s.sym and clears len[]: every lane ranks its symbols against all others.
// All lanes of the warp call it; returns the number of used symbols.
__device__ int huff_sort(const uint32_t* freq, int n, uint8_t* len, HuffScratch& s) {
  const int lane = int(threadIdx.x & 31);
  int m = 0;
  for (int i0 = 0; i0 < n; i0 += 32) {
    const int i = i0 + lane;
    m += __popc(__ballot_sync(kAll, i < n && freq[i] != 0));
    if (i < n) len[i] = 0;
  }
  for (int i = lane; i < n; i += 32) {
    const uint32_t fi = freq[i];
    if (!fi) continue;
    int r = 0;
    for (int j = 0; j < n; ++j) {
      const uint32_t fj = freq[j];
      r += (fj != 0 && (fj < fi || (fj == fi && j < i))) ? 1 : 0;
    }
    s.sym[r] = uint16_t(i);
  }
  __syncwarp();
  return m;
}

// Code lengths of the m sorted symbols (one lane; after huff_sort).
__device__ void huff_lengths(const uint32_t* freq, int m, uint8_t* len, int limit, HuffScratch& s) {
  if (m == 0) return;
  if (m == 1) { len[s.sym[0]] = 1; return; }
  int li = 0, ni = 0;
  for (int k = 0; k < m - 1; ++k) {
    uint32_t wsum = 0;
    for (int pick = 0; pick < 2; ++pick) {
      const bool leaf_ok = li < m;
      const bool node_ok = ni < k;
      bool take_leaf;
      if (leaf_ok && node_ok) take_leaf = freq[s.sym[li]] <= s.w[ni];
      else take_leaf = leaf_ok;
      if (take_leaf) { wsum += freq[s.sym[li]]; s.par[li] = uint16_t(m + k); ++li; }
      else { wsum += s.w[ni]; s.par[m + ni] = uint16_t(m + k); ++ni; }
    }
    s.w[k] = wsum;
  }
  const int root = m + m - 2;
  s.dep[root] = 0;
  for (int k = m - 3; k >= 0; --k) s.dep[m + k] = uint8_t(min(63, s.dep[s.par[m + k]] + 1));
  int maxd = 0;
  for (int i = 0; i < m; ++i) {
    s.dep[i] = uint8_t(min(63, s.dep[s.par[i]] + 1));
    maxd = max(maxd, int(s.dep[i]));
  }
  if (maxd <= limit) {
    for (int i = 0; i < m; ++i) len[s.sym[i]] = s.dep[i];
    return;
  }
  for (int d = 0; d < 64; ++d) s.cnt[d] = 0;
  for (int i = 0; i < m; ++i) ++s.cnt[s.dep[i]];
  for (int i = maxd; i > limit; --i) {
    while (s.cnt[i] > 0) {
      int j = i - 2;
      while (s.cnt[j] == 0) --j;
      s.cnt[i] -= 2;
      s.cnt[i - 1] += 1;
      s.cnt[j + 1] += 2;
      s.cnt[j] -= 1;
    }
  }
  int idx = 0;
  for (int l = limit; l >= 1; --l)
    for (uint32_t k = 0; k < s.cnt[l]; ++k) len[s.sym[idx++]] = uint8_t(l);
}

// Canonical codes (RFC 1951 3.2.2), reversed for LSB-first output.
__device__ void canon(const uint8_t* len, int n, uint32_t* out /* code | len << 16 */) {
  uint32_t bl[16] = {0};
  for (int i = 0; i < n; ++i) bl[len[i]] += len[i] ? 1 : 0;
  uint32_t next[16];
  uint32_t code = 0;
  next[0] = 0;
  for (int b = 1; b < 16; ++b) { code = (code + bl[b - 1]) << 1; next[b] = code; }
  for (int i = 0; i < n; ++i) {
    const uint32_t l = len[i];
    out[i] = l ? (rev_bits(next[l]++, l) | (l << 16)) : 0u;
  }
}

struct BitOut {
  uint32_t* w;
  uint32_t pos;
  __device__ void put(uint32_t v, uint32_t n) {
    if (!n) return;
    v &= n == 32 ? kAll : ((1u << n) - 1);
    const uint32_t i = pos >> 5, sh = pos & 31;
    w[i] |= v << sh;
    if (sh + n > 32) w[i + 1] |= v >> (32 - sh);
    pos += n;
  }
};

__constant__ uint8_t c_len_extra[29] = {0, 0, 0, 0, 0, 0, 0, 0, 1, 1, 1, 1, 2, 2, 2, 2, 3, 3, 3, 3, 4, 4, 4, 4, 5, 5, 5, 5, 0};
__constant__ uint8_t c_dist_extra[30] = {0, 0, 0, 0, 1, 1, 2, 2, 3, 3, 4, 4, 5, 5, 6, 6, 7, 7, 8, 8, 9, 9, 10, 10, 11, 11, 12, 12, 13, 13};
__constant__ uint8_t c_cl_order[19] = {16, 17, 18, 0, 8, 7, 9, 6, 10, 5, 11, 4, 12, 3, 13, 2, 14, 1, 15};

constexpr int kHuffWarps = 4;
struct HuffSmem {
  uint32_t freq[320];
  uint8_t ll[288], dl[32], cl[19];
  uint8_t seq[320];
  uint8_t rsym[320], rext[320];
  uint32_t clf[19];
  uint32_t clc[19];
  HuffScratch hs;
};

__global__ void __launch_bounds__(kHuffWarps * 32) k_huff(Work wk, const uint32_t* __restrict__ list, uint32_t nlist) {
  __shared__ HuffSmem S[kHuffWarps];
  const uint32_t wid = threadIdx.x >> 5, lane = threadIdx.x & 31;
  const uint32_t si = blockIdx.x * kHuffWarps + wid;
  if (si >= nlist) return;
  HuffSmem& H = S[wid];
  Segment* gp = wk.segs + list[si];
  const Segment sg = *gp;
  for (uint32_t b = lane; b < 320; b += 32) {
    uint32_t f = 0;
    for (uint32_t t = sg.tile_first; t < sg.tile_first + sg.tile_count; ++t)
      f += reinterpret_cast<const uint32_t*>(wk.scratch + wk.tiles[t].hist)[b];
    H.freq[b] = f;
  }
  uint32_t mt = 0;
  for (uint32_t t = sg.tile_first + lane; t < sg.tile_first + sg.tile_count; t += 32) mt += wk.tiles[t].fin_matches;
#pragma unroll
  for (int o = 16; o; o >>= 1) mt += __shfl_xor_sync(kAll, mt, o);
  uint32_t* codes = reinterpret_cast<uint32_t*>(wk.scratch + sg.codes);
  uint32_t* hdr = reinterpret_cast<uint32_t*>(wk.scratch + sg.hdr_off);
  for (uint32_t i = lane; i < 256; i += 32) hdr[i] = 0;
  if (lane == 0) H.freq[256] = 1;  // EOB
  __syncwarp();
  const bool all_literal = (sg.flags & kSegWholeBuf) && mt == 0;  // warp-uniform
  int m_ll = 0, m_dl = 0;
  if (!all_literal) {
    // the symbol sorts of both alphabets, by the whole warp
    m_ll = huff_sort(H.freq, 288, H.ll, H.hs);
    if (lane == 0) huff_lengths(H.freq, m_ll, H.ll, 15, H.hs);
    __syncwarp();
    m_dl = huff_sort(H.freq + 288, 32, H.dl, H.hs);
    if (lane == 0) huff_lengths(H.freq + 288, m_dl, H.dl, 15, H.hs);
    __syncwarp();
  }
  if (lane != 0) return;

  uint32_t type;
  uint32_t hbits = 0, eob = 0;
  const uint32_t pieces = sg.len ? (sg.len + 65534) / 65535 : 1;
  const uint64_t stored_bits = (uint64_t(sg.len) + 5ull * pieces) * 8;
  if (all_literal) {
    type = kBlkStored;  // all-literal parse (block_compressor.cpp:60-61)
  } else {
    // fixed cost (deflate_block.cpp:50-70)
    uint64_t ext = 0;
    for (int i = 0; i < 29; ++i) ext += uint64_t(c_len_extra[i]) * H.freq[257 + i];
    for (int i = 0; i < 30; ++i) ext += uint64_t(c_dist_extra[i]) * H.freq[288 + i];
    uint64_t fixed_bits = 3 + ext;
    for (int i = 0; i < 288; ++i) fixed_bits += uint64_t(i < 144 ? 8 : i < 256 ? 9 : i < 280 ? 7 : 8) * H.freq[i];
    for (int i = 0; i < 30; ++i) fixed_bits += 5ull * H.freq[288 + i];
    // dynamic code (deflate_block.cpp:347-383 conventions); the lengths of
    // both alphabets were built above
    if (H.ll[256] == 0) H.ll[256] = 1;
    bool any = false;
    for (int i = 0; i < 32; ++i) any |= H.dl[i] != 0;
    if (!any) H.dl[0] = 1;
    int hlit = 288, hdist = 32;
    while (hlit > 257 && H.ll[hlit - 1] == 0) --hlit;
    while (hdist > 1 && H.dl[hdist - 1] == 0) --hdist;
    // run-length code of the lengths (deflate_block.cpp:212-242)
    for (int i = 0; i < hlit; ++i) H.seq[i] = H.ll[i];
    for (int i = 0; i < hdist; ++i) H.seq[hlit + i] = H.dl[i];
    const int total = hlit + hdist;
    int nr = 0;
    for (int i = 0; i < total;) {
      const uint8_t v = H.seq[i];
      int run = 1;
      while (i + run < total && H.seq[i + run] == v && run < 138) ++run;
      if (v == 0 && run >= 3) {
        H.rsym[nr] = run <= 10 ? 17 : 18;
        H.rext[nr++] = uint8_t(run <= 10 ? run - 3 : run - 11);
        i += run;
      } else if (v != 0 && run >= 4) {
        H.rsym[nr] = v; H.rext[nr++] = 0xFF;
        ++i;
        const int rep = min(run - 1, 6);
        H.rsym[nr] = 16; H.rext[nr++] = uint8_t(rep - 3);
        i += rep;
      } else {
        H.rsym[nr] = v; H.rext[nr++] = 0xFF;
        ++i;
      }
    }
    for (int i = 0; i < 19; ++i) H.clf[i] = 0;
    for (int i = 0; i < nr; ++i) ++H.clf[H.rsym[i]];
    int m_cl = 0;
    for (int i = 0; i < 19; ++i) {  // 19 symbols: sorted on this lane (insertion by (frequency, symbol))
      H.cl[i] = 0;
      if (!H.clf[i]) continue;
      int j = m_cl++;
      while (j > 0 && H.clf[H.hs.sym[j - 1]] > H.clf[i]) { H.hs.sym[j] = H.hs.sym[j - 1]; --j; }
      H.hs.sym[j] = uint16_t(i);
    }
    huff_lengths(H.clf, m_cl, H.cl, 7, H.hs);
    canon(H.cl, 19, H.clc);
    int hclen = 19;
    while (hclen > 4 && H.cl[c_cl_order[hclen - 1]] == 0) --hclen;
    BitOut bo{hdr, 0};
    bo.put(uint32_t(hlit - 257), 5);
    bo.put(uint32_t(hdist - 1), 5);
    bo.put(uint32_t(hclen - 4), 4);
    for (int i = 0; i < hclen; ++i) bo.put(H.cl[c_cl_order[i]], 3);
    for (int i = 0; i < nr; ++i) {
      const uint32_t c = H.clc[H.rsym[i]];
      bo.put(c & 0xFFFFu, c >> 16);
      if (H.rext[i] != 0xFF) bo.put(H.rext[i], H.rsym[i] == 16 ? 2 : H.rsym[i] == 17 ? 3 : 7);
    }
    hbits = bo.pos;
    uint64_t dyn_bits = 3 + hbits + ext;
    for (int i = 0; i < 288; ++i) dyn_bits += uint64_t(H.ll[i]) * H.freq[i];
    for (int i = 0; i < 32; ++i) dyn_bits += uint64_t(H.dl[i]) * H.freq[288 + i];
    if (stored_bits <= fixed_bits && stored_bits <= dyn_bits) type = kBlkStored;
    else if (fixed_bits <= dyn_bits) type = kBlkFixed;
    else type = kBlkDynamic;
  }
  if (type == kBlkFixed) {
    for (int i = 0; i < 288; ++i) H.ll[i] = uint8_t(i < 144 ? 8 : i < 256 ? 9 : i < 280 ? 7 : 8);
    for (int i = 0; i < 32; ++i) H.dl[i] = 5;
  }
  if (type != kBlkStored) {
    canon(H.ll, 288, codes);
    canon(H.dl, 32, codes + 288);
    eob = codes[256];
  }
  gp->block_type = type;
  gp->hdr_bits = type == kBlkDynamic ? hbits : 0;
  gp->eob = eob;
}

// ---------------------------------------------------------------- k_enc
__device__ __forceinline__ void ring_put(uint32_t* ring, uint32_t bp, uint32_t v, uint32_t n) {
  if (!n) return;
  const uint32_t w = bp >> 5, sh = bp & 31;
  atomicOr(&ring[w & 127], v << sh);
  if (sh + n > 32) atomicOr(&ring[(w + 1) & 127], v >> (32 - sh));
}

constexpr int kEncWarps = 4;
__global__ void __launch_bounds__(kEncWarps * 32) k_enc(Work wk, const uint32_t* __restrict__ list, uint32_t nlist,
                                                        uint32_t* __restrict__ counter) {
  __shared__ uint32_t tab[kEncWarps][320];
  __shared__ uint32_t rings[kEncWarps][128];
  const uint32_t wid = threadIdx.x >> 5, lane = threadIdx.x & 31;
  uint32_t* code = tab[wid];
  uint32_t* ring = rings[wid];
  for (;;) {
    uint32_t i = 0;
    if (lane == 0) i = atomicAdd(counter, 1u);
    i = __shfl_sync(kAll, i, 0);
    if (i >= nlist) break;
    Tile* tp = wk.tiles + list[i];
    const Tile t = *tp;
    const Segment sg = wk.segs[t.seg];
    if (sg.block_type == kBlkStored) {
      if (lane == 0) { tp->spec_bits = 0; tp->spec_exit = t.start + t.len; }
      continue;
    }
    const uint32_t* gc = reinterpret_cast<const uint32_t*>(wk.scratch + sg.codes);
    for (uint32_t k = lane; k < 320; k += 32) code[k] = gc[k];
    for (uint32_t k = lane; k < 128; k += 32) ring[k] = 0;
    __syncwarp();
    const uint32_t* tok = reinterpret_cast<const uint32_t*>(wk.scratch + t.tok);
    uint32_t* out = reinterpret_cast<uint32_t*>(wk.scratch + t.scratch);
    const uint64_t o = sg.in_off;
    const SegBytes sb{reinterpret_cast<const uint32_t*>(wk.in + (o & ~uint64_t(3))), uint32_t(o & 3)};
    uint32_t np = 0, cursor = 0, flushed = 0;
    const uint32_t nwin = (t.len + 31) >> 5;
    for (uint32_t w = 0; w < nwin; ++w) {
      const uint32_t wpos = w << 5;
      const uint32_t lim = min(32u, t.len - wpos);
      if (np >= wpos + lim) continue;
      const uint32_t tk = lane < lim ? tok[wpos + lane] : 0u;
      const uint32_t M = __ballot_sync(kAll, tk != 0);
      const uint32_t limmask = lim == 32 ? kAll : ((1u << lim) - 1);
      uint32_t cur = np - wpos, vis = 0;
      while (cur < lim) {
        const uint32_t nm = M & limmask & (kAll << cur);
        if (!nm) { vis |= limmask & (kAll << cur); cur = lim; break; }
        const uint32_t j = __ffs(nm) - 1;
        vis |= (kAll << cur) & ((2u << j) - 1u);
        cur = j + ((__shfl_sync(kAll, tk, j) >> 16) & 0x1FFu);
      }
      uint32_t a = 0, na = 0, b = 0, nb = 0;  // two parts of one token
      if ((vis >> lane) & 1u) {
        if (tk) {
          const uint32_t len = (tk >> 16) & 0x1FFu, dist = tk & 0xFFFFu;
          uint32_t li, le, lv, dc, de, dv;
          length_code(len, li, le, lv);
          dist_code(dist, dc, de, dv);
          const uint32_t lc = code[257 + li], dcw = code[288 + dc];
          a = (lc & 0xFFFFu) | (lv << (lc >> 16));
          na = (lc >> 16) + le;
          b = (dcw & 0xFFFFu) | (dv << (dcw >> 16));
          nb = (dcw >> 16) + de;
        } else {
          const uint32_t c = code[sb.byte(t.start + wpos + lane)];
          a = c & 0xFFFFu;
          na = c >> 16;
        }
      }
      uint32_t incl = na + nb;
#pragma unroll
      for (int s = 1; s < 32; s <<= 1) {
        const uint32_t x = __shfl_up_sync(kAll, incl, s);
        if (lane >= uint32_t(s)) incl += x;
      }
      const uint32_t total = __shfl_sync(kAll, incl, 31);
      const uint32_t bp = cursor + incl - na - nb;
      ring_put(ring, bp, a, na);
      ring_put(ring, bp + na, b, nb);
      cursor += total;
      np = wpos + cur;
      __syncwarp();
      while ((cursor >> 5) >= flushed + 32) {
        out[flushed + lane] = ring[(flushed + lane) & 127];
        ring[(flushed + lane) & 127] = 0;
        flushed += 32;
        __syncwarp();
      }
    }
    const uint32_t nwords = (cursor + 31) >> 5;
    for (uint32_t k = flushed + lane; k < nwords; k += 32) out[k] = ring[k & 127];
    __syncwarp();
    if (lane == 0) {
      tp->spec_bits = cursor;
      tp->spec_exit = t.start + t.len;
    }
  }
}

int launch_lazy(const Work& wk, const LazyLists& L, cudaStream_t st, int sms, Marks* mk) {
  if (!L.n_tiles) return 0;
  static std::atomic<bool> attr_set[64];
  const int ds = device_slot();
  if (!attr_set[ds].load(std::memory_order_relaxed)) {
    if (cudaFuncSetAttribute(k_lz, cudaFuncAttributeMaxDynamicSharedMemorySize, int(kSmemLz)) == cudaSuccess)
      attr_set[ds].store(true, std::memory_order_relaxed);
  }
  k_lz<<<L.n_runs, 1024, kSmemLz, st>>>(wk, L.runs, L.n_runs);
  mk->mark(kPhLazyLz, st);
  k_huff<<<(L.n_segs + kHuffWarps - 1) / kHuffWarps, kHuffWarps * 32, 0, st>>>(wk, L.segs, L.n_segs);
  mk->mark(kPhLazyHuff, st);
  uint32_t blocks = uint32_t(sms) * 8;
  const uint32_t need = (L.n_tiles + kEncWarps - 1) / kEncWarps;
  if (blocks > need) blocks = need;
  k_enc<<<blocks, kEncWarps * 32, 0, st>>>(wk, L.tiles, L.n_tiles, L.counter);
  mk->mark(kPhLazyEnc, st);
  return 3;
}

}  // namespace orotb
