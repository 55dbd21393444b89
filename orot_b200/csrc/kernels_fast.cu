// kernels_fast.cu -- LZ77 for levels 1-3 (orot's "fast path") on sm_100a.
//
// Reference semantics (src/deflate/lz77.cpp:163-191, 378-406): greedy
// parsing, a single head[] table of 2^hash_bits absolute positions, every
// position p <= n-4 inserted in order, candidate = head[hash(p)] (0 = empty),
// dist = (p - cand) & 0x7FFF, first-byte check at cand, match length measured
// at p - dist, matches shorter than 3 rejected.  Because every position is
// inserted whether the parse visits it or not, the candidate of p is simply
// "the last earlier position with the same hash": it does not depend on the
// parse.  That is what makes the path parallel:
//
//   k_lastocc     per tile, last position of every hash (shared atomics)
//   k_carry_scan  per segment, exclusive prefix-max of those tables
//   k_cand        one warp per tile, head[] in shared memory (18 walkers of
//                 12.4 KB per SM at 12 hash bits): 32 positions per step;
//                 hash, head lookup, insert by store and read-back (a
//                 window with a repeated hash groups its lanes with
//                 __match_any); the candidate distance of every position (2 bytes)
//                 and the run period of every 32-position window.
//   k_parse       one warp per tile, no table (16 warps of 0.6 KB per CTA,
//                 two CTAs per SM): capped match lengths per lane, greedy
//                 parse resolved with ballots, fixed Huffman bits packed with
//                 shared atomics and flushed as coalesced 128-byte stores.
//                 The parse starts at the tile's first byte (speculation) and
//                 one record per 32 positions remembers where it entered that
//                 window; windows a match covers cost only that record.
//   k_cand_parse  (the default) both passes in one persistent kernel: 16
//                 walkers (4 at 14 hash bits) and the rest of 32 warps as
//                 parsers per SM; a parser takes a tile once a walker has
//                 published its candidates.
//   k_fix1/k_fix2 re-walk a tile from the true entry (where the previous
//                 tile's parse ended; k_fix1 all tiles at once assuming the
//                 previous speculation held, k_fix2 one warp per multi-tile
//                 segment, tiles in order, where it did not) until it
//                 meets the speculative parse at a window boundary; from
//                 there the speculative bits are exact.
//
// The output is therefore token-for-token the reference's.
#include <cuda_runtime.h>
#include <cstdint>
#include <cstdlib>
#include "engine.cuh"
#include "deflate_device.cuh"
#include "kernels.cuh"

namespace orotb {

constexpr uint32_t kFull = 0xFFFFFFFFu;

__device__ __forceinline__ uint32_t hash_fast(uint32_t v, int hb) { return (v * 0x9E3779B1u) >> (32 - hb); }

// ---------------------------------------------------------------- k_lastocc
// Each thread hashes 16 consecutive positions from 5 loaded words; a position
// followed by one with the same hash (runs) needs no atomic, since the later
// position wins the max anyway.
template <int HB>
__global__ void __launch_bounds__(256) k_lastocc(Work wk, const uint32_t* __restrict__ list, uint32_t nlist) {
  extern __shared__ uint32_t tbl[];
  constexpr int H = 1 << HB;
  if (blockIdx.x >= nlist) return;
  const Tile t = wk.tiles[list[blockIdx.x]];
  const Segment sg = wk.segs[t.seg];
  for (int i = threadIdx.x; i < H; i += blockDim.x) tbl[i] = 0;
  __syncthreads();
  const uint64_t a = sg.in_off;
  const uint32_t* w = reinterpret_cast<const uint32_t*>(wk.in + (a & ~uint64_t(3)));
  const uint32_t boff = uint32_t(a & 3);
  const uint32_t end = t.start + t.len;
  const uint32_t lim = sg.len >= 4 ? min(end, sg.len - 3) : t.start;  // positions with 4 bytes
  // 16 positions per thread from word-aligned loads: the byte offsets of the
  // funnel shifts are then constants.  Positions before the tile start or
  // without 4 bytes are masked.
  const uint32_t q0 = (t.start + boff) & ~3u;
  for (uint32_t qb = q0 + 16 * threadIdx.x; qb < lim + boff; qb += 16 * blockDim.x) {
    const uint32_t* qw = w + (qb >> 2);
    uint32_t W[5];
#pragma unroll
    for (int j = 0; j < 5; ++j) W[j] = __ldg(qw + j);
    uint32_t h[16];
#pragma unroll
    for (int i = 0; i < 16; ++i) h[i] = hash_fast(__funnelshift_r(W[i >> 2], W[(i >> 2) + 1], (i & 3) * 8), HB);
    const uint32_t p0 = qb - boff;  // position of byte 0 (may be below the tile start)
#pragma unroll
    for (int i = 0; i < 16; ++i) {
      const bool in = p0 + i >= t.start && p0 + i < lim;
      const bool next_in = i < 15 && p0 + i + 1 >= t.start && p0 + i + 1 < lim;
      if (in && !(next_in && h[i] == h[i + 1])) atomicMax(&tbl[h[i]], p0 + i);
    }
  }
  __syncthreads();
  uint32_t* slot = reinterpret_cast<uint32_t*>(wk.scratch + t.slot);
  for (int i = threadIdx.x; i < H; i += blockDim.x) slot[i] = tbl[i];
}

// ---------------------------------------------------------------- k_carry_scan
// Exclusive prefix-max over the tiles of a segment: afterwards the slot of
// tile k holds max(last positions of tiles 0..k), i.e. the head[] state at the
// start of tile k+1.
template <int HB>
__global__ void __launch_bounds__(256) k_carry_scan(Work wk, const uint32_t* __restrict__ seglist, uint32_t nseg) {
  constexpr int H = 1 << HB;
  const uint32_t h = blockIdx.x * blockDim.x + threadIdx.x;
  if (h >= uint32_t(H)) return;
  for (uint32_t si = blockIdx.y; si < nseg; si += gridDim.y) {
    const Segment sg = wk.segs[seglist[si]];
    uint32_t run = 0;
    // eight tiles at a time: their loads are issued before the dependent
    // running maximum and the stores (one memory latency per eight tiles)
    constexpr uint32_t B = 8;
    const uint32_t nt = sg.tile_count ? sg.tile_count - 1 : 0;
    for (uint32_t k0 = 0; k0 < nt; k0 += B) {
      uint32_t* slot[B];
      uint32_t v[B];
#pragma unroll
      for (uint32_t j = 0; j < B; ++j)
        slot[j] = k0 + j < nt ? reinterpret_cast<uint32_t*>(wk.scratch + wk.tiles[sg.tile_first + k0 + j].slot) : nullptr;
#pragma unroll
      for (uint32_t j = 0; j < B; ++j) v[j] = slot[j] ? slot[j][h] : 0u;
#pragma unroll
      for (uint32_t j = 0; j < B; ++j) {
        run = max(run, v[j]);
        if (slot[j]) slot[j][h] = run;
      }
    }
  }
}

// ---------------------------------------------------------------- the walker
// Per-warp shared state: head[] (walk only), the bit ring, and the staged
// bytes around the current window: 24 words starting 32 bytes before the
// window (so runs with a period up to 32 can be checked) and reaching 64
// bytes past its start (the p side of every capped match length).
constexpr uint32_t kRing = 128, kWbuf = 24;
constexpr uint32_t kCapMax = 48;  // capped match length of lane 0 (48 - lane)

struct WinState {
  uint32_t np, cursor, flushed, matches, tokens;
};

// Staging starts at segment position max(wpos - 32, 0), rounded down to a
// word.  Returns the byte offset of wpos inside wbuf.
__device__ __forceinline__ uint32_t stage_base_word(const SegBytes& sb, uint32_t wpos) {
  return (sb.boff + (wpos >= 32 ? wpos - 32 : 0)) >> 2;
}
__device__ __forceinline__ uint32_t prefetch_window(const SegBytes& sb, uint32_t wpos, uint32_t lane) {
  return lane < kWbuf ? __ldg(sb.w + stage_base_word(sb, wpos) + lane) : 0u;
}
__device__ __forceinline__ uint32_t stage_window(const SegBytes& sb, uint32_t wpos, uint32_t* wbuf, uint32_t lane,
                                                 uint32_t pre) {
  if (lane < kWbuf) wbuf[lane] = pre;
  __syncwarp();
  return sb.boff + wpos - 4 * stage_base_word(sb, wpos);
}
__device__ __forceinline__ uint32_t wload4(const uint32_t* wbuf, uint32_t off) {
  return __funnelshift_r(wbuf[off >> 2], wbuf[(off >> 2) + 1], (off & 3) * 8);
}

// Capped common-prefix length of the bytes at p (staged at wbuf offset po)
// and at q (global), at most cap <= kCapMax.  The first 4 q-side words are
// loaded in one batch (one memory latency covers matches up to ~12 bytes);
// longer matches fetch one more word per step.  The loop runs while any lane
// of the warp is still matching, so its trip count follows the longest match
// in the window rather than the cap.  Every lane of the warp must call it.
__device__ __forceinline__ uint32_t lcp_window(const SegBytes& sb, const uint32_t* wbuf, uint32_t po, uint32_t q,
                                               uint32_t cap, bool active) {
  constexpr int PRE = 4;
  const uint32_t qa = q + sb.boff;
  const uint32_t* qw = sb.w + (qa >> 2);
  const uint32_t qs = (qa & 3) * 8;
  const uint32_t* pw = wbuf + (po >> 2);  // p side: staged words, each loaded once
  const uint32_t ps = (po & 3) * 8;
  uint32_t v[PRE];
#pragma unroll
  for (int j = 0; j < PRE; ++j) v[j] = active && uint32_t(j) * 4 < cap + 4 ? __ldg(qw + j) : 0u;
  uint32_t n = 0;
  bool open = active && cap > 0;
  uint32_t plo = pw[0];
#pragma unroll
  for (int j = 0; j < PRE - 1; ++j) {
    if (!__any_sync(kFull, open)) break;
    // staged words (po >> 2) + j + 1 <= 23 < kWbuf: in bounds for every lane
    const uint32_t phi = pw[j + 1];
    const uint32_t x = __funnelshift_r(plo, phi, ps) ^ __funnelshift_r(v[j], v[j + 1], qs);
    plo = phi;
    n += open ? (x ? (__ffs(x) - 1) >> 3 : 4u) : 0u;
    open = open && !x && n < cap;
  }
  uint32_t lo = v[PRE - 1];
  for (uint32_t j = PRE - 1; __any_sync(kFull, open); ++j) {
    if (open) {
      const uint32_t hi = __ldg(qw + j + 1);
      const uint32_t phi = pw[j + 1];
      const uint32_t x = __funnelshift_r(plo, phi, ps) ^ __funnelshift_r(lo, hi, qs);
      plo = phi;
      lo = hi;
      if (x) { n += (__ffs(x) - 1) >> 3; open = false; } else { n += 4; }
      if (n >= cap) open = false;
    }
  }
  return n < cap ? n : cap;
}

// Fixed-Huffman code tables for the parse kernels: literal b at [b], match
// length L (3..258) at [256 + L]; each entry is the LSB-first bits | count << 16
// (a length entry holds the length symbol and its extra bits).  Distance
// codes at [kDistTab + (d - 1)] for d - 1 < 256, else at
// [kDistTab + 256 + ((d - 1) >> 7)] (the code of a larger distance depends only
// on its bits above the 7th): the 5-bit code reversed | extra-bit count << 8.
constexpr uint32_t kDistTab = 256 + 259;
constexpr uint32_t kCodeTab = kDistTab + 512;
__device__ __forceinline__ void fill_code_tab(uint32_t* tab) {
  for (uint32_t i = threadIdx.x; i < kCodeTab; i += blockDim.x) {
    uint32_t bits = 0, nb = 0;
    if (i >= kDistTab) {
      const uint32_t t = i - kDistTab, dm1 = t < 256 ? t : (t - 256) << 7;
      uint32_t dc, de, dv;
      dist_code(dm1 + 1, dc, de, dv);
      tab[i] = rev_bits(dc, 5) | (de << 8);
      continue;
    }
    if (i < 256) {
      fixed_literal(i, bits, nb);
    } else if (i >= 256 + 3) {
      uint32_t li, le, lv;
      length_code(i - 256, li, le, lv);
      const uint32_t sym = 257 + li;
      const uint32_t c = sym <= 279 ? sym - 256 : 0xC0u + (sym - 280), cl = sym <= 279 ? 7u : 8u;
      bits = rev_bits(c, cl) | (lv << cl);
      nb = cl + le;
    }
    tab[i] = bits | (nb << 16);
  }
}
__device__ __forceinline__ void tab_match(const uint32_t* tab, uint32_t len, uint32_t dist, uint32_t& bits,
                                          uint32_t& nb) {
  const uint32_t t = tab[256 + len];
  const uint32_t dm1 = dist - 1;
  const uint32_t e = tab[kDistTab + (dm1 < 256 ? dm1 : 256 + (dm1 >> 7))];
  const uint32_t ne = e >> 8;
  bits = (t & 0xFFFFu) | ((e & 31u) << (t >> 16));
  nb = (t >> 16) + 5;
  bits |= (dm1 & ((1u << ne) - 1u)) << nb;
  nb += ne;
}

// head[] entry: the candidate's position mod 32768 with a valid bit (u16)
// beside its first byte (u8).  That is all the reference's fast path uses of
// a candidate (distance = (p - cand) & 0x7FFF, first-byte check at cand), and
// keeping the byte saves a dependent load.  Position 0 stays invalid (head
// value 0 means empty in src/deflate/lz77.cpp:178).
struct HeadTab {
  uint16_t* pos;   // (pos & 0x7FFF) | 0x8000 when valid, 0 when empty
  uint8_t* byte;
  __device__ __forceinline__ void put(uint32_t h, uint32_t p, uint32_t b) const {
    pos[h] = p ? uint16_t((p & 0x7FFFu) | 0x8000u) : uint16_t(0);
    byte[h] = uint8_t(b);
  }
};
// Shared-memory words per warp of a walker: head table (2 + 1 bytes per
// entry), bit ring and staged window.
template <int HB>
__host__ __device__ constexpr uint32_t walker_words() { return ((1u << HB) * 3 + 3) / 4 + kRing + kWbuf; }

// Greedy parse and fixed-Huffman emission of one 32-position window.  Lane
// `lane` holds position wpos+lane; `d` is its candidate distance (0 = none).
__device__ __forceinline__ void parse_window(const SegBytes& sb, uint32_t n, uint32_t wpos, uint32_t lim,
                                             uint32_t lane, const uint32_t* wbuf, uint32_t woff, uint32_t d,
                                             uint32_t* ring, uint32_t* out, WinState& st,
                                             const uint32_t* ctab = nullptr) {
  const uint32_t p = wpos + lane;
  uint32_t clen = 0;
  bool exact = true;
  const bool want = d && p >= st.np && lane < lim;
  const uint32_t maxm = want ? min(258u, n - p) : 0u;
  const uint32_t cap = want ? min(maxm, max(3u, kCapMax - lane)) : 0u;
  if (__any_sync(kFull, want)) {
    clen = lcp_window(sb, wbuf, woff + lane, want ? p - d : p, cap, want);
    if (want) {
      exact = clen < cap || cap == maxm;
      if (clen < 3) clen = 0;
    } else {
      clen = 0;
    }
  }
  const uint32_t M = __ballot_sync(kFull, clen >= 3);
  const uint32_t limmask = lim == 32 ? kFull : ((1u << lim) - 1);
  uint32_t cur = st.np - wpos, visited = 0;
  int xl = -1;
  while (cur < lim) {
    const uint32_t nm = M & limmask & (kFull << cur);
    if (!nm) { visited |= limmask & (kFull << cur); cur = lim; break; }
    const uint32_t j = __ffs(nm) - 1;
    visited |= (kFull << cur) & ((2u << j) - 1u);
    const uint32_t lj = __shfl_sync(kFull, clen, j);
    const bool ej = __shfl_sync(kFull, exact, j);
    if (ej) { cur = j + lj; } else { xl = int(j); break; }
  }
  uint32_t full = 0;
  if (xl >= 0) {
    // warp-cooperative extension, 128 bytes per round
    const uint32_t pj = wpos + xl;
    const uint32_t dj = __shfl_sync(kFull, d, xl);
    const uint32_t c0 = __shfl_sync(kFull, clen, xl);
    const uint32_t maxm = min(258u, n - pj);
    full = c0;
    for (uint32_t base = c0; base < maxm; base += 128) {
      const uint32_t off = base + 4 * lane;
      uint32_t stop = kFull;
      if (off < maxm) {
        const uint32_t x = sb.load4(pj + off) ^ sb.load4(pj - dj + off);
        const uint32_t m = x ? ((__ffs(x) - 1) >> 3) : 4u;
        const uint32_t l4 = min(4u, maxm - off);
        if (m < l4) stop = off + m;
        else if (off + 4 >= maxm) stop = maxm;
      }
      const uint32_t b = __ballot_sync(kFull, stop != kFull);
      if (b) { full = __shfl_sync(kFull, stop, __ffs(b) - 1); break; }
    }
    cur = uint32_t(xl) + full;
  }
  const bool vis = (visited >> lane) & 1u;
  const bool ism = vis && ((M >> lane) & 1u);
  uint32_t code = 0, nb = 0;
  if (ctab) {
    if (visited & M) {  // a match in the window: both codes, selected per lane
      uint32_t mc, mn;
      tab_match(ctab, ism ? (int(lane) == xl ? full : clen) : 3u, ism ? d : 1u, mc, mn);
      const uint32_t t = ctab[wload4(wbuf, woff + lane) & 0xFFu];
      code = !vis ? 0u : ism ? mc : (t & 0xFFFFu);
      nb = !vis ? 0u : ism ? mn : (t >> 16);
    } else if (vis) {
      const uint32_t t = ctab[wload4(wbuf, woff + lane) & 0xFFu];
      code = t & 0xFFFFu;
      nb = t >> 16;
    }
  } else if (vis) {
    if (ism) {
      fixed_match(int(lane) == xl ? full : clen, d, code, nb);
    } else {
      fixed_literal(wload4(wbuf, woff + lane) & 0xFFu, code, nb);
    }
  }
  uint32_t incl = nb;
#pragma unroll
  for (int o = 1; o < 32; o <<= 1) {
    const uint32_t t = __shfl_up_sync(kFull, incl, o);
    if (lane >= uint32_t(o)) incl += t;
  }
  const uint32_t total = __shfl_sync(kFull, incl, 31);
  if (nb) {
    const uint32_t bp = st.cursor + incl - nb, wd = bp >> 5, sh = bp & 31;
    atomicOr(&ring[wd & (kRing - 1)], code << sh);
    if (sh + nb > 32) atomicOr(&ring[(wd + 1) & (kRing - 1)], code >> (32 - sh));
  }
  st.cursor += total;
  st.tokens += __popc(visited);
  st.matches += __popc(visited & M);
  st.np = wpos + cur;
  __syncwarp();
  while ((st.cursor >> 5) >= st.flushed + 32) {
    out[st.flushed + lane] = ring[(st.flushed + lane) & (kRing - 1)];
    ring[(st.flushed + lane) & (kRing - 1)] = 0;
    st.flushed += 32;
    __syncwarp();
  }
}

__device__ __forceinline__ void flush_tail(uint32_t* ring, uint32_t* out, const WinState& st, uint32_t lane) {
  const uint32_t nwords = (st.cursor + 31) >> 5;
  for (uint32_t i = st.flushed + lane; i < nwords; i += 32) out[i] = ring[i & (kRing - 1)];
  __syncwarp();
}

struct TileView {
  SegBytes sb;
  uint32_t n, ts, tl;
};

__device__ __forceinline__ TileView tile_view(const Work& wk, const Tile& t, const Segment& sg) {
  const uint64_t o = sg.in_off;
  return TileView{SegBytes{reinterpret_cast<const uint32_t*>(wk.in + (o & ~uint64_t(3))), uint32_t(o & 3)}, sg.len,
                  t.start, t.len};
}

// Speculative walk of one tile (parse entry = tile start): inserts every
// position into head[], records the candidate distance of every position and
// the parse entry (and run period) of every window, emits the fixed-Huffman
// bits.  `carry` holds full segment positions (0 = empty).
template <int HB>
__device__ WinState walk_tile(const TileView& tv, const uint32_t* carry, uint32_t* smem_warp, uint32_t* ring,
                              uint32_t* wbuf, uint32_t* out, WinRec* rec, uint16_t* cand16) {
  constexpr int H = 1 << HB;
  const uint32_t lane = threadIdx.x & 31;
  const uint32_t lt = (1u << lane) - 1;
  const HeadTab head{reinterpret_cast<uint16_t*>(smem_warp), reinterpret_cast<uint8_t*>(smem_warp) + 2 * H};
  if (carry) {
#pragma unroll 8
    for (int i = lane; i < H; i += 32) {
      const uint32_t pos = __ldg(carry + i);
      head.put(i, pos, pos ? tv.sb.byte(pos) : 0u);
    }
  } else {
    for (int i = lane; i < H; i += 32) head.put(i, 0, 0);
  }
  for (uint32_t i = lane; i < kRing; i += 32) ring[i] = 0;
  __syncwarp();
  WinState st{tv.ts, 0, 0, 0, 0};
  const uint32_t tend = tv.ts + tv.tl;
  const uint32_t nwin = (tv.tl + 31) >> 5;
  uint32_t pre = prefetch_window(tv.sb, tv.ts, lane);
  for (uint32_t w = 0; w < nwin; ++w) {
    const uint32_t wpos = tv.ts + (w << 5);
    const uint32_t woff = stage_window(tv.sb, wpos, wbuf, lane, pre);
    if (w + 1 < nwin) pre = prefetch_window(tv.sb, wpos + 32, lane);
    const WinRec rc{st.np - tv.ts, st.cursor, st.matches, 0};
    const uint32_t p = wpos + lane;
    const bool ins = p < tend && p + 4 <= tv.n;
    const uint32_t v4 = wload4(wbuf, woff + lane);
    const uint32_t h = ins ? hash_fast(v4, HB) : kFull;
    const uint32_t peers = __match_any_sync(kFull, h);
    const uint32_t before = peers & lt;
    const uint32_t src = before ? 31 - __clz(before) : lane;
    const uint32_t vb = __shfl_sync(kFull, v4, src);
    uint32_t cpos = 0, cbyte = 0;  // candidate: position mod 32768 | valid bit, first byte
    if (ins) {
      if (before) {
        const uint32_t c = wpos + src;
        cpos = c ? ((c & 0x7FFFu) | 0x8000u) : 0u;
        cbyte = vb & 0xFFu;
      } else {
        cpos = head.pos[h];
        cbyte = head.byte[h];
      }
    }
    __syncwarp();
    if (ins && (peers >> lane) == 1u) head.put(h, p, v4 & 0xFFu);
    // candidate distance after the first-byte check at the candidate itself
    uint32_t d = 0;
    if (cpos & 0x8000u) {
      const uint32_t dist = (p - (cpos & 0x7FFFu)) & 0x7FFFu;
      if (dist != 0 && cbyte == (v4 & 0xFFu)) d = dist;
    }
    if (cand16 && p < tend) cand16[p - tv.ts] = uint16_t(d);
    if (rec) {
      // run window: every position has the same short distance D and its
      // four bytes equal the four bytes D earlier
      const uint32_t D = __shfl_sync(kFull, d, 0);
      const bool ok = wpos >= 32 && D != 0 && D <= 32 && d == D && p + 4 <= tend &&
                      wload4(wbuf, woff + lane - D) == v4;
      const uint32_t all = __ballot_sync(kFull, ok);
      if (lane == 0) rec[w] = WinRec{rc.entry, rc.bit, rc.matches, all == kFull ? D : 0u};
    }
    __syncwarp();
    const uint32_t lim = min(32u, tend - wpos);
    if (st.np < wpos + lim) parse_window(tv.sb, tv.n, wpos, lim, lane, wbuf, woff, d, ring, out, st);
  }
  flush_tail(ring, out, st, lane);
  return st;
}

// Re-parse of one tile from `entry` using the recorded candidate distances,
// until the parse meets the speculative one at a window boundary.  Inside
// runs of short period (see WinRec::run) every match is (258, D), so the
// re-parse steps through them arithmetically.
struct FixOut {
  uint32_t bits, matches, exit, merged, merge_win;
};
__device__ FixOut fix_tile(const TileView& tv, uint32_t entry, const WinRec* rec, const uint16_t* cand16,
                           uint32_t* ring, uint32_t* wbuf, uint32_t* out) {
  const uint32_t lane = threadIdx.x & 31;
  for (uint32_t i = lane; i < kRing; i += 32) ring[i] = 0;
  __syncwarp();
  WinState st{entry, 0, 0, 0, 0};
  FixOut r{};
  const uint32_t tend = tv.ts + tv.tl;
  const uint32_t nwin = (tv.tl + 31) >> 5;
  for (uint32_t w = (entry - tv.ts) >> 5; w < nwin; ++w) {
    const uint32_t wpos = tv.ts + (w << 5);
    const WinRec rc = rec[w];
    if (st.np == tv.ts + rc.entry) { r.merged = 1; r.merge_win = w; break; }
    const uint32_t lim = min(32u, tend - wpos);
    if (st.np >= wpos + lim) continue;
    if (rc.run) {
      // the run's period and the first window after it (recorded by k_cand)
      const uint32_t D = rc.run & 0xFFu;
      const uint32_t wend = rc.run >> 8;
      const uint32_t rend = tv.ts + (wend << 5);  // bytes before rend all repeat at distance D
      if (st.np + 258 <= rend) {
        const uint32_t k = (rend - st.np) / 258;
        uint32_t code, nb;
        fixed_match(258, D, code, nb);
        for (uint32_t t0 = 0; t0 < k; t0 += 32) {
          const uint32_t cnt = min(32u, k - t0);
          if (lane < cnt) {
            const uint32_t bp = st.cursor + lane * nb, wd = bp >> 5, sh = bp & 31;
            atomicOr(&ring[wd & (kRing - 1)], code << sh);
            if (sh + nb > 32) atomicOr(&ring[(wd + 1) & (kRing - 1)], code >> (32 - sh));
          }
          st.cursor += cnt * nb;
          __syncwarp();
          while ((st.cursor >> 5) >= st.flushed + 32) {
            out[st.flushed + lane] = ring[(st.flushed + lane) & (kRing - 1)];
            ring[(st.flushed + lane) & (kRing - 1)] = 0;
            st.flushed += 32;
            __syncwarp();
          }
        }
        st.np += 258 * k;
        st.matches += k;
        st.tokens += k;
        w = ((st.np - tv.ts) >> 5) - 1;  // continue at the window holding np
        continue;
      }
    }
    const uint32_t pre = prefetch_window(tv.sb, wpos, lane);
    const uint32_t woff = stage_window(tv.sb, wpos, wbuf, lane, pre);
    const uint32_t d = lane < lim ? cand16[(w << 5) + lane] : 0u;
    parse_window(tv.sb, tv.n, wpos, lim, lane, wbuf, woff, d, ring, out, st);
  }
  flush_tail(ring, out, st, lane);
  r.bits = st.cursor;
  r.matches = st.matches;
  r.exit = st.np;
  return r;
}

// ---------------------------------------------------------------- k_cand
// Candidate pass of one tile: inserts every position into head[] in order
// (the table is carried in from earlier tiles) and records, per position, the
// candidate distance that passed the first-byte check (0 = literal) and, per
// window, its run period (WinRec::run: D when all 32 positions have distance
// D <= 32 and equal the bytes D earlier, with the first window after the run
// in bits 8 and up; 0 for other windows).  Only this pass needs the head
// table, so only it is limited to the walkers whose tables fit in shared
// memory; the parse runs as a separate kernel with far more warps per SM.
template <int HB>
__device__ void cand_tile(const TileView& tv, const uint32_t* carry, uint32_t* smem_warp, uint32_t* wbuf, WinRec* rec,
                          uint16_t* cand16) {
  constexpr int H = 1 << HB;
  const uint32_t lane = threadIdx.x & 31;
  const uint32_t lt = (1u << lane) - 1;
  const HeadTab head{reinterpret_cast<uint16_t*>(smem_warp), reinterpret_cast<uint8_t*>(smem_warp) + 2 * H};
  if (carry) {
#pragma unroll 8
    for (int i = lane; i < H; i += 32) {
      const uint32_t pos = __ldg(carry + i);
      head.put(i, pos, pos ? tv.sb.byte(pos) : 0u);
    }
  } else {
    for (int i = lane; i < H; i += 32) head.put(i, 0, 0);
  }
  __syncwarp();
  const uint32_t tend = tv.ts + tv.tl;
  const uint32_t nwin = (tv.tl + 31) >> 5;
  uint32_t seg_D = 0, seg_start = 0;  // the run being recorded: its period and first window
  uint32_t pre = prefetch_window(tv.sb, tv.ts, lane);
  uint32_t prevD = 0;  // run period of the previous window (0 = not a run)
  for (uint32_t w = 0; w < nwin; ++w) {
    const uint32_t wpos = tv.ts + (w << 5);
    const uint32_t woff = stage_window(tv.sb, wpos, wbuf, lane, pre);
    if (w + 1 < nwin) pre = prefetch_window(tv.sb, wpos + 32, lane);
    const uint32_t p = wpos + lane;
    const bool ins = p < tend && p + 4 <= tv.n;
    const uint32_t v4 = wload4(wbuf, woff + lane);
    const uint32_t h = ins ? hash_fast(v4, HB) : 0u;
    const uint32_t mine = p ? ((p & 0x7FFFu) | 0x8000u) : 0u;  // this position as a table entry
    uint32_t d = 0, runD = 0;  // candidate distance (0 = none), run period of this window
    uint32_t cpos = 0, cbyte = 0;  // the table's candidate: position mod 32768 | valid bit, first byte
    bool done = false, have_c = false;
    // A window that continues the previous window's run of period D (every
    // position's 4 bytes equal those D earlier) has hashes repeating with
    // period D.  When the last D lanes' hashes are distinct, every position's
    // latest same-hash position is the one D earlier and the last D lanes
    // hold the table's new entries, so the window is done without the
    // same-hash search.  Period 1 needs no check.
    if (prevD && __all_sync(kFull, p + 4 <= tend && wload4(wbuf, woff + lane - prevD) == v4)) {
      const bool top = lane >= 32 - prevD;
      if (prevD == 1) {
        done = true;
      } else {
        cpos = head.pos[h];
        cbyte = head.byte[h];
        have_c = true;
        __syncwarp();
        if (top) head.pos[h] = uint16_t(mine);
        __syncwarp();
        done = !__any_sync(kFull, top && head.pos[h] != mine);
      }
      if (done) {
        if (prevD == 1 && top) head.pos[h] = uint16_t(mine);
        if (top) head.byte[h] = uint8_t(v4);
        d = prevD;
        runD = prevD;
      }
    }
    if (!done) {
      // the table's candidate (the latest position of the hash in earlier
      // windows), read before any entry of this window is stored
      if (!have_c) {
        cpos = ins ? head.pos[h] : 0u;
        cbyte = ins ? head.byte[h] : 0u;
        __syncwarp();
      }
      // Every lane stores its position and reads the entry back.  Positions
      // differ, so all read back their own exactly when no two lanes of the
      // window share a hash; only then may the table's candidate stand for
      // every lane and every lane's entry stay.  Otherwise (repeats within
      // 32 bytes) the lanes of each hash are found with __match_any_sync,
      // whose cost grows with the number of distinct hashes in the warp: the
      // nearest earlier lane is the candidate and the last lane's entry
      // stays.  After a run window (repeats all but certain) the probe is
      // skipped.
      bool clash = true, last = ins;
      if (!prevD && !have_c) {
        if (ins) head.pos[h] = uint16_t(mine);
        __syncwarp();
        clash = __any_sync(kFull, ins && head.pos[h] != mine);
      }
      if (clash) {
        const uint32_t peers = __match_any_sync(kFull, ins ? h : kFull);
        const uint32_t before = peers & lt;
        const uint32_t src = before ? 31 - __clz(before) : lane;
        const uint32_t vb = __shfl_sync(kFull, v4, src);
        if (ins && before) {
          const uint32_t c = wpos + src;
          cpos = c ? ((c & 0x7FFFu) | 0x8000u) : 0u;
          cbyte = vb & 0xFFu;
        }
        last = ins && (peers >> lane) == 1u;
        __syncwarp();
        if (last) head.pos[h] = uint16_t(mine);
      }
      if (last) head.byte[h] = uint8_t(v4);
      // candidate distance after the first-byte check at the candidate itself
      if (cpos & 0x8000u) {
        const uint32_t dist = (p - (cpos & 0x7FFFu)) & 0x7FFFu;
        if (dist != 0 && cbyte == (v4 & 0xFFu)) d = dist;
      }
      // run window: every position has the same distance D <= 32 and its
      // four bytes equal the four bytes D earlier (checked only when every
      // lane has a distance of at most 32)
      if (wpos >= 32 && __all_sync(kFull, d != 0 && d <= 32 && p + 4 <= tend)) {
        const uint32_t D = __shfl_sync(kFull, d, 0);
        runD = __all_sync(kFull, d == D && wload4(wbuf, woff + lane - D) == v4) ? D : 0u;
      }
    }
    if (p < tend) cand16[p - tv.ts] = uint16_t(d);
    // consecutive run windows of one period form a run; when it ends, each of
    // its windows records the period and the window after the run, so the
    // fix-up crosses a run without scanning it
    if (runD != seg_D) {
      if (seg_D)
        for (uint32_t k = seg_start + lane; k < w; k += 32) rec[k].run = seg_D | (w << 8);
      seg_D = runD;
      seg_start = w;
    }
    prevD = runD;
    if (!runD && lane == 0) rec[w].run = 0;
  }
  if (seg_D)
    for (uint32_t k = seg_start + lane; k < nwin; k += 32) rec[k].run = seg_D | (nwin << 8);
}

template <int HB, int WARPS>
__global__ void __launch_bounds__(WARPS * 32) k_cand(Work wk, const uint32_t* __restrict__ list, uint32_t nlist,
                                                      uint32_t* __restrict__ counter) {
  extern __shared__ uint32_t sm[];
  constexpr uint32_t HW = ((1u << HB) * 3 + 3) / 4;
  const uint32_t wid = threadIdx.x >> 5, lane = threadIdx.x & 31;
  uint32_t* head = sm + wid * (HW + kWbuf);
  uint32_t* wbuf = head + HW;
  for (;;) {
    uint32_t i = 0;
    if (lane == 0) i = atomicAdd(counter, 1u);
    i = __shfl_sync(kFull, i, 0);
    if (i >= nlist) break;
    const Tile t = wk.tiles[list[i]];
    const Segment sg = wk.segs[t.seg];
    const TileView tv = tile_view(wk, t, sg);
    const uint32_t* carry = t.index ? reinterpret_cast<const uint32_t*>(wk.scratch + t.carry) : nullptr;
    cand_tile<HB>(tv, carry, head, wbuf, reinterpret_cast<WinRec*>(wk.scratch + t.rec),
                  reinterpret_cast<uint16_t*>(wk.scratch + t.cand));
  }
}

// ---------------------------------------------------------------- k_parse
// Speculative parse of one tile (parse entry = tile start) from the recorded
// candidates: greedy parse, fixed-Huffman bits, and per window the parse
// entry, bit offset and match count for the fix-up.  Windows that a match
// covers entirely cost only that record.  Shared memory per warp is the bit
// ring and the staged bytes, so many warps share an SM.  The candidates are
// read at L2 (ld.global.cg): in the fused kernel they were written by other
// SMs during the same launch.
__device__ void parse_tile(const Work& wk, Tile* tp, uint32_t* ring, uint32_t* wbuf, const uint32_t* ctab) {
  const uint32_t lane = threadIdx.x & 31;
  const Tile t = *tp;
  const Segment sg = wk.segs[t.seg];
  const TileView tv = tile_view(wk, t, sg);
  WinRec* rec = reinterpret_cast<WinRec*>(wk.scratch + t.rec);
  const uint16_t* c16 = reinterpret_cast<const uint16_t*>(wk.scratch + t.cand);
  uint32_t* out = reinterpret_cast<uint32_t*>(wk.scratch + t.scratch);
  for (uint32_t k = lane; k < kRing; k += 32) ring[k] = 0;
  __syncwarp();
  WinState st{tv.ts, 0, 0, 0, 0};
  const uint32_t tend = tv.ts + tv.tl;
  const uint32_t nwin = (tv.tl + 31) >> 5;
  // the next window's bytes and candidates are loaded one window ahead
  uint32_t pre = prefetch_window(tv.sb, tv.ts, lane);
  uint32_t dnext = lane < tv.tl ? __ldcg(c16 + lane) : 0u;
  uint32_t pre_w = 0;
  for (uint32_t w = 0; w < nwin; ++w) {
    const uint32_t wpos = tv.ts + (w << 5);
    const uint32_t lim = min(32u, tend - wpos);
    // parse state where the parse enters this window (lanes 0-2 write one field each)
    const uint32_t f = lane == 0 ? st.np - tv.ts : lane == 1 ? st.cursor : st.matches;
    if (lane < 3) reinterpret_cast<uint32_t*>(rec + w)[lane] = f;
    if (st.np >= wpos + lim) continue;  // covered by a match
    uint32_t woff, d;
    if (pre_w == w) {
      woff = stage_window(tv.sb, wpos, wbuf, lane, pre);
      d = dnext;
    } else {
      woff = stage_window(tv.sb, wpos, wbuf, lane, prefetch_window(tv.sb, wpos, lane));
      d = lane < lim ? __ldcg(c16 + (w << 5) + lane) : 0u;
    }
    if (w + 1 < nwin) {
      pre = prefetch_window(tv.sb, wpos + 32, lane);
      const uint32_t q = ((w + 1) << 5) + lane;
      dnext = q < tv.tl ? __ldcg(c16 + q) : 0u;
      pre_w = w + 1;
    }
    parse_window(tv.sb, tv.n, wpos, lim, lane, wbuf, woff, d, ring, out, st, ctab);
  }
  flush_tail(ring, out, st, lane);
  if (lane == 0) {
    tp->spec_bits = st.cursor;
    tp->spec_matches = st.matches;
    tp->spec_exit = st.np;
    tp->spec_tokens = st.tokens;
    tp->fix_bits = 0;
    tp->splice_bit = 0;
    tp->fin_matches = st.matches;
    tp->fin_exit = st.np;
    tp->fix_entry = t.start;
  }
}

template <int WARPS>
__global__ void __launch_bounds__(WARPS * 32, 2) k_parse(Work wk, const uint32_t* __restrict__ list, uint32_t nlist,
                                                          uint32_t* __restrict__ counter) {
  __shared__ uint32_t sm[WARPS][kRing + kWbuf];
  __shared__ uint32_t ctab[kCodeTab];
  const uint32_t wid = threadIdx.x >> 5, lane = threadIdx.x & 31;
  uint32_t* ring = sm[wid];
  uint32_t* wbuf = ring + kRing;
  fill_code_tab(ctab);
  __syncthreads();
  for (;;) {
    uint32_t i = 0;
    if (lane == 0) i = atomicAdd(counter, 1u);
    i = __shfl_sync(kFull, i, 0);
    if (i >= nlist) break;
    parse_tile(wk, wk.tiles + list[i], ring, wbuf, ctab);
  }
}

// ---------------------------------------------------------------- k_cand_parse
// The candidate pass and the parse in one persistent kernel, one CTA of 32
// warps per SM: the first CW warps are candidate walkers (head tables in
// shared memory), the others parse, and a walker whose candidate work is
// exhausted parses too.  Walkers take tiles in list order and publish each
// finished tile in `ready`; parsers take tiles in the same order and wait for
// its flag.  The two kinds of warp have complementary limits (walkers:
// shared-memory and warp-collective latency; parsers: instruction issue), so
// an SM running both issues more than it does running either alone.  A walker
// never waits, so every flag a parser waits for is set by a running warp; the
// wait is bounded all the same (kReadyWaitNs; the first parser that gives up
// makes every later wait of the launch give up at once), and a parser that
// gives up marks the tile's segment failed and leaves the tile as empty.
__device__ __forceinline__ uint32_t ld_acquire_gpu(const uint32_t* p) {
  uint32_t v;
  asm volatile("ld.acquire.gpu.global.u32 %0, [%1];" : "=r"(v) : "l"(p) : "memory");
  return v;
}
__device__ __forceinline__ void st_release_gpu(uint32_t* p, uint32_t v) {
  asm volatile("st.release.gpu.global.u32 [%0], %1;" ::"l"(p), "r"(v) : "memory");
}
__device__ __forceinline__ uint64_t fast_global_ns() {
  uint64_t t;
  asm volatile("mov.u64 %0, %%globaltimer;" : "=l"(t));
  return t;
}
constexpr uint64_t kReadyWaitNs = 1000000000ull;
// Waits for `flag`; false after kReadyWaitNs, or at once when another
// parser of the launch has already given up (`abort`, which it then sets).
__device__ __noinline__ bool wait_ready(const uint32_t* flag, uint32_t* abort) {
  if (ld_acquire_gpu(flag)) return true;
  const uint64_t t0 = fast_global_ns();
  uint32_t nap = 64;
  for (;;) {
    __nanosleep(nap);
    if (nap < 2048) nap <<= 1;
    if (ld_acquire_gpu(flag)) return true;
    if (*reinterpret_cast<volatile uint32_t*>(abort) || fast_global_ns() - t0 > kReadyWaitNs) {
      atomicExch(abort, 1u);
      return false;
    }
  }
}
template <int HB>
__host__ __device__ constexpr uint32_t cand_parse_words(int cw) {
  return kCodeTab + uint32_t(cw) * (((1u << HB) * 3 + 3) / 4 + kWbuf) + uint32_t(32 - cw) * (kRing + kWbuf);
}
template <int HB, int CW>
__global__ void __launch_bounds__(1024, 1) k_cand_parse(Work wk, const uint32_t* __restrict__ list, uint32_t nlist,
                                                         uint32_t* __restrict__ counter, uint32_t* __restrict__ ready) {
  extern __shared__ uint32_t sm[];
  constexpr uint32_t HW = ((1u << HB) * 3 + 3) / 4;
  const uint32_t wid = threadIdx.x >> 5, lane = threadIdx.x & 31;
  uint32_t* ctab = sm;
  uint32_t* own = wid < CW ? sm + kCodeTab + wid * (HW + kWbuf)
                           : sm + kCodeTab + CW * (HW + kWbuf) + (wid - CW) * (kRing + kWbuf);
  fill_code_tab(ctab);
  __syncthreads();
  if (wid < CW) {
    for (;;) {
      uint32_t i = 0;
      if (lane == 0) i = atomicAdd(counter, 1u);
      i = __shfl_sync(kFull, i, 0);
      if (i >= nlist) break;
      const Tile t = wk.tiles[list[i]];
      const Segment sg = wk.segs[t.seg];
      const TileView tv = tile_view(wk, t, sg);
      const uint32_t* carry = t.index ? reinterpret_cast<const uint32_t*>(wk.scratch + t.carry) : nullptr;
      cand_tile<HB>(tv, carry, own, own + HW, reinterpret_cast<WinRec*>(wk.scratch + t.rec),
                    reinterpret_cast<uint16_t*>(wk.scratch + t.cand));
      __threadfence();  // this lane's candidates and records, before the flag
      __syncwarp();
      if (lane == 0) st_release_gpu(ready + i, 1u);
    }
  }
  uint32_t* ring = own;  // a walker's head-table space holds a parser's ring and staged bytes
  uint32_t* wbuf = own + kRing;
  for (;;) {
    uint32_t i = 0;
    if (lane == 0) i = atomicAdd(counter + 6, 1u);
    i = __shfl_sync(kFull, i, 0);
    if (i >= nlist) break;
    Tile* tp = wk.tiles + list[i];
    uint32_t ok = 1;
    if (lane == 0) ok = wait_ready(ready + i, counter + 12) ? 1u : 0u;
    ok = __shfl_sync(kFull, ok, 0);
    __syncwarp();
    if (!ok) {
      if (lane == 0) {
        atomicOr(&wk.segs[tp->seg].flags, kSegFault);
        tp->spec_bits = 0;
        tp->spec_matches = 0;
        tp->spec_exit = tp->start + tp->len;
        tp->spec_tokens = 0;
        tp->fix_bits = 0;
        tp->splice_bit = 0;
        tp->fin_matches = 0;
        tp->fin_exit = tp->start + tp->len;
        tp->fix_entry = tp->start;
      }
      __syncwarp();
      continue;
    }
    parse_tile(wk, tp, ring, wbuf, ctab);
  }
}

// ---------------------------------------------------------------- fix-up
// Applies the re-parse of tile t from `entry` and returns its true exit.
__device__ uint32_t fix_apply(const Work& wk, Tile* tp, uint32_t entry, uint32_t* ring, uint32_t* wbuf) {
  const Tile t = *tp;
  const Segment sg = wk.segs[t.seg];
  const uint32_t lane = threadIdx.x & 31;
  uint32_t fix_bits = 0, splice = 0, fin_m = t.spec_matches, fin_x = t.spec_exit;
  if (entry >= t.start + t.len) {  // a match of the previous tile covers this one
    splice = t.spec_bits;
    fin_m = 0;
    fin_x = entry;
  } else if (entry != t.start) {
    const TileView tv = tile_view(wk, t, sg);
    const WinRec* rec = reinterpret_cast<const WinRec*>(wk.scratch + t.rec);
    const uint16_t* c16 = reinterpret_cast<const uint16_t*>(wk.scratch + t.cand);
    uint32_t* out = reinterpret_cast<uint32_t*>(wk.scratch + t.scratch + tile_stream_bytes(t.len));
    const FixOut r = fix_tile(tv, entry, rec, c16, ring, wbuf, out);
    fix_bits = r.bits;
    if (r.merged) {
      const WinRec rc = rec[r.merge_win];
      splice = rc.bit;
      fin_m = r.matches + (t.spec_matches - rc.matches);
      fin_x = t.spec_exit;
    } else {
      splice = t.spec_bits;
      fin_m = r.matches;
      fin_x = r.exit;
    }
  }
  if (lane == 0) {
    tp->fix_bits = fix_bits;
    tp->splice_bit = splice;
    tp->fin_matches = fin_m;
    tp->fin_exit = fin_x;
    tp->fix_entry = entry;
  }
  __syncwarp();
  return fin_x;
}

// Round 1: every tile after the first, in parallel, assuming the previous
// tile's speculative parse was the true one.
template <int WARPS>
__global__ void __launch_bounds__(WARPS * 32) k_fix1(Work wk, const uint32_t* __restrict__ list, uint32_t nlist,
                                                      uint32_t* __restrict__ counter) {
  __shared__ uint32_t sm[WARPS][kRing + kWbuf];
  const uint32_t wid = threadIdx.x >> 5, lane = threadIdx.x & 31;
  for (;;) {
    uint32_t i = 0;
    if (lane == 0) i = atomicAdd(counter, 1u);
    i = __shfl_sync(kFull, i, 0);
    if (i >= nlist) break;
    Tile* tp = wk.tiles + list[i];
    if (tp->index == 0) continue;
    fix_apply(wk, tp, tp[-1].spec_exit, sm[wid], sm[wid] + kRing);
  }
}

// Round 2: per segment, in order; a tile is redone only when its
// predecessor's true exit differs from the entry round 1 assumed.
template <int WARPS>
__global__ void __launch_bounds__(WARPS * 32) k_fix2(Work wk, const uint32_t* __restrict__ seglist, uint32_t nseg) {
  __shared__ uint32_t sm[WARPS][kRing + kWbuf];
  const uint32_t wid = threadIdx.x >> 5;
  const uint32_t si = blockIdx.x * WARPS + wid;
  if (si >= nseg) return;
  const Segment sg = wk.segs[seglist[si]];
  const uint32_t lane = threadIdx.x & 31;
  uint32_t exit = wk.tiles[sg.tile_first].fin_exit;
  // The entries and exits of 32 tiles are loaded at once (one memory latency
  // instead of one per tile) and followed through shuffles; fix_apply changes
  // only its own tile, so the loaded values of the later tiles stay valid.
  for (uint32_t k0 = 1; k0 < sg.tile_count; k0 += 32) {
    const uint32_t cnt = min(32u, sg.tile_count - k0);
    uint32_t ent = 0, ext = 0;
    if (lane < cnt) {
      const Tile* t = wk.tiles + sg.tile_first + k0 + lane;
      ent = t->fix_entry;
      ext = t->fin_exit;
    }
    for (uint32_t j = 0; j < cnt; ++j) {
      const uint32_t ej = __shfl_sync(kFull, ent, j);
      const uint32_t xj = __shfl_sync(kFull, ext, j);
      if (ej == exit) { exit = xj; continue; }
      exit = fix_apply(wk, wk.tiles + sg.tile_first + k0 + j, exit, sm[wid], sm[wid] + kRing);
    }
  }
}

// ---------------------------------------------------------------- launchers
// The fused candidate + parse kernel is the default; OROT_B200_FUSED=0 runs
// the two passes as separate kernels (same bytes).
static bool fused_cand_parse() {
  static const bool on = [] {
    const char* e = getenv("OROT_B200_FUSED");
    return !(e && e[0] == '0');
  }();
  return on;
}
template <int HB>
static void launch_fast_t(const Work& wk, const FastLists& L, cudaStream_t st, int sms, Marks* mk) {
  constexpr int H = 1 << HB;
  // Walkers per CTA: shared memory bounds them (12.9 KB each at 12 hash
  // bits), and one CTA of 17 (219 KB) holds one more per SM than four CTAs
  // of four, since every CTA also reserves 1 KB; 5% faster.  At 14 hash bits
  // (49.7 KB each) four fit either way.
  constexpr int WARPS = HB <= 12 ? 18 : 4;
  const size_t tbl_bytes = size_t(H) * 4;
  constexpr uint32_t HW = ((1u << HB) * 3 + 3) / 4;
  const size_t csm = size_t(WARPS) * (HW + kWbuf) * 4;  // head table + staged bytes per walker
  // walker CTAs per SM, and the kernels' shared-memory limits, once per device
  static std::atomic<int> walk_per_sm[64];
  const int ds = device_slot();
  int per_sm = walk_per_sm[ds].load(std::memory_order_relaxed);
  if (!per_sm) {
    cudaFuncSetAttribute(k_lastocc<HB>, cudaFuncAttributeMaxDynamicSharedMemorySize, int(tbl_bytes));
    cudaFuncSetAttribute(k_cand<HB, WARPS>, cudaFuncAttributeMaxDynamicSharedMemorySize, int(csm));
    cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, k_cand<HB, WARPS>, WARPS * 32, csm);
    if (per_sm < 1) per_sm = 1;
    walk_per_sm[ds].store(per_sm, std::memory_order_relaxed);
  }
  if (L.n_lastocc) k_lastocc<HB><<<L.n_lastocc, 256, tbl_bytes, st>>>(wk, L.lastocc, L.n_lastocc);
  if (L.n_multi) {
    dim3 g((H + 255) / 256, L.n_multi < 65535u ? L.n_multi : 65535u);
    k_carry_scan<HB><<<g, 256, 0, st>>>(wk, L.multi, L.n_multi);
  }
  mk->mark(kPhPre, st);
  if (L.n_walk && L.ready && fused_cand_parse()) {
    // one persistent CTA per SM: CW walkers and 32 - CW parsers
    constexpr int CW = HB <= 12 ? 16 : 4;
    const size_t fsm = size_t(cand_parse_words<HB>(CW)) * 4;
    static std::atomic<int> fused_attr[64];
    if (!fused_attr[ds].load(std::memory_order_relaxed)) {
      cudaFuncSetAttribute(k_cand_parse<HB, CW>, cudaFuncAttributeMaxDynamicSharedMemorySize, int(fsm));
      fused_attr[ds].store(1, std::memory_order_relaxed);
    }
    uint32_t blocks = uint32_t(sms);
    const uint32_t need = (L.n_walk + CW - 1) / CW;
    if (blocks > need) blocks = need;
    mk->mark(kPhCand, st);
    k_cand_parse<HB, CW><<<blocks, 1024, fsm, st>>>(wk, L.walk, L.n_walk, L.counter, L.ready);
  } else if (L.n_walk) {
    uint32_t blocks = uint32_t(per_sm) * uint32_t(sms);
    const uint32_t need = (L.n_walk + WARPS - 1) / WARPS;
    if (blocks > need) blocks = need;
    k_cand<HB, WARPS><<<blocks, WARPS * 32, csm, st>>>(wk, L.walk, L.n_walk, L.counter);
    mk->mark(kPhCand, st);
    constexpr int PW = 16;
    static std::atomic<int> parse_per_sm[64];
    int pps = parse_per_sm[ds].load(std::memory_order_relaxed);
    if (!pps) {
      cudaOccupancyMaxActiveBlocksPerMultiprocessor(&pps, k_parse<PW>, PW * 32, 0);
      if (pps < 1) pps = 1;
      parse_per_sm[ds].store(pps, std::memory_order_relaxed);
    }
    uint32_t pblocks = uint32_t(sms) * uint32_t(pps);
    const uint32_t pneed = (L.n_walk + PW - 1) / PW;
    if (pblocks > pneed) pblocks = pneed;
    k_parse<PW><<<pblocks, PW * 32, 0, st>>>(wk, L.walk, L.n_walk, L.counter + 6);
  }
  mk->mark(kPhWalk, st);
  if (L.n_multi) {
    constexpr int FW = 8;
    uint32_t blocks = uint32_t(sms) * 8;
    const uint32_t need = (L.n_walk + FW - 1) / FW;
    if (blocks > need) blocks = need;
    k_fix1<FW><<<blocks, FW * 32, 0, st>>>(wk, L.walk, L.n_walk, L.counter + 4);
    k_fix2<FW><<<(L.n_multi + FW - 1) / FW, FW * 32, 0, st>>>(wk, L.multi, L.n_multi);
  }
  mk->mark(kPhFix, st);
}

bool fast_launches_fused() { return fused_cand_parse(); }

void launch_fast(const Work& wk, const FastLists& L, int hash_bits, cudaStream_t st, int sms, Marks* mk) {
  if (hash_bits == 12) launch_fast_t<12>(wk, L, st, sms, mk);
  else launch_fast_t<14>(wk, L, st, sms, mk);
}

}  // namespace orotb

// ====================================================================== no-allocation entry point
// Some callers cannot let a library allocate device memory: code that runs
// inside another framework's memory pool or under a fixed device-memory
// budget, where every byte on the GPU is owned by the caller.  They can still
// use the fast levels through deflate_gpu_compress_noalloc(): the caller
// passes device pointers for the input, the output and the output size, and
// the only working memory is the file-scope array below, which every GPU
// that loads this library holds until the process exits.  It keeps a padded
// copy of the input (so no read ever runs past the caller's buffer) and the
// token bit stream.  The kernel writes every word of it that it later reads,
// so nothing has to start at zero, but all calls share it: two calls whose
// kernels overlap on the GPU (different streams, or different host threads)
// race on it and must be ordered by the caller.
#include <mutex>
#include <string>
#include "../../include/orot_b200.h"

namespace orotb {

void set_error(const std::string& e);  // engine.cu

constexpr uint32_t kNoAllocInBytes = DEFLATE_GPU_NOALLOC_MAX_INPUT + 256;
constexpr uint32_t kNoAllocBitBytes = DEFLATE_GPU_NOALLOC_MAX_INPUT / 8 * 9 + 256;
static __device__ __align__(256) uint32_t g_noalloc_scratch[(kNoAllocInBytes + kNoAllocBitBytes) / 4];

template <int HB>
__global__ void __launch_bounds__(256) k_noalloc(const uint8_t* __restrict__ in, uint32_t n, uint8_t* __restrict__ out,
                                                  int level_arg, int lv, int fmt, uint32_t* scratch,
                                                  unsigned long long* out_size) {
  extern __shared__ uint32_t sm[];
  constexpr uint32_t HW = ((1u << HB) * 3 + 3) / 4;
  uint32_t* head = sm;
  uint32_t* ring = head + HW;
  uint32_t* wbuf = ring + kRing;
  __shared__ uint32_t crc_tab[256];
  __shared__ uint32_t part_crc[224], part_a[224], part_b[224], part_len[224];
  __shared__ uint32_t x2k[64];
  __shared__ uint32_t s_bits, s_matches;
  const uint32_t tid = threadIdx.x, lane = tid & 31, wid = tid >> 5;
  uint8_t* cin = reinterpret_cast<uint8_t*>(scratch);
  uint32_t* bits = scratch + kNoAllocInBytes / 4;

  // padded copy of the input; the tail is zeroed so over-reads see zeros
  for (uint32_t i = tid; i < n + 256; i += blockDim.x) cin[i] = i < n ? in[i] : 0;
  for (uint32_t i = tid; i < 256; i += blockDim.x) {
    uint32_t c = i;
    for (int k = 0; k < 8; ++k) c = (c & 1) ? (c >> 1) ^ kCrcPoly : (c >> 1);
    crc_tab[i] = c;
  }
  if (tid == 0) {
    uint32_t x = 0x40000000u;
    for (int k = 0; k < 64; ++k) { x2k[k] = x; x = gf2_mulmod(x, x); }
    s_bits = 0;
    s_matches = 0;
  }
  __syncthreads();

  if (wid == 0) {
    if (lv >= 1) {
      const TileView tv{SegBytes{reinterpret_cast<const uint32_t*>(cin), 0}, n, 0, n};
      const WinState r = walk_tile<HB>(tv, nullptr, head, ring, wbuf, bits, nullptr, nullptr);
      if (lane == 0) { s_bits = r.cursor; s_matches = r.matches; }
    }
  } else {
    // checksum partials over 224 contiguous parts
    const uint32_t t = tid - 32, per = (n + 223) / 224;
    const uint32_t b0 = min(n, t * per), b1 = min(n, b0 + per);
    uint32_t crc = 0, A = 0, B = 0;
    for (uint32_t i = b0; i < b1; ++i) {
      const uint32_t by = cin[i];
      crc = crc_tab[(crc ^ by) & 0xFF] ^ (crc >> 8);
      A += by;
      if (A >= 65521u) A -= 65521u;
      B += A;
      if (B >= 65521u) B -= 65521u;
    }
    part_crc[t] = crc;
    part_a[t] = A;
    part_b[t] = B;
    part_len[t] = b1 - b0;
  }
  __syncthreads();

  __shared__ uint32_t s_type, s_check;
  __shared__ unsigned long long s_total;
  if (tid == 0) {
    CrcPowers pw;
    for (int k = 0; k < 64; ++k) pw.x2k[k] = x2k[k];
    uint32_t crc = 0;
    uint64_t s1 = 1, s2 = 0;
    for (int t = 0; t < 224; ++t) {
      if (!part_len[t]) continue;
      crc = gf2_mulmod(xpow8n(pw, part_len[t]), crc) ^ part_crc[t];
      s2 = (s2 + uint64_t(part_len[t] % 65521u) * s1 + part_b[t]) % 65521u;
      s1 = (s1 + part_a[t]) % 65521u;
    }
    s_check = fmt == kFmtGzip ? ~(gf2_mulmod(xpow8n(pw, n), 0xFFFFFFFFu) ^ crc) : uint32_t(s2 << 16) | uint32_t(s1);
    // block type: level 0 and all-literal parses are stored
    // (src/compress/block_compressor.cpp:53-63, src/deflate/deflate_block.cpp:414-421)
    uint32_t type = kBlkStored;
    if (lv >= 1 && s_matches) {
      const uint64_t fixed_bits = 3ull + s_bits + 7;
      const uint64_t stored_bits = (uint64_t(n) + 5) * 8;
      type = stored_bits <= fixed_bits ? kBlkStored : kBlkFixed;
    }
    s_type = type;
    const uint64_t hdr = fmt == kFmtZlib ? 2 : fmt == kFmtGzip ? 10 : 0;
    const uint64_t trl = fmt == kFmtZlib ? 4 : fmt == kFmtGzip ? 8 : 0;
    const uint64_t pieces = n ? (n + 65534) / 65535 : 1;
    const uint64_t raw = type == kBlkStored ? uint64_t(n) + 5 * pieces : (3ull + s_bits + 7 + 7) / 8;
    s_total = hdr + raw + trl;
  }
  __syncthreads();
  const uint32_t hdr = fmt == kFmtZlib ? 2 : fmt == kFmtGzip ? 10 : 0;
  const uint64_t total = s_total;
  const uint32_t trl = fmt == kFmtZlib ? 4 : fmt == kFmtGzip ? 8 : 0;
  uint8_t* raw = out + hdr;
  const uint64_t raw_len = total - hdr - trl;
  if (s_type == kBlkFixed) {
    // 3 header bits (BFINAL=1, BTYPE=01), the token bits, 7 zero bits of EOB
    const uint32_t nb = s_bits;
    for (uint64_t k = tid; k < raw_len; k += blockDim.x) {
      uint32_t v = 0;
      const int64_t s = int64_t(k) * 8 - 3;  // token bit of output bit 0 of this byte
      for (int j = 0; j < 8; ++j) {
        const int64_t b = s + j;
        uint32_t bit;
        if (b < 0) bit = (3u >> (j)) & 1u;       // the 3 header bits: value 0b011
        else if (uint64_t(b) < nb) bit = (bits[b >> 5] >> (b & 31)) & 1u;
        else bit = 0;                            // EOB and padding
        v |= bit << j;
      }
      raw[k] = uint8_t(v);
    }
  } else {
    // stored pieces of at most 65535 bytes (deflate_block.cpp:107-132)
    for (uint64_t k = tid; k < raw_len; k += blockDim.x) {
      const uint64_t piece = k / 65540, off = k % 65540;
      const uint64_t start = piece * 65535;
      const uint32_t len = uint32_t(min(uint64_t(65535), uint64_t(n) - min(uint64_t(n), start)));
      uint8_t v;
      if (off == 0) v = (start + len == n) ? 1 : 0;
      else if (off == 1) v = uint8_t(len);
      else if (off == 2) v = uint8_t(len >> 8);
      else if (off == 3) v = uint8_t(~len);
      else if (off == 4) v = uint8_t(~len >> 8);
      else v = cin[start + off - 5];
      raw[k] = v;
    }
  }
  if (tid == 0) {
    if (fmt == kFmtZlib) {
      out[0] = 0x78; out[1] = 0x9C;
      for (int i = 0; i < 4; ++i) out[total - 4 + i] = uint8_t(s_check >> (24 - 8 * i));
    } else if (fmt == kFmtGzip) {
      const uint8_t xfl = level_arg >= 9 ? 2 : (level_arg <= 2 ? 4 : 0);
      const uint8_t h[10] = {0x1F, 0x8B, 8, 0, 0, 0, 0, 0, xfl, 0xFF};
      for (int i = 0; i < 10; ++i) out[i] = h[i];
      for (int i = 0; i < 4; ++i) {
        out[total - 8 + i] = uint8_t(s_check >> (8 * i));
        out[total - 4 + i] = uint8_t(n >> (8 * i));
      }
    }
    *out_size = total;
  }
}

// Device address of g_noalloc_scratch, looked up once per device (with that
// device current) on the first call made on it.
static uint32_t* noalloc_scratch_ptr(int dev) {
  static std::mutex mu;
  static uint32_t* ptrs[64] = {};
  static bool init[64] = {};
  if (dev < 0 || dev >= 64) {
    set_error("deflate_gpu_compress_noalloc: CUDA device index above 63");
    return nullptr;
  }
  std::lock_guard<std::mutex> lk(mu);
  if (!init[dev]) {
    void* p = nullptr;
    const cudaError_t e = cudaGetSymbolAddress(&p, g_noalloc_scratch);
    if (e != cudaSuccess) {
      cudaGetLastError();
      set_error(std::string("cudaGetSymbolAddress(g_noalloc_scratch): ") + cudaGetErrorString(e));
      return nullptr;
    }
    ptrs[dev] = static_cast<uint32_t*>(p);
    init[dev] = true;
  }
  return ptrs[dev];
}

}  // namespace orotb

extern "C" int deflate_gpu_compress_noalloc(const void* d_in, size_t in_size, void* d_out, size_t out_capacity,
                                            int level, deflate_format format, unsigned long long* d_out_size,
                                            void* cuda_stream) {
  using namespace orotb;
  const int fmt = int(format);
  if ((in_size && !d_in) || !d_out || !d_out_size || fmt < 0 || fmt > 2) {
    set_error("deflate_gpu_compress_noalloc: null pointer or unknown format");
    return -1;
  }
  if (in_size > DEFLATE_GPU_NOALLOC_MAX_INPUT) {
    set_error("deflate_gpu_compress_noalloc: input larger than DEFLATE_GPU_NOALLOC_MAX_INPUT (1 MiB)");
    return -2;
  }
  const int lv = level < 0 ? 0 : level > 12 ? 12 : level;
  if (lv > 3) {
    set_error("deflate_gpu_compress_noalloc: only levels 0-3 are available without allocation");
    return -3;
  }
  const size_t bound = in_size + (in_size >> 12) + (in_size >> 14) + (in_size >> 25) + 13 +
                       (fmt == kFmtZlib ? 6 : fmt == kFmtGzip ? 18 : 0);
  if (out_capacity < bound) {
    set_error("deflate_gpu_compress_noalloc: out_capacity below deflate_compress_bound()");
    return -4;
  }
  int dev = 0;
  if (cudaGetDevice(&dev) != cudaSuccess) { cudaGetLastError(); set_error("no CUDA device"); return -5; }
  uint32_t* scratch = noalloc_scratch_ptr(dev);
  if (!scratch) return -5;
  cudaStream_t st = static_cast<cudaStream_t>(cuda_stream);
  const uint8_t* in = static_cast<const uint8_t*>(d_in);
  uint8_t* out = static_cast<uint8_t*>(d_out);
  const uint32_t n = uint32_t(in_size);
  if (lv == 1 || lv == 0) {
    const size_t smem = size_t(walker_words<12>()) * 4;
    k_noalloc<12><<<1, 256, smem, st>>>(in, n, out, level, lv, fmt, scratch, d_out_size);
  } else {
    const size_t smem = size_t(walker_words<14>()) * 4;
    const cudaError_t a = cudaFuncSetAttribute(k_noalloc<14>, cudaFuncAttributeMaxDynamicSharedMemorySize, int(smem));
    if (a != cudaSuccess) {
      cudaGetLastError();
      set_error(std::string("deflate_gpu_compress_noalloc shared-memory set-up: ") + cudaGetErrorString(a));
      return -6;
    }
    k_noalloc<14><<<1, 256, smem, st>>>(in, n, out, level, lv, fmt, scratch, d_out_size);
  }
  const cudaError_t e = cudaGetLastError();
  if (e != cudaSuccess) {
    set_error(std::string("deflate_gpu_compress_noalloc launch: ") + cudaGetErrorString(e));
    return -6;
  }
  return 0;
}
