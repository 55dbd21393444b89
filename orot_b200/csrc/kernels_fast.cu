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
//   k_walk        one warp per tile: 32 positions per step; hash, __match_any
//                 for same-hash lanes, head[] in shared memory, capped match
//                 lengths per lane, greedy parse resolved with ballots, fixed
//                 Huffman bits packed with shared atomics and flushed as
//                 coalesced 128-byte stores.  The parse starts at the tile's
//                 first byte (speculation) and one record per 32 positions
//                 remembers where it entered that window.
//   k_fixup       one warp per multi-tile segment, tiles in order: re-walks a
//                 tile from the true entry (where the previous tile's parse
//                 ended) until it meets the speculative parse at a window
//                 boundary; from there the speculative bits are exact.
//
// The output is therefore token-for-token the reference's.
#include <cuda_runtime.h>
#include <cstdint>
#include "engine.cuh"
#include "deflate_device.cuh"
#include "kernels.cuh"

namespace orotb {

constexpr uint32_t kFull = 0xFFFFFFFFu;

__device__ __forceinline__ uint32_t hash_fast(uint32_t v, int hb) { return (v * 0x9E3779B1u) >> (32 - hb); }

// ---------------------------------------------------------------- k_lastocc
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
  const SegBytes sb{reinterpret_cast<const uint32_t*>(wk.in + (a & ~uint64_t(3))), uint32_t(a & 3)};
  const uint32_t end = t.start + t.len;
  for (uint32_t base = t.start + (threadIdx.x & ~31u); base < end; base += blockDim.x) {
    const uint32_t p = base + (threadIdx.x & 31);
    const bool ins = p < end && p + 4 <= sg.len;
    const uint32_t h = ins ? hash_fast(sb.load4(p), HB) : kFull;
    const uint32_t peers = __match_any_sync(kFull, h);
    if (ins && (peers >> (threadIdx.x & 31)) == 1u) atomicMax(&tbl[h], p);
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
  const uint32_t si = blockIdx.y;
  if (si >= nseg) return;
  const Segment sg = wk.segs[seglist[si]];
  const uint32_t h = blockIdx.x * blockDim.x + threadIdx.x;
  if (h >= uint32_t(H)) return;
  uint32_t run = 0;
  for (uint32_t k = 0; k + 1 < sg.tile_count; ++k) {
    uint32_t* slot = reinterpret_cast<uint32_t*>(wk.scratch + wk.tiles[sg.tile_first + k].slot);
    run = max(run, slot[h]);
    slot[h] = run;
  }
}

// ---------------------------------------------------------------- the walker
struct WalkIn {
  SegBytes sb;
  uint32_t n;            // segment length
  uint32_t ts, tl;       // tile start (segment-relative) and length
  uint32_t entry;        // parse start, segment-relative, in [ts, ts+tl)
  const uint32_t* carry; // head[] at tile start, nullptr = empty
  uint32_t* out;         // bit-stream words
  WinRec* rec_out;       // speculative walk: per-window records (may be null)
  const WinRec* rec_in;  // fix-up walk: the speculative records
};
struct WalkOut {
  uint32_t bits, matches, tokens, exit;
  uint32_t merged, merge_win;
};

template <int HB>
__device__ WalkOut walk_tile(const WalkIn& a, uint32_t* __restrict__ head, uint32_t* __restrict__ ring) {
  constexpr int H = 1 << HB;
  const uint32_t lane = threadIdx.x & 31;
  const uint32_t lt = (1u << lane) - 1;
  if (a.carry) {
    for (int i = lane; i < H; i += 32) head[i] = __ldg(a.carry + i);
  } else {
    for (int i = lane; i < H; i += 32) head[i] = 0;
  }
  for (int i = lane; i < 128; i += 32) ring[i] = 0;
  __syncwarp();

  WalkOut r{};
  uint32_t np = a.entry, cursor = 0, flushed = 0, matches = 0, tokens = 0;
  const uint32_t tend = a.ts + a.tl;
  const uint32_t nwin = (a.tl + 31) >> 5;
  for (uint32_t w = 0; w < nwin; ++w) {
    const uint32_t wpos = a.ts + (w << 5);
    if (a.rec_in) {
      const uint32_t se = a.ts + a.rec_in[w].entry;
      if (np == se) { r.merged = 1; r.merge_win = w; break; }
    }
    if (a.rec_out && lane == 0) a.rec_out[w] = WinRec{np - a.ts, cursor, matches, tokens};

    // -- insert the 32 positions of this window into head[]
    const uint32_t p = wpos + lane;
    const bool in_tile = p < tend;
    const bool ins = in_tile && p + 4 <= a.n;
    uint32_t v4 = 0, h = kFull;
    if (ins) { v4 = a.sb.load4(p); h = hash_fast(v4, HB); }
    const uint32_t peers = __match_any_sync(kFull, h);
    const uint32_t before = peers & lt;
    uint32_t cand = 0;
    if (ins) cand = before ? (wpos + 31 - __clz(before)) : head[h];
    __syncwarp();
    if (ins && (peers >> lane) == 1u) head[h] = p;
    __syncwarp();

    // -- greedy parse over the window
    const uint32_t lim = min(32u, tend - wpos);
    if (np >= wpos + lim) continue;
    uint32_t clen = 0, dist = 0;
    bool exact = true;
    if (ins && p >= np && cand != 0) {
      dist = (p - cand) & 0x7FFFu;
      if (dist != 0 && a.sb.byte(cand) == (v4 & 0xFFu)) {
        const uint32_t maxm = min(258u, a.n - p);
        const uint32_t cap = min(maxm, max(3u, 32u - lane));
        clen = lcp_capped(a.sb, p, p - dist, cap);
        exact = clen < cap || cap == maxm;
        if (clen < 3) clen = 0;
      }
    }
    const uint32_t M = __ballot_sync(kFull, clen >= 3);
    const uint32_t limmask = lim == 32 ? kFull : ((1u << lim) - 1);
    uint32_t cur = np - wpos, visited = 0;
    int xl = -1;  // lane whose match runs past the window and needs its full length
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
      const uint32_t dj = __shfl_sync(kFull, dist, xl);
      const uint32_t c0 = __shfl_sync(kFull, clen, xl);
      const uint32_t maxm = min(258u, a.n - pj);
      full = c0;
      for (uint32_t base = c0; base < maxm; base += 128) {
        const uint32_t off = base + 4 * lane;
        uint32_t stop = kFull;
        if (off < maxm) {
          const uint32_t x = a.sb.load4(pj + off) ^ a.sb.load4(pj - dj + off);
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

    // -- emit the visited tokens
    const bool vis = (visited >> lane) & 1u;
    const bool ism = vis && ((M >> lane) & 1u);
    uint32_t code = 0, nb = 0;
    if (vis) {
      if (ism) fixed_match(int(lane) == xl ? full : clen, dist, code, nb);
      else fixed_literal(ins ? (v4 & 0xFFu) : a.sb.byte(p), code, nb);
    }
    uint32_t incl = nb;
#pragma unroll
    for (int o = 1; o < 32; o <<= 1) {
      const uint32_t t = __shfl_up_sync(kFull, incl, o);
      if (lane >= uint32_t(o)) incl += t;
    }
    const uint32_t total = __shfl_sync(kFull, incl, 31);
    if (nb) {
      const uint32_t bp = cursor + incl - nb, wd = bp >> 5, sh = bp & 31;
      atomicOr(&ring[wd & 127], code << sh);
      if (sh + nb > 32) atomicOr(&ring[(wd + 1) & 127], code >> (32 - sh));
    }
    cursor += total;
    tokens += __popc(visited);
    matches += __popc(visited & M);
    np = wpos + cur;
    __syncwarp();
    while ((cursor >> 5) >= flushed + 32) {
      a.out[flushed + lane] = ring[(flushed + lane) & 127];
      ring[(flushed + lane) & 127] = 0;
      flushed += 32;
      __syncwarp();
    }
  }
  const uint32_t nwords = (cursor + 31) >> 5;
  for (uint32_t i = flushed + lane; i < nwords; i += 32) a.out[i] = ring[i & 127];
  __syncwarp();
  r.bits = cursor;
  r.matches = matches;
  r.tokens = tokens;
  r.exit = np;
  return r;
}

__device__ __forceinline__ WalkIn walk_args(const Work& wk, const Tile& t, const Segment& sg) {
  WalkIn a;
  const uint64_t o = sg.in_off;
  a.sb = SegBytes{reinterpret_cast<const uint32_t*>(wk.in + (o & ~uint64_t(3))), uint32_t(o & 3)};
  a.n = sg.len;
  a.ts = t.start;
  a.tl = t.len;
  a.entry = t.start;
  a.carry = t.index ? reinterpret_cast<const uint32_t*>(wk.scratch + t.carry) : nullptr;
  a.out = reinterpret_cast<uint32_t*>(wk.scratch + t.scratch);
  a.rec_out = nullptr;
  a.rec_in = nullptr;
  return a;
}

// ---------------------------------------------------------------- k_walk
template <int HB, int WARPS>
__global__ void __launch_bounds__(WARPS * 32) k_walk(Work wk, const uint32_t* __restrict__ list, uint32_t nlist,
                                                      uint32_t* __restrict__ counter) {
  extern __shared__ uint32_t sm[];
  constexpr int H = 1 << HB;
  const uint32_t wid = threadIdx.x >> 5, lane = threadIdx.x & 31;
  uint32_t* head = sm + wid * (H + 128);
  uint32_t* ring = head + H;
  for (;;) {
    uint32_t i = 0;
    if (lane == 0) i = atomicAdd(counter, 1u);
    i = __shfl_sync(kFull, i, 0);
    if (i >= nlist) break;
    Tile* tp = wk.tiles + list[i];
    const Tile t = *tp;
    const Segment sg = wk.segs[t.seg];
    WalkIn a = walk_args(wk, t, sg);
    if (t.index) a.rec_out = reinterpret_cast<WinRec*>(wk.scratch + t.rec);
    const WalkOut r = walk_tile<HB>(a, head, ring);
    if (lane == 0) {
      tp->spec_bits = r.bits;
      tp->spec_matches = r.matches;
      tp->spec_exit = r.exit;
      tp->spec_tokens = r.tokens;
      tp->fix_bits = 0;
      tp->splice_bit = 0;
      tp->fin_matches = r.matches;
      tp->fin_exit = r.exit;
    }
  }
}

// ---------------------------------------------------------------- k_fixup
template <int HB, int WARPS>
__global__ void __launch_bounds__(WARPS * 32) k_fixup(Work wk, const uint32_t* __restrict__ seglist, uint32_t nseg) {
  extern __shared__ uint32_t sm[];
  constexpr int H = 1 << HB;
  const uint32_t wid = threadIdx.x >> 5, lane = threadIdx.x & 31;
  uint32_t* head = sm + wid * (H + 128);
  uint32_t* ring = head + H;
  const uint32_t si = blockIdx.x * WARPS + wid;
  if (si >= nseg) return;
  const Segment sg = wk.segs[seglist[si]];
  uint32_t exit = wk.tiles[sg.tile_first].fin_exit;
  for (uint32_t k = 1; k < sg.tile_count; ++k) {
    Tile* tp = wk.tiles + sg.tile_first + k;
    const Tile t = *tp;
    uint32_t fix_bits = 0, splice = 0, fin_m = t.spec_matches, fin_x = t.spec_exit;
    if (exit >= t.start + t.len) {          // a match of the previous tile covers this one
      splice = t.spec_bits; fin_m = 0; fin_x = exit;
    } else if (exit != t.start) {
      WalkIn a = walk_args(wk, t, sg);
      a.entry = exit;
      a.out = reinterpret_cast<uint32_t*>(wk.scratch + t.scratch + tile_stream_bytes(t.len));
      a.rec_in = reinterpret_cast<const WinRec*>(wk.scratch + t.rec);
      const WalkOut r = walk_tile<HB>(a, head, ring);
      fix_bits = r.bits;
      if (r.merged) {
        const WinRec rc = a.rec_in[r.merge_win];
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
    }
    exit = fin_x;
    __syncwarp();
  }
}

// ---------------------------------------------------------------- launchers
template <int HB>
static void launch_fast_t(const Work& wk, const FastLists& L, cudaStream_t st, int sms) {
  constexpr int H = 1 << HB;
  constexpr int WARPS = HB <= 12 ? 4 : 1;
  const size_t tbl_bytes = size_t(H) * 4;
  if (L.n_lastocc) {
    cudaFuncSetAttribute(k_lastocc<HB>, cudaFuncAttributeMaxDynamicSharedMemorySize, int(tbl_bytes));
    k_lastocc<HB><<<L.n_lastocc, 256, tbl_bytes, st>>>(wk, L.lastocc, L.n_lastocc);
  }
  if (L.n_multi) {
    dim3 g((H + 255) / 256, L.n_multi);
    k_carry_scan<HB><<<g, 256, 0, st>>>(wk, L.multi, L.n_multi);
  }
  const size_t wsm = size_t(WARPS) * (H + 128) * 4;
  if (L.n_walk) {
    cudaFuncSetAttribute(k_walk<HB, WARPS>, cudaFuncAttributeMaxDynamicSharedMemorySize, int(wsm));
    int per_sm = 0;
    cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, k_walk<HB, WARPS>, WARPS * 32, wsm);
    if (per_sm < 1) per_sm = 1;
    uint32_t blocks = uint32_t(per_sm) * uint32_t(sms);
    const uint32_t need = (L.n_walk + WARPS - 1) / WARPS;
    if (blocks > need) blocks = need;
    k_walk<HB, WARPS><<<blocks, WARPS * 32, wsm, st>>>(wk, L.walk, L.n_walk, L.counter);
  }
  if (L.n_multi) {
    cudaFuncSetAttribute(k_fixup<HB, WARPS>, cudaFuncAttributeMaxDynamicSharedMemorySize, int(wsm));
    k_fixup<HB, WARPS><<<(L.n_multi + WARPS - 1) / WARPS, WARPS * 32, wsm, st>>>(wk, L.multi, L.n_multi);
  }
}

void launch_fast(const Work& wk, const FastLists& L, int hash_bits, cudaStream_t st, int sms) {
  if (hash_bits == 12) launch_fast_t<12>(wk, L, st, sms);
  else launch_fast_t<14>(wk, L, st, sms);
}

}  // namespace orotb
