// kernels_common.cu -- block planning, output assembly and checksums.
//
//   k_plan_*    block type of every segment (the reference's rules,
//               src/deflate/deflate_block.cpp:389-474 and
//               src/compress/block_compressor.cpp:53-63), bit offset of every
//               block, and the list of bit-range copies that assemble the
//               stream; output size and capacity check (one warp per segment
//               or stream, see below).
//   k_zero      clears the words the streams will occupy.
//   k_ck_block  CRC-32 (slicing-by-4) and Adler-32 partial sums of 64 KiB
//               blocks, 256 bytes per thread, folded with the GF(2) shift /
//               Adler weight identities.
//   k_ck_fold   folds the blocks of each stream: runs of blocks per thread,
//               then a tree over the runs (one CTA per stream).
//   k_join      one warp per copy: funnel-shifted 32-bit words, plain stores
//               inside a copy, atomicOr on the two boundary words it shares.
//   k_frame     zlib / gzip header and trailer bytes.
#include <cuda_runtime.h>
#include <algorithm>
#include <mutex>
#include <cstdint>
#include "engine.cuh"
#include "deflate_device.cuh"
#include "kernels.cuh"

namespace orotb {

constexpr uint32_t kFullMask = 0xFFFFFFFFu;

__host__ __device__ inline uint32_t fmt_header_bytes(uint32_t fmt) { return fmt == kFmtZlib ? 2 : fmt == kFmtGzip ? 10 : 0; }
__host__ __device__ inline uint32_t fmt_trailer_bytes(uint32_t fmt) { return fmt == kFmtZlib ? 4 : fmt == kFmtGzip ? 8 : 0; }

// ---------------------------------------------------------------- planning
// Three kernels, so that a stream of thousands of segments (a pigz-style
// stream) or a segment of thousands of tiles (a large whole buffer) is
// planned in parallel:
//   k_plan_seg     one warp per segment: token bits and matches summed over
//                  its tiles, the block type, and the block's length when it
//                  does not depend on its bit alignment (Huffman blocks).
//   k_plan_stream  one warp per stream: block offsets in order (32 segments
//                  loaded at a time, followed through shuffles; a stored
//                  block's padding depends on where it starts), stream size,
//                  capacity check, the closing sync point of an open part.
//   k_plan_pieces  one warp per segment: its bit-range copies, at slots the
//                  host reserved for the segment (Segment::piece_off); unused
//                  slots are left empty (nbits 0).

// Bits a stored block of `len` bytes starting at bit c occupies: per piece of
// at most 65535 bytes, 3 header bits, padding to a byte, LEN/NLEN and the
// bytes (deflate_block.cpp:107-132).
__device__ __forceinline__ uint64_t stored_bits_at(uint64_t c, uint32_t len) {
  const uint64_t pieces = len ? (uint64_t(len) + 65534) / 65535 : 1;
  return (((c + 3 + 7) & ~uint64_t(7)) - c) + 32 + uint64_t(len) * 8 + (pieces - 1) * 40;
}

__device__ __forceinline__ uint32_t seg_piece_slots(const Segment& sg) {
  const uint32_t stored_pieces = max(1u, (sg.len + 65534u) / 65535u);
  return 1 + 2 * sg.tile_count + 2 + 3 * stored_pieces;
}

__global__ void k_plan_seg(Work wk) {
  const uint32_t g = (blockIdx.x * blockDim.x + threadIdx.x) >> 5, lane = threadIdx.x & 31;
  if (g >= wk.nsegs) return;
  const Segment sg = wk.segs[g];
  unsigned long long tok = 0, matches = 0;
  if (sg.level > 0) {
    for (uint32_t t = sg.tile_first + lane; t < sg.tile_first + sg.tile_count; t += 32) {
      const Tile& tl = wk.tiles[t];
      tok += uint64_t(tl.fix_bits) + (tl.spec_bits - tl.splice_bit);
      matches += tl.fin_matches;
    }
  }
#pragma unroll
  for (int o = 16; o > 0; o >>= 1) {
    tok += __shfl_xor_sync(kFullMask, tok, o);
    matches += __shfl_xor_sync(kFullMask, matches, o);
  }
  if (lane) return;
  uint32_t type = kBlkStored;
  uint64_t bits = 0;
  if (sg.level > 0) {
    if (sg.level >= 4) {
      type = sg.block_type;  // chosen by the lazy pipeline
    } else if ((sg.flags & kSegWholeBuf) && matches == 0) {
      type = kBlkStored;     // all-literal parse (block_compressor.cpp:60-61)
    } else {
      const uint64_t fixed_bits = 3 + tok + 7;      // header + tokens + EOB
      const uint64_t stored = (uint64_t(sg.len) + 5) * 8;
      type = stored <= fixed_bits ? kBlkStored : kBlkFixed;
    }
  }
  if (type == kBlkFixed) bits = 3 + tok + 7;                       // EOB is code 0000000
  else if (type == kBlkDynamic) bits = 3 + sg.hdr_bits + tok + (sg.eob >> 16);
  wk.segs[g].block_type = type;
  wk.segs[g].bits = bits;
}

__global__ void k_plan_stream(Work wk) {
  const uint32_t si = (blockIdx.x * blockDim.x + threadIdx.x) >> 5, lane = threadIdx.x & 31;
  if (si >= wk.nstreams) return;
  Stream s = wk.streams[si];
  const bool bare = (s.mode & kStreamBare) != 0;
  const uint32_t hdr = bare ? 0 : fmt_header_bytes(s.fmt), trl = bare ? 0 : fmt_trailer_bytes(s.fmt);
  uint64_t c = 0;  // bits from the start of the raw DEFLATE stream
  bool fault = false;  // a kernel could not finish one of the stream's segments
  for (uint32_t g0 = s.seg_first; g0 < s.seg_first + s.seg_count; g0 += 32) {
    const uint32_t cnt = min(32u, s.seg_first + s.seg_count - g0);
    uint32_t type = 0, len = 0, last = 0;
    uint64_t bits = 0;
    if (lane < cnt) {
      const Segment& sg = wk.segs[g0 + lane];
      type = sg.block_type;
      len = sg.len;
      last = sg.flags & kSegLast;
      bits = sg.bits;
      if (sg.flags & kSegFault) fault = true;
    }
    uint64_t my_off = 0, my_bits = 0;
    for (uint32_t j = 0; j < cnt; ++j) {
      const uint32_t tj = __shfl_sync(kFullMask, type, j), lj = __shfl_sync(kFullMask, len, j);
      const uint32_t fj = __shfl_sync(kFullMask, last, j);
      const uint64_t bj = __shfl_sync(kFullMask, bits, j);
      const uint64_t start = c;
      c += tj == kBlkStored ? stored_bits_at(c, lj) : bj;
      if (fj) c = (c + 7) & ~uint64_t(7);
      if (lane == j) { my_off = start; my_bits = c - start; }
    }
    if (lane < cnt) {
      wk.segs[g0 + lane].bit_off = my_off;
      wk.segs[g0 + lane].bits = my_bits;
    }
  }
  fault = __any_sync(kFullMask, fault);
  if (lane) return;
  Piece* tail = wk.pieces + s.piece_first + s.piece_count - 2;  // the open part's sync point
  const uint64_t sync_at = c;
  if (s.mode & kStreamOpen) c = ((c + 3 + 7) & ~uint64_t(7)) + 32;  // empty stored block, BFINAL = 0
  const uint64_t size = uint64_t(hdr) + c / 8 + trl;
  s.raw_bits = c;
  s.error = fault ? kErrInternal : size > s.out_cap ? kErrCapacity : kErrNone;
  s.out_size = s.error ? 0 : size;
  if (s.mode & kStreamOpen) {
    uint32_t* dst = reinterpret_cast<uint32_t*>(wk.out + s.out_off);
    const uint64_t base = uint64_t(hdr) * 8;
    tail[0] = Piece{nullptr, dst, 0, base + sync_at, s.error ? 0u : 3u, 0u};
    tail[1] = Piece{nullptr, dst, 0, base + ((sync_at + 3 + 7) & ~uint64_t(7)), s.error ? 0u : 32u, 0xFFFF0000u};
  }
  wk.streams[si] = s;
}

__global__ void k_plan_pieces(Work wk) {
  const uint32_t g = (blockIdx.x * blockDim.x + threadIdx.x) >> 5, lane = threadIdx.x & 31;
  if (g >= wk.nsegs) return;
  const Segment sg = wk.segs[g];
  const Stream& s = wk.streams[sg.stream];
  const bool bare = (s.mode & kStreamBare) != 0;
  const uint32_t hdr = bare ? 0 : fmt_header_bytes(s.fmt);
  uint32_t* dst = reinterpret_cast<uint32_t*>(wk.out + s.out_off);
  Piece* pc = wk.pieces + s.piece_first + sg.piece_off;
  const uint32_t slots = seg_piece_slots(sg);
  const uint64_t c = uint64_t(hdr) * 8 + sg.bit_off;  // block start in the output slot
  const bool last = (sg.flags & kSegLast) != 0;
  for (uint32_t i = lane; i < slots; i += 32) pc[i].nbits = 0;
  __syncwarp();
  if (s.error) return;
  if (sg.block_type == kBlkStored) {
    const uint32_t P = max(1u, (sg.len + 65534u) / 65535u);
    const uint64_t c1 = ((c + 3 + 7) & ~uint64_t(7)) + 32 + 8ull * 65535;  // start of piece 1 (when P > 1)
    for (uint32_t i = lane; i < P; i += 32) {
      const uint64_t ci = i == 0 ? c : c1 + uint64_t(i - 1) * (40 + 8ull * 65535);
      const uint32_t off = i * 65535u, n = min(sg.len - off, 65535u);
      const bool fin = last && off + n == sg.len;
      const uint64_t lenpos = (ci + 3 + 7) & ~uint64_t(7);
      const uint64_t a = sg.in_off + off;
      pc[3 * i] = Piece{nullptr, dst, 0, ci, 3, fin ? 1u : 0u};
      pc[3 * i + 1] = Piece{nullptr, dst, 0, lenpos, 32, n | ((~n & 0xFFFFu) << 16)};
      pc[3 * i + 2] = Piece{reinterpret_cast<const uint32_t*>(wk.in + (a & ~uint64_t(3))), dst, (a & 3) * 8,
                            lenpos + 32, n * 8, 0};
    }
    return;
  }
  // BFINAL + BTYPE (write_bits(type, 2) puts the low bit first), then the
  // code-length header of a dynamic block (written by the Huffman kernel)
  uint64_t at = c + 3;
  if (lane == 0) pc[0] = Piece{nullptr, dst, 0, c, 3, (last ? 1u : 0u) | (sg.block_type << 1)};
  if (sg.block_type == kBlkDynamic) {
    if (lane == 0)
      pc[1] = Piece{reinterpret_cast<const uint32_t*>(wk.scratch + sg.hdr_off), dst, 0, at, sg.hdr_bits, 0};
    at += sg.hdr_bits;
  }
  // two copies per tile (fix-up bits, then the speculative bits from the
  // splice point), at offsets from a prefix sum over the tiles
  for (uint32_t t0 = 0; t0 < sg.tile_count; t0 += 32) {
    const uint32_t t = t0 + lane;
    uint32_t fb = 0, sb = 0, sp = 0;
    const Tile* tl = nullptr;
    if (t < sg.tile_count) {
      tl = wk.tiles + sg.tile_first + t;
      fb = tl->fix_bits;
      sp = tl->splice_bit;
      sb = tl->spec_bits - sp;
    }
    unsigned long long incl = uint64_t(fb) + sb;
#pragma unroll
    for (int o = 1; o < 32; o <<= 1) {
      const unsigned long long v = __shfl_up_sync(kFullMask, incl, o);
      if (lane >= uint32_t(o)) incl += v;
    }
    const uint64_t mine = at + incl - (uint64_t(fb) + sb);
    if (tl) {
      const uint32_t* spec = reinterpret_cast<const uint32_t*>(wk.scratch + tl->scratch);
      const uint32_t* fix = reinterpret_cast<const uint32_t*>(wk.scratch + tl->scratch + tile_stream_bytes(tl->len));
      pc[2 + 2 * t] = Piece{fix, dst, 0, mine, fb, 0};
      pc[3 + 2 * t] = Piece{spec, dst, sp, mine + fb, sb, 0};
    }
    at += __shfl_sync(kFullMask, incl, 31);
  }
  if (lane == 0 && sg.block_type == kBlkDynamic) {
    const uint32_t eob = sg.eob;  // dynamic EOB: code | (len << 16)
    pc[2 + 2 * sg.tile_count] = Piece{nullptr, dst, 0, at, eob >> 16, eob & 0xFFFFu};
  }
}

// ---------------------------------------------------------------- k_zero
// Clears the words every stream will occupy (the join ORs boundary words):
// blockIdx.y splits a stream into gridDim.y parts, so one large stream is
// cleared by many CTAs.
__global__ void k_zero(Work wk) {
  const uint32_t si = blockIdx.x;
  if (si >= wk.nstreams) return;
  const Stream s = wk.streams[si];
  if (s.error) return;
  uint4* o = reinterpret_cast<uint4*>(wk.out + s.out_off);
  const uint64_t n16 = (s.out_size + 15) / 16;
  const uint64_t per = (n16 + gridDim.y - 1) / gridDim.y;
  const uint64_t b = per * blockIdx.y, e = min(n16, b + per);
  for (uint64_t i = b + threadIdx.x; i < e; i += blockDim.x) o[i] = make_uint4(0, 0, 0, 0);
}

// ---------------------------------------------------------------- checksums
__constant__ uint32_t c_crc_slice[4][256];
__constant__ uint32_t c_crc_sub[9];   // x^(8*256*2^s), s = 0..8
__constant__ uint32_t c_crc_block;    // x^(8*65536)

constexpr uint32_t kAdlerMod = 65521u;
constexpr uint32_t kCkBlock = 65536u;
constexpr uint32_t kCkSub = 256u;

__global__ void __launch_bounds__(256) k_ck_block(Work wk, CrcPowers pw) {
  __shared__ uint32_t tb[4][256];
  __shared__ uint32_t sc[256], sa[256], sb2[256], sl[256];
  for (int i = threadIdx.x; i < 1024; i += blockDim.x) tb[i >> 8][i & 255] = c_crc_slice[i >> 8][i & 255];
  __syncthreads();
  const uint32_t bi = blockIdx.x;
  if (bi >= wk.nck) return;
  CkBlock b = wk.ck[bi];
  const uint32_t t = threadIdx.x;
  const uint32_t o0 = t * kCkSub;
  const uint32_t len = o0 < b.len ? min(kCkSub, b.len - o0) : 0u;
  const uint8_t* p = wk.in + b.in_off + o0;
  uint32_t crc = 0, A = 0, B = 0;
  uint32_t i = 0;
  const uint32_t what = b.what;  // uniform over the block
  // one 32-bit word: CRC slicing-by-4; Adler A += bytes, B += 4A + 4,3,2,1-weighted bytes
  auto word = [&](uint32_t v) {
    if (what & kCkCrc) {
      crc ^= v;
      crc = tb[3][crc & 0xFF] ^ tb[2][(crc >> 8) & 0xFF] ^ tb[1][(crc >> 16) & 0xFF] ^ tb[0][crc >> 24];
    }
    if (what & kCkAdler) {
      B += 4 * A + __dp4a(v, 0x01020304u, 0u);
      A += __dp4a(v, 0x01010101u, 0u);
    }
  };
  const uint64_t ab = b.in_off + o0;
  if ((ab & 15) == 0) {
    const uint4* p16 = reinterpret_cast<const uint4*>(wk.in + ab);
    for (; i + 16 <= len; i += 16) {
      const uint4 v = __ldg(p16 + (i >> 4));
      word(v.x);
      word(v.y);
      word(v.z);
      word(v.w);
    }
  }
  // aligned words, funnel-shifted when the block does not start on a word
  const uint32_t* pw4 = reinterpret_cast<const uint32_t*>(wk.in + (ab & ~uint64_t(3)));
  const uint32_t sh = uint32_t(ab & 3) * 8;
  for (; i + 4 <= len; i += 4)
    word(sh ? __funnelshift_r(__ldg(pw4 + (i >> 2)), __ldg(pw4 + (i >> 2) + 1), sh) : __ldg(pw4 + (i >> 2)));
  for (; i < len; ++i) {
    const uint32_t by = p[i];
    crc = tb[0][(crc ^ by) & 0xFF] ^ (crc >> 8);
    A += by;
    B += A;
  }
  // B so far is sum_j (prefix sums) = sum_i (len - i) d_i, as the fold wants.
  sc[t] = crc;
  sa[t] = A % kAdlerMod;
  sb2[t] = B % kAdlerMod;
  sl[t] = len;
  __syncthreads();
  int lvl = 0;
  for (uint32_t s = 1; s < 256; s <<= 1, ++lvl) {
    if ((t & (2 * s - 1)) == 0 && t + s < 256) {
      const uint32_t lr = sl[t + s];
      if (lr) {
        if (what & kCkCrc) {
          const uint32_t shift = (lr == kCkSub * s) ? c_crc_sub[lvl] : xpow8n(pw, lr);
          sc[t] = gf2_mulmod(shift, sc[t]) ^ sc[t + s];
        }
        if (what & kCkAdler) {
          sb2[t] = uint32_t((uint64_t(sb2[t]) + uint64_t(lr % kAdlerMod) * sa[t] + sb2[t + s]) % kAdlerMod);
          sa[t] = (sa[t] + sa[t + s]) % kAdlerMod;
        }
        sl[t] += lr;
      }
    }
    __syncthreads();
  }
  if (t == 0) {
    b.crc = sc[0];
    b.a = sa[0];
    b.b = sb2[0];
    wk.ck[bi] = b;
  }
}

// Checksum partial of a byte range: the raw CRC register from 0, Adler sums
// A = sum of bytes and B = sum of (len - i) * byte_i (mod 65521), and length.
struct CkPartial {
  uint32_t crc, a, b;
  uint64_t len;
};
constexpr int kFoldThreads = 128;

// Folds blocks blk[0, n) in order into one partial: every thread of the CTA
// (kFoldThreads threads) folds a contiguous run of blocks, then the runs are
// combined in a tree (appending R multiplies the CRC register by x^(8|R|) and
// adds |R| * A to B).  Every thread must call it; thread 0 gets the result.
__device__ CkPartial fold_blocks(const CkBlock* blk, uint32_t n, uint32_t what, const CrcPowers& pw,
                                 CkPartial* sh) {
  const uint32_t t = threadIdx.x;
  const uint32_t per = (n + kFoldThreads - 1) / kFoldThreads;
  const uint32_t b0 = min(n, t * per), b1 = min(n, b0 + per);
  CkPartial p{0, 0, 0, 0};
  for (uint32_t i = b0; i < b1; ++i) {
    const CkBlock b = blk[i];
    if (what & kCkCrc) p.crc = gf2_mulmod(b.len == kCkBlock ? c_crc_block : xpow8n(pw, b.len), p.crc) ^ b.crc;
    if (what & kCkAdler) {
      p.b = uint32_t((uint64_t(p.b) + uint64_t(b.len % kAdlerMod) * p.a + b.b) % kAdlerMod);
      p.a = (p.a + b.a) % kAdlerMod;
    }
    p.len += b.len;
  }
  sh[t] = p;
  __syncthreads();
  for (uint32_t s = 1; s < uint32_t(kFoldThreads); s <<= 1) {
    if ((t & (2 * s - 1)) == 0 && t + s < uint32_t(kFoldThreads)) {
      CkPartial l = sh[t];
      const CkPartial r = sh[t + s];
      if (r.len) {
        if (what & kCkCrc) l.crc = gf2_mulmod(xpow8n(pw, r.len), l.crc) ^ r.crc;
        if (what & kCkAdler) {
          l.b = uint32_t((uint64_t(l.b) + (r.len % kAdlerMod) * l.a + r.b) % kAdlerMod);
          l.a = (l.a + r.a) % kAdlerMod;
        }
        l.len += r.len;
        sh[t] = l;
      }
    }
    __syncthreads();
  }
  return sh[0];
}

// One CTA per stream.
__global__ void __launch_bounds__(kFoldThreads) k_ck_fold(Work wk, CrcPowers pw) {
  __shared__ CkPartial sh[kFoldThreads];
  const uint32_t si = blockIdx.x;
  if (si >= wk.nstreams) return;
  const Stream& s = wk.streams[si];
  if (s.fmt == kFmtRaw) return;
  const uint32_t what = s.fmt == kFmtGzip ? kCkCrc : kCkAdler;
  const CkPartial p = fold_blocks(wk.ck + s.ck_first, s.ck_count, what, pw, sh);
  if (threadIdx.x) return;
  uint32_t check;
  if (s.fmt == kFmtGzip) {
    // crc32(0, data) = ~(x^(8n) * ~0 + raw(data))
    check = ~(gf2_mulmod(xpow8n(pw, s.in_len), 0xFFFFFFFFu) ^ p.crc);
  } else {
    // Adler-32 from 1: s1 = 1 + A, s2 = n + B
    const uint64_t s1 = (1 + p.a) % kAdlerMod, s2 = (s.in_len % kAdlerMod + p.b) % kAdlerMod;
    check = uint32_t(s2 << 16) | uint32_t(s1);
  }
  wk.streams[si].checksum = check;
}

// Single-stream checksum with an arbitrary initial value (deflate_crc32 /
// deflate_adler32): result written to *res.  One CTA.
__global__ void __launch_bounds__(kFoldThreads) k_ck_single(const CkBlock* ck, uint32_t nck, uint64_t total,
                                                            uint32_t init, int adler, CrcPowers pw, uint32_t* res) {
  __shared__ CkPartial sh[kFoldThreads];
  if (blockIdx.x) return;
  const CkPartial p = fold_blocks(ck, nck, adler ? kCkAdler : kCkCrc, pw, sh);
  if (threadIdx.x) return;
  if (adler) {
    const uint64_t a0 = (init & 0xFFFFu) % kAdlerMod, b0 = (init >> 16) % kAdlerMod;
    const uint64_t s1 = (a0 + p.a) % kAdlerMod;
    const uint64_t s2 = (b0 + (total % kAdlerMod) * a0 + p.b) % kAdlerMod;
    *res = uint32_t(s2 << 16) | uint32_t(s1);
  } else {
    *res = ~(gf2_mulmod(xpow8n(pw, total), ~init) ^ p.crc);
  }
}

// ---------------------------------------------------------------- k_join
__global__ void __launch_bounds__(256) k_join(Work wk, uint32_t* counter) {
  const uint32_t lane = threadIdx.x & 31;
  for (;;) {
    uint32_t i = 0;
    if (lane == 0) i = atomicAdd(counter, 1u);
    i = __shfl_sync(kFullMask, i, 0);
    if (i >= wk.npieces) break;
    const Piece pc = wk.pieces[i];
    if (pc.nbits == 0) continue;
    uint32_t* dst = pc.dst;
    if (pc.src == nullptr) {
      if (lane == 0) {
        const uint64_t w = pc.dst_bit >> 5;
        const uint32_t sh = uint32_t(pc.dst_bit & 31);
        const uint32_t v = pc.nbits == 32 ? pc.value : (pc.value & ((1u << pc.nbits) - 1));
        atomicOr(dst + w, v << sh);
        if (sh + pc.nbits > 32) atomicOr(dst + w + 1, v >> (32 - sh));
      }
      continue;
    }
    const uint64_t d0 = pc.dst_bit, d1 = pc.dst_bit + pc.nbits;
    const uint64_t w0 = d0 >> 5, w1 = (d1 - 1) >> 5;
    const int64_t delta = int64_t(pc.src_bit) - int64_t(d0);
    for (uint64_t w = w0 + lane; w <= w1; w += 32) {
      const int64_t sbit = int64_t(w) * 32 + delta;
      const int64_t sw = sbit >> 5;  // floor
      const uint32_t sh = uint32_t(sbit & 31);
      const uint32_t lo = sw >= 0 ? __ldg(pc.src + sw) : 0u;
      const uint32_t hi = __ldg(pc.src + sw + 1);
      const uint32_t v = __funnelshift_r(lo, hi, sh);
      const uint64_t x0 = w * 32;
      const uint32_t lb = uint32_t((d0 > x0 ? d0 : x0) - x0);
      const uint32_t hb = uint32_t((d1 < x0 + 32 ? d1 : x0 + 32) - x0);
      if (lb == 0 && hb == 32) {
        dst[w] = v;
      } else {
        const uint32_t m = (hb - lb == 32) ? kFullMask : (((1u << (hb - lb)) - 1) << lb);
        atomicOr(dst + w, v & m);
      }
    }
  }
}

// ---------------------------------------------------------------- k_frame
__global__ void k_frame(Work wk) {
  const uint32_t si = blockIdx.x * blockDim.x + threadIdx.x;
  if (si >= wk.nstreams) return;
  const Stream s = wk.streams[si];
  if (s.error || s.fmt == kFmtRaw || (s.mode & kStreamBare)) return;
  uint8_t* o = wk.out + s.out_off;
  const uint64_t end = s.out_size;
  if (s.fmt == kFmtZlib) {
    // header 78 9C (zlib_wrapper.cpp:21-22), Adler-32 big-endian trailer
    o[0] = 0x78; o[1] = 0x9C;
    for (int i = 0; i < 4; ++i) o[end - 4 + i] = uint8_t(s.checksum >> (24 - 8 * i));
  } else {
    // 1F 8B 08 00 mtime=0 XFL OS=FF (gzip_wrapper.cpp:31-43); the parallel
    // path always writes XFL 0 (parallel_compressor.cpp:96-98)
    const uint8_t xfl = s.parallel ? 0 : (s.level >= 9 ? 2 : (s.level <= 2 ? 4 : 0));
    const uint8_t h[10] = {0x1F, 0x8B, 8, 0, 0, 0, 0, 0, xfl, 0xFF};
    for (int i = 0; i < 10; ++i) o[i] = h[i];
    const uint32_t isz = uint32_t(s.in_len);
    for (int i = 0; i < 4; ++i) {
      o[end - 8 + i] = uint8_t(s.checksum >> (8 * i));
      o[end - 4 + i] = uint8_t(isz >> (8 * i));
    }
  }
}

// ---------------------------------------------------------------- launchers
// The constant tables live in each device's own constant memory, so they are
// uploaded once per device (under a lock: engines of one device may be
// created by several host threads at once).
bool upload_crc_tables() {
  static std::mutex mu;
  static bool done[64] = {};
  int dev = 0;
  if (cudaGetDevice(&dev) != cudaSuccess || dev < 0 || dev >= 64) return false;
  std::lock_guard<std::mutex> lk(mu);
  if (done[dev]) return true;
  uint32_t t[4][256];
  for (uint32_t i = 0; i < 256; ++i) {
    uint32_t c = i;
    for (int k = 0; k < 8; ++k) c = (c & 1) ? (c >> 1) ^ kCrcPoly : (c >> 1);
    t[0][i] = c;
  }
  for (int s = 1; s < 4; ++s)
    for (int i = 0; i < 256; ++i) t[s][i] = (t[s - 1][i] >> 8) ^ t[0][t[s - 1][i] & 0xFF];
  CrcPowers pw = host_crc_powers();
  uint32_t sub[9];
  for (int s = 0; s < 9; ++s) sub[s] = xpow8n(pw, uint64_t(kCkSub) << s);
  const uint32_t blk = xpow8n(pw, kCkBlock);
  if (cudaMemcpyToSymbol(c_crc_slice, t, sizeof t) != cudaSuccess ||
      cudaMemcpyToSymbol(c_crc_sub, sub, sizeof sub) != cudaSuccess ||
      cudaMemcpyToSymbol(c_crc_block, &blk, sizeof blk) != cudaSuccess) {
    cudaGetLastError();
    return false;
  }
  done[dev] = true;
  return true;
}

CrcPowers host_crc_powers() {
  CrcPowers pw;
  uint32_t x = 0x40000000u;  // the polynomial x
  for (int k = 0; k < 64; ++k) { pw.x2k[k] = x; x = gf2_mulmod(x, x); }
  return pw;
}

void launch_plan(const Work& wk, uint64_t max_out, cudaStream_t st) {
  if (!wk.nstreams) return;
  if (wk.nsegs) k_plan_seg<<<(wk.nsegs + 7) / 8, 256, 0, st>>>(wk);
  k_plan_stream<<<(wk.nstreams + 7) / 8, 256, 0, st>>>(wk);
  if (wk.nsegs) k_plan_pieces<<<(wk.nsegs + 7) / 8, 256, 0, st>>>(wk);
  // about 1 MiB of output per clearing CTA for the largest stream
  const uint32_t parts = uint32_t(std::min<uint64_t>(256, std::max<uint64_t>(1, max_out >> 20)));
  k_zero<<<dim3(wk.nstreams, parts), 256, 0, st>>>(wk);
}

void launch_checksums(const Work& wk, cudaStream_t st) {
  const CrcPowers pw = host_crc_powers();
  if (wk.nck) k_ck_block<<<wk.nck, 256, 0, st>>>(wk, pw);
  if (wk.nstreams) k_ck_fold<<<wk.nstreams, kFoldThreads, 0, st>>>(wk, pw);
}

void launch_ck_single(const CkBlock* ck, uint32_t nck, uint64_t total, uint32_t init, int adler, uint32_t* res,
                      const Work& wk, cudaStream_t st) {
  const CrcPowers pw = host_crc_powers();
  if (nck) k_ck_block<<<nck, 256, 0, st>>>(wk, pw);
  k_ck_single<<<1, kFoldThreads, 0, st>>>(ck, nck, total, init, adler, pw, res);
}

void launch_join(const Work& wk, uint32_t* counter, cudaStream_t st, int sms) {
  if (!wk.npieces) return;
  uint32_t blocks = uint32_t(sms) * 8;
  const uint32_t need = (wk.npieces + 7) / 8;
  if (blocks > need) blocks = need;
  k_join<<<blocks, 256, 0, st>>>(wk, counter);
}

void launch_frame(const Work& wk, cudaStream_t st) {
  if (!wk.nstreams) return;
  k_frame<<<(wk.nstreams + 127) / 128, 128, 0, st>>>(wk);
}

}  // namespace orotb
