// kernels_common.cu -- block planning, output assembly and checksums.
//
//   k_plan      one thread per stream: block type of every segment (the
//               reference's rules, src/deflate/deflate_block.cpp:389-474 and
//               src/compress/block_compressor.cpp:53-63), bit offset of every
//               block, and the list of bit-range copies that assemble the
//               stream; output size and capacity check.
//   k_zero      clears the words the stream will occupy.
//   k_ck_block  CRC-32 (slicing-by-4) and Adler-32 partial sums of 64 KiB
//               blocks, 256 bytes per thread, folded with the GF(2) shift /
//               Adler weight identities.
//   k_ck_fold   folds the blocks of each stream in order.
//   k_join      one warp per copy: funnel-shifted 32-bit words, plain stores
//               inside a copy, atomicOr on the two boundary words it shares.
//   k_frame     zlib / gzip header and trailer bytes.
#include <cuda_runtime.h>
#include <mutex>
#include <cstdint>
#include "engine.cuh"
#include "deflate_device.cuh"
#include "kernels.cuh"

namespace orotb {

constexpr uint32_t kFullMask = 0xFFFFFFFFu;

__host__ __device__ inline uint32_t fmt_header_bytes(uint32_t fmt) { return fmt == kFmtZlib ? 2 : fmt == kFmtGzip ? 10 : 0; }
__host__ __device__ inline uint32_t fmt_trailer_bytes(uint32_t fmt) { return fmt == kFmtZlib ? 4 : fmt == kFmtGzip ? 8 : 0; }

// ---------------------------------------------------------------- k_plan
__device__ __forceinline__ void put_piece(Piece* pc, uint32_t& k, uint32_t kmax, const uint32_t* src, uint32_t* dst,
                                          uint64_t sbit, uint64_t dbit, uint32_t nbits, uint32_t value) {
  if (nbits == 0) return;
  if (k < kmax) pc[k] = Piece{src, dst, sbit, dbit, nbits, value};
  ++k;
}

__global__ void k_plan(Work wk) {
  const uint32_t si = blockIdx.x * blockDim.x + threadIdx.x;
  if (si >= wk.nstreams) return;
  Stream s = wk.streams[si];
  const bool bare = (s.mode & kStreamBare) != 0;
  const uint32_t hdr = bare ? 0 : fmt_header_bytes(s.fmt), trl = bare ? 0 : fmt_trailer_bytes(s.fmt);
  uint32_t* dst = reinterpret_cast<uint32_t*>(wk.out + s.out_off);
  Piece* pc = wk.pieces + s.piece_first;
  uint32_t k = 0;
  const uint32_t kmax = s.piece_count;
  const uint64_t base = uint64_t(hdr) * 8;
  uint64_t c = 0;  // bits from the start of the raw DEFLATE stream
  bool bad = false;
  for (uint32_t g = s.seg_first; g < s.seg_first + s.seg_count; ++g) {
    Segment sg = wk.segs[g];
    const bool last = (sg.flags & kSegLast) != 0;
    uint32_t type = kBlkStored;
    uint64_t tok_bits = 0, matches = 0;
    if (sg.level > 0) {
      for (uint32_t t = sg.tile_first; t < sg.tile_first + sg.tile_count; ++t) {
        const Tile& tl = wk.tiles[t];
        tok_bits += uint64_t(tl.fix_bits) + (tl.spec_bits - tl.splice_bit);
        matches += tl.fin_matches;
      }
      if (sg.level >= 4) {
        type = sg.block_type;  // chosen by the lazy pipeline
      } else if ((sg.flags & kSegWholeBuf) && matches == 0) {
        type = kBlkStored;     // all-literal parse (block_compressor.cpp:60-61)
      } else {
        const uint64_t fixed_bits = 3 + tok_bits + 7;      // header + tokens + EOB
        const uint64_t stored_bits = (uint64_t(sg.len) + 5) * 8;
        type = stored_bits <= fixed_bits ? kBlkStored : kBlkFixed;
      }
    }
    const uint64_t start = c;
    if (type == kBlkStored) {
      uint32_t off = 0;
      for (;;) {
        const uint32_t n = min(sg.len - off, 65535u);
        const bool fin = last && off + n == sg.len;
        put_piece(pc, k, kmax, nullptr, dst, 0, base + c, 3, fin ? 1u : 0u);
        c += 3;
        c = (c + 7) & ~uint64_t(7);
        put_piece(pc, k, kmax, nullptr, dst, 0, base + c, 32, n | ((~n & 0xFFFFu) << 16));
        c += 32;
        const uint64_t a = sg.in_off + off;
        put_piece(pc, k, kmax, reinterpret_cast<const uint32_t*>(wk.in + (a & ~uint64_t(3))), dst, (a & 3) * 8,
                  base + c, n * 8, 0);
        c += uint64_t(n) * 8;
        off += n;
        if (n == 0 || off >= sg.len) break;
      }
    } else {
      // BFINAL + BTYPE (write_bits(type, 2) puts the low bit first)
      if (type == kBlkFixed) {
        put_piece(pc, k, kmax, nullptr, dst, 0, base + c, 3, (last ? 1u : 0u) | (1u << 1));
        c += 3;
      } else {
        // code-length header written by the Huffman kernel
        const uint32_t* hsrc = reinterpret_cast<const uint32_t*>(wk.scratch + sg.hdr_off);
        put_piece(pc, k, kmax, nullptr, dst, 0, base + c, 3, (last ? 1u : 0u) | (2u << 1));
        c += 3;
        put_piece(pc, k, kmax, hsrc, dst, 0, base + c, sg.hdr_bits, 0);
        c += sg.hdr_bits;
      }
      for (uint32_t t = sg.tile_first; t < sg.tile_first + sg.tile_count; ++t) {
        const Tile& tl = wk.tiles[t];
        const uint32_t* spec = reinterpret_cast<const uint32_t*>(wk.scratch + tl.scratch);
        const uint32_t* fix = reinterpret_cast<const uint32_t*>(wk.scratch + tl.scratch + tile_stream_bytes(tl.len));
        put_piece(pc, k, kmax, fix, dst, 0, base + c, tl.fix_bits, 0);
        c += tl.fix_bits;
        put_piece(pc, k, kmax, spec, dst, tl.splice_bit, base + c, tl.spec_bits - tl.splice_bit, 0);
        c += tl.spec_bits - tl.splice_bit;
      }
      if (type == kBlkFixed) {
        c += 7;  // EOB is code 0000000
      } else {
        const uint32_t eob = sg.eob;  // dynamic EOB: code | (len << 16)
        put_piece(pc, k, kmax, nullptr, dst, 0, base + c, eob >> 16, eob & 0xFFFFu);
        c += eob >> 16;
      }
    }
    if (last) c = (c + 7) & ~uint64_t(7);
    sg.block_type = type;
    sg.bit_off = start;
    sg.bits = c - start;
    wk.segs[g] = sg;
  }
  if (s.mode & kStreamOpen) {
    // sync point: empty stored block, BFINAL = 0, LEN 0000 NLEN FFFF
    put_piece(pc, k, kmax, nullptr, dst, 0, base + c, 3, 0u);
    c = (c + 3 + 7) & ~uint64_t(7);
    put_piece(pc, k, kmax, nullptr, dst, 0, base + c, 32, 0xFFFF0000u);
    c += 32;
  }
  bad = k > kmax;
  const uint64_t size = uint64_t(hdr) + c / 8 + trl;
  s.raw_bits = c;
  s.error = kErrNone;
  if (bad) s.error = kErrInternal;
  else if (size > s.out_cap) s.error = kErrCapacity;
  s.out_size = s.error ? 0 : size;
  if (s.error) k = 0;
  for (uint32_t i = (k < kmax ? k : kmax); i < kmax; ++i) pc[i].nbits = 0;
  wk.streams[si] = s;
}

// ---------------------------------------------------------------- k_zero
__global__ void k_zero(Work wk) {
  const uint32_t si = blockIdx.x;
  if (si >= wk.nstreams) return;
  const Stream s = wk.streams[si];
  if (s.error) return;
  uint4* o = reinterpret_cast<uint4*>(wk.out + s.out_off);
  const uint64_t n16 = (s.out_size + 15) / 16;
  for (uint64_t i = threadIdx.x; i < n16; i += blockDim.x) o[i] = make_uint4(0, 0, 0, 0);
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

__global__ void k_ck_fold(Work wk, CrcPowers pw) {
  const uint32_t si = blockIdx.x * blockDim.x + threadIdx.x;
  if (si >= wk.nstreams) return;
  Stream s = wk.streams[si];
  if (s.fmt == kFmtRaw) return;
  uint32_t crc = 0;
  uint64_t s1 = 1, s2 = 0;
  for (uint32_t i = s.ck_first; i < s.ck_first + s.ck_count; ++i) {
    const CkBlock b = wk.ck[i];
    const uint32_t shift = b.len == kCkBlock ? c_crc_block : xpow8n(pw, b.len);
    crc = gf2_mulmod(shift, crc) ^ b.crc;
    s2 = (s2 + uint64_t(b.len % kAdlerMod) * s1 + b.b) % kAdlerMod;
    s1 = (s1 + b.a) % kAdlerMod;
  }
  if (s.fmt == kFmtGzip) {
    // crc32(0, data) = ~(x^(8n) * ~0 + raw(data))
    s.checksum = ~(gf2_mulmod(xpow8n(pw, s.in_len), 0xFFFFFFFFu) ^ crc);
  } else {
    s.checksum = uint32_t(s2 << 16) | uint32_t(s1);
  }
  wk.streams[si].checksum = s.checksum;
}

// Single-stream checksum with an arbitrary initial value (deflate_crc32 /
// deflate_adler32): result written to *res.
__global__ void k_ck_single(const CkBlock* ck, uint32_t nck, uint64_t total, uint32_t init, int adler, CrcPowers pw,
                            uint32_t* res) {
  if (threadIdx.x || blockIdx.x) return;
  uint32_t crc = 0;
  uint64_t s1 = (init & 0xFFFFu) % kAdlerMod, s2 = (init >> 16) % kAdlerMod;
  for (uint32_t i = 0; i < nck; ++i) {
    const CkBlock b = ck[i];
    const uint32_t shift = b.len == kCkBlock ? c_crc_block : xpow8n(pw, b.len);
    crc = gf2_mulmod(shift, crc) ^ b.crc;
    s2 = (s2 + uint64_t(b.len % kAdlerMod) * s1 + b.b) % kAdlerMod;
    s1 = (s1 + b.a) % kAdlerMod;
  }
  if (adler) *res = uint32_t(s2 << 16) | uint32_t(s1);
  else *res = ~(gf2_mulmod(xpow8n(pw, total), ~init) ^ crc);
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

void launch_plan(const Work& wk, cudaStream_t st) {
  if (!wk.nstreams) return;
  k_plan<<<(wk.nstreams + 127) / 128, 128, 0, st>>>(wk);
  k_zero<<<wk.nstreams, 256, 0, st>>>(wk);
}

void launch_checksums(const Work& wk, cudaStream_t st) {
  const CrcPowers pw = host_crc_powers();
  if (wk.nck) k_ck_block<<<wk.nck, 256, 0, st>>>(wk, pw);
  if (wk.nstreams) k_ck_fold<<<(wk.nstreams + 127) / 128, 128, 0, st>>>(wk, pw);
}

void launch_ck_single(const CkBlock* ck, uint32_t nck, uint64_t total, uint32_t init, int adler, uint32_t* res,
                      const Work& wk, cudaStream_t st) {
  const CrcPowers pw = host_crc_powers();
  if (nck) k_ck_block<<<nck, 256, 0, st>>>(wk, pw);
  k_ck_single<<<1, 32, 0, st>>>(ck, nck, total, init, adler, pw, res);
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
