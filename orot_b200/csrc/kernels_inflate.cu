// kernels_inflate.cu -- DEFLATE decoding (RFC 1951) on sm_100a.
//
// Decoding a DEFLATE stream is sequential: each code's length is known only
// after the previous one is decoded.  The parallel unit is therefore the
// stream: one warp per stream, warps take streams from a counter (largest
// first, so the longest decode starts first).  Inside the warp, lane 0 reads
// bits and decodes symbols, writing literals itself; the 32 lanes build the
// Huffman lookup tables together and copy every match together (a copy of
// length L at distance D reads only bytes before the copy, out[p - D + i % D],
// so all lanes copy at once even when D < L).
//
// Codes are decoded with a 9-bit lookup table (codes up to 9 bits, nearly all
// symbols of real data) and, for longer codes, the canonical rule of RFC 1951
// 3.2.2 walked bit by bit: codes of one length are consecutive integers and
// shorter codes precede longer ones, so per length the code is compared
// against the first code and the number of codes of that length.
//
// The kernel does not read the zlib / gzip framing; the host strips it and
// checks the trailer against a checksum of the output (src/formats/*:
// zlib_decompress, gzip_decompress semantics).
#include <cuda_runtime.h>
#include <cstdint>
#include "engine.cuh"
#include "kernels.cuh"

namespace orotb {

namespace {

constexpr uint32_t kAll = 0xFFFFFFFFu;
constexpr int kFastBits = 9;
constexpr uint32_t kFast = 1u << kFastBits;
constexpr uint32_t kWin = 8192;   // recent output kept in shared memory per warp
constexpr int kInfWarps = 4;      // warps per CTA

// RFC 1951 3.2.5: base lengths / distances and extra bits of symbols 257..285
// and distance codes 0..29.
__constant__ uint16_t c_len_base[29] = {3,  4,  5,  6,  7,  8,  9,  10, 11,  13,  15,  17,  19,  23, 27,
                                        31, 35, 43, 51, 59, 67, 83, 99, 115, 131, 163, 195, 227, 258};
__constant__ uint8_t c_len_extra[29] = {0, 0, 0, 0, 0, 0, 0, 0, 1, 1, 1, 1, 2, 2, 2, 2, 3, 3, 3, 3, 4, 4, 4, 4, 5, 5, 5, 5, 0};
__constant__ uint16_t c_dist_base[30] = {1,   2,   3,   4,   5,   7,    9,    13,   17,   25,   33,   49,   65,    97,    129,
                                         193, 257, 385, 513, 769, 1025, 1537, 2049, 3073, 4097, 6145, 8193, 12289, 16385, 24577};
__constant__ uint8_t c_dist_extra[30] = {0, 0, 0, 0, 1, 1, 2, 2, 3, 3, 4, 4, 5, 5, 6, 6, 7, 7, 8, 8, 9, 9, 10, 10, 11, 11, 12, 12, 13, 13};
// order of the code-length code lengths in a dynamic block header (3.2.7)
__constant__ uint8_t c_cl_order[19] = {16, 17, 18, 0, 8, 7, 9, 6, 10, 5, 11, 4, 12, 3, 13, 2, 14, 1, 15};

// One Huffman code: lookup table for codes up to 9 bits ((len << 12) | sym,
// 0 = longer code), code counts per length and the symbols in code order.
struct Code {
  uint16_t* fast;
  uint16_t* count;  // [16]
  uint16_t* sym;    // [nsym]
};

// Per-warp shared memory.  Output goes to global memory and to `win`: a match
// whose source lies in the window reads shared memory instead of waiting for
// the bytes this warp has just stored to come back from L2.
struct WarpMem {
  uint16_t lfast[kFast], dfast[kFast];
  uint16_t lcount[16], dcount[16];
  uint16_t lsym[288], dsym[32];
  uint16_t first[16], offs[16];  // builder scratch: first code and first index per length
  uint8_t lens[320];
  uint32_t bad;                  // builder result
  uint8_t win[kWin];             // the last kWin output bytes, at position & (kWin - 1)
};

// Builds `c` from code lengths lens[0..n) (all lanes).  Returns false for an
// over-subscribed set of lengths; an incomplete set is accepted (a code that
// is not assigned is reported when it is read).
__device__ bool build_code(const Code& c, const uint8_t* lens, uint32_t n, WarpMem& m, uint32_t lane) {
  for (uint32_t i = lane; i < kFast; i += 32) c.fast[i] = 0;
  if (lane == 0) {
    for (int l = 0; l < 16; ++l) c.count[l] = 0;
    for (uint32_t s = 0; s < n; ++s) c.count[lens[s]]++;
    c.count[0] = 0;
    int left = 1;  // codes still available at the current length
    uint32_t bad = 0;
    for (int l = 1; l < 16; ++l) {
      left = (left << 1) - c.count[l];
      if (left < 0) bad = 1;
    }
    m.offs[1] = 0;
    for (int l = 1; l < 15; ++l) m.offs[l + 1] = m.offs[l] + c.count[l];
    uint32_t code = 0;
    for (int l = 1; l < 16; ++l) {
      m.first[l] = uint16_t(code);
      code = (code + c.count[l]) << 1;
    }
    for (uint32_t s = 0; s < n; ++s)
      if (lens[s]) c.sym[m.offs[lens[s]]++] = uint16_t(s);
    // offs now holds the index one past each length's symbols; restore
    for (int l = 15; l >= 1; --l) m.offs[l] -= c.count[l];
    m.bad = bad;
  }
  __syncwarp();
  if (m.bad) return false;
  // fill the lookup table: symbol i (in code order) of length l <= 9
  uint32_t total = 0;
  for (int l = 1; l < 16; ++l) total += c.count[l];
  for (uint32_t i = lane; i < total; i += 32) {
    const uint32_t s = c.sym[i];
    const uint32_t l = lens[s];
    if (l > uint32_t(kFastBits)) continue;
    const uint32_t code = m.first[l] + (i - m.offs[l]);
    const uint32_t rev = __brev(code) >> (32 - l);  // codes are sent most significant bit first
    for (uint32_t k = rev; k < kFast; k += 1u << l) c.fast[k] = uint16_t((l << 12) | s);
  }
  __syncwarp();
  return true;
}

// LSB-first bit reader over [p, end); reads whole aligned words (the buffers
// carry padding after their last byte) and counts bits taken past the end.
struct BitIn {
  const uint8_t* base;
  uint64_t pos, end;  // byte positions relative to base
  uint64_t buf;
  uint32_t cnt;
  __device__ __forceinline__ void refill() {
    if (cnt > 32) return;
    uint32_t v = 0;
    if (pos < end) {
      const uint64_t a = reinterpret_cast<uint64_t>(base) + pos;
      const uint32_t* w = reinterpret_cast<const uint32_t*>(a & ~uint64_t(3));
      v = __funnelshift_r(__ldg(w), __ldg(w + 1), uint32_t(a & 3) * 8);
      if (pos + 4 > end) v &= (1u << (8 * uint32_t(end - pos))) - 1u;
    }
    buf |= uint64_t(v) << cnt;
    cnt += 32;
    pos += 4;
  }
  __device__ __forceinline__ uint32_t take(uint32_t n) {  // n <= 32, needs n bits buffered
    const uint32_t v = uint32_t(buf) & (n == 32 ? kAll : ((1u << n) - 1u));
    buf >>= n;
    cnt -= n;
    return v;
  }
  // bytes consumed so far
  __device__ __forceinline__ uint64_t used() const { return pos - cnt / 8; }
};

// Decodes one symbol (lane 0).  Returns 0xFFFF for a code that is not assigned.
__device__ __forceinline__ uint32_t decode(BitIn& b, const Code& c) {
  b.refill();
  const uint32_t e = c.fast[uint32_t(b.buf) & (kFast - 1)];
  if (e) {
    b.take(e >> 12);
    return e & 0xFFFu;
  }
  int code = 0, first = 0, index = 0;
  for (int l = 1; l < 16; ++l) {
    code |= int(b.take(1));
    const int count = c.count[l];
    if (code - first < count) return c.sym[index + (code - first)];
    index += count;
    first = (first + count) << 1;
    code <<= 1;
  }
  return 0xFFFFu;
}

}  // namespace

// status: kInfOk, kInfData (corrupt), kInfOutput (output full), kInfInput (input exhausted)
__global__ void __launch_bounds__(kInfWarps * 32) k_inflate(const uint8_t* __restrict__ in, uint8_t* __restrict__ out,
                                                 InflateJob* jobs, const uint32_t* __restrict__ order, uint32_t njobs,
                                                 uint32_t* counter) {
  __shared__ WarpMem wm[kInfWarps];
  const uint32_t lane = threadIdx.x & 31, wid = threadIdx.x >> 5;
  WarpMem& m = wm[wid];
  const Code lit{m.lfast, m.lcount, m.lsym}, dst{m.dfast, m.dcount, m.dsym};
  for (;;) {
    uint32_t k = 0;
    if (lane == 0) k = atomicAdd(counter, 1u);
    k = __shfl_sync(kAll, k, 0);
    if (k >= njobs) break;
    InflateJob* jp = jobs + order[k];
    const InflateJob job = *jp;
    uint8_t* o = out + job.out_off;
    BitIn b{in + job.in_off, 0, job.in_len, 0, 0};
    uint64_t op = 0;  // output position
    int32_t status = kInfOk;
    bool last = false;
    while (!last && status == kInfOk) {
      // block header (lane 0 reads, every lane learns the type)
      uint32_t hdr = 0;
      if (lane == 0) {
        b.refill();
        hdr = b.take(3);
      }
      hdr = __shfl_sync(kAll, hdr, 0);
      last = hdr & 1u;
      const uint32_t type = hdr >> 1;
      if (type == 3) { status = kInfData; break; }
      if (type == 0) {
        // stored: byte-align, LEN, NLEN, LEN raw bytes
        uint64_t src = 0;
        uint32_t len = 0, ok = 1;
        if (lane == 0) {
          b.take(b.cnt & 7);
          b.refill();
          const uint32_t ln = b.take(32);
          len = ln & 0xFFFFu;
          ok = ((ln >> 16) ^ 0xFFFFu) == len;
          src = b.used();  // the bytes left in the buffer are the block's first bytes
          b.buf = 0;
          b.cnt = 0;
          b.pos = src + len;
        }
        len = __shfl_sync(kAll, len, 0);
        ok = __shfl_sync(kAll, ok, 0);
        src = __shfl_sync(kAll, src, 0);
        if (!ok) { status = kInfData; break; }
        if (src + len > job.in_len) { status = kInfInput; break; }
        if (op + len > job.out_cap) { status = kInfOutput; break; }
        const uint8_t* s = in + job.in_off + src;
        for (uint32_t i = lane; i < len; i += 32) {
          const uint8_t v = s[i];
          o[op + i] = v;
          m.win[(op + i) & (kWin - 1)] = v;
        }
        op += len;
        __syncwarp();
        continue;
      }
      // Huffman block: tables
      if (type == 1) {
        for (uint32_t i = lane; i < 320; i += 32) m.lens[i] = i < 144 ? 8 : i < 256 ? 9 : i < 280 ? 7 : i < 288 ? 8 : 5;
        __syncwarp();
        build_code(lit, m.lens, 288, m, lane);
        build_code(dst, m.lens + 288, 30, m, lane);
      } else {
        uint32_t hlit = 0, hdist = 0, err = 0;
        if (lane == 0) {
          b.refill();
          hlit = b.take(5) + 257;
          hdist = b.take(5) + 1;
          const uint32_t hclen = b.take(4) + 4;
          for (int i = 0; i < 19; ++i) m.lens[300 + i] = 0;
          for (uint32_t i = 0; i < hclen; ++i) {
            b.refill();
            m.lens[300 + c_cl_order[i]] = uint8_t(b.take(3));
          }
        }
        __syncwarp();
        hlit = __shfl_sync(kAll, hlit, 0);
        hdist = __shfl_sync(kAll, hdist, 0);
        // the code-length code lives in the literal table while the lengths are read
        if (hlit > 286 || hdist > 30 || !build_code(lit, m.lens + 300, 19, m, lane)) err = 1;
        if (lane == 0 && !err) {
          uint32_t i = 0;
          const uint32_t n = hlit + hdist;
          while (i < n) {
            const uint32_t sym = decode(b, lit);
            if (sym < 16) {
              m.lens[i++] = uint8_t(sym);
              continue;
            }
            uint32_t rep = 0, val = 0;
            b.refill();
            if (sym == 16) {
              if (i == 0) { err = 1; break; }
              val = m.lens[i - 1];
              rep = 3 + b.take(2);
            } else if (sym == 17) {
              rep = 3 + b.take(3);
            } else if (sym == 18) {
              rep = 11 + b.take(7);
            } else {
              err = 1;
              break;
            }
            if (i + rep > n) { err = 1; break; }
            while (rep--) m.lens[i++] = uint8_t(val);
          }
          if (!err && m.lens[256] == 0) err = 1;  // no end-of-block code
          // distance lengths follow the literal lengths; move them to 288..
          if (!err) {
            for (uint32_t j = hdist; j-- > 0;) m.lens[288 + j] = m.lens[hlit + j];  // ranges may overlap
            for (uint32_t j = hlit; j < 288; ++j) m.lens[j] = 0;
            for (uint32_t j = hdist; j < 32; ++j) m.lens[288 + j] = 0;
          }
        }
        err = __shfl_sync(kAll, err, 0);
        __syncwarp();
        if (err) { status = kInfData; break; }
        if (!build_code(lit, m.lens, 288, m, lane) || !build_code(dst, m.lens + 288, 30, m, lane)) {
          status = kInfData;
          break;
        }
      }
      // symbols: lane 0 decodes literals until a match or the end of the block
      for (;;) {
        uint32_t cmd = 0, len = 0, dist = 0;  // cmd: 0 end of block, 1 match, 2 error
        int32_t st = kInfOk;
        if (lane == 0) {
          for (;;) {
            const uint32_t sym = decode(b, lit);
            if (sym < 256) {
              if (op >= job.out_cap) { st = kInfOutput; cmd = 2; break; }
              o[op] = uint8_t(sym);
              m.win[op & (kWin - 1)] = uint8_t(sym);
              ++op;
              continue;
            }
            if (sym == 256) { cmd = 0; break; }
            if (sym > 285) { st = kInfData; cmd = 2; break; }
            b.refill();
            len = c_len_base[sym - 257] + b.take(c_len_extra[sym - 257]);
            const uint32_t ds = decode(b, dst);
            if (ds > 29) { st = kInfData; cmd = 2; break; }
            b.refill();
            dist = c_dist_base[ds] + b.take(c_dist_extra[ds]);
            if (dist > op) { st = kInfData; cmd = 2; break; }
            if (op + len > job.out_cap) { st = kInfOutput; cmd = 2; break; }
            cmd = 1;
            break;
          }
          if (b.used() > job.in_len && st == kInfOk) { st = kInfInput; cmd = 2; }
        }
        cmd = __shfl_sync(kAll, cmd, 0);
        if (cmd != 1) {
          status = __shfl_sync(kAll, st, 0);
          break;
        }
        len = __shfl_sync(kAll, len, 0);
        dist = __shfl_sync(kAll, dist, 0);
        const uint64_t p0 = __shfl_sync(kAll, op, 0);
        __syncwarp();
        // sources lie before p0; in the window unless the copy's own writes
        // could reach the slots other lanes read (dist + len > kWin)
        const bool in_win = dist + len <= kWin;
        for (uint32_t i = lane; i < len; i += 32) {
          const uint64_t src = p0 - dist + (i < dist ? i : i % dist);
          const uint8_t v = in_win ? m.win[src & (kWin - 1)] : o[src];
          o[p0 + i] = v;
          m.win[(p0 + i) & (kWin - 1)] = v;
        }
        __syncwarp();
        if (lane == 0) op += len;
      }
      op = __shfl_sync(kAll, op, 0);
    }
    if (lane == 0) {
      if (status == kInfOk && b.used() > job.in_len) status = kInfInput;
      jp->out_len = op;
      jp->in_used = status == kInfOk ? b.used() : 0;
      jp->status = status;
    }
    __syncwarp();
  }
}

// Compares decoded bytes with the original input, one warp per stream.
__global__ void __launch_bounds__(256) k_inflate_compare(const uint8_t* __restrict__ a, const uint8_t* __restrict__ b,
                                                         InflateJob* jobs, const uint64_t* __restrict__ ref_off,
                                                         const uint64_t* __restrict__ ref_len, uint32_t njobs) {
  const uint32_t lane = threadIdx.x & 31;
  const uint32_t j = (blockIdx.x * blockDim.x + threadIdx.x) >> 5;
  if (j >= njobs) return;
  InflateJob job = jobs[j];
  if (job.status != kInfOk) return;
  bool same = job.out_len == ref_len[j];
  if (same) {
    const uint8_t* x = a + job.out_off;
    const uint8_t* y = b + ref_off[j];
    for (uint64_t i = lane; i < job.out_len && same; i += 32) same = x[i] == y[i];
  }
  same = __all_sync(kAll, same);
  if (lane == 0 && !same) jobs[j].status = kInfMismatch;
}

// Framing of compressed streams (one thread per stream): zlib 78 9C header and
// big-endian Adler-32 trailer, gzip 1F 8B 08 header, little-endian CRC-32 and
// ISIZE; the trailer must carry the stream's checksum and length.
__global__ void k_frame_check(const uint8_t* __restrict__ out, const Stream* __restrict__ st, InflateJob* jobs,
                              uint32_t n) {
  const uint32_t i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= n) return;
  const Stream s = st[i];
  if (s.error || jobs[i].status != kInfOk || s.fmt == kFmtRaw) return;
  const uint8_t* o = out + s.out_off;
  const uint8_t* t = o + s.out_size;
  bool good;
  if (s.fmt == kFmtZlib) {
    const uint32_t a = (uint32_t(t[-4]) << 24) | (uint32_t(t[-3]) << 16) | (uint32_t(t[-2]) << 8) | t[-1];
    good = o[0] == 0x78 && o[1] == 0x9C && a == s.checksum;
  } else {
    const uint32_t c = uint32_t(t[-8]) | (uint32_t(t[-7]) << 8) | (uint32_t(t[-6]) << 16) | (uint32_t(t[-5]) << 24);
    const uint32_t z = uint32_t(t[-4]) | (uint32_t(t[-3]) << 8) | (uint32_t(t[-2]) << 16) | (uint32_t(t[-1]) << 24);
    good = o[0] == 0x1F && o[1] == 0x8B && o[2] == 8 && c == s.checksum && z == uint32_t(s.in_len);
  }
  if (!good) jobs[i].status = kInfMismatch;
}

void launch_frame_check(const uint8_t* out, const Stream* streams, InflateJob* jobs, uint32_t n, cudaStream_t st) {
  if (n) k_frame_check<<<(n + 255) / 256, 256, 0, st>>>(out, streams, jobs, n);
}

void launch_inflate(const uint8_t* in, uint8_t* out, InflateJob* jobs, const uint32_t* order, uint32_t njobs,
                    uint32_t* counter, int sms, cudaStream_t st) {
  if (!njobs) return;
  cudaMemsetAsync(counter, 0, 4, st);
  uint32_t blocks = uint32_t(sms) * 4;  // 4 CTAs of 4 warps per SM (shared memory)
  const uint32_t need = (njobs + kInfWarps - 1) / kInfWarps;
  if (blocks > need) blocks = need;
  k_inflate<<<blocks, kInfWarps * 32, 0, st>>>(in, out, jobs, order, njobs, counter);
}

void launch_inflate_compare(const uint8_t* decoded, const uint8_t* ref, InflateJob* jobs, const uint64_t* ref_off,
                            const uint64_t* ref_len, uint32_t njobs, cudaStream_t st) {
  if (!njobs) return;
  k_inflate_compare<<<(njobs + 7) / 8, 256, 0, st>>>(decoded, ref, jobs, ref_off, ref_len, njobs);
}

}  // namespace orotb
