// kernels_inflate.cu -- DEFLATE decoding (RFC 1951) on sm_100a.
//
// Decoding a DEFLATE stream is sequential: each code's length is known only
// after the previous one is decoded.  The parallel unit across streams is the
// stream: one warp per stream, warps take streams from a counter (largest
// first, so the longest decode starts first).
//
// Inside the warp the symbols are decoded speculatively, a window of 64 bit
// offsets at a time: every lane decodes the token that would start at two of
// the offsets (a literal, the end of the block, or a length code with its
// extra bits followed by a distance code with its extra bits, at most 48
// bits), then the warp follows the chain of tokens from the window's first
// bit with one shuffle per token, writing each literal from one lane and
// copying each match with all 32 lanes (a copy of length L at distance D reads
// only bytes before the copy, out[p - D + i % D], so all lanes copy at once
// even when D < L).  Tokens off the chain are discarded; a window advances by
// the bits its chain consumed.
//
// Codes are looked up in 9-bit tables whose entries carry everything a token
// needs (code bits, base length or distance, extra bits).  Longer codes (rare
// in real data, absent from the fixed code) are resolved when the chain
// reaches them, by the canonical rule of RFC 1951 3.2.2: codes of one length
// are consecutive integers and shorter codes precede longer ones, so per
// length the code is compared against the first code and the number of codes
// of that length.  Block headers (stored lengths, the code-length code and
// the code lengths of a dynamic block) are read by lane 0.
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
constexpr uint32_t kSpan = 64;    // bit offsets decoded speculatively per window (two per lane)

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

// Lookup-table entries (0: the code is longer than kFastBits or not assigned).
//   code-length code: [0,4) code bits, [16,32) symbol
//   literal/length:   [0,4) code bits, [4,6) kind (0 literal, 1 length,
//                     2 end of block, 3 symbol 286/287), [6,11) code + extra
//                     bits, [11,14) extra bits, [16,32) literal or base length
//   distance:         [0,4) code bits, [4,8) extra bits, [8,13) code + extra
//                     bits, bit 15 symbol 30/31, [16,32) base distance
enum : uint32_t { kTabCl = 0, kTabLit = 1, kTabDist = 2 };

__device__ __forceinline__ uint32_t make_entry(uint32_t tab, uint32_t s, uint32_t n) {
  if (tab == kTabCl) return n | (s << 16);
  if (tab == kTabLit) {
    if (s < 256) return n | (n << 6) | (s << 16);
    if (s == 256) return n | (2u << 4) | (n << 6);
    if (s > 285) return n | (3u << 4) | (n << 6);
    const uint32_t x = c_len_extra[s - 257];
    return n | (1u << 4) | ((n + x) << 6) | (x << 11) | (uint32_t(c_len_base[s - 257]) << 16);
  }
  if (s > 29) return n | 0x8000u;
  const uint32_t x = c_dist_extra[s];
  return n | (x << 4) | ((n + x) << 8) | (uint32_t(c_dist_base[s]) << 16);
}

// One Huffman code: lookup table, code counts per length and the symbols in
// code order.
struct Code {
  uint32_t* fast;
  uint16_t* count;  // [16]
  uint16_t* sym;    // [nsym]
};

// Per-warp shared memory.  Output goes to global memory and to `win`: a match
// whose source lies in the window reads shared memory instead of waiting for
// the bytes this warp has just stored to come back from L2.
struct WarpMem {
  uint32_t lfast[kFast], dfast[kFast];
  uint16_t lcount[16], dcount[16];
  uint16_t lsym[288], dsym[32];
  uint16_t first[16], offs[16];  // builder scratch: first code and first index per length
  uint8_t lens[320];
  uint32_t bad;                  // builder result
  uint8_t win[kWin];             // the last kWin output bytes, at position & (kWin - 1)
};
constexpr size_t kInfSmem = sizeof(WarpMem) * kInfWarps;

// Builds `c` from code lengths lens[0..n) (all lanes); `tab` selects the
// entry layout.  Returns false for an over-subscribed set of lengths; an
// incomplete set is accepted (a code that is not assigned is reported when
// it is read).
__device__ bool build_code(const Code& c, const uint8_t* lens, uint32_t n, uint32_t tab, WarpMem& m, uint32_t lane) {
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
  // fill the lookup table: symbol i (in code order) of length l <= kFastBits
  uint32_t total = 0;
  for (int l = 1; l < 16; ++l) total += c.count[l];
  for (uint32_t i = lane; i < total; i += 32) {
    const uint32_t s = c.sym[i];
    const uint32_t l = lens[s];
    if (l > uint32_t(kFastBits)) continue;
    const uint32_t code = m.first[l] + (i - m.offs[l]);
    const uint32_t rev = __brev(code) >> (32 - l);  // codes are sent most significant bit first
    const uint32_t e = make_entry(tab, s, l);
    for (uint32_t k = rev; k < kFast; k += 1u << l) c.fast[k] = e;
  }
  __syncwarp();
  return true;
}

// LSB-first bit reader over [p, end) for the block headers (lane 0); reads
// whole aligned words (the buffers carry padding after their last byte) and
// counts bits taken past the end.
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
  // bits consumed so far
  __device__ __forceinline__ uint64_t bits() const { return pos * 8 - cnt; }
  // bytes consumed so far
  __device__ __forceinline__ uint64_t used() const { return pos - cnt / 8; }
};

// A reader positioned at bit `p` of the stream.
__device__ __forceinline__ BitIn bitin_at(const uint8_t* base, uint64_t end, uint64_t p) {
  BitIn b{base, p >> 3, end, 0, 0};
  b.refill();
  b.take(uint32_t(p & 7));
  return b;
}

// Decodes one symbol of the code-length code (lane 0).  Returns 0xFFFF for a
// code that is not assigned.
__device__ __forceinline__ uint32_t decode(BitIn& b, const Code& c) {
  b.refill();
  const uint32_t e = c.fast[uint32_t(b.buf) & (kFast - 1)];
  if (e) {
    b.take(e & 15u);
    return e >> 16;
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

// Canonical decode of the code at the low bits of `w` without the table;
// returns the symbol and its code length, or 0xFFFF for a code that is not
// assigned.
__device__ __forceinline__ uint32_t canon_peek(uint64_t w, const uint16_t* count, const uint16_t* sym, uint32_t& n) {
  int code = 0, first = 0, index = 0;
  for (int l = 1; l < 16; ++l) {
    code |= int((w >> (l - 1)) & 1u);
    const int cnt = count[l];
    if (code - first < cnt) {
      n = uint32_t(l);
      return sym[index + (code - first)];
    }
    index += cnt;
    first = (first + cnt) << 1;
    code <<= 1;
  }
  n = 0;
  return 0xFFFFu;
}

// Tokens: [0,6) bits, [6,8) kind (0 literal, 1 match, 2 end of block, 3 not
// decoded); literal: [8,16) byte; match: [8,17) length, [17,32) distance - 1;
// not decoded: [8,16) 0 = a code longer than the tables, 1 = invalid code.
constexpr uint32_t kTokSlow = 3u << 6, kTokBad = (3u << 6) | (1u << 8);

// Decodes the token at the low bits of `w` (up to 48 bits).  Without Slow a
// code missing from a table gives kTokSlow; with Slow it is decoded by the
// canonical rule.
template <bool Slow>
__device__ __forceinline__ uint32_t token(uint64_t w, const WarpMem& m) {
  uint32_t e = m.lfast[uint32_t(w) & (kFast - 1)];
  if (!(e & 15u)) {
    if (!Slow) return kTokSlow;
    uint32_t n;
    const uint32_t s = canon_peek(w, m.lcount, m.lsym, n);
    if (s == 0xFFFFu) return kTokBad;
    e = make_entry(kTabLit, s, n);
  }
  const uint32_t n = e & 15u, kind = (e >> 4) & 3u;
  if (kind != 1) return kind == 3 ? kTokBad : (n | (kind << 6) | ((e >> 16) << 8));
  const uint32_t tot = (e >> 6) & 31u, x = (e >> 11) & 7u;
  const uint32_t len = (e >> 16) + (uint32_t(w >> n) & ((1u << x) - 1u));
  const uint64_t w2 = w >> tot;
  uint32_t d = m.dfast[uint32_t(w2) & (kFast - 1)];
  if (!(d & 15u)) {
    if (!Slow) return kTokSlow;
    uint32_t dn;
    const uint32_t s = canon_peek(w2, m.dcount, m.dsym, dn);
    if (s == 0xFFFFu) return kTokBad;
    d = make_entry(kTabDist, s, dn);
  }
  if (d & 0x8000u) return kTokBad;
  const uint32_t dn = d & 15u, dx = (d >> 4) & 15u;
  const uint32_t dist = (d >> 16) + (uint32_t(w2 >> dn) & ((1u << dx) - 1u));
  return (tot + ((d >> 8) & 31u)) | (1u << 6) | (len << 8) | ((dist - 1u) << 17);
}

// Aligned input word j of a stream whose last bit is at absolute bit `endb`
// (bits at or past it read as zero).
__device__ __forceinline__ uint32_t word_at(const uint32_t* a, uint64_t j, uint64_t endb) {
  const uint64_t b0 = j * 32;
  if (b0 >= endb) return 0;
  uint32_t v = __ldg(a + j);
  if (endb - b0 < 32) v &= (1u << uint32_t(endb - b0)) - 1u;
  return v;
}

// 64 bits starting at bit `rel` (< 96) of the five words w0..w4.
__device__ __forceinline__ uint64_t bits_at(uint32_t w0, uint32_t w1, uint32_t w2, uint32_t w3, uint32_t w4,
                                            uint32_t rel) {
  const uint32_t q = rel >> 5, s = rel & 31u;
  const uint32_t x0 = q == 0 ? w0 : q == 1 ? w1 : w2;
  const uint32_t x1 = q == 0 ? w1 : q == 1 ? w2 : w3;
  const uint32_t x2 = q == 0 ? w2 : q == 1 ? w3 : w4;
  return (uint64_t(__funnelshift_r(x1, x2, s)) << 32) | __funnelshift_r(x0, x1, s);
}

}  // namespace

// status: kInfOk, kInfData (corrupt), kInfOutput (output full), kInfInput (input exhausted)
__global__ void __launch_bounds__(kInfWarps * 32) k_inflate(const uint8_t* __restrict__ in, uint8_t* __restrict__ out,
                                                 InflateJob* jobs, const uint32_t* __restrict__ order, uint32_t njobs,
                                                 uint32_t* counter) {
  extern __shared__ __align__(16) uint8_t inf_smem[];
  const uint32_t lane = threadIdx.x & 31, wid = threadIdx.x >> 5;
  WarpMem& m = reinterpret_cast<WarpMem*>(inf_smem)[wid];
  const Code lit{m.lfast, m.lcount, m.lsym}, dst{m.dfast, m.dcount, m.dsym};
  for (;;) {
    uint32_t k = 0;
    if (lane == 0) k = atomicAdd(counter, 1u);
    k = __shfl_sync(kAll, k, 0);
    if (k >= njobs) break;
    InflateJob* jp = jobs + order[k];
    const InflateJob job = *jp;
    uint8_t* o = out + job.out_off;
    const uint8_t* base = in + job.in_off;
    // the stream as aligned words: its first bit is bit s0 of word 0
    const uint32_t* aw = reinterpret_cast<const uint32_t*>(reinterpret_cast<uint64_t>(base) & ~uint64_t(3));
    const uint64_t s0 = (reinterpret_cast<uint64_t>(base) & 3) * 8;
    const uint64_t endb = s0 + job.in_len * 8;
    uint64_t P = 0;   // bits consumed
    uint64_t op = 0;  // output position
    int32_t status = kInfOk;
    bool last = false;
    while (!last && status == kInfOk) {
      // block header (lane 0 reads, every lane learns the type)
      BitIn b{base, 0, job.in_len, 0, 0};
      uint32_t hdr = 0;
      if (lane == 0) {
        b = bitin_at(base, job.in_len, P);
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
        }
        len = __shfl_sync(kAll, len, 0);
        ok = __shfl_sync(kAll, ok, 0);
        src = __shfl_sync(kAll, src, 0);
        if (!ok) { status = kInfData; break; }
        if (src + len > job.in_len) { status = kInfInput; break; }
        if (op + len > job.out_cap) { status = kInfOutput; break; }
        const uint8_t* s = base + src;
        for (uint32_t i = lane; i < len; i += 32) {
          const uint8_t v = s[i];
          o[op + i] = v;
          m.win[(op + i) & (kWin - 1)] = v;
        }
        op += len;
        P = (src + len) * 8;
        __syncwarp();
        continue;
      }
      // Huffman block: tables
      if (type == 1) {
        for (uint32_t i = lane; i < 320; i += 32) m.lens[i] = i < 144 ? 8 : i < 256 ? 9 : i < 280 ? 7 : i < 288 ? 8 : 5;
        __syncwarp();
        build_code(lit, m.lens, 288, kTabLit, m, lane);
        build_code(dst, m.lens + 288, 30, kTabDist, m, lane);
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
        if (hlit > 286 || hdist > 30 || !build_code(lit, m.lens + 300, 19, kTabCl, m, lane)) err = 1;
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
        if (!build_code(lit, m.lens, 288, kTabLit, m, lane) || !build_code(dst, m.lens + 288, 30, kTabDist, m, lane)) {
          status = kInfData;
          break;
        }
      }
      P = __shfl_sync(kAll, b.bits(), 0);
      // symbols, a window of kSpan bit offsets at a time
      bool block_end = false;
      while (!block_end && status == kInfOk) {
        const uint64_t A = s0 + P;  // the window's first bit, counted from aw
        const uint64_t q = A >> 5;
        const uint32_t w0 = word_at(aw, q, endb), w1 = word_at(aw, q + 1, endb), w2 = word_at(aw, q + 2, endb),
                       w3 = word_at(aw, q + 3, endb), w4 = word_at(aw, q + 4, endb);
        const uint32_t r = uint32_t(A & 31);
        const uint32_t t_lo = token<false>(bits_at(w0, w1, w2, w3, w4, r + lane), m);
        const uint32_t t_hi = token<false>(bits_at(w0, w1, w2, w3, w4, r + lane + 32), m);
        uint32_t cur = 0;  // offset of the next token on the chain
        uint32_t nl = 0;   // literals decoded but not written yet: lane j holds the j-th in lb
        uint32_t lb = 0;
        // bits of the stream from the window's first bit on (capped: every
        // token on the chain ends before bit kSpan + 48)
        const uint32_t lim = A >= endb ? 0u : endb - A >= 256 ? 256u : uint32_t(endb - A);
        while (cur < kSpan) {
          uint32_t t = __shfl_sync(kAll, cur < 32 ? t_lo : t_hi, cur & 31);
          uint32_t tb = t & 63u;
          if (((t >> 6) & 3u) == 0 && cur + tb <= lim && nl < 32) {  // a literal: keep it in lane nl
            if (lane == nl) lb = t >> 8;
            ++nl;
            cur += tb;
            continue;
          }
          // anything else writes the pending literals first
          if (nl) {
            if (op + nl > job.out_cap) { status = kInfOutput; break; }
            if (lane < nl) {
              o[op + lane] = uint8_t(lb);
              m.win[(op + lane) & (kWin - 1)] = uint8_t(lb);
            }
            op += nl;
            nl = 0;
          }
          if (((t >> 6) & 3u) == 3u) {
            if (t != kTokSlow) { status = kInfData; break; }
            t = token<true>(bits_at(w0, w1, w2, w3, w4, r + cur), m);
            if (t == kTokBad) { status = kInfData; break; }
            tb = t & 63u;
          }
          const uint32_t kind = (t >> 6) & 3u;
          if (cur + tb > lim) { status = kInfInput; break; }
          cur += tb;
          if (kind == 0) {
            if (lane == 0) lb = t >> 8;
            nl = 1;
            continue;
          }
          if (kind == 2) { block_end = true; break; }
          const uint32_t len = (t >> 8) & 511u, dist = (t >> 17) + 1u;
          if (dist > op) { status = kInfData; break; }
          if (op + len > job.out_cap) { status = kInfOutput; break; }
          __syncwarp();
          // sources lie before op; in the window unless the copy's own writes
          // could reach the slots other lanes read (dist + len > kWin)
          const bool in_win = dist + len <= kWin;
          for (uint32_t i = lane; i < len; i += 32) {
            const uint64_t src = op - dist + (i < dist ? i : i % dist);
            const uint8_t v = in_win ? m.win[src & (kWin - 1)] : o[src];
            o[op + i] = v;
            m.win[(op + i) & (kWin - 1)] = v;
          }
          __syncwarp();
          op += len;
        }
        if (nl && status == kInfOk) {
          if (op + nl > job.out_cap) {
            status = kInfOutput;
          } else {
            if (lane < nl) {
              o[op + lane] = uint8_t(lb);
              m.win[(op + lane) & (kWin - 1)] = uint8_t(lb);
            }
            op += nl;
          }
        }
        __syncwarp();
        P += cur;
      }
      __syncwarp();
    }
    if (lane == 0) {
      const uint64_t used = (P + 7) >> 3;
      if (status == kInfOk && used > job.in_len) status = kInfInput;
      jp->out_len = op;
      jp->in_used = status == kInfOk ? used : 0;
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
  static std::atomic<bool> attr_set[64];
  const int ds = device_slot();
  if (!attr_set[ds].load(std::memory_order_relaxed)) {
    if (cudaFuncSetAttribute(k_inflate, cudaFuncAttributeMaxDynamicSharedMemorySize, int(kInfSmem)) == cudaSuccess)
      attr_set[ds].store(true, std::memory_order_relaxed);
  }
  k_inflate<<<blocks, kInfWarps * 32, kInfSmem, st>>>(in, out, jobs, order, njobs, counter);
}

void launch_inflate_compare(const uint8_t* decoded, const uint8_t* ref, InflateJob* jobs, const uint64_t* ref_off,
                            const uint64_t* ref_len, uint32_t njobs, cudaStream_t st) {
  if (!njobs) return;
  k_inflate_compare<<<(njobs + 7) / 8, 256, 0, st>>>(decoded, ref, jobs, ref_off, ref_len, njobs);
}

}  // namespace orotb
