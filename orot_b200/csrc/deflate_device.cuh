// deflate_device.cuh -- device helpers for the sm_100a DEFLATE kernels.
#pragma once
#include <cstdint>

namespace orotb {

// ---------------------------------------------------------------- input access
// Segment bytes are addressed through 4-byte words so that every load is an
// aligned 32-bit read-only load; `boff` is the byte offset of the segment's
// first byte inside words[0].  The input arena carries 64 bytes of padding, so
// reading one word past the last used byte is always in bounds.
struct SegBytes {
  const uint32_t* __restrict__ w;
  uint32_t boff;
  __device__ __forceinline__ uint32_t load4(uint32_t p) const {
    const uint32_t q = p + boff;
    const uint32_t lo = __ldg(w + (q >> 2)), hi = __ldg(w + (q >> 2) + 1);
    return __funnelshift_r(lo, hi, (q & 3) * 8);
  }
  __device__ __forceinline__ uint32_t byte(uint32_t p) const {
    const uint32_t q = p + boff;
    return (__ldg(w + (q >> 2)) >> ((q & 3) * 8)) & 0xFFu;
  }
};

// Common-prefix length of the bytes at p and q, at most cap (cap <= 258).
__device__ __forceinline__ uint32_t lcp_capped(const SegBytes& s, uint32_t p, uint32_t q, uint32_t cap) {
  uint32_t n = 0;
  while (n < cap) {
    const uint32_t x = s.load4(p + n) ^ s.load4(q + n);
    if (x) { n += (__ffs(x) - 1) >> 3; break; }
    n += 4;
  }
  return n < cap ? n : cap;
}

// ---------------------------------------------------------------- fixed Huffman
// RFC 1951 section 3.2.6 fixed code, bit-reversed for LSB-first packing.
__device__ __forceinline__ uint32_t rev_bits(uint32_t code, uint32_t len) { return __brev(code) >> (32 - len); }

__device__ __forceinline__ void fixed_literal(uint32_t b, uint32_t& bits, uint32_t& nb) {
  if (b < 144) { bits = rev_bits(0x30u + b, 8); nb = 8; }
  else { bits = rev_bits(0x190u + (b - 144), 9); nb = 9; }
}

// Length 3..258 -> code index 0..28, extra-bit count and value (RFC 1951 3.2.5).
__device__ __forceinline__ void length_code(uint32_t len, uint32_t& li, uint32_t& ne, uint32_t& ev) {
  if (len == 258) { li = 28; ne = 0; ev = 0; return; }
  const uint32_t d = len - 3;
  if (d < 8) { li = d; ne = 0; ev = 0; return; }
  const uint32_t e = (31 - __clz(d)) - 2;
  li = 4 * e + (d >> e);
  ne = e;
  ev = d & ((1u << e) - 1);
}
// Distance 1..32768 -> code 0..29, extra-bit count and value.
__device__ __forceinline__ void dist_code(uint32_t dist, uint32_t& dc, uint32_t& ne, uint32_t& ev) {
  const uint32_t d = dist - 1;
  if (d < 4) { dc = d; ne = 0; ev = 0; return; }
  const uint32_t e = (31 - __clz(d)) - 1;
  dc = 2 * e + 2 + ((d >> e) & 1);
  ne = e;
  ev = d & ((1u << e) - 1);
}

// Whole fixed-Huffman match token (<= 31 bits) packed LSB-first.
__device__ __forceinline__ void fixed_match(uint32_t len, uint32_t dist, uint32_t& bits, uint32_t& nb) {
  uint32_t li, le, lv, dc, de, dv;
  length_code(len, li, le, lv);
  dist_code(dist, dc, de, dv);
  const uint32_t sym = 257 + li;
  uint32_t c, cl;
  if (sym <= 279) { c = sym - 256; cl = 7; } else { c = 0xC0u + (sym - 280); cl = 8; }
  bits = rev_bits(c, cl) | (lv << cl);
  nb = cl + le;
  bits |= rev_bits(dc, 5) << nb;
  nb += 5;
  bits |= dv << nb;
  nb += de;
}

// ---------------------------------------------------------------- CRC-32 algebra
// Polynomials over GF(2) in the reflected representation of the IEEE CRC-32
// (bit 31 holds the coefficient of x^0).  crc(A||B) = (crc(A) * x^(8|B|)) +
// crc(B) for the unconditioned register; the conditioning (~init, ~result)
// is applied around it.  This is the standard combination identity of
// cyclic codes.
constexpr uint32_t kCrcPoly = 0xEDB88320u;

__host__ __device__ inline uint32_t gf2_mulmod(uint32_t a, uint32_t b) {
  uint32_t p = 0;
  for (int i = 0; i < 32; ++i) {
    if (a & 0x80000000u) p ^= b;
    a <<= 1;
    b = (b & 1u) ? (b >> 1) ^ kCrcPoly : (b >> 1);
  }
  return p;
}

// x^(2^k) mod P for k = 0..63, filled by the host.
struct CrcPowers { uint32_t x2k[64]; };

__host__ __device__ inline uint32_t xpow8n(const CrcPowers& t, uint64_t n) {
  uint32_t r = 0x80000000u;  // the polynomial 1
  int k = 3;                 // x^(8n) = prod over set bits of n of x^(2^(k))
  while (n && k < 64) {
    if (n & 1) r = gf2_mulmod(r, t.x2k[k]);
    n >>= 1;
    ++k;
  }
  return r;
}

}  // namespace orotb
