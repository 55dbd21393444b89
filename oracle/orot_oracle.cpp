// orot_oracle.cpp -- CPU restatement of orot's DEFLATE *compress* path.
//
// TEST INFRASTRUCTURE ONLY.  This file is the parity checker for the CUDA
// engine in orot_b200/: only tests/, __graft_entry__.smoke() and bench.py's
// CPU-baseline leg may load it.  The product never links or calls it.
//
// Every function restates the reference algorithm named in its comment
// (paths are relative to the daramkun/orot source tree).  One deliberate
// difference: when a Huffman tree is deeper than the code-length limit the
// reference clamps the depths and emits an over-subscribed (invalid) code
// (src/deflate/huffman.cpp:307-356).  Here the limit is enforced with the
// bit-count adjustment of ITU-T T.81 (JPEG) Annex K.3, which always yields a
// complete prefix code.  A second difference: the binary-tree search of
// levels 10-12 (src/deflate/lz77.cpp:309-316) starts each comparison after
// min(len_left, len_right) bytes it assumes equal; the covered-position
// inserts of lz77.cpp:428-431 link nodes without keeping the tree ordered, so
// that assumption fails and the reference emits matches whose bytes differ
// (its streams then inflate to different data).  Here every comparison starts
// at byte 0.  oracle_set_mode(0) restores both reference behaviours so byte
// identity with the reference can be tested.
//
// Exported C ABI (loaded with ctypes by the tests):
//   oracle_crc32 / oracle_adler32            checksums
//   oracle_compress_bound / oracle_compress   whole-buffer API
//   oracle_parallel_compress                  pigz-style API (single thread)
//   oracle_lz77                               token stream of one segment
//   oracle_huffman_lengths                    code-length builder
//   oracle_set_mode / oracle_limiter_events
//   oracle_block_types                        block types of a raw stream (an
//                                             RFC 1951 walker, test helper)

#include <algorithm>
#include <cstdint>
#include <cstring>
#include <vector>

namespace {

// ---------------------------------------------------------------- tables
// RFC 1951 section 3.2.5 length/distance alphabets (the same constants the
// reference holds in src/deflate/huffman.cpp:15-32).
const uint16_t kLenBase[29] = {3, 4, 5, 6, 7, 8, 9, 10, 11, 13, 15, 17, 19, 23, 27, 31,
                               35, 43, 51, 59, 67, 83, 99, 115, 131, 163, 195, 227, 258};
const uint8_t kLenExtra[29] = {0, 0, 0, 0, 0, 0, 0, 0, 1, 1, 1, 1, 2, 2, 2, 2,
                               3, 3, 3, 3, 4, 4, 4, 4, 5, 5, 5, 5, 0};
const uint16_t kDistBase[30] = {1, 2, 3, 4, 5, 7, 9, 13, 17, 25, 33, 49, 65, 97, 129,
                                193, 257, 385, 513, 769, 1025, 1537, 2049, 3073, 4097,
                                6145, 8193, 12289, 16385, 24577};
const uint8_t kDistExtra[30] = {0, 0, 0, 0, 1, 1, 2, 2, 3, 3, 4, 4, 5, 5, 6,
                                6, 7, 7, 8, 8, 9, 9, 10, 10, 11, 11, 12, 12, 13, 13};

int len_code(int len) {  // 3..258 -> 0..28  (huffman.cpp:109-113)
  int c = 0;
  while (c < 28 && kLenBase[c + 1] <= len) ++c;
  if (len == 258) c = 28;
  return c;
}
int dist_code(int dist) {  // 1..32768 -> 0..29  (huffman.cpp:115-119)
  int c = 0;
  while (c < 29 && kDistBase[c + 1] <= dist) ++c;
  return c;
}

constexpr int kLitLenSyms = 288, kDistSyms = 32, kClSyms = 19;
constexpr int kMaxBits = 15, kMaxClBits = 7;

int g_mode = 1;                // 1 = corrected, 0 = reference defects kept
long g_limiter_events = 0;     // trees that exceeded their length limit

// ---------------------------------------------------------------- checksums
// Sarwate table CRC-32, reflected polynomial 0xEDB88320, pre/post inverted
// (src/simd/simd_detect.cpp:33-50).
uint32_t crc_table[256];
bool crc_ready = false;
void crc_init() {
  for (uint32_t i = 0; i < 256; ++i) {
    uint32_t c = i;
    for (int k = 0; k < 8; ++k) c = (c & 1) ? (c >> 1) ^ 0xEDB88320u : (c >> 1);
    crc_table[i] = c;
  }
  crc_ready = true;
}
uint32_t crc32(uint32_t crc, const uint8_t* p, size_t n) {
  if (!crc_ready) crc_init();
  crc = ~crc;
  for (size_t i = 0; i < n; ++i) crc = crc_table[(crc ^ p[i]) & 0xFF] ^ (crc >> 8);
  return ~crc;
}
// Adler-32 modulo 65521, reduced every 5552 bytes (simd_detect.cpp:52-70).
uint32_t adler32(uint32_t a, const uint8_t* p, size_t n) {
  uint32_t s1 = a & 0xFFFF, s2 = a >> 16;
  while (n) {
    size_t k = n < 5552 ? n : 5552;
    for (size_t i = 0; i < k; ++i) { s1 += p[i]; s2 += s1; }
    s1 %= 65521u; s2 %= 65521u;
    p += k; n -= k;
  }
  return (s2 << 16) | s1;
}

// ---------------------------------------------------------------- LZ77
// Token word: bit 31 = match, bits 24:16 = length, bits 15:0 = distance;
// literal = byte value (src/deflate/lz77.hpp:26-43).
inline uint32_t tok_lit(uint8_t b) { return b; }
inline uint32_t tok_match(int len, int dist) { return 0x80000000u | (uint32_t(len) << 16) | uint32_t(dist); }

struct Lz77Cfg { int max_chain, nice_len, lazy_depth; bool bt4, fast; int hash_bits, miss_limit; };
// Per-level table of src/deflate/lz77.cpp:18-32 (values must be equal for parity).
const Lz77Cfg kCfg[13] = {
    {0, 0, 0, false, false, 16, 8},      {1, 32, 0, false, true, 12, 8},
    {16, 64, 0, false, true, 14, 8},     {32, 128, 0, false, true, 14, 8},
    {64, 128, 1, false, false, 16, 5},   {128, 128, 1, false, false, 16, 5},
    {128, 258, 1, false, false, 16, 5},  {256, 258, 2, false, false, 16, 6},
    {512, 258, 2, false, false, 16, 6},  {768, 258, 3, false, false, 16, 6},
    {1024, 258, 4, true, false, 16, 8},  {2048, 258, 4, true, false, 16, 8},
    {4096, 258, 4, true, false, 16, 8}};
Lz77Cfg cfg_for(int level) { return kCfg[level < 0 ? 0 : level > 12 ? 12 : level]; }

constexpr int kWin = 32768, kWinMask = kWin - 1;

inline uint32_t load32(const uint8_t* p) { uint32_t v; std::memcpy(&v, p, 4); return v; }
inline uint32_t hash4(const uint8_t* p, int bits) { return (load32(p) * 0x9E3779B1u) >> (32 - bits); }

// Common-prefix length of a and b, at most max_len (simd_detect.cpp:12-31).
inline int common_prefix(const uint8_t* a, const uint8_t* b, int max_len) {
  int n = 0;
  while (n < max_len && a[n] == b[n]) ++n;
  return n;
}

struct State {
  std::vector<uint32_t> head, prev, right;
  explicit State(int hash_bits) : head(size_t(1) << hash_bits, 0), prev(kWin, 0), right(kWin, 0) {}
};

// Chain search of the standard path (lz77.cpp:66-156).  The 8-byte and
// best_len-byte rejects of the reference only skip candidates that cannot
// beat best_len, so they are omitted; the 4-byte reject and its
// consecutive-miss abort do change results and are kept.
int chain_search(const uint8_t* s, int pos, int n, const State& st, int max_chain,
                 const Lz77Cfg& c, int& best_dist) {
  const int max_match = std::min(258, n - pos);
  if (max_match < 3 || n - pos < 4) return 0;
  int best = 2;
  best_dist = 0;
  uint32_t cur = st.head[hash4(s + pos, 16)];
  int steps = max_chain, misses = 0;
  while (steps-- > 0 && cur != 0) {
    const int dist = (pos - int(cur)) & kWinMask;
    if (dist == 0) break;
    const uint8_t* cand = s + pos - dist;
    bool miss = (pos + 3 < n) ? (load32(cand) != load32(s + pos)) : (cand[0] != s[pos]);
    if (miss) {
      if (++misses >= c.miss_limit) break;
      cur = st.prev[cur & kWinMask];
      continue;
    }
    misses = 0;
    const int len = common_prefix(s + pos, cand, max_match);
    if (len > best) {
      best = len;
      best_dist = dist;
      if (len >= c.nice_len) break;
    }
    cur = st.prev[cur & kWinMask];
  }
  return best;
}

inline void insert_chain(const uint8_t* s, int pos, int n, State& st) {  // lz77.cpp:199-207
  if (pos + 4 > n) return;
  const uint32_t h = hash4(s + pos, 16);
  st.prev[pos & kWinMask] = st.head[h];
  st.head[h] = uint32_t(pos);
}
inline void insert_bt(const uint8_t* s, int pos, int n, State& st) {  // lz77.cpp:213-222
  if (pos + 4 > n) return;
  const uint32_t h = hash4(s + pos, 16);
  st.prev[pos & kWinMask] = st.head[h];
  st.right[pos & kWinMask] = 0;
  st.head[h] = uint32_t(pos);
}

// Binary-tree search + insert of levels 10-12 (lz77.cpp:235-350).
int bt4_search(const uint8_t* s, int pos, int n, State& st, const Lz77Cfg& c, int& best_dist) {
  const int max_match = std::min(258, n - pos);
  if (max_match < 3 || n - pos < 4) {
    if (pos + 4 <= n) insert_bt(s, pos, n, st);
    return 0;
  }
  int best = 2;
  best_dist = 0;
  const uint32_t h = hash4(s + pos, 16);
  uint32_t cur = st.head[h];
  st.head[h] = uint32_t(pos);
  uint32_t* lslot = &st.prev[pos & kWinMask];
  uint32_t* rslot = &st.right[pos & kWinMask];
  int known_l = 0, known_r = 0, steps = c.max_chain, misses = 0;
  while (steps-- > 0 && cur != 0) {
    const int dist = (pos - int(cur)) & kWinMask;
    if (dist == 0) break;
    const uint8_t* cand = s + pos - dist;
    if (cand[0] != s[pos]) {
      if (++misses >= c.miss_limit) { *lslot = 0; *rslot = 0; return best; }
      if (cand[0] < s[pos]) {
        *lslot = cur; lslot = &st.right[cur & kWinMask]; cur = st.right[cur & kWinMask]; known_l = 0;
      } else {
        *rslot = cur; rslot = &st.prev[cur & kWinMask]; cur = st.prev[cur & kWinMask]; known_r = 0;
      }
      continue;
    }
    misses = 0;
    const int skip = g_mode == 0 ? std::min(known_l, known_r) : 0;
    int len = skip;
    if (skip < max_match) len = skip + common_prefix(s + pos + skip, cand + skip, max_match - skip);
    if (len > best) {
      best = len;
      best_dist = dist;
      if (len >= c.nice_len) {
        *lslot = st.prev[cur & kWinMask];
        *rslot = st.right[cur & kWinMask];
        return best;
      }
    }
    if (pos + len < n && cand[len] < s[pos + len]) {
      *lslot = cur; lslot = &st.right[cur & kWinMask]; cur = st.right[cur & kWinMask]; known_l = len;
    } else {
      *rslot = cur; rslot = &st.prev[cur & kWinMask]; cur = st.prev[cur & kWinMask]; known_r = len;
    }
  }
  *lslot = 0;
  *rslot = 0;
  return best;
}

// One LZ77 pass over one segment with a fresh dictionary (lz77.cpp:352-499).
size_t lz77(const uint8_t* s, size_t n_in, uint32_t* out, int level) {
  const Lz77Cfg c = cfg_for(level);
  if (n_in == 0) return 0;
  if (c.max_chain == 0) {
    for (size_t i = 0; i < n_in; ++i) out[i] = tok_lit(s[i]);
    return n_in;
  }
  const int n = int(n_in);
  State st(c.hash_bits);
  size_t nt = 0;
  int pos = 0;
  if (c.fast) {
    // Greedy, head-only lookup; every position is hashed (lz77.cpp:378-406).
    while (pos < n) {
      if (pos + 3 > n || n - pos < 4) { out[nt++] = tok_lit(s[pos++]); continue; }
      const int max_match = std::min(258, n - pos);
      const uint32_t h = hash4(s + pos, c.hash_bits);
      const uint32_t cand = st.head[h];
      st.head[h] = uint32_t(pos);
      int len = 0, dist = 0;
      if (cand != 0) {
        dist = (pos - int(cand)) & kWinMask;
        if (dist != 0 && s[cand] == s[pos]) len = common_prefix(s + pos, s + pos - dist, max_match);
      }
      if (len < 3) { out[nt++] = tok_lit(s[pos++]); continue; }
      out[nt++] = tok_match(len, dist);
      const int end = pos + len;
      for (int i = pos + 1; i < end && i + 4 <= n; ++i) st.head[hash4(s + i, c.hash_bits)] = uint32_t(i);
      pos = end;
    }
  } else if (c.bt4) {
    while (pos < n) {
      if (pos + 3 > n) { out[nt++] = tok_lit(s[pos++]); continue; }
      int dist = 0;
      const int len = bt4_search(s, pos, n, st, c, dist);
      if (len < 3) { out[nt++] = tok_lit(s[pos++]); continue; }
      out[nt++] = tok_match(len, dist);
      const int end = pos + len;
      for (int i = pos + 1; i < end && i + 3 <= n; ++i) insert_bt(s, i, n, st);
      pos = end;
    }
  } else {
    // Chain search with lazy evaluation; lookahead searches use half the
    // chain budget and need a gain of two bytes (lz77.cpp:435-495).
    const int lazy_chain = std::max(1, c.max_chain >> 1);
    while (pos < n) {
      if (pos + 3 > n) { out[nt++] = tok_lit(s[pos++]); continue; }
      int dist = 0;
      int len = chain_search(s, pos, n, st, c.max_chain, c, dist);
      if (len < 3) {
        insert_bt(s, pos, n, st);
        out[nt++] = tok_lit(s[pos++]);
        continue;
      }
      int lazy = c.lazy_depth;
      while (lazy > 0 && pos + len + 1 < n && pos + 4 <= n) {
        int nd = 0;
        const int nl = chain_search(s, pos + 1, n, st, lazy_chain, c, nd);
        if (nl > len + 1) {
          insert_bt(s, pos, n, st);
          out[nt++] = tok_lit(s[pos++]);
          len = nl;
          dist = nd;
          --lazy;
        } else {
          break;
        }
      }
      out[nt++] = tok_match(len, dist);
      const int end = pos + len;
      for (int i = pos; i < end && i + 3 <= n; ++i) insert_chain(s, i, n, st);
      pos = end;
    }
  }
  return nt;
}

// ---------------------------------------------------------------- Huffman
// Code lengths from frequencies (src/deflate/huffman.cpp:180-368): symbols
// with non-zero frequency are ordered by std::sort on frequency, a binary
// heap (std::make_heap / pop_heap / push_heap, min on weight) merges the two
// lightest nodes, and each leaf's depth is its length.  A single used symbol
// gets length 1.
void huffman_lengths(const uint32_t* freq, int nsym, uint8_t* lens, int max_bits) {
  std::memset(lens, 0, size_t(nsym));
  int act[kLitLenSyms];
  int n = 0;
  for (int i = 0; i < nsym; ++i)
    if (freq[i]) act[n++] = i;
  if (n == 0) return;
  if (n == 1) { lens[act[0]] = 1; return; }
  std::sort(act, act + n, [&](int a, int b) { return freq[a] < freq[b]; });
  struct Node { uint64_t w; int l, r; };
  Node nodes[2 * kLitLenSyms];
  int heap[2 * kLitLenSyms];
  for (int i = 0; i < n; ++i) { nodes[i] = {freq[act[i]], -1, i}; heap[i] = i; }
  int nn = n, nh = n;
  auto gt = [&](int a, int b) { return nodes[a].w > nodes[b].w; };
  std::make_heap(heap, heap + nh, gt);
  while (nh > 1) {
    std::pop_heap(heap, heap + nh, gt);
    const int a = heap[--nh];
    std::pop_heap(heap, heap + nh, gt);
    const int b = heap[--nh];
    nodes[nn] = {nodes[a].w + nodes[b].w, a, b};
    heap[nh++] = nn++;
    std::push_heap(heap, heap + nh, gt);
  }
  int depth[2 * kLitLenSyms];
  int maxd = 0;
  depth[nn - 1] = 0;
  for (int i = nn - 1; i >= n; --i) {  // parents are created after children
    depth[nodes[i].l] = depth[i] + 1;
    depth[nodes[i].r] = depth[i] + 1;
  }
  for (int i = 0; i < n; ++i) maxd = std::max(maxd, depth[i]);
  if (maxd <= max_bits) {
    for (int i = 0; i < n; ++i) lens[act[nodes[i].r]] = uint8_t(depth[i]);
    return;
  }
  ++g_limiter_events;
  if (g_mode == 0) {  // reference behaviour: clamp (over-subscribed)
    for (int i = 0; i < n; ++i) lens[act[nodes[i].r]] = uint8_t(std::min(depth[i], max_bits));
    return;
  }
  // ITU-T T.81 Annex K.3 (Figure K.3, "Adjust_BITS"): move pairs of codes
  // from too-long lengths up one level by splitting a shorter code.
  int count[64] = {0};
  for (int i = 0; i < n; ++i) ++count[depth[i]];
  for (int i = maxd; i > max_bits; --i) {
    while (count[i] > 0) {
      int j = i - 2;
      while (count[j] == 0) --j;
      count[i] -= 2;
      count[i - 1] += 1;
      count[j + 1] += 2;
      count[j] -= 1;
    }
  }
  // Longest codes go to the least frequent symbols: act[] is ascending by
  // frequency, so walk it from the front while handing out lengths from the
  // longest down.
  int idx = 0;
  for (int l = max_bits; l >= 1; --l)
    for (int k = 0; k < count[l]; ++k) lens[act[idx++]] = uint8_t(l);
}

// Canonical codes, bit-reversed for LSB-first output (huffman.cpp:374-397).
void canonical_codes(const uint8_t* lens, int nsym, uint16_t* codes) {
  int bl[kMaxBits + 1] = {0};
  for (int i = 0; i < nsym; ++i)
    if (lens[i]) ++bl[lens[i]];
  uint16_t next[kMaxBits + 2] = {0};
  uint16_t code = 0;  // 16-bit arithmetic, as in the reference
  for (int b = 1; b <= kMaxBits; ++b) { code = uint16_t((code + bl[b - 1]) << 1); next[b] = code; }
  for (int i = 0; i < nsym; ++i) {
    if (!lens[i]) { codes[i] = 0; continue; }
    uint32_t c = next[lens[i]]++, r = 0;
    for (int k = 0; k < lens[i]; ++k) { r = (r << 1) | (c & 1); c >>= 1; }
    codes[i] = uint16_t(r);
  }
}

void fixed_lengths(uint8_t* ll, uint8_t* dl) {  // RFC 1951 section 3.2.6
  for (int i = 0; i < 288; ++i) ll[i] = i < 144 ? 8 : i < 256 ? 9 : i < 280 ? 7 : 8;
  for (int i = 0; i < 32; ++i) dl[i] = 5;
}

// ---------------------------------------------------------------- bit writer
// LSB-first bit packing with zero padding at flush (src/deflate/bit_writer.hpp).
struct Bits {
  uint8_t* dst;
  size_t cap, pos = 0;
  uint64_t acc = 0;
  int cnt = 0;
  bool overflow = false;
  Bits(uint8_t* d, size_t c) : dst(d), cap(c) {}
  void put_byte(uint8_t b) { if (pos < cap) dst[pos] = b; else overflow = true; ++pos; }
  void put(uint32_t v, int n) {
    if (n == 0) return;
    acc |= uint64_t(v & ((n == 32) ? 0xFFFFFFFFu : ((1u << n) - 1))) << cnt;
    cnt += n;
    while (cnt >= 8) { put_byte(uint8_t(acc)); acc >>= 8; cnt -= 8; }
  }
  void align() { if (cnt & 7) put(0, 8 - (cnt & 7)); }
  uint64_t bit_pos() const { return uint64_t(pos) * 8 + uint64_t(cnt); }
};

// ---------------------------------------------------------------- blocks
struct Stats { uint32_t lit[kLitLenSyms]; uint32_t dist[kDistSyms]; };

void block_stats(const uint32_t* t, size_t nt, Stats& s) {  // deflate_block.cpp:21-44
  std::memset(&s, 0, sizeof s);
  for (size_t i = 0; i < nt; ++i) {
    if (t[i] >> 31) {
      ++s.lit[257 + len_code((t[i] >> 16) & 0x1FF)];
      ++s.dist[dist_code(t[i] & 0xFFFF)];
    } else {
      ++s.lit[t[i] & 0xFF];
    }
  }
  ++s.lit[256];
}

uint64_t cost_with(const Stats& s, const uint8_t* ll, const uint8_t* dl) {
  uint64_t b = 0;
  for (int i = 0; i < kLitLenSyms; ++i) b += uint64_t(ll[i]) * s.lit[i];
  for (int i = 0; i < kDistSyms; ++i) b += uint64_t(dl[i]) * s.dist[i];
  for (int i = 0; i < 29; ++i) b += uint64_t(kLenExtra[i]) * s.lit[257 + i];
  for (int i = 0; i < 30; ++i) b += uint64_t(kDistExtra[i]) * s.dist[i];
  return b;
}
// estimate_fixed_bits (deflate_block.cpp:50-70)
uint64_t fixed_cost(const Stats& s) {
  uint8_t ll[288], dl[32];
  fixed_lengths(ll, dl);
  return 3 + cost_with(s, ll, dl);
}
// estimate_dynamic_bits_from_lens: flat header guess (deflate_block.cpp:74-92)
uint64_t dynamic_cost(const Stats& s, const uint8_t* ll, const uint8_t* dl) {
  return 3 + 5 + 5 + 4 + 19 * 3 + 3 * (kLitLenSyms + kDistSyms) + cost_with(s, ll, dl);
}

void emit_stored(const uint8_t* raw, size_t len, Bits& bw, bool last) {  // deflate_block.cpp:107-132
  size_t off = 0;
  do {
    const size_t k = std::min<size_t>(len - off, 65535);
    bw.put((last && off + k == len) ? 1 : 0, 1);
    bw.put(0, 2);
    bw.align();
    bw.put(uint32_t(k), 16);
    bw.put(uint32_t(~k) & 0xFFFF, 16);
    for (size_t i = 0; i < k; ++i) bw.put_byte(raw[off + i]);
    off += k;
    if (k == 0) break;
  } while (off < len);
}

void emit_tokens(const uint32_t* t, size_t nt, const uint8_t* ll, const uint16_t* lc,
                 const uint8_t* dl, const uint16_t* dc, Bits& bw) {  // deflate_block.cpp:138-160
  for (size_t i = 0; i < nt; ++i) {
    if (!(t[i] >> 31)) {
      const int b = t[i] & 0xFF;
      bw.put(lc[b], ll[b]);
      continue;
    }
    const int len = (t[i] >> 16) & 0x1FF, dist = t[i] & 0xFFFF;
    const int li = len_code(len), di = dist_code(dist);
    bw.put(lc[257 + li], ll[257 + li]);
    bw.put(uint32_t(len - kLenBase[li]), kLenExtra[li]);
    bw.put(dc[di], dl[di]);
    bw.put(uint32_t(dist - kDistBase[di]), kDistExtra[di]);
  }
  bw.put(lc[256], ll[256]);
}

// Run-length coding of the code lengths and the code-length code
// (deflate_block.cpp:196-290).  Runs are capped at 138; zero runs of 3..10
// use symbol 17, 11..138 symbol 18; a non-zero run of 4 or more is sent as
// the length itself plus one symbol 16 repeating up to 6 copies.
void encode_code_lengths(const uint8_t* ll, int hlit, const uint8_t* dl, int hdist, Bits& bw) {
  uint8_t seq[kLitLenSyms + kDistSyms];
  std::memcpy(seq, ll, size_t(hlit));
  std::memcpy(seq + hlit, dl, size_t(hdist));
  const int total = hlit + hdist;
  uint8_t sym[kLitLenSyms + kDistSyms], extra[kLitLenSyms + kDistSyms];
  int nr = 0;
  for (int i = 0; i < total;) {
    const uint8_t v = seq[i];
    int run = 1;
    while (i + run < total && seq[i + run] == v && run < 138) ++run;
    if (v == 0 && run >= 3) {
      sym[nr] = run <= 10 ? 17 : 18;
      extra[nr++] = uint8_t(run <= 10 ? run - 3 : run - 11);
      i += run;
    } else if (v != 0 && run >= 4) {
      sym[nr] = v; extra[nr++] = 0xFF;
      ++i;
      const int rep = std::min(run - 1, 6);
      sym[nr] = 16; extra[nr++] = uint8_t(rep - 3);
      i += rep;
    } else {
      sym[nr] = v; extra[nr++] = 0xFF;
      ++i;
    }
  }
  uint32_t cf[kClSyms] = {0};
  for (int i = 0; i < nr; ++i) ++cf[sym[i]];
  uint8_t cl[kClSyms];
  uint16_t cc[kClSyms];
  huffman_lengths(cf, kClSyms, cl, kMaxClBits);
  canonical_codes(cl, kClSyms, cc);
  static const int order[kClSyms] = {16, 17, 18, 0, 8, 7, 9, 6, 10, 5, 11, 4, 12, 3, 13, 2, 14, 1, 15};
  int hclen = kClSyms;
  while (hclen > 4 && cl[order[hclen - 1]] == 0) --hclen;
  bw.put(uint32_t(hlit - 257), 5);
  bw.put(uint32_t(hdist - 1), 5);
  bw.put(uint32_t(hclen - 4), 4);
  for (int i = 0; i < hclen; ++i) bw.put(cl[order[i]], 3);
  for (int i = 0; i < nr; ++i) {
    bw.put(cc[sym[i]], cl[sym[i]]);
    if (extra[i] != 0xFF) bw.put(extra[i], sym[i] == 16 ? 2 : sym[i] == 17 ? 3 : 7);
  }
}

enum Hint { kStored, kFixed, kAuto };

// Block-type choice and emission (deflate_block.cpp:389-474).
void encode_block(const uint32_t* t, size_t nt, const uint8_t* raw, size_t raw_len, Bits& bw,
                  bool last, Hint hint) {
  int type = 0;  // 0 stored, 1 fixed, 2 dynamic
  uint8_t dll[kLitLenSyms] = {0}, ddl[kDistSyms] = {0};
  if (hint != kStored) {
    const uint64_t stored_bits = (uint64_t(raw_len) + 5) * 8;
    Stats s;
    block_stats(t, nt, s);
    if (hint == kFixed) {
      type = stored_bits <= fixed_cost(s) ? 0 : 1;
    } else {
      const uint64_t fb = fixed_cost(s);
      huffman_lengths(s.lit, kLitLenSyms, dll, kMaxBits);
      huffman_lengths(s.dist, kDistSyms, ddl, kMaxBits);
      const uint64_t db = dynamic_cost(s, dll, ddl);
      type = (stored_bits <= fb && stored_bits <= db) ? 0 : (fb <= db ? 1 : 2);
    }
  }
  if (type == 0) {
    emit_stored(raw, raw_len, bw, last);
  } else if (type == 1) {
    uint8_t ll[288], dl[32];
    uint16_t lc[288], dc[32];
    fixed_lengths(ll, dl);
    canonical_codes(ll, 288, lc);
    canonical_codes(dl, 32, dc);
    bw.put(last ? 1 : 0, 1);
    bw.put(1, 2);
    emit_tokens(t, nt, ll, lc, dl, dc, bw);
  } else {
    // Dynamic block (deflate_block.cpp:347-383): EOB always gets a code, a
    // block without matches still sends one distance code of length 1.
    if (dll[256] == 0) dll[256] = 1;
    bool any = false;
    for (int i = 0; i < kDistSyms; ++i) any |= ddl[i] != 0;
    if (!any) ddl[0] = 1;
    int hlit = kLitLenSyms, hdist = kDistSyms;
    while (hlit > 257 && dll[hlit - 1] == 0) --hlit;
    while (hdist > 1 && ddl[hdist - 1] == 0) --hdist;
    bw.put(last ? 1 : 0, 1);
    bw.put(2, 2);
    encode_code_lengths(dll, hlit, ddl, hdist, bw);
    uint16_t lc[288], dc[32];
    canonical_codes(dll, kLitLenSyms, lc);
    canonical_codes(ddl, kDistSyms, dc);
    emit_tokens(t, nt, dll, lc, ddl, dc, bw);
  }
  if (last) bw.align();
}

Hint hint_for(int level) { return level <= 0 ? kStored : level <= 3 ? kFixed : kAuto; }  // level_config.hpp:15-28

// Whole-buffer raw DEFLATE (block_compressor.cpp:16-73): one block for the
// whole input; an all-literal token stream is always stored.
size_t raw_compress(const uint8_t* src, size_t n, uint8_t* dst, size_t cap, int level) {
  Bits bw(dst, cap);
  const Hint h = hint_for(level);
  if (h == kStored) {
    emit_stored(src, n, bw, true);
  } else {
    std::vector<uint32_t> tok(n ? n : 1);
    const size_t nt = lz77(src, n, tok.data(), level);
    if (nt == n) emit_stored(src, n, bw, true);
    else encode_block(tok.data(), nt, src, n, bw, true, h);
  }
  bw.align();
  return bw.overflow ? 0 : bw.pos;
}

size_t raw_bound(size_t n) { return n + (n >> 12) + (n >> 14) + (n >> 25) + 13; }  // raw_deflate.cpp:9-12

}  // namespace

extern "C" {

uint32_t oracle_crc32(uint32_t init, const void* p, size_t n) { return crc32(init, (const uint8_t*)p, n); }
uint32_t oracle_adler32(uint32_t init, const void* p, size_t n) { return adler32(init, (const uint8_t*)p, n); }
void oracle_set_mode(int m) { g_mode = m; }
long oracle_limiter_events(void) { return g_limiter_events; }

// deflate_compress_bound (src/api/deflate_api.cpp:81-98)
size_t oracle_compress_bound(size_t n, int fmt) {
  return raw_bound(n) + (fmt == 1 ? 6 : fmt == 2 ? 18 : 0);
}

size_t oracle_lz77(const void* in, size_t n, int level, uint32_t* tokens) {
  return lz77((const uint8_t*)in, n, tokens, level);
}

void oracle_huffman_lengths(const uint32_t* freq, int nsym, uint8_t* lens, int max_bits) {
  huffman_lengths(freq, nsym, lens, max_bits);
}

// deflate_compress with the raw/zlib/gzip wrappers
// (src/formats/{raw_deflate,zlib_wrapper,gzip_wrapper}.cpp).
size_t oracle_compress(const void* in, size_t n, void* out, size_t cap, int level, int fmt) {
  const uint8_t* src = (const uint8_t*)in;
  uint8_t* dst = (uint8_t*)out;
  if (cap < oracle_compress_bound(n, fmt)) return 0;
  if (fmt == 0) return raw_compress(src, n, dst, cap, level);
  if (fmt == 1) {
    dst[0] = 0x78; dst[1] = 0x9C;
    const size_t r = raw_compress(src, n, dst + 2, cap - 6, level);
    if (!r) return 0;
    const uint32_t a = adler32(1, src, n);
    for (int i = 0; i < 4; ++i) dst[2 + r + i] = uint8_t(a >> (24 - 8 * i));
    return r + 6;
  }
  if (fmt == 2) {
    const uint8_t xfl = level >= 9 ? 2 : level <= 2 ? 4 : 0;
    const uint8_t hdr[10] = {0x1F, 0x8B, 8, 0, 0, 0, 0, 0, xfl, 0xFF};
    std::memcpy(dst, hdr, 10);
    const size_t r = raw_compress(src, n, dst + 10, cap - 18, level);
    if (!r) return 0;
    const uint32_t c = crc32(0, src, n), isz = uint32_t(n);
    for (int i = 0; i < 4; ++i) { dst[10 + r + i] = uint8_t(c >> (8 * i)); dst[14 + r + i] = uint8_t(isz >> (8 * i)); }
    return r + 18;
  }
  return 0;
}

// deflate_parallel_compress (src/parallel/parallel_compressor.cpp:36-150):
// independent chunks with fresh dictionaries, blocks joined bit-contiguously
// with no all-literal shortcut, only the last block final and byte-aligned;
// gzip XFL is always 0.  block_size 0 selects 128 KiB / 512 KiB / 1 MiB by
// level (parallel_compressor.cpp:16-20).  Threads do not change the bytes, so
// the chunks are compressed in order on the calling thread.
size_t oracle_parallel_compress(const void* in, size_t n, void* out, size_t cap, int level, int fmt,
                                size_t block_size) {
  const uint8_t* src = (const uint8_t*)in;
  uint8_t* dst = (uint8_t*)out;
  if (block_size == 0) block_size = level <= 3 ? 131072 : level <= 6 ? 524288 : 1048576;
  const size_t nblk = n ? (n + block_size - 1) / block_size : 1;
  size_t w = 0;
  if (fmt == 1) { if (cap < 6) return 0; dst[0] = 0x78; dst[1] = 0x9C; w = 2; }
  if (fmt == 2) {
    const uint8_t hdr[10] = {0x1F, 0x8B, 8, 0, 0, 0, 0, 0, 0, 0xFF};
    if (cap < 10) return 0;
    std::memcpy(dst, hdr, 10);
    w = 10;
  }
  const size_t trailer = fmt == 1 ? 4 : fmt == 2 ? 8 : 0;
  if (w + trailer > cap) return 0;
  Bits bw(dst + w, cap - w - trailer);
  const Hint h = hint_for(level);
  std::vector<uint32_t> tok;
  for (size_t b = 0; b < nblk; ++b) {
    const size_t off = b * block_size, len = n ? std::min(block_size, n - off) : 0;
    tok.resize(len ? len : 1);
    const size_t nt = lz77(src + off, len, tok.data(), level);
    encode_block(tok.data(), nt, src + off, len, bw, b + 1 == nblk, h);
  }
  if (bw.overflow) return 0;
  w += bw.pos;
  if (fmt == 1) {
    const uint32_t a = adler32(1, src, n);
    for (int i = 0; i < 4; ++i) dst[w++] = uint8_t(a >> (24 - 8 * i));
  } else if (fmt == 2) {
    const uint32_t c = crc32(0, src, n), isz = uint32_t(n);
    for (int i = 0; i < 4; ++i) dst[w++] = uint8_t(c >> (8 * i));
    for (int i = 0; i < 4; ++i) dst[w++] = uint8_t(isz >> (8 * i));
  }
  return w;
}

}  // extern "C"

// ---------------------------------------------------------------- block walker
// Not a restatement of the reference: an RFC 1951 reader that only walks a raw
// DEFLATE stream's blocks (symbols are decoded and skipped, nothing is
// written) and records each block's type.  The tests use it to say which
// streams contain a stored block after a Huffman-coded block, the pattern the
// reference's inflate misreads.
namespace blockwalk {

struct Reader {
  const uint8_t* p;
  size_t n, bit = 0;
  bool bad = false;
  uint32_t get(int k) {
    uint32_t v = 0;
    for (int i = 0; i < k; ++i, ++bit) {
      if ((bit >> 3) >= n) { bad = true; return 0; }
      v |= uint32_t((p[bit >> 3] >> (bit & 7)) & 1u) << i;
    }
    return v;
  }
};

// Canonical code by counts per length and symbols in code order (RFC 1951
// section 3.2.2): decoding reads one bit at a time and compares with the
// first code of each length.
struct Code {
  int count[16] = {};
  int sym[320] = {};
  bool build(const uint8_t* len, int n) {
    for (int i = 0; i < n; ++i) count[len[i]]++;
    count[0] = 0;
    int offs[16] = {}, left = 1;
    for (int l = 1; l < 16; ++l) {
      left = left * 2 - count[l];
      if (left < 0) return false;
      offs[l] = l == 1 ? 0 : offs[l - 1] + count[l - 1];
    }
    for (int i = 0; i < n; ++i)
      if (len[i]) sym[offs[len[i]]++] = i;
    return true;
  }
  int decode(Reader& r) const {
    int code = 0, first = 0, index = 0;
    for (int l = 1; l < 16; ++l) {
      code |= int(r.get(1));
      if (r.bad) return -1;
      const int c = count[l];
      if (code - first < c) return sym[index + code - first];
      index += c;
      first = (first + c) << 1;
      code <<= 1;
    }
    return -1;
  }
};

const int kLenExtra[29] = {0, 0, 0, 0, 0, 0, 0, 0, 1, 1, 1, 1, 2, 2, 2, 2, 3, 3, 3, 3, 4, 4, 4, 4, 5, 5, 5, 5, 0};
const int kDistExtra[30] = {0, 0, 0, 0, 1, 1, 2, 2, 3, 3, 4, 4, 5, 5, 6, 6, 7, 7, 8, 8, 9, 9, 10, 10, 11, 11, 12, 12, 13, 13};

bool skip_symbols(Reader& r, const Code& lit, const Code& dist) {
  for (;;) {
    const int s = lit.decode(r);
    if (s < 0 || s > 285) return false;
    if (s == 256) return true;
    if (s > 256) {
      r.get(kLenExtra[s - 257]);
      const int d = dist.decode(r);
      if (d < 0 || d > 29) return false;
      r.get(kDistExtra[d]);
      if (r.bad) return false;
    }
  }
}

}  // namespace blockwalk

extern "C" {

// Writes the type (0 stored, 1 fixed, 2 dynamic) of every block of the raw
// DEFLATE stream p[0, n) into types[0, max); returns the number of blocks, or
// -1 when the stream is malformed.
long oracle_block_types(const void* data, size_t n, uint8_t* types, long max) {
  using namespace blockwalk;
  Reader r{static_cast<const uint8_t*>(data), n};
  long nb = 0;
  for (;;) {
    const uint32_t last = r.get(1), type = r.get(2);
    if (r.bad || type == 3) return -1;
    if (nb < max) types[nb] = uint8_t(type);
    ++nb;
    if (type == 0) {
      r.bit = (r.bit + 7) & ~size_t(7);
      const uint32_t len = r.get(16), nlen = r.get(16);
      if (r.bad || (len ^ 0xFFFFu) != nlen) return -1;
      r.bit += size_t(len) * 8;
      if ((r.bit >> 3) > n) return -1;
    } else {
      uint8_t lens[320] = {};
      Code lit, dist;
      if (type == 1) {
        for (int i = 0; i < 288; ++i) lens[i] = i < 144 ? 8 : i < 256 ? 9 : i < 280 ? 7 : 8;
        for (int i = 0; i < 30; ++i) lens[288 + i] = 5;
        if (!lit.build(lens, 288) || !dist.build(lens + 288, 30)) return -1;
      } else {
        const int hlit = int(r.get(5)) + 257, hdist = int(r.get(5)) + 1, hclen = int(r.get(4)) + 4;
        static const int order[19] = {16, 17, 18, 0, 8, 7, 9, 6, 10, 5, 11, 4, 12, 3, 13, 2, 14, 1, 15};
        uint8_t cl[19] = {};
        for (int i = 0; i < hclen; ++i) cl[order[i]] = uint8_t(r.get(3));
        Code clc;
        if (r.bad || !clc.build(cl, 19)) return -1;
        int i = 0;
        while (i < hlit + hdist) {
          const int s = clc.decode(r);
          if (s < 0) return -1;
          if (s < 16) { lens[i++] = uint8_t(s); continue; }
          int rep = 0, val = 0;
          if (s == 16) { if (i == 0) return -1; val = lens[i - 1]; rep = 3 + int(r.get(2)); }
          else if (s == 17) rep = 3 + int(r.get(3));
          else rep = 11 + int(r.get(7));
          if (r.bad || i + rep > hlit + hdist) return -1;
          while (rep--) lens[i++] = uint8_t(val);
        }
        uint8_t ll[288] = {}, dl[32] = {};
        std::memcpy(ll, lens, size_t(hlit));
        std::memcpy(dl, lens + hlit, size_t(hdist));
        if (!lit.build(ll, hlit) || !dist.build(dl, hdist)) return -1;
      }
      if (!skip_symbols(r, lit, dist)) return -1;
    }
    if (last) return nb;
  }
}

}  // extern "C"
