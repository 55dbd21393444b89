// synth.cpp -- seeded synthetic inputs for the DEFLATE benchmarks and tests.
//
// No public corpus is named for this workload, so inputs are generated:
//   kind 0  Zipf text: a 4,096-word vocabulary (word length U{3..10}, letters
//           U{a..z}, fixed vocabulary seed), ranks drawn with P(r) ~ r^-1.1,
//           words joined by single spaces; a line target is drawn from
//           U{60..100} and when the running line length reaches it the
//           separator becomes '\n' and a new target is drawn.
//   kind 1  little-endian u32 values v[i] = v[i-1] + U{0..255} (wrapping).
//   kind 2  zero bytes.
//   kind 3  uniform random bytes.
//   kind 4  mixed: 1 MiB segments rotating kinds 0,1,2,3, each segment with
//           its own seed derived from (seed, segment index).
//   kind 5  periodic: a random 8-byte pattern, each byte replaced by a
//           uniform random byte with probability 1/100.
// The generator is splitmix64 (Steele, Lea, Flood 2014), which is fast and
// fully specified; all outputs are deterministic functions of (kind, seed, n).

#include <cmath>
#include <cstdint>
#include <cstring>
#include <string>
#include <vector>

namespace {

struct Rng {
  uint64_t s;
  explicit Rng(uint64_t seed) : s(seed ^ 0x6A09E667F3BCC909ull) {}
  uint64_t next() {
    uint64_t z = (s += 0x9E3779B97F4A7C15ull);
    z = (z ^ (z >> 30)) * 0xBF58476D1CE4E5B9ull;
    z = (z ^ (z >> 27)) * 0x94D049BB133111EBull;
    return z ^ (z >> 31);
  }
  uint32_t below(uint32_t n) { return uint32_t((next() >> 32) * n >> 32); }
  double unit() { return double(next() >> 11) * (1.0 / 9007199254740992.0); }
};

constexpr int kVocab = 4096;
constexpr uint64_t kVocabSeed = 0x766F636162ull;  // fixed: every text shares one vocabulary

struct Vocab {
  std::vector<std::string> words;
  std::vector<double> cdf;
  std::vector<uint16_t> bucket;  // 65536-way index into cdf for O(1) sampling
  Vocab() {
    Rng r(kVocabSeed);
    words.resize(kVocab);
    for (auto& w : words) {
      const int len = 3 + int(r.below(8));
      w.resize(size_t(len));
      for (auto& ch : w) ch = char('a' + r.below(26));
    }
    cdf.resize(kVocab);
    double acc = 0;
    for (int i = 0; i < kVocab; ++i) { acc += std::pow(double(i + 1), -1.1); cdf[i] = acc; }
    for (auto& c : cdf) c /= acc;
    cdf.back() = 1.0;
    bucket.resize(65537);
    int k = 0;
    for (int b = 0; b <= 65536; ++b) {
      const double u = double(b) / 65536.0;
      while (k < kVocab - 1 && cdf[size_t(k)] <= u) ++k;
      bucket[size_t(b)] = uint16_t(k);
    }
  }
  int draw(Rng& r) const {  // inverse CDF
    const double u = r.unit();
    int k = bucket[size_t(u * 65536.0)];
    while (k < kVocab - 1 && cdf[size_t(k)] <= u) ++k;
    return k;
  }
};

const Vocab& vocab() { static const Vocab v; return v; }

void fill_text(uint8_t* d, size_t n, uint64_t seed) {
  const Vocab& v = vocab();
  Rng r(seed);
  size_t o = 0;
  int line = 0, target = 60 + int(r.below(41));
  while (o < n) {
    const std::string& w = v.words[size_t(v.draw(r))];
    for (size_t i = 0; i < w.size() && o < n; ++i) d[o++] = uint8_t(w[i]);
    line += int(w.size());
    if (o >= n) break;
    if (line >= target) {
      d[o++] = '\n';
      line = 0;
      target = 60 + int(r.below(41));
    } else {
      d[o++] = ' ';
      ++line;
    }
  }
}

void fill_ints(uint8_t* d, size_t n, uint64_t seed) {
  Rng r(seed);
  uint32_t v = 0;
  size_t o = 0;
  bool first = true;
  while (o < n) {
    if (!first) v += uint32_t(r.below(256));
    first = false;
    for (int i = 0; i < 4 && o < n; ++i) d[o++] = uint8_t(v >> (8 * i));
  }
}

void fill_random(uint8_t* d, size_t n, uint64_t seed) {
  Rng r(seed);
  size_t o = 0;
  for (; o + 8 <= n; o += 8) { const uint64_t x = r.next(); std::memcpy(d + o, &x, 8); }
  if (o < n) { const uint64_t x = r.next(); std::memcpy(d + o, &x, n - o); }
}

void fill_periodic(uint8_t* d, size_t n, uint64_t seed) {
  Rng r(seed);
  uint8_t pat[8];
  for (auto& b : pat) b = uint8_t(r.below(256));
  for (size_t i = 0; i < n; ++i) d[i] = (r.below(100) == 0) ? uint8_t(r.below(256)) : pat[i & 7];
}

uint64_t mix(uint64_t seed, uint64_t k) { return seed * 0x100000001B3ull + k * 0x9E3779B97F4A7C15ull + 1; }

void fill(uint8_t* d, size_t n, int kind, uint64_t seed) {
  switch (kind) {
    case 0: fill_text(d, n, seed); break;
    case 1: fill_ints(d, n, seed); break;
    case 2: std::memset(d, 0, n); break;
    case 3: fill_random(d, n, seed); break;
    case 4: {
      const size_t seg = size_t(1) << 20;
      for (size_t o = 0, k = 0; o < n; o += seg, ++k) {
        const size_t len = n - o < seg ? n - o : seg;
        fill(d + o, len, int(k % 4), mix(seed, k));
      }
      break;
    }
    case 5: fill_periodic(d, n, seed); break;
    default: std::memset(d, 0, n);
  }
}

}  // namespace

extern "C" {

void synth_fill(void* dst, size_t n, int kind, uint64_t seed) { fill(static_cast<uint8_t*>(dst), n, kind, seed); }

// Sizes exp(U(ln lo, ln hi)) rounded down, for batches of uneven buffers.
void synth_loguniform_sizes(uint64_t* out, size_t count, uint64_t lo, uint64_t hi, uint64_t seed) {
  Rng r(seed);
  const double a = std::log(double(lo)), b = std::log(double(hi));
  for (size_t i = 0; i < count; ++i) {
    uint64_t v = uint64_t(std::exp(a + (b - a) * r.unit()));
    out[i] = v < lo ? lo : v > hi ? hi : v;
  }
}

}  // extern "C"
