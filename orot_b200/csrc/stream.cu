// stream.cu -- the streaming compress API over the GPU engine.
//
// Same entry points and return codes as the reference's deflate_stream_*
// (include/orot/deflate.h:92-108, src/api/stream_api.cpp:134-247), built the
// way the engine works best: input accumulates into chunks of kChunk bytes and
// every chunk is compressed on the GPU as one part of a pigz-style stream
// (independent chunks; a part that is not the last ends with an empty stored
// block, so every part ends on a byte boundary and can be handed out at once).
//   DEFLATE_NO_FLUSH    compress whenever a chunk is full
//   DEFLATE_SYNC_FLUSH  also compress the partial chunk: all input given so far
//   DEFLATE_FULL_FLUSH  is decodable from the output given so far (chunks never
//                       reference earlier chunks, so both flushes are "full")
//   DEFLATE_FINISH      the last part (BFINAL) and the zlib / gzip trailer from
//                       the chunk checksums combined; then DEFLATE_STREAM_END
// Returns DEFLATE_OK when all input is consumed and nothing is pending,
// DEFLATE_NEED_OUTPUT when the output buffer filled first.
#include <cuda_runtime.h>
#include <algorithm>
#include <cstring>
#include <mutex>
#include <new>
#include <vector>
#include "engine_host.h"
#include "../../include/orot_b200.h"

using namespace orotb;

struct deflate_stream {
  static constexpr size_t kChunk = size_t(1) << 20;
  int level = 6;
  int fmt = 0;
  std::vector<uint8_t> in;       // the chunk being filled
  std::vector<uint8_t> pending;  // output not yet handed out
  size_t pend_pos = 0;
  std::vector<uint8_t> part;     // scratch for one compressed part
  bool header_done = false, finished = false;
  uint32_t check = 0;            // running Adler-32 (zlib) / CRC-32 (gzip)
  uint64_t total = 0;            // input bytes so far

  void push(const uint8_t* p, size_t n) { pending.insert(pending.end(), p, p + n); }

  // Compresses the accumulated chunk as one part; false on a device error.
  bool emit(bool final_part) {
    if (!header_done) {
      if (fmt == int(DEFLATE_FORMAT_ZLIB)) {
        const uint8_t h[2] = {0x78, 0x9C};
        push(h, 2);
      } else if (fmt == int(DEFLATE_FORMAT_GZIP)) {
        const uint8_t h[10] = {0x1F, 0x8B, 8, 0, 0, 0, 0, 0, 0, 0xFF};
        push(h, 10);
      }
      header_done = true;
    }
    size_t n = 0;
    uint32_t ck = 0;
    part.resize(deflate_compress_bound(in.size(), DEFLATE_FORMAT_RAW) + 4096);
    if (deflate_gpu_parallel_shard(in.data(), in.size(), level, deflate_format(fmt), 0, final_part ? 1 : 0, part.data(),
                                   part.size(), &n, &ck) != 0)
      return false;
    push(part.data(), n);
    if (!in.empty()) {
      if (fmt == int(DEFLATE_FORMAT_ZLIB)) check = deflate_adler32_combine(check, ck, in.size());
      else if (fmt == int(DEFLATE_FORMAT_GZIP)) check = deflate_crc32_combine(check, ck, in.size());
    }
    total += in.size();
    in.clear();
    if (final_part) {
      if (fmt == int(DEFLATE_FORMAT_ZLIB)) {
        const uint8_t t[4] = {uint8_t(check >> 24), uint8_t(check >> 16), uint8_t(check >> 8), uint8_t(check)};
        push(t, 4);
      } else if (fmt == int(DEFLATE_FORMAT_GZIP)) {
        const uint32_t z = uint32_t(total);
        const uint8_t t[8] = {uint8_t(check), uint8_t(check >> 8), uint8_t(check >> 16), uint8_t(check >> 24),
                              uint8_t(z),     uint8_t(z >> 8),     uint8_t(z >> 16),     uint8_t(z >> 24)};
        push(t, 8);
      }
      finished = true;
    }
    return true;
  }
};

extern "C" {

deflate_stream* deflate_stream_new(int level, deflate_format format) {
  if (int(format) < 0 || int(format) > 2) return nullptr;
  auto* s = new (std::nothrow) deflate_stream();
  if (!s) return nullptr;
  s->level = level;
  s->fmt = int(format);
  s->check = format == DEFLATE_FORMAT_ZLIB ? 1u : 0u;
  s->in.reserve(deflate_stream::kChunk);
  return s;
}

void deflate_stream_free(deflate_stream* s) { delete s; }

deflate_result deflate_stream_compress(deflate_stream* s, const uint8_t** next_in, size_t* avail_in,
                                       uint8_t** next_out, size_t* avail_out, deflate_flush flush) {
  if (!s || !next_in || !avail_in || !next_out || !avail_out || (*avail_in && !*next_in) ||
      (*avail_out && !*next_out) || int(flush) < 0 || int(flush) > 3)
    return DEFLATE_PARAM_ERROR;
  if (s->finished && *avail_in) return DEFLATE_PARAM_ERROR;  // input after the stream ended
  for (;;) {
    // 1. hand out pending output
    if (s->pend_pos < s->pending.size()) {
      const size_t k = std::min(*avail_out, s->pending.size() - s->pend_pos);
      if (k) std::memcpy(*next_out, s->pending.data() + s->pend_pos, k);
      *next_out += k;
      *avail_out -= k;
      s->pend_pos += k;
      if (s->pend_pos < s->pending.size()) return DEFLATE_NEED_OUTPUT;
    }
    s->pending.clear();
    s->pend_pos = 0;
    if (s->finished) return DEFLATE_STREAM_END;
    // 2. take input into the chunk
    if (*avail_in) {
      const size_t k = std::min(*avail_in, deflate_stream::kChunk - s->in.size());
      s->in.insert(s->in.end(), *next_in, *next_in + k);
      *next_in += k;
      *avail_in -= k;
    }
    // 3. compress a full chunk, or what the flush asks for
    const bool full = s->in.size() == deflate_stream::kChunk;
    const bool last = flush == DEFLATE_FINISH && *avail_in == 0;
    const bool sync = (flush == DEFLATE_SYNC_FLUSH || flush == DEFLATE_FULL_FLUSH) && *avail_in == 0 && !s->in.empty();
    if (last || full || sync) {
      if (!s->emit(last)) return DEFLATE_MEM_ERROR;
      continue;
    }
    return DEFLATE_OK;
  }
}

}  // extern "C"
