// shard.cu -- one pigz-style stream compressed by several GPUs.
//
// The chunks of a parallel stream are independent (every chunk starts from an
// empty dictionary, src/parallel/parallel_compressor.cpp:66-80), so a stream
// splits into contiguous chunk ranges, one per rank.  Each rank compresses its
// range into a bare part (no header or trailer); every part but the last ends
// with an empty stored block (a sync point), which leaves it on a byte
// boundary, so the parts concatenate without any bit shifting.  What the
// ranks exchange is small: the part sizes and the checksum of every range,
// which combine with the identities below.
//
//   deflate_gpu_parallel_shard   this rank's part (GPU)
//   deflate_crc32_combine        CRC-32 of A||B from CRC-32(A), CRC-32(B), |B|
//   deflate_adler32_combine      Adler-32 of A||B from Adler-32(A), Adler-32(B), |B|
#include <cuda_runtime.h>
#include <cstdint>
#include <mutex>
#include "engine_host.h"
#include "deflate_device.cuh"
#include "../../include/orot_b200.h"

using namespace orotb;

extern "C" {

int deflate_gpu_parallel_shard(const void* in, size_t in_size, int level, deflate_format format, size_t block_size,
                               int final_part, void* out, size_t out_capacity, size_t* out_size, uint32_t* checksum) {
  const int fmt = int(format);
  if ((in_size && !in) || !out || !out_size || !checksum || fmt < 0 || fmt > 2) return -1;
  *out_size = 0;
  *checksum = fmt == int(DEFLATE_FORMAT_ZLIB) ? 1u : 0u;  // checksums of an empty range
  if (in_size == 0 && !final_part) return 0;             // a rank without chunks adds nothing
  EngineLease e;
  if (!e) return -2;
  Stream s{};
  const uint32_t mode = kStreamBare | (final_part ? 0u : kStreamOpen);
  const size_t r = e->compress_host(in, in_size, out, out_capacity, level, fmt, true, block_size, mode, &s);
  if (r == 0) return s.error == kErrCapacity || s.out_size > out_capacity ? -3 : -2;
  *out_size = r;
  if (fmt != int(DEFLATE_FORMAT_RAW)) *checksum = s.checksum;
  return 0;
}

uint32_t deflate_crc32_combine(uint32_t crc1, uint32_t crc2, uint64_t len2) {
  // appending len2 bytes multiplies the register by x^(8 len2) mod P; the
  // pre- and post-inversions of both values cancel in the sum
  static const CrcPowers pw = host_crc_powers();
  return gf2_mulmod(xpow8n(pw, len2), crc1) ^ crc2;
}

uint32_t deflate_adler32_combine(uint32_t adler1, uint32_t adler2, uint64_t len2) {
  // a = 1 + sum of bytes, b = sum of a after every byte: appending B gives
  // a = a1 + a2 - 1 and b = b1 + b2 + |B| (a1 - 1)
  constexpr uint64_t M = 65521;
  const uint64_t a1 = adler1 & 0xFFFFu, b1 = adler1 >> 16, a2 = adler2 & 0xFFFFu, b2 = adler2 >> 16;
  const uint64_t a = (a1 + a2 + M - 1) % M;
  const uint64_t b = (b1 + b2 + (len2 % M) * ((a1 + M - 1) % M)) % M;
  return uint32_t(b << 16 | a);
}

}  // extern "C"
