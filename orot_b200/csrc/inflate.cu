// inflate.cu -- deflate_decompress on the GPU and on-device verification of
// a compressed batch.
//
// deflate_decompress follows the reference's whole-buffer decompress
// (src/api/deflate_api.cpp:138-219 with src/formats/raw_deflate.cpp:25-55,
// zlib_wrapper.cpp:104-142, gzip_wrapper.cpp:76-139): the framing is checked
// on the host, the raw stream is decoded by k_inflate, the trailer is checked
// against a checksum of the output computed on the device.  Corrupt input, a
// stream that needs more input and an output buffer that is too small all
// return DEFLATE_DATA_ERROR, as in the reference.
#include <cuda_runtime.h>
#include <algorithm>
#include <cstdint>
#include <cstring>
#include <mutex>
#include <numeric>
#include <vector>
#include "engine_host.h"
#include "kernels.cuh"
#include "../../include/orot_b200.h"

namespace orotb {

// Raw DEFLATE range of a framed stream, checked like the reference's wrappers.
static deflate_result frame_range(const uint8_t* s, size_t n, int fmt, size_t* off, size_t* len) {
  if (fmt == int(DEFLATE_FORMAT_RAW)) {
    *off = 0;
    *len = n;
    return DEFLATE_OK;
  }
  if (fmt == int(DEFLATE_FORMAT_ZLIB)) {
    if (n < 6) return DEFLATE_DATA_ERROR;
    if ((s[0] & 0x0F) != 8) return DEFLATE_DATA_ERROR;                        // CM = 8
    if (((uint32_t(s[0]) << 8) | s[1]) % 31 != 0) return DEFLATE_DATA_ERROR;  // FCHECK
    if (s[1] & 0x20) return DEFLATE_DATA_ERROR;                               // no preset dictionary
    *off = 2;
    *len = n - 6;
    return DEFLATE_OK;
  }
  if (n < 18 || s[0] != 0x1F || s[1] != 0x8B || s[2] != 8) return DEFLATE_DATA_ERROR;
  const uint8_t flags = s[3];
  size_t o = 10;
  if (flags & 0x04) {  // FEXTRA
    if (o + 2 > n) return DEFLATE_DATA_ERROR;
    o += 2 + (size_t(s[o]) | (size_t(s[o + 1]) << 8));
  }
  if (flags & 0x08) {  // FNAME
    while (o < n && s[o] != 0) ++o;
    ++o;
  }
  if (flags & 0x10) {  // FCOMMENT
    while (o < n && s[o] != 0) ++o;
    ++o;
  }
  if (flags & 0x02) o += 2;  // FHCRC
  if (o + 8 > n) return DEFLATE_DATA_ERROR;
  *off = o;
  *len = n - o - 8;
  return DEFLATE_OK;
}

deflate_result gzip_members_decompress(Engine& e, const uint8_t* in, size_t n, uint8_t* out, size_t cap,
                                       size_t* actual);

// Decodes the raw DEFLATE bytes raw[0, len) on the device into d_out + out_off
// (at most cap bytes).  Returns false on a device error; the job holds the
// status, the bytes written and the input bytes the stream occupied.
static bool decode_raw(Engine& e, const uint8_t* raw, size_t len, size_t out_off, size_t cap, InflateJob* job) {
  const size_t tbl = align_up(sizeof(InflateJob), 256) + 256;
  if (!e.d_tables.ensure(tbl) || !e.h_stage.ensure(std::max<size_t>(len, 16))) return false;
  uint8_t* dt = static_cast<uint8_t*>(e.d_tables.p);
  InflateJob* d_job = reinterpret_cast<InflateJob*>(dt);
  uint32_t* d_order = reinterpret_cast<uint32_t*>(dt + align_up(sizeof(InflateJob), 256));
  uint32_t* d_counter = d_order + 1;
  *job = InflateJob{};
  job->in_len = len;
  job->out_off = out_off;
  job->out_cap = cap;
  const uint32_t zero = 0;
  if (len) std::memcpy(e.h_stage.p, raw, len);
  if ((len && cudaMemcpyAsync(e.d_in.p, e.h_stage.p, len, cudaMemcpyHostToDevice, e.stream) != cudaSuccess) ||
      cudaMemcpyAsync(d_job, job, sizeof *job, cudaMemcpyHostToDevice, e.stream) != cudaSuccess ||
      cudaMemcpyAsync(d_order, &zero, 4, cudaMemcpyHostToDevice, e.stream) != cudaSuccess) {
    set_error("H2D failed");
    return false;
  }
  launch_inflate(static_cast<const uint8_t*>(e.d_in.p), static_cast<uint8_t*>(e.d_out.p), d_job, d_order, 1,
                 d_counter, e.sms, e.stream);
  if (cudaMemcpyAsync(job, d_job, sizeof *job, cudaMemcpyDeviceToHost, e.stream) != cudaSuccess ||
      cudaStreamSynchronize(e.stream) != cudaSuccess) {
    set_error(std::string("device error: ") + cudaGetErrorString(cudaGetLastError()));
    return false;
  }
  return true;
}

// Most bytes n bytes of DEFLATE data can decode to: the densest token is a
// 258-byte match coded in 2 bits (1-bit length and distance codes, no extra
// bits), 1032 bytes per input byte; stored blocks expand less.
static size_t max_inflated(size_t n) { return n > (SIZE_MAX - 64) / 1032 ? SIZE_MAX - 64 : n * 1032 + 64; }

static uint32_t le32(const uint8_t* t) {
  return uint32_t(t[0]) | (uint32_t(t[1]) << 8) | (uint32_t(t[2]) << 16) | (uint32_t(t[3]) << 24);
}

// gzip members one after another, each ending where its DEFLATE stream ends:
// accepts every concatenation of members, also where a member's data happens
// to contain a header-like byte pattern that the parallel path splits on.
static deflate_result gzip_members_sequential(Engine& e, const uint8_t* in, size_t n, uint8_t* out, size_t cap,
                                              size_t* actual) {
  cap = std::min(cap, max_inflated(n));
  if (!e.ensure_io(align_up(n, 16) + 64, align_up(cap, 16) + 64)) return DEFLATE_MEM_ERROR;
  size_t pos = 0, total = 0;
  while (pos < n) {
    size_t off = 0, rlen = 0;
    if (frame_range(in + pos, n - pos, int(DEFLATE_FORMAT_GZIP), &off, &rlen) != DEFLATE_OK) return DEFLATE_DATA_ERROR;
    InflateJob job;
    if (!decode_raw(e, in + pos + off, rlen, total, cap - total, &job)) return DEFLATE_MEM_ERROR;
    if (job.status != kInfOk) return DEFLATE_DATA_ERROR;
    const uint8_t* t = in + pos + off + job.in_used;  // the member's trailer
    if (pos + off + job.in_used + 8 > n) return DEFLATE_DATA_ERROR;
    if (e.checksum_device(0, static_cast<const uint8_t*>(e.d_out.p) + total, job.out_len, false) != le32(t) ||
        le32(t + 4) != uint32_t(job.out_len & 0xFFFFFFFFu))
      return DEFLATE_DATA_ERROR;
    total += job.out_len;
    pos += off + job.in_used + 8;
  }
  if (total && cudaMemcpy(out, e.d_out.p, total, cudaMemcpyDeviceToHost) != cudaSuccess) {
    set_error("D2H failed");
    return DEFLATE_MEM_ERROR;
  }
  if (actual) *actual = total;
  return DEFLATE_OK;
}

static deflate_result decompress_one(Engine& e, const uint8_t* in, size_t n, uint8_t* out, size_t cap, size_t* actual,
                                     int fmt);

static deflate_result decompress_host(Engine& e, const uint8_t* in, size_t n, uint8_t* out, size_t cap,
                                      size_t* actual, int fmt) {
  // gzip of 256 KiB or more: independent members decode in parallel when there
  // are at least two (src/api/deflate_api.cpp:203-211).  The member scan can
  // split on a header-like pattern inside compressed data (the reference then
  // fails the file); here the file is decoded as one stream, or member after
  // member, before an error is returned.
  bool members_too_big = false;
  if (fmt == int(DEFLATE_FORMAT_GZIP) && n >= (size_t(256) << 10)) {
    const deflate_result r = gzip_members_decompress(e, in, n, out, cap, actual);
    if (r == DEFLATE_OK) return r;
    members_too_big = r == DEFLATE_MEM_ERROR;
  }
  const deflate_result r = decompress_one(e, in, n, out, cap, actual, fmt);
  // the reference's answer for members whose sizes exceed the output buffer
  return r == DEFLATE_DATA_ERROR && members_too_big ? DEFLATE_MEM_ERROR : r;
}

static deflate_result decompress_one(Engine& e, const uint8_t* in, size_t n, uint8_t* out, size_t cap, size_t* actual,
                                     int fmt) {
  size_t off = 0, rlen = 0;
  const deflate_result fr = frame_range(in, n, fmt, &off, &rlen);
  if (fr != DEFLATE_OK) return fr;
  // The device arena holds at most what rlen bytes can expand to (not the
  // caller's whole capacity, which may exceed free device memory).
  const size_t dcap = std::min(cap, max_inflated(rlen));
  if (!e.ensure_io(align_up(rlen, 16) + 64, align_up(dcap, 16) + 64)) return DEFLATE_MEM_ERROR;
  InflateJob job;
  if (!decode_raw(e, in + off, rlen, 0, dcap, &job)) return DEFLATE_MEM_ERROR;
  bool good = job.status == kInfOk;
  const uint8_t* t = in + n;  // trailer
  if (good && fmt == int(DEFLATE_FORMAT_ZLIB)) {
    const uint32_t want = (uint32_t(t[-4]) << 24) | (uint32_t(t[-3]) << 16) | (uint32_t(t[-2]) << 8) | t[-1];
    good = e.checksum_device(1, static_cast<const uint8_t*>(e.d_out.p), job.out_len, true) == want;
  } else if (good && fmt == int(DEFLATE_FORMAT_GZIP)) {
    good = e.checksum_device(0, static_cast<const uint8_t*>(e.d_out.p), job.out_len, false) == le32(t - 8) &&
           le32(t - 4) == uint32_t(job.out_len & 0xFFFFFFFFu);
  }
  if (!good) {
    // a gzip file of several members: decode them in order
    if (fmt == int(DEFLATE_FORMAT_GZIP) && job.status == kInfOk && off + job.in_used + 8 < n)
      return gzip_members_sequential(e, in, n, out, cap, actual);
    return DEFLATE_DATA_ERROR;
  }
  if (job.out_len && cudaMemcpy(out, e.d_out.p, job.out_len, cudaMemcpyDeviceToHost) != cudaSuccess) {
    set_error("D2H failed");
    return DEFLATE_MEM_ERROR;
  }
  if (actual) *actual = job.out_len;
  return DEFLATE_OK;
}

}  // namespace orotb

using namespace orotb;

extern "C" deflate_result deflate_decompress(const void* in, size_t in_size, void* out, size_t out_capacity,
                                             size_t* actual_out_size, deflate_format format) {
  const int fmt = int(format);
  if (fmt < 0 || fmt > 2 || (in_size && !in) || (out_capacity && !out)) return DEFLATE_PARAM_ERROR;
  EngineLease e;
  if (!e) return DEFLATE_MEM_ERROR;
  return decompress_host(*e, static_cast<const uint8_t*>(in), in_size, static_cast<uint8_t*>(out),
                         out_capacity, actual_out_size, fmt);
}
