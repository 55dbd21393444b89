// members.cu -- gzip files made of independent members.
//
// Compression (no counterpart in the reference's compress API): the input is
// cut into members of member_size bytes and every member is a complete gzip
// stream, all compressed in one pass of the batch engine.  The concatenation
// is one valid gzip file for any reader.
//
// Decompression follows the reference's parallel gzip path
// (src/decompress/parallel_decompress.cpp:19-150, used by deflate_decompress
// for gzip inputs of 256 KiB and more, src/api/deflate_api.cpp:203-211):
// members are located by scanning for a valid header; the 8 bytes before the
// next member are the trailer; with at least two members every member is
// decoded into place (output offsets from the ISIZE fields), each must fill
// exactly its ISIZE and match its CRC-32.  Here the members are decoded by
// k_inflate, one warp per member, and their CRC-32s are computed by the
// checksum kernels.
#include <cuda_runtime.h>
#include <algorithm>
#include <cstring>
#include <mutex>
#include <vector>
#include "engine_host.h"
#include "kernels.cuh"
#include "../../include/orot_b200.h"

namespace orotb {

// Offset just past a gzip header at s, or 0 (parallel_decompress.cpp:19-50
// rules: reserved flag bits rejected, 8 trailer bytes must fit).
static size_t member_header(const uint8_t* s, size_t n) {
  if (n < 18 || s[0] != 0x1F || s[1] != 0x8B || s[2] != 8 || s[3] >= 0x20) return 0;
  const uint8_t flags = s[3];
  size_t o = 10;
  if (flags & 0x04) {
    if (o + 2 > n) return 0;
    o += 2 + (size_t(s[o]) | (size_t(s[o + 1]) << 8));
  }
  if (flags & 0x08) {
    while (o < n && s[o] != 0) ++o;
    ++o;
  }
  if (flags & 0x10) {
    while (o < n && s[o] != 0) ++o;
    ++o;
  }
  if (flags & 0x02) o += 2;
  if (o + 8 > n) return 0;
  return o;
}

struct Member {
  size_t start, end, hdr, out_off, out_size;
};

// Member boundaries as the reference finds them (parallel_decompress.cpp:78-108).
static std::vector<Member> find_members(const uint8_t* in, size_t n) {
  std::vector<Member> ms;
  size_t pos = 0;
  while (pos < n) {
    const size_t h = member_header(in + pos, n - pos);
    if (h == 0) break;
    size_t next = n;
    for (size_t i = pos + h; i + 2 < n; ++i)
      if (in[i] == 0x1F && in[i + 1] == 0x8B && i + 3 < n && in[i + 2] == 8 && member_header(in + i, n - i)) {
        next = i;
        break;
      }
    if (next < 8 || next - 8 < pos + h) break;
    const uint8_t* t = in + next - 8;
    Member m{pos, next, h, 0, size_t(uint32_t(t[4]) | (uint32_t(t[5]) << 8) | (uint32_t(t[6]) << 16) | (uint32_t(t[7]) << 24))};
    ms.push_back(m);
    if (next >= n) break;
    pos = next;
  }
  return ms;
}

// DEFLATE_DATA_ERROR when the input is not (at least) two members or any
// member fails, as the reference's parallel path.
deflate_result gzip_members_decompress(Engine& e, const uint8_t* in, size_t n, uint8_t* out, size_t cap,
                                       size_t* actual) {
  std::vector<Member> ms = find_members(in, n);
  if (ms.size() < 2) return DEFLATE_DATA_ERROR;
  size_t total = 0;
  for (Member& m : ms) {
    m.out_off = total;
    total += m.out_size;
  }
  if (total > cap) return DEFLATE_MEM_ERROR;
  const size_t k = ms.size();
  if (!e.ensure_io(align_up(n, 16) + 64, align_up(total, 16) + 64) || !e.h_stage.ensure(n)) return DEFLATE_MEM_ERROR;
  // decode jobs, largest first
  std::vector<InflateJob> jobs(k);
  std::vector<uint32_t> order(k);
  for (size_t i = 0; i < k; ++i) {
    jobs[i].in_off = ms[i].start + ms[i].hdr;
    jobs[i].in_len = ms[i].end - 8 - jobs[i].in_off;
    jobs[i].out_off = ms[i].out_off;
    jobs[i].out_cap = ms[i].out_size;
    order[i] = uint32_t(i);
  }
  std::stable_sort(order.begin(), order.end(), [&](uint32_t a, uint32_t b) { return jobs[a].in_len > jobs[b].in_len; });
  // checksum tables: one gzip "stream" per member over the decoded bytes
  std::vector<Stream> st(k);
  std::vector<CkBlock> ck;
  for (size_t i = 0; i < k; ++i) {
    st[i].in_off = ms[i].out_off;
    st[i].in_len = ms[i].out_size;
    st[i].fmt = kFmtGzip;
    st[i].ck_first = uint32_t(ck.size());
    for (uint64_t o = 0; o < ms[i].out_size; o += 65536) {
      CkBlock c{};
      c.in_off = ms[i].out_off + o;
      c.len = uint32_t(std::min<uint64_t>(65536, ms[i].out_size - o));
      c.stream = uint32_t(i);
      c.what = kCkCrc;
      ck.push_back(c);
    }
    st[i].ck_count = uint32_t(ck.size()) - st[i].ck_first;
  }
  const size_t o_jobs = 0, o_order = align_up(k * sizeof(InflateJob), 256);
  const size_t o_st = o_order + align_up(k * 4 + 8, 256), o_ck = o_st + align_up(k * sizeof(Stream), 256);
  const size_t o_cnt = o_ck + align_up(ck.size() * sizeof(CkBlock) + 1, 256);
  if (!e.d_tables.ensure(o_cnt + 256)) return DEFLATE_MEM_ERROR;
  uint8_t* dt = static_cast<uint8_t*>(e.d_tables.p);
  InflateJob* d_jobs = reinterpret_cast<InflateJob*>(dt + o_jobs);
  uint32_t* d_order = reinterpret_cast<uint32_t*>(dt + o_order);
  Stream* d_st = reinterpret_cast<Stream*>(dt + o_st);
  CkBlock* d_ck = reinterpret_cast<CkBlock*>(dt + o_ck);
  uint32_t* d_cnt = reinterpret_cast<uint32_t*>(dt + o_cnt);
  std::memcpy(e.h_stage.p, in, n);
  cudaStream_t s = e.stream;
  if (cudaMemcpyAsync(e.d_in.p, e.h_stage.p, n, cudaMemcpyHostToDevice, s) != cudaSuccess ||
      cudaMemcpyAsync(d_jobs, jobs.data(), k * sizeof(InflateJob), cudaMemcpyHostToDevice, s) != cudaSuccess ||
      cudaMemcpyAsync(d_order, order.data(), k * 4, cudaMemcpyHostToDevice, s) != cudaSuccess ||
      cudaMemcpyAsync(d_st, st.data(), k * sizeof(Stream), cudaMemcpyHostToDevice, s) != cudaSuccess ||
      (!ck.empty() && cudaMemcpyAsync(d_ck, ck.data(), ck.size() * sizeof(CkBlock), cudaMemcpyHostToDevice, s) != cudaSuccess)) {
    set_error("H2D failed");
    return DEFLATE_MEM_ERROR;
  }
  uint8_t* dec = static_cast<uint8_t*>(e.d_out.p);
  launch_inflate(static_cast<const uint8_t*>(e.d_in.p), dec, d_jobs, d_order, uint32_t(k), d_cnt, e.sms, s);
  Work w{};
  w.in = dec;
  w.streams = d_st;
  w.nstreams = uint32_t(k);
  w.ck = d_ck;
  w.nck = uint32_t(ck.size());
  launch_checksums(w, s);
  if (cudaMemcpyAsync(jobs.data(), d_jobs, k * sizeof(InflateJob), cudaMemcpyDeviceToHost, s) != cudaSuccess ||
      cudaMemcpyAsync(st.data(), d_st, k * sizeof(Stream), cudaMemcpyDeviceToHost, s) != cudaSuccess ||
      cudaStreamSynchronize(s) != cudaSuccess) {
    set_error(std::string("device error: ") + cudaGetErrorString(cudaGetLastError()));
    return DEFLATE_MEM_ERROR;
  }
  for (size_t i = 0; i < k; ++i) {
    const uint8_t* t = in + ms[i].end - 8;
    const uint32_t crc = uint32_t(t[0]) | (uint32_t(t[1]) << 8) | (uint32_t(t[2]) << 16) | (uint32_t(t[3]) << 24);
    if (jobs[i].status != kInfOk || jobs[i].out_len != ms[i].out_size || st[i].checksum != crc) return DEFLATE_DATA_ERROR;
  }
  if (total && cudaMemcpy(out, dec, total, cudaMemcpyDeviceToHost) != cudaSuccess) {
    set_error("D2H failed");
    return DEFLATE_MEM_ERROR;
  }
  if (actual) *actual = total;
  return DEFLATE_OK;
}

}  // namespace orotb

using namespace orotb;

extern "C" {

size_t deflate_gzip_members_bound(size_t in_size, size_t member_size) {
  if (!member_size) return 0;
  const size_t k = in_size ? (in_size + member_size - 1) / member_size : 1;
  return k * framed_bound(std::min(in_size, member_size), int(DEFLATE_FORMAT_GZIP));
}

size_t deflate_gpu_compress_gzip_members(const void* in, size_t in_size, int level, size_t member_size, void* out,
                                         size_t out_capacity) {
  if ((in_size && !in) || !out || !member_size) return 0;
  if (out_capacity < deflate_gzip_members_bound(in_size, member_size)) return 0;
  const size_t k = in_size ? (in_size + member_size - 1) / member_size : 1;
  std::vector<size_t> sizes(k);
  for (size_t i = 0; i < k; ++i) sizes[i] = std::min(member_size, in_size - std::min(in_size, i * member_size));
  const size_t pb = deflate_gpu_packed_bound(sizes.data(), k, DEFLATE_FORMAT_GZIP);
  std::vector<uint8_t> packed(pb);
  std::vector<uint64_t> offs(k + 1);
  std::vector<size_t> osz(k);
  if (!deflate_gpu_compress_packed(in, sizes.data(), k, level, DEFLATE_FORMAT_GZIP, packed.data(), pb, offs.data(),
                                   osz.data()))
    return 0;
  // members back to back (the packed layout aligns each to 16 bytes)
  uint8_t* o = static_cast<uint8_t*>(out);
  size_t pos = 0;
  for (size_t i = 0; i < k; ++i) {
    if (osz[i] == 0 || pos + osz[i] > out_capacity) return 0;
    std::memcpy(o + pos, packed.data() + offs[i], osz[i]);
    pos += osz[i];
  }
  return pos;
}

}  // extern "C"
