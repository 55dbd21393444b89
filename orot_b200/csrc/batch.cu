// batch.cu -- device-resident batches of independent buffers.
//
// The reference compresses many buffers with one deflate_compress call each
// (src/api/deflate_api.cpp:100-136).  Here a batch of buffers is one pass of
// the engine: every buffer is a stream, all tiles of all streams share the
// same persistent kernels, and the pass can be captured once into a CUDA graph
// and replayed.  For host-to-host use the outputs are packed on the device at
// 16-byte aligned offsets so that one device-to-host copy returns them all.
#include <cuda_runtime.h>
#include <algorithm>
#include <cstring>
#include <mutex>
#include <new>
#include <vector>
#include "engine_host.h"
#include "../../include/orot_b200.h"

namespace orotb {

// Exclusive scan of the stream sizes (rounded to 16 bytes) -> pack offsets.
__global__ void k_pack_offsets(const Stream* __restrict__ st, uint32_t n, uint64_t* __restrict__ off) {
  __shared__ uint64_t part[1024];
  const uint32_t t = threadIdx.x;
  const uint32_t per = (n + 1023) / 1024;
  const uint32_t b = t * per, e = min(n, b + per);
  uint64_t s = 0;
  for (uint32_t i = b; i < e; ++i) s += (st[i].out_size + 15) & ~uint64_t(15);
  part[t] = s;
  __syncthreads();
  for (uint32_t o = 1; o < 1024; o <<= 1) {
    const uint64_t v = t >= o ? part[t - o] : 0;
    __syncthreads();
    part[t] += v;
    __syncthreads();
  }
  uint64_t run = t ? part[t - 1] : 0;
  for (uint32_t i = b; i < e; ++i) {
    off[i] = run;
    run += (st[i].out_size + 15) & ~uint64_t(15);
  }
  if (t == 1023) off[n] = part[1023];
}

__global__ void k_pack(const Stream* __restrict__ st, uint32_t n, const uint64_t* __restrict__ off,
                       const uint8_t* __restrict__ out, uint8_t* __restrict__ packed);

__global__ void k_sizes(const Stream* __restrict__ st, uint32_t n, uint64_t* __restrict__ sizes) {
  const uint32_t i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i < n) sizes[i] = st[i].error ? 0 : st[i].out_size;
}

void launch_pack(const Work& w, uint64_t* d_off, uint64_t* d_sizes, uint8_t* d_packed, cudaStream_t st) {
  k_pack_offsets<<<1, 1024, 0, st>>>(w.streams, w.nstreams, d_off);
  k_pack<<<w.nstreams, 256, 0, st>>>(w.streams, w.nstreams, d_off, w.out, d_packed);
  if (d_sizes) k_sizes<<<(w.nstreams + 255) / 256, 256, 0, st>>>(w.streams, w.nstreams, d_sizes);
}

__global__ void k_pack(const Stream* __restrict__ st, uint32_t n, const uint64_t* __restrict__ off,
                       const uint8_t* __restrict__ out, uint8_t* __restrict__ packed) {
  const uint32_t i = blockIdx.x;
  if (i >= n) return;
  const Stream s = st[i];
  const uint4* src = reinterpret_cast<const uint4*>(out + s.out_off);
  uint4* dst = reinterpret_cast<uint4*>(packed + off[i]);
  const uint64_t n16 = (s.out_size + 15) / 16;
  for (uint64_t k = threadIdx.x; k < n16; k += blockDim.x) dst[k] = src[k];
}

}  // namespace orotb

using namespace orotb;

struct deflate_gpu_batch {
  Engine eng;
  DevBuf d_verify, d_vtab;  // on-device verification: decoded bytes, job tables
  std::vector<Job> jobs;
  cudaGraph_t graph = nullptr;
  cudaGraphExec_t gexec = nullptr;
  cudaStream_t graph_stream = nullptr;
  int launches = 0;
  bool ran = false;
  ~deflate_gpu_batch() {
    if (gexec) cudaGraphExecDestroy(gexec);
    if (graph) cudaGraphDestroy(graph);
  }
};

static void drop_graph(deflate_gpu_batch* b) {
  if (b->gexec) cudaGraphExecDestroy(b->gexec);
  if (b->graph) cudaGraphDestroy(b->graph);
  b->gexec = nullptr;
  b->graph = nullptr;
}

// Lays out `count` buffers, uploads them, plans the pass.  With `concat`
// set, the buffers are back to back in caller memory and are copied to the
// device in one transfer (DMA straight from the caller when it is pinned);
// otherwise each buffer is staged at a 16-byte aligned offset.
static bool batch_setup(deflate_gpu_batch* b, const void* const* in, const uint8_t* concat, const size_t* sizes,
                        size_t count, int level, int fmt, bool parallel, size_t block, cudaStream_t st) {
  Engine& e = b->eng;
  drop_graph(b);
  b->jobs.assign(count, Job{});
  uint64_t in_total = 0, out_total = 0;
  for (size_t i = 0; i < count; ++i) {
    Job& j = b->jobs[i];
    j.in_off = in_total;
    j.in_len = sizes[i];
    j.out_off = out_total;
    j.out_cap = parallel ? parallel_bound(sizes[i], fmt, level, block) : framed_bound(sizes[i], fmt);
    j.level = level;
    j.fmt = fmt;
    j.parallel = parallel;
    j.block_size = block;
    in_total += concat ? sizes[i] : align_up(sizes[i], 16);
    out_total += align_up(j.out_cap, 16);
  }
  if (!e.ensure_io(in_total, out_total)) return false;
  if (concat) {
    if (in_total && cudaMemcpyAsync(e.d_in.p, concat, in_total, cudaMemcpyHostToDevice, st) != cudaSuccess) {
      set_error("H2D failed");
      return false;
    }
  } else {
    if (!e.h_stage.ensure(std::max<uint64_t>(in_total, 16))) return false;
    uint8_t* sp = static_cast<uint8_t*>(e.h_stage.p);
    for (size_t i = 0; i < count; ++i)
      if (sizes[i]) std::memcpy(sp + b->jobs[i].in_off, in[i], sizes[i]);
    if (in_total && cudaMemcpyAsync(e.d_in.p, sp, in_total, cudaMemcpyHostToDevice, st) != cudaSuccess) {
      set_error("H2D failed");
      return false;
    }
    if (cudaStreamSynchronize(st) != cudaSuccess) { set_error("H2D sync failed"); return false; }
  }
  return e.plan(b->jobs);
}

// Packs every stream's output at 16-byte aligned offsets in e.d_pack and
// copies sizes + offsets + packed bytes to the host.
static bool batch_pack_to_host(deflate_gpu_batch* b, cudaStream_t st, void* host_out, size_t host_cap,
                               uint64_t* offsets, size_t* sizes_out, uint64_t* total_out) {
  Engine& e = b->eng;
  const Work w = e.work();
  const size_t count = e.streams.size();
  uint64_t out_total = 0;
  for (const Job& j : b->jobs) out_total += align_up(j.out_cap, 16);
  if (!e.d_pack.ensure(align_up(out_total, 256) + (count + 1) * 8 + 256)) return false;
  uint64_t* d_off = reinterpret_cast<uint64_t*>(static_cast<uint8_t*>(e.d_pack.p) + align_up(out_total, 256));
  k_pack_offsets<<<1, 1024, 0, st>>>(w.streams, w.nstreams, d_off);
  k_pack<<<w.nstreams, 256, 0, st>>>(w.streams, w.nstreams, d_off, w.out, static_cast<uint8_t*>(e.d_pack.p));
  std::vector<Stream> s(count);
  if (cudaMemcpyAsync(s.data(), w.streams, count * sizeof(Stream), cudaMemcpyDeviceToHost, st) != cudaSuccess ||
      cudaMemcpyAsync(offsets, d_off, (count + 1) * 8, cudaMemcpyDeviceToHost, st) != cudaSuccess ||
      cudaStreamSynchronize(st) != cudaSuccess) {
    set_error("D2H failed");
    return false;
  }
  const uint64_t total = offsets[count];
  if (total > host_cap) { set_error("packed output larger than the host buffer"); return false; }
  if (total && (cudaMemcpyAsync(host_out, e.d_pack.p, total, cudaMemcpyDeviceToHost, st) != cudaSuccess ||
                cudaStreamSynchronize(st) != cudaSuccess)) {
    set_error("D2H failed");
    return false;
  }
  for (size_t i = 0; i < count; ++i) sizes_out[i] = s[i].error ? 0 : s[i].out_size;
  *total_out = total;
  return true;
}

// The batch that the host-to-host batch calls reuse, one per device (that of
// the calling thread), created on first use; callers hold global_mutex().
static deflate_gpu_batch* host_batch() {
  static deflate_gpu_batch* per_dev[kMaxDevices] = {};
  const int dev = current_device();
  if (dev < 0) return nullptr;
  if (!per_dev[dev]) {
    auto* b = new (std::nothrow) deflate_gpu_batch();
    if (!b || !b->eng.ok) { delete b; return nullptr; }
    per_dev[dev] = b;
  }
  return per_dev[dev];
}

extern "C" {

deflate_gpu_batch* deflate_gpu_batch_new(void) {
  int n = 0;
  if (cudaGetDeviceCount(&n) != cudaSuccess || n == 0) { cudaGetLastError(); set_error("no CUDA device"); return nullptr; }
  auto* b = new (std::nothrow) deflate_gpu_batch();
  if (b && !b->eng.ok) { delete b; return nullptr; }
  return b;
}

void deflate_gpu_batch_free(deflate_gpu_batch* b) { delete b; }

int deflate_gpu_batch_load(deflate_gpu_batch* b, const void* concat, const size_t* sizes, size_t count, int level,
                           deflate_format format, int parallel, size_t block_size) {
  if (!b || (count && (!sizes || !concat)) || int(format) < 0 || int(format) > 2) return -1;
  DeviceScope dev_scope(b->eng.device);
  std::vector<const void*> ptrs(count);
  const uint8_t* p = static_cast<const uint8_t*>(concat);
  for (size_t i = 0; i < count; ++i) { ptrs[i] = p; p += sizes[i]; }
  return batch_setup(b, ptrs.data(), nullptr, sizes, count, level, int(format), parallel != 0, block_size, b->eng.stream)
             ? 0
             : -1;
}

int deflate_gpu_batch_run(deflate_gpu_batch* b, void* cuda_stream, int use_graph) {
  if (!b) return -1;
  DeviceScope dev_scope(b->eng.device);
  Engine& e = b->eng;
  cudaStream_t st = cuda_stream ? static_cast<cudaStream_t>(cuda_stream) : e.stream;
  if (!use_graph) {
    if (!e.launch(st)) return -1;
    b->launches = e.launches;
    b->ran = true;
    return 0;
  }
  if (!b->gexec) {
    cudaStream_t cap;
    if (cudaStreamCreateWithFlags(&cap, cudaStreamNonBlocking) != cudaSuccess) { set_error("stream"); return -1; }
    if (cudaStreamBeginCapture(cap, cudaStreamCaptureModeThreadLocal) != cudaSuccess) {
      cudaStreamDestroy(cap);
      set_error("begin capture failed");
      return -1;
    }
    const bool ok = e.launch(cap);
    cudaGraph_t g = nullptr;
    const cudaError_t ce = cudaStreamEndCapture(cap, &g);
    cudaStreamDestroy(cap);
    if (!ok || ce != cudaSuccess || !g) { cudaGetLastError(); set_error("capture failed"); return -1; }
    if (cudaGraphInstantiate(&b->gexec, g, 0) != cudaSuccess) {
      cudaGraphDestroy(g);
      set_error("graph instantiate failed");
      return -1;
    }
    b->graph = g;
  }
  if (cudaGraphLaunch(b->gexec, st) != cudaSuccess) { set_error("graph launch failed"); return -1; }
  b->launches = e.launches;
  b->ran = true;
  return 0;
}

int deflate_gpu_batch_sizes(deflate_gpu_batch* b, size_t* out_sizes) {
  if (!b || !b->ran) return -1;
  DeviceScope dev_scope(b->eng.device);
  Engine& e = b->eng;
  if (cudaDeviceSynchronize() != cudaSuccess) { set_error(cudaGetErrorString(cudaGetLastError())); return -1; }
  std::vector<Stream> s(e.streams.size());
  if (!s.empty() && cudaMemcpy(s.data(), static_cast<uint8_t*>(e.d_tables.p) + e.off_streams, s.size() * sizeof(Stream),
                               cudaMemcpyDeviceToHost) != cudaSuccess) {
    set_error("D2H failed");
    return -1;
  }
  for (size_t i = 0; i < s.size(); ++i) out_sizes[i] = s[i].error ? 0 : s[i].out_size;
  return 0;
}

int deflate_gpu_batch_verify(deflate_gpu_batch* b, int* ok) {
  if (!b || !b->ran || !ok) return -1;
  DeviceScope dev_scope(b->eng.device);
  Engine& e = b->eng;
  if (cudaDeviceSynchronize() != cudaSuccess) { set_error(cudaGetErrorString(cudaGetLastError())); return -1; }
  const size_t n = e.streams.size();
  std::vector<Stream> s(n);
  if (n && cudaMemcpy(s.data(), static_cast<uint8_t*>(e.d_tables.p) + e.off_streams, n * sizeof(Stream),
                      cudaMemcpyDeviceToHost) != cudaSuccess) {
    set_error("D2H failed");
    return -1;
  }
  // one decode job per stream (framing stripped), largest streams first
  std::vector<InflateJob> jobs(n);
  std::vector<uint64_t> ref_off(n), ref_len(n);
  std::vector<uint32_t> order;
  uint64_t vbytes = 0;
  for (size_t i = 0; i < n; ++i) {
    const uint32_t hdr = s[i].fmt == kFmtZlib ? 2 : s[i].fmt == kFmtGzip ? 10 : 0;
    const uint32_t trl = s[i].fmt == kFmtZlib ? 4 : s[i].fmt == kFmtGzip ? 8 : 0;
    InflateJob& j = jobs[i];
    ref_off[i] = s[i].in_off;
    ref_len[i] = s[i].in_len;
    if (s[i].error || s[i].out_size < hdr + trl + 2) {
      j.status = kInfData;
      continue;
    }
    j.in_off = s[i].out_off + hdr;
    j.in_len = s[i].out_size - hdr - trl;
    j.out_off = vbytes;
    j.out_cap = s[i].in_len;
    vbytes += align_up(s[i].in_len, 16);
    order.push_back(uint32_t(i));
  }
  std::stable_sort(order.begin(), order.end(), [&](uint32_t a, uint32_t c) { return jobs[a].in_len > jobs[c].in_len; });
  const size_t o_jobs = 0, o_order = align_up(n * sizeof(InflateJob), 256);
  const size_t o_roff = o_order + align_up(n * 4 + 8, 256), o_rlen = o_roff + align_up(n * 8, 256);
  const size_t o_cnt = o_rlen + align_up(n * 8, 256);
  if (!b->d_verify.ensure(vbytes + 256) || !b->d_vtab.ensure(o_cnt + 256)) return -1;
  uint8_t* vt = static_cast<uint8_t*>(b->d_vtab.p);
  InflateJob* d_jobs = reinterpret_cast<InflateJob*>(vt + o_jobs);
  uint32_t* d_order = reinterpret_cast<uint32_t*>(vt + o_order);
  uint64_t* d_roff = reinterpret_cast<uint64_t*>(vt + o_roff);
  uint64_t* d_rlen = reinterpret_cast<uint64_t*>(vt + o_rlen);
  uint32_t* d_cnt = reinterpret_cast<uint32_t*>(vt + o_cnt);
  cudaStream_t st = e.stream;
  if ((n && cudaMemcpyAsync(d_jobs, jobs.data(), n * sizeof(InflateJob), cudaMemcpyHostToDevice, st) != cudaSuccess) ||
      (!order.empty() && cudaMemcpyAsync(d_order, order.data(), order.size() * 4, cudaMemcpyHostToDevice, st) != cudaSuccess) ||
      (n && cudaMemcpyAsync(d_roff, ref_off.data(), n * 8, cudaMemcpyHostToDevice, st) != cudaSuccess) ||
      (n && cudaMemcpyAsync(d_rlen, ref_len.data(), n * 8, cudaMemcpyHostToDevice, st) != cudaSuccess)) {
    set_error("H2D failed");
    return -1;
  }
  uint8_t* dec = static_cast<uint8_t*>(b->d_verify.p);
  launch_inflate(static_cast<const uint8_t*>(e.d_out.p), dec, d_jobs, d_order, uint32_t(order.size()), d_cnt, e.sms, st);
  launch_inflate_compare(dec, static_cast<const uint8_t*>(e.d_in.p), d_jobs, d_roff, d_rlen, uint32_t(n), st);
  launch_frame_check(static_cast<const uint8_t*>(e.d_out.p),
                     reinterpret_cast<const Stream*>(static_cast<uint8_t*>(e.d_tables.p) + e.off_streams), d_jobs,
                     uint32_t(n), st);
  if (n && cudaMemcpyAsync(jobs.data(), d_jobs, n * sizeof(InflateJob), cudaMemcpyDeviceToHost, st) != cudaSuccess) return -1;
  if (cudaStreamSynchronize(st) != cudaSuccess) {
    set_error(std::string("device error: ") + cudaGetErrorString(cudaGetLastError()));
    return -1;
  }
  int bad = 0;
  for (size_t i = 0; i < n; ++i) {
    ok[i] = jobs[i].status == kInfOk ? 1 : 0;
    bad += 1 - ok[i];
  }
  return bad;
}

size_t deflate_gpu_batch_output(deflate_gpu_batch* b, size_t i, void* dst, size_t cap) {
  if (!b || !b->ran || i >= b->eng.streams.size()) return 0;
  DeviceScope dev_scope(b->eng.device);
  Engine& e = b->eng;
  Stream s{};
  if (cudaDeviceSynchronize() != cudaSuccess ||
      cudaMemcpy(&s, static_cast<uint8_t*>(e.d_tables.p) + e.off_streams + i * sizeof(Stream), sizeof s,
                 cudaMemcpyDeviceToHost) != cudaSuccess) {
    set_error("D2H failed");
    return 0;
  }
  if (s.error || s.out_size > cap) return 0;
  if (cudaMemcpy(dst, static_cast<uint8_t*>(e.d_out.p) + s.out_off, s.out_size, cudaMemcpyDeviceToHost) != cudaSuccess) {
    set_error("D2H failed");
    return 0;
  }
  return s.out_size;
}

int deflate_gpu_batch_launches(const deflate_gpu_batch* b) { return b ? b->launches : 0; }

int deflate_gpu_batch_profile(deflate_gpu_batch* b, int enable) {
  if (!b) return -1;
  DeviceScope dev_scope(b->eng.device);
  b->eng.marks.on = enable != 0;
  drop_graph(b);  // a captured graph carries no event records
  return 0;
}

int deflate_gpu_batch_phase_ms(deflate_gpu_batch* b, float* ms, int max) {
  if (!b || !ms || max < int(kNumPhases)) return -1;
  DeviceScope dev_scope(b->eng.device);
  if (cudaDeviceSynchronize() != cudaSuccess) return -1;
  b->eng.phase_ms(ms);
  return int(kNumPhases);
}

const char* deflate_gpu_phase_name(int i) {
  static const char* names[kNumPhases] = {"hash_carry", "candidates", "parse", "fixup", "lazy_match", "lazy_huffman",
                                          "lazy_encode", "plan", "join", "checksum", "frame"};
  return i >= 0 && i < int(kNumPhases) ? names[i] : "";
}

size_t deflate_gpu_compress_batch(const void* const* in, const size_t* in_sizes, void* const* out, const size_t* out_caps,
                                  size_t* out_sizes, size_t count, int level, deflate_format format) {
  if (!count) return 0;
  if (!in || !in_sizes || !out || !out_caps || !out_sizes || int(format) < 0 || int(format) > 2) return 0;
  std::lock_guard<std::mutex> lk(global_mutex());
  deflate_gpu_batch* b = host_batch();
  if (!b) return 0;
  Engine& e = b->eng;
  if (!batch_setup(b, in, nullptr, in_sizes, count, level, int(format), false, 0, e.stream)) return 0;
  if (!e.launch(e.stream)) return 0;
  std::vector<uint64_t> off(count + 1);
  std::vector<size_t> sz(count);
  uint64_t bound = 0;
  for (const Job& j : b->jobs) bound += align_up(j.out_cap, 16);
  if (!e.h_stage.ensure(bound + 16)) return 0;
  uint64_t total = 0;
  if (!batch_pack_to_host(b, e.stream, e.h_stage.p, bound + 16, off.data(), sz.data(), &total)) return 0;
  size_t done = 0;
  for (size_t i = 0; i < count; ++i) {
    if (sz[i] && sz[i] <= out_caps[i]) {
      std::memcpy(out[i], static_cast<uint8_t*>(e.h_stage.p) + off[i], sz[i]);
      out_sizes[i] = sz[i];
      ++done;
    } else {
      out_sizes[i] = 0;
    }
  }
  return done;
}

size_t deflate_gpu_compress_packed(const void* in_concat, const size_t* in_sizes, size_t count, int level,
                                   deflate_format format, void* out_packed, size_t out_capacity, uint64_t* out_offsets,
                                   size_t* out_sizes) {
  if (!count || !in_sizes || !out_packed || !out_offsets || !out_sizes || int(format) < 0 || int(format) > 2) return 0;
  uint64_t total_in = 0;
  for (size_t i = 0; i < count; ++i) total_in += in_sizes[i];
  if (total_in && !in_concat) return 0;
  std::lock_guard<std::mutex> lk(global_mutex());
  deflate_gpu_batch* b = host_batch();
  if (!b) return 0;
  Engine& e = b->eng;
  if (!batch_setup(b, nullptr, static_cast<const uint8_t*>(in_concat), in_sizes, count, level, int(format), false, 0,
                   e.stream))
    return 0;
  if (!e.launch(e.stream)) return 0;
  uint64_t total = 0;
  if (!batch_pack_to_host(b, e.stream, out_packed, out_capacity, out_offsets, out_sizes, &total)) return 0;
  return size_t(total);
}

size_t deflate_gpu_packed_bound(const size_t* in_sizes, size_t count, deflate_format format) {
  uint64_t t = 0;
  for (size_t i = 0; i < count; ++i) t += align_up(framed_bound(in_sizes[i], int(format)), 16);
  return size_t(t);
}

}  // extern "C"
