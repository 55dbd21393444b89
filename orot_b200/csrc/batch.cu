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

// Lays out `count` buffers, uploads them, plans the pass.
static bool batch_setup(deflate_gpu_batch* b, const void* const* in, const size_t* sizes, size_t count, int level,
                        int fmt, bool parallel, size_t block) {
  Engine& e = b->eng;
  drop_graph(b);
  b->jobs.assign(count, Job{});
  uint64_t in_total = 0, out_total = 0;
  for (size_t i = 0; i < count; ++i) {
    Job& j = b->jobs[i];
    j.in_off = in_total;
    j.in_len = sizes[i];
    j.out_off = out_total;
    j.out_cap = framed_bound(sizes[i], fmt);
    j.level = level;
    j.fmt = fmt;
    j.parallel = parallel;
    j.block_size = block;
    in_total += align_up(sizes[i], 16);
    out_total += align_up(j.out_cap, 16);
  }
  if (!e.ensure_io(in_total, out_total) || !e.h_stage.ensure(std::max<uint64_t>(in_total, 16))) return false;
  uint8_t* st = static_cast<uint8_t*>(e.h_stage.p);
  for (size_t i = 0; i < count; ++i)
    if (sizes[i]) std::memcpy(st + b->jobs[i].in_off, in[i], sizes[i]);
  if (in_total && cudaMemcpyAsync(e.d_in.p, st, in_total, cudaMemcpyHostToDevice, e.stream) != cudaSuccess) {
    set_error("H2D failed");
    return false;
  }
  if (cudaStreamSynchronize(e.stream) != cudaSuccess) { set_error("H2D sync failed"); return false; }
  return e.plan(b->jobs);
}

extern "C" {

deflate_gpu_batch* deflate_gpu_batch_new(void) {
  int n = 0;
  if (cudaGetDeviceCount(&n) != cudaSuccess || n == 0) { cudaGetLastError(); set_error("no CUDA device"); return nullptr; }
  return new (std::nothrow) deflate_gpu_batch();
}

void deflate_gpu_batch_free(deflate_gpu_batch* b) { delete b; }

int deflate_gpu_batch_load(deflate_gpu_batch* b, const void* concat, const size_t* sizes, size_t count, int level,
                           deflate_format format, int parallel, size_t block_size) {
  if (!b || (count && (!sizes || !concat)) || int(format) < 0 || int(format) > 2) return -1;
  std::vector<const void*> ptrs(count);
  const uint8_t* p = static_cast<const uint8_t*>(concat);
  for (size_t i = 0; i < count; ++i) { ptrs[i] = p; p += sizes[i]; }
  return batch_setup(b, ptrs.data(), sizes, count, level, int(format), parallel != 0, block_size) ? 0 : -1;
}

int deflate_gpu_batch_run(deflate_gpu_batch* b, void* cuda_stream, int use_graph) {
  if (!b) return -1;
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

size_t deflate_gpu_batch_output(deflate_gpu_batch* b, size_t i, void* dst, size_t cap) {
  if (!b || !b->ran || i >= b->eng.streams.size()) return 0;
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

size_t deflate_gpu_compress_batch(const void* const* in, const size_t* in_sizes, void* const* out, const size_t* out_caps,
                                  size_t* out_sizes, size_t count, int level, deflate_format format) {
  if (!count) return 0;
  if (!in || !in_sizes || !out || !out_caps || !out_sizes || int(format) < 0 || int(format) > 2) return 0;
  std::lock_guard<std::mutex> lk(global_mutex());
  static deflate_gpu_batch* gb = new deflate_gpu_batch();
  deflate_gpu_batch* b = gb;
  Engine& e = b->eng;
  if (!batch_setup(b, in, in_sizes, count, level, int(format), false, 0)) return 0;
  if (!e.launch(e.stream)) return 0;
  // pack on the device, one copy back
  const Work w = e.work();
  DevBuf& pk = e.d_pack;
  uint64_t out_total = 0;
  for (const Job& j : b->jobs) out_total += align_up(j.out_cap, 16);
  if (!pk.ensure(out_total + 16 + (count + 1) * 8)) return 0;
  uint64_t* d_off = reinterpret_cast<uint64_t*>(static_cast<uint8_t*>(pk.p) + align_up(out_total, 256));
  k_pack_offsets<<<1, 1024, 0, e.stream>>>(w.streams, w.nstreams, d_off);
  k_pack<<<w.nstreams, 256, 0, e.stream>>>(w.streams, w.nstreams, d_off, w.out, static_cast<uint8_t*>(pk.p));
  std::vector<Stream> s(count);
  std::vector<uint64_t> off(count + 1);
  if (cudaMemcpyAsync(s.data(), w.streams, count * sizeof(Stream), cudaMemcpyDeviceToHost, e.stream) != cudaSuccess ||
      cudaMemcpyAsync(off.data(), d_off, (count + 1) * 8, cudaMemcpyDeviceToHost, e.stream) != cudaSuccess ||
      cudaStreamSynchronize(e.stream) != cudaSuccess) {
    set_error("D2H failed");
    return 0;
  }
  if (!e.h_stage.ensure(off[count] + 16)) return 0;
  if (off[count] && (cudaMemcpyAsync(e.h_stage.p, pk.p, off[count], cudaMemcpyDeviceToHost, e.stream) != cudaSuccess ||
                     cudaStreamSynchronize(e.stream) != cudaSuccess)) {
    set_error("D2H failed");
    return 0;
  }
  size_t done = 0;
  for (size_t i = 0; i < count; ++i) {
    const uint64_t n = s[i].error ? 0 : s[i].out_size;
    if (n && n <= out_caps[i]) {
      std::memcpy(out[i], static_cast<uint8_t*>(e.h_stage.p) + off[i], n);
      out_sizes[i] = n;
      ++done;
    } else {
      out_sizes[i] = 0;
    }
  }
  return done;
}

}  // extern "C"
