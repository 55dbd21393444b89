// server.cu -- passes in flight: a continuous-batching compression server and
// the pipelined host-to-host batch.
//
// A Lane is one engine (its own CUDA stream and device arenas) running one
// pass at a time: host planning, one host-to-device copy, the kernels, the
// device-side packing of every output, a small copy of sizes and offsets,
// then one device-to-host copy of the packed bytes.  Several lanes are in
// flight at once, so the copies of one pass overlap the kernels of another
// (H2D and D2H use the two copy engines).
//
// The server (deflate_gpu_server_*) owns a host thread that polls its lanes
// and, whenever a lane is free and the device-memory budget allows, admits
// every pending request (up to a group cap) into a new pass: requests that
// arrive while others are on the GPU join the next pass, and passes overlap
// on the device.  Each request is its own stream with deflate_compress
// semantics at its own level, so its bytes do not depend on what it was
// batched with.  A request whose output buffer is too small fails alone.
#include <cuda_runtime.h>
#include <algorithm>
#include <atomic>
#include <chrono>
#include <condition_variable>
#include <cstring>
#include <deque>
#include <mutex>
#include <new>
#include <thread>
#include <unordered_map>
#include <vector>
#include "engine_host.h"
#include "host_copy.h"
#include "../../include/orot_b200.h"

namespace orotb {

using Clock = std::chrono::steady_clock;

// Device bytes a buffer of n bytes needs in a pass (input, output slot,
// scratch), used for admission against the budget.
static uint64_t device_estimate(uint64_t n, int level) {
  const int lv = clamp_level(level);
  return align_up(n, 16) + align_up(framed_bound(n, 2), 16) + (lv >= 4 ? 7 : 6) * n + 4096;
}

struct Lane {
  Engine eng;
  std::vector<Job> jobs;
  HostBuf h_in, h_out, h_meta;
  cudaEvent_t ev_meta = nullptr, ev_data = nullptr;
  int state = 0;            // 0 idle, 1 waiting for sizes, 2 waiting for data
  uint64_t total = 0;       // packed bytes
  uint64_t est = 0;         // device bytes charged to the budget
  uint8_t* dst = nullptr;   // where the packed bytes go (h_out or the caller)
  std::vector<void*> reqs;  // server: the requests of this pass
  size_t first = 0;         // pipelined batch: first buffer of this pass
  Lane() {
    eng.use_stream_ordered_arenas();  // a lane's work runs on its engine's stream only
    cudaEventCreateWithFlags(&ev_meta, cudaEventDisableTiming);
    cudaEventCreateWithFlags(&ev_data, cudaEventDisableTiming);
  }
  ~Lane() {
    if (ev_meta) cudaEventDestroy(ev_meta);
    if (ev_data) cudaEventDestroy(ev_data);
    h_in.release();
    h_out.release();
    h_meta.release();
  }
  uint64_t* offsets() { return static_cast<uint64_t*>(h_meta.p); }
  uint64_t* sizes() { return static_cast<uint64_t*>(h_meta.p) + jobs.size() + 1; }
};

// Starts a pass over `count` buffers whose bytes are back to back at `src`
// (pinned or pageable host memory).  Jobs use deflate_compress semantics.
static bool lane_start(Lane& L, const uint8_t* src, const size_t* sizes, const int* levels, const int* fmts,
                       const size_t* caps, size_t count) {
  Engine& e = L.eng;
  L.jobs.assign(count, Job{});
  uint64_t in_total = 0, out_total = 0;
  for (size_t i = 0; i < count; ++i) {
    Job& j = L.jobs[i];
    j.in_off = in_total;
    j.in_len = sizes[i];
    j.out_off = out_total;
    const uint64_t bound = framed_bound(sizes[i], fmts[i]);
    j.out_cap = caps ? std::min<uint64_t>(caps[i], bound) : bound;
    j.level = levels[i];
    j.fmt = fmts[i];
    j.parallel = false;
    in_total += sizes[i];
    out_total += align_up(bound, 16);
  }
  if (!e.ensure_io(in_total, out_total)) return false;
  if (!e.d_pack.ensure(align_up(out_total, 256) + (2 * count + 1) * 8 + 256)) return false;
  if (!L.h_meta.ensure((2 * count + 1) * 8 + 64)) return false;
  if (in_total && cudaMemcpyAsync(e.d_in.p, src, in_total, cudaMemcpyHostToDevice, e.stream) != cudaSuccess) {
    set_error("H2D failed");
    return false;
  }
  if (!e.plan(L.jobs) || !e.launch(e.stream)) return false;
  const Work w = e.work();
  uint8_t* meta = static_cast<uint8_t*>(e.d_pack.p) + align_up(out_total, 256);
  uint64_t* d_off = reinterpret_cast<uint64_t*>(meta);
  uint64_t* d_sz = d_off + count + 1;
  launch_pack(w, d_off, d_sz, static_cast<uint8_t*>(e.d_pack.p), e.stream);
  if (cudaMemcpyAsync(L.h_meta.p, d_off, (2 * count + 1) * 8, cudaMemcpyDeviceToHost, e.stream) != cudaSuccess ||
      cudaEventRecord(L.ev_meta, e.stream) != cudaSuccess) {
    set_error("D2H failed");
    return false;
  }
  L.state = 1;
  return true;
}

// Advances a lane: once the sizes are on the host, queues the copy of the
// packed bytes to `L.dst` (needs capacity `cap`).  Returns true when the pass
// is complete.
static bool lane_poll(Lane& L, uint64_t cap, bool* failed) {
  if (L.state == 1) {
    const cudaError_t q = cudaEventQuery(L.ev_meta);
    if (q == cudaErrorNotReady) return false;
    if (q != cudaSuccess) { *failed = true; L.state = 0; return true; }
    L.total = L.offsets()[L.jobs.size()];
    if (L.total > cap) { set_error("packed output larger than its buffer"); *failed = true; L.state = 0; return true; }
    if (L.total && cudaMemcpyAsync(L.dst, L.eng.d_pack.p, L.total, cudaMemcpyDeviceToHost, L.eng.stream) != cudaSuccess) {
      *failed = true;
      L.state = 0;
      return true;
    }
    cudaEventRecord(L.ev_data, L.eng.stream);
    L.state = 2;
    return false;
  }
  if (L.state == 2) {
    const cudaError_t q = cudaEventQuery(L.ev_data);
    if (q == cudaErrorNotReady) return false;
    if (q != cudaSuccess) *failed = true;
    L.state = 0;
    return true;
  }
  return false;
}

// Runs a pass over synthetic zero bytes so that a lane's host and device
// arenas reach the size of a full group before traffic arrives (growing them
// later would free device memory, which waits for every pass in flight).
static bool lane_warm(Lane& L, uint64_t bytes, int level, uint64_t per_job) {
  const size_t count = size_t(std::max<uint64_t>(1, bytes / per_job));
  std::vector<size_t> sz(count, size_t(per_job));
  std::vector<int> lv(count, level), fm(count, int(DEFLATE_FORMAT_RAW));
  uint64_t ob = 0;
  for (size_t i = 0; i < count; ++i) ob += align_up(framed_bound(per_job, 0), 16);
  if (!L.h_in.ensure(per_job * count) || !L.h_out.ensure(ob + 16)) return false;
  std::memset(L.h_in.p, 0, per_job * count);
  L.dst = static_cast<uint8_t*>(L.h_out.p);
  if (!lane_start(L, static_cast<uint8_t*>(L.h_in.p), sz.data(), lv.data(), fm.data(), nullptr, count)) return false;
  bool failed = false;
  while (!lane_poll(L, L.h_out.cap, &failed)) std::this_thread::sleep_for(std::chrono::microseconds(50));
  return !failed;
}

// ---------------------------------------------------------------- server
struct Req {
  uint64_t id;
  const uint8_t* in;
  size_t n;
  uint8_t* out;
  size_t cap;
  int level, fmt;
  Clock::time_point t_submit, t_done;
  int status = 0;  // 0 pending, 1 done, -1 failed
  size_t out_size = 0;
};

struct Server {
  std::vector<Lane*> lanes;
  uint64_t budget, in_use = 0;
  uint64_t max_group;
  std::mutex mu;
  std::condition_variable cv_work, cv_done;
  std::deque<Req*> pending;
  std::unordered_map<uint64_t, Req*> reqs;
  uint64_t next_id = 1;
  bool stop = false;
  std::thread th;
  int device = 0;
  std::atomic<uint64_t> passes{0}, max_in_flight{0};
  CopyPool* copies = nullptr;

  void run();
};

void Server::run() {
  cudaSetDevice(device);
  std::vector<int> lv;
  std::vector<int> fm;
  std::vector<size_t> sz, cp;
  std::vector<Copy> moves;
  while (true) {
    bool progressed = false;
    // 1. advance lanes in flight; copy finished outputs to their requests
    for (Lane* L : lanes) {
      if (L->state == 0) continue;
      bool failed = false;
      if (!lane_poll(*L, L->h_out.cap, &failed)) continue;
      progressed = true;
      const uint64_t* off = L->offsets();
      const uint64_t* s = L->sizes();
      moves.clear();
      for (size_t i = 0; !failed && i < L->reqs.size(); ++i) {
        Req* r = static_cast<Req*>(L->reqs[i]);
        if (s[i] && s[i] <= r->cap) moves.push_back({r->out, static_cast<uint8_t*>(L->h_out.p) + off[i], size_t(s[i])});
      }
      copies->run(moves);
      std::lock_guard<std::mutex> lk(mu);
      const auto now = Clock::now();
      for (size_t i = 0; i < L->reqs.size(); ++i) {
        Req* r = static_cast<Req*>(L->reqs[i]);
        if (!failed && s[i] && s[i] <= r->cap) {
          r->out_size = s[i];
          r->status = 1;
        } else {
          r->status = -1;
        }
        r->t_done = now;
      }
      L->reqs.clear();
      in_use -= L->est;
      cv_done.notify_all();
    }
    // 2. admit pending requests into free lanes
    {
      std::unique_lock<std::mutex> lk(mu);
      if (stop && pending.empty()) {
        bool busy = false;
        for (Lane* L : lanes) busy |= L->state != 0;
        if (!busy) break;
      }
      for (Lane* L : lanes) {
        if (L->state != 0 || pending.empty()) continue;
        std::vector<Req*> group;
        uint64_t bytes = 0, est = 0;
        while (!pending.empty()) {
          Req* r = pending.front();
          const uint64_t e1 = device_estimate(r->n, r->level);
          if (!group.empty() && (bytes + r->n > max_group || in_use + est + e1 > budget)) break;
          if (group.empty() && in_use + e1 > budget && in_use > 0) break;  // wait for memory
          group.push_back(r);
          pending.pop_front();
          bytes += r->n;
          est += e1;
        }
        if (group.empty()) break;
        in_use += est;
        L->est = est;
        lk.unlock();
        // stage inputs back to back in pinned memory, then one pass
        uint64_t tot = 0, obound = 0;
        for (Req* r : group) { tot += r->n; obound += align_up(framed_bound(r->n, r->fmt), 16); }
        bool ok = L->h_in.ensure(std::max<uint64_t>(tot, 16)) && L->h_out.ensure(obound + 16);
        sz.resize(group.size());
        lv.resize(group.size());
        fm.resize(group.size());
        cp.resize(group.size());
        uint64_t o = 0;
        moves.clear();
        for (size_t i = 0; ok && i < group.size(); ++i) {
          moves.push_back({static_cast<uint8_t*>(L->h_in.p) + o, group[i]->in, group[i]->n});
          o += group[i]->n;
          sz[i] = group[i]->n;
          lv[i] = group[i]->level;
          fm[i] = group[i]->fmt;
          cp[i] = group[i]->cap;
        }
        if (ok) copies->run(moves);
        L->reqs.assign(group.begin(), group.end());
        L->dst = static_cast<uint8_t*>(L->h_out.p);
        if (ok) ok = lane_start(*L, static_cast<uint8_t*>(L->h_in.p), sz.data(), lv.data(), fm.data(), cp.data(),
                                group.size());
        passes++;
        lk.lock();
        if (!ok) {
          for (Req* r : group) { r->status = -1; r->t_done = Clock::now(); }
          L->reqs.clear();
          L->state = 0;
          in_use -= est;
          cv_done.notify_all();
        }
        uint64_t nf = 0;
        for (Lane* X : lanes) nf += X->state != 0;
        if (nf > max_in_flight) max_in_flight = nf;
        progressed = true;
      }
      if (!progressed) {
        bool busy = false;
        for (Lane* L : lanes) busy |= L->state != 0;
        if (!busy && pending.empty() && !stop) cv_work.wait_for(lk, std::chrono::milliseconds(2));
      }
    }
    if (!progressed) std::this_thread::sleep_for(std::chrono::microseconds(20));
  }
}

}  // namespace orotb

using namespace orotb;

struct deflate_gpu_server {
  Server s;
};

extern "C" {

deflate_gpu_server* deflate_gpu_server_new(size_t device_budget, int lanes) {
  int n = 0;
  if (cudaGetDeviceCount(&n) != cudaSuccess || n == 0) { cudaGetLastError(); set_error("no CUDA device"); return nullptr; }
  auto* srv = new (std::nothrow) deflate_gpu_server();
  if (!srv) return nullptr;
  Server& s = srv->s;
  cudaGetDevice(&s.device);
  s.budget = device_budget ? device_budget : (size_t(16) << 30);
  const int nl = lanes > 0 ? std::min(lanes, 8) : 3;
  // Groups of at most 256 MiB keep the queueing delay of a pass to a few ms;
  // a smaller budget shrinks them so that every lane can hold one.
  s.max_group = std::min<uint64_t>(256ull << 20, std::max<uint64_t>(16ull << 20, s.budget / (uint64_t(nl) * 10)));
  for (int i = 0; i < nl; ++i) {
    Lane* L = new (std::nothrow) Lane();
    if (!L) break;
    s.lanes.push_back(L);
    // size the arenas for a full group: one large lazy-level buffer, then
    // many small fast-level ones (per-buffer tables).  The lazy-level buffer
    // is 1/8 larger than a group: a group of many requests has one partial
    // tile per request more than one buffer of the same size, and growing an
    // arena mid-traffic frees device memory, which waits for every pass in
    // flight (two lanes regrowing once each cost up to 2x in L6 throughput).
    const uint64_t lazy_warm = s.max_group + s.max_group / 8;
    if (!lane_warm(*L, lazy_warm, 6, lazy_warm) || !lane_warm(*L, s.max_group, 1, 4096)) {
      for (Lane* X : s.lanes) delete X;
      delete srv;
      return nullptr;
    }
  }
  const unsigned hw = std::thread::hardware_concurrency();
  s.copies = new CopyPool(int(std::min(6u, hw / 4)));
  s.th = std::thread([&s] { s.run(); });
  return srv;
}

void deflate_gpu_server_free(deflate_gpu_server* srv) {
  if (!srv) return;
  Server& s = srv->s;
  {
    std::lock_guard<std::mutex> lk(s.mu);
    s.stop = true;
  }
  s.cv_work.notify_all();
  if (s.th.joinable()) s.th.join();
  delete s.copies;
  for (Lane* L : s.lanes) delete L;
  for (auto& kv : s.reqs) delete kv.second;
  delete srv;
}

uint64_t deflate_gpu_server_submit(deflate_gpu_server* srv, const void* in, size_t n, void* out, size_t cap, int level,
                                   deflate_format format) {
  if (!srv || (n && !in) || !out || int(format) < 0 || int(format) > 2) return 0;
  if (n > (size_t(1) << 31)) { set_error("request larger than 2 GiB"); return 0; }
  Server& s = srv->s;
  Req* r = new (std::nothrow) Req();
  if (!r) return 0;
  r->in = static_cast<const uint8_t*>(in);
  r->n = n;
  r->out = static_cast<uint8_t*>(out);
  r->cap = cap;
  r->level = level;
  r->fmt = int(format);
  r->t_submit = Clock::now();
  {
    std::lock_guard<std::mutex> lk(s.mu);
    if (s.stop) { delete r; return 0; }
    r->id = s.next_id++;
    s.reqs[r->id] = r;
    s.pending.push_back(r);
  }
  s.cv_work.notify_one();
  return r->id;
}

int deflate_gpu_server_wait(deflate_gpu_server* srv, uint64_t ticket, size_t* out_size, double* latency_s,
                            double timeout_s) {
  if (!srv) return -1;
  Server& s = srv->s;
  std::unique_lock<std::mutex> lk(s.mu);
  auto it = s.reqs.find(ticket);
  if (it == s.reqs.end()) return -1;
  Req* r = it->second;
  const auto deadline = Clock::now() + std::chrono::duration_cast<Clock::duration>(std::chrono::duration<double>(
                                          timeout_s > 0 ? timeout_s : 1e9));
  while (r->status == 0) {
    if (s.cv_done.wait_until(lk, deadline) == std::cv_status::timeout && r->status == 0) return 1;
  }
  const int st = r->status;
  if (out_size) *out_size = st == 1 ? r->out_size : 0;
  if (latency_s) *latency_s = std::chrono::duration<double>(r->t_done - r->t_submit).count();
  s.reqs.erase(it);
  delete r;
  return st == 1 ? 0 : -2;
}

int deflate_gpu_server_stats(deflate_gpu_server* srv, uint64_t* passes, uint64_t* max_in_flight) {
  if (!srv) return -1;
  if (passes) *passes = srv->s.passes.load();
  if (max_in_flight) *max_in_flight = srv->s.max_in_flight.load();
  return 0;
}

// Pipelined host-to-host batch: the buffers are split into groups of about
// group_bytes; lanes overlap the copies of one group with the kernels of
// another.  Outputs land in out_packed at 16-byte aligned offsets, each
// group's region starting where the bound of the previous groups ends.
size_t deflate_gpu_compress_pipelined(const void* in_concat, const size_t* in_sizes, size_t count, int level,
                                      deflate_format format, void* out_packed, size_t out_capacity,
                                      uint64_t* out_offsets, size_t* out_sizes, size_t group_bytes, int lanes) {
  if (!count || !in_sizes || !out_packed || !out_offsets || !out_sizes || int(format) < 0 || int(format) > 2) return 0;
  std::lock_guard<std::mutex> lk(global_mutex());
  // lanes are kept per device (the calling thread's) and reused across calls
  static std::vector<Lane*> pools[kMaxDevices];
  const int dev = current_device();
  if (dev < 0) return 0;
  std::vector<Lane*>& pool = pools[dev];
  const int nl = lanes > 0 ? std::min(lanes, 8) : 6;
  while (int(pool.size()) < nl) {
    Lane* L = new (std::nothrow) Lane();
    if (!L || !L->eng.ok) { delete L; set_error("lane set-up failed"); return 0; }
    pool.push_back(L);
  }
  // defaults measured on B200 over PCIe 5 (10,000 buffers, 5.13 GB): 256 MiB
  // groups with 6 lanes keep both copy directions busier than 512 MiB with 4
  if (!group_bytes) group_bytes = size_t(256) << 20;
  // groups: contiguous buffer ranges
  std::vector<size_t> gfirst, gcount;
  std::vector<uint64_t> gsrc, gdst, gcap;
  uint64_t src = 0, dst = 0, total = 0;
  for (size_t i = 0; i < count; ++i) total += in_sizes[i];
  // Group sizes ramp up (1/8, 1/4, 1/2 of group_bytes) at the start and down
  // at the end, so that the first kernels start after a short copy and the
  // last copies out follow a short pass: the pipeline fills and drains fast.
  const uint64_t G = group_bytes;
  for (size_t i = 0; i < count;) {
    const uint64_t left = total - src;
    const size_t gi = gfirst.size();
    uint64_t target = gi < 3 ? (G >> (3 - gi)) : G;
    if (left <= G / 8) target = left;
    else if (left <= 3 * G / 8) target = std::min(target, left - G / 8);
    else if (left <= 7 * G / 8) target = std::min(target, left - 3 * G / 8);
    else if (left - target < 7 * G / 8) target = left - 7 * G / 8;
    size_t j = i;
    uint64_t b = 0, ob = 0;
    while (j < count && (j == i || b + in_sizes[j] <= target)) {
      b += in_sizes[j];
      ob += align_up(framed_bound(in_sizes[j], int(format)), 16);
      ++j;
    }
    gfirst.push_back(i);
    gcount.push_back(j - i);
    gsrc.push_back(src);
    gdst.push_back(dst);
    gcap.push_back(ob);
    src += b;
    dst += ob;
    i = j;
  }
  if (dst > out_capacity) { set_error("out_capacity below deflate_gpu_packed_bound()"); return 0; }
  const uint8_t* in = static_cast<const uint8_t*>(in_concat);
  uint8_t* out = static_cast<uint8_t*>(out_packed);
  // Pageable caller memory goes through each lane's pinned buffers, copied by
  // the copy threads (a DMA from pageable memory is staged by the driver on
  // one thread); pinned caller memory is read and written by DMA directly.
  auto pageable = [](const void* p) {
    cudaPointerAttributes a{};
    if (cudaPointerGetAttributes(&a, p) != cudaSuccess) {
      cudaGetLastError();
      return true;
    }
    return a.type == cudaMemoryTypeUnregistered;
  };
  const bool stage_in = total && pageable(in), stage_out = pageable(out);
  std::vector<int> lv(count, level), fm(count, int(format));
  std::vector<int> lane_group(nl, -1);
  size_t next = 0, done_groups = 0;
  bool ok = true;
  uint64_t end = 0;
  while (done_groups < gfirst.size() && ok) {
    bool progressed = false;
    for (int k = 0; k < nl; ++k) {
      Lane& L = *pool[k];
      if (L.state != 0) {
        bool failed = false;
        if (lane_poll(L, gcap[lane_group[k]], &failed)) {
          progressed = true;
          if (failed) { ok = false; break; }
          const int g = lane_group[k];
          for (size_t i = 0; i < gcount[g]; ++i) {
            out_offsets[gfirst[g] + i] = gdst[g] + L.offsets()[i];
            out_sizes[gfirst[g] + i] = L.sizes()[i];
          }
          if (stage_out) host_copy(out + gdst[g], L.h_out.p, L.total);
          end = std::max<uint64_t>(end, gdst[g] + L.total);
          ++done_groups;
          lane_group[k] = -1;
        }
      }
      if (L.state == 0 && next < gfirst.size()) {
        const size_t g = next++;
        lane_group[k] = int(g);
        const uint8_t* gin = in + gsrc[g];
        const uint64_t gbytes = (g + 1 < gfirst.size() ? gsrc[g + 1] : total) - gsrc[g];
        if (stage_in) {
          if (!L.h_in.ensure(std::max<uint64_t>(gbytes, 16))) { ok = false; break; }
          host_copy(L.h_in.p, gin, gbytes);
          gin = static_cast<const uint8_t*>(L.h_in.p);
        }
        if (stage_out) {
          if (!L.h_out.ensure(std::max<uint64_t>(gcap[g], 16))) { ok = false; break; }
          L.dst = static_cast<uint8_t*>(L.h_out.p);
        } else {
          L.dst = out + gdst[g];
        }
        if (!lane_start(L, gin, in_sizes + gfirst[g], lv.data(), fm.data(), nullptr, gcount[g])) {
          ok = false;
          break;
        }
        progressed = true;
      }
    }
    if (!progressed) std::this_thread::sleep_for(std::chrono::microseconds(10));
  }
  if (!ok) {
    for (Lane* L : pool) {
      cudaStreamSynchronize(L->eng.stream);
      L->state = 0;
    }
    return 0;
  }
  out_offsets[count] = end;
  return size_t(end);
}

}  // extern "C"
