// batch.cu - many independent jobs, each an input with its own sequence of pairs, run as
// segmented launches of the super-tile kernel; and the request loop that serves them.
//
// A batch is a set of jobs resident in one device arena. Round r applies every job's r-th
// pair: per carry class (free; bordered L <= 4; bordered 5 <= L <= 32) ONE segmented launch
// covers the super-tiles of all jobs of that class, work split by super-tiles, not by jobs.
// Lengths pass between rounds in device memory (n_dev / len_out), so the rounds of a batch
// are a fixed sequence of launches over fixed tables: it is captured once as a CUDA graph
// per round count and replayed for every batch. Per job the device holds its input and two
// ping-pong buffers; a job whose output outgrows them is flagged by the kernel (nothing is
// written out of range) and run again through a Session, which sizes exactly.
//
// Serving: submit() copies the request into page-locked memory and queues it; a dispatcher
// thread forms a batch from the queue whenever one of two slots is free, admitting requests
// in arrival order while their device footprint fits the arena (the HBM budget); a
// completion thread downloads the results of a finished batch and releases its memory. So
// requests that arrive while a batch is on the GPU form the next batch and run beside it.
#include <cuda_runtime.h>

#include <algorithm>
#include <atomic>
#include <chrono>
#include <condition_variable>
#include <cstdint>
#include <cstring>
#include <deque>
#include <map>
#include <memory>
#include <mutex>
#include <string>
#include <thread>
#include <unordered_map>
#include <vector>

#include "cuda_replace.h"
#include "host_pool.h"
#include "replace_kernels.h"

#define CR_EXPORT extern "C" __attribute__((visibility("default")))

namespace {

using crb::ApplyResult;
using crb::SegJob;
using crb::SegLaunch;
using crb::SegPair;
using crb::TileIncl;

constexpr int kClasses = 3;     // free; small with L <= 4; small with 5 <= L <= 32
constexpr int kMaxRounds = 16;  // pairs per job in a segmented batch; longer chains use a Session
constexpr int kSlots = 2;       // batches in flight
constexpr size_t kAlign = 256;

size_t rup(size_t x, size_t q) { return (x + q - 1) / q * q; }

double now_us() {
  return std::chrono::duration<double, std::micro>(std::chrono::steady_clock::now().time_since_epoch()).count();
}

int pair_class(const SegPair& q) { return q.mode == crb::kModeFree ? 0 : (q.L <= 4 ? 1 : 2); }
const uint32_t kClassLmax[kClasses] = {crb::kSegMaxL, 4, crb::kSegMaxL};

// ------------------------------------------------------------------ device arena
// First-fit allocator over one device allocation (the HBM budget of a server).
class Arena {
 public:
  ~Arena() {
    if (base_) cudaFree(base_);
  }
  cudaError_t init(size_t bytes) {
    bytes = rup(bytes, 2u << 20);
    cudaError_t e = cudaMalloc(&base_, bytes);
    if (e != cudaSuccess) return e;
    size_ = bytes;
    free_[0] = bytes;
    return cudaSuccess;
  }
  bool alloc(size_t n, size_t* off) {
    n = rup(n ? n : 1, kAlign);
    for (auto it = free_.begin(); it != free_.end(); ++it) {
      if (it->second >= n) {
        *off = it->first;
        const size_t rest = it->second - n;
        const size_t at = it->first + n;
        free_.erase(it);
        if (rest) free_[at] = rest;
        used_[*off] = n;
        in_use_ += n;
        return true;
      }
    }
    return false;
  }
  void release(size_t off) {
    auto u = used_.find(off);
    if (u == used_.end()) return;
    size_t start = off, len = u->second;
    in_use_ -= len;
    used_.erase(u);
    auto nx = free_.lower_bound(start);
    if (nx != free_.end() && start + len == nx->first) {
      len += nx->second;
      nx = free_.erase(nx);
    }
    if (nx != free_.begin()) {
      auto pv = std::prev(nx);
      if (pv->first + pv->second == start) {
        start = pv->first;
        len += pv->second;
        free_.erase(pv);
      }
    }
    free_[start] = len;
  }
  uint8_t* base() const { return base_; }
  size_t size() const { return size_; }
  size_t in_use() const { return in_use_; }

 private:
  uint8_t* base_ = nullptr;
  size_t size_ = 0, in_use_ = 0;
  std::map<size_t, size_t> free_, used_;
};

// ------------------------------------------------------------------ jobs
struct Job {
  unsigned long long ticket = 0;
  std::vector<std::vector<uint8_t>> pats, reps;
  std::vector<SegPair> seg;  // one per pair when the job fits segmented launches
  bool seg_ok = false;
  uint8_t* hin = nullptr;    // page-locked copy of the input
  size_t n = 0;
  size_t cap = 0;            // capacity of each ping-pong buffer
  size_t off_in = 0, off_a = 0, off_b = 0;
  bool placed = false;
  // result
  uint8_t* hout = nullptr;
  size_t out_len = 0;
  int rc = 0;
  bool done = false;
  bool via_session = false;
  int retries = 0;           // segmented reruns after an overflow
  double t_submit = 0, t_done = 0;
  unsigned int tenant = 0;   // admission is counted against this tenant's budget (0: no budget)
  size_t charged = 0;        // arena bytes counted against the tenant while the job is placed
};

constexpr int kCancelled = -8;       // the request was cancelled before it reached the device
constexpr int kOverTenantBudget = -9;  // the request alone needs more than its tenant's budget

// Largest intermediate length of a job's chain in the worst case (every pattern position a
// match), capped at `lim`.
long double chain_worst(const Job& j, long double lim) {
  long double wc = (long double)j.n, mx = wc;
  for (const SegPair& q : j.seg) {
    if (q.R > q.L) wc += (long double)((unsigned long long)wc / q.L) * (long double)(q.R - q.L);
    mx = std::max(mx, wc);
    if (mx > lim) break;
  }
  return std::min(mx, lim);
}

// Output capacity of a job's ping-pong buffers: the worst case of its chain when that is at
// most 4n + 1 MiB (no overflow possible), else 4n + 1 MiB (an overflow reruns the job).
size_t job_capacity(const Job& j) {
  const long double lim = 4.0L * (long double)j.n + (long double)(1u << 20);
  return rup((size_t)chain_worst(j, lim) + 16, kAlign);
}

// ------------------------------------------------------------------ autotuning
struct ClassCfg {
  uint32_t nsub = 8;
  int grid = 0;  // CTAs of the persistent grid
  float us = 0;  // measured time of the chosen candidate on the tuning batch
};

struct Tuning {
  ClassCfg cls[kClasses];
  bool done = false;
};

std::mutex g_tune_mu;
std::map<int, Tuning> g_tuning;  // by device

// ------------------------------------------------------------------ slots
struct Slot {
  cudaStream_t st = nullptr;
  cudaEvent_t ev_meta = nullptr;
  cudaEvent_t ev_t0 = nullptr, ev_t1 = nullptr;  // batch start / rounds done (timing)
  int max_jobs = 0;
  SegJob* d_jobs = nullptr;  // [kMaxRounds][kClasses][max_jobs]
  SegJob* h_jobs = nullptr;
  unsigned int* d_njobs = nullptr;  // [kMaxRounds * kClasses]
  unsigned int* h_njobs = nullptr;
  SegPair* d_pairs = nullptr;  // [max_jobs * kMaxRounds]
  SegPair* h_pairs = nullptr;
  ApplyResult* d_res = nullptr;  // [max_jobs]
  ApplyResult* h_res = nullptr;
  unsigned long long* d_lens = nullptr;  // [max_jobs * 2]
  unsigned long long* h_lens = nullptr;
  unsigned int* d_ctl = nullptr;  // total, sched[2], epoch[2]
  unsigned int* d_tile_job = nullptr;
  uint32_t* status = nullptr;
  TileIncl* incl = nullptr;
  unsigned long long* agg = nullptr;
  long long* tile_last = nullptr;
  unsigned long long* rec = nullptr;
  size_t max_tiles = 0;
  cudaGraphExec_t graphs[kMaxRounds + 1] = {};
  std::vector<Job*> jobs;  // the batch in flight
  int rounds = 0;
  bool busy = false;
  double t_launch = 0;

  SegLaunch launch_desc(int r, int c, const Tuning& tu) const {
    SegLaunch sl{};
    sl.jobs = d_jobs + ((size_t)r * kClasses + c) * max_jobs;
    sl.njobs = d_njobs + r * kClasses + c;
    sl.pairs = d_pairs;
    sl.res = d_res;
    sl.total = d_ctl;
    sl.sched = d_ctl + 1;
    sl.epoch = d_ctl + 3;
    sl.tile_job = d_tile_job;
    sl.status = status;
    sl.incl = incl;
    sl.agg = agg;
    sl.tile_last = tile_last;
    sl.rec = rec;
    sl.max_tiles = (unsigned int)max_tiles;
    sl.agg_stride = crb::kSegMaxL;
    sl.mode = c == 0 ? crb::kModeFree : crb::kModeSmall;
    sl.Lmax = kClassLmax[c];
    sl.Rmax = crb::kSegMaxR;
    sl.nsub = tu.cls[c].nsub;
    return sl;
  }

  void drop_graphs() {
    for (auto& g : graphs)
      if (g) {
        cudaGraphExecDestroy(g);
        g = nullptr;
      }
  }

  void free_scratch() {
    for (void* q : {(void*)d_tile_job, (void*)status, (void*)incl, (void*)agg, (void*)tile_last, (void*)rec})
      if (q) cudaFree(q);
    d_tile_job = nullptr;
    status = nullptr;
    incl = nullptr;
    agg = nullptr;
    tile_last = nullptr;
    rec = nullptr;
    max_tiles = 0;
  }

  cudaError_t ensure_tiles(size_t need) {
    if (need <= max_tiles) return cudaSuccess;
    drop_graphs();  // the graphs hold the old pointers
    free_scratch();
    const size_t cap = rup(need + need / 4 + 256, 1024);
    cudaError_t e = cudaMalloc(&d_tile_job, cap * sizeof(unsigned int));
    if (e == cudaSuccess) e = cudaMalloc(&status, cap * sizeof(uint32_t));
    if (e == cudaSuccess) e = cudaMalloc(&incl, cap * sizeof(TileIncl));
    if (e == cudaSuccess) e = cudaMalloc(&agg, cap * crb::kSegMaxL * sizeof(unsigned long long));
    if (e == cudaSuccess) e = cudaMalloc(&tile_last, cap * sizeof(long long));
    if (e == cudaSuccess) e = cudaMalloc(&rec, cap * 2 * sizeof(unsigned long long));
    if (e == cudaSuccess) e = cudaMemsetAsync(status, 0, cap * sizeof(uint32_t), st);
    if (e == cudaSuccess) e = cudaMemsetAsync(rec, 0, cap * 2 * sizeof(unsigned long long), st);
    if (e == cudaSuccess) e = cudaStreamSynchronize(st);
    if (e != cudaSuccess) {
      free_scratch();
      return e;
    }
    max_tiles = cap;
    return cudaSuccess;
  }

  cudaError_t init(int mj) {
    max_jobs = mj;
    const size_t tables = (size_t)kMaxRounds * kClasses * max_jobs;
    cudaError_t e = cudaStreamCreateWithFlags(&st, cudaStreamNonBlocking);
    if (e == cudaSuccess) e = cudaEventCreateWithFlags(&ev_meta, cudaEventDisableTiming);
    if (e == cudaSuccess) e = cudaEventCreate(&ev_t0);
    if (e == cudaSuccess) e = cudaEventCreate(&ev_t1);
    if (e == cudaSuccess) e = cudaMalloc(&d_jobs, tables * sizeof(SegJob));
    if (e == cudaSuccess) e = cudaMallocHost(&h_jobs, tables * sizeof(SegJob));
    if (e == cudaSuccess) e = cudaMalloc(&d_njobs, kMaxRounds * kClasses * sizeof(unsigned int));
    if (e == cudaSuccess) e = cudaMallocHost(&h_njobs, kMaxRounds * kClasses * sizeof(unsigned int));
    if (e == cudaSuccess) e = cudaMalloc(&d_pairs, (size_t)max_jobs * kMaxRounds * sizeof(SegPair));
    if (e == cudaSuccess) e = cudaMallocHost(&h_pairs, (size_t)max_jobs * kMaxRounds * sizeof(SegPair));
    if (e == cudaSuccess) e = cudaMalloc(&d_res, (size_t)max_jobs * sizeof(ApplyResult));
    if (e == cudaSuccess) e = cudaMallocHost(&h_res, (size_t)max_jobs * sizeof(ApplyResult));
    if (e == cudaSuccess) e = cudaMalloc(&d_lens, (size_t)max_jobs * 2 * sizeof(unsigned long long));
    if (e == cudaSuccess) e = cudaMallocHost(&h_lens, (size_t)max_jobs * 2 * sizeof(unsigned long long));
    if (e == cudaSuccess) e = cudaMalloc(&d_ctl, 8 * sizeof(unsigned int));
    if (e == cudaSuccess) e = cudaMemsetAsync(d_ctl, 0, 8 * sizeof(unsigned int), st);
    if (e == cudaSuccess) e = cudaStreamSynchronize(st);
    return e;
  }

  void destroy() {
    if (st) cudaStreamSynchronize(st);
    drop_graphs();
    free_scratch();
    for (void* q : {(void*)d_jobs, (void*)d_njobs, (void*)d_pairs, (void*)d_res, (void*)d_lens, (void*)d_ctl})
      if (q) cudaFree(q);
    for (void* q : {(void*)h_jobs, (void*)h_njobs, (void*)h_pairs, (void*)h_res, (void*)h_lens})
      if (q) cudaFreeHost(q);
    if (ev_meta) cudaEventDestroy(ev_meta);
    if (ev_t0) cudaEventDestroy(ev_t0);
    if (ev_t1) cudaEventDestroy(ev_t1);
    if (st) cudaStreamDestroy(st);
    st = nullptr;
  }
};

// ------------------------------------------------------------------ engine
// Device side of a server: arena, two slots, tuning. Not thread-safe by itself.
class Engine {
 public:
  int device = 0;
  Arena arena;
  Slot slots[kSlots];
  Tuning tune;
  int max_jobs = 0;
  crb::HostArena* hstage = nullptr;  // page-locked staging of inputs and results

  // page-locked host memory: the staging area first, the pool when it is full
  uint8_t* host_get(size_t n, cudaError_t* e) {
    *e = cudaSuccess;
    uint8_t* p = hstage ? hstage->alloc(n) : nullptr;
    return p ? p : static_cast<uint8_t*>(crb::host_pinned_pool().get(n, e));
  }
  std::atomic<unsigned long long> seg_launches{0}, graph_launches{0};
  // uploads + rounds on the device; result downloads (host wall), in microseconds
  std::atomic<unsigned long long> gpu_us{0}, download_us{0};

  cudaError_t init(size_t budget, int mj) {
    cudaGetDevice(&device);
    max_jobs = mj;
    cudaError_t e = arena.init(budget);
    if (e == cudaSuccess) {
      hstage = new crb::HostArena();
      e = hstage->init(std::min<size_t>(8ull << 30, std::max<size_t>(64u << 20, budget / 4)));
      if (e != cudaSuccess) {
        delete hstage;
        hstage = nullptr;
      } else {
        crb::host_arena_register(hstage);
      }
    }
    for (int i = 0; i < kSlots && e == cudaSuccess; ++i) e = slots[i].init(max_jobs);
    if (e == cudaSuccess) e = autotune();
    return e;
  }
  void destroy() {
    for (auto& s : slots) s.destroy();
    if (hstage) crb::host_arena_close(hstage);  // freed once the callers release its last block
    hstage = nullptr;
  }

  // Device footprint of a job: input + two ping-pong buffers (each + 64 B of read slack).
  static size_t footprint(const Job& j) {
    return rup(j.n + 64, kAlign) + 2 * rup(j.cap + 64, kAlign);
  }

  bool place(Job& j) {
    size_t a, b, c;
    if (!arena.alloc(j.n + 64, &a)) return false;
    if (!arena.alloc(j.cap + 64, &b)) {
      arena.release(a);
      return false;
    }
    if (!arena.alloc(j.cap + 64, &c)) {
      arena.release(a);
      arena.release(b);
      return false;
    }
    j.off_in = a;
    j.off_a = b;
    j.off_b = c;
    j.placed = true;
    return true;
  }
  void unplace(Job& j) {
    if (!j.placed) return;
    arena.release(j.off_in);
    arena.release(j.off_a);
    arena.release(j.off_b);
    j.placed = false;
  }

  // Enqueue a batch on slot s: uploads, the rounds (graph), read-back of lengths and flags.
  cudaError_t launch(Slot& s, std::vector<Job*>& batch) {
    const int nj = (int)batch.size();
    int rounds = 0;
    size_t tiles = 0;
    for (Job* j : batch) {
      rounds = std::max(rounds, (int)j->seg.size());
      tiles += (j->cap + crb::kTile - 1) / crb::kTile + 1;
    }
    cudaError_t e = s.ensure_tiles(tiles);
    if (e != cudaSuccess) return e;
    uint8_t* base = arena.base();
    // tables
    memset(s.h_njobs, 0, kMaxRounds * kClasses * sizeof(unsigned int));
    for (int i = 0; i < nj; ++i) {
      Job& j = *batch[(size_t)i];
      s.h_lens[2 * i] = j.n;
      s.h_lens[2 * i + 1] = 0;
      for (int r = 0; r < (int)j.seg.size(); ++r) {
        const SegPair& q = j.seg[(size_t)r];
        const int pi = i * kMaxRounds + r;
        s.h_pairs[pi] = q;
        const int c = pair_class(q);
        const int k = (int)s.h_njobs[r * kClasses + c]++;
        SegJob& J = s.h_jobs[((size_t)r * kClasses + c) * s.max_jobs + k];
        memset(&J, 0, sizeof(J));
        J.in = base + (r == 0 ? j.off_in : ((r & 1) ? j.off_a : j.off_b));
        J.out = base + ((r & 1) ? j.off_b : j.off_a);
        J.n_dev = s.d_lens + 2 * i + (r & 1);
        J.len_out = s.d_lens + 2 * i + ((r + 1) & 1);
        J.out_cap = j.cap;
        J.pair = (unsigned int)pi;
        J.res = (unsigned int)i;
      }
    }
    // uploads: inputs, lengths, pairs, job tables, counts; results cleared
    e = cudaEventRecord(s.ev_t0, s.st);
    for (int i = 0; i < nj && e == cudaSuccess; ++i) {
      Job& j = *batch[(size_t)i];
      if (j.n) e = cudaMemcpyAsync(base + j.off_in, j.hin, j.n, cudaMemcpyHostToDevice, s.st);
    }
    if (e == cudaSuccess)
      e = cudaMemcpyAsync(s.d_lens, s.h_lens, (size_t)nj * 2 * sizeof(unsigned long long), cudaMemcpyHostToDevice,
                          s.st);
    if (e == cudaSuccess && rounds > 0)
      e = cudaMemcpyAsync(s.d_pairs, s.h_pairs, (size_t)nj * kMaxRounds * sizeof(SegPair), cudaMemcpyHostToDevice,
                          s.st);
    for (int r = 0; r < rounds && e == cudaSuccess; ++r)
      for (int c = 0; c < kClasses && e == cudaSuccess; ++c) {
        const unsigned int k = s.h_njobs[r * kClasses + c];
        const size_t off = ((size_t)r * kClasses + c) * s.max_jobs;
        if (k) e = cudaMemcpyAsync(s.d_jobs + off, s.h_jobs + off, k * sizeof(SegJob), cudaMemcpyHostToDevice, s.st);
      }
    if (e == cudaSuccess)
      e = cudaMemcpyAsync(s.d_njobs, s.h_njobs, kMaxRounds * kClasses * sizeof(unsigned int), cudaMemcpyHostToDevice,
                          s.st);
    if (e == cudaSuccess) e = cudaMemsetAsync(s.d_res, 0, (size_t)nj * sizeof(ApplyResult), s.st);
    if (e != cudaSuccess) return e;
    // the rounds
    if (rounds > 0) {
      e = run_rounds(s, rounds);
      if (e != cudaSuccess) return e;
    }
    e = cudaEventRecord(s.ev_t1, s.st);
    if (e != cudaSuccess) return e;
    // lengths and flags back
    e = cudaMemcpyAsync(s.h_lens, s.d_lens, (size_t)nj * 2 * sizeof(unsigned long long), cudaMemcpyDeviceToHost, s.st);
    if (e == cudaSuccess)
      e = cudaMemcpyAsync(s.h_res, s.d_res, (size_t)nj * sizeof(ApplyResult), cudaMemcpyDeviceToHost, s.st);
    if (e == cudaSuccess) e = cudaEventRecord(s.ev_meta, s.st);
    s.rounds = rounds;
    return e;
  }

  // The launch sequence of `rounds` rounds, from a graph captured at its first use.
  cudaError_t run_rounds(Slot& s, int rounds) {
    if (!s.graphs[rounds]) {
      cudaGraph_t g = nullptr;
      cudaError_t e = cudaStreamBeginCapture(s.st, cudaStreamCaptureModeThreadLocal);
      if (e != cudaSuccess) return e;
      cudaError_t le = cudaSuccess;
      for (int r = 0; r < rounds && le == cudaSuccess; ++r)
        for (int c = 0; c < kClasses && le == cudaSuccess; ++c)
          le = crb::launch_seg(s.launch_desc(r, c, tune), s.st, tune.cls[c].grid);
      e = cudaStreamEndCapture(s.st, &g);
      if (le != cudaSuccess) {
        if (g) cudaGraphDestroy(g);
        return le;
      }
      if (e != cudaSuccess) return e;
      e = cudaGraphInstantiate(&s.graphs[rounds], g, 0);
      cudaGraphDestroy(g);
      if (e != cudaSuccess) {
        s.graphs[rounds] = nullptr;
        return e;
      }
    }
    seg_launches += 2ull * rounds * kClasses;
    ++graph_launches;
    return cudaGraphLaunch(s.graphs[rounds], s.st);
  }

  // After ev_meta: download every job's output; jobs that failed on the device are returned
  // for a Session run. The caller releases the batch's arena memory.
  cudaError_t finish(Slot& s, std::vector<Job*>* rerun) {
    cudaError_t e = cudaEventSynchronize(s.ev_meta);
    if (e != cudaSuccess) return e;
    float ms = 0;
    if (cudaEventElapsedTime(&ms, s.ev_t0, s.ev_t1) == cudaSuccess) gpu_us += (unsigned long long)(ms * 1000.0f);
    const double t_dl = now_us();
    uint8_t* base = arena.base();
    const int nj = (int)s.jobs.size();
    for (int i = 0; i < nj && e == cudaSuccess; ++i) {
      Job& j = *s.jobs[(size_t)i];
      const ApplyResult& r = s.h_res[i];
      const int k = (int)j.seg.size();
      if (r.error_epoch != 0u || r.overflow_epoch != 0u) {
        if (r.error_epoch == 0u) {
          // overflow: the length that did not fit is in one of the two length slots
          j.out_len = (size_t)std::max(s.h_lens[2 * i], s.h_lens[2 * i + 1]);
        } else {
          j.out_len = 0;
          j.retries = 1 << 20;  // an error: no segmented rerun
        }
        rerun->push_back(&j);
        continue;
      }
      const size_t len = (size_t)s.h_lens[2 * i + (k & 1)];
      const size_t off = k == 0 ? j.off_in : ((k & 1) ? j.off_a : j.off_b);
      j.out_len = len;
      if (len) {
        j.hout = host_get(len, &e);
        if (!j.hout) break;
        e = cudaMemcpyAsync(j.hout, base + off, len, cudaMemcpyDeviceToHost, s.st);
      }
    }
    if (e == cudaSuccess) e = cudaStreamSynchronize(s.st);
    download_us += (unsigned long long)(now_us() - t_dl);
    return e;
  }

 private:
  // Pick the super-tile size of each class by timing segmented launches of a synthetic batch
  // (48 jobs of 2 MiB over a 16-symbol alphabet, one pair of the class each).
  cudaError_t autotune() {
    {
      std::lock_guard<std::mutex> g(g_tune_mu);
      auto it = g_tuning.find(device);
      if (it != g_tuning.end() && it->second.done) {
        tune = it->second;
        return cudaSuccess;
      }
    }
    int sms = 0;
    cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, device);
    Slot& s = slots[0];
    const int nj = std::min(48, max_jobs);
    const size_t n = 2u << 20;
    uint8_t* buf = nullptr;
    unsigned long long* lens = nullptr;
    cudaError_t e = cudaMalloc(&buf, (size_t)nj * 2 * (n + 4096));
    if (e != cudaSuccess) return e;
    e = cudaMalloc(&lens, (size_t)nj * 2 * sizeof(unsigned long long));
    std::vector<uint8_t> host(n);
    uint32_t x = 12345u;
    for (size_t i = 0; i < n; ++i) {
      x = x * 1664525u + 1013904223u;
      host[i] = (uint8_t)('a' + ((x >> 24) & 15u));
    }
    for (int i = 0; i < nj && e == cudaSuccess; ++i)
      e = cudaMemcpy(buf + (size_t)i * 2 * (n + 4096), host.data(), n, cudaMemcpyHostToDevice);
    if (e == cudaSuccess) e = s.ensure_tiles((size_t)nj * (n / crb::kTile + 2));
    // two representative pairs per class, at the short and the long end of its pattern
    // lengths (the candidate test and the tables cost differently there): borderless L = 2 and
    // L = 12; bordered L = 2 and L = 4; bordered L = 6 and L = 24
    const uint8_t p0[4] = {'a', 'b', 'c', 'd'}, p0b[12] = {'a', 'b', 'c', 'd', 'e', 'f', 'g', 'h', 'i', 'j', 'k', 'l'};
    const uint8_t p1[2] = {'a', 'a'}, p1b[4] = {'a', 'b', 'a', 'b'};
    const uint8_t p2[6] = {'a', 'b', 'c', 'a', 'b', 'c'};
    uint8_t p2b[24];
    for (int i = 0; i < 24; ++i) p2b[i] = (uint8_t)("abac"[i % 4]);
    const uint8_t rp[8] = {'X', 'Y', 'Z', 'W', 'V', 'U', 'T', 'S'};
    SegPair q[kClasses][2];
    crb::make_seg_pair(q[0][0], p0, 2, rp, 6);
    crb::make_seg_pair(q[0][1], p0b, 12, rp, 3);
    crb::make_seg_pair(q[1][0], p1, 2, rp, 1);
    crb::make_seg_pair(q[1][1], p1b, 4, rp, 2);
    crb::make_seg_pair(q[2][0], p2, 6, rp, 3);
    crb::make_seg_pair(q[2][1], p2b, 24, rp, 5);
    cudaEvent_t e0 = nullptr, e1 = nullptr;
    if (e == cudaSuccess) e = cudaEventCreate(&e0);
    if (e == cudaSuccess) e = cudaEventCreate(&e1);
    for (int c = 0; c < kClasses && e == cudaSuccess; ++c) {
      std::vector<uint32_t> cands;
      for (uint32_t ns : {2u, 4u, 8u})
        if (c == 0 || ns * kClassLmax[c] <= 128u) cands.push_back(ns);
      if (c == 2) cands = {1u, 2u, 4u};
      float best = 1e30f;
      ClassCfg pick;
      // super-tile size x CTAs per SM (the full occupancy, one less, half), each timed on both
      // representative pairs; the sum decides
      for (uint32_t ns : cands)
      for (int occ_step = 0; occ_step < 3 && e == cudaSuccess; ++occ_step) {
      float tot = 0;
      int grid = 0;
      for (int qv = 0; qv < 2 && e == cudaSuccess; ++qv) {
        memset(s.h_njobs, 0, kMaxRounds * kClasses * sizeof(unsigned int));
        s.h_njobs[c] = (unsigned int)nj;
        std::vector<unsigned long long> hl((size_t)nj * 2, 0);
        for (int i = 0; i < nj; ++i) {
          SegJob& J = s.h_jobs[(size_t)c * s.max_jobs + i];
          memset(&J, 0, sizeof(J));
          J.in = buf + (size_t)i * 2 * (n + 4096);
          J.out = buf + (size_t)i * 2 * (n + 4096) + n + 4096;
          J.n_dev = lens + 2 * i;
          J.len_out = lens + 2 * i + 1;
          J.out_cap = n + 2048;
          J.pair = 0;
          J.res = (unsigned int)i;
          hl[(size_t)2 * i] = n;
        }
        s.h_pairs[0] = q[c][qv];
        Tuning tu = tune;
        tu.cls[c].nsub = ns;
        SegLaunch sl = s.launch_desc(0, c, tu);
        const int per_sm = crb::seg_ctas_per_sm(sl);
        if (per_sm < 0) {
          e = cudaErrorUnknown;
          break;
        }
        const int occ = occ_step == 0 ? per_sm : (occ_step == 1 ? per_sm - 1 : per_sm / 2);
        if (occ < 1 || (occ_step == 2 && occ == per_sm - 1)) {
          tot = 1e30f;  // not a distinct candidate
          break;
        }
        grid = occ * sms;
        e = cudaMemcpy(lens, hl.data(), hl.size() * sizeof(unsigned long long), cudaMemcpyHostToDevice);
        if (e == cudaSuccess)
          e = cudaMemcpy(s.d_jobs + (size_t)c * s.max_jobs, s.h_jobs + (size_t)c * s.max_jobs, nj * sizeof(SegJob),
                         cudaMemcpyHostToDevice);
        if (e == cudaSuccess)
          e = cudaMemcpy(s.d_njobs, s.h_njobs, kMaxRounds * kClasses * sizeof(unsigned int), cudaMemcpyHostToDevice);
        if (e == cudaSuccess) e = cudaMemcpy(s.d_pairs, s.h_pairs, sizeof(SegPair), cudaMemcpyHostToDevice);
        for (int it = 0; it < 4 && e == cudaSuccess; ++it) {
          e = cudaMemsetAsync(s.d_res, 0, (size_t)nj * sizeof(ApplyResult), s.st);
          if (e == cudaSuccess) e = cudaEventRecord(e0, s.st);
          if (e == cudaSuccess) e = crb::launch_seg(sl, s.st, grid);
          if (e == cudaSuccess) e = cudaEventRecord(e1, s.st);
          if (e == cudaSuccess) e = cudaEventSynchronize(e1);
          float ms = 0;
          if (e == cudaSuccess) e = cudaEventElapsedTime(&ms, e0, e1);
          if (it > 0) tot += ms;  // the first run warms up
        }
      }
        if (e != cudaSuccess) break;
        if (tot < best) {
          best = tot;
          pick.nsub = ns;
          pick.grid = grid;
          pick.us = tot / 6.0f * 1000.0f;
        }
      }
      tune.cls[c] = pick;
    }
    if (e0) cudaEventDestroy(e0);
    if (e1) cudaEventDestroy(e1);
    cudaFree(buf);
    if (lens) cudaFree(lens);
    if (e != cudaSuccess) return e;
    tune.done = true;
    std::lock_guard<std::mutex> g(g_tune_mu);
    g_tuning[device] = tune;
    return cudaSuccess;
  }
};

// ------------------------------------------------------------------ Session path
// A job outside the segmented limits, or one whose output outgrew its buffers, runs
// through a Session (exact sizing), one pair at a time on the device.
int run_with_session(Job& j, Engine& eng) {
  void* h = nullptr;
  int rc = cuda_replace_open(&h, j.hin, j.n);
  if (rc != 0) return rc;
  const int k = (int)j.pats.size();
  std::vector<const uint8_t*> pp((size_t)std::max(k, 1)), rr((size_t)std::max(k, 1));
  std::vector<int> pl((size_t)std::max(k, 1)), rl((size_t)std::max(k, 1));
  for (int i = 0; i < k; ++i) {
    pp[(size_t)i] = j.pats[(size_t)i].data();
    pl[(size_t)i] = (int)j.pats[(size_t)i].size();
    rr[(size_t)i] = j.reps[(size_t)i].data();
    rl[(size_t)i] = (int)j.reps[(size_t)i].size();
  }
  size_t nl = 0;
  if (k) rc = cuda_replace_apply_batch(h, pp.data(), pl.data(), rr.data(), rl.data(), k, &nl);
  if (rc == 0) rc = cuda_replace_length(h, &nl);
  if (rc == 0 && nl) {
    cudaError_t e;
    j.hout = eng.host_get(nl, &e);  // page-locked staging, not a fresh pinned block
    if (!j.hout) rc = (int)e;
    if (rc == 0) rc = cuda_replace_result_into(h, j.hout, nl, &j.out_len);
  } else if (rc == 0) {
    j.out_len = 0;
  }
  cuda_replace_close(h);
  j.via_session = true;
  return rc;
}

// ------------------------------------------------------------------ server
class Server {
 public:
  explicit Server(int device) : device_(device) {}

  int open(size_t budget, int max_jobs) {
    cudaSetDevice(device_);
    cudaError_t e = eng_.init(budget, max_jobs);
    if (e != cudaSuccess) {
      eng_.destroy();
      return (int)e;
    }
    run_ = true;
    dispatcher_ = std::thread([this] { dispatch_loop(); });
    completer_ = std::thread([this] { complete_loop(); });
    fallback_ = std::thread([this] { fallback_loop(); });
    return 0;
  }

  // Finishes every submitted request, then stops the threads and frees the device memory.
  void close() {
    {
      std::unique_lock<std::mutex> lk(mu_);
      cv_.wait(lk, [&] { return drained(); });
      run_ = false;
    }
    cv_.notify_all();
    if (dispatcher_.joinable()) dispatcher_.join();
    if (completer_.joinable()) completer_.join();
    if (fallback_.joinable()) fallback_.join();
    cudaSetDevice(device_);
    for (auto& kv : jobs_) {
      crb::host_free(kv.second->hin);
      crb::host_free(kv.second->hout);
    }
    jobs_.clear();
    eng_.destroy();
  }

  int submit(const uint8_t* src, size_t n, const uint8_t** pats, const int* pat_lens, const uint8_t** reps,
             const int* rep_lens, int count, unsigned long long* ticket, unsigned int tenant = 0) {
    auto j = std::make_unique<Job>();
    j->t_submit = now_us();
    j->n = n;
    j->tenant = tenant;
    j->seg_ok = count <= kMaxRounds;
    for (int i = 0; i < count; ++i) {
      if (pat_lens[i] < 0 || rep_lens[i] < 0 || (pat_lens[i] && !pats[i]) || (rep_lens[i] && !reps[i])) return -1;
      if ((uint32_t)pat_lens[i] > crb::kMaxLen || (uint32_t)rep_lens[i] > crb::kMaxLen) return -4;
      j->pats.emplace_back(pats[i], pats[i] + pat_lens[i]);
      j->reps.emplace_back(reps[i], reps[i] + rep_lens[i]);
      SegPair q;
      if (j->seg_ok && crb::make_seg_pair(q, pats[i], (uint32_t)pat_lens[i], reps[i], (uint32_t)rep_lens[i]))
        j->seg.push_back(q);
      else
        j->seg_ok = false;
    }
    if (!j->seg_ok) j->seg.clear();
    cudaError_t e;
    j->hin = eng_.host_get(n ? n : 1, &e);
    if (!j->hin) return (int)e;
    if (n) crb::parallel_memcpy(j->hin, src, n);
    if (j->seg_ok) j->cap = job_capacity(*j);
    std::lock_guard<std::mutex> g(mu_);
    if (j->seg_ok && tenant) {
      const auto b = tenant_budget_.find(tenant);
      if (b != tenant_budget_.end() && Engine::footprint(*j) > b->second) {
        crb::host_free(j->hin);  // it could never be admitted within the tenant's budget
        return kOverTenantBudget;
      }
    }
    j->ticket = ++next_ticket_;
    *ticket = j->ticket;
    Job* raw = j.get();
    jobs_[j->ticket] = std::move(j);
    if (raw->seg_ok && Engine::footprint(*raw) <= eng_.arena.size())
      pending_.push_back(raw);
    else
      fallback_q_.push_back(raw);
    cv_.notify_all();
    return 0;
  }

  // 0: done (*out_host/*out_len filled, ownership passes to the caller); 1: not done within
  // timeout_ms (< 0: wait without limit); -1: unknown ticket; other: the job's error code.
  int wait(unsigned long long ticket, int timeout_ms, uint8_t** out_host, size_t* out_len) {
    std::unique_lock<std::mutex> lk(mu_);
    auto it = jobs_.find(ticket);
    if (it == jobs_.end()) return -1;
    Job* j = it->second.get();
    auto ready = [&] { return j->done; };
    if (timeout_ms < 0)
      cv_.wait(lk, ready);
    else if (!cv_.wait_for(lk, std::chrono::milliseconds(timeout_ms), ready))
      return 1;
    const int rc = j->rc;
    *out_host = j->hout;
    *out_len = j->out_len;
    j->hout = nullptr;
    jobs_.erase(it);
    return rc;
  }

  // 0: the request was still queued and is cancelled (a wait then returns kCancelled); 1: it is
  // on the device, running or done, and completes normally; -1: unknown ticket.
  int cancel(unsigned long long ticket) {
    std::lock_guard<std::mutex> g(mu_);
    auto it = jobs_.find(ticket);
    if (it == jobs_.end()) return -1;
    Job* j = it->second.get();
    if (j->done) return 1;
    auto pi = std::find(pending_.begin(), pending_.end(), j);
    if (pi != pending_.end()) {
      pending_.erase(pi);
    } else {
      auto fi = std::find(fallback_q_.begin(), fallback_q_.end(), j);
      if (fi == fallback_q_.end()) return 1;
      fallback_q_.erase(fi);
    }
    crb::host_free(j->hin);
    j->hin = nullptr;
    if (j->hout) {
      crb::host_free(j->hout);
      j->hout = nullptr;
    }
    j->out_len = 0;
    j->rc = kCancelled;
    j->done = true;
    ++cancelled_;
    cv_.notify_all();
    return 0;
  }

  // Device bytes (arena) the tenant's requests may hold at once; 0 removes the limit.
  void set_tenant_budget(unsigned int tenant, size_t bytes) {
    std::lock_guard<std::mutex> g(mu_);
    if (bytes)
      tenant_budget_[tenant] = bytes;
    else
      tenant_budget_.erase(tenant);
    cv_.notify_all();
  }
  void tenant_usage(unsigned int tenant, unsigned long long* in_use, unsigned long long* peak) {
    std::lock_guard<std::mutex> g(mu_);
    auto u = tenant_inuse_.find(tenant);
    auto k = tenant_peak_.find(tenant);
    *in_use = u == tenant_inuse_.end() ? 0 : u->second;
    *peak = k == tenant_peak_.end() ? 0 : k->second;
  }

  void stats(CudaReplaceServerStats* st) {
    std::lock_guard<std::mutex> g(mu_);
    memset(st, 0, sizeof(*st));
    st->jobs_done = jobs_done_;
    st->jobs_via_session = jobs_session_;
    st->batches = batches_;
    st->bytes_in = bytes_in_;
    st->bytes_out = bytes_out_;
    st->kernel_launches = eng_.seg_launches;
    st->graph_launches = eng_.graph_launches;
    st->pending = (unsigned long long)(pending_.size() + fallback_q_.size());
    st->cancelled = cancelled_;
    st->arena_bytes = eng_.arena.size();
    st->arena_peak_bytes = arena_peak_;
    st->gpu_us = (double)eng_.gpu_us.load();
    st->download_us = (double)eng_.download_us.load();
    st->session_us = session_us_;
    std::vector<double> l = lat_;
    if (!l.empty()) {
      std::sort(l.begin(), l.end());
      auto q = [&](double f) { return l[std::min(l.size() - 1, (size_t)(f * (double)(l.size() - 1) + 0.5))]; };
      st->p50_us = q(0.50);
      st->p99_us = q(0.99);
      st->max_us = l.back();
    }
    for (int c = 0; c < 3; ++c) {
      st->tile_bytes[c] = eng_.tune.cls[c].nsub * (unsigned int)crb::kTile;
      st->grid_ctas[c] = eng_.tune.cls[c].grid;
    }
  }

  void reset_stats() {
    std::lock_guard<std::mutex> g(mu_);
    lat_.clear();
    jobs_done_ = jobs_session_ = batches_ = bytes_in_ = bytes_out_ = 0;
    session_us_ = 0;
    eng_.gpu_us = 0;
    eng_.download_us = 0;
  }

 private:
  void mark_done(Job* j, int rc) {
    std::lock_guard<std::mutex> g(mu_);
    j->rc = rc;
    j->t_done = now_us();
    j->done = true;
    lat_.push_back(j->t_done - j->t_submit);
    ++jobs_done_;
    if (j->via_session) ++jobs_session_;
    bytes_in_ += j->n;
    bytes_out_ += j->out_len;
    crb::host_free(j->hin);
    j->hin = nullptr;
    cv_.notify_all();
  }

  void uncharge(Job* j) {  // with mu_ held
    if (j->tenant && j->charged) {
      unsigned long long& u = tenant_inuse_[j->tenant];
      u = u >= j->charged ? u - j->charged : 0;
    }
    j->charged = 0;
  }

  int free_slot() const {
    for (int i = 0; i < kSlots; ++i)
      if (!eng_.slots[i].busy) return i;
    return -1;
  }
  bool drained() const {
    if (!pending_.empty() || !fallback_q_.empty() || !launched_.empty() || running_fallback_) return false;
    for (int i = 0; i < kSlots; ++i)
      if (eng_.slots[i].busy) return false;
    return true;
  }

  void dispatch_loop() {
    cudaSetDevice(device_);
    std::unique_lock<std::mutex> lk(mu_);
    for (;;) {
      cv_.wait(lk, [&] { return !run_ || (!pending_.empty() && free_slot() >= 0); });
      if (!run_) break;
      const int si = free_slot();
      Slot& s = eng_.slots[si];
      std::vector<Job*> batch;
      // admit in arrival order while the job table and the arena (the HBM budget) have room; a
      // request whose tenant has its budget in use waits without holding back other tenants
      Job* blocked_front = nullptr;  // the oldest request not held back by its tenant
      for (auto it = pending_.begin(); it != pending_.end() && (int)batch.size() < eng_.max_jobs;) {
        Job* j = *it;
        const auto b = j->tenant ? tenant_budget_.find(j->tenant) : tenant_budget_.end();
        const size_t fp = Engine::footprint(*j);
        if (b != tenant_budget_.end() && tenant_inuse_[j->tenant] + fp > b->second) {
          ++it;
          continue;
        }
        if (!eng_.place(*j)) {
          blocked_front = j;
          break;
        }
        j->charged = fp;
        if (j->tenant) {
          const unsigned long long u = (tenant_inuse_[j->tenant] += fp);
          unsigned long long& pk = tenant_peak_[j->tenant];
          pk = std::max(pk, u);
        }
        batch.push_back(j);
        it = pending_.erase(it);
      }
      if (batch.empty()) {
        bool in_flight = false;
        for (int i = 0; i < kSlots; ++i) in_flight = in_flight || eng_.slots[i].busy;
        if (in_flight) {
          // the oldest request does not fit beside the batches in flight, or every queued
          // request waits for its tenant's requests in flight: wait for a batch to end
          const unsigned long long c0 = completions_;
          cv_.wait(lk, [&] { return !run_ || completions_ != c0; });
        } else if (blocked_front) {
          // it does not fit in the empty arena (fragmentation or a large request): Session path
          pending_.erase(std::find(pending_.begin(), pending_.end(), blocked_front));
          fallback_q_.push_back(blocked_front);
          cv_.notify_all();
        } else {
          // nothing in flight holds a tenant's budget now (a budget was lowered meanwhile): the
          // oldest request goes to the Session path rather than wait for nothing
          fallback_q_.push_back(pending_.front());
          pending_.pop_front();
          cv_.notify_all();
        }
        continue;
      }
      arena_peak_ = std::max(arena_peak_, (unsigned long long)eng_.arena.in_use());
      s.busy = true;
      s.jobs = batch;
      s.t_launch = now_us();
      ++batches_;
      lk.unlock();
      const cudaError_t e = eng_.launch(s, s.jobs);
      if (e != cudaSuccess) cudaStreamSynchronize(s.st);
      lk.lock();
      if (e != cudaSuccess) {
        // nothing of the batch is trusted: every job goes to the Session path
        for (Job* j : s.jobs) {
          eng_.unplace(*j);
          uncharge(j);
          fallback_q_.push_back(j);
        }
        s.jobs.clear();
        s.busy = false;
        ++completions_;
        cv_.notify_all();
        continue;
      }
      launched_.push_back(si);
      cv_.notify_all();
    }
  }

  void complete_loop() {
    cudaSetDevice(device_);
    std::unique_lock<std::mutex> lk(mu_);
    for (;;) {
      cv_.wait(lk, [&] { return !run_ || !launched_.empty(); });
      if (launched_.empty()) break;  // only when closing, after the queues drained
      const int si = launched_.front();
      launched_.pop_front();
      Slot& s = eng_.slots[si];
      lk.unlock();
      std::vector<Job*> rerun;
      const cudaError_t e = eng_.finish(s, &rerun);
      for (Job* j : s.jobs)
        if (std::find(rerun.begin(), rerun.end(), j) == rerun.end()) mark_done(j, e == cudaSuccess ? 0 : (int)e);
      lk.lock();
      for (Job* j : s.jobs) {
        eng_.unplace(*j);
        uncharge(j);
      }
      // an overflowed job runs again, first in the queue, with buffers grown past the length
      // that overflowed (at most twice); otherwise, and after an error, through a Session
      for (auto it = rerun.rbegin(); it != rerun.rend(); ++it) {
        Job* j = *it;
        if (j->retries < 2) {
          const long double need = (long double)j->out_len * 1.5L + (long double)(1u << 20);
          const long double grown = std::max(need, 2.0L * (long double)j->cap);
          j->cap = rup((size_t)std::min(grown, chain_worst(*j, grown)) + 16, kAlign);
          ++j->retries;
          j->out_len = 0;
          if (Engine::footprint(*j) <= eng_.arena.size()) {
            pending_.push_front(j);
            continue;
          }
        }
        fallback_q_.push_back(j);
      }
      s.jobs.clear();
      s.busy = false;
      ++completions_;
      cv_.notify_all();
    }
  }

  void fallback_loop() {
    cudaSetDevice(device_);
    std::unique_lock<std::mutex> lk(mu_);
    for (;;) {
      cv_.wait(lk, [&] { return !run_ || !fallback_q_.empty(); });
      if (fallback_q_.empty()) break;  // only when closing, after the queues drained
      Job* j = fallback_q_.front();
      fallback_q_.pop_front();
      running_fallback_ = true;
      lk.unlock();
      if (j->hout) {
        crb::host_free(j->hout);
        j->hout = nullptr;
      }
      const double t0 = now_us();
      const int rc = run_with_session(*j, eng_);
      const double dt = now_us() - t0;
      mark_done(j, rc);
      lk.lock();
      session_us_ += dt;
      running_fallback_ = false;
      cv_.notify_all();
    }
  }

  int device_;
  Engine eng_;
  std::mutex mu_;
  std::condition_variable cv_;
  bool run_ = false;
  std::thread dispatcher_, completer_, fallback_;
  std::deque<Job*> pending_, fallback_q_;
  std::deque<int> launched_;
  unsigned long long completions_ = 0;
  bool running_fallback_ = false;
  std::unordered_map<unsigned long long, std::unique_ptr<Job>> jobs_;
  unsigned long long next_ticket_ = 0;
  std::vector<double> lat_;
  unsigned long long jobs_done_ = 0, jobs_session_ = 0, batches_ = 0, bytes_in_ = 0, bytes_out_ = 0;
  unsigned long long arena_peak_ = 0;
  unsigned long long cancelled_ = 0;
  double session_us_ = 0;
  std::unordered_map<unsigned int, size_t> tenant_budget_;
  std::unordered_map<unsigned int, unsigned long long> tenant_inuse_, tenant_peak_;
};

size_t default_budget() {
  size_t fr = 0, tot = 0;
  if (cudaMemGetInfo(&fr, &tot) != cudaSuccess) return 1ull << 30;
  return std::max<size_t>(64u << 20, fr / 10 * 4);  // 40% of the free memory
}

}  // namespace

CR_EXPORT int cuda_replace_server_open(void** srv, size_t hbm_budget, int max_jobs_per_batch) {
  if (!srv) return -1;
  *srv = nullptr;
  int dev = 0;
  cudaError_t e = cudaGetDevice(&dev);
  if (e != cudaSuccess) return (int)e;
  auto* s = new (std::nothrow) Server(dev);
  if (!s) return -2;
  const int mj = max_jobs_per_batch > 0 ? std::min(max_jobs_per_batch, 65536) : 4096;
  const int rc = s->open(hbm_budget ? hbm_budget : default_budget(), mj);
  if (rc != 0) {
    delete s;
    return rc;
  }
  *srv = s;
  return 0;
}

CR_EXPORT int cuda_replace_server_submit(void* srv, const uint8_t* src, size_t n, const uint8_t** pats,
                                         const int* pat_lens, const uint8_t** reps, const int* rep_lens, int count,
                                         unsigned long long* ticket) {
  if (!srv || !ticket || (n && !src) || count < 0 || (count > 0 && (!pats || !pat_lens || !reps || !rep_lens)))
    return -1;
  return static_cast<Server*>(srv)->submit(src, n, pats, pat_lens, reps, rep_lens, count, ticket);
}

CR_EXPORT int cuda_replace_server_submit_tenant(void* srv, unsigned int tenant, const uint8_t* src, size_t n,
                                                const uint8_t** pats, const int* pat_lens, const uint8_t** reps,
                                                const int* rep_lens, int count, unsigned long long* ticket) {
  if (!srv || !ticket || (n && !src) || count < 0 || (count > 0 && (!pats || !pat_lens || !reps || !rep_lens)))
    return -1;
  return static_cast<Server*>(srv)->submit(src, n, pats, pat_lens, reps, rep_lens, count, ticket, tenant);
}

CR_EXPORT int cuda_replace_server_cancel(void* srv, unsigned long long ticket) {
  if (!srv) return -1;
  return static_cast<Server*>(srv)->cancel(ticket);
}

CR_EXPORT int cuda_replace_server_set_tenant_budget(void* srv, unsigned int tenant, size_t bytes) {
  if (!srv || tenant == 0) return -1;
  static_cast<Server*>(srv)->set_tenant_budget(tenant, bytes);
  return 0;
}

CR_EXPORT int cuda_replace_server_tenant_usage(void* srv, unsigned int tenant, unsigned long long* in_use,
                                               unsigned long long* peak) {
  if (!srv || !in_use || !peak) return -1;
  static_cast<Server*>(srv)->tenant_usage(tenant, in_use, peak);
  return 0;
}

CR_EXPORT int cuda_replace_server_wait(void* srv, unsigned long long ticket, int timeout_ms, uint8_t** out_host,
                                       size_t* out_len) {
  if (!srv || !out_host || !out_len) return -1;
  *out_host = nullptr;
  *out_len = 0;
  return static_cast<Server*>(srv)->wait(ticket, timeout_ms, out_host, out_len);
}

CR_EXPORT int cuda_replace_server_stats(void* srv, CudaReplaceServerStats* st) {
  if (!srv || !st) return -1;
  static_cast<Server*>(srv)->stats(st);
  return 0;
}

CR_EXPORT int cuda_replace_server_reset_stats(void* srv) {
  if (!srv) return -1;
  static_cast<Server*>(srv)->reset_stats();
  return 0;
}

CR_EXPORT void cuda_replace_server_close(void* srv) {
  if (!srv) return;
  auto* s = static_cast<Server*>(srv);
  s->close();
  delete s;
}

namespace {
// One server per device shared by every cuda_replace_jobs call, opened at the first call and
// reopened larger when a call's inputs need more device memory; calls are serialised. Released
// by cuda_replace_jobs_release (the process exit reclaims it otherwise).
constexpr int kJobsDevices = 64;
std::mutex g_jobs_mu;
void* g_jobs_srv[kJobsDevices] = {};
size_t g_jobs_budget[kJobsDevices] = {};
}  // namespace

CR_EXPORT int cuda_replace_jobs(int njobs, const uint8_t** srcs, const size_t* src_lens, const int* pair_counts,
                                const uint8_t** pats, const int* pat_lens, const uint8_t** reps, const int* rep_lens,
                                uint8_t** out_hosts, size_t* out_lens) {
  if (njobs < 0 || (njobs > 0 && (!srcs || !src_lens || !pair_counts || !out_hosts || !out_lens))) return -1;
  if (njobs == 0) return 0;
  size_t total_pairs = 0, total_bytes = 0, largest = 0;
  for (int i = 0; i < njobs; ++i) {
    if (pair_counts[i] < 0) return -1;
    total_pairs += (size_t)pair_counts[i];
    total_bytes += src_lens[i];
    largest = std::max(largest, src_lens[i]);
    out_hosts[i] = nullptr;
    out_lens[i] = 0;
  }
  if (total_pairs && (!pats || !pat_lens || !reps || !rep_lens)) return -1;
  int dev = 0;
  cudaError_t e = cudaGetDevice(&dev);
  if (e != cudaSuccess) return (int)e;
  if (dev < 0 || dev >= kJobsDevices) return (int)cudaErrorInvalidDevice;
  std::lock_guard<std::mutex> g(g_jobs_mu);
  // device memory for this call: its inputs with their ping-pong buffers (about 9 bytes per input
  // byte), at least room for its largest job, within 40% of the free memory
  const size_t want = std::max<size_t>(64u << 20, std::min<size_t>(9 * total_bytes, 9 * largest + (512u << 20)));
  if (!g_jobs_srv[dev] || g_jobs_budget[dev] < std::min(want, default_budget() + g_jobs_budget[dev])) {
    if (g_jobs_srv[dev]) {
      cuda_replace_server_close(g_jobs_srv[dev]);
      g_jobs_srv[dev] = nullptr;
    }
    const size_t budget = std::min(default_budget(), std::max(want, (size_t)256 << 20));
    int rc = cuda_replace_server_open(&g_jobs_srv[dev], budget, 4096);
    if (rc != 0) {
      g_jobs_srv[dev] = nullptr;
      return rc;
    }
    g_jobs_budget[dev] = budget;
  }
  void* srv = g_jobs_srv[dev];
  std::vector<unsigned long long> tickets((size_t)njobs, 0);
  size_t p = 0;
  int rc = 0;
  for (int i = 0; i < njobs && rc == 0; ++i) {
    rc = cuda_replace_server_submit(srv, srcs[i], src_lens[i], pats ? pats + p : nullptr,
                                    pat_lens ? pat_lens + p : nullptr, reps ? reps + p : nullptr,
                                    rep_lens ? rep_lens + p : nullptr, pair_counts[i], &tickets[(size_t)i]);
    p += (size_t)pair_counts[i];
  }
  int first_err = rc;
  for (int i = 0; i < njobs; ++i) {
    if (!tickets[(size_t)i]) continue;
    const int r = cuda_replace_server_wait(srv, tickets[(size_t)i], -1, &out_hosts[i], &out_lens[i]);
    if (r != 0 && first_err == 0) first_err = r;
  }
  if (first_err != 0)
    for (int i = 0; i < njobs; ++i)
      if (out_hosts[i]) {
        cuda_free_host(out_hosts[i]);
        out_hosts[i] = nullptr;
        out_lens[i] = 0;
      }
  return first_err;
}

CR_EXPORT void cuda_replace_jobs_release(void) {
  std::lock_guard<std::mutex> g(g_jobs_mu);
  for (int d = 0; d < kJobsDevices; ++d)
    if (g_jobs_srv[d]) {
      int cur = 0;
      cudaGetDevice(&cur);
      cudaSetDevice(d);
      cuda_replace_server_close(g_jobs_srv[d]);
      cudaSetDevice(cur);
      g_jobs_srv[d] = nullptr;
      g_jobs_budget[d] = 0;
    }
}
