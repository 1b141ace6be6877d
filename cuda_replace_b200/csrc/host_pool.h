// host_pool.h - page-locked host memory handed to callers (freed with cuda_free_host).
#pragma once

#include <cuda_runtime.h>

#include <cstddef>
#include <cstdint>
#include <condition_variable>
#include <cstring>
#include <iterator>
#include <map>
#include <mutex>
#include <thread>
#include <unordered_map>
#include <vector>

namespace crb {

static inline size_t pool_round_up(size_t x, size_t q) { return (x + q - 1) / q * q; }

// Results are handed to the caller in page-locked memory that it frees with cuda_free_host.
// Pinning fresh memory for every result costs far more than the copy itself, so freed
// blocks are kept (up to kMaxIdle bytes) and reused for later results of similar size.
class PinnedPool {
 public:
  void* get(size_t n, cudaError_t* err) {
    const size_t want = pool_round_up(n ? n : 1, 64 << 10);
    {
      std::lock_guard<std::mutex> g(mu_);
      auto it = idle_.lower_bound(want);
      if (it != idle_.end() && it->first <= want + want / 2 + (64ull << 20)) {
        void* p = it->second.first;
        idle_bytes_ -= it->first;
        lru_.erase(it->second.second);
        idle_.erase(it);
        *err = cudaSuccess;
        return p;
      }
    }
    void* p = nullptr;
    *err = cudaMallocHost(&p, want);
    if (*err != cudaSuccess) return nullptr;
    std::lock_guard<std::mutex> g(mu_);
    sizes_[p] = want;
    return p;
  }
  // Keep p for reuse. Over kMaxIdle idle bytes, the blocks idle the longest are released first
  // (so a large block handed back, the one most likely wanted again soon, is kept).
  void put(void* p) {
    if (!p) return;
    std::vector<void*> evict;
    {
      std::lock_guard<std::mutex> g(mu_);
      auto s = sizes_.find(p);
      if (s == sizes_.end()) {
        evict.push_back(p);  // not ours: release directly
      } else {
        const unsigned long long seq = ++seq_;
        idle_.emplace(s->second, std::make_pair(p, seq));
        lru_.emplace(seq, std::make_pair(s->second, p));
        idle_bytes_ += s->second;
        while (idle_bytes_ > kMaxIdle && !lru_.empty()) {
          auto old = lru_.begin();
          if (old->first == seq && lru_.size() > 1) old = std::next(old);  // not the block just returned
          const size_t sz = old->second.first;
          void* q = old->second.second;
          auto range = idle_.equal_range(sz);
          for (auto it = range.first; it != range.second; ++it)
            if (it->second.first == q) {
              idle_.erase(it);
              break;
            }
          idle_bytes_ -= sz;
          sizes_.erase(q);
          evict.push_back(q);
          lru_.erase(old);
        }
      }
    }
    for (void* q : evict) cudaFreeHost(q);
  }

 private:
  static constexpr size_t kMaxIdle = 24ull << 30;
  std::mutex mu_;
  std::multimap<size_t, std::pair<void*, unsigned long long>> idle_;  // size -> (block, put order)
  std::map<unsigned long long, std::pair<size_t, void*>> lru_;        // put order -> (size, block)
  std::unordered_map<void*, size_t> sizes_;
  size_t idle_bytes_ = 0;
  unsigned long long seq_ = 0;
};

// The process-wide pool (never destroyed: CUDA may be torn down first at exit).
PinnedPool& host_pinned_pool();

// A few persistent host threads for large memcpys (pageable <-> page-locked staging, result
// copies): spawning threads per copy would cost more than the copy of a 32 MiB chunk.
class CopyWorkers {
 public:
  static CopyWorkers& get() {
    static CopyWorkers* w = new CopyWorkers();  // never destroyed (threads parked at exit)
    return *w;
  }
  // dst[0, n) = src[0, n), split across the workers and the calling thread
  void copy(void* dst, const void* src, size_t n) {
    const size_t kMin = 8u << 20;
    const unsigned parts = nthreads_ + 1;
    if (n < kMin || nthreads_ == 0) {
      memcpy(dst, src, n);
      return;
    }
    const size_t part = pool_round_up((n + parts - 1) / parts, 4096);
    std::unique_lock<std::mutex> lk(mu_);
    caller_.wait(lk, [&] { return !busy_; });  // one parallel copy at a time
    busy_ = true;
    dst_ = static_cast<char*>(dst);
    src_ = static_cast<const char*>(src);
    n_ = n;
    part_ = part;
    next_ = 1;  // part 0 is the caller's
    pending_ = 0;
    for (unsigned i = 1; i < parts; ++i)
      if (part * i < n) ++pending_;
    ++gen_;
    work_.notify_all();
    lk.unlock();
    memcpy(dst, src, part < n ? part : n);
    lk.lock();
    done_.wait(lk, [&] { return pending_ == 0; });
    busy_ = false;
    caller_.notify_one();
  }

 private:
  CopyWorkers() {
    const unsigned hw = std::thread::hardware_concurrency();
    nthreads_ = hw > 1 ? (hw - 1 < 15u ? hw - 1 : 15u) : 0u;
    for (unsigned i = 0; i < nthreads_; ++i) std::thread([this] { loop(); }).detach();
  }
  void loop() {
    unsigned long long seen = 0;
    std::unique_lock<std::mutex> lk(mu_);
    for (;;) {
      work_.wait(lk, [&] { return gen_ != seen && busy_ && next_ * part_ < n_; });
      const size_t i = next_++;
      if (next_ * part_ >= n_ || next_ > nthreads_) seen = gen_;
      char* d = dst_;
      const char* s = src_;
      const size_t a = i * part_, len = part_ < n_ - a ? part_ : n_ - a;
      lk.unlock();
      memcpy(d + a, s + a, len);
      lk.lock();
      if (--pending_ == 0) done_.notify_all();
    }
  }
  std::mutex mu_;
  std::condition_variable work_, done_, caller_;
  unsigned nthreads_ = 0;
  bool busy_ = false;
  char* dst_ = nullptr;
  const char* src_ = nullptr;
  size_t n_ = 0, part_ = 0, next_ = 0, pending_ = 0;
  unsigned long long gen_ = 0;
};

// memcpy split over the copy workers when it is large.
inline void parallel_memcpy(void* dst, const void* src, size_t n) { CopyWorkers::get().copy(dst, src, n); }

// Copies ranges of page-locked host memory into pageable caller memory as their downloads
// land: push() queues (dst, src, n) behind an event recorded after the range's device-to-host
// copy; a thread of its own waits for each event in turn and copies the range on the copy
// workers, so the copy of one chunk's output overlaps the downloads and kernels of the next.
// The downloads themselves go at the link's rate into a page-locked block (a DMA into pageable
// memory is staged by the driver at a fraction of it). finish() waits for every queued range.
class CopyOut {
 public:
  void open(int device) {
    th_ = std::thread([this, device] { loop(device); });
  }
  void push(uint8_t* dst, const uint8_t* src, size_t n, cudaEvent_t ready) {
    if (!n) return;
    std::lock_guard<std::mutex> g(mu_);
    q_.push_back(Item{dst, src, n, ready});
    cv_.notify_all();
  }
  // waits for every queued range; the first error met (later ranges are skipped after one)
  cudaError_t finish() {
    {
      std::lock_guard<std::mutex> g(mu_);
      closed_ = true;
      cv_.notify_all();
    }
    if (th_.joinable()) th_.join();
    return err_;
  }
  ~CopyOut() { finish(); }

 private:
  struct Item {
    uint8_t* dst;
    const uint8_t* src;
    size_t n;
    cudaEvent_t ready;
  };
  void loop(int device) {
    if (cudaSetDevice(device) != cudaSuccess) err_ = cudaErrorInvalidDevice;
    for (;;) {
      Item it;
      {
        std::unique_lock<std::mutex> lk(mu_);
        cv_.wait(lk, [&] { return !q_.empty() || closed_; });
        if (q_.empty()) break;
        it = q_.front();
        q_.erase(q_.begin());
      }
      if (err_ != cudaSuccess) continue;
      if (it.ready) err_ = cudaEventSynchronize(it.ready);
      if (err_ == cudaSuccess) parallel_memcpy(it.dst, it.src, it.n);
    }
  }
  std::thread th_;
  std::mutex mu_;
  std::condition_variable cv_;
  std::vector<Item> q_;
  bool closed_ = false;
  cudaError_t err_ = cudaSuccess;  // written by the thread only until finish() joins it
};

// First-fit sub-allocator over one page-locked block: a server's host staging area, pinned
// once instead of per request. Blocks handed to callers are released with cuda_free_host
// (host_free below finds the owning area); an area closed by its server is freed when its
// last block comes back.
class HostArena {
 public:
  ~HostArena() {
    if (base_) cudaFreeHost(base_);
  }
  cudaError_t init(size_t bytes) {
    bytes = pool_round_up(bytes ? bytes : 1, 2u << 20);
    cudaError_t e = cudaMallocHost(&base_, bytes);
    if (e != cudaSuccess) {
      base_ = nullptr;
      return e;
    }
    size_ = bytes;
    free_[0] = bytes;
    return cudaSuccess;
  }
  uint8_t* alloc(size_t n) {
    n = pool_round_up(n ? n : 1, 256);
    std::lock_guard<std::mutex> g(mu_);
    for (auto it = free_.begin(); it != free_.end(); ++it) {
      if (it->second >= n) {
        const size_t off = it->first, rest = it->second - n;
        free_.erase(it);
        if (rest) free_[off + n] = rest;
        used_[off] = n;
        return base_ + off;
      }
    }
    return nullptr;
  }
  bool contains(const void* p) const {
    const uint8_t* q = static_cast<const uint8_t*>(p);
    return base_ && q >= base_ && q < base_ + size_;
  }
  // returns true when the area is closed and now empty
  bool release(const void* p) {
    std::lock_guard<std::mutex> g(mu_);
    size_t start = (size_t)(static_cast<const uint8_t*>(p) - base_);
    auto u = used_.find(start);
    if (u == used_.end()) return false;
    size_t len = u->second;
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
    return closed_ && used_.empty();
  }
  // the owner is gone; true when nothing is outstanding (the area can be freed now)
  bool close() {
    std::lock_guard<std::mutex> g(mu_);
    closed_ = true;
    return used_.empty();
  }

 private:
  std::mutex mu_;
  uint8_t* base_ = nullptr;
  size_t size_ = 0;
  bool closed_ = false;
  std::map<size_t, size_t> free_, used_;
};

// Registry of the live host areas (defined in capi.cu).
void host_arena_register(HostArena* a);
// The owner closes its area: freed now, or when its last block is released.
void host_arena_close(HostArena* a);
// Release a block handed to a caller: into its host area, else into the pool.
void host_free(void* p);

}  // namespace crb
