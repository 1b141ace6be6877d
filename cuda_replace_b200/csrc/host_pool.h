// host_pool.h - page-locked host memory handed to callers (freed with cuda_free_host).
#pragma once

#include <cuda_runtime.h>

#include <cstddef>
#include <cstdint>
#include <iterator>
#include <map>
#include <mutex>
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
        void* p = it->second;
        idle_bytes_ -= it->first;
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
  void put(void* p) {
    if (!p) return;
    std::vector<void*> evict;
    {
      std::lock_guard<std::mutex> g(mu_);
      auto s = sizes_.find(p);
      if (s == sizes_.end()) {
        evict.push_back(p);  // not ours: release directly
      } else {
        idle_.emplace(s->second, p);
        idle_bytes_ += s->second;
        while (idle_bytes_ > kMaxIdle && !idle_.empty()) {
          auto big = std::prev(idle_.end());
          idle_bytes_ -= big->first;
          sizes_.erase(big->second);
          evict.push_back(big->second);
          idle_.erase(big);
        }
      }
    }
    for (void* q : evict) cudaFreeHost(q);
  }

 private:
  static constexpr size_t kMaxIdle = 24ull << 30;
  std::mutex mu_;
  std::multimap<size_t, void*> idle_;
  std::unordered_map<void*, size_t> sizes_;
  size_t idle_bytes_ = 0;
};

// The process-wide pool (never destroyed: CUDA may be torn down first at exit).
PinnedPool& host_pinned_pool();

}  // namespace crb
