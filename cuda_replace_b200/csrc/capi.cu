// capi.cu - sessions, memory management and the C ABI of libcuda_replace.so.
//
// Mirrors the exports of RAZZULLIX/cuda_replace (cuda_replace.cu:2164-2603): same names,
// signatures, ownership rules and return codes (see include/cuda_replace.h). The session
// keeps two device buffers that swap roles after every apply (input -> output), a small
// look-back scratch area (per-tile status, function tables, inclusive prefixes) that
// grows with the input, and a device result block read back once per apply.
//
// Differences from the reference that callers can observe, all towards bytes.replace:
//  * An empty pattern inserts the replacement before every byte and at the end, as
//    bytes.replace does; the reference leaves the buffer unchanged (cuda_replace.cu:2104).
//  * apply_seeded honours negative carry-ins (the reference's default fused path ignores
//    them, cuda_replace.cu:859) and reports the real last kept start.
//  * Positions, counts and offsets are 64-bit end to end (the reference truncates to int
//    at cuda_replace.cu:159-160, 609, 668, 1418).
#include <cuda_runtime.h>

#include <algorithm>
#include <atomic>
#include <condition_variable>
#include <cstdint>
#include <cstdlib>
#include <cstring>
#include <map>
#include <mutex>
#include <new>
#include <thread>
#include <unordered_map>
#include <vector>

#include "cuda_replace.h"
#include "host_pool.h"
#include "replace_kernels.h"

namespace crb {
PinnedPool& host_pinned_pool() {
  static PinnedPool* pool = new PinnedPool();  // never destroyed: CUDA may be torn down first at exit
  return *pool;
}

namespace {
std::mutex g_arena_mu;
std::vector<HostArena*>& arenas() {
  static auto* v = new std::vector<HostArena*>();  // never destroyed, like the pool
  return *v;
}
}  // namespace

void host_arena_register(HostArena* a) {
  std::lock_guard<std::mutex> g(g_arena_mu);
  arenas().push_back(a);
}

void host_arena_close(HostArena* a) {
  std::lock_guard<std::mutex> g(g_arena_mu);
  if (a->close()) {
    auto& v = arenas();
    v.erase(std::remove(v.begin(), v.end(), a), v.end());
    delete a;
  }
}

void host_free(void* p) {
  if (!p) return;
  {
    std::lock_guard<std::mutex> g(g_arena_mu);
    auto& v = arenas();
    for (auto it = v.begin(); it != v.end(); ++it) {
      if ((*it)->contains(p)) {
        HostArena* a = *it;
        if (a->release(p)) {  // closed and empty: the last block of a closed server's area
          v.erase(it);
          delete a;
        }
        return;
      }
    }
  }
  host_pinned_pool().put(p);
}
}  // namespace crb

#define CR_EXPORT extern "C" __attribute__((visibility("default")))

// unified() takes its chunked path (uploads, replaces and downloads of successive chunks
// overlapped) for page-locked inputs from kUnifiedChunkedMin bytes, in at most kUnifiedChunks
// chunks of at least 32 MiB.
constexpr size_t kUnifiedChunkedMin = (size_t)256 << 20;
constexpr int kUnifiedChunks = 16;

namespace {

using crb::ApplyResult;
using crb::ReplaceParams;
using crb::TileIncl;

constexpr int kErrUnknown = 999;  // cudaErrorUnknown
constexpr int kFallback = -100;   // internal: the fast path does not apply, use the general one
constexpr size_t kAllocQuantum = 2ull << 20;

size_t round_up(size_t x, size_t q) { return (x + q - 1) / q * q; }

// apply_batch runs runs of pairs proved independent in one pass each (multi-pattern stages)
// unless the environment sets CUDA_REPLACE_STAGES=0 (every pair then gets its own pass).
bool stages_enabled() {
  const char* v = getenv("CUDA_REPLACE_STAGES");
  return !(v && v[0] == '0');
}

// ------------------------------------------------------------------ page-locked host pool
using crb::CopyOut;
using crb::PinnedPool;
PinnedPool& pinned_pool() { return crb::host_pinned_pool(); }

// ------------------------------------------------------------------ session
struct Session {
  std::mutex mtx;
  bool alive = true;
  int device = 0;
  cudaStream_t stream = nullptr;

  uint8_t* buf = nullptr;  // current contents (len bytes)
  size_t buf_cap = 0;
  uint8_t* alt = nullptr;  // output of the next apply; holds the previous input afterwards
  size_t alt_cap = 0;
  size_t len = 0;

  uint32_t* status = nullptr;  // look-back scratch
  TileIncl* incl = nullptr;
  size_t tiles_cap = 0;
  unsigned long long* agg = nullptr;
  size_t agg_cap = 0;
  long long* tile_last = nullptr;  // per super-tile (same capacity as status)
  unsigned long long* rec = nullptr;  // 16-byte look-back record per super-tile
  ApplyResult* res = nullptr;       // device
  ApplyResult* res_host = nullptr;  // page-locked mirror
  uint8_t* ext = nullptr;           // device copy of long patterns / replacements
  size_t ext_cap = 0;
  uint8_t* ext_host = nullptr;
  size_t ext_host_cap = 0;

  uint32_t epoch = 0;
  unsigned long long launches = 0;
  unsigned long long kept_last = 0;

  unsigned long long* lens = nullptr;       // device: lengths along an apply_batch chain
  unsigned long long* lens_host = nullptr;  // page-locked mirror
  size_t lens_cap = 0;
  unsigned long long buf_version = 1;       // changes whenever the contents of buf change
  uint32_t* pres = nullptr;                 // presence index of buf (cuda_replace_build_index)
  size_t pres_cap = 0;                      // words
  uint32_t pres_shift = 20;
  unsigned long long pres_version = 0;      // buf_version the index describes (0: none)
  crb::MultiTable* mtab = nullptr;          // device: pair tables of an apply_batch's stages
  crb::MultiTable* mtab_host = nullptr;     // page-locked mirror
  size_t mtab_cap = 0;
  cudaStream_t async_stream = nullptr;  // stream of the last cuda_replace_apply_device_async
  uint32_t async_epoch = 0;
  bool async_copy = false;          // the last async call copied its input (n < pattern length)
  unsigned long long async_n = 0;   // ... and this many bytes
  cudaEvent_t ev_order = nullptr;   // orders the session stream and a caller stream

  // the most recent apply, for query_prefix: 0 none, 1 no match possible, 2 kernel, 3 empty pattern
  int q_kind = 0;
  unsigned long long q_n = 0;
  ReplaceParams q_params;

  // unified() on a large page-locked input: upload and download streams, one event per chunk
  cudaStream_t up = nullptr, down = nullptr;
  cudaEvent_t ev_up[kUnifiedChunks] = {}, ev_done[kUnifiedChunks] = {};
  cudaEvent_t ev_dl[kUnifiedChunks] = {};   // a chunk's download is done (unified into caller memory)
  cudaEvent_t ev_stage[3] = {};             // a pageable input's staging slots (chunked unified)
  unsigned int* carry2 = nullptr;           // device: carry into / out of the current chunk
  unsigned long long* olen_dev = nullptr;   // device: output end of the current chunk
};

cudaError_t dev_grow(uint8_t** ptr, size_t* cap, size_t need, bool keep, size_t keep_len, cudaStream_t st) {
  if (*cap >= need && *ptr) return cudaSuccess;
  const size_t new_cap = round_up(need + need / 8 + 4096, kAllocQuantum);
  uint8_t* p = nullptr;
  cudaError_t e = cudaMalloc(&p, new_cap);
  if (e != cudaSuccess) {
    // retry without headroom before giving up
    const size_t tight = round_up(need + 4096, 4096);
    e = cudaMalloc(&p, tight);
    if (e != cudaSuccess) return e;
    *cap = tight;
  } else {
    *cap = new_cap;
  }
  if (keep && *ptr && keep_len) {
    e = cudaMemcpyAsync(p, *ptr, keep_len, cudaMemcpyDeviceToDevice, st);
    if (e == cudaSuccess) e = cudaStreamSynchronize(st);
    if (e != cudaSuccess) {
      cudaFree(p);
      return e;
    }
  }
  if (*ptr) cudaFree(*ptr);
  *ptr = p;
  return cudaSuccess;
}

cudaError_t ensure_scratch(Session* s, size_t tiles, size_t entries_per_tile) {
  if (tiles > s->tiles_cap) {
    const size_t cap = tiles + tiles / 8 + 64;
    uint32_t* st = nullptr;
    TileIncl* in = nullptr;
    long long* tl = nullptr;
    cudaError_t e = cudaMalloc(&st, cap * sizeof(uint32_t));
    if (e != cudaSuccess) return e;
    e = cudaMalloc(&in, cap * sizeof(TileIncl));
    if (e != cudaSuccess) {
      cudaFree(st);
      return e;
    }
    e = cudaMalloc(&tl, cap * sizeof(long long));
    if (e != cudaSuccess) {
      cudaFree(st);
      cudaFree(in);
      return e;
    }
    unsigned long long* rc = nullptr;
    e = cudaMalloc(&rc, cap * 2 * sizeof(unsigned long long));
    if (e == cudaSuccess) e = cudaMemsetAsync(rc, 0, cap * 2 * sizeof(unsigned long long), s->stream);
    if (e != cudaSuccess) {
      cudaFree(st);
      cudaFree(in);
      cudaFree(tl);
      if (rc) cudaFree(rc);
      return e;
    }
    e = cudaMemsetAsync(st, 0, cap * sizeof(uint32_t), s->stream);
    if (e != cudaSuccess) {
      cudaFree(st);
      cudaFree(in);
      return e;
    }
    if (s->status) cudaFree(s->status);
    if (s->incl) cudaFree(s->incl);
    if (s->tile_last) cudaFree(s->tile_last);
    if (s->rec) cudaFree(s->rec);
    s->status = st;
    s->incl = in;
    s->tile_last = tl;
    s->rec = rc;
    s->tiles_cap = cap;
  }
  const size_t entries = tiles * entries_per_tile;
  if (entries > s->agg_cap) {
    const size_t cap = entries + entries / 8 + 1024;
    unsigned long long* a = nullptr;
    cudaError_t e = cudaMalloc(&a, cap * sizeof(unsigned long long));
    if (e != cudaSuccess) return e;
    if (s->agg) cudaFree(s->agg);
    s->agg = a;
    s->agg_cap = cap;
  }
  return cudaSuccess;
}

uint32_t next_epoch(Session* s) {
  // Status words hold the epoch (30 bits), look-back records its low 24 bits: when either
  // wraps, clear both so a stale word from 2^24 launches ago can never look current.
  if (s->epoch >= (1u << 30) - 2 || ((s->epoch + 1) & 0xFFFFFFu) == 0) {
    cudaMemsetAsync(s->status, 0, s->tiles_cap * sizeof(uint32_t), s->stream);
    if (s->rec) cudaMemsetAsync(s->rec, 0, s->tiles_cap * 2 * sizeof(unsigned long long), s->stream);
    if (s->epoch >= (1u << 30) - 2) s->epoch = 0;
    ++s->epoch;  // skip the value whose record tag would be 0
  }
  return ++s->epoch;
}

void session_free(Session* s) {
  if (!s) return;
  cudaSetDevice(s->device);
  if (s->stream) cudaStreamSynchronize(s->stream);
  if (s->buf) cudaFree(s->buf);
  if (s->alt) cudaFree(s->alt);
  if (s->status) cudaFree(s->status);
  if (s->incl) cudaFree(s->incl);
  if (s->tile_last) cudaFree(s->tile_last);
  if (s->rec) cudaFree(s->rec);
  if (s->agg) cudaFree(s->agg);
  if (s->res) cudaFree(s->res);
  if (s->res_host) cudaFreeHost(s->res_host);
  if (s->ext) cudaFree(s->ext);
  if (s->ext_host) cudaFreeHost(s->ext_host);
  if (s->lens) cudaFree(s->lens);
  if (s->lens_host) cudaFreeHost(s->lens_host);
  if (s->pres) cudaFree(s->pres);
  if (s->mtab) cudaFree(s->mtab);
  if (s->mtab_host) cudaFreeHost(s->mtab_host);
  for (int k = 0; k < 3; ++k)
    if (s->ev_stage[k]) cudaEventDestroy(s->ev_stage[k]);
  for (int k = 0; k < kUnifiedChunks; ++k) {
    if (s->ev_up[k]) cudaEventDestroy(s->ev_up[k]);
    if (s->ev_done[k]) cudaEventDestroy(s->ev_done[k]);
    if (s->ev_dl[k]) cudaEventDestroy(s->ev_dl[k]);
  }
  if (s->up) {
    cudaStreamSynchronize(s->up);
    cudaStreamDestroy(s->up);
  }
  if (s->down) {
    cudaStreamSynchronize(s->down);
    cudaStreamDestroy(s->down);
  }
  if (s->ev_order) cudaEventDestroy(s->ev_order);
  if (s->carry2) cudaFree(s->carry2);
  if (s->olen_dev) cudaFree(s->olen_dev);
  if (s->stream) cudaStreamDestroy(s->stream);
  delete s;
}

int session_create(Session** out) {
  *out = nullptr;
  Session* s = new (std::nothrow) Session();
  if (!s) return -2;
  cudaError_t e = cudaGetDevice(&s->device);
  if (e == cudaSuccess) e = cudaStreamCreateWithFlags(&s->stream, cudaStreamNonBlocking);
  if (e == cudaSuccess) e = cudaMalloc(&s->res, sizeof(ApplyResult));
  if (e == cudaSuccess) e = cudaMemsetAsync(s->res, 0, sizeof(ApplyResult), s->stream);
  if (e == cudaSuccess) e = cudaMallocHost(&s->res_host, sizeof(ApplyResult));
  if (e == cudaSuccess) e = cudaStreamSynchronize(s->stream);
  if (e != cudaSuccess) {
    session_free(s);
    return (int)e;
  }
  *out = s;
  return 0;
}

// Upload src[0, len) into the session buffer.
bool host_is_pinned(const void* p) {
  cudaPointerAttributes a;
  if (cudaPointerGetAttributes(&a, p) != cudaSuccess) {
    cudaGetLastError();
    return false;
  }
  return a.type == cudaMemoryTypeHost;
}

// Host -> device copy of len bytes. A large pageable source is staged through two page-locked
// 32 MiB buffers filled by several host threads, so the copy runs near the host link's speed
// (a pageable cudaMemcpy goes through the driver's single-threaded staging).
cudaError_t upload_host(uint8_t* dst, const uint8_t* src, size_t len, cudaStream_t st) {
  const size_t kChunk = 32u << 20;
  if (len < (8u << 20) || host_is_pinned(src)) return cudaMemcpyAsync(dst, src, len, cudaMemcpyHostToDevice, st);
  cudaError_t e = cudaSuccess;
  uint8_t* stage[2] = {nullptr, nullptr};
  cudaEvent_t ev[2] = {nullptr, nullptr};
  for (int b = 0; b < 2 && e == cudaSuccess; ++b) {
    stage[b] = static_cast<uint8_t*>(pinned_pool().get(kChunk, &e));
    if (e == cudaSuccess) e = cudaEventCreateWithFlags(&ev[b], cudaEventDisableTiming);
  }
  for (size_t off = 0, i = 0; off < len && e == cudaSuccess; off += kChunk, ++i) {
    const int b = (int)(i & 1);
    const size_t m = std::min(kChunk, len - off);
    if (i >= 2) e = cudaEventSynchronize(ev[b]);  // stage[b] has reached the device
    if (e != cudaSuccess) break;
    crb::parallel_memcpy(stage[b], src + off, m);
    e = cudaMemcpyAsync(dst + off, stage[b], m, cudaMemcpyHostToDevice, st);
    if (e == cudaSuccess) e = cudaEventRecord(ev[b], st);
  }
  const cudaError_t se = cudaStreamSynchronize(st);  // the staging goes back to the pool
  for (int b = 0; b < 2; ++b) {
    if (ev[b]) cudaEventDestroy(ev[b]);
    if (stage[b]) pinned_pool().put(stage[b]);
  }
  return e != cudaSuccess ? e : se;
}

int session_load(Session* s, const uint8_t* src, size_t len) {
  if (len && !src) return -1;
  cudaError_t e = dev_grow(&s->buf, &s->buf_cap, len ? len : 1, false, 0, s->stream);
  if (e != cudaSuccess) return (int)e;
  if (len) {
    e = upload_host(s->buf, src, len, s->stream);
    if (e != cudaSuccess) return (int)e;
  }
  e = cudaStreamSynchronize(s->stream);
  if (e != cudaSuccess) return (int)e;
  s->len = len;
  ++s->buf_version;
  s->q_kind = 0;
  return 0;
}

// Copy host bytes that do not fit in the launch parameters to the device.
cudaError_t upload_ext(Session* s, const uint8_t* pat, uint32_t L, const uint8_t* rep, uint32_t R) {
  const size_t need = round_up(L, 16) + round_up(R, 16) + 32;
  if (need > s->ext_host_cap) {
    if (s->ext_host) {
      cudaStreamSynchronize(s->stream);
      cudaFreeHost(s->ext_host);
      s->ext_host = nullptr;
    }
    cudaError_t e = cudaMallocHost(&s->ext_host, need);
    if (e != cudaSuccess) return e;
    s->ext_host_cap = need;
  }
  if (need > s->ext_cap) {
    cudaStreamSynchronize(s->stream);
    if (s->ext) cudaFree(s->ext);
    s->ext = nullptr;
    cudaError_t e = cudaMalloc(&s->ext, need);
    if (e != cudaSuccess) return e;
    s->ext_cap = need;
  }
  cudaError_t e = cudaStreamSynchronize(s->stream);  // staging may still feed an earlier copy
  if (e != cudaSuccess) return e;
  if (L) memcpy(s->ext_host, pat, L);
  if (R) memcpy(s->ext_host + round_up(L, 16), rep, R);
  return cudaMemcpyAsync(s->ext, s->ext_host, need, cudaMemcpyHostToDevice, s->stream);
}

// Worst-case output length of one apply, saturating at SIZE_MAX.
size_t output_bound(size_t n, uint32_t L, uint32_t R) {
  if (L == 0) {
    const unsigned __int128 b = (unsigned __int128)n * (R + 1ull) + R;
    return b > (unsigned __int128)SIZE_MAX ? SIZE_MAX : (size_t)b;
  }
  if (R <= L) return n;
  const unsigned __int128 b = (unsigned __int128)n + (unsigned __int128)(n / L) * (R - L);
  return b > (unsigned __int128)SIZE_MAX ? SIZE_MAX : (size_t)b;
}

void swap_buffers(Session* s) {
  std::swap(s->buf, s->alt);
  std::swap(s->buf_cap, s->alt_cap);
}

// Start of the last kept match of the launch described by p (after it completed).
long long last_kept_of(const ReplaceParams& p, const ApplyResult& r) {
  if (!p.nsub) return r.last_kept;
  if ((r.last_tagged >> 40) != (unsigned long long)p.epoch) return -1;
  return (long long)(r.last_tagged & ((1ull << 40) - 1)) - 1;
}

// One apply. block_before: candidates starting before it are not taken.
int apply_one(Session* s, const uint8_t* pat, int pat_len, const uint8_t* rep, int rep_len,
              unsigned long long block_before, long long* out_last, size_t* new_len) {
  if (pat_len < 0 || rep_len < 0) return -1;
  if ((pat_len > 0 && !pat) || (rep_len > 0 && !rep)) return -1;
  const uint32_t L = (uint32_t)pat_len, R = (uint32_t)rep_len;
  if (L > crb::kMaxLen || R > crb::kMaxLen) return -4;
  const size_t n = s->len;
  cudaError_t e;

  if (L == 0) {  // bytes.replace(b"", rep)
    const size_t out_n = output_bound(n, 0, R);
    if (out_n == SIZE_MAX) return (int)cudaErrorMemoryAllocation;
    e = dev_grow(&s->alt, &s->alt_cap, out_n ? out_n : 1, false, 0, s->stream);
    if (e != cudaSuccess) return (int)e;
    if (R) {
      e = upload_ext(s, nullptr, 0, rep, R);
      if (e != cudaSuccess) return (int)e;
    }
    if (out_n) {
      e = crb::launch_empty_pattern(s->buf, n, s->ext, R, s->alt, s->stream);
      if (e != cudaSuccess) return (int)e;
      ++s->launches;
    }
    e = cudaStreamSynchronize(s->stream);
    if (e != cudaSuccess) return (int)e;
    swap_buffers(s);
    ++s->buf_version;
    s->len = out_n;
    s->q_kind = 3;
    s->q_n = n;
    s->kept_last = n + 1;
    if (out_last) *out_last = (long long)n;
    if (new_len) *new_len = out_n;
    return 0;
  }

  if (n < L) {  // no occurrence possible: the buffer is unchanged
    s->q_kind = 1;
    s->q_n = n;
    s->kept_last = 0;
    if (out_last) *out_last = -1;
    if (new_len) *new_len = n;
    return 0;
  }

  ReplaceParams p;
  memset(&p, 0, sizeof(p));
  crb::prepare_pattern_fields(p, pat, L);
  p.R = R;
  p.nsub = crb::super_nsub(p.mode, L);
  const size_t tile_bytes = (size_t)crb::kTile * (p.nsub ? p.nsub : 1u);
  const size_t tiles = (n + tile_bytes - 1) / tile_bytes;
  if (tiles > 0xFFFFFFF0ull) return (int)cudaErrorInvalidValue;
  p.num_tiles = (uint32_t)tiles;
  e = ensure_scratch(s, tiles, p.agg_entries);
  if (e != cudaSuccess) return (int)e;
  p.tile_last = s->tile_last;
  p.rec = s->rec;

  const size_t bound = output_bound(n, L, R);
  size_t want = bound;
  const size_t generous = std::max<size_t>(4 * n, n + (256ull << 20));
  if (bound > generous) want = std::max<size_t>(s->alt_cap, std::min<size_t>(bound, 2 * n + (64ull << 20)));
  e = dev_grow(&s->alt, &s->alt_cap, want ? want : 1, false, 0, s->stream);
  if (e != cudaSuccess) return (int)e;

  if (L > (uint32_t)crb::kInlineMax || R > (uint32_t)crb::kInlineMax) {
    e = upload_ext(s, pat, L, rep, R);
    if (e != cudaSuccess) return (int)e;
    p.pat_ext = s->ext;
    p.rep_ext = s->ext + round_up(L, 16);
  }
  if (L <= (uint32_t)crb::kInlineMax) memcpy(p.pat, pat, L);
  if (R <= (uint32_t)crb::kInlineMax && R) memcpy(p.rep, rep, R);
  p.in = s->buf;
  p.n = n;
  p.block_before = block_before;
  if (s->pres_version == s->buf_version && p.nsub) {  // the presence index describes this input
    p.presence = s->pres;
    p.presence_shift = s->pres_shift;
  }
  p.status = s->status;
  p.incl = s->incl;
  p.agg = s->agg;
  p.res = s->res;

  for (int attempt = 0; attempt < 2; ++attempt) {
    p.out = s->alt;
    p.out_cap = s->alt_cap;
    p.epoch = next_epoch(s);
    e = p.nsub ? crb::launch_replace_super(p, s->stream, nullptr) : crb::launch_replace(p, s->stream, nullptr);
    if (e != cudaSuccess) return (int)e;
    ++s->launches;
    e = cudaMemcpyAsync(s->res_host, s->res, sizeof(ApplyResult), cudaMemcpyDeviceToHost, s->stream);
    if (e != cudaSuccess) return (int)e;
    e = cudaStreamSynchronize(s->stream);
    if (e != cudaSuccess) return (int)e;
    const ApplyResult r = *s->res_host;
    if (r.error_epoch == p.epoch) return kErrUnknown;
    if (r.overflow_epoch == p.epoch) {
      if (attempt == 1) return kErrUnknown;
      e = dev_grow(&s->alt, &s->alt_cap, r.out_len, false, 0, s->stream);
      if (e != cudaSuccess) return (int)e;
      continue;
    }
    swap_buffers(s);
    ++s->buf_version;
    s->len = (size_t)r.out_len;
    s->q_kind = 2;
    s->q_n = n;
    s->q_params = p;
    s->kept_last = r.kept;
    if (out_last) *out_last = r.kept ? last_kept_of(p, r) : -1;
    if (new_len) *new_len = s->len;
    return 0;
  }
  return kErrUnknown;
}

// apply_batch with the lengths chained on the device: one launch per stage (one pair, or a run
// of pairs applied in one pass) and a single read-back at the end, instead of a host round trip
// per pair. Used when every pair fits the super-tile kernel with inline pattern bytes and the
// worst-case lengths along the chain fit in memory; returns kFallback when the caller must use
// one apply per pair.
int apply_batch_chained(Session* s, const uint8_t** pats, const int* pat_lens, const uint8_t** reps,
                        const int* rep_lens, int count, size_t* new_len) {
  if (count <= 0 || !pats || !reps || !pat_lens || !rep_lens) return kFallback;
  for (int k = 0; k < count; ++k) {
    const int pl = pat_lens[k], rl = rep_lens[k];
    if (pl < 1 || rl < 0 || pl > crb::kInlineMax || rl > crb::kInlineMax || !pats[k] || (rl && !reps[k])) return kFallback;
  }
  // Stages: runs of pairs proved to give in one pass what they give one after the other
  // (crb::plan_stages). The last pair runs alone, so query_prefix and the kept count after the
  // batch describe the last pair's pass, as after the reference's per-pair loop (cu:2480-2519).
  std::vector<int> stage_of((size_t)count);
  int nst = count;
  if (stages_enabled())
    nst = crb::plan_stages(pats, pat_lens, reps, rep_lens, count, true, stage_of.data());
  else
    for (int k = 0; k < count; ++k) stage_of[(size_t)k] = k;
  std::vector<ReplaceParams> ps((size_t)nst);
  std::vector<crb::MultiTable> tabs;
  std::vector<int> tab_of((size_t)nst, -1);
  size_t b = s->len, maxb = s->len, tiles_max = 1, entries_max = 1;
  for (int st = 0, k = 0; st < nst; ++st) {
    int k1 = k;
    while (k1 < count && stage_of[(size_t)k1] == st) ++k1;
    ReplaceParams& p = ps[(size_t)st];
    memset(&p, 0, sizeof(p));
    size_t bnext;
    if (k1 - k >= 2) {  // one pass over every pair of the stage
      tabs.emplace_back();
      crb::MultiTable& T = tabs.back();
      crb::build_multi_table(T, pats + k, pat_lens + k, reps + k, rep_lens + k, k1 - k);
      tab_of[(size_t)st] = (int)tabs.size() - 1;
      p.mode = crb::kModeMulti;
      p.L = T.Lmax;
      p.R = 0;
      p.agg_entries = 1;
      p.multi_ratio = T.ratio;
      p.nsub = crb::super_nsub(crb::kModeFree, 1);
      bnext = (size_t)crb::multi_output_bound(T, b);
      // the look-back sums sum(R - L) plus a bias per super-tile in 38-bit fields
      if ((b / ((size_t)crb::kTile * p.nsub) + 2) * crb::kMultiBias + bnext >= (1ull << 37)) return kFallback;
    } else {
      const int pl = pat_lens[k], rl = rep_lens[k];
      crb::prepare_pattern_fields(p, pats[k], (uint32_t)pl);
      p.R = (uint32_t)rl;
      p.nsub = crb::super_nsub(p.mode, p.L);
      if (!p.nsub) return kFallback;
      memcpy(p.pat, pats[k], (size_t)pl);
      if (rl) memcpy(p.rep, reps[k], (size_t)rl);
      bnext = output_bound(b, p.L, p.R);
    }
    const size_t tb = (size_t)crb::kTile * p.nsub;
    const size_t tiles = (b + tb - 1) / tb;
    p.num_tiles = (uint32_t)(tiles ? tiles : 1);
    tiles_max = std::max(tiles_max, (size_t)p.num_tiles);
    entries_max = std::max(entries_max, (size_t)p.num_tiles * p.agg_entries);
    if (bnext == SIZE_MAX) return kFallback;
    b = bnext;
    maxb = std::max(maxb, b);
    k = k1;
  }
  if (maxb > std::max<size_t>(4 * s->len, s->len + (1ull << 30))) return kFallback;
  cudaError_t e = dev_grow(&s->buf, &s->buf_cap, maxb ? maxb : 1, true, s->len, s->stream);
  if (e == cudaSuccess) e = dev_grow(&s->alt, &s->alt_cap, maxb ? maxb : 1, false, 0, s->stream);
  if (e == cudaSuccess) e = ensure_scratch(s, tiles_max, entries_max);
  if (e != cudaSuccess) return (int)e;
  if ((size_t)count + 1 > s->lens_cap) {
    if (s->lens) cudaFree(s->lens);
    if (s->lens_host) cudaFreeHost(s->lens_host);
    s->lens = nullptr;
    s->lens_host = nullptr;
    const size_t cap = (size_t)count + 64;
    e = cudaMalloc(&s->lens, cap * sizeof(unsigned long long));
    if (e == cudaSuccess) e = cudaMallocHost(&s->lens_host, cap * sizeof(unsigned long long));
    if (e != cudaSuccess) {
      s->lens_cap = 0;
      return (int)e;
    }
    s->lens_cap = cap;
  }
  if (tabs.size() > s->mtab_cap) {
    if (s->pres) cudaFree(s->pres);
  if (s->mtab) cudaFree(s->mtab);
    if (s->mtab_host) cudaFreeHost(s->mtab_host);
    s->mtab = nullptr;
    s->mtab_host = nullptr;
    const size_t cap = tabs.size() + 8;
    e = cudaMalloc(&s->mtab, cap * sizeof(crb::MultiTable));
    if (e == cudaSuccess) e = cudaMallocHost(&s->mtab_host, cap * sizeof(crb::MultiTable));
    if (e != cudaSuccess) {
      s->mtab_cap = 0;
      return (int)e;
    }
    s->mtab_cap = cap;
  }
  e = cudaStreamSynchronize(s->stream);  // the page-locked mirrors may feed an earlier copy
  if (e != cudaSuccess) return (int)e;
  s->lens_host[0] = s->len;
  e = cudaMemcpyAsync(s->lens, s->lens_host, sizeof(unsigned long long), cudaMemcpyHostToDevice, s->stream);
  if (e == cudaSuccess && !tabs.empty()) {
    memcpy(s->mtab_host, tabs.data(), tabs.size() * sizeof(crb::MultiTable));
    e = cudaMemcpyAsync(s->mtab, s->mtab_host, tabs.size() * sizeof(crb::MultiTable), cudaMemcpyHostToDevice,
                        s->stream);
  }
  if (e != cudaSuccess) return (int)e;
  uint8_t* bufs[2] = {s->buf, s->alt};
  const size_t cap = std::min(s->buf_cap, s->alt_cap);
  uint32_t first_epoch = 0;
  for (int k = 0; k < nst; ++k) {
    ReplaceParams& p = ps[(size_t)k];
    p.in = bufs[k & 1];
    p.out = bufs[(k + 1) & 1];
    p.n_dev = s->lens + k;
    p.len_out = s->lens + k + 1;
    p.out_cap = cap;
    p.status = s->status;
    p.incl = s->incl;
    p.agg = s->agg;
    p.res = s->res;
    p.tile_last = s->tile_last;
    p.rec = s->rec;
    p.epoch = next_epoch(s);
    if (k == 0) {
      first_epoch = p.epoch;
      if (s->pres_version == s->buf_version) {  // the presence index describes the first input
        p.presence = s->pres;
        p.presence_shift = s->pres_shift;
      }
    }
    if (tab_of[(size_t)k] >= 0) {
      p.multi = s->mtab + tab_of[(size_t)k];
      e = crb::launch_replace_multi(p, s->stream, nullptr);
    } else {
      e = crb::launch_replace_super(p, s->stream, nullptr);
    }
    if (e != cudaSuccess) return (int)e;
    ++s->launches;
  }
  e = cudaMemcpyAsync(s->lens_host, s->lens, ((size_t)nst + 1) * sizeof(unsigned long long),
                      cudaMemcpyDeviceToHost, s->stream);
  if (e == cudaSuccess)
    e = cudaMemcpyAsync(s->res_host, s->res, sizeof(ApplyResult), cudaMemcpyDeviceToHost, s->stream);
  if (e == cudaSuccess) e = cudaStreamSynchronize(s->stream);
  if (e != cudaSuccess) return (int)e;
  const ApplyResult r = *s->res_host;
  const uint32_t last_epoch = ps[(size_t)nst - 1].epoch;
  if ((r.error_epoch >= first_epoch && r.error_epoch <= last_epoch) ||
      (r.overflow_epoch >= first_epoch && r.overflow_epoch <= last_epoch))
    return kErrUnknown;
  if (nst & 1) swap_buffers(s);
  ++s->buf_version;
  s->len = (size_t)s->lens_host[nst];
  ReplaceParams q = ps[(size_t)nst - 1];  // a single pair (the last pair runs alone)
  q.n = s->lens_host[nst - 1];
  q.n_dev = nullptr;
  q.len_out = nullptr;
  s->q_kind = q.mode == crb::kModeMulti ? 0 : 2;
  s->q_n = q.n;
  s->q_params = q;
  s->kept_last = r.kept;
  if (new_len) *new_len = s->len;
  return 0;
}

int query_prefix64(Session* s, size_t limit, long long* kept, long long* last) {
  *kept = 0;
  *last = -1;
  if (s->q_kind == 0 || s->q_kind == 1) return 0;
  const unsigned long long lim = std::min<unsigned long long>(limit, s->q_n);
  if (lim == 0) return 0;
  if (s->q_kind == 3) {  // empty pattern: an (empty) match at every position 0..n
    *kept = (long long)lim;
    *last = (long long)lim - 1;
    return 0;
  }
  cudaError_t e;
  if (s->q_params.nsub) {
    ReplaceParams p = s->q_params;
    p.in = s->alt;  // the input of the last apply
    p.query_limit64 = lim;
    e = crb::launch_query_super(p, s->stream);
    if (e != cudaSuccess) return (int)e;
    ++s->launches;
    e = cudaMemcpyAsync(s->res_host, s->res, sizeof(ApplyResult), cudaMemcpyDeviceToHost, s->stream);
    if (e == cudaSuccess) e = cudaStreamSynchronize(s->stream);
    if (e != cudaSuccess) return (int)e;
    if (s->res_host->error_epoch == p.epoch) return kErrUnknown;
    *kept = (long long)s->res_host->q_kept;
    *last = s->res_host->q_last;
    return 0;
  }
  const unsigned long long t = lim / crb::kTile, rel = lim % crb::kTile;
  if (rel == 0) {
    TileIncl ti;
    e = cudaMemcpyAsync(&ti, s->incl + (t - 1), sizeof(TileIncl), cudaMemcpyDeviceToHost, s->stream);
    if (e == cudaSuccess) e = cudaStreamSynchronize(s->stream);
    if (e != cudaSuccess) return (int)e;
    *kept = (long long)ti.kept;
    *last = ti.last;
    return 0;
  }
  ReplaceParams p = s->q_params;
  p.in = s->alt;  // the input of the last apply
  p.query_tile = (uint32_t)t;
  p.query_limit = (uint32_t)rel;
  e = crb::launch_query(p, s->stream);
  if (e != cudaSuccess) return (int)e;
  ++s->launches;
  e = cudaMemcpyAsync(s->res_host, s->res, sizeof(ApplyResult), cudaMemcpyDeviceToHost, s->stream);
  if (e == cudaSuccess) e = cudaStreamSynchronize(s->stream);
  if (e != cudaSuccess) return (int)e;
  if (s->res_host->error_epoch == p.epoch) return kErrUnknown;
  *kept = (long long)s->res_host->q_kept;
  *last = s->res_host->q_last;
  return 0;
}

int result_to_pinned(Session* s, uint8_t** out_host, size_t* outlen) {
  *out_host = nullptr;
  *outlen = s->len;
  if (s->len == 0) return 0;
  cudaError_t e;
  void* host = pinned_pool().get(s->len, &e);
  if (!host) {
    *outlen = 0;
    return (int)e;
  }
  e = cudaMemcpyAsync(host, s->buf, s->len, cudaMemcpyDeviceToHost, s->stream);
  if (e == cudaSuccess) e = cudaStreamSynchronize(s->stream);
  if (e != cudaSuccess) {
    pinned_pool().put(host);
    *outlen = 0;
    return (int)e;
  }
  *out_host = (uint8_t*)host;
  return 0;
}

// Idle sessions reused by cuda_replace_unified, so a one-shot call pays no allocation.
std::mutex g_cache_mu;
std::vector<Session*> g_cache;

Session* cache_take(int device) {
  std::lock_guard<std::mutex> g(g_cache_mu);
  for (size_t i = 0; i < g_cache.size(); ++i) {
    if (g_cache[i]->device == device) {
      Session* s = g_cache[i];
      g_cache.erase(g_cache.begin() + i);
      return s;
    }
  }
  return nullptr;
}

void cache_give(Session* s) {
  {
    std::lock_guard<std::mutex> g(g_cache_mu);
    if (g_cache.size() < 8) {
      g_cache.push_back(s);
      return;
    }
  }
  session_free(s);
}

#define SESSION_GUARD(h)                              \
  if (!(h)) return -1;                                \
  Session* s = static_cast<Session*>(h);              \
  std::lock_guard<std::mutex> lock_(s->mtx);          \
  if (!s->alive) return -3;                           \
  cudaSetDevice(s->device)

}  // namespace

CR_EXPORT const char* cuda_replace_version(void) { return "cuda_replace_b200 1.0 sm_100a single-pass look-back"; }

CR_EXPORT int cuda_replace_plan_stages(const uint8_t** pats, const int* pat_lens, const uint8_t** reps,
                                       const int* rep_lens, int count, int keep_last_alone, int* stage_of) {
  if (count < 0 || (count > 0 && (!pats || !pat_lens || !reps || !rep_lens || !stage_of))) return -1;
  for (int k = 0; k < count; ++k)
    if (pat_lens[k] < 0 || rep_lens[k] < 0 || (pat_lens[k] && !pats[k]) || (rep_lens[k] && !reps[k])) return -1;
  if (count == 0) return 0;
  return crb::plan_stages(pats, pat_lens, reps, rep_lens, count, keep_last_alone != 0, stage_of);
}

CR_EXPORT void cuda_replace_host_copy(void* dst, const void* src, size_t n) {
  if (dst && src && n) crb::parallel_memcpy(dst, src, n);
}

CR_EXPORT void cuda_free_host(void* p) {
  if (p) crb::host_free(p);
}

CR_EXPORT int cuda_replace_open(void** ph, const uint8_t* src, size_t len) {
  if (!ph) return -1;
  *ph = nullptr;
  Session* s = nullptr;
  int rc = session_create(&s);
  if (rc != 0) return rc;
  rc = session_load(s, src, len);
  if (rc != 0) {
    session_free(s);
    return rc;
  }
  *ph = s;
  return 0;
}

CR_EXPORT int cuda_replace_reset(void* h, const uint8_t* src, size_t len) {
  SESSION_GUARD(h);
  return session_load(s, src, len);
}

CR_EXPORT int cuda_replace_build_index(void* h, size_t chunk_size) {
  SESSION_GUARD(h);
  // chunk: the reference's default of 1 MiB (DEFAULT_CHUNK_SIZE, cu:70), else the next power of
  // two of at least 16 KiB (a sub-tile of the kernel must lie inside one chunk)
  uint32_t shift = 20;
  if (chunk_size) {
    shift = 14;
    while (shift < 40 && ((size_t)1 << shift) < chunk_size) ++shift;
  }
  s->pres_version = 0;
  if (s->len == 0) return 0;
  const size_t chunks = (s->len + ((size_t)1 << shift) - 1) >> shift;
  if (chunks * 8 > s->pres_cap) {
    if (s->pres) cudaFree(s->pres);
    s->pres = nullptr;
    s->pres_cap = 0;
    cudaError_t e = cudaMalloc(&s->pres, chunks * 8 * sizeof(uint32_t));
    if (e != cudaSuccess) return (int)e;
    s->pres_cap = chunks * 8;
  }
  cudaError_t e = crb::launch_presence(s->buf, s->len, shift, s->pres, s->stream);
  if (e == cudaSuccess) e = cudaStreamSynchronize(s->stream);
  if (e != cudaSuccess) return (int)e;
  ++s->launches;
  s->pres_shift = shift;
  s->pres_version = s->buf_version;
  return 0;
}

CR_EXPORT int cuda_replace_apply(void* h, const uint8_t* pat, int pat_len, const uint8_t* rep, int rep_len,
                                 size_t* new_len) {
  SESSION_GUARD(h);
  return apply_one(s, pat, pat_len, rep, rep_len, 0, nullptr, new_len);
}

CR_EXPORT int cuda_replace_apply_seeded(void* h, const uint8_t* pat, int pat_len, const uint8_t* rep,
                                        int rep_len, long long prev_last_rel, long long* out_last_rel,
                                        size_t* new_len) {
  SESSION_GUARD(h);
  const long long b = (pat_len > 0) ? prev_last_rel + (long long)pat_len : 0;
  const unsigned long long block_before = b > 0 ? (unsigned long long)b : 0ull;
  long long last = -1;
  const int rc = apply_one(s, pat, pat_len, rep, rep_len, block_before, &last, new_len);
  if (rc == 0 && out_last_rel) *out_last_rel = last;
  return rc;
}

CR_EXPORT int cuda_replace_query_prefix(void* h, size_t limit, int* kept_before_limit,
                                        int* last_kept_before_limit) {
  SESSION_GUARD(h);
  long long k = 0, l = -1;
  const int rc = query_prefix64(s, limit, &k, &l);
  if (rc != 0) return rc;
  if (k > 0x7FFFFFFFll || l > 0x7FFFFFFFll) return -5;
  if (kept_before_limit) *kept_before_limit = (int)k;
  if (last_kept_before_limit) *last_kept_before_limit = (int)l;
  return 0;
}

CR_EXPORT int cuda_replace_query_prefix64(void* h, size_t limit, long long* kept_before_limit,
                                          long long* last_kept_before_limit) {
  SESSION_GUARD(h);
  long long k = 0, l = -1;
  const int rc = query_prefix64(s, limit, &k, &l);
  if (rc != 0) return rc;
  if (kept_before_limit) *kept_before_limit = k;
  if (last_kept_before_limit) *last_kept_before_limit = l;
  return 0;
}

CR_EXPORT int cuda_replace_apply_batch(void* h, const uint8_t** pats, const int* pat_lens, const uint8_t** reps,
                                       const int* rep_lens, int count, size_t* new_len) {
  SESSION_GUARD(h);
  if (count > 1) {
    const int rc = apply_batch_chained(s, pats, pat_lens, reps, rep_lens, count, new_len);
    if (rc != kFallback) return rc;
  }
  for (int i = 0; i < count; ++i) {
    const uint8_t* p = pats ? pats[i] : nullptr;
    const uint8_t* r = reps ? reps[i] : nullptr;
    const int pl = pat_lens ? pat_lens[i] : 0;
    const int rl = rep_lens ? rep_lens[i] : 0;
    const int rc = apply_one(s, p, pl, r, rl, 0, nullptr, nullptr);
    if (rc != 0) return rc;
  }
  if (new_len) *new_len = s->len;
  return 0;
}

CR_EXPORT int cuda_replace_result(void* h, uint8_t** out_host, size_t* outlen_host) {
  if (!h || !out_host || !outlen_host) return -1;
  SESSION_GUARD(h);
  return result_to_pinned(s, out_host, outlen_host);
}

CR_EXPORT int cuda_replace_result_into(void* h, uint8_t* dst, size_t cap, size_t* len) {
  SESSION_GUARD(h);
  if (len) *len = s->len;
  if (s->len == 0) return 0;
  if (!dst) return -1;
  if (cap < s->len) return (int)cudaErrorInvalidValue;
  cudaError_t e = cudaMemcpyAsync(dst, s->buf, s->len, cudaMemcpyDeviceToHost, s->stream);
  if (e == cudaSuccess) e = cudaStreamSynchronize(s->stream);
  return (int)e;
}

CR_EXPORT int cuda_replace_length(void* h, size_t* len) {
  if (!len) return -1;
  SESSION_GUARD(h);
  *len = s->len;
  return 0;
}

CR_EXPORT int cuda_replace_stats(void* h, unsigned long long* kept_last_apply, unsigned long long* kernel_launches) {
  SESSION_GUARD(h);
  if (kept_last_apply) *kept_last_apply = s->kept_last;
  if (kernel_launches) *kernel_launches = s->launches;
  return 0;
}

CR_EXPORT int cuda_replace_apply_device_async(void* h, const uint8_t* d_in, size_t n, const uint8_t* pat,
                                               int pat_len, const uint8_t* rep, int rep_len, uint8_t* d_out,
                                               size_t out_cap, void* stream) {
  SESSION_GUARD(h);
  if (pat_len <= 0 || rep_len < 0) return -1;
  if (pat_len > crb::kInlineMax || rep_len > crb::kInlineMax) return -4;
  if ((n && !d_in) || !d_out || !pat || (rep_len && !rep)) return -1;
  if (((uintptr_t)d_in & 15u) || ((uintptr_t)d_out & 15u)) return (int)cudaErrorInvalidValue;
  const uint32_t L = (uint32_t)pat_len, R = (uint32_t)rep_len;
  if (out_cap < output_bound(n, L, R)) return (int)cudaErrorInvalidValue;
  cudaStream_t st = stream ? static_cast<cudaStream_t>(stream) : s->stream;
  cudaError_t e = cudaSuccess;
  if (!s->ev_order) {
    e = cudaEventCreateWithFlags(&s->ev_order, cudaEventDisableTiming);
    if (e != cudaSuccess) return (int)e;
  }
  if ((size_t)L > n) {  // no occurrence possible: the output is the input, as bytes.replace gives
    if (n) e = cudaMemcpyAsync(d_out, d_in, n, cudaMemcpyDeviceToDevice, st);
    if (e != cudaSuccess) return (int)e;
    s->async_stream = st;
    s->async_epoch = 1;
    s->async_copy = true;
    s->async_n = n;
    s->q_kind = 0;
    return 0;
  }
  ReplaceParams p;
  memset(&p, 0, sizeof(p));
  crb::prepare_pattern_fields(p, pat, L);
  p.R = R;
  p.nsub = crb::super_nsub(p.mode, L);
  const size_t tile_bytes = (size_t)crb::kTile * (p.nsub ? p.nsub : 1u);
  const size_t tiles = (n + tile_bytes - 1) / tile_bytes;
  if (tiles > 0xFFFFFFF0ull) return (int)cudaErrorInvalidValue;
  p.num_tiles = (uint32_t)tiles;
  e = ensure_scratch(s, tiles, p.agg_entries);
  if (e != cudaSuccess) return (int)e;
  p.tile_last = s->tile_last;
  p.rec = s->rec;
  memcpy(p.pat, pat, L);
  if (R) memcpy(p.rep, rep, R);
  p.in = d_in;
  p.out = d_out;
  p.n = n;
  p.out_cap = out_cap;
  p.status = s->status;
  p.incl = s->incl;
  p.agg = s->agg;
  p.res = s->res;
  p.epoch = next_epoch(s);
  if (st != s->stream) {
    // ensure_scratch and next_epoch clear look-back scratch on the session stream: the kernel
    // on the caller's stream must not start before those clears have landed.
    e = cudaEventRecord(s->ev_order, s->stream);
    if (e == cudaSuccess) e = cudaStreamWaitEvent(st, s->ev_order, 0);
    if (e != cudaSuccess) return (int)e;
  }
  e = p.nsub ? crb::launch_replace_super(p, st, nullptr) : crb::launch_replace(p, st, nullptr);
  if (e != cudaSuccess) return (int)e;
  ++s->launches;
  if (st != s->stream) {
    // later work of this handle on its own stream (clears, other applies) waits for the kernel
    e = cudaEventRecord(s->ev_order, st);
    if (e == cudaSuccess) e = cudaStreamWaitEvent(s->stream, s->ev_order, 0);
    if (e != cudaSuccess) return (int)e;
  }
  s->async_stream = st;
  s->async_epoch = p.epoch;
  s->async_copy = false;
  s->q_kind = 0;
  return 0;
}

CR_EXPORT int cuda_replace_device_result(void* h, size_t* out_len, unsigned long long* kept) {
  SESSION_GUARD(h);
  if (!s->async_epoch) return -1;
  cudaStream_t st = s->async_stream ? s->async_stream : s->stream;
  cudaError_t e = cudaStreamSynchronize(st);
  if (e != cudaSuccess) return (int)e;
  if (s->async_copy) {
    if (out_len) *out_len = (size_t)s->async_n;
    if (kept) *kept = 0;
    return 0;
  }
  e = cudaMemcpy(s->res_host, s->res, sizeof(ApplyResult), cudaMemcpyDeviceToHost);
  if (e != cudaSuccess) return (int)e;
  const ApplyResult r = *s->res_host;
  if (r.error_epoch == s->async_epoch || r.overflow_epoch == s->async_epoch) return kErrUnknown;
  if (out_len) *out_len = (size_t)r.out_len;
  if (kept) *kept = r.kept;
  return 0;
}

CR_EXPORT void cuda_replace_close(void* h) {
  if (!h) return;
  Session* s = static_cast<Session*>(h);
  {
    std::lock_guard<std::mutex> lock(s->mtx);
    if (!s->alive) return;
    s->alive = false;
  }
  session_free(s);
}

// unified() for a large page-locked input and a pattern the super-tile kernel takes: every
// chunk's upload is queued at once; each chunk is replaced as soon as it is on the device (its
// last L - 1 bytes held back for the next chunk, the coverage carried across on the device)
// into the session's output buffer, and its output is downloaded into the result while the
// next chunks upload. With dst (pageable caller memory of at least the worst-case output
// length), each chunk's output is also copied from that page-locked block into dst by a
// CopyOut thread as soon as its download lands, while later chunks upload, replace and
// download; the block goes back to the pool. Returns kFallback when
// the call does not qualify (the caller takes the single-launch path), else 0 or an error code
// (a cudaError_t, or 999).
int unified_chunked(Session* s, const uint8_t* src, size_t n, const uint8_t* pat, uint32_t L, const uint8_t* rep,
                    uint32_t R, uint8_t** out_host, size_t* out_len, uint8_t* dst = nullptr, size_t dst_cap = 0) {
  if (n < kUnifiedChunkedMin || L == 0 || L > (uint32_t)crb::kInlineMax || R > (uint32_t)crb::kInlineMax)
    return kFallback;
  const bool pinned = host_is_pinned(src);
  ReplaceParams proto;
  memset(&proto, 0, sizeof(proto));
  crb::prepare_pattern_fields(proto, pat, L);
  proto.R = R;
  proto.nsub = crb::super_nsub(proto.mode, L);
  if (!proto.nsub) return kFallback;
  const size_t bound = output_bound(n, L, R);
  if (bound > 4 * n + ((size_t)64 << 20)) return kFallback;  // a large expansion: the single-launch path sizes it
  if (dst && dst_cap < bound) return kFallback;  // the single-launch path checks the exact length
  memcpy(proto.pat, pat, L);
  if (R) memcpy(proto.rep, rep, R);
  const size_t P = L - 1;  // bytes held back at the end of every chunk but the last
  const size_t chunk = std::max<size_t>((size_t)32 << 20, round_up((n + kUnifiedChunks - 1) / kUnifiedChunks, 1u << 20));
  // Chunk k uploads input [bnd(k), bnd(k + 1)) with bnd(k) = k * chunk + P for 0 < k: its
  // replace then starts P bytes earlier, at k * chunk, a 16-byte boundary as the loads need.
  size_t nchunks = (n + chunk - 1) / chunk;
  while (nchunks > 1 && (nchunks - 1) * chunk + P >= n) --nchunks;
  if (nchunks > (size_t)kUnifiedChunks) return kFallback;
  auto bnd = [&](size_t k) -> size_t { return k == 0 ? 0 : (k >= nchunks ? n : k * chunk + P); };
  const size_t tile_bytes = (size_t)crb::kTile * proto.nsub;

  cudaError_t e = cudaSuccess;
  if (!s->up) e = cudaStreamCreateWithFlags(&s->up, cudaStreamNonBlocking);
  if (e == cudaSuccess && !s->down) e = cudaStreamCreateWithFlags(&s->down, cudaStreamNonBlocking);
  for (int k = 0; k < kUnifiedChunks && e == cudaSuccess; ++k) {
    if (!s->ev_up[k]) e = cudaEventCreateWithFlags(&s->ev_up[k], cudaEventDisableTiming);
    if (e == cudaSuccess && !s->ev_done[k]) e = cudaEventCreateWithFlags(&s->ev_done[k], cudaEventDisableTiming);
    if (e == cudaSuccess && dst && !s->ev_dl[k]) e = cudaEventCreateWithFlags(&s->ev_dl[k], cudaEventDisableTiming);
  }
  if (e == cudaSuccess && !s->carry2) e = cudaMalloc(&s->carry2, 2 * sizeof(unsigned int));
  if (e == cudaSuccess && !s->olen_dev) e = cudaMalloc(&s->olen_dev, sizeof(unsigned long long));
  if (e == cudaSuccess) e = dev_grow(&s->buf, &s->buf_cap, n, false, 0, s->stream);
  if (e == cudaSuccess) e = dev_grow(&s->alt, &s->alt_cap, bound ? bound : 1, false, 0, s->stream);
  if (e == cudaSuccess) e = ensure_scratch(s, (2 * chunk + P + tile_bytes - 1) / tile_bytes + 1, proto.agg_entries);
  if (e == cudaSuccess) e = cudaMemsetAsync(s->carry2, 0, 2 * sizeof(unsigned int), s->stream);
  if (e != cudaSuccess) return (int)e;
  uint8_t* host = static_cast<uint8_t*>(pinned_pool().get(bound ? bound : 1, &e));
  if (!host) {
    cudaGetLastError();  // a page-locked block of the worst case was refused: the single-launch
    return kFallback;            // path allocates the result at its exact size
  }
  CopyOut copyout;
  if (dst) copyout.open(s->device);
  // Uploads. A page-locked input: every chunk's copy is queued at once. A pageable one: a
  // producer thread copies each chunk (on the copy workers) into one of kStageSlots page-locked
  // staging buffers and queues its upload from there, while this thread replaces and downloads
  // the chunks already up; ready counts the chunks whose upload (and event) is queued.
  constexpr int kStageSlots = 3;
  uint8_t* stage[kStageSlots] = {};
  std::mutex rmu;
  std::condition_variable rcv;
  size_t ready = 0;
  cudaError_t prod_err = cudaSuccess;
  std::atomic<bool> stop{false};
  std::thread producer;
  if (pinned) {
    for (size_t k = 0; k < nchunks && e == cudaSuccess; ++k) {
      const size_t a = bnd(k), m = bnd(k + 1) - a;
      e = cudaMemcpyAsync(s->buf + a, src + a, m, cudaMemcpyHostToDevice, s->up);
      if (e == cudaSuccess) e = cudaEventRecord(s->ev_up[k], s->up);
    }
    ready = nchunks;
  } else {
    for (int i = 0; i < kStageSlots && e == cudaSuccess; ++i) {
      if (!s->ev_stage[i]) e = cudaEventCreateWithFlags(&s->ev_stage[i], cudaEventDisableTiming);
      if (e == cudaSuccess) stage[i] = static_cast<uint8_t*>(pinned_pool().get(chunk + P, &e));
    }
    if (e == cudaSuccess) {
      const int dev = s->device;
      producer = std::thread([&, dev]() {
        cudaSetDevice(dev);
        cudaError_t pe = cudaSuccess;
        for (size_t k = 0; k < nchunks && pe == cudaSuccess && !stop.load(); ++k) {
          const int slot = (int)(k % kStageSlots);
          const size_t a = bnd(k), m = bnd(k + 1) - a;
          if (k >= (size_t)kStageSlots) pe = cudaEventSynchronize(s->ev_stage[slot]);  // the slot's upload is done
          if (pe != cudaSuccess) break;
          crb::parallel_memcpy(stage[slot], src + a, m);
          pe = cudaMemcpyAsync(s->buf + a, stage[slot], m, cudaMemcpyHostToDevice, s->up);
          if (pe == cudaSuccess) pe = cudaEventRecord(s->ev_up[k], s->up);
          if (pe == cudaSuccess) pe = cudaEventRecord(s->ev_stage[slot], s->up);
          std::lock_guard<std::mutex> g(rmu);
          if (pe == cudaSuccess) ready = k + 1;
          prod_err = pe;
          rcv.notify_all();
        }
        std::lock_guard<std::mutex> g(rmu);
        if (pe != cudaSuccess) prod_err = pe;
        rcv.notify_all();
      });
    }
  }
  int rc = (int)e;
  size_t O = 0;
  for (size_t k = 0; k < nchunks && rc == 0; ++k) {
    const size_t a = bnd(k), m = bnd(k + 1) - a;
    const bool first = k == 0, final = k + 1 == nchunks;
    if (!pinned) {  // wait until the producer has queued this chunk's upload
      std::unique_lock<std::mutex> lk(rmu);
      rcv.wait(lk, [&] { return ready > k || prod_err != cudaSuccess; });
      if (ready <= k) {
        rc = (int)prod_err;
        break;
      }
    }
    const size_t held = first ? 0 : P;  // the previous chunk's last bytes, matched again here
    ReplaceParams p = proto;
    p.in = s->buf + (a - held);  // k * chunk: 16-byte aligned
    p.n = held + m;
    p.hold = final ? 0 : P;
    p.carry0_dev = s->carry2 + (k & 1);
    p.carry_out = s->carry2 + ((k & 1) ^ 1);
    p.out = s->alt;
    p.out_cap = s->alt_cap;
    p.len_bias = O;
    p.len_out = s->olen_dev;
    p.num_tiles = (uint32_t)((p.n + tile_bytes - 1) / tile_bytes + 1);
    p.status = s->status;
    p.incl = s->incl;
    p.agg = s->agg;
    p.res = s->res;
    p.tile_last = s->tile_last;
    p.rec = s->rec;
    p.epoch = next_epoch(s);
    e = cudaStreamWaitEvent(s->stream, s->ev_up[k], 0);
    if (e == cudaSuccess) e = crb::launch_replace_super(p, s->stream, nullptr);
    if (e == cudaSuccess) {
      ++s->launches;
      e = cudaMemcpyAsync(s->res_host, s->res, sizeof(ApplyResult), cudaMemcpyDeviceToHost, s->stream);
    }
    if (e == cudaSuccess) e = cudaStreamSynchronize(s->stream);
    if (e != cudaSuccess) {
      rc = (int)e;
      break;
    }
    const ApplyResult r = *s->res_host;
    if (r.error_epoch == p.epoch || r.overflow_epoch == p.epoch) {
      rc = kErrUnknown;  // a bounded wait gave up (the buffer holds the worst case: no overflow)
      break;
    }
    const size_t olen = (size_t)r.out_len;
    if (olen) {
      e = cudaEventRecord(s->ev_done[k], s->stream);
      if (e == cudaSuccess) e = cudaStreamWaitEvent(s->down, s->ev_done[k], 0);
      if (e == cudaSuccess) e = cudaMemcpyAsync(host + O, s->alt + O, olen, cudaMemcpyDeviceToHost, s->down);
      if (e == cudaSuccess && dst) {
        e = cudaEventRecord(s->ev_dl[k], s->down);
        if (e == cudaSuccess) copyout.push(dst + O, host + O, olen, s->ev_dl[k]);
      }
      if (e != cudaSuccess) {
        rc = (int)e;
        break;
      }
    }
    O += olen;
  }
  stop.store(true);
  if (producer.joinable()) producer.join();
  const cudaError_t e0 = dst ? copyout.finish() : cudaSuccess;
  if (rc == 0 && e0 != cudaSuccess) rc = (int)e0;
  const cudaError_t e1 = cudaStreamSynchronize(s->down);
  const cudaError_t e2 = cudaStreamSynchronize(s->up);
  if (rc == 0 && e1 != cudaSuccess) rc = (int)e1;
  if (rc == 0 && e2 != cudaSuccess) rc = (int)e2;
  for (int i = 0; i < kStageSlots; ++i)
    if (stage[i]) pinned_pool().put(stage[i]);  // its uploads finished with the stream above
  s->len = 0;  // the session's buffers hold no complete content now
  ++s->buf_version;
  s->q_kind = 0;
  if (dst) {
    pinned_pool().put(host);  // its downloads and copies are done (both waited for above)
    if (rc == 0) *out_len = O;
    return rc;
  }
  if (rc != 0 || O == 0) {
    pinned_pool().put(host);
    return rc;
  }
  *out_host = host;
  *out_len = O;
  return 0;
}

CR_EXPORT int cuda_replace_unified(const uint8_t* src, size_t src_len, const uint8_t* pat, int pat_len,
                                   const uint8_t* rep, int rep_len, uint8_t** out_host, size_t* out_len) {
  if (!out_host || !out_len) return -1;
  *out_host = nullptr;
  *out_len = 0;
  int dev = 0;
  cudaError_t e = cudaGetDevice(&dev);
  if (e != cudaSuccess) return (int)e;
  Session* s = cache_take(dev);
  int rc = 0;
  if (!s) {
    rc = session_create(&s);
    if (rc != 0) return rc;
  }
  if (pat_len > 0 && rep_len >= 0 && pat && (rep || rep_len == 0)) {
    rc = unified_chunked(s, src, src_len, pat, (uint32_t)pat_len, rep, (uint32_t)rep_len, out_host, out_len);
    if (rc != kFallback) {
      if (rc == 0) {
        cache_give(s);
      } else {
        session_free(s);
        *out_host = nullptr;
        *out_len = 0;
      }
      return rc;
    }
    rc = 0;
  }
  rc = session_load(s, src, src_len);
  if (rc == 0) rc = apply_one(s, pat, pat_len, rep, rep_len, 0, nullptr, nullptr);
  if (rc == 0) rc = result_to_pinned(s, out_host, out_len);
  if (rc == 0) {
    cache_give(s);
  } else {
    session_free(s);
    *out_host = nullptr;
    *out_len = 0;
  }
  return rc;
}

CR_EXPORT int cuda_replace_output_bound(size_t src_len, int pat_len, int rep_len, size_t* bound) {
  if (!bound || pat_len < 0 || rep_len < 0) return -1;
  *bound = output_bound(src_len, (uint32_t)pat_len, (uint32_t)rep_len);
  return 0;
}

CR_EXPORT int cuda_replace_unified_into(const uint8_t* src, size_t src_len, const uint8_t* pat, int pat_len,
                                        const uint8_t* rep, int rep_len, uint8_t* dst, size_t dst_cap,
                                        size_t* out_len) {
  if (!out_len || pat_len < 0 || rep_len < 0 || (!src && src_len) || (!pat && pat_len) || (!rep && rep_len))
    return -1;
  *out_len = 0;
  if (pat_len > crb::kInlineMax || rep_len > crb::kInlineMax) return -4;
  int dev = 0;
  cudaError_t e = cudaGetDevice(&dev);
  if (e != cudaSuccess) return (int)e;
  Session* s = cache_take(dev);
  int rc = 0;
  if (!s) {
    rc = session_create(&s);
    if (rc != 0) return rc;
  }
  if (pat_len > 0 && dst) {
    uint8_t* unused = nullptr;
    rc = unified_chunked(s, src, src_len, pat, (uint32_t)pat_len, rep, (uint32_t)rep_len, &unused, out_len, dst,
                         dst_cap);
    if (rc != kFallback) {
      if (rc == 0) {
        cache_give(s);
      } else {
        session_free(s);
        *out_len = 0;
      }
      return rc;
    }
    rc = 0;
  }
  rc = session_load(s, src, src_len);
  if (rc == 0) rc = apply_one(s, pat, pat_len, rep, rep_len, 0, nullptr, nullptr);
  bool too_small = false;
  if (rc == 0) {
    *out_len = s->len;
    if (s->len > dst_cap) {
      too_small = true;
      rc = (int)cudaErrorInvalidValue;  // *out_len tells the length needed
    } else if (s->len >= ((size_t)32 << 20)) {
      // downloaded in up to kUnifiedChunks pieces into a pooled page-locked block, each piece
      // copied into dst as soon as it lands while the next ones download
      uint8_t* host = static_cast<uint8_t*>(pinned_pool().get(s->len, &e));
      const size_t piece = round_up((s->len + kUnifiedChunks - 1) / kUnifiedChunks, (size_t)1 << 20);
      CopyOut copyout;
      if (host) copyout.open(s->device);
      for (size_t off = 0, k = 0; host && e == cudaSuccess && off < s->len; off += piece, ++k) {
        const size_t m = std::min(piece, s->len - off);
        if (!s->ev_dl[k]) e = cudaEventCreateWithFlags(&s->ev_dl[k], cudaEventDisableTiming);
        if (e == cudaSuccess) e = cudaMemcpyAsync(host + off, s->buf + off, m, cudaMemcpyDeviceToHost, s->stream);
        if (e == cudaSuccess) e = cudaEventRecord(s->ev_dl[k], s->stream);
        if (e == cudaSuccess) copyout.push(dst + off, host + off, m, s->ev_dl[k]);
      }
      const cudaError_t e0 = copyout.finish();
      const cudaError_t e1 = cudaStreamSynchronize(s->stream);
      if (e == cudaSuccess) e = e0 != cudaSuccess ? e0 : e1;
      if (host) pinned_pool().put(host);
      rc = (int)e;
    } else if (s->len) {
      e = cudaMemcpyAsync(dst, s->buf, s->len, cudaMemcpyDeviceToHost, s->stream);
      if (e == cudaSuccess) e = cudaStreamSynchronize(s->stream);
      rc = (int)e;
    }
  }
  if (rc == 0 || too_small) {
    cache_give(s);
  } else {
    session_free(s);
    *out_len = 0;
  }
  return rc;
}
