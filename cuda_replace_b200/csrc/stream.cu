// stream.cu - replacement of an input larger than device memory: chunk-major, every pair
// applied to a chunk before the next chunk is read.
//
// The reference streams pair-major (cuda_replace_wrapper.py:305-366): for each pair it
// uploads every chunk, applies, queries and downloads, so the data crosses the host link
// twice per pair, and it drops the replacement of a match that straddles a chunk boundary
// (cuda_replace_wrapper.py:356). Here each pair is a stage of a chain that every chunk
// flows through on the device:
//
//   stage input  = [P held bytes][piece]      P = L - 1, piece = the previous stage's output
//   launch       : matches start before the held tail and may run into it; the output covers
//                  the same range; the carry says how many leading bytes a match kept in the
//                  previous chunk already covers (neither matched nor emitted); the last tile
//                  reports the coverage past the output range as the next chunk's carry
//   afterwards   : the last P bytes become the next chunk's held bytes
//
// At the first chunk the P held bytes do not exist; an initial carry of P covers them. The
// last chunk holds nothing back. Lengths between stages stay in device memory; the host reads
// them once per chunk. Carries and held bytes are double-buffered by chunk parity, so a chunk
// whose output overflowed a buffer runs again from intact inputs after the buffer grows. The
// next chunk's upload overlaps this chunk's stages and the previous chunk's download.
#include <cuda_runtime.h>

#include <unistd.h>

#include <algorithm>
#include <cerrno>
#include <cstdint>
#include <cstring>
#include <thread>
#include <vector>

#include "cuda_replace.h"
#include "host_pool.h"
#include "replace_kernels.h"

#define CR_EXPORT extern "C" __attribute__((visibility("default")))

namespace {

using crb::ApplyResult;
using crb::ReplaceParams;
using crb::TileIncl;

constexpr int kErrUnknown = 999;  // cudaErrorUnknown
constexpr int kUnsupported = -7;  // a pair outside the limits of this path
constexpr int kIoError = -10;     // reading the input or writing the output file failed (errno is kept)

size_t rup(size_t x, size_t q) { return (x + q - 1) / q * q; }

using crb::parallel_memcpy;

bool is_pinned(const void* p) {
  cudaPointerAttributes a;
  if (cudaPointerGetAttributes(&a, p) != cudaSuccess) {
    cudaGetLastError();
    return false;
  }
  return a.type == cudaMemoryTypeHost;
}

struct Stage {
  ReplaceParams proto;                    // pattern fields for every launch of this stage
  uint32_t P = 0;                         // held bytes (L - 1)
  uint8_t* pend[2] = {nullptr, nullptr};  // held bytes, by chunk parity
  double grow = 1.0;                      // output estimate factor, raised when this stage overflows
};

struct Stream {
  int count = 0;
  size_t chunk = 0;
  cudaStream_t comp = nullptr, h2d = nullptr, d2h = nullptr;
  std::vector<Stage> st;
  uint8_t* in0[2] = {nullptr, nullptr};  // stage 0 inputs [P held][chunk], by chunk parity
  size_t in0_cap = 0;
  uint8_t* x[2] = {nullptr, nullptr};    // inputs of stages >= 1 [P held][piece]; stage k writes x[k & 1]
  size_t xcap = 0;
  uint8_t* out[2] = {nullptr, nullptr};  // last stage outputs, by chunk parity
  size_t out_cap = 0;
  unsigned long long* lens = nullptr;    // [count]: input length of stage k (k >= 1)
  unsigned long long* outlen = nullptr;  // [2]
  unsigned int* carry = nullptr;         // [2 * count]: carry into stage k, by chunk parity
  uint32_t* status = nullptr;
  TileIncl* incl = nullptr;
  long long* tile_last = nullptr;
  unsigned long long* rec = nullptr;
  unsigned long long* agg = nullptr;
  size_t tiles_cap = 0, agg_cap = 0;
  ApplyResult* res = nullptr;
  ApplyResult* res_host = nullptr;
  unsigned long long* meta_host = nullptr;  // [count + 1]
  uint8_t* hin[2] = {nullptr, nullptr};     // page-locked staging of a pageable source
  cudaEvent_t ev_h2d[2] = {nullptr, nullptr}, ev_stage0[2] = {nullptr, nullptr}, ev_d2h[2] = {nullptr, nullptr};
  uint32_t epoch = 0;
  unsigned long long launches = 0;

  ~Stream() {
    if (comp) cudaStreamSynchronize(comp);
    if (h2d) cudaStreamSynchronize(h2d);
    if (d2h) cudaStreamSynchronize(d2h);
    for (auto& s : st)
      for (int b = 0; b < 2; ++b)
        if (s.pend[b]) cudaFree(s.pend[b]);
    for (int b = 0; b < 2; ++b) {
      if (in0[b]) cudaFree(in0[b]);
      if (x[b]) cudaFree(x[b]);
      if (out[b]) cudaFree(out[b]);
      if (hin[b]) crb::host_pinned_pool().put(hin[b]);
      if (ev_h2d[b]) cudaEventDestroy(ev_h2d[b]);
      if (ev_stage0[b]) cudaEventDestroy(ev_stage0[b]);
      if (ev_d2h[b]) cudaEventDestroy(ev_d2h[b]);
    }
    for (void* q : {(void*)lens, (void*)outlen, (void*)carry, (void*)status, (void*)incl, (void*)tile_last,
                    (void*)rec, (void*)agg, (void*)res})
      if (q) cudaFree(q);
    if (res_host) cudaFreeHost(res_host);
    if (meta_host) cudaFreeHost(meta_host);
    if (comp) cudaStreamDestroy(comp);
    if (h2d) cudaStreamDestroy(h2d);
    if (d2h) cudaStreamDestroy(d2h);
  }

  size_t tile_bytes(int k) const { return (size_t)crb::kTile * st[(size_t)k].proto.nsub; }

  // Output capacity planned for stage k with input capacity in_cap: a quarter over the
  // chunk, scaled by the stage's growth factor, never above the worst case of the pair.
  size_t out_estimate(int k, size_t in_cap) const {
    const Stage& s = st[(size_t)k];
    const size_t L = s.proto.L, R = s.proto.R;
    const size_t worst = R > L ? in_cap + (in_cap / L) * (R - L) : in_cap;
    const double est = (double)(chunk + chunk / 4 + (1u << 20)) * s.grow;
    return std::max<size_t>(16, est >= (double)worst ? worst : (size_t)est);
  }

  static cudaError_t regrow(uint8_t** p, size_t* cap, size_t want) {
    if (want <= *cap && *p) return cudaSuccess;
    if (*p) cudaFree(*p);
    *p = nullptr;
    const size_t c = rup(want, 1u << 20);
    const cudaError_t e = cudaMalloc(p, c + 64);  // + 64: reads rounded up to 16 bytes stay inside
    if (e == cudaSuccess) *cap = c;
    return e;
  }

  // (Re)allocate stage buffers and scratch for the current growth factors; only grows.
  cudaError_t size_buffers() {
    size_t in_cap = in0_cap, want_x = 0, want_out = 0, need_tiles = 1, need_agg = 1;
    for (int k = 0; k < count; ++k) {
      const size_t tiles = (in_cap + tile_bytes(k) - 1) / tile_bytes(k) + 1;
      need_tiles = std::max(need_tiles, tiles);
      need_agg = std::max(need_agg, tiles * st[(size_t)k].proto.agg_entries);
      const size_t est = out_estimate(k, in_cap);
      if (k + 1 < count) {
        want_x = std::max(want_x, st[(size_t)k + 1].P + est);
        in_cap = std::max(want_x, xcap);
      } else {
        want_out = est;
      }
    }
    cudaError_t e = cudaSuccess;
    if (want_x > xcap) {
      size_t c0 = xcap, c1 = xcap;
      e = regrow(&x[0], &c0, want_x);
      if (e == cudaSuccess) e = regrow(&x[1], &c1, want_x);
      if (e != cudaSuccess) return e;
      xcap = std::min(c0, c1);
    }
    if (want_out > out_cap) {
      size_t c0 = out_cap, c1 = out_cap;
      e = regrow(&out[0], &c0, want_out);
      if (e == cudaSuccess) e = regrow(&out[1], &c1, want_out);
      if (e != cudaSuccess) return e;
      out_cap = std::min(c0, c1);
    }
    if (need_tiles > tiles_cap) {
      for (void* q : {(void*)status, (void*)incl, (void*)tile_last, (void*)rec})
        if (q) cudaFree(q);
      status = nullptr;
      incl = nullptr;
      tile_last = nullptr;
      rec = nullptr;
      const size_t cap = need_tiles + 64;
      e = cudaMalloc(&status, cap * sizeof(uint32_t));
      if (e == cudaSuccess) e = cudaMalloc(&incl, cap * sizeof(TileIncl));
      if (e == cudaSuccess) e = cudaMalloc(&tile_last, cap * sizeof(long long));
      if (e == cudaSuccess) e = cudaMalloc(&rec, cap * 2 * sizeof(unsigned long long));
      if (e == cudaSuccess) e = cudaMemsetAsync(status, 0, cap * sizeof(uint32_t), comp);
      if (e == cudaSuccess) e = cudaMemsetAsync(rec, 0, cap * 2 * sizeof(unsigned long long), comp);
      if (e != cudaSuccess) return e;
      tiles_cap = cap;
    }
    if (need_agg > agg_cap) {
      if (agg) cudaFree(agg);
      agg = nullptr;
      e = cudaMalloc(&agg, (need_agg + 1024) * sizeof(unsigned long long));
      if (e != cudaSuccess) return e;
      agg_cap = need_agg + 1024;
    }
    return cudaSuccess;
  }

  // Make the next k epochs consecutive and free of a record-tag (24-bit) or status (30-bit)
  // wrap, so that the launches of one chunk carry epochs first .. first + k - 1.
  cudaError_t reserve_epochs(uint32_t k) {
    const bool tag_wrap = (epoch & 0xFFFFFFu) + k + 1u >= 0x1000000u;
    const bool st_wrap = epoch + k + 2u >= (1u << 30);
    if (!tag_wrap && !st_wrap) return cudaSuccess;
    cudaError_t e = cudaMemsetAsync(status, 0, tiles_cap * sizeof(uint32_t), comp);
    if (e == cudaSuccess) e = cudaMemsetAsync(rec, 0, tiles_cap * 2 * sizeof(unsigned long long), comp);
    if (e == cudaSuccess && st_wrap) e = cudaMemsetAsync(res, 0, sizeof(ApplyResult), comp);
    epoch = st_wrap ? 0u : (epoch | 0xFFFFFFu) + 1u;  // tag 0 is the cleared state: never issued
    return e;
  }

  // Enqueue every stage of one chunk (m new bytes in in0[b] after the P_0 held bytes).
  cudaError_t run_chunk(int b, size_t m, bool first, bool final, uint32_t* first_epoch) {
    cudaError_t e = reserve_epochs((uint32_t)count);
    if (e != cudaSuccess) return e;
    *first_epoch = epoch + 1;
    for (int k = 0; k < count; ++k) {
      Stage& s = st[(size_t)k];
      uint8_t* in = k == 0 ? in0[b] : x[(k - 1) & 1];
      if (s.P) {
        e = cudaMemcpyAsync(in, s.pend[b], s.P, cudaMemcpyDeviceToDevice, comp);
        if (e != cudaSuccess) return e;
      }
      ReplaceParams p = s.proto;
      p.in = in;
      size_t in_cap;
      if (k == 0) {
        p.n = s.P + m;
        in_cap = p.n;
      } else {
        p.n_dev = lens + k;
        p.n_cap = xcap;
        in_cap = xcap;
      }
      p.num_tiles = (uint32_t)((in_cap + tile_bytes(k) - 1) / tile_bytes(k) + 1);
      p.hold = final ? 0 : s.P;
      // At the first chunk the held bytes are placeholders: no match may start in them (the
      // carry covers them too, but a pattern without a border keeps every occurrence it finds).
      p.block_before = first ? s.P : 0;
      p.carry0_dev = carry + 2 * k + b;
      p.carry_out = carry + 2 * k + (b ^ 1);
      if (k + 1 < count) {
        p.out = x[k & 1];
        p.out_cap = xcap;
        p.len_out = lens + k + 1;
        p.len_bias = st[(size_t)k + 1].P;  // the next stage's held bytes go in front
      } else {
        e = cudaStreamWaitEvent(comp, ev_d2h[b], 0);  // out[b] may still feed a download
        if (e != cudaSuccess) return e;
        p.out = out[b];
        p.out_cap = out_cap;
        p.len_out = outlen + b;
        p.len_bias = 0;
      }
      p.status = status;
      p.incl = incl;
      p.agg = agg;
      p.res = res;
      p.tile_last = tile_last;
      p.rec = rec;
      p.epoch = ++epoch;
      e = crb::launch_replace_super(p, comp, nullptr);
      if (e != cudaSuccess) return e;
      ++launches;
      if (k == 0) {
        e = cudaEventRecord(ev_stage0[b], comp);
        if (e != cudaSuccess) return e;
      }
      if (s.P && !final) {
        if (k == 0) {
          e = cudaMemcpyAsync(s.pend[b ^ 1], in + m, s.P, cudaMemcpyDeviceToDevice, comp);
        } else {
          e = crb::launch_move_tail(in, lens + k, xcap, s.P, s.pend[b ^ 1], comp);
          ++launches;
        }
        if (e != cudaSuccess) return e;
      }
    }
    // meta_host[1, count): stage input lengths, [count]: this chunk's output length
    e = cudaMemcpyAsync(meta_host, lens, (size_t)count * sizeof(unsigned long long), cudaMemcpyDeviceToHost, comp);
    if (e == cudaSuccess)
      e = cudaMemcpyAsync(meta_host + count, outlen + b, sizeof(unsigned long long), cudaMemcpyDeviceToHost, comp);
    if (e == cudaSuccess) e = cudaMemcpyAsync(res_host, res, sizeof(ApplyResult), cudaMemcpyDeviceToHost, comp);
    return e;
  }
};

// Pair checks, buffers, streams and initial carries of a chunk-major stream over chunks of
// `chunk` bytes. staging: page-locked buffers for the chunks (S.hin) are needed.
int stream_setup(Stream& S, const uint8_t** pats, const int* pat_lens, const uint8_t** reps, const int* rep_lens,
                 int count, size_t chunk, bool staging) {
  crb::PinnedPool& pool = crb::host_pinned_pool();
  S.count = count;
  S.st.resize((size_t)count);
  for (int k = 0; k < count; ++k) {
    const int pl = pat_lens[k], rl = rep_lens[k];
    if (pl < 0 || rl < 0 || (pl && !pats[k]) || (rl && !reps[k])) return -1;
    if (pl == 0 || pl > crb::kInlineMax || rl > crb::kInlineMax) return kUnsupported;
    ReplaceParams& p = S.st[(size_t)k].proto;
    memset(&p, 0, sizeof(p));
    crb::prepare_pattern_fields(p, pats[k], (uint32_t)pl);
    p.R = (uint32_t)rl;
    p.nsub = crb::super_nsub(p.mode, p.L);
    if (!p.nsub) return kUnsupported;  // bordered pattern longer than the super-tile kernel takes
    memcpy(p.pat, pats[k], (size_t)pl);
    if (rl) memcpy(p.rep, reps[k], (size_t)rl);
    S.st[(size_t)k].P = (uint32_t)pl - 1;
  }
  S.chunk = chunk;
  cudaError_t e = cudaStreamCreateWithFlags(&S.comp, cudaStreamNonBlocking);
  if (e == cudaSuccess) e = cudaStreamCreateWithFlags(&S.h2d, cudaStreamNonBlocking);
  if (e == cudaSuccess) e = cudaStreamCreateWithFlags(&S.d2h, cudaStreamNonBlocking);
  for (int b = 0; b < 2 && e == cudaSuccess; ++b) {
    e = cudaEventCreateWithFlags(&S.ev_h2d[b], cudaEventDisableTiming);
    if (e == cudaSuccess) e = cudaEventCreateWithFlags(&S.ev_stage0[b], cudaEventDisableTiming);
    if (e == cudaSuccess) e = cudaEventCreateWithFlags(&S.ev_d2h[b], cudaEventDisableTiming);
  }
  S.in0_cap = S.st[0].P + S.chunk;
  for (int b = 0; b < 2 && e == cudaSuccess; ++b) {
    e = cudaMalloc(&S.in0[b], rup(S.in0_cap, 1u << 20) + 64);
    if (e == cudaSuccess && staging) S.hin[b] = static_cast<uint8_t*>(pool.get(S.chunk, &e));
  }
  for (int k = 0; k < count && e == cudaSuccess; ++k)
    for (int b = 0; b < 2 && e == cudaSuccess; ++b) {
      e = cudaMalloc(&S.st[(size_t)k].pend[b], 256);
      if (e == cudaSuccess) e = cudaMemsetAsync(S.st[(size_t)k].pend[b], 0, 256, S.comp);
    }
  if (e == cudaSuccess) e = cudaMalloc(&S.lens, (size_t)(count + 1) * sizeof(unsigned long long));
  if (e == cudaSuccess) e = cudaMemsetAsync(S.lens, 0, (size_t)(count + 1) * sizeof(unsigned long long), S.comp);
  if (e == cudaSuccess) e = cudaMalloc(&S.outlen, 2 * sizeof(unsigned long long));
  if (e == cudaSuccess) e = cudaMalloc(&S.carry, (size_t)2 * count * sizeof(unsigned int));
  if (e == cudaSuccess) e = cudaMalloc(&S.res, sizeof(ApplyResult));
  if (e == cudaSuccess) e = cudaMemsetAsync(S.res, 0, sizeof(ApplyResult), S.comp);
  if (e == cudaSuccess) e = cudaMallocHost(&S.res_host, sizeof(ApplyResult));
  if (e == cudaSuccess) e = cudaMallocHost(&S.meta_host, (size_t)(count + 2) * sizeof(unsigned long long));
  if (e == cudaSuccess) e = S.size_buffers();
  if (e != cudaSuccess) return (int)e;
  // every stage starts with its P held bytes covered: at the first chunk they do not exist
  std::vector<unsigned int> c0((size_t)2 * count, 0u);
  for (int k = 0; k < count; ++k) c0[(size_t)2 * k] = S.st[(size_t)k].P;
  e = cudaMemcpyAsync(S.carry, c0.data(), c0.size() * sizeof(unsigned int), cudaMemcpyHostToDevice, S.comp);
  if (e == cudaSuccess) e = cudaStreamSynchronize(S.comp);
  return (int)e;
}

// Enqueue every stage of chunk c (in parity b, m new bytes), wait for it, and grow the buffer
// that overflowed and run it again until it fits. after_enqueue runs once, on the host, while
// the first attempt computes (the next chunk's upload, file I/O). Returns 0 or an error code.
template <typename F>
int run_chunk_fitting(Stream& S, int b, size_t m, bool first, bool final, F&& after_enqueue) {
  for (int attempt = 0;; ++attempt) {
    cudaError_t e = cudaStreamWaitEvent(S.comp, S.ev_h2d[b], 0);
    uint32_t e0 = 0;
    if (e == cudaSuccess) e = S.run_chunk(b, m, first, final, &e0);
    if (e == cudaSuccess && attempt == 0) e = after_enqueue();  // overlaps this chunk's stages
    if (e == cudaSuccess) e = cudaStreamSynchronize(S.comp);
    if (e != cudaSuccess) return (int)e;
    const ApplyResult r = *S.res_host;
    const uint32_t e1 = e0 + (uint32_t)S.count - 1u;
    if (r.error_epoch >= e0 && r.error_epoch <= e1) return kErrUnknown;  // a bounded wait gave up
    if (!(r.overflow_epoch >= e0 && r.overflow_epoch <= e1)) return 0;
    // The chunk's inputs (in0[b], pend[b], the carries of parity b) are intact: grow the buffer
    // that overflowed and run the chunk again. The first stage whose output length passed its
    // buffer is the one that overflowed (later stages read a clamped input); that length is
    // exact, so one regrow per stage suffices.
    int k = S.count - 1;
    unsigned long long need = S.meta_host[S.count];
    for (int j = 0; j + 1 < S.count; ++j)
      if (S.meta_host[j + 1] > S.xcap) {
        k = j;
        need = S.meta_host[j + 1];
        break;
      }
    const double base = (double)(S.chunk + S.chunk / 4 + (1u << 20));
    const double g = std::max(S.st[(size_t)k].grow * 2.0, 1.125 * (double)need / base);
    for (int j = k; j < S.count; ++j) S.st[(size_t)j].grow = std::max(S.st[(size_t)j].grow, g);
    if (attempt >= 2 * S.count + 8) return kErrUnknown;
    e = cudaStreamSynchronize(S.d2h);  // out[] may be replaced
    if (e == cudaSuccess) e = S.size_buffers();
    if (e != cudaSuccess) return (int)e;
  }
}

int stream_replace(const uint8_t* src, size_t n, const uint8_t** pats, const int* pat_lens, const uint8_t** reps,
                   const int* rep_lens, int count, size_t chunk_bytes, uint8_t** out_host, size_t* out_len) {
  crb::PinnedPool& pool = crb::host_pinned_pool();
  Stream S;
  for (int k = 0; k < count; ++k)
    if (pat_lens[k] < 0 || rep_lens[k] < 0 || (pat_lens[k] && !pats[k]) || (rep_lens[k] && !reps[k])) return -1;
  if (n == 0) {  // nothing matches in an empty input; the pairs must still be ones this path takes
    for (int k = 0; k < count; ++k)
      if (pat_lens[k] == 0 || pat_lens[k] > crb::kInlineMax || rep_lens[k] > crb::kInlineMax) return kUnsupported;
    for (int k = 0; k < count; ++k) {
      ReplaceParams q;
      memset(&q, 0, sizeof(q));
      crb::prepare_pattern_fields(q, pats[k], (uint32_t)pat_lens[k]);
      if (!crb::super_nsub(q.mode, q.L)) return kUnsupported;
    }
    return 0;
  }
  const bool src_pinned = is_pinned(src);
  const int src_rc = stream_setup(S, pats, pat_lens, reps, rep_lens, count,
                                  std::max<size_t>(1, std::min(chunk_bytes ? chunk_bytes : (256u << 20), n)),
                                  !src_pinned);
  if (src_rc != 0) return src_rc;
  cudaError_t e;

  // the result: page-locked, from the pool; grows by half when a chunk does not fit. One pair:
  // sized for the most matches it can keep (n / L of them), up to four times the input.
  size_t ocap = n + n / 8 + (64u << 20), written = 0;
  if (count == 1) {
    const size_t L = (size_t)pat_lens[0], R = (size_t)rep_lens[0];
    const size_t bound = R > L ? n + (n / L) * (R - L) : n;
    ocap = std::min(bound, 4 * n + (64u << 20)) + 64;
  }
  uint8_t* hout = static_cast<uint8_t*>(pool.get(ocap, &e));
  if (!hout) return (int)e;

  const size_t nchunks = (n + S.chunk - 1) / S.chunk;
  auto upload = [&](size_t c) -> cudaError_t {
    const int b = (int)(c & 1);
    const size_t pos = c * S.chunk, m = std::min(S.chunk, n - pos);
    const uint8_t* from = src + pos;
    cudaError_t err;
    if (!src_pinned) {
      err = cudaEventSynchronize(S.ev_h2d[b]);  // hin[b] is free once its previous upload finished
      if (err != cudaSuccess) return err;
      parallel_memcpy(S.hin[b], from, m);
      from = S.hin[b];
    }
    err = cudaStreamWaitEvent(S.h2d, S.ev_stage0[b], 0);  // in0[b] no longer read
    if (err == cudaSuccess) err = cudaMemcpyAsync(S.in0[b] + S.st[0].P, from, m, cudaMemcpyHostToDevice, S.h2d);
    if (err == cudaSuccess) err = cudaEventRecord(S.ev_h2d[b], S.h2d);
    return err;
  };
  int rc = 0;
  e = upload(0);
  if (e != cudaSuccess) rc = (int)e;
  for (size_t c = 0; c < nchunks && rc == 0; ++c) {
    const int b = (int)(c & 1);
    const size_t m = std::min(S.chunk, n - c * S.chunk);
    const bool final = c + 1 == nchunks;
    rc = run_chunk_fitting(S, b, m, c == 0, final, [&]() { return final ? cudaSuccess : upload(c + 1); });
    if (rc) break;
    const size_t olen = (size_t)S.meta_host[count];
    if (written + olen > ocap) {
      e = cudaStreamSynchronize(S.d2h);
      const size_t ncap = std::max(written + olen, ocap + ocap / 2);
      uint8_t* bigger = e == cudaSuccess ? static_cast<uint8_t*>(pool.get(ncap, &e)) : nullptr;
      if (!bigger) {
        rc = (int)e;
        break;
      }
      parallel_memcpy(bigger, hout, written);
      pool.put(hout);
      hout = bigger;
      ocap = ncap;
    }
    if (olen) {
      e = cudaMemcpyAsync(hout + written, S.out[b], olen, cudaMemcpyDeviceToHost, S.d2h);
      if (e != cudaSuccess) {
        rc = (int)e;
        break;
      }
    }
    e = cudaEventRecord(S.ev_d2h[b], S.d2h);
    if (e != cudaSuccess) {
      rc = (int)e;
      break;
    }
    written += olen;
  }
  if (rc == 0) {
    e = cudaStreamSynchronize(S.d2h);
    if (e == cudaSuccess) e = cudaStreamSynchronize(S.h2d);
    if (e != cudaSuccess) rc = (int)e;
  }
  if (rc != 0) {
    cudaStreamSynchronize(S.d2h);
    pool.put(hout);
    return rc;
  }
  if (written == 0) {
    pool.put(hout);
    hout = nullptr;
  }
  *out_host = hout;
  *out_len = written;
  return 0;
}

// read() until m bytes are in or the input ends; the bytes read, or -1 on an error (errno set).
long long read_full(int fd, uint8_t* dst, size_t m) {
  size_t got = 0;
  while (got < m) {
    const ssize_t r = ::read(fd, dst + got, m - got);
    if (r < 0) {
      if (errno == EINTR) continue;
      return -1;
    }
    if (r == 0) break;
    got += (size_t)r;
  }
  return (long long)got;
}

bool write_full(int fd, const uint8_t* src, size_t m) {
  size_t put = 0;
  while (put < m) {
    const ssize_t w = ::write(fd, src + put, m - put);
    if (w < 0) {
      if (errno == EINTR) continue;
      return false;
    }
    put += (size_t)w;
  }
  return true;
}

// The chunk-major stream between two file descriptors: chunks are read into two page-locked
// buffers (the next one while the current one is on the device), every pair is applied to a
// chunk on the device, and each chunk's output is downloaded into one of two page-locked
// buffers and written out while the next chunk computes. Neither the input nor the output is
// held whole in memory, and the input may be a pipe (its end is found by reading ahead).
int stream_fd(int in_fd, int out_fd, const uint8_t** pats, const int* pat_lens, const uint8_t** reps,
              const int* rep_lens, int count, size_t chunk_bytes, unsigned long long* in_bytes,
              unsigned long long* out_bytes) {
  crb::PinnedPool& pool = crb::host_pinned_pool();
  Stream S;
  int rc = stream_setup(S, pats, pat_lens, reps, rep_lens, count, chunk_bytes ? chunk_bytes : (256u << 20), true);
  if (rc != 0) return rc;
  uint8_t* obuf[2] = {nullptr, nullptr};
  size_t ocap[2] = {0, 0};
  unsigned long long tin = 0, tout = 0;
  auto upload = [&](int b, size_t m) -> cudaError_t {
    cudaError_t err = cudaStreamWaitEvent(S.h2d, S.ev_stage0[b], 0);  // in0[b] no longer read
    if (err == cudaSuccess) err = cudaMemcpyAsync(S.in0[b] + S.st[0].P, S.hin[b], m, cudaMemcpyHostToDevice, S.h2d);
    if (err == cudaSuccess) err = cudaEventRecord(S.ev_h2d[b], S.h2d);
    return err;
  };
  long long m_cur = read_full(in_fd, S.hin[0], S.chunk);
  if (m_cur < 0) return kIoError;
  cudaError_t e = cudaSuccess;
  int prev_b = -1;  // a downloaded chunk not written yet
  size_t prev_len = 0;
  bool io_fail = false;
  auto flush_prev = [&]() -> cudaError_t {
    if (prev_b < 0) return cudaSuccess;
    const cudaError_t err = cudaEventSynchronize(S.ev_d2h[prev_b]);
    if (err != cudaSuccess) return err;
    if (prev_len && !write_full(out_fd, obuf[prev_b], prev_len)) io_fail = true;
    prev_b = -1;
    return cudaSuccess;
  };
  if (m_cur > 0) {
    tin = (unsigned long long)m_cur;
    e = upload(0, (size_t)m_cur);
    if (e != cudaSuccess) rc = (int)e;
  }
  for (size_t c = 0; m_cur > 0 && rc == 0 && !io_fail; ++c) {
    const int b = (int)(c & 1);
    e = cudaEventSynchronize(S.ev_h2d[b ^ 1]);  // hin[b ^ 1] fed the previous chunk's upload
    if (e != cudaSuccess) {
      rc = (int)e;
      break;
    }
    const long long m_next = read_full(in_fd, S.hin[b ^ 1], S.chunk);  // read ahead: is this the last?
    if (m_next < 0) {
      io_fail = true;
      break;
    }
    const bool final = m_next == 0;
    rc = run_chunk_fitting(S, b, (size_t)m_cur, c == 0, final, [&]() {
      cudaError_t err = final ? cudaSuccess : upload(b ^ 1, (size_t)m_next);
      if (err == cudaSuccess) err = flush_prev();  // the previous chunk's output, while this one computes
      return err;
    });
    if (rc) break;
    e = flush_prev();  // (a chunk that needed a rerun reached here without the write)
    if (e != cudaSuccess) {
      rc = (int)e;
      break;
    }
    const size_t olen = (size_t)S.meta_host[count];
    if (olen > ocap[b]) {
      if (obuf[b]) pool.put(obuf[b]);
      obuf[b] = static_cast<uint8_t*>(pool.get(olen + olen / 8, &e));
      if (!obuf[b]) {
        rc = (int)e;
        break;
      }
      ocap[b] = olen + olen / 8;
    }
    if (olen) e = cudaMemcpyAsync(obuf[b], S.out[b], olen, cudaMemcpyDeviceToHost, S.d2h);
    if (e == cudaSuccess) e = cudaEventRecord(S.ev_d2h[b], S.d2h);
    if (e != cudaSuccess) {
      rc = (int)e;
      break;
    }
    prev_b = b;
    prev_len = olen;
    tout += olen;
    m_cur = m_next;
    tin += (unsigned long long)m_next;
  }
  if (rc == 0) {
    e = flush_prev();
    if (e != cudaSuccess) rc = (int)e;
  }
  cudaStreamSynchronize(S.d2h);
  cudaStreamSynchronize(S.h2d);
  for (int b = 0; b < 2; ++b)
    if (obuf[b]) pool.put(obuf[b]);
  if (rc == 0 && io_fail) rc = kIoError;
  if (in_bytes) *in_bytes = tin;
  if (out_bytes) *out_bytes = tout;
  return rc;
}

}  // namespace

CR_EXPORT int cuda_replace_stream_fd(int in_fd, int out_fd, const uint8_t** pats, const int* pat_lens,
                                     const uint8_t** reps, const int* rep_lens, int count, size_t chunk_bytes,
                                     unsigned long long* in_bytes, unsigned long long* out_bytes) {
  if (in_fd < 0 || out_fd < 0 || count < 0 || (count > 0 && (!pats || !pat_lens || !reps || !rep_lens))) return -1;
  if (in_bytes) *in_bytes = 0;
  if (out_bytes) *out_bytes = 0;
  if (count == 0) {  // no pair: the output is the input
    std::vector<uint8_t> buf((size_t)8 << 20);
    unsigned long long total = 0;
    for (;;) {
      const long long m = read_full(in_fd, buf.data(), buf.size());
      if (m < 0) return kIoError;
      if (m == 0) break;
      if (!write_full(out_fd, buf.data(), (size_t)m)) return kIoError;
      total += (unsigned long long)m;
    }
    if (in_bytes) *in_bytes = total;
    if (out_bytes) *out_bytes = total;
    return 0;
  }
  return stream_fd(in_fd, out_fd, pats, pat_lens, reps, rep_lens, count, chunk_bytes, in_bytes, out_bytes);
}

CR_EXPORT int cuda_replace_stream(const uint8_t* src, size_t n, const uint8_t** pats, const int* pat_lens,
                                  const uint8_t** reps, const int* rep_lens, int count, size_t chunk_bytes,
                                  uint8_t** out_host, size_t* out_len) {
  if (!out_host || !out_len || (n && !src) || count < 0 || (count > 0 && (!pats || !pat_lens || !reps || !rep_lens)))
    return -1;
  *out_host = nullptr;
  *out_len = 0;
  if (count == 0) {
    if (n == 0) return 0;
    cudaError_t e;
    uint8_t* h = static_cast<uint8_t*>(crb::host_pinned_pool().get(n, &e));
    if (!h) return (int)e;
    parallel_memcpy(h, src, n);
    *out_host = h;
    *out_len = n;
    return 0;
  }
  return stream_replace(src, n, pats, pat_lens, reps, rep_lens, count, chunk_bytes, out_host, out_len);
}
