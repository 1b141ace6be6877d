// noalloc.cu - a replace entry point that allocates no memory.
//
// Some callers cannot allocate device memory at the moment they need a replace: code
// running under a memory pool or arena that owns the whole device budget, real-time or
// plugin hosts that forbid cudaMalloc/cudaFree (both can synchronise the device and stall
// other streams), and code paths that must not fail on an out-of-memory error halfway
// through. cuda_replace_apply_device_noalloc serves them: the caller passes device input
// and output buffers, and the look-back scratch that the single-pass kernel needs (tile
// status words, inclusive prefixes, tile carry functions, the result block) lives in one
// file-scope __device__ array of fixed size, which every GPU that loads this library
// holds until the process exits.
//
// Limits (checked before anything is launched; see cuda_replace.h):
//   input  <= CUDA_REPLACE_NOALLOC_MAX_INPUT bytes (64 MiB = 4096 tiles of 16 KiB)
//   pattern 1..64 bytes, replacement 0..256 bytes
// The array is shared by every call on a device and keeps the previous call's contents.
// Tile status words carry a per-call epoch, so stale words are never mistaken for fresh
// ones; the two scheduler counters that must start at zero are cleared by each call.
// Calls whose work overlaps on the GPU (two streams, two host threads) race on the array
// and must not be issued; successive calls on one stream are fine.
#include <cuda_runtime.h>

#include <atomic>
#include <cstdint>
#include <cstring>
#include <mutex>

#include "cuda_replace.h"
#include "replace_kernels.h"

#define CR_EXPORT extern "C" __attribute__((visibility("default")))

namespace {

constexpr size_t kMaxInput = (size_t)CUDA_REPLACE_NOALLOC_MAX_INPUT;
constexpr uint32_t kMaxPat = 64;
constexpr uint32_t kMaxRep = 256;
constexpr size_t kTiles = kMaxInput / crb::kTile;
constexpr size_t kStatusOff = 0;
constexpr size_t kInclOff = (kStatusOff + kTiles * sizeof(unsigned int) + 255) / 256 * 256;
constexpr size_t kAggOff = (kInclOff + kTiles * sizeof(crb::TileIncl) + 255) / 256 * 256;
constexpr size_t kResOff = (kAggOff + kTiles * kMaxPat * sizeof(unsigned long long) + 255) / 256 * 256;
constexpr size_t kScratchBytes = kResOff + (sizeof(crb::ApplyResult) + 255) / 256 * 256;

static_assert(kMaxInput % crb::kTile == 0, "whole tiles");

// The only storage this entry point uses on the device (about 2.1 MiB).
static __device__ __align__(256) unsigned char g_noalloc_scratch[kScratchBytes];

constexpr int kMaxDevices = 64;

struct DeviceSlot {
  std::once_flag once;
  cudaError_t setup_err = cudaSuccess;
  unsigned char* base = nullptr;  // device address of g_noalloc_scratch on this device
  std::atomic<uint32_t> epoch{0};
};

DeviceSlot g_slots[kMaxDevices];

// Knuth-Morris-Pratt failure function on a stack array (pattern <= kMaxPat bytes).
bool pattern_has_border(const uint8_t* pat, uint32_t L) {
  if (L < 2) return false;
  uint32_t fail[kMaxPat];
  fail[0] = 0;
  uint32_t k = 0;
  for (uint32_t i = 1; i < L; ++i) {
    while (k > 0 && pat[i] != pat[k]) k = fail[k - 1];
    if (pat[i] == pat[k]) ++k;
    fail[i] = k;
  }
  return fail[L - 1] > 0;
}

}  // namespace

CR_EXPORT int cuda_replace_apply_device_noalloc(const uint8_t* d_in, size_t n, const uint8_t* pat, int pat_len,
                                                const uint8_t* rep, int rep_len, uint8_t* d_out, size_t out_cap,
                                                size_t* out_len, void* stream) {
  if (!out_len || !pat || !d_out || (n && !d_in) || (rep_len > 0 && !rep)) return -1;
  if (pat_len < 1 || rep_len < 0) return -1;
  if ((uint32_t)pat_len > kMaxPat || (uint32_t)rep_len > kMaxRep || n > kMaxInput) return -6;
  if (((uintptr_t)d_in & 15u) || ((uintptr_t)d_out & 15u)) return (int)cudaErrorInvalidValue;
  const uint32_t L = (uint32_t)pat_len, R = (uint32_t)rep_len;
  const size_t bound = R > L ? n + (n / L) * (R - L) : n;
  if (out_cap < bound) return (int)cudaErrorInvalidValue;
  cudaStream_t st = static_cast<cudaStream_t>(stream);
  *out_len = 0;
  if (n < L) {  // no occurrence possible: the output is the input
    if (n) {
      cudaError_t e = cudaMemcpyAsync(d_out, d_in, n, cudaMemcpyDeviceToDevice, st);
      if (e == cudaSuccess) e = cudaStreamSynchronize(st);
      if (e != cudaSuccess) return (int)e;
    }
    *out_len = n;
    return 0;
  }

  int dev = 0;
  cudaError_t e = cudaGetDevice(&dev);
  if (e != cudaSuccess) return (int)e;
  if (dev < 0 || dev >= kMaxDevices) return (int)cudaErrorInvalidDevice;
  DeviceSlot& slot = g_slots[dev];
  // First call on this device: look up the device address of the array (the device is current).
  std::call_once(slot.once, [&slot]() {
    void* p = nullptr;
    slot.setup_err = cudaGetSymbolAddress(&p, g_noalloc_scratch);
    slot.base = static_cast<unsigned char*>(p);
  });
  if (slot.setup_err != cudaSuccess) return (int)slot.setup_err;

  crb::ReplaceParams p;
  memset(&p, 0, sizeof(p));
  p.L = L;
  p.R = R;
  p.mode = pattern_has_border(pat, L) ? crb::kModeSmall : crb::kModeFree;
  for (uint32_t i = 0; i < 4 && i < L; ++i) {
    p.p4 |= (uint32_t)pat[i] << (8 * i);
    p.m4 |= 0xFFu << (8 * i);
  }
  p.inv_l = L < 64 ? (65536u + L - 1) / L : 0u;
  p.stride_mask = 1ull;
  if (L < 64) {
    p.stride_mask = 0;
    for (uint32_t b = 0; b < 64; b += L) p.stride_mask |= 1ull << b;
  }
  p.agg_entries = p.mode == crb::kModeFree ? 1u : L;
  memcpy(p.pat, pat, L);
  if (R) memcpy(p.rep, rep, R);
  p.in = d_in;
  p.out = d_out;
  p.n = n;
  p.out_cap = out_cap;
  p.num_tiles = (uint32_t)((n + crb::kTile - 1) / crb::kTile);
  p.status = reinterpret_cast<unsigned int*>(slot.base + kStatusOff);
  p.incl = reinterpret_cast<crb::TileIncl*>(slot.base + kInclOff);
  p.agg = reinterpret_cast<unsigned long long*>(slot.base + kAggOff);
  p.res = reinterpret_cast<crb::ApplyResult*>(slot.base + kResOff);

  uint32_t epoch = slot.epoch.fetch_add(1) + 1;
  if (epoch >= (1u << 30) - 2) {  // epoch wrap: clear the status words, restart at 1
    e = cudaMemsetAsync(p.status, 0, kTiles * sizeof(unsigned int), st);
    if (e != cudaSuccess) return (int)e;
    slot.epoch.store(1);
    epoch = 1;
  }
  p.epoch = epoch;
  // the dynamic tile scheduler and the exit counter must start at zero
  e = cudaMemsetAsync(&p.res->tile_counter, 0, 2 * sizeof(unsigned int), st);
  if (e != cudaSuccess) return (int)e;
  e = crb::launch_replace(p, st, nullptr);
  if (e != cudaSuccess) return (int)e;
  crb::ApplyResult r;
  e = cudaMemcpyAsync(&r, p.res, sizeof(r), cudaMemcpyDeviceToHost, st);
  if (e == cudaSuccess) e = cudaStreamSynchronize(st);
  if (e != cudaSuccess) return (int)e;
  if (r.error_epoch == epoch || r.overflow_epoch == epoch) return 999;
  *out_len = (size_t)r.out_len;
  return 0;
}
