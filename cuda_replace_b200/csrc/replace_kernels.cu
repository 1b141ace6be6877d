// replace_kernels.cu - sm_100a kernels for leftmost, non-overlapping byte-pattern
// replacement (bytes.replace semantics) in one pass over HBM.
//
// Reference behaviour being replaced (RAZZULLIX/cuda_replace, cuda_replace.cu):
//   mark      cuda_replace.cu:447-477, 717-734   (one thread per position, bool[n] bitmap)
//   suppress  cuda_replace.cu:737-884, 905-968   (thread-0 / <<<1,1>>> serial greedy)
//   scan      cuda_replace.cu:237-352, 1223-1244 (three-stage scan, 32-bit local offsets)
//   scatter   cuda_replace.cu:1391-1608          (u16 padded array, range-sliced expand)
// Here all four are one launch:
//   1. TMA (cp.async.bulk) stages a 16 KiB tile plus an (L-1)-byte halo in shared memory.
//   2. Each thread owns 64 bytes; it compares the first min(L,4) pattern bytes at all 64
//      positions with funnel shifts over 32-bit words and verifies the rest only for the
//      survivors, producing a 64-bit candidate mask.
//   3. The greedy leftmost rule is a function of the carry "blocked until" (how many
//      leading bytes are covered by an earlier kept match). Each thread tabulates its
//      segment's function over every carry in [0, L) by walking the candidate mask run
//      by run; warps and then the tile compose the tables; the tile publishes its
//      function and resolves its exact carry-in and 64-bit kept-count prefix with a
//      decoupled look-back over its predecessors (bounded waits).
//   4. With the exact carry each thread re-walks its mask to get the kept starts, a
//      block scan gives every thread its output offset, the output is assembled in a
//      shared-memory window aligned to the global 16-byte grid and written with TMA
//      bulk stores (edge bytes with plain byte stores).
// There is no floating point and no tensor-core work: the path is HBM-bound byte work.
#include "replace_kernels.h"

#include <algorithm>
#include <cstring>
#include <mutex>

namespace crb {

namespace {

constexpr unsigned long long kSpinLimitNs = 2000000000ull;  // 2 s per bounded wait

__host__ __device__ __forceinline__ uint32_t align_up_u32(uint32_t x, uint32_t a) { return (x + a - 1) / a * a; }

// ---------------------------------------------------------------- shared memory layout
struct Layout {
  uint32_t tile, pat, rep, outb, masks, segtab, srec, wtab, wrec, ttab, segcarry, total;
  uint32_t eseg;  // segment-table entries per segment (carries 0 .. eseg-1)
  uint32_t rs;    // segment-table row stride in entries (odd: conflict-free column access)
};

__host__ __device__ __forceinline__ Layout make_layout(uint32_t mode, uint32_t L, uint32_t R) {
  Layout s{};
  uint32_t off = 0;
  s.tile = off;
  off += align_up_u32(kTile + (L > 1 ? L - 1 : 0), 16) + 32;  // + slack for the 17th word read
  s.pat = off;
  off += align_up_u32(L > 0 ? L : 1, 16);
  s.rep = off;
  off += align_up_u32(R > 0 ? R : 1, 16);
  s.outb = off;
  off += kOutWin + 32;
  s.masks = off;
  off += kThreads * 8;
  if (mode != kModeFree) {
    s.eseg = L < 64 ? L : 64;
    s.rs = s.eseg | 1u;
    s.segtab = off;
    off += align_up_u32(kThreads * s.rs * 4, 16);
    if (mode == kModeSmall) {
      s.srec = off;
      off += align_up_u32(kThreads * L, 16);
      s.wtab = off;
      off += align_up_u32(kWarps * L * 4, 16);
      s.wrec = off;
      off += align_up_u32(kWarps * L, 16);
      s.ttab = off;
      off += align_up_u32(L * 8, 16);
    } else {
      s.segcarry = off;
      off += kThreads * 4;
    }
  }
  s.total = off;
  return s;
}

// ---------------------------------------------------------------- PTX wrappers
__device__ __forceinline__ uint32_t smem_u32(const void* p) {
  return static_cast<uint32_t>(__cvta_generic_to_shared(p));
}
__device__ __forceinline__ void mbar_init(uint64_t* bar, uint32_t count) {
  asm volatile("mbarrier.init.shared::cta.b64 [%0], %1;" ::"r"(smem_u32(bar)), "r"(count) : "memory");
}
__device__ __forceinline__ void fence_mbar_init() {
  asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
}
__device__ __forceinline__ void mbar_arrive_expect_tx(uint64_t* bar, uint32_t bytes) {
  asm volatile("mbarrier.arrive.expect_tx.shared::cta.b64 _, [%0], %1;" ::"r"(smem_u32(bar)), "r"(bytes)
               : "memory");
}
__device__ __forceinline__ bool mbar_try_wait(uint64_t* bar, uint32_t parity) {
  uint32_t ok;
  asm volatile(
      "{\n\t.reg .pred p;\n\t"
      "mbarrier.try_wait.parity.shared::cta.b64 p, [%1], %2;\n\t"
      "selp.u32 %0, 1, 0, p;\n\t}"
      : "=r"(ok)
      : "r"(smem_u32(bar)), "r"(parity)
      : "memory");
  return ok != 0;
}
__device__ __forceinline__ void bulk_load(void* dst_smem, const void* src_gmem, uint32_t bytes, uint64_t* bar) {
  asm volatile(
      "cp.async.bulk.shared::cluster.global.mbarrier::complete_tx::bytes [%0], [%1], %2, [%3];" ::"r"(
          smem_u32(dst_smem)),
      "l"(src_gmem), "r"(bytes), "r"(smem_u32(bar))
      : "memory");
}
__device__ __forceinline__ void bulk_store(void* dst_gmem, const void* src_smem, uint32_t bytes) {
  asm volatile("cp.async.bulk.global.shared::cta.bulk_group [%0], [%1], %2;" ::"l"(dst_gmem),
               "r"(smem_u32(src_smem)), "r"(bytes)
               : "memory");
}
__device__ __forceinline__ void bulk_commit() { asm volatile("cp.async.bulk.commit_group;" ::: "memory"); }
__device__ __forceinline__ void bulk_wait_read_all() {
  asm volatile("cp.async.bulk.wait_group.read 0;" ::: "memory");
}
__device__ __forceinline__ void bulk_wait_all() { asm volatile("cp.async.bulk.wait_group 0;" ::: "memory"); }
__device__ __forceinline__ void fence_proxy_async_smem() {
  asm volatile("fence.proxy.async.shared::cta;" ::: "memory");
}
__device__ __forceinline__ uint32_t ld_acquire_u32(const uint32_t* p) {
  uint32_t v;
  asm volatile("ld.acquire.gpu.global.u32 %0, [%1];" : "=r"(v) : "l"(p) : "memory");
  return v;
}
__device__ __forceinline__ void st_release_u32(uint32_t* p, uint32_t v) {
  asm volatile("st.release.gpu.global.u32 [%0], %1;" ::"l"(p), "r"(v) : "memory");
}
__device__ __forceinline__ unsigned long long global_ns() {
  unsigned long long t;
  asm volatile("mov.u64 %0, %%globaltimer;" : "=l"(t));
  return t;
}

// ---------------------------------------------------------------- small helpers
__device__ __forceinline__ uint64_t low_bits(uint32_t b) { return b >= 64 ? ~0ull : ((1ull << b) - 1ull); }

// Tile function entry (global, 64-bit): [0,32) kept count, [32,48) carry-out, [48,64) last kept + 1.
__host__ __device__ __forceinline__ unsigned long long pack_tile(uint32_t cnt, uint32_t carry, uint32_t last1) {
  return (unsigned long long)cnt | ((unsigned long long)carry << 32) | ((unsigned long long)last1 << 48);
}
__device__ __forceinline__ uint32_t tile_cnt(unsigned long long e) { return (uint32_t)e; }
__device__ __forceinline__ uint32_t tile_carry(unsigned long long e) { return (uint32_t)(e >> 32) & 0xFFFFu; }
__device__ __forceinline__ uint32_t tile_last1(unsigned long long e) { return (uint32_t)(e >> 48); }

// Segment entry (shared, 32-bit): [0,7) kept count, [7,14) last kept + 1, [14,32) carry-out.
__device__ __forceinline__ uint32_t pack_seg(uint32_t cnt, uint32_t carry, uint32_t last1) {
  return cnt | (last1 << 7) | (carry << 14);
}
// Warp entry (shared, 32-bit): [0,12) kept count, [12,24) last kept + 1, [24,32) carry-out.
__device__ __forceinline__ uint32_t pack_warp(uint32_t cnt, uint32_t carry, uint32_t last1) {
  return cnt | (last1 << 12) | (carry << 24);
}

// Candidate mask of one 64-byte segment: bit i set when the first min(L,4) pattern bytes
// match at segment byte i. s is 16-byte aligned in shared memory; reads 68 bytes.
__device__ __forceinline__ uint64_t seg_candidates4(const uint8_t* s, uint32_t p4, uint32_t m4) {
  uint32_t w[17];
  const uint4* v = reinterpret_cast<const uint4*>(s);
#pragma unroll
  for (int i = 0; i < 4; ++i) {
    const uint4 q = v[i];
    w[4 * i + 0] = q.x;
    w[4 * i + 1] = q.y;
    w[4 * i + 2] = q.z;
    w[4 * i + 3] = q.w;
  }
  w[16] = *reinterpret_cast<const uint32_t*>(s + 64);
  uint32_t lo = 0, hi = 0;
#pragma unroll
  for (int i = 0; i < 16; ++i) {
#pragma unroll
    for (int j = 0; j < 4; ++j) {
      const uint32_t x = (j == 0) ? w[i] : __funnelshift_r(w[i], w[i + 1], 8 * j);
      const uint32_t hit = (((x ^ p4) & m4) == 0u) ? 1u : 0u;
      const int pos = 4 * i + j;
      if (pos < 32)
        lo |= hit << pos;
      else
        hi |= hit << (pos - 32);
    }
  }
  return ((uint64_t)hi << 32) | lo;
}

// Drop candidates whose pattern bytes [4, L) do not match.
__device__ __forceinline__ uint64_t verify_tail(uint64_t mask, const uint8_t* s, const uint8_t* pat, uint32_t L) {
  uint64_t m = mask;
  while (m) {
    const int p = __ffsll((long long)m) - 1;
    m &= m - 1;
    const uint8_t* a = s + p + 4;
    for (uint32_t k = 0; k + 4 < L; ++k) {
      if (a[k] != pat[4 + k]) {
        mask &= ~(1ull << p);
        break;
      }
    }
  }
  return mask;
}

struct Walk {
  uint64_t kept;   // kept starts (bits)
  uint32_t cnt;    // number kept
  uint32_t end;    // blocked-until, relative to the segment start (carry-out = end - 64 when > 64)
};

// Greedy leftmost selection over one 64-bit candidate mask, starting blocked until x.
// Consecutive candidates form runs; inside a run [p, q) the kept starts are p, p+L, ...
// so the walk costs one step per run, not per match.
__device__ __forceinline__ Walk seg_walk(uint64_t mask, uint32_t x, uint32_t L, uint32_t inv_l, uint64_t stride) {
  Walk w{0ull, 0u, x};
  while (x < 64) {
    const uint64_t m = mask >> x;
    if (m == 0) break;
    const uint32_t p = x + (uint32_t)(__ffsll((long long)m) - 1);
    const uint64_t r = ~(mask >> p);
    const uint32_t q = r ? p + (uint32_t)(__ffsll((long long)r) - 1) : 64u;
    const uint32_t run = q - p;
    const uint32_t k = (L >= 64) ? 1u : (((run + L - 1) * inv_l) >> 16);
    const uint32_t span = (k - 1) * L;
    w.kept |= (stride << p) & low_bits(p + span + 1);
    w.cnt += k;
    x = p + k * L;
  }
  w.end = x;
  return w;
}

// Segment function over carries c in [0, eseg): entry c = result of the walk started at
// the first candidate at or after c. Only one walk per distinct first candidate.
__device__ __forceinline__ void build_seg_table(uint64_t mask, uint32_t L, uint32_t eseg, uint32_t inv_l,
                                                uint64_t stride, uint32_t* row) {
  uint32_t c = 0;
  while (c < eseg) {
    const uint64_t m = mask >> c;
    if (m == 0) {
      for (; c < eseg; ++c) row[c] = pack_seg(0, 0, 0);
      break;
    }
    const uint32_t e = c + (uint32_t)(__ffsll((long long)m) - 1);
    const Walk w = seg_walk(mask, e, L, inv_l, stride);
    const uint32_t carry = w.end > 64 ? w.end - 64 : 0;
    const uint32_t last1 = 64u - (uint32_t)__clzll((long long)w.kept);
    const uint32_t v = pack_seg(w.cnt, carry, last1);
    const uint32_t hi = min(e + 1, eseg);
    for (; c < hi; ++c) row[c] = v;
  }
}

template <typename Op>
__device__ __forceinline__ uint32_t warp_incl_scan(uint32_t v, Op op) {
  const uint32_t lane = threadIdx.x & 31;
#pragma unroll
  for (int d = 1; d < 32; d <<= 1) {
    const uint32_t o = __shfl_up_sync(0xffffffffu, v, d);
    if (lane >= (uint32_t)d) v = op(v, o);
  }
  return v;
}

// Block-wide exclusive scan with a commutative, associative op. scratch holds kWarps words.
template <typename Op>
__device__ __forceinline__ uint32_t block_excl_scan(uint32_t v, uint32_t identity, Op op, uint32_t* scratch,
                                                    uint32_t* total) {
  const uint32_t lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
  const uint32_t inc = warp_incl_scan(v, op);
  if (lane == 31) scratch[warp] = inc;
  __syncthreads();
  uint32_t wpre = identity, tot = identity;
#pragma unroll
  for (int w = 0; w < kWarps; ++w) {
    const uint32_t s = scratch[w];
    if ((uint32_t)w < warp) wpre = op(wpre, s);
    tot = op(tot, s);
  }
  __syncthreads();
  uint32_t ex = __shfl_up_sync(0xffffffffu, inc, 1);
  if (lane == 0) ex = identity;
  *total = tot;
  return op(wpre, ex);
}

struct OpSum {
  __device__ __forceinline__ uint32_t operator()(uint32_t a, uint32_t b) const { return a + b; }
};
struct OpMax {
  __device__ __forceinline__ uint32_t operator()(uint32_t a, uint32_t b) const { return a > b ? a : b; }
};

__device__ __forceinline__ void set_error(const ReplaceParams& p) {
  atomicExch(&p.res->error_epoch, p.epoch);
}
__device__ __forceinline__ bool aborted(const ReplaceParams& p) {
  return *reinterpret_cast<volatile unsigned int*>(&p.res->error_epoch) == p.epoch;
}

// Bounded wait for the TMA load of the current tile.
__device__ __forceinline__ bool wait_tile(uint64_t* bar, uint32_t phase) {
  if (mbar_try_wait(bar, phase)) return true;
  const unsigned long long t0 = global_ns();
  for (;;) {
    if (mbar_try_wait(bar, phase)) return true;
    if (global_ns() - t0 > kSpinLimitNs) return false;
  }
}

// Bounded wait until tile j of this epoch has published at least its aggregate.
// Returns the state (kStAgg or kStInc) or 0 when the wait gave up.
__device__ __forceinline__ uint32_t wait_status(const ReplaceParams& p, uint32_t j) {
  const uint32_t want = p.epoch << 2;
  uint32_t s = ld_acquire_u32(p.status + j);
  if ((s & ~3u) == want && (s & 3u)) return s & 3u;
  const unsigned long long t0 = global_ns();
  uint32_t ns = 32;
  for (;;) {
    __nanosleep(ns);
    if (ns < 1024) ns <<= 1;
    s = ld_acquire_u32(p.status + j);
    if ((s & ~3u) == want && (s & 3u)) return s & 3u;
    if (aborted(p)) return 0;
    if (global_ns() - t0 > kSpinLimitNs) {
      set_error(p);
      return 0;
    }
  }
}

// Entry of tile i's published function for carry-in c; *carry_out receives its carry-out.
template <int MODE>
__device__ __forceinline__ unsigned long long agg_lookup(const ReplaceParams& p, uint32_t i, uint32_t c,
                                                         uint32_t* carry_out) {
  if (MODE == kModeFree) {
    const unsigned long long e = __ldcg(p.agg + i);
    const uint32_t shifted = c > (uint32_t)kTile ? c - (uint32_t)kTile : 0u;
    const uint32_t lco = tile_carry(e);
    *carry_out = shifted > lco ? shifted : lco;
    return e;
  } else {
    const uint32_t E = p.agg_entries;
    if (c < E) {
      const unsigned long long e = __ldcg(p.agg + (unsigned long long)i * E + c);
      *carry_out = tile_carry(e);
      return e;
    }
    *carry_out = c - (uint32_t)kTile;  // c >= E == kTile: the whole tile is covered
    return 0ull;
  }
}

// Copy len bytes to output positions [o, o + len), clipped to the window [w0, w1).
__device__ __forceinline__ void copy_clip(uint8_t* ob, uint32_t o, const uint8_t* src, uint32_t len,
                                          uint32_t w0, uint32_t w1) {
  uint32_t a = o > w0 ? o : w0;
  const uint32_t b = (o + len) < w1 ? (o + len) : w1;
  for (; a < b; ++a) ob[a - w0] = src[a - o];
}

}  // namespace

// ============================================================================ main kernel
template <int MODE>
__global__ void __launch_bounds__(kThreads) replace_tiles_kernel(const __grid_constant__ ReplaceParams p) {
  extern __shared__ __align__(128) uint8_t smem[];
  __shared__ __align__(8) uint64_t s_bar;
  __shared__ uint32_t s_tile;
  __shared__ uint32_t s_scan[kWarps];
  __shared__ unsigned long long s_kexcl;
  __shared__ long long s_lastexcl;
  __shared__ uint32_t s_cin;
  __shared__ uint32_t s_own_cnt, s_own_lco, s_own_last1;
  __shared__ uint32_t s_fail;

  const uint32_t L = p.L, R = p.R;
  const Layout lay = make_layout(MODE, L, R);
  uint8_t* tb = smem + lay.tile;
  uint8_t* ps = smem + lay.pat;
  uint8_t* rs = smem + lay.rep;
  uint8_t* ob = smem + lay.outb;
  const uint32_t tid = threadIdx.x, lane = tid & 31u, warp = tid >> 5;
  const uint32_t sb = tid * kSeg;

  {
    const uint8_t* psrc = L <= (uint32_t)kInlineMax ? p.pat : p.pat_ext;
    const uint8_t* rsrc = R <= (uint32_t)kInlineMax ? p.rep : p.rep_ext;
    for (uint32_t i = tid; i < L; i += kThreads) ps[i] = psrc[i];
    for (uint32_t i = tid; i < R; i += kThreads) rs[i] = rsrc[i];
  }
  if (tid == 0) {
    mbar_init(&s_bar, 1);
    fence_mbar_init();
  }
  uint32_t phase = 0;
  const unsigned long long n = p.n;
  const unsigned long long n16 = (n + 15ull) & ~15ull;
  const uint32_t want_bytes = align_up_u32(kTile + (L > 1 ? L - 1 : 0), 16);

  for (;;) {
    __syncthreads();
    if (tid == 0) {
      s_tile = atomicAdd(&p.res->tile_counter, 1u);
      s_fail = 0;
    }
    __syncthreads();
    const uint32_t t = s_tile;
    if (t >= p.num_tiles) break;
    const unsigned long long tstart = (unsigned long long)t * kTile;

    // ---- 1. stage tile + halo with one bulk copy
    if (tid == 0) {
      const unsigned long long avail = n16 - tstart;
      const uint32_t bytes = avail < want_bytes ? (uint32_t)avail : want_bytes;
      fence_proxy_async_smem();
      mbar_arrive_expect_tx(&s_bar, bytes);
      bulk_load(tb, p.in + tstart, bytes, &s_bar);
    }
    if (!wait_tile(&s_bar, phase)) {
      if (tid == 0) {
        set_error(p);
        s_fail = 1;
      }
    }
    phase ^= 1u;

    // ---- 2. candidates of this thread's 64-byte segment
    const unsigned long long gseg = tstart + sb;
    uint64_t mask = seg_candidates4(tb + sb, p.p4, p.m4);
    {
      uint32_t lo = 0, hi = 0;
      if (p.block_before > gseg) {
        const unsigned long long d = p.block_before - gseg;
        lo = d < 64ull ? (uint32_t)d : 64u;
      }
      if (n >= L && n - L + 1 > gseg) {
        const unsigned long long d = n - L + 1 - gseg;
        hi = d < 64ull ? (uint32_t)d : 64u;
      }
      mask &= low_bits(hi) & ~low_bits(lo);
    }
    if (L > 4) mask = verify_tail(mask, tb + sb, ps, L);

    // ---- 3. tile function, aggregate publication
    uint32_t pre_cend = 0;  // kModeFree: max cover end (tile-relative) of earlier segments
    if (MODE == kModeFree) {
      const uint32_t cnt = (uint32_t)__popcll(mask);
      const uint32_t last = mask ? 63u - (uint32_t)__clzll((long long)mask) : 0u;
      const uint32_t cend = mask ? sb + last + L : 0u;
      const uint32_t last1 = mask ? sb + last + 1u : 0u;
      uint32_t tot_cend, tot_cnt, tot_last1;
      pre_cend = block_excl_scan(cend, 0u, OpMax(), s_scan, &tot_cend);
      (void)block_excl_scan(cnt, 0u, OpSum(), s_scan, &tot_cnt);
      (void)block_excl_scan(last1, 0u, OpMax(), s_scan, &tot_last1);
      if (tid == 0) {
        s_own_cnt = tot_cnt;
        s_own_lco = tot_cend > (uint32_t)kTile ? tot_cend - (uint32_t)kTile : 0u;
        s_own_last1 = tot_last1;
        if (t > 0) {
          __stcg(p.agg + t, pack_tile(tot_cnt, s_own_lco, tot_last1));
          __threadfence();
          st_release_u32(p.status + t, (p.epoch << 2) | kStAgg);
        }
      }
    } else if (MODE == kModeSmall) {
      uint32_t* segtab = reinterpret_cast<uint32_t*>(smem + lay.segtab);
      build_seg_table(mask, L, lay.eseg, p.inv_l, p.stride_mask, segtab + tid * lay.rs);
      __syncthreads();
      uint8_t* srec = smem + lay.srec;
      uint32_t* wtab = reinterpret_cast<uint32_t*>(smem + lay.wtab);
      for (uint32_t c = lane; c < L; c += 32) {
        uint32_t x = c, cnt = 0, last1 = 0;
        const uint32_t seg0 = warp * 32u;
#pragma unroll 4
        for (uint32_t k = 0; k < 32; ++k) {
          const uint32_t seg = seg0 + k;
          srec[seg * L + c] = (uint8_t)x;
          const uint32_t v = segtab[seg * lay.rs + x];
          const uint32_t vc = v & 127u;
          if (vc) {
            cnt += vc;
            last1 = k * 64u + ((v >> 7) & 127u);
          }
          x = v >> 14;
        }
        wtab[warp * L + c] = pack_warp(cnt, x, last1);
      }
      __syncthreads();
      if (warp == 0) {
        uint8_t* wrec = smem + lay.wrec;
        unsigned long long* ttab = reinterpret_cast<unsigned long long*>(smem + lay.ttab);
        for (uint32_t c = lane; c < L; c += 32) {
          uint32_t x = c, cnt = 0, last1 = 0;
#pragma unroll
          for (uint32_t w = 0; w < (uint32_t)kWarps; ++w) {
            wrec[w * L + c] = (uint8_t)x;
            const uint32_t v = wtab[w * L + x];
            const uint32_t vc = v & 4095u;
            if (vc) {
              cnt += vc;
              last1 = w * 2048u + ((v >> 12) & 4095u);
            }
            x = v >> 24;
          }
          const unsigned long long e = pack_tile(cnt, x, last1);
          ttab[c] = e;
          if (t > 0) __stcg(p.agg + (unsigned long long)t * L + c, e);
        }
        __threadfence();
      }
      __syncthreads();
      if (tid == 0 && t > 0) st_release_u32(p.status + t, (p.epoch << 2) | kStAgg);
    } else {  // kModeLarge
      uint32_t* segtab = reinterpret_cast<uint32_t*>(smem + lay.segtab);
      build_seg_table(mask, L, lay.eseg, p.inv_l, p.stride_mask, segtab + tid * lay.rs);
      __syncthreads();
      if (t > 0) {
        const uint32_t E = p.agg_entries;
        for (uint32_t c = tid; c < E; c += kThreads) {
          uint32_t x = c, cnt = 0, last1 = 0;
          for (uint32_t seg = 0; seg < (uint32_t)kThreads; ++seg) {
            if (x >= 64u) {
              x -= 64u;
              continue;
            }
            const uint32_t v = segtab[seg * lay.rs + x];
            const uint32_t vc = v & 127u;
            if (vc) {
              cnt += vc;
              last1 = seg * 64u + ((v >> 7) & 127u);
            }
            x = v >> 14;
          }
          __stcg(p.agg + (unsigned long long)t * E + c, pack_tile(cnt, x, last1));
        }
        __threadfence();
      }
      __syncthreads();
      if (tid == 0 && t > 0) st_release_u32(p.status + t, (p.epoch << 2) | kStAgg);
    }

    // ---- 4. decoupled look-back: exact carry-in and kept prefix of this tile
    if (tid == 0) {
      unsigned long long K = 0;
      long long last = -1;
      uint32_t c = 0;
      if (t > 0) {
        uint32_t j = t - 1;
        bool ok = true;
        for (;;) {
          const uint32_t st = wait_status(p, j);
          if (st == 0) {
            ok = false;
            break;
          }
          if (st == kStInc) break;
          --j;  // tile 0 always publishes an inclusive prefix, so j never passes 0
        }
        if (ok) {
          const TileIncl* in = p.incl + j;
          K = __ldcg(&in->kept);
          last = __ldcg(&in->last);
          c = __ldcg(&in->carry);
          for (uint32_t i = j + 1; i < t; ++i) {
            uint32_t co;
            const unsigned long long e = agg_lookup<MODE>(p, i, c, &co);
            K += tile_cnt(e);
            const uint32_t l1 = tile_last1(e);
            if (l1) last = (long long)((unsigned long long)i * kTile + l1 - 1);
            c = co;
          }
        } else {
          s_fail = 1;
        }
      }
      s_kexcl = K;
      s_lastexcl = last;
      s_cin = c;

      // own inclusive prefix
      uint32_t own_cnt = 0, own_carry = 0, own_last1 = 0;
      if (MODE == kModeFree) {
        own_cnt = s_own_cnt;
        const uint32_t shifted = c > (uint32_t)kTile ? c - (uint32_t)kTile : 0u;
        own_carry = shifted > s_own_lco ? shifted : s_own_lco;
        own_last1 = s_own_last1;
      } else if (MODE == kModeSmall) {
        const unsigned long long e = reinterpret_cast<unsigned long long*>(smem + lay.ttab)[c];
        own_cnt = tile_cnt(e);
        own_carry = tile_carry(e);
        own_last1 = tile_last1(e);
      } else {
        const uint32_t* segtab = reinterpret_cast<const uint32_t*>(smem + lay.segtab);
        uint32_t* segcarry = reinterpret_cast<uint32_t*>(smem + lay.segcarry);
        uint32_t x = c;
        for (uint32_t seg = 0; seg < (uint32_t)kThreads; ++seg) {
          segcarry[seg] = x;
          if (x >= 64u) {
            x -= 64u;
            continue;
          }
          const uint32_t v = segtab[seg * lay.rs + x];
          const uint32_t vc = v & 127u;
          if (vc) {
            own_cnt += vc;
            own_last1 = seg * 64u + ((v >> 7) & 127u);
          }
          x = v >> 14;
        }
        own_carry = x;
      }
      TileIncl* mine = p.incl + t;
      __stcg(&mine->kept, K + own_cnt);
      __stcg(&mine->last, own_last1 ? (long long)(tstart + own_last1 - 1) : last);
      __stcg(&mine->carry, own_carry);
      __threadfence();
      st_release_u32(p.status + t, (p.epoch << 2) | kStInc);
    }
    __syncthreads();
    const uint32_t cin = s_cin;
    const unsigned long long kexcl = s_kexcl;

    // ---- 5. exact kept starts of this segment
    uint32_t x_in;
    uint64_t kept;
    uint32_t cnt;
    if (MODE == kModeFree) {
      const uint32_t cov = cin > pre_cend ? cin : pre_cend;
      x_in = cov > sb ? cov - sb : 0u;
      kept = mask;
      cnt = (uint32_t)__popcll(mask);
    } else {
      if (MODE == kModeSmall) {
        const uint32_t cw = (smem + lay.wrec)[warp * L + cin];
        x_in = (smem + lay.srec)[tid * L + cw];
      } else {
        x_in = reinterpret_cast<const uint32_t*>(smem + lay.segcarry)[tid];
      }
      if (x_in >= 64u) {
        kept = 0;
        cnt = 0;
      } else {
        const Walk w = seg_walk(mask, x_in, L, p.inv_l, p.stride_mask);
        kept = w.kept;
        cnt = w.cnt;
      }
    }

    // ---- 6. output length and offset of this segment
    const uint32_t V = gseg >= n ? 0u : ((n - gseg) < 64ull ? (uint32_t)(n - gseg) : 64u);
    uint32_t covered = x_in < V ? x_in : V;
    if (cnt) {
      const uint32_t lastk = 63u - (uint32_t)__clzll((long long)kept);
      const uint32_t over = (lastk + L > V) ? lastk + L - V : 0u;
      covered += cnt * L - over;
    }
    const uint32_t olen = V - covered + cnt * R;
    uint32_t tile_olen;
    const uint32_t ooff = block_excl_scan(olen, 0u, OpSum(), s_scan, &tile_olen);
    const long long delta = (long long)R - (long long)L;
    const unsigned long long O_t =
        (unsigned long long)((long long)(tstart + cin) + (long long)kexcl * delta);

    if (tid == 0 && t == p.num_tiles - 1) {
      TileIncl* mine = p.incl + t;
      p.res->out_len = O_t + tile_olen;
      p.res->kept = __ldcg(&mine->kept);
      p.res->last_kept = __ldcg(&mine->last);
    }
    const bool fits = (O_t + tile_olen <= p.out_cap) && (O_t <= p.out_cap);
    if (!fits && tid == 0) atomicExch(&p.res->overflow_epoch, p.epoch);
    if (!fits || s_fail) continue;

    // ---- 7. assemble output windows in shared memory, store with TMA
    for (uint32_t w0 = 0; w0 < tile_olen; w0 += kOutWin) {
      const uint32_t w1 = (w0 + kOutWin) < tile_olen ? (w0 + kOutWin) : tile_olen;
      const unsigned long long g0 = O_t + w0;
      const uint32_t sh = (uint32_t)(g0 & 15ull);
      uint8_t* obw = ob + sh;  // output byte o lives at obw[o - w0]
      if (olen && ooff < w1 && ooff + olen > w0) {
        const uint8_t* src = tb + sb;
        uint32_t o = ooff;
        uint32_t pos = x_in < V ? x_in : V;
        while (pos < V) {
          const uint64_t km = pos < 64u ? (kept >> pos) : 0ull;
          uint32_t nk = km ? pos + (uint32_t)(__ffsll((long long)km) - 1) : V;
          if (nk > V) nk = V;
          copy_clip(obw, o, src + pos, nk - pos, w0, w1);
          o += nk - pos;
          if (nk >= V) break;
          copy_clip(obw, o, rs, R, w0, w1);
          o += R;
          pos = nk + L;
        }
      }
      fence_proxy_async_smem();
      __syncthreads();
      const unsigned long long gend = O_t + w1;
      const unsigned long long a0 = (g0 + 15ull) & ~15ull;
      const unsigned long long a1 = gend & ~15ull;
      if (a1 > a0) {
        if (tid == 0) {
          bulk_store(p.out + a0, ob + sh + (uint32_t)(a0 - g0), (uint32_t)(a1 - a0));
          bulk_commit();
        }
        if (tid < (uint32_t)(a0 - g0)) p.out[g0 + tid] = obw[tid];
        if (tid >= 32u && tid - 32u < (uint32_t)(gend - a1))
          p.out[a1 + (tid - 32u)] = obw[(uint32_t)(a1 - g0) + (tid - 32u)];
      } else {
        for (uint32_t i = tid; i < (uint32_t)(gend - g0); i += kThreads) p.out[g0 + i] = obw[i];
      }
      if (tid == 0) bulk_wait_read_all();
      __syncthreads();
    }
  }

  // ---- exit: drain bulk stores, reset the tile scheduler when the last CTA leaves
  if (tid == 0) {
    bulk_wait_all();
    __threadfence();
    const unsigned int d = atomicAdd(&p.res->done_ctas, 1u);
    if (d == gridDim.x - 1) {
      atomicExch(&p.res->tile_counter, 0u);
      atomicExch(&p.res->done_ctas, 0u);
      __threadfence();
    }
  }
}

// ============================================================================ query kernel
// One CTA re-derives the kept starts of one tile from the tile records of the last apply
// (exact carry-in from the predecessor's inclusive prefix) and counts those before limit.
template <int MODE>
__global__ void __launch_bounds__(kThreads) query_tile_kernel(const __grid_constant__ ReplaceParams p) {
  extern __shared__ __align__(128) uint8_t smem[];
  __shared__ __align__(8) uint64_t s_bar;
  __shared__ uint32_t s_ok;
  const uint32_t L = p.L;
  const Layout lay = make_layout(kModeFree, L, p.R);
  uint8_t* tb = smem + lay.tile;
  uint8_t* ps = smem + lay.pat;
  uint64_t* masks = reinterpret_cast<uint64_t*>(smem + lay.masks);
  const uint32_t tid = threadIdx.x;
  const uint32_t sb = tid * kSeg;
  const uint32_t t = p.query_tile;
  const unsigned long long tstart = (unsigned long long)t * kTile;
  const unsigned long long n = p.n;
  {
    const uint8_t* psrc = L <= (uint32_t)kInlineMax ? p.pat : p.pat_ext;
    for (uint32_t i = tid; i < L; i += kThreads) ps[i] = psrc[i];
  }
  if (tid == 0) {
    mbar_init(&s_bar, 1);
    fence_mbar_init();
    s_ok = 1;
  }
  __syncthreads();
  if (tid == 0) {
    const unsigned long long n16 = (n + 15ull) & ~15ull;
    const uint32_t want = align_up_u32(kTile + (L > 1 ? L - 1 : 0), 16);
    const unsigned long long avail = n16 - tstart;
    const uint32_t bytes = avail < want ? (uint32_t)avail : want;
    fence_proxy_async_smem();
    mbar_arrive_expect_tx(&s_bar, bytes);
    bulk_load(tb, p.in + tstart, bytes, &s_bar);
  }
  if (!wait_tile(&s_bar, 0)) {
    if (tid == 0) s_ok = 0;
  }
  const unsigned long long gseg = tstart + sb;
  uint64_t mask = seg_candidates4(tb + sb, p.p4, p.m4);
  {
    uint32_t lo = 0, hi = 0;
    if (p.block_before > gseg) {
      const unsigned long long d = p.block_before - gseg;
      lo = d < 64ull ? (uint32_t)d : 64u;
    }
    if (n >= L && n - L + 1 > gseg) {
      const unsigned long long d = n - L + 1 - gseg;
      hi = d < 64ull ? (uint32_t)d : 64u;
    }
    mask &= low_bits(hi) & ~low_bits(lo);
  }
  if (L > 4) mask = verify_tail(mask, tb + sb, ps, L);
  masks[tid] = mask;
  __syncthreads();
  if (tid == 0) {
    unsigned long long K = 0;
    long long last = -1;
    uint32_t x = 0;
    if (t > 0) {
      K = __ldcg(&p.incl[t - 1].kept);
      last = __ldcg(&p.incl[t - 1].last);
      x = __ldcg(&p.incl[t - 1].carry);
    }
    const uint32_t lim = p.query_limit;
    for (uint32_t seg = 0; seg < (uint32_t)kThreads; ++seg) {
      const uint32_t base = seg * 64u;
      if (base >= lim) break;
      uint64_t kept;
      uint32_t xn;
      if (MODE == kModeFree) {
        kept = masks[seg];
        xn = 0;
      } else if (x >= 64u) {
        kept = 0;
        xn = x - 64u;
      } else {
        const Walk w = seg_walk(masks[seg], x, L, p.inv_l, p.stride_mask);
        kept = w.kept;
        xn = w.end > 64u ? w.end - 64u : 0u;
      }
      const uint64_t kb = kept & low_bits(lim - base);
      K += (unsigned long long)__popcll(kb);
      if (kb) last = (long long)(tstart + base + 63u - (uint32_t)__clzll((long long)kb));
      x = xn;
    }
    p.res->q_kept = K;
    p.res->q_last = last;
    if (!s_ok) set_error(p);
  }
}

// ============================================================================ empty pattern
// bytes.replace(b"", rep): rep before every input byte and once at the end.
__global__ void empty_pattern_kernel(const uint8_t* __restrict__ in, unsigned long long n,
                                     const uint8_t* __restrict__ rep, uint32_t R, uint8_t* __restrict__ out) {
  const unsigned long long step = (unsigned long long)R + 1ull;
  const unsigned long long total = n * step + R;
  for (unsigned long long o = (unsigned long long)blockIdx.x * blockDim.x + threadIdx.x; o < total;
       o += (unsigned long long)gridDim.x * blockDim.x) {
    const unsigned long long q = o / step;
    const unsigned long long r = o - q * step;
    out[o] = r < R ? rep[r] : in[q];
  }
}

// ============================================================================ host side
namespace {

bool has_proper_border(const uint8_t* pat, uint32_t L) {
  if (L < 2) return false;
  // Knuth-Morris-Pratt failure function; the longest proper border of pat is fail[L-1].
  uint32_t* fail = new uint32_t[L];
  fail[0] = 0;
  uint32_t k = 0;
  for (uint32_t i = 1; i < L; ++i) {
    while (k > 0 && pat[i] != pat[k]) k = fail[k - 1];
    if (pat[i] == pat[k]) ++k;
    fail[i] = k;
  }
  const bool b = fail[L - 1] > 0;
  delete[] fail;
  return b;
}

template <int MODE>
struct KernelCache {
  std::once_flag once;
  cudaError_t attr_err = cudaSuccess;
};

int device_sm_count() {
  int dev = 0, sms = 0;
  cudaGetDevice(&dev);
  cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev);
  return sms > 0 ? sms : 1;
}

template <int MODE>
cudaError_t launch_mode(const ReplaceParams& p, cudaStream_t st, int* grid_out) {
  static std::mutex mu;
  static int attr_dev_mask = 0;  // bit per device index that has the attribute set
  const uint32_t smem = tile_kernel_smem_bytes(MODE, p.L, p.R);
  int dev = 0;
  cudaGetDevice(&dev);
  {
    std::lock_guard<std::mutex> g(mu);
    if (!(attr_dev_mask & (1 << (dev & 31)))) {
      cudaError_t e = cudaFuncSetAttribute(replace_tiles_kernel<MODE>,
                                           cudaFuncAttributeMaxDynamicSharedMemorySize, 200 * 1024);
      if (e != cudaSuccess) return e;
      e = cudaFuncSetAttribute(query_tile_kernel<MODE>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                               200 * 1024);
      if (e != cudaSuccess) return e;
      attr_dev_mask |= 1 << (dev & 31);
    }
  }
  int per_sm = 0;
  cudaError_t e = cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, replace_tiles_kernel<MODE>, kThreads,
                                                                smem);
  if (e != cudaSuccess) return e;
  if (per_sm < 1) per_sm = 1;
  long long grid = (long long)per_sm * device_sm_count();
  if (grid > (long long)p.num_tiles) grid = p.num_tiles;
  if (grid < 1) grid = 1;
  replace_tiles_kernel<MODE><<<(unsigned)grid, kThreads, smem, st>>>(p);
  if (grid_out) *grid_out = (int)grid;
  return cudaGetLastError();
}

}  // namespace

void prepare_pattern_fields(ReplaceParams& p, const uint8_t* pat, uint32_t L) {
  p.L = L;
  const bool border = has_proper_border(pat, L);
  p.mode = !border ? kModeFree : (L <= 64 ? kModeSmall : kModeLarge);
  uint32_t p4 = 0, m4 = 0;
  for (uint32_t i = 0; i < 4 && i < L; ++i) {
    p4 |= (uint32_t)pat[i] << (8 * i);
    m4 |= 0xFFu << (8 * i);
  }
  p.p4 = p4;
  p.m4 = m4;
  p.inv_l = L > 0 && L < 64 ? (65536u + L - 1) / L : 0u;
  unsigned long long stride = 1ull;
  if (L > 0 && L < 64) {
    stride = 0;
    for (uint32_t b = 0; b < 64; b += L) stride |= 1ull << b;
  }
  p.stride_mask = stride;
  p.agg_entries = p.mode == kModeFree ? 1u : (L < (uint32_t)kTile ? L : (uint32_t)kTile);
}

uint32_t tile_kernel_smem_bytes(uint32_t mode, uint32_t L, uint32_t R) { return make_layout(mode, L, R).total; }

cudaError_t launch_replace(const ReplaceParams& p, cudaStream_t st, int* grid_ctas_out) {
  switch (p.mode) {
    case kModeFree: return launch_mode<kModeFree>(p, st, grid_ctas_out);
    case kModeSmall: return launch_mode<kModeSmall>(p, st, grid_ctas_out);
    default: return launch_mode<kModeLarge>(p, st, grid_ctas_out);
  }
}

cudaError_t launch_query(const ReplaceParams& p, cudaStream_t st) {
  const uint32_t smem = make_layout(kModeFree, p.L, p.R).total;
  // the attribute is set by the first launch_replace of the same mode on this device
  switch (p.mode) {
    case kModeFree: query_tile_kernel<kModeFree><<<1, kThreads, smem, st>>>(p); break;
    case kModeSmall: query_tile_kernel<kModeSmall><<<1, kThreads, smem, st>>>(p); break;
    default: query_tile_kernel<kModeLarge><<<1, kThreads, smem, st>>>(p); break;
  }
  return cudaGetLastError();
}

cudaError_t launch_empty_pattern(const uint8_t* in, unsigned long long n, const uint8_t* rep_dev, uint32_t R,
                                 uint8_t* out, cudaStream_t st) {
  const unsigned long long total = n * ((unsigned long long)R + 1ull) + R;
  unsigned long long blocks = (total + 255ull) / 256ull;
  const unsigned long long cap = (unsigned long long)device_sm_count() * 8ull;
  if (blocks > cap) blocks = cap;
  if (blocks < 1) blocks = 1;
  empty_pattern_kernel<<<(unsigned)blocks, 256, 0, st>>>(in, n, rep_dev, R, out);
  return cudaGetLastError();
}

}  // namespace crb
