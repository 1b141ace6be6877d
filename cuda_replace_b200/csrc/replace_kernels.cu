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
#include <climits>
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
// L2 policies for the super-tile kernel: its input is read twice (pass A from HBM, pass B again
// a super-tile later), so pass A's loads ask L2 to keep the lines (evict_last) and pass B's
// loads and the output stores let them go first (evict_first).
__device__ __forceinline__ uint64_t l2_policy_evict_last() {
  uint64_t p;
  asm("createpolicy.fractional.L2::evict_last.b64 %0, 1.0;" : "=l"(p));
  return p;
}
__device__ __forceinline__ uint64_t l2_policy_evict_first() {
  uint64_t p;
  asm("createpolicy.fractional.L2::evict_first.b64 %0, 1.0;" : "=l"(p));
  return p;
}
__device__ __forceinline__ void bulk_load_hint(void* dst_smem, const void* src_gmem, uint32_t bytes, uint64_t* bar,
                                               uint64_t policy) {
  asm volatile(
      "cp.async.bulk.shared::cluster.global.mbarrier::complete_tx::bytes.L2::cache_hint [%0], [%1], %2, [%3], %4;" ::
          "r"(smem_u32(dst_smem)),
      "l"(src_gmem), "r"(bytes), "r"(smem_u32(bar)), "l"(policy)
      : "memory");
}
// 16-byte output store that L2 may evict first (the output is not read again by this kernel).
__device__ __forceinline__ void st_out16(uint8_t* dst, const uint4& v) {
  asm volatile("st.global.L1::no_allocate.L2::cache_hint.v4.u32 [%0], {%1, %2, %3, %4}, %5;" ::"l"(dst), "r"(v.x),
               "r"(v.y), "r"(v.z), "r"(v.w), "l"(l2_policy_evict_first())
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

// ============================================================================ segmented plan
// One CTA before every segmented launch: draw the launch's epoch (clearing the look-back
// scratch when the 24-bit record tag or the 30-bit status epoch wraps), read every job's
// input length, give each job its range of super-tiles and fill the super-tile -> job map.
// A job whose input is empty gets no super-tile and an empty output; a job whose result
// block holds an error or overflow epoch (an earlier launch of its chain failed) gets no
// super-tile and its lengths stay as they were (the host reads the length that overflowed).
__global__ void __launch_bounds__(1024) seg_plan_kernel(const __grid_constant__ SegLaunch sl) {
  __shared__ uint32_t s_warp[32];
  __shared__ uint32_t s_epoch, s_clear;
  const uint32_t tid = threadIdx.x, lane = tid & 31u, warp = tid >> 5;
  if (tid == 0) {
    uint32_t e = sl.epoch[1] + 1u;
    uint32_t clear = 0;
    if (e >= (1u << 30) - 2u) {
      e = 1;
      clear = 1;
    } else if ((e & 0xFFFFFFu) == 0) {
      e += 1;  // tag 0 is the cleared state
      clear = 1;
    }
    s_epoch = e;
    s_clear = clear;
  }
  __syncthreads();
  if (s_clear) {
    for (unsigned long long i = tid; i < sl.max_tiles; i += blockDim.x) {
      sl.status[i] = 0;
      sl.rec[2 * i] = 0;
      sl.rec[2 * i + 1] = 0;
    }
  }
  const uint32_t nj = *sl.njobs;
  const unsigned long long S = (unsigned long long)sl.nsub * kTile;
  uint32_t run = 0;  // super-tiles of the jobs before this chunk
  for (uint32_t c0 = 0; c0 < nj; c0 += blockDim.x) {
    const uint32_t j = c0 + tid;
    uint32_t nt = 0;
    if (j < nj) {
      SegJob& J = sl.jobs[j];
      const ApplyResult& r = sl.res[J.res];
      const bool failed = r.error_epoch != 0u || r.overflow_epoch != 0u;
      const unsigned long long n = failed ? 0ull : *J.n_dev;
      const unsigned long long t = (n + S - 1ull) / S;
      nt = t < 0xFFFFFFFFull ? (uint32_t)t : 0xFFFFFFFFu;
      if (nt == 0 && !failed) *J.len_out = 0;  // a failed job keeps the length that overflowed
    }
    // block exclusive scan of nt
    uint32_t x = nt;
#pragma unroll
    for (int d = 1; d < 32; d <<= 1) {
      const uint32_t o = __shfl_up_sync(0xffffffffu, x, d);
      if (lane >= (uint32_t)d) x += o;
    }
    if (lane == 31) s_warp[warp] = x;
    __syncthreads();
    if (warp == 0) {
      uint32_t y = lane < (blockDim.x >> 5) ? s_warp[lane] : 0u;
#pragma unroll
      for (int d = 1; d < 32; d <<= 1) {
        const uint32_t o = __shfl_up_sync(0xffffffffu, y, d);
        if (lane >= (uint32_t)d) y += o;
      }
      s_warp[lane] = y;
    }
    __syncthreads();
    const uint32_t excl = (warp ? s_warp[warp - 1] : 0u) + x - nt;
    const uint32_t chunk_total = s_warp[31];
    if (j < nj) {
      SegJob& J = sl.jobs[j];
      const uint32_t base = run + excl;
      J.tile_base = base;
      J.ntiles = nt;
      if ((unsigned long long)base + nt <= sl.max_tiles)
        for (uint32_t i = 0; i < nt; ++i) sl.tile_job[base + i] = j;
    }
    run += chunk_total;
    __syncthreads();
  }
  if (tid == 0) {
    if (run > sl.max_tiles) {
      // more super-tiles than the scratch holds: run nothing, fail every job
      *sl.total = 0;
      for (uint32_t j = 0; j < nj; ++j) sl.res[sl.jobs[j].res].error_epoch = 0xFFFFFFFFu;
    } else {
      *sl.total = run;
    }
    sl.epoch[0] += 1u;
    sl.epoch[1] = s_epoch;
  }
}

// ============================================================================ held tail
// Streaming: copy the last P bytes of buf[0, min(*total, cap)) to dst, where *total is the
// length a previous launch left in device memory. Bytes before position 0 read as zero.
__global__ void move_tail_kernel(const uint8_t* __restrict__ buf, const unsigned long long* __restrict__ total,
                                 unsigned long long cap, uint32_t P, uint8_t* __restrict__ dst) {
  unsigned long long t = *total;
  if (t > cap) t = cap;
  const unsigned long long from = t >= P ? t - P : 0ull;
  for (uint32_t i = threadIdx.x; i < P; i += blockDim.x) dst[i] = (from + i < t) ? buf[from + i] : (uint8_t)0;
}

// ============================================================================ empty pattern
// bytes.replace(b"", rep): rep before every input byte and once at the end.
// One CTA per chunk of 2^shift bytes: the set of byte values present. Each warp keeps its own
// 256-bit set in shared memory and sets a bit only when it is not set yet (text reaches its few
// dozen byte values within the first kilobytes, after which the pass is reads and tests).
__global__ void __launch_bounds__(256) presence_kernel(const uint8_t* __restrict__ in, unsigned long long n,
                                                       uint32_t shift, uint32_t* __restrict__ masks) {
  __shared__ uint32_t wm[8][8];
  const uint32_t warp = threadIdx.x >> 5, lane = threadIdx.x & 31u;
  if (lane < 8) wm[warp][lane] = 0;
  __syncwarp();
  const unsigned long long c0 = (unsigned long long)blockIdx.x << shift;
  const unsigned long long len = min(n - c0, 1ull << shift);
  volatile uint32_t* w = wm[warp];
  const uint4* v = reinterpret_cast<const uint4*>(in + c0);  // chunk starts are 16-byte aligned
  const unsigned long long nv = len >> 4;
  for (unsigned long long i = threadIdx.x; i < nv; i += blockDim.x) {
    const uint4 q = v[i];
    const uint32_t words[4] = {q.x, q.y, q.z, q.w};
#pragma unroll
    for (int k = 0; k < 4; ++k)
#pragma unroll
      for (int j = 0; j < 4; ++j) {
        const uint32_t b = (words[k] >> (8 * j)) & 0xFFu;
        const uint32_t bit = 1u << (b & 31u);
        if (!(w[b >> 5] & bit)) atomicOr(const_cast<uint32_t*>(&w[b >> 5]), bit);
      }
  }
  for (unsigned long long i = (nv << 4) + threadIdx.x; i < len; i += blockDim.x) {
    const uint32_t b = in[c0 + i];
    atomicOr(const_cast<uint32_t*>(&w[b >> 5]), 1u << (b & 31u));
  }
  __syncthreads();
  if (threadIdx.x < 8) {
    uint32_t m = 0;
    for (int k = 0; k < 8; ++k) m |= wm[k][threadIdx.x];
    masks[(unsigned long long)blockIdx.x * 8ull + threadIdx.x] = m;
  }
}

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

// ============================================================================ super-tile kernel
// One look-back per super-tile of nsub 16 KiB sub-tiles. Pass A streams the sub-tiles in
// from HBM, keeps their candidate masks in shared memory and composes the super-tile's
// carry function; after the look-back, pass B streams the same sub-tiles again (they are
// still in L2) and writes the output. Loads run kNBuf ahead through a ring of buffers.
namespace {

constexpr int kNBuf = 2;
constexpr int kMaxSub = 8;


struct LayoutS {
  uint32_t in0, outb, masks, pat, rep, tab16, segtab, srec, wtab, wrec, subrec, total;  // buffer b at in0 + b * inbytes
  uint32_t masks_set, srec_set, wtab_set, wrec_set, subrec_set;  // bytes of one set of per-super-tile tables
  uint32_t mtab;                    // kModeMulti: the stage's pair table
  uint32_t rs, inbytes;
  uint32_t wstage_words;  // padded staging words per warp (its 2 KiB of input may grow 3x)
  uint32_t wstage_cap;    // bytes one warp can stage (before the padding words)
};

// Output bytes one 16 KiB sub-tile can produce, capped at three times its input.
__host__ __device__ __forceinline__ uint32_t stage_ratio(uint32_t L, uint32_t R) {
  if (L == 0 || R <= L) return 1;
  const uint32_t r = (R + L - 1) / L;
  return r < 3 ? r : 3;
}

// ratio: output staging per input byte (0: from L and R; a segmented launch passes the largest).
// sets: per-super-tile tables held at once (2 when one super-tile's pass A overlaps the
// previous one's look-back and pass B).
__host__ __device__ __forceinline__ LayoutS make_layout_s(uint32_t mode, uint32_t L, uint32_t R, uint32_t nsub,
                                                          uint32_t ratio = 0, uint32_t sets = 1) {
  LayoutS s{};
  uint32_t off = 0;
  s.inbytes = align_up_u32(kTile + (L > 1 ? L - 1 : 0), 16) + 32;
  s.in0 = off;
  off += kNBuf * s.inbytes;
  {
    const uint32_t words = (2048u * (ratio ? ratio : stage_ratio(L, R)) + 48u) / 4u;
    s.wstage_words = words + words / 32u + 2u;
    s.wstage_cap = words * 4u;
  }
  s.outb = off;
  off += align_up_u32(kWarps * s.wstage_words * 4u, 16);
  s.masks = off;
  s.masks_set = nsub * kThreads * 8;
  off += sets * s.masks_set;
  s.pat = off;
  off += align_up_u32(L ? L : 1, 16);
  s.rep = off;
  off += align_up_u32(R + 16, 16);
  s.tab16 = off;  // replacement repeated, 16 bytes from every phase (R <= 64)
  off += (R >= 1 && R <= 64) ? R * 16 : 0;
  if (mode == kModeSmall) {
    s.rs = L | 1u;
    if (L > 4) {
      s.segtab = off;
      off += align_up_u32(kThreads * s.rs * 2, 16);
    }
    s.srec = off;
    s.srec_set = align_up_u32(nsub * kThreads * L, 16);
    off += sets * s.srec_set;
    s.wtab = off;
    s.wtab_set = align_up_u32(nsub * kWarps * L * 4, 16);
    off += sets * s.wtab_set;
    s.wrec = off;
    s.wrec_set = align_up_u32(nsub * kWarps * L, 16);
    off += sets * s.wrec_set;
    s.subrec = off;
    s.subrec_set = align_up_u32(nsub * L, 16);
    off += sets * s.subrec_set;
  }
  if (mode == kModeMulti) {
    s.mtab = off;
    off += align_up_u32((uint32_t)sizeof(MultiTable), 16);
  }
  s.total = off;
  return s;
}

// Segment function as 16-bit entries (kept count in the low byte, carry-out in the high
// byte) over carries [0, L), L <= 32.
__device__ __forceinline__ void build_seg_table16(uint64_t mask, uint32_t L, uint32_t inv_l, uint64_t stride,
                                                  uint16_t* row) {
  uint32_t c = 0;
  while (c < L) {
    const uint64_t m = mask >> c;
    if (m == 0) {
      for (; c < L; ++c) row[c] = 0;
      break;
    }
    const uint32_t e = c + (uint32_t)(__ffsll((long long)m) - 1);
    const Walk w = seg_walk(mask, e, L, inv_l, stride);
    const uint32_t carry = w.end > 64 ? w.end - 64 : 0;
    const uint16_t v = (uint16_t)(w.cnt | (carry << 8));
    const uint32_t hi = min(e + 1, L);
    for (; c < hi; ++c) row[c] = v;
  }
}

// The 17 words (68 bytes) starting at this thread's 64-byte segment; the 17th word is the
// next lane's first word (read from shared memory only by the last lane of each warp), so
// no load has lanes 64 bytes apart on the same bank.
__device__ __forceinline__ void load_seg_words(const uint8_t* s, uint32_t w[17]) {
  const uint4* v = reinterpret_cast<const uint4*>(s);
#pragma unroll
  for (int i = 0; i < 4; ++i) {
    const uint4 q = v[i];
    w[4 * i + 0] = q.x;
    w[4 * i + 1] = q.y;
    w[4 * i + 2] = q.z;
    w[4 * i + 3] = q.w;
  }
  const uint32_t nxt = __shfl_down_sync(0xffffffffu, w[0], 1);
  w[16] = ((threadIdx.x & 31u) == 31u) ? *reinterpret_cast<const uint32_t*>(s + 64) : nxt;
}

__device__ __forceinline__ uint64_t candidates_from_words(const uint32_t w[17], uint32_t p4, uint32_t m4) {
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

// 4 bytes at an arbitrary shared-memory byte address (two aligned loads and a funnel shift).
__device__ __forceinline__ uint32_t ld_u32_unaligned(const uint8_t* p) {
  const uintptr_t a = reinterpret_cast<uintptr_t>(p);
  const uint32_t* q = reinterpret_cast<const uint32_t*>(a & ~uintptr_t(3));
  const uint32_t sh = (uint32_t)(a & 3u) * 8u;
  return sh ? __funnelshift_r(q[0], q[1], sh) : q[0];
}

// 4-bit mask of the bytes of w equal to the byte replicated in rep (bit i: byte i). Exact per
// byte: (x & 0x7f) + 0x7f sets bit 7 of a byte iff its low 7 bits are nonzero, with no carry
// into the next byte; the multiply gathers the four bit-7 flags into bits 28-31.
__device__ __forceinline__ uint32_t eq_nibble(uint32_t w, uint32_t rep) {
  const uint32_t x = w ^ rep;
  const uint32_t nz = ((x & 0x7F7F7F7Fu) + 0x7F7F7F7Fu) | x;
  return ((~nz & 0x80808080u) * 0x00204081u) >> 28;
}

// Candidate starts of the 64-byte segment at seg (shared memory), comparing the first min(L, 4)
// pattern bytes (as candidates_from_words) with fewer instructions: the positions holding the
// first pattern byte come from four bytes per operation; L = 1 needs nothing more and a
// doubled first byte (L = 2, e.g. "aa") a shift; otherwise each such position is checked with
// one unaligned 4-byte read, unless a lane of the warp has many of them (dense text), where
// every window is compared. The segment is read without bank conflicts: lanes 64 bytes apart
// would hit the same banks four at a time, so each pair of lanes starts at another of its four
// 16-byte chunks; the first-byte mask is built in that rotated order and rotated back (a 64-bit
// rotate). Only the rare dense branch reads the segment in order.
// try_run (the pattern's first min(L, 4) bytes all equal its first byte b0): first test, one OR
// per word, whether the warp's whole 2 KiB region is the byte b0 repeated (*uniform). Then
// every window starting in the region matches those bytes, except the last lane's final
// min(L, 4) - 1 positions, which also need the bytes after the region.
__device__ __forceinline__ uint64_t candidates_seg(const uint8_t* seg, uint32_t p4, uint32_t m4, uint32_t L,
                                                   bool try_run, bool* uniform) {
  const uint32_t lane = threadIdx.x & 31u;
  const uint32_t rot = (lane >> 1) & 3u;
  const uint4* v = reinterpret_cast<const uint4*>(seg);
  const uint4 q0 = v[rot], q1 = v[(rot + 1u) & 3u], q2 = v[(rot + 2u) & 3u], q3 = v[(rot + 3u) & 3u];
  const uint32_t b0 = p4 & 0xFFu, rep = b0 * 0x01010101u;
  *uniform = false;
  if (try_run) {
    const uint32_t d = ((q0.x ^ rep) | (q0.y ^ rep) | (q0.z ^ rep) | (q0.w ^ rep)) |
                       ((q1.x ^ rep) | (q1.y ^ rep) | (q1.z ^ rep) | (q1.w ^ rep)) |
                       ((q2.x ^ rep) | (q2.y ^ rep) | (q2.z ^ rep) | (q2.w ^ rep)) |
                       ((q3.x ^ rep) | (q3.y ^ rep) | (q3.z ^ rep) | (q3.w ^ rep));
    if (__all_sync(0xffffffffu, d == 0u)) {
      *uniform = true;
      uint64_t mask = ~0ull;
      const uint32_t lp = L < 4u ? L : 4u;
      if (lane == 31u && lp > 1u) {
        // leading bytes b0 of the 4 bytes after the region (the next region's, or the halo)
        const uint32_t z = (uint32_t)__ffs(~eq_nibble(*reinterpret_cast<const uint32_t*>(seg + 64), rep) & 0x1Fu) - 1u;
        for (uint32_t k = 1; k < lp; ++k)  // position 64 - k needs lp - k following bytes
          if (lp - k > z) mask &= ~(1ull << (64u - k));
      }
      return mask;
    }
  }
  if (L >= 3u || (L == 2u && ((p4 >> 8) & 0xFFu) != b0)) {
    // Positions of the first byte, kept in a transposed order that costs fewer operations:
    // bit 8j + i of t0 (t1) is byte j of rotated word i (i + 8). ~((((w ^ rep) & 0x7f..) +
    // 0x7f..) | (w ^ rep)) has bit 7 of a byte set exactly when the byte equals b0; a shift
    // moves those bits to 8j + i and a masked OR adds them.
    uint32_t t0 = 0, t1 = 0;
#define CRB_FIRST_BYTE(word, acc, i)                                                 \
    {                                                                                \
      const uint32_t x_ = (word) ^ rep;                                              \
      const uint32_t f_ = ~(((x_ & 0x7F7F7F7Fu) + 0x7F7F7F7Fu) | x_);                \
      acc |= (f_ >> (7u - (i))) & (0x01010101u << (i));                              \
    }
    CRB_FIRST_BYTE(q0.x, t0, 0u) CRB_FIRST_BYTE(q0.y, t0, 1u) CRB_FIRST_BYTE(q0.z, t0, 2u) CRB_FIRST_BYTE(q0.w, t0, 3u)
    CRB_FIRST_BYTE(q1.x, t0, 4u) CRB_FIRST_BYTE(q1.y, t0, 5u) CRB_FIRST_BYTE(q1.z, t0, 6u) CRB_FIRST_BYTE(q1.w, t0, 7u)
    CRB_FIRST_BYTE(q2.x, t1, 0u) CRB_FIRST_BYTE(q2.y, t1, 1u) CRB_FIRST_BYTE(q2.z, t1, 2u) CRB_FIRST_BYTE(q2.w, t1, 3u)
    CRB_FIRST_BYTE(q3.x, t1, 4u) CRB_FIRST_BYTE(q3.y, t1, 5u) CRB_FIRST_BYTE(q3.z, t1, 6u) CRB_FIRST_BYTE(q3.w, t1, 7u)
#undef CRB_FIRST_BYTE
    if (__any_sync(0xffffffffu, __popc(t0) + __popc(t1) > 12)) {
      uint32_t w[17];
      load_seg_words(seg, w);
      return candidates_from_words(w, p4, m4);
    }
    uint64_t out = 0;
    // one loop over both halves (t0's positions, then t1's): a warp iterates as often as its
    // busiest lane has positions in all
    while (t0 | t1) {
      const uint32_t h = t0 ? 0u : 1u;
      const uint32_t m = h ? t1 : t0;
      const uint32_t b = (uint32_t)(__ffs(m) - 1);
      if (h) t1 = m & (m - 1u); else t0 = m & (m - 1u);
      const uint32_t i = (b & 7u) + 8u * h;                              // rotated word
      const uint32_t nat = (((rot + (i >> 2)) & 3u) << 2) | (i & 3u);  // natural word
      const uint32_t pos = 4u * nat + (b >> 3);
      if (((ld_u32_unaligned(seg + pos) ^ p4) & m4) == 0u) out |= 1ull << pos;
    }
    return out;
  }
  const uint32_t lo = eq_nibble(q0.x, rep) | (eq_nibble(q0.y, rep) << 4) | (eq_nibble(q0.z, rep) << 8) |
                      (eq_nibble(q0.w, rep) << 12) | (eq_nibble(q1.x, rep) << 16) | (eq_nibble(q1.y, rep) << 20) |
                      (eq_nibble(q1.z, rep) << 24) | (eq_nibble(q1.w, rep) << 28);
  const uint32_t hi = eq_nibble(q2.x, rep) | (eq_nibble(q2.y, rep) << 4) | (eq_nibble(q2.z, rep) << 8) |
                      (eq_nibble(q2.w, rep) << 12) | (eq_nibble(q3.x, rep) << 16) | (eq_nibble(q3.y, rep) << 20) |
                      (eq_nibble(q3.z, rep) << 24) | (eq_nibble(q3.w, rep) << 28);
  const uint64_t er = ((uint64_t)hi << 32) | lo;  // chunk (rot + k) & 3 at bits 16k
  const uint32_t sh = 16u * rot;
  const uint64_t e0 = sh ? ((er << sh) | (er >> (64u - sh))) : er;
  if (L == 1u) return e0;
  if (L == 2u && ((p4 >> 8) & 0xFFu) == b0) {
    // byte 64: the next lane's first word (chunk 0 of the next segment), from shared memory
    // for the last lane
    const uint32_t nat0 = rot == 0u ? q0.x : (rot == 1u ? q3.x : (rot == 2u ? q2.x : q1.x));
    uint32_t w64 = __shfl_down_sync(0xffffffffu, nat0, 1);
    if (lane == 31u) w64 = *reinterpret_cast<const uint32_t*>(seg + 64);
    const uint64_t next = (w64 & 0xFFu) == b0 ? 1ull : 0ull;
    return e0 & ((e0 >> 1) | (next << 63));
  }
  if (__any_sync(0xffffffffu, __popcll(e0) > 12)) {
    uint32_t w[17];
    load_seg_words(seg, w);
    return candidates_from_words(w, p4, m4);
  }
  uint64_t m = e0, out = 0;
  while (m) {
    const int b = __ffsll((long long)m) - 1;
    m &= m - 1;
    if (((ld_u32_unaligned(seg + b) ^ p4) & m4) == 0u) out |= 1ull << b;
  }
  return out;
}

// ---- kModeMulti helpers
// Positions of the 64-byte segment at seg holding one of the stage's nfirst (1..4) distinct
// first pattern bytes (`firsts`, one per byte lane): the four-bytes-per-operation byte test of
// candidates_seg once per distinct byte, with the same conflict-free rotated reads.
__device__ __forceinline__ uint64_t multi_first_mask(const uint8_t* seg, uint32_t firsts, uint32_t nfirst) {
  const uint32_t lane = threadIdx.x & 31u;
  const uint32_t rot = (lane >> 1) & 3u;
  const uint4* v = reinterpret_cast<const uint4*>(seg);
  const uint4 q0 = v[rot], q1 = v[(rot + 1u) & 3u], q2 = v[(rot + 2u) & 3u], q3 = v[(rot + 3u) & 3u];
  uint64_t er = 0;
  for (uint32_t k = 0; k < nfirst; ++k) {
    const uint32_t rep = ((firsts >> (8u * k)) & 0xFFu) * 0x01010101u;
    const uint32_t lo = eq_nibble(q0.x, rep) | (eq_nibble(q0.y, rep) << 4) | (eq_nibble(q0.z, rep) << 8) |
                        (eq_nibble(q0.w, rep) << 12) | (eq_nibble(q1.x, rep) << 16) | (eq_nibble(q1.y, rep) << 20) |
                        (eq_nibble(q1.z, rep) << 24) | (eq_nibble(q1.w, rep) << 28);
    const uint32_t hi = eq_nibble(q2.x, rep) | (eq_nibble(q2.y, rep) << 4) | (eq_nibble(q2.z, rep) << 8) |
                        (eq_nibble(q2.w, rep) << 12) | (eq_nibble(q3.x, rep) << 16) | (eq_nibble(q3.y, rep) << 20) |
                        (eq_nibble(q3.z, rep) << 24) | (eq_nibble(q3.w, rep) << 28);
    er |= ((uint64_t)hi << 32) | lo;  // chunk (rot + k) & 3 at bits 16k
  }
  const uint32_t sh = 16u * rot;
  return sh ? ((er << sh) | (er >> (64u - sh))) : er;
}

// The pair of the stage whose pattern occurs at s (shared memory), or -1. room = input bytes
// from s to the end of the buffer (a pattern must fit in them). No two patterns of a stage can
// occur at one position (none is a prefix of another), so the first pair that matches is the
// only one. One-byte patterns are found by their byte; longer ones through a hash of their
// first two bytes, then compared.
__device__ __forceinline__ int multi_identify(const MultiTable& T, const uint8_t* s, unsigned long long room) {
  const uint32_t b0 = s[0];
  uint32_t id = T.one[b0];
  if (id) return (int)id - 1;
  if (room < 2ull) return -1;
  const uint32_t w = ld_u32_unaligned(s);
  id = T.head[multi_hash(b0, (w >> 8) & 0xFFu)];
  while (id) {
    const uint32_t k = id - 1u;
    const uint32_t L = T.L[k];
    if ((unsigned long long)L <= room && ((w ^ T.p4[k]) & T.m4[k]) == 0u) {
      bool ok = true;
      for (uint32_t i = 4; i < L; ++i)
        if (s[i] != T.pat[k][i]) {
          ok = false;
          break;
        }
      if (ok) return (int)k;
    }
    id = T.next[k];
  }
  return -1;
}

// Output staging: a word buffer with one padding word after every 32, so threads that
// write their (contiguous) outputs word by word land on different banks.
__device__ __forceinline__ uint32_t stg_pad(uint32_t w) { return w + (w >> 5); }


// Streams one thread's output bytes into the staging buffer: whole words are stored as
// words; the partial first and last words (shared with the neighbouring threads) byte by
// byte. `pend` holds the nb (0..3) bytes of the current word not yet stored; appending four
// bytes leaves nb unchanged, so the word loop has no branches.
struct Emitter {
  uint32_t* stg;
  uint32_t pend;  // pending bytes (low nb bytes; the first `skip` belong to the previous thread)
  uint32_t nb;
  uint32_t wpos;  // staging word that pend will complete
  uint32_t skip;  // nonzero until the first (partial) word has been stored

  __device__ __forceinline__ void init(uint32_t* s, uint32_t start_byte) {
    stg = s;
    pend = 0;
    nb = start_byte & 3u;
    wpos = start_byte >> 2;
    skip = nb;
  }
  __device__ __forceinline__ void store_bytes(uint32_t word, uint32_t from, uint32_t to) {
    uint8_t* b = reinterpret_cast<uint8_t*>(stg + stg_pad(wpos));
    for (uint32_t i = from; i < to; ++i) b[i] = (uint8_t)(word >> (8 * i));
  }
  __device__ __forceinline__ void put_word(uint32_t word) {
    if (skip) {
      store_bytes(word, skip, 4);
      skip = 0;
    } else {
      stg[stg_pad(wpos)] = word;
    }
    ++wpos;
  }
  __device__ __forceinline__ void append4(uint32_t v) {
    const uint32_t s = 8u * nb;
    put_word(pend | (v << s));
    pend = __funnelshift_rc(v, 0u, 32u - s);
  }
  __device__ __forceinline__ void append1(uint32_t b) {
    pend |= (b & 0xFFu) << (8u * nb);
    if (++nb == 4u) {
      put_word(pend);
      pend = 0;
      nb = 0;
    }
  }
  __device__ __forceinline__ void finish() {
    if (nb > skip) store_bytes(pend, skip, nb);
  }
};

// Literal bytes src[0, len) from shared memory.
__device__ __forceinline__ void emit_literal(Emitter& e, const uint8_t* src, uint32_t len) {
  uint32_t i = 0;
  for (; i + 4 <= len; i += 4) e.append4(ld_u32_unaligned(src + i));
  for (; i < len; ++i) e.append1(src[i]);
}

// r copies of the replacement: rrep holds the replacement repeated (at least R + 8 bytes);
// step4 = 4 mod R. When R divides 4 every word of the run is the same.
__device__ __forceinline__ void emit_repeat(Emitter& e, const uint8_t* rrep, uint32_t R, uint32_t step4,
                                            uint32_t r) {
  uint32_t total = r * R;
  if (step4 == 0u) {
    const uint32_t w = *reinterpret_cast<const uint32_t*>(rrep);
    for (; total >= 4; total -= 4) e.append4(w);
  } else {
    uint32_t ph = 0;
    for (; total >= 4; total -= 4) {
      e.append4(ld_u32_unaligned(rrep + ph));
      ph += step4;
      if (ph >= R) ph -= R;
    }
    for (; total; --total) {
      e.append1(rrep[ph]);
      if (++ph == R) ph = 0;
    }
    return;
  }
  for (uint32_t ph = 0; total; --total) {
    e.append1(rrep[ph]);
    if (++ph == R) ph = 0;
  }
}

// ---- short bordered patterns (L <= 4): segment functions packed in registers.
// Entry c (carry-in c) is 16 bits: kept count in bits 0-13, carry-out in bits 14-15; entries
// 0,1 live in t0 and 2,3 in t1. Composition is a few selects, so a warp composes its 32
// segment functions with a Kogge-Stone scan of shuffles instead of a 32-step walk.
__device__ __forceinline__ uint32_t ks_get(uint32_t t0, uint32_t t1, uint32_t c) {
  const uint32_t w = (c & 2u) ? t1 : t0;
  return (c & 1u) ? (w >> 16) : (w & 0xFFFFu);
}

// Block-wide exclusive scan with ONE barrier: buf alternates between two scratch arrays so
// the next scan cannot overwrite totals still being read.
template <typename Op>
__device__ __forceinline__ uint32_t block_excl_scan1(uint32_t v, uint32_t identity, Op op, uint32_t* buf,
                                                     uint32_t* total) {
  const uint32_t lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
  const uint32_t inc = warp_incl_scan(v, op);
  if (lane == 31) buf[warp] = inc;
  __syncthreads();
  uint32_t wpre = identity, tot = identity;
#pragma unroll
  for (int w = 0; w < kWarps; ++w) {
    const uint32_t s = buf[w];
    if ((uint32_t)w < warp) wpre = op(wpre, s);
    tot = op(tot, s);
  }
  uint32_t ex = __shfl_up_sync(0xffffffffu, inc, 1);
  if (lane == 0) ex = identity;
  *total = tot;
  return op(wpre, ex);
}

// Warp-level bounded wait over the window of predecessors j = base - lane (j < 0 is the
// virtual tile before tile 0, treated as inclusive with K = 0, carry = 0). Returns the lane
// of the nearest inclusive tile (32 if none) once every nearer lane has at least its
// aggregate, or -1 when the wait gave up. *st receives this lane's state.
__device__ __forceinline__ int warp_wait_window(const ReplaceParams& p, long long base, uint32_t* st) {
  const uint32_t lane = threadIdx.x & 31u;
  const long long j = base - (long long)lane;
  const uint32_t want = p.epoch << 2;
  unsigned long long t0 = 0;
  uint32_t ns = 32;
  for (;;) {
    uint32_t s = 0;
    if (j < 0) {
      s = kStInc;
    } else {
      const uint32_t v = ld_acquire_u32(p.status + j);
      if ((v & ~3u) == want) s = v & 3u;
    }
    const uint32_t ready = __ballot_sync(0xffffffffu, s != 0);
    const uint32_t incm = __ballot_sync(0xffffffffu, s == kStInc);
    const uint32_t pl = incm ? (uint32_t)(__ffs(incm) - 1) : 32u;
    const uint32_t need = pl == 32u ? 0xffffffffu : ((1u << pl) - 1u);
    if ((ready & need) == need) {
      *st = s;
      return (int)pl;
    }
    if (aborted(p)) return -1;
    const unsigned long long now = global_ns();
    if (t0 == 0) {
      t0 = now;
    } else if (now - t0 > kSpinLimitNs) {
      if (lane == 0) set_error(p);
      return -1;
    }
    __nanosleep(ns);
    if (ns < 256) ns <<= 1;
  }
}

// ---- one-round-trip look-back records (kModeFree, and kModeSmall with L <= 4).
// Tile t's record is 16 bytes, rec[2t] and rec[2t+1]; each word carries the launch tag
// (low 24 bits of the epoch, bits 40-63) and the state (bits 38-39) next to 38 payload
// bits, so a reader validates a record with one 16-byte load: both tags current and both
// states equal (a torn read of an AGG -> INC update fails that test and is retried).
// AGG payload: free mode (count, cover); small mode the 4-entry table (19 bits per entry:
// count 17 bits, carry-out 2 bits). INC payload: (kept prefix, carry-out).
__device__ __forceinline__ unsigned long long rec_word(uint32_t tag, uint32_t state, unsigned long long d) {
  return ((unsigned long long)tag << 40) | ((unsigned long long)state << 38) | (d & ((1ull << 38) - 1ull));
}
__device__ __forceinline__ void rec_store(unsigned long long* rec, uint32_t t, unsigned long long w0,
                                          unsigned long long w1) {
  asm volatile("st.volatile.global.v2.u64 [%0], {%1, %2};" ::"l"(rec + 2ull * t), "l"(w0), "l"(w1) : "memory");
}
__device__ __forceinline__ void rec_load(const unsigned long long* rec, uint32_t t, unsigned long long* w0,
                                         unsigned long long* w1) {
  asm volatile("ld.volatile.global.v2.u64 {%0, %1}, [%2];" : "=l"(*w0), "=l"(*w1) : "l"(rec + 2ull * t) : "memory");
}
__device__ __forceinline__ unsigned long long rec_data(unsigned long long w) { return w & ((1ull << 38) - 1ull); }

// Window of predecessors j = base - lane read from the records (j < 0: virtual inclusive
// tile with zero payload). Returns the nearest inclusive lane (32 if none) once every
// nearer lane holds a valid record, or -1 when the wait gave up; d0/d1 receive the payload.
__device__ __forceinline__ int warp_read_window(const ReplaceParams& p, long long base, unsigned long long* d0,
                                                unsigned long long* d1, uint32_t carry0) {
  const uint32_t lane = threadIdx.x & 31u;
  const long long j = base - (long long)lane;
  const uint32_t tag = p.epoch & 0xFFFFFFu;
  unsigned long long t0 = 0;
  uint32_t ns = 32;
  for (;;) {
    uint32_t st = 0;
    unsigned long long w0 = 0, w1 = 0;
    if (j < 0) {
      st = kStInc;
      w1 = carry0;  // the virtual tile before tile 0 leaves carry0 bytes covered
    } else {
      rec_load(p.rec, (uint32_t)j, &w0, &w1);
      const uint32_t s0 = (uint32_t)(w0 >> 38) & 3u, s1 = (uint32_t)(w1 >> 38) & 3u;
      if ((uint32_t)(w0 >> 40) == tag && (uint32_t)(w1 >> 40) == tag && s0 == s1) st = s0;
    }
    const uint32_t ready = __ballot_sync(0xffffffffu, st != 0);
    const uint32_t incm = __ballot_sync(0xffffffffu, st == kStInc);
    const uint32_t pl = incm ? (uint32_t)(__ffs(incm) - 1) : 32u;
    const uint32_t need = pl == 32u ? 0xffffffffu : ((1u << pl) - 1u);
    if ((ready & need) == need) {
      *d0 = rec_data(w0);
      *d1 = rec_data(w1);
      return (int)pl;
    }
    if (aborted(p)) return -1;
    const unsigned long long now = global_ns();
    if (t0 == 0) {
      t0 = now;
    } else if (now - t0 > kSpinLimitNs) {
      if (lane == 0) set_error(p);
      return -1;
    }
    __nanosleep(ns);
    if (ns < 256) ns <<= 1;
  }
}

__device__ __forceinline__ bool lookback_free_rec(const ReplaceParams& p, uint32_t t, unsigned long long S,
                                                  unsigned long long* K_out, uint32_t* c_out, uint32_t carry0) {
  const uint32_t lane = threadIdx.x & 31u;
  unsigned long long acc_cnt = 0;
  long long acc_cover = 0;
  unsigned long long acc_span = 0;
  long long base = (long long)t - 1;
  for (;;) {
    unsigned long long d0, d1;
    const int plr = warp_read_window(p, base, &d0, &d1, carry0);
    if (plr < 0) return false;
    const uint32_t pl = (uint32_t)plr;
    unsigned long long cnt = 0;
    long long val = LLONG_MIN / 4;
    if (lane <= pl && lane < 32u) {
      cnt = d0;
      val = (long long)d1 - (long long)(lane * S);
    }
#pragma unroll
    for (int d = 16; d >= 1; d >>= 1) {
      cnt += __shfl_xor_sync(0xffffffffu, cnt, d);
      const long long o = __shfl_xor_sync(0xffffffffu, val, d);
      val = o > val ? o : val;
    }
    if (pl < 32) {
      const long long c1 = val - (long long)acc_span;
      const long long c = c1 > acc_cover ? c1 : acc_cover;
      *K_out = cnt + acc_cnt;
      *c_out = c > 0 ? (uint32_t)c : 0u;
      return true;
    }
    const long long cov = val - (long long)acc_span;
    acc_cover = cov > acc_cover ? cov : acc_cover;
    acc_cnt += cnt;
    acc_span += 32ull * S;
    base -= 32;
  }
}

// entry c of a packed 4-entry table (two 38-bit payloads)
__device__ __forceinline__ uint32_t tab4_entry(unsigned long long d0, unsigned long long d1, uint32_t c) {
  const unsigned long long w = (c & 2u) ? d1 : d0;
  return (uint32_t)((c & 1u) ? (w >> 19) : w) & 0x7FFFFu;
}

// A warp region whose 2 KiB are all candidates (a run such as "aaaa" for "aa", L <= 4): from
// carry-in c the greedy keeps c, c + L, c + 2L, ..., so its tables have closed forms, and pass
// A records only that the region is dense. Region entry (kept count | carry-out << 16):
__device__ __forceinline__ uint32_t dense_region_entry(uint32_t c, uint32_t L) {
  const uint32_t cnt = (2048u - c + L - 1u) / L;
  return cnt | ((c + cnt * L - 2048u) << 16);
}
// ... and the carry into the segment at byte `off` of the region:
__device__ __forceinline__ uint32_t dense_seg_carry(uint32_t c, uint32_t off, uint32_t L) {
  const uint32_t q = off > c ? (off - c + L - 1u) / L : 0u;  // kept starts before the segment
  return c + q * L - off;
}

// Functions over carries 0..LL-1 (patterns of LL <= 4 bytes) with wide counts, one register
// per entry: kept count in bits 0-23, carry-out in bits 24-31.
template <int LL>
__device__ __forceinline__ uint32_t fn_at(const uint32_t g[4], uint32_t k) {
  if (LL == 2) return k == 0u ? g[0] : g[1];
  if (LL == 3) return k == 0u ? g[0] : (k == 1u ? g[1] : g[2]);
  return k == 0u ? g[0] : (k == 1u ? g[1] : (k == 2u ? g[2] : g[3]));
}
// g := g applied after o (o covers the earlier bytes)
template <int LL>
__device__ __forceinline__ void fn_after(uint32_t g[4], const uint32_t o[4]) {
  uint32_t r[4];
#pragma unroll
  for (int y = 0; y < LL; ++y) {
    const uint32_t m = fn_at<LL>(g, o[y] >> 24);
    r[y] = ((o[y] & 0xFFFFFFu) + (m & 0xFFFFFFu)) | (m & 0xFF000000u);
  }
#pragma unroll
  for (int y = 0; y < LL; ++y) g[y] = r[y];
}
// One step of an inclusive scan of functions over lanes, earlier bytes in lower lanes: within
// groups of `width` lanes (pos: the lane's place in its group) or across groups (width 32).
template <int LL>
__device__ __forceinline__ void fn_scan_up(uint32_t g[4], uint32_t step, uint32_t width, uint32_t pos) {
  uint32_t o[4];
#pragma unroll
  for (int y = 0; y < LL; ++y) o[y] = __shfl_up_sync(0xffffffffu, g[y], step, width);
  if (pos >= step) fn_after<LL>(g, o);
}
// The same with earlier bytes in higher lanes.
template <int LL>
__device__ __forceinline__ void fn_scan_down(uint32_t g[4], uint32_t step) {
  uint32_t o[4];
#pragma unroll
  for (int y = 0; y < LL; ++y) o[y] = __shfl_down_sync(0xffffffffu, g[y], step);
  if ((threadIdx.x & 31u) + step < 32u) fn_after<LL>(g, o);
}


// Window of 64 predecessors, two per lane: lane l reads super-tiles base - 2l and base - 2l - 1
// (distances 2l and 2l + 1; distance < 0: the virtual inclusive tile before tile 0). Returns the
// distance of the nearest inclusive record (64 if none) once every nearer record is valid, or
// -1 when the wait gave up; d0/d1 receive the payloads. Both loads of a lane are in flight
// together, so a window costs one round trip.
__device__ __forceinline__ int warp_read_window2(const ReplaceParams& p, long long base, unsigned long long d0[2],
                                                 unsigned long long d1[2], uint32_t carry0) {
  const uint32_t lane = threadIdx.x & 31u;
  const uint32_t tag = p.epoch & 0xFFFFFFu;
  unsigned long long t0 = 0;
  uint32_t ns = 32;
  for (;;) {
    uint32_t st[2];
#pragma unroll
    for (int r = 0; r < 2; ++r) {
      const long long j = base - 2 * (long long)lane - r;
      st[r] = 0;
      d0[r] = 0;
      d1[r] = 0;
      if (j < 0) {
        st[r] = kStInc;
        d1[r] = carry0;  // the virtual tile before tile 0 leaves carry0 bytes covered
      } else {
        rec_load(p.rec, (uint32_t)j, &d0[r], &d1[r]);
      }
    }
#pragma unroll
    for (int r = 0; r < 2; ++r) {
      if (base - 2 * (long long)lane - r >= 0) {
        const unsigned long long w0 = d0[r], w1 = d1[r];
        const uint32_t s0 = (uint32_t)(w0 >> 38) & 3u, s1 = (uint32_t)(w1 >> 38) & 3u;
        st[r] = ((uint32_t)(w0 >> 40) == tag && (uint32_t)(w1 >> 40) == tag && s0 == s1) ? s0 : 0u;
        d0[r] = rec_data(w0);
        d1[r] = rec_data(w1);
      }
    }
    // this lane's nearest inclusive record (2: none) and whether every nearer one is valid
    const uint32_t fi = st[0] == kStInc ? 0u : (st[1] == kStInc ? 1u : 2u);
    const bool pre = (fi < 1u || st[0] != 0u) && (fi < 2u || st[1] != 0u);
    const uint32_t incm = __ballot_sync(0xffffffffu, fi < 2u);
    const uint32_t okm = __ballot_sync(0xffffffffu, pre);
    const uint32_t pl = incm ? (uint32_t)(__ffs(incm) - 1) : 32u;
    const uint32_t need = pl >= 31u ? 0xffffffffu : ((2u << pl) - 1u);  // lanes 0..pl
    if ((okm & need) == need) {
      const uint32_t fpl = __shfl_sync(0xffffffffu, fi, pl & 31u);
      return pl == 32u ? 64 : (int)(2u * pl + fpl);
    }
    if (aborted(p)) return -1;
    const unsigned long long now = global_ns();
    if (t0 == 0) {
      t0 = now;
    } else if (now - t0 > kSpinLimitNs) {
      if (lane == 0) set_error(p);
      return -1;
    }
    __nanosleep(ns);
    if (ns < 256) ns <<= 1;
  }
}

// Look-back for patterns of LL <= 4 bytes over the 16-byte records, in windows of 64
// predecessors (warp_read_window2): each lane first composes its two super-tiles' functions
// (the older applied first), then a scan over lanes (lane l: super-tiles t - 1 - 2l and
// t - 2 - 2l, the identity at and beyond the nearest inclusive one) composes the window, so a
// window costs a few shuffle steps whatever its length. Counts stay within 24 bits: 64
// super-tiles of at most 2^15 kept starts.
template <int LL>
__device__ __forceinline__ bool lookback_small_rec(const ReplaceParams& p, uint32_t t, unsigned long long* K_out,
                                                    uint32_t* c_out, uint32_t carry0) {
  const uint32_t lane = threadIdx.x & 31u;
  unsigned long long acc_cnt = 0;  // lane c < LL: function of the super-tiles between the window and t
  uint32_t acc_carry = lane;
  long long base = (long long)t - 1;
  for (;;) {
    unsigned long long d0[2], d1[2];
    const int D = warp_read_window2(p, base, d0, d1, carry0);
    if (D < 0) return false;
    uint32_t g[4], f[4];
#pragma unroll
    for (uint32_t y = 0; y < (uint32_t)LL; ++y) {
      g[y] = y << 24;
      f[y] = y << 24;
      if (2u * lane + 1u < (uint32_t)D) {  // the older record of the lane
        const uint32_t e = tab4_entry(d0[1], d1[1], y);
        g[y] = (e & 0x1FFFFu) | ((e >> 17) << 24);
      }
      if (2u * lane < (uint32_t)D) {  // the nearer one
        const uint32_t e = tab4_entry(d0[0], d1[0], y);
        f[y] = (e & 0x1FFFFu) | ((e >> 17) << 24);
      }
    }
    fn_after<LL>(f, g);  // the nearer applied after the older
    fn_scan_down<LL>(f, 1);
    fn_scan_down<LL>(f, 2);
    fn_scan_down<LL>(f, 4);
    fn_scan_down<LL>(f, 8);
    fn_scan_down<LL>(f, 16);
    // lane 0 now holds the window's function (its oldest super-tile applied first)
    if (D < 64) {
      const uint32_t ln = (uint32_t)D >> 1;
      const bool older = (D & 1) != 0;
      const unsigned long long K = __shfl_sync(0xffffffffu, older ? d0[1] : d0[0], ln);  // the inclusive one
      const uint32_t x = (uint32_t)__shfl_sync(0xffffffffu, older ? d1[1] : d1[0], ln);
      const uint32_t e = __shfl_sync(0xffffffffu, fn_at<LL>(f, x), 0);
      const uint32_t xc = e >> 24;
      *K_out = K + (e & 0xFFFFFFu) + __shfl_sync(0xffffffffu, acc_cnt, xc);
      *c_out = __shfl_sync(0xffffffffu, acc_carry, xc);
      return true;
    }
    uint32_t w[4];
#pragma unroll
    for (uint32_t y = 0; y < (uint32_t)LL; ++y) w[y] = __shfl_sync(0xffffffffu, f[y], 0);
    const uint32_t e = fn_at<LL>(w, lane < (uint32_t)LL ? lane : 0u);  // entry `lane` of the window
    const uint32_t y = e >> 24;
    const unsigned long long ac = __shfl_sync(0xffffffffu, acc_cnt, y);
    const uint32_t ax = __shfl_sync(0xffffffffu, acc_carry, y);
    acc_cnt = (e & 0xFFFFFFu) + ac;
    acc_carry = ax;
    base -= 64;
  }
}

// Fold of a super-tile of m <= 4 sub-tiles for patterns of LL <= 4 bytes (warp 1): lane r
// holds the function of warp region r % 8 of sub-tile r / 8 (idle lanes: the identity). Scans
// over each group of 8 lanes give the carry into every region from its sub-tile's carry-in
// (wrec), scans over the sub-tile functions the carry into every sub-tile from the
// super-tile's carry-in (subrec) and the super-tile function (entry `lane`). Checked when
// `whole`: some region is not covered end to end from some carry (*bad), or is neither covered
// nor free of kept starts (*mixed).
template <int LL>
__device__ __forceinline__ void fold_small_rec(const uint32_t* wt, const uint8_t* dense, uint8_t* wrec,
                                               uint8_t* subrec, uint32_t m, bool whole, bool* bad, bool* mixed,
                                               uint32_t* sup_cnt, uint32_t* sup_carry) {
  const uint32_t lane = threadIdx.x & 31u, jr = lane >> 3, wr = lane & 7u;
  const bool act = jr < m;
  uint32_t g[4];
#pragma unroll
  for (uint32_t y = 0; y < (uint32_t)LL; ++y) {
    g[y] = y << 24;
    if (act) {
      const uint32_t v = dense[lane] ? dense_region_entry(y, LL) : wt[lane * LL + y];
      const uint32_t wc = v & 0xFFFFu, co = v >> 16;
      g[y] = wc | (co << 24);
      if (whole && 2048u - y - wc * LL + co != 0u) {
        *bad = true;
        if (wc != 0u) *mixed = true;
      }
    }
  }
  fn_scan_up<LL>(g, 1, 8, wr);
  fn_scan_up<LL>(g, 2, 8, wr);
  fn_scan_up<LL>(g, 4, 8, wr);
  uint32_t h[4];
#pragma unroll
  for (uint32_t y = 0; y < (uint32_t)LL; ++y) {
    uint32_t x = __shfl_up_sync(0xffffffffu, g[y], 1, 8);
    if (wr == 0) x = y << 24;
    if (act) wrec[lane * LL + y] = (uint8_t)(x >> 24);
    h[y] = __shfl_sync(0xffffffffu, g[y], lane | 7u);  // the sub-tile's function
  }
  fn_scan_up<LL>(h, 8, 32, lane);
  fn_scan_up<LL>(h, 16, 32, lane);
#pragma unroll
  for (uint32_t y = 0; y < (uint32_t)LL; ++y) {
    uint32_t xe = __shfl_up_sync(0xffffffffu, h[y], 8);
    if (jr == 0) xe = y << 24;
    if (act && wr == 0) subrec[jr * LL + y] = (uint8_t)(xe >> 24);
    const uint32_t e = __shfl_sync(0xffffffffu, h[y], 31);  // entry y of the super-tile function
    if (lane == y) {
      *sup_cnt = e & 0xFFFFFFu;
      *sup_carry = e >> 24;
    }
  }
}

// Mode small (L <= 32): tile functions are tables over carries; lane c holds entry c.
// acc is the function of the tiles between the current window and t.
__device__ __forceinline__ bool lookback_small(const ReplaceParams& p, uint32_t t, uint32_t L,
                                               unsigned long long* K_out, uint32_t* c_out, uint32_t carry0) {
  const uint32_t lane = threadIdx.x & 31u;
  unsigned long long acc_cnt = 0;
  uint32_t acc_carry = lane;
  long long base = (long long)t - 1;
  for (;;) {
    uint32_t st;
    const int plr = warp_wait_window(p, base, &st);
    if (plr < 0) return false;
    const uint32_t pl = (uint32_t)plr;
    uint32_t e[32];
#pragma unroll
    for (int i = 0; i < 32; ++i) {
      e[i] = 0;
      if ((uint32_t)i < pl && lane < L) {
        const unsigned long long v = __ldcg(p.agg + (unsigned long long)(base - i) * L + lane);
        e[i] = (uint32_t)(v & 0x00FFFFFFull) | ((uint32_t)(v >> 32) << 24);
      }
    }
    if (pl < 32) {
      unsigned long long K = 0;
      uint32_t x = carry0;
      const long long jp = base - (long long)pl;
      if (jp >= 0) {
        K = __ldcg(&p.incl[jp].kept);
        x = __ldcg(&p.incl[jp].carry);
      }
#pragma unroll
      for (int i = 31; i >= 0; --i) {
        if ((uint32_t)i < pl) {
          const uint32_t v = __shfl_sync(0xffffffffu, e[i], x);
          K += v & 0x00FFFFFFu;
          x = v >> 24;
        }
      }
      *K_out = K + __shfl_sync(0xffffffffu, acc_cnt, x);
      *c_out = __shfl_sync(0xffffffffu, acc_carry, x);
      return true;
    }
    // the whole window holds aggregates: compose it and put it in front of acc
    uint32_t y = lane < L ? lane : 0u;
    unsigned long long wc = 0;
#pragma unroll
    for (int i = 31; i >= 0; --i) {
      const uint32_t v = __shfl_sync(0xffffffffu, e[i], y);
      wc += v & 0x00FFFFFFu;
      y = v >> 24;
    }
    const unsigned long long ac = __shfl_sync(0xffffffffu, acc_cnt, y);
    const uint32_t ax = __shfl_sync(0xffffffffu, acc_carry, y);
    acc_cnt = wc + ac;
    acc_carry = ax;
    base -= 32;
  }
}

template <int LL>
__device__ __forceinline__ void ks_compose_n(uint32_t& t0, uint32_t& t1, uint32_t o0, uint32_t o1) {
  uint32_t r[4] = {0u, 0u, 0u, 0u};
#pragma unroll
  for (uint32_t c = 0; c < (uint32_t)LL; ++c) {
    const uint32_t o = ks_get(o0, o1, c);
    const uint32_t m = ks_get(t0, t1, o >> 14);
    r[c] = ((o & 0x3FFFu) + (m & 0x3FFFu)) | (m & 0xC000u);
  }
  t0 = r[0] | (r[1] << 16);
  t1 = r[2] | (r[3] << 16);
}

// Kogge-Stone scan of the warp's 32 segment functions (L = LL <= 4): srec row of this
// segment (carry into it for each warp carry-in) and, from lane 31, the warp function.
// *dense (written by lane 0) tells whether the region is all candidates; then no table is
// written and every reader uses the closed forms.
template <int LL>
__device__ __forceinline__ void ks_warp_tables(uint64_t mask, uint32_t inv_l, uint64_t stride, uint8_t* srec_row,
                                               uint32_t* wtab_row, uint8_t* dense) {
  const uint32_t lane = threadIdx.x & 31u;
  const bool all = __all_sync(0xffffffffu, mask == ~0ull);
  if (lane == 0) *dense = all ? 1u : 0u;
  if (all) return;  // closed forms (dense_region_entry, dense_seg_carry): no tables
  uint32_t ent[4] = {0u, 0u, 0u, 0u};
#pragma unroll
  for (uint32_t c = 0; c < (uint32_t)LL; ++c) {
    const uint64_t mm = mask >> c;
    if (mm) {
      const uint32_t e = c + (uint32_t)(__ffsll((long long)mm) - 1);
      const Walk w = seg_walk(mask, e, LL, inv_l, stride);
      const uint32_t carry = w.end > 64 ? w.end - 64 : 0;
      ent[c] = w.cnt | (carry << 14);
    }
  }
  uint32_t t0 = ent[0] | (ent[1] << 16), t1 = ent[2] | (ent[3] << 16);
#pragma unroll
  for (int d = 1; d < 32; d <<= 1) {
    const uint32_t o0 = __shfl_up_sync(0xffffffffu, t0, d);
    const uint32_t o1 = __shfl_up_sync(0xffffffffu, t1, d);
    if (lane >= (uint32_t)d) ks_compose_n<LL>(t0, t1, o0, o1);
  }
  const uint32_t x0 = __shfl_up_sync(0xffffffffu, t0, 1), x1 = __shfl_up_sync(0xffffffffu, t1, 1);
#pragma unroll
  for (uint32_t c = 0; c < (uint32_t)LL; ++c)
    srec_row[c] = (uint8_t)(lane == 0 ? c : (ks_get(x0, x1, c) >> 14));
  if (lane == 31) {
#pragma unroll
    for (uint32_t c = 0; c < (uint32_t)LL; ++c) {
      const uint32_t v = ks_get(t0, t1, c);
      wtab_row[c] = (v & 0x3FFFu) | ((v >> 14) << 16);
    }
  }
}

// 16 bytes starting r = 4q + sh/8 bytes into the 32 bytes (A, B); q is warp-uniform.
__device__ __forceinline__ uint4 extract16(const uint4& A, const uint4& B, uint32_t q, uint32_t sh) {
  uint4 o;
  switch (q) {
    case 0:
      o.x = __funnelshift_r(A.x, A.y, sh); o.y = __funnelshift_r(A.y, A.z, sh);
      o.z = __funnelshift_r(A.z, A.w, sh); o.w = __funnelshift_r(A.w, B.x, sh);
      break;
    case 1:
      o.x = __funnelshift_r(A.y, A.z, sh); o.y = __funnelshift_r(A.z, A.w, sh);
      o.z = __funnelshift_r(A.w, B.x, sh); o.w = __funnelshift_r(B.x, B.y, sh);
      break;
    case 2:
      o.x = __funnelshift_r(A.z, A.w, sh); o.y = __funnelshift_r(A.w, B.x, sh);
      o.z = __funnelshift_r(B.x, B.y, sh); o.w = __funnelshift_r(B.y, B.z, sh);
      break;
    default:
      o.x = __funnelshift_r(A.w, B.x, sh); o.y = __funnelshift_r(B.x, B.y, sh);
      o.z = __funnelshift_r(B.y, B.z, sh); o.w = __funnelshift_r(B.z, B.w, sh);
      break;
  }
  return o;
}

// Exclusive / inclusive scan over lanes 0..7 (the warps of a CTA), done by every warp.
__device__ __forceinline__ void lanes8_sum(uint32_t v, uint32_t* excl, uint32_t* incl) {
  const uint32_t lane = threadIdx.x & 31u;
  uint32_t x = lane < 8u ? v : 0u;
#pragma unroll
  for (int d = 1; d < 8; d <<= 1) {
    const uint32_t o = __shfl_up_sync(0xffffffffu, x, d);
    if (lane >= (uint32_t)d) x += o;
  }
  *incl = x;
  uint32_t e = __shfl_up_sync(0xffffffffu, x, 1);
  *excl = lane == 0 ? 0u : e;
}
__device__ __forceinline__ uint32_t lanes8_excl_max(uint32_t v) {
  const uint32_t lane = threadIdx.x & 31u;
  uint32_t x = lane < 8u ? v : 0u;
#pragma unroll
  for (int d = 1; d < 8; d <<= 1) {
    const uint32_t o = __shfl_up_sync(0xffffffffu, x, d);
    if (lane >= (uint32_t)d) x = o > x ? o : x;
  }
  const uint32_t e = __shfl_up_sync(0xffffffffu, x, 1);
  return lane == 0 ? 0u : e;
}

}  // namespace

// Number of 16 KiB sub-tiles in super-tile `tile`.
__device__ __forceinline__ uint32_t subs_in_tile(uint32_t tile, unsigned long long S, unsigned long long n,
                                                 uint32_t nsub) {
  const unsigned long long rem = n - (unsigned long long)tile * S;
  const unsigned long long m = (rem + kTile - 1) / kTile;
  return m < nsub ? (uint32_t)m : nsub;
}

// Ring of kNBuf shared-memory buffers fed by 1-D TMA loads. Every thread keeps the same
// `consumed` count; only thread 0 issues (and tracks the issue position).
struct LoadRing {
  uint32_t issued, consumed;
  uint32_t ij;   // next sub-tile of the head phase
  uint32_t qh;   // head of the phase queue
  uint32_t nph;  // phases queued (at most kPhases)
  uint32_t halo_b;  // pass-B loads include the halo (kModeMulti: a match's pattern is looked up again)
  uint32_t* q;   // the queue in shared memory: super-tile << 1 | kind (0: pass A, 1: pass B)
  static constexpr uint32_t kPhases = 4;

  __device__ __forceinline__ void init(uint32_t* qs, bool halo_in_b = false) {
    issued = consumed = 0;
    ij = qh = nph = 0;
    halo_b = halo_in_b ? 1u : 0u;
    q = qs;
  }
  // Thread 0: queue the loads of one pass over super-tile t (kind 0: sub-tiles with their
  // halo, for pass A; kind 1: sub-tiles, for pass B), consumed in the order queued.
  __device__ __forceinline__ void push(uint32_t t, uint32_t kind) {
    q[(qh + nph) & (kPhases - 1u)] = (t << 1) | kind;
    ++nph;
  }
  // Thread 0: keep up to kNBuf loads in flight.
  __device__ __forceinline__ void issue(const ReplaceParams& p, uint8_t* smem, const LayoutS& lay, uint64_t* bars,
                                        unsigned long long S, unsigned long long n16, uint32_t want_a,
                                        unsigned long long n, uint32_t nsub) {
    while (issued - consumed < (uint32_t)kNBuf && nph > 0) {
      const uint32_t e = q[qh];
      const uint32_t t = e >> 1, kind = e & 1u;
      const uint32_t m = subs_in_tile(t, S, n, nsub);
      const unsigned long long start = (unsigned long long)t * S + (unsigned long long)ij * kTile;
      const unsigned long long avail = n16 - start;
      const uint32_t want = (kind == 0 || halo_b) ? want_a : (uint32_t)kTile;
      const uint32_t bytes = avail < want ? (uint32_t)avail : want;
      const uint32_t b = issued % kNBuf;
      // no proxy fence: the buffer's earlier contents were only read, and every read of them
      // completed before the block barrier that freed it (a write cannot reach a finished read)
      mbar_arrive_expect_tx(&bars[b], bytes);
      bulk_load_hint(smem + lay.in0 + b * lay.inbytes, p.in + start, bytes, &bars[b],
                     kind == 0 ? l2_policy_evict_last() : l2_policy_evict_first());
      ++issued;
      if (++ij == m) {
        ij = 0;
        qh = (qh + 1u) & (kPhases - 1u);
        --nph;
      }
    }
  }
  // Wait for the next load in consumption order; returns its buffer.
  __device__ __forceinline__ uint8_t* wait(const ReplaceParams& p, uint8_t* smem, const LayoutS& lay,
                                           uint64_t* bars, uint32_t* fail) {
    const uint32_t b = consumed % kNBuf;
    const uint32_t parity = (consumed / kNBuf) & 1u;
    if (!wait_tile(&bars[b], parity)) {
      if (threadIdx.x == 0) {
        set_error(p);
        *fail = 1;
      }
    }
    return smem + lay.in0 + b * lay.inbytes;
  }
  // After a block barrier: every thread is done with the current buffer.
  __device__ __forceinline__ void release() { ++consumed; }
};

// k output chunks of one lane of warp_emit_literal, 512 bytes apart (the warp's 32 lanes
// interleaved): the word offset Q of the source within its 16-byte chunk is the same for every
// chunk of a call, so the loop is instantiated per offset (no selection inside it) and kept
// rolled (unrolled copies of the four instances spilled registers).
template <int Q>
__device__ __forceinline__ void literal_chunks(uint8_t* dst, const uint8_t* src, uint32_t k, uint32_t sh) {
#pragma unroll 1
  for (; k; --k) {
    const uint4 A = *reinterpret_cast<const uint4*>(src);
    const uint4 B = *reinterpret_cast<const uint4*>(src + 16u);
    st_out16(dst, extract16(A, B, (uint32_t)Q, sh));
    src += 512u;
    dst += 512u;
  }
}

// One warp's output when it is a copy of its input: wtot bytes from tile byte srcw, written at
// out[g0, g0 + wtot) with aligned 16-byte stores (funnel-shifted from shared memory); the
// partial 16-byte chunks at both ends one byte per lane (the neighbouring regions own their
// other bytes).
__device__ __forceinline__ void warp_emit_literal(uint8_t* out, const uint8_t* tb, unsigned long long g0,
                                                  uint32_t wtot, uint32_t srcw) {
  const uint32_t lane = threadIdx.x & 31u;
  const unsigned long long ga = g0 & ~15ull;
  const unsigned long long gend = g0 + wtot;
  const uint32_t c0 = (uint32_t)((g0 - ga + 15ull) >> 4);  // first whole 16-byte chunk
  const uint32_t c1 = (uint32_t)((gend - ga) >> 4);        // end of the whole chunks
  const uint32_t off0 = srcw + (uint32_t)(ga + ((unsigned long long)c0 << 4) - g0);
  const uint32_t r = off0 & 15u, q = r >> 2, sh = (r & 3u) * 8u;
  {
    const uint32_t c = c0 + lane;
    if (c < c1) {
      const uint32_t k = (c1 - c + 31u) >> 5;  // this lane's chunks c, c + 32, ...
      const uint8_t* src = tb + (off0 - r + ((c - c0) << 4));
      uint8_t* dst = out + ga + ((unsigned long long)c << 4);
      switch (q) {  // the same in every lane
        case 0: literal_chunks<0>(dst, src, k, sh); break;
        case 1: literal_chunks<1>(dst, src, k, sh); break;
        case 2: literal_chunks<2>(dst, src, k, sh); break;
        default: literal_chunks<3>(dst, src, k, sh); break;
      }
    }
  }
  unsigned long long b;
  bool ok;
  if (c0 < c1) {
    b = lane < 16u ? g0 + lane : ga + ((unsigned long long)c1 << 4) + (lane - 16u);
    ok = lane < 16u ? (b < ga + ((unsigned long long)c0 << 4)) : (b < gend);
  } else {
    b = g0 + lane;
    ok = b < gend;
  }
  if (ok) out[b] = tb[srcw + (uint32_t)(b - g0)];
}

// x mod R for x < 2^26 and 1 <= R <= 64, with rmag = ceil(2^32 / R) (0 for R = 1): the
// quotient is the high word of x * rmag (its error, below x / 2^32, stays under 1/R).
__host__ __device__ __forceinline__ uint32_t mod_magic(uint32_t R) {
  return R > 1u ? (uint32_t)((0x100000000ull + R - 1u) / R) : 0u;
}
__device__ __forceinline__ uint32_t mod_small(uint32_t x, uint32_t R, uint32_t rmag) {
  return R > 1u ? x - __umulhi(x, rmag) * R : 0u;
}

// One warp's output when it is a run of replacements: 16 bytes per phase from the table t16
// (the replacement repeated from every phase), the partial chunks from rs byte by byte.
__device__ __forceinline__ void warp_emit_replace(uint8_t* out, const uint4* t16, const uint8_t* rs, uint32_t R,
                                                  uint32_t step512, uint32_t rmag, unsigned long long g0,
                                                  uint32_t wtot, uint32_t ph0 = 0) {
  const uint32_t lane = threadIdx.x & 31u;
  const unsigned long long ga = g0 & ~15ull;
  const unsigned long long gend = g0 + wtot;
  const uint32_t c0 = (uint32_t)((g0 - ga + 15ull) >> 4);
  const uint32_t c1 = (uint32_t)((gend - ga) >> 4);
  uint32_t c = c0 + lane;
  // phase of chunk c: its distance from g0, plus the phase ph0 < R at g0, modulo R
  uint32_t ph = mod_small(((c << 4) - (uint32_t)(g0 - ga)) + ph0, R, rmag);
  // (both loops kept rolled: unrolled, they cost registers elsewhere in the kernel and measured
  // 3% slower on aa->X)
  if (step512 == 0u) {  // every chunk of this lane has the same phase
    const uint4 v = t16[ph];
#pragma unroll 1
    for (; c < c1; c += 32u) st_out16(out + ga + ((unsigned long long)c << 4), v);
  } else {
#pragma unroll 1
    for (; c < c1; c += 32u) {
      st_out16(out + ga + ((unsigned long long)c << 4), t16[ph]);
      ph += step512;
      if (ph >= R) ph -= R;
    }
  }
  unsigned long long b;
  bool ok;
  if (c0 < c1) {
    b = lane < 16u ? g0 + lane : ga + ((unsigned long long)c1 << 4) + (lane - 16u);
    ok = lane < 16u ? (b < ga + ((unsigned long long)c0 << 4)) : (b < gend);
  } else {
    b = g0 + lane;
    ok = b < gend;
  }
  if (ok) out[b] = rs[mod_small((uint32_t)(b - g0) + ph0, R, rmag)];
}

// Input length, output range and super-tile count of the job described by p.
struct JobDims {
  unsigned long long n_all, n, n16;
  uint32_t NT, carry0, want_a;
};
__device__ __forceinline__ JobDims job_dims(const ReplaceParams& p, unsigned long long S) {
  JobDims d;
  // n_all bytes are in the buffer (matches may reach up to it); output covers the first n
  d.n_all = p.n_dev ? min(*p.n_dev, p.n_cap ? p.n_cap : ~0ull) : p.n;
  d.n = d.n_all > p.hold ? d.n_all - p.hold : 0ull;
  d.n16 = (d.n_all + 15ull) & ~15ull;
  d.NT = (uint32_t)min((d.n + S - 1ull) / S, (unsigned long long)p.num_tiles);
  d.carry0 = p.carry0_dev ? *p.carry0_dev : p.carry0;
  d.want_a = align_up_u32(kTile + (p.L > 1 ? p.L - 1 : 0), 16);
  return d;
}

// Segmented launch, thread 0: claim the next super-tile of the launch; when it belongs to
// another job than the one in sj, describe that job in sj. Returns the job-local super-tile
// index, or 0xFFFFFFFF when the launch has no super-tile left.
__device__ __forceinline__ uint32_t seg_claim(const SegLaunch& sl, ReplaceParams& sj, uint32_t* cur_job,
                                              uint32_t* newjob) {
  const uint32_t g = atomicAdd(sl.sched, 1u);
  if (g >= *sl.total) return 0xFFFFFFFFu;
  const uint32_t j = sl.tile_job[g];
  const SegJob& J = sl.jobs[j];
  const uint32_t base = J.tile_base;
  if (j != *cur_job) {
    *cur_job = j;
    *newjob = 1u;
    const SegPair& Q = sl.pairs[J.pair];
    sj.in = J.in;
    sj.out = J.out;
    sj.n = *J.n_dev;
    sj.out_cap = J.out_cap;
    sj.block_before = 0;
    sj.stride_mask = Q.stride_mask;
    sj.L = Q.L;
    sj.R = Q.R;
    sj.mode = Q.mode;
    sj.num_tiles = J.ntiles;
    sj.epoch = sl.epoch[1];
    sj.agg_entries = Q.agg_entries;
    sj.p4 = Q.p4;
    sj.m4 = Q.m4;
    sj.inv_l = Q.inv_l;
    sj.nsub = sl.nsub;
    sj.status = sl.status + base;
    sj.incl = sl.incl + base;
    sj.agg = sl.agg + (unsigned long long)base * sl.agg_stride;
    sj.res = sl.res + J.res;
    sj.tile_last = sl.tile_last + base;
    sj.rec = sl.rec + 2ull * base;
    sj.n_dev = nullptr;
    sj.len_out = J.len_out;
    sj.carry0_dev = nullptr;
    sj.carry_out = nullptr;
    sj.hold = 0;
    sj.n_cap = 0;
    sj.len_bias = 0;
    sj.carry0 = 0;
    sj.pat_ext = Q.pat;
    sj.rep_ext = Q.rep;
    sj.multi = nullptr;
    sj.presence = nullptr;
  }
  return g - base;
}

// One kernel for one apply (SEG = false: the job is the launch parameter pk) and for a
// segmented launch over a job table (SEG = true: the job of each super-tile is looked up
// and described in shared memory).
template <int MODE, bool SEG>
__global__ void __launch_bounds__(kThreads, 3)
    replace_super_kernel(const __grid_constant__ ReplaceParams pk, const __grid_constant__ SegLaunch sl) {
  extern __shared__ __align__(128) uint8_t smem[];
  __shared__ ReplaceParams s_job;           // segmented launch: the job of the current super-tile
  __shared__ uint32_t s_jobid, s_newjob;    // segmented launch: that job's index; its pattern is not staged yet
  __shared__ __align__(8) uint64_t s_bar[kNBuf];
  __shared__ uint32_t s_scan2[2][kWarps];  // alternating buffers of block_excl_scan1
  __shared__ uint32_t s_q[2];               // the super-tile this CTA works on
  __shared__ unsigned long long s_kexcl;
  __shared__ uint32_t s_cin;
  __shared__ uint32_t s_tcnt, s_cout;       // kept starts in the super-tile looked back for; its carry-out
  __shared__ uint32_t s_fail;
  __shared__ uint32_t s_cutlen;             // exact output length of the warp region cut at n
  // per-super-tile tables, two sets: one super-tile's pass A runs while the previous one
  // looks back and writes its output (one set in a segmented launch)
  __shared__ uint32_t s_sub_lco[2 * kMaxSub];
  __shared__ uint32_t s_wcnt[2 * kMaxSub * kWarps];   // kModeFree: kept count per (sub-tile, warp)
  __shared__ uint32_t s_wcend[2 * kMaxSub * kWarps];  // kModeFree: max cover end per (sub-tile, warp)
  __shared__ int s_wd[2 * kMaxSub * kWarps];          // kModeMulti: sum of R - L per (sub-tile, warp)
  __shared__ unsigned long long s_frcnt[2];          // kModeFree: super-tile function (count, local carry-out)
  __shared__ long long s_frlco[2];
  __shared__ uint32_t s_supc[2][32], s_supx[2][32];  // kModeSmall: super-tile table over carries
  __shared__ uint32_t s_noin[2];
  __shared__ uint8_t s_dense[2][kMaxSub * kWarps];  // kModeSmall, L <= 4: region (j, w) is dense  // pass B mode: 0 general, 1 table-driven without input, 2 table-driven
  __shared__ uint32_t s_phq[LoadRing::kPhases];

  const ReplaceParams& p = SEG ? s_job : pk;
  unsigned int* const sched = SEG ? sl.sched : &pk.res->tile_counter;  // claim counter, then finished CTAs
  const uint32_t nsub = SEG ? sl.nsub : pk.nsub;
  const LayoutS lay =
      SEG ? make_layout_s(MODE, sl.Lmax, sl.Rmax, nsub, 3u)
          : make_layout_s(MODE, pk.L, pk.R, nsub, MODE == kModeMulti ? pk.multi_ratio : 0u, 2u);
  uint8_t* ps = smem + lay.pat;
  uint8_t* rs = smem + lay.rep;
  uint8_t* ob = smem + lay.outb;
  uint64_t* masks = reinterpret_cast<uint64_t*>(smem + lay.masks);
  // kModeMulti follows the free-mode paths (every occurrence kept), with per-pair lengths
  constexpr bool kFreeLike = MODE == kModeFree || MODE == kModeMulti;
  const MultiTable& MT = *reinterpret_cast<const MultiTable*>(smem + lay.mtab);
  const uint32_t tid = threadIdx.x, lane = tid & 31u, warp = tid >> 5;
  const uint32_t sb = tid * kSeg;
  const unsigned long long S = (unsigned long long)nsub * kTile;
  // the job's dimensions and pattern: once (one apply) or whenever the job changes (segmented)
  uint32_t L = 0, R = 0, NT = 0, carry0 = 0, want_a = 0, step4 = 0, step512 = 0, rmag = 0;
  unsigned long long n_all = 0, n = 0, n16 = 0;
  bool rep_table = false;
  bool run_pat = false;  // the pattern's first min(L, 4) bytes are its first byte repeated
  auto setup_job = [&]() {
    const JobDims d = job_dims(p, S);
    n_all = d.n_all;
    n = d.n;
    n16 = d.n16;
    NT = d.NT;
    carry0 = d.carry0;
    want_a = d.want_a;
    L = p.L;
    R = p.R;
    rep_table = R >= 1u && R <= 64u;
    run_pat = ((p.p4 ^ ((p.p4 & 0xFFu) * 0x01010101u)) & p.m4) == 0u;
    step4 = R ? 4u % R : 0u;
    step512 = R ? 512u % R : 0u;
    rmag = mod_magic(R);
    const uint8_t* psrc = (!SEG && L <= (uint32_t)kInlineMax) ? p.pat : p.pat_ext;
    const uint8_t* rsrc = (!SEG && R <= (uint32_t)kInlineMax) ? p.rep : p.rep_ext;
    for (uint32_t i = tid; i < L; i += kThreads) ps[i] = psrc[i];
    // the replacement repeated: rs[i] = rep[i mod R] for i < R + 16
    for (uint32_t i = tid; i < R + 16; i += kThreads) rs[i] = R ? rsrc[i % R] : (uint8_t)0;
    if (rep_table) {
      uint8_t* t16 = smem + lay.tab16;
      for (uint32_t i = tid; i < R * 16u; i += kThreads) t16[i] = rsrc[((i >> 4) + (i & 15u)) % R];
    }
    if constexpr (MODE == kModeMulti) {  // the stage's pair table
      const uint4* src = reinterpret_cast<const uint4*>(p.multi);
      uint4* dst = reinterpret_cast<uint4*>(smem + lay.mtab);
      for (uint32_t i = tid; i < (uint32_t)(sizeof(MultiTable) / 16u); i += kThreads) dst[i] = src[i];
    }
  };
  if (!SEG) {
    setup_job();
    if (NT == 0 && blockIdx.x == 0 && threadIdx.x == 0) {  // nothing to emit: still report
      if (p.len_out) *p.len_out = p.len_bias;
      if (p.carry_out) *p.carry_out = carry0 > n ? carry0 - (uint32_t)n : 0u;
      p.res->out_len = 0;
      p.res->kept = 0;
    }
  }
  uint32_t nscan = 0;  // block_excl_scan1 calls so far (selects the scratch buffer)

  // ---- load ring: thread 0 queues the loads of each pass in the order they are consumed
  LoadRing ring;
  ring.init(s_phq, MODE == kModeMulti);

  // pass A of super-tile t and its function (published as an aggregate record); tables in set `set`
  auto tile_front = [&](const uint32_t t, const uint32_t set) {
    const uint32_t m = subs_in_tile(t, S, n, nsub);
    const unsigned long long tstart = (unsigned long long)t * S;
    uint64_t* const masks_s = masks + (size_t)set * nsub * kThreads;
    uint32_t* const wcnt_s = s_wcnt + set * (kMaxSub * kWarps);
    uint32_t* const wcend_s = s_wcend + set * (kMaxSub * kWarps);
    uint32_t* const sublco_s = s_sub_lco + set * kMaxSub;
    uint8_t* const srec_b = smem + lay.srec + set * lay.srec_set;
    uint8_t* const wtab_b = smem + lay.wtab + set * lay.wtab_set;
    uint8_t* const wrec_b = smem + lay.wrec + set * lay.wrec_set;
    uint8_t* const subrec_b = smem + lay.subrec + set * lay.subrec_set;
    // ================= pass A: candidates and per-warp functions of every sub-tile
    bool run_try = run_pat;  // re-armed for every super-tile
    // bounds: candidates p in [block_before, lim); a super-tile inside both needs no masking
    // (kModeMulti: p < n here; each pattern's own length is checked against n_all when found)
    const unsigned long long lim =
        MODE == kModeMulti ? n : ((n_all >= L) ? min(n_all - L + 1, n) : 0ull);  // candidates p < lim
    const bool edge = tstart < p.block_before || tstart + (unsigned long long)m * kTile > lim;
    // (this and the other per-sub-tile loops are kept rolled: their bodies are large, and
    // unrolled copies measured about 1% slower)
#pragma unroll 1
    for (uint32_t j = 0; j < m; ++j) {
      uint8_t* tb = ring.wait(p, smem, lay, s_bar, &s_fail);
      const unsigned long long gseg = tstart + (unsigned long long)j * kTile + sb;
      bool uni = false;
      uint64_t mask;
      // presence index: no candidate can start in a sub-tile whose chunk lacks the first byte
      const bool absent = !SEG && MODE != kModeMulti && p.presence &&
                          !((p.presence[((tstart + (unsigned long long)j * kTile) >> p.presence_shift) * 8ull +
                                        ((p.p4 & 0xFFu) >> 5)] >> (p.p4 & 31u)) & 1u);
      if constexpr (MODE == kModeMulti) {
        mask = multi_first_mask(tb + sb, MT.firsts, MT.nfirst);
      } else {
        mask = absent ? 0ull : candidates_seg(tb + sb, p.p4, p.m4, L, run_try, &uni);
      }
      run_try = uni;  // keep testing while the text is runs of b0
      const unsigned long long sub0 = tstart + (unsigned long long)j * kTile;
      if (edge && (sub0 < p.block_before || sub0 + kTile > lim)) {
        uint32_t lo = 0, hi = 0;
        if (p.block_before > gseg) {
          const unsigned long long d = p.block_before - gseg;
          lo = d < 64ull ? (uint32_t)d : 64u;
        }
        if (lim > gseg) {
          const unsigned long long d = lim - gseg;
          hi = d < 64ull ? (uint32_t)d : 64u;
        }
        mask &= low_bits(hi) & ~low_bits(lo);
      }
      if constexpr (MODE == kModeMulti) {
        // each position holding a first pattern byte: which pattern occurs there, if any; every
        // occurrence is kept. Per thread: D = sum of R - L, and where its last match ends.
        uint64_t kept = 0;
        int dsum = 0;
        uint32_t lastend = 0;
        while (mask) {
          const uint32_t b = (uint32_t)(__ffsll((long long)mask) - 1);
          mask &= mask - 1ull;
          const int k = multi_identify(MT, tb + sb + b, n_all - (gseg + b));
          if (k >= 0) {
            kept |= 1ull << b;
            dsum += (int)MT.R[k] - (int)MT.L[k];
            lastend = b + MT.L[k];
          }
        }
        mask = kept;
        masks_s[j * kThreads + tid] = mask;
        const uint32_t cnt = __reduce_add_sync(0xffffffffu, (uint32_t)__popcll(mask));
        const int wd = __reduce_add_sync(0xffffffffu, dsum);
        const uint32_t cend = __reduce_max_sync(0xffffffffu, mask ? sb + lastend : 0u);
        if (lane == 0) {
          wcnt_s[j * kWarps + warp] = cnt;
          s_wd[set * (kMaxSub * kWarps) + j * kWarps + warp] = wd;
          wcend_s[j * kWarps + warp] = cend;
        }
      } else {
      if (L > 4) mask = verify_tail(mask, tb + sb, ps, L);
      masks_s[j * kThreads + tid] = mask;
      if (MODE == kModeFree) {
        // every candidate is kept: per warp, the count and how far its last match reaches
        const uint32_t cnt = __reduce_add_sync(0xffffffffu, (uint32_t)__popcll(mask));
        const uint32_t cend = __reduce_max_sync(
            0xffffffffu, mask ? sb + (63u - (uint32_t)__clzll((long long)mask)) + L : 0u);
        if (lane == 0) {
          wcnt_s[j * kWarps + warp] = cnt;
          wcend_s[j * kWarps + warp] = cend;
        }
      } else {
        uint8_t* srec = srec_b + (size_t)j * kThreads * L;
        uint32_t* wtab = reinterpret_cast<uint32_t*>(wtab_b) + (size_t)(j * kWarps + warp) * L;
        if (L == 2u) {
          ks_warp_tables<2>(mask, p.inv_l, p.stride_mask, srec + tid * 2u, wtab, &s_dense[set][j * kWarps + warp]);
        } else if (L == 3u) {
          ks_warp_tables<3>(mask, p.inv_l, p.stride_mask, srec + tid * 3u, wtab, &s_dense[set][j * kWarps + warp]);
        } else if (L == 4u) {
          ks_warp_tables<4>(mask, p.inv_l, p.stride_mask, srec + tid * 4u, wtab, &s_dense[set][j * kWarps + warp]);
        } else {
          // segment tables in shared memory, then lanes-over-carries walks of the warp's
          // own 32 segments (only rows of this warp are read: a warp barrier suffices)
          uint16_t* segtab = reinterpret_cast<uint16_t*>(smem + lay.segtab);
          build_seg_table16(mask, L, p.inv_l, p.stride_mask, segtab + tid * lay.rs);
          __syncwarp();
          if (lane < L) {
            uint32_t x = lane, cnt = 0;
            const uint32_t seg0 = warp * 32u;
#pragma unroll 8
            for (uint32_t k = 0; k < 32; ++k) {
              const uint32_t seg = seg0 + k;
              srec[seg * L + lane] = (uint8_t)x;
              const uint32_t v = segtab[seg * lay.rs + x];
              cnt += v & 0xFFu;
              x = v >> 8;
            }
            wtab[lane] = cnt | (x << 16);
          }
        }
      }
      }  // not kModeMulti
      __syncthreads();
      ring.release();
      if (tid == 0) ring.issue(p, smem, lay, s_bar, S, n16, want_a, n, nsub);
    }

    // ================= fold the sub-tiles into the super-tile function
    // (warp 1, so that warp 0 can start the previous super-tile's look-back at the same time)
    const bool use_rec = kFreeLike || L <= 4u;
    const uint32_t tag = p.epoch & 0xFFFFFFu;
    unsigned long long fr_cnt = 0;  // kModeFree: lane 0 of warp 1
    long long fr_lco = 0;
    uint32_t sup_cnt = 0, sup_carry = lane;  // kModeSmall: warp 1, lane = carry-in
    // Pass B of a whole super-tile is table-driven when every warp region's output is a run of
    // replacements (the kept matches cover every byte; nothing when R = 0) or a copy of its
    // input (no kept start): the tables alone place every region. With no copies (mode 1) pass B
    // reads no input: the super-tile's second loads, their waits and its per-sub-tile barriers
    // are skipped; with copies (mode 2) the loads stay. Free mode checks
    // the carry 0 (full cover of the first region needs a match at byte 0, so no match
    // of the previous super-tile can reach into it), small mode every carry into every region.
    const bool whole = !SEG && m == nsub && nsub * kWarps <= 32u && tstart + S <= n && L <= 64u &&
                       (R == 0u || rep_table);
    uint32_t noin = 0;
    if (kFreeLike) {
      if (warp == 1) {
        // lane r stands for warp region r % 8 of sub-tile j0 + r / 8 (groups of 8 lanes)
        const uint32_t wr = lane & 7u;
        bool ok = whole;   // every region covered end to end (whole: m <= 4, one round)
        bool tin = whole;  // every region covered end to end or free of kept starts
        uint32_t cnt_sum = 0;
        int dsum = 0;      // kModeMulti: sum of R - L over the super-tile's matches
        long long lco_max = LLONG_MIN;
#pragma unroll 1
        for (uint32_t j0 = 0; j0 < m; j0 += 4u) {
          const uint32_t jr = j0 + (lane >> 3);
          const bool act = jr < m;
          const uint32_t wc = act ? wcnt_s[jr * kWarps + wr] : 0u;
          const uint32_t ce = act ? wcend_s[jr * kWarps + wr] : 0u;
          uint32_t gmax = ce, pre = ce;  // sub-tile max reach; inclusive max over earlier regions
#pragma unroll
          for (int d = 1; d < 8; d <<= 1) {
            const uint32_t x = __shfl_xor_sync(0xffffffffu, gmax, d, 8);
            gmax = x > gmax ? x : gmax;
            const uint32_t o = __shfl_up_sync(0xffffffffu, pre, d, 8);
            if (wr >= (uint32_t)d) pre = o > pre ? o : pre;
          }
          pre = __shfl_up_sync(0xffffffffu, pre, 1, 8);
          if (wr == 0) pre = 0;
          const uint32_t lco = gmax > (uint32_t)kTile ? gmax - (uint32_t)kTile : 0u;  // reach past the sub-tile
          if (act && wr == 0) sublco_s[jr] = lco;
          cnt_sum += __reduce_add_sync(0xffffffffu, wc);
          if (MODE == kModeMulti)
            dsum += __reduce_add_sync(0xffffffffu, act ? s_wd[set * (kMaxSub * kWarps) + jr * kWarps + wr] : 0);
          // the super-tile's reach: max over sub-tiles of their reach, less the sub-tiles after them
          const long long v = act ? (long long)lco - (long long)(m - 1u - jr) * kTile : LLONG_MIN;
          lco_max = v > lco_max ? v : lco_max;
          if (ok) {
            // carry into the sub-tile from carry 0: the previous sub-tile's reach (L <= 64)
            uint32_t csj = __shfl_up_sync(0xffffffffu, lco, 8);
            if (jr == 0) csj = 0;
            const uint32_t covs = csj > pre ? csj : pre;  // reach of everything before the region
            const uint32_t wlo = wr * 2048u;
            uint32_t wcov = covs > wlo ? covs - wlo : 0u;
            wcov = wcov < 2048u ? wcov : 2048u;
            const uint32_t over = ce > wlo + 2048u ? ce - (wlo + 2048u) : 0u;
            // (kModeMulti: the replacements differ, so no region is a run of one replacement)
            const bool full = MODE != kModeMulti && 2048u - wcov - wc * L + over == 0u;
            ok = __all_sync(0xffffffffu, !act || full);
            // (kModeFree: a region with at most 16 matches is written as pieces in mode 2)
            tin = __all_sync(0xffffffffu, !act || full || wc == 0u || (MODE == kModeFree && wc <= 16u));
          }
        }
#pragma unroll
        for (int d = 16; d >= 1; d >>= 1) {
          const long long o = __shfl_xor_sync(0xffffffffu, lco_max, d);
          lco_max = o > lco_max ? o : lco_max;
        }
        // kModeMulti: the look-back sums sum(R - L) + kMultiBias per super-tile (a payload >= 0)
        fr_cnt = MODE == kModeMulti ? (unsigned long long)((long long)dsum + (long long)kMultiBias) : cnt_sum;
        fr_lco = lco_max;
        noin = ok ? 1u : (tin ? 2u : 0u);
        if (lane == 0 && t > 0)
          rec_store(p.rec, t, rec_word(tag, kStAgg, fr_cnt), rec_word(tag, kStAgg, (unsigned long long)fr_lco));
      }
    } else if (warp == 1) {
      const uint32_t* wt = reinterpret_cast<const uint32_t*>(wtab_b);
      bool bad = false;    // some region is not covered from some carry
      bool mixed = false;  // some region is neither covered nor free of kept starts
      if (use_rec && m <= 4u) {
        if (L == 2u)
          fold_small_rec<2>(wt, s_dense[set], wrec_b, subrec_b, m, whole, &bad, &mixed, &sup_cnt, &sup_carry);
        else if (L == 3u)
          fold_small_rec<3>(wt, s_dense[set], wrec_b, subrec_b, m, whole, &bad, &mixed, &sup_cnt, &sup_carry);
        else
          fold_small_rec<4>(wt, s_dense[set], wrec_b, subrec_b, m, whole, &bad, &mixed, &sup_cnt, &sup_carry);
      } else
#pragma unroll 1
      for (uint32_t j = 0; j < m; ++j) {
        uint8_t* wrec = wrec_b + (size_t)j * kWarps * L;
        uint32_t y = lane < L ? lane : 0u, cnt = 0;
#pragma unroll
        for (uint32_t w = 0; w < (uint32_t)kWarps; ++w) {
          if (lane < L) wrec[w * L + lane] = (uint8_t)y;
          const uint32_t v = (L <= 4u && s_dense[set][j * kWarps + w]) ? dense_region_entry(y, L)
                                                                       : wt[(j * kWarps + w) * L + y];
          cnt += v & 0xFFFFu;
          y = v >> 16;
        }
        if (lane < L) (subrec_b)[j * L + lane] = (uint8_t)sup_carry;
        if (whole && lane < L) {
#pragma unroll
          for (uint32_t w = 0; w < (uint32_t)kWarps; ++w) {
            const uint32_t v = (L <= 4u && s_dense[set][j * kWarps + w])  // region w from carry `lane`
                                   ? dense_region_entry(lane, L)
                                   : wt[(j * kWarps + w) * L + lane];
            const uint32_t wc = v & 0xFFFFu, co = v >> 16;
            if (2048u - lane - wc * L + co != 0u) {
              bad = true;
              if (wc != 0u) mixed = true;
            }
          }
        }
        const uint32_t tc = __shfl_sync(0xffffffffu, cnt, sup_carry);
        const uint32_t tx = __shfl_sync(0xffffffffu, y, sup_carry);
        sup_cnt += tc;
        sup_carry = tx;
      }
      noin = !whole ? 0u : (!__any_sync(0xffffffffu, bad) ? 1u : (!__any_sync(0xffffffffu, mixed) ? 2u : 0u));
      if (use_rec) {
        unsigned long long e = lane < L ? ((unsigned long long)sup_cnt | ((unsigned long long)sup_carry << 17)) : 0ull;
        const unsigned long long e1 = __shfl_sync(0xffffffffu, e, 1), e2 = __shfl_sync(0xffffffffu, e, 2),
                                 e3 = __shfl_sync(0xffffffffu, e, 3);
        if (lane == 0 && t > 0)
          rec_store(p.rec, t, rec_word(tag, kStAgg, e | (e1 << 19)), rec_word(tag, kStAgg, e2 | (e3 << 19)));
      } else {
        if (t > 0 && lane < L)
          __stcg(p.agg + (unsigned long long)t * L + lane, (unsigned long long)sup_cnt |
                                                                ((unsigned long long)sup_carry << 32));
        __threadfence();
        __syncwarp();
        if (t > 0 && lane == 0) st_release_u32(p.status + t, (p.epoch << 2) | kStAgg);
      }
    }

    if (kFreeLike) {
      if (tid == 32u) {
        s_frcnt[set] = fr_cnt;
        s_frlco[set] = fr_lco;
        s_noin[set] = noin;
      }
    } else if (warp == 1) {
      s_supc[set][lane] = sup_cnt;
      s_supx[set][lane] = sup_carry;
      if (lane == 0) s_noin[set] = noin;
    }
  };

  constexpr uint32_t kNone = 0xFFFFFFFFu;
  // Thread 0, one apply: claim the next super-tile and queue its pass-A loads, then the pass-B
  // loads of super-tile tcur (whose pass A filled set cset) unless its pass B reads no input.
  auto claim_next = [&]() {
    const uint32_t c = atomicAdd(sched, 1u);
    const uint32_t nx = c < NT ? c : kNone;
    s_q[0] = nx;
    if (nx != kNone) ring.push(nx, 0);
  };
  auto schedule = [&](const uint32_t tcur, const uint32_t cset) {
    claim_next();
    if (s_noin[cset] != 1u) ring.push(tcur, 1);
    ring.issue(p, smem, lay, s_bar, S, n16, want_a, n, nsub);
  };

  // Output of one warp region with at most 16 matches (kFreeLike): literal runs between its
  // replacements. Each run is copied by the whole warp (aligned 16-byte stores, like a
  // copy-only region), each replacement by as many lanes as it has bytes; no staging of the
  // whole output. kept: this thread's kept starts in its 64-byte segment of the sub-tile at tb
  // (global position gseg); x0r: bytes at the region start covered by an earlier match; vend:
  // input bytes of the region; the output is out[g0, g0 + wtot). Returns false, writing
  // nothing, when the region has more than 16 matches; when the pieces do not add up to wtot
  // (which the arithmetic rules out) it writes nothing and reports an error.
  auto emit_pieces = [&](const uint8_t* tb, uint64_t kept, unsigned long long gseg, uint32_t x0r, uint32_t vend,
                         unsigned long long g0, uint32_t wtot) -> bool {
    const uint32_t cnt = (uint32_t)__popcll(kept);
    const uint32_t M = __reduce_add_sync(0xffffffffu, cnt);
    if (M > 16u) return false;
    uint32_t* desc = reinterpret_cast<uint32_t*>(ob) + (size_t)warp * lay.wstage_words;
    const uint32_t mb = warp_incl_scan(cnt, OpSum()) - cnt;  // this lane's first match index
    uint32_t i = 0;
    for (uint64_t km = kept; km; km &= km - 1ull, ++i) {
      const uint32_t b = (uint32_t)(__ffsll((long long)km) - 1);
      int k = 0;  // the match's pair (kModeMulti)
      if constexpr (MODE == kModeMulti) k = multi_identify(MT, tb + sb + b, n_all - (gseg + b));
      desc[2 * (mb + i)] = lane * 64u + b;  // start within the region
      desc[2 * (mb + i) + 1] = (uint32_t)(k < 0 ? 0 : k);
    }
    __syncwarp();
    // piece j (lane j <= M): the literal run before match j (after the last match for j = M)
    uint32_t lstart = 0, llen = 0, rlen = 0, pid = 0;
    if (lane <= M) {
      uint32_t st0 = x0r;
      if (lane > 0) {
        const uint32_t pk = desc[2 * (lane - 1) + 1];
        st0 = desc[2 * (lane - 1)] + (MODE == kModeMulti ? (uint32_t)MT.L[pk] : L);
      }
      const uint32_t en = lane < M ? desc[2 * lane] : vend;
      lstart = st0;
      llen = en > st0 ? en - st0 : 0u;
      if (lane < M) {
        pid = desc[2 * lane + 1];
        rlen = MODE == kModeMulti ? (uint32_t)MT.R[pid] : R;
      }
    }
    const uint32_t piece = llen + rlen;
    const uint32_t poff = warp_incl_scan(piece, OpSum()) - piece;
    // the pieces fill exactly the region's slot (the same sum as the threads' lengths);
    // otherwise nothing is written and the launch reports an error
    const bool pieces_ok = __shfl_sync(0xffffffffu, poff + piece, 31) == wtot;
    if (!pieces_ok && lane == 0) set_error(p);
#pragma unroll 1  // (rolled: each piece inlines the four copy loops of warp_emit_literal)
    for (uint32_t jp = 0; pieces_ok && jp <= M; ++jp) {
      const uint32_t ls = __shfl_sync(0xffffffffu, lstart, jp);
      const uint32_t ll = __shfl_sync(0xffffffffu, llen, jp);
      const uint32_t po = __shfl_sync(0xffffffffu, poff, jp);
      if (ll) warp_emit_literal(p.out, tb, g0 + po, ll, warp * 2048u + ls);
      if (jp < M) {
        const uint32_t rl = __shfl_sync(0xffffffffu, rlen, jp);
        const uint32_t pk = __shfl_sync(0xffffffffu, pid, jp);
        const uint8_t* rb = MODE == kModeMulti ? MT.rep[pk] : rs;  // rs: the replacement (and more)
        for (uint32_t q = lane; q < rl; q += 32u) p.out[g0 + po + ll + q] = rb[q];
      }
    }
    __syncwarp();
    return true;
  };

  // look-back, pass B and records of super-tile t, whose pass A filled set `set`; after the
  // look-back, thread 0 schedules past super-tile tnext (set nset) when there is one
  auto tile_back = [&](const uint32_t t, const uint32_t set, const uint32_t tnext, const uint32_t nset) {
    const uint32_t m = subs_in_tile(t, S, n, nsub);
    const unsigned long long tstart = (unsigned long long)t * S;
    uint64_t* const masks_s = masks + (size_t)set * nsub * kThreads;
    uint32_t* const wcnt_s = s_wcnt + set * (kMaxSub * kWarps);
    uint32_t* const wcend_s = s_wcend + set * (kMaxSub * kWarps);
    uint32_t* const sublco_s = s_sub_lco + set * kMaxSub;
    uint8_t* const srec_b = smem + lay.srec + set * lay.srec_set;
    uint8_t* const wtab_b = smem + lay.wtab + set * lay.wtab_set;
    uint8_t* const wrec_b = smem + lay.wrec + set * lay.wrec_set;
    uint8_t* const subrec_b = smem + lay.subrec + set * lay.subrec_set;
    const bool use_rec = kFreeLike || L <= 4u;
    const uint32_t tag = p.epoch & 0xFFFFFFu;
    // ================= look back, publish the inclusive prefix
    if (warp == 0) {
      unsigned long long K = 0;
      uint32_t c = carry0;
      bool ok = true;
      if (t > 0) {
        if (kFreeLike)
          ok = lookback_free_rec(p, t, S, &K, &c, carry0);
        else if (L == 2u)
          ok = lookback_small_rec<2>(p, t, &K, &c, carry0);
        else if (L == 3u)
          ok = lookback_small_rec<3>(p, t, &K, &c, carry0);
        else if (L == 4u)
          ok = lookback_small_rec<4>(p, t, &K, &c, carry0);
        else
          ok = lookback_small(p, t, L, &K, &c, carry0);
      }
      if (!ok) {
        K = 0;
        c = 0;
        if (lane == 0) s_fail = 1;
      }
      unsigned long long Kin;
      uint32_t cout;
      if (kFreeLike) {
        const unsigned long long fcnt = s_frcnt[set];
        const long long flco = s_frlco[set];
        const long long sh = (long long)c - (long long)m * kTile;  // span of this super-tile
        const long long co = sh > flco ? sh : flco;
        Kin = K + fcnt;
        cout = co > 0 ? (uint32_t)co : 0u;
      } else {
        Kin = K + s_supc[set][c];
        cout = s_supx[set][c];
      }
      if (lane == 0) {
        if (use_rec) rec_store(p.rec, t, rec_word(tag, kStInc, Kin), rec_word(tag, kStInc, cout));
        __stcg(&p.incl[t].kept, Kin);
        __stcg(&p.incl[t].carry, cout);
        if (!use_rec) {
          __threadfence();
          st_release_u32(p.status + t, (p.epoch << 2) | kStInc);
        }
        s_kexcl = K;
        s_cin = c;
        s_tcnt = (uint32_t)(Kin - K);
        s_cout = cout;
      }
    }
    __syncthreads();
    if (tid == 0 && tnext != kNone) schedule(tnext, nset);
    const uint32_t pbm = s_noin[set];  // pass B mode
    const bool noin = pbm == 1u;
    const uint32_t cin = s_cin;
    const unsigned long long kexcl = s_kexcl;
    const long long delta = (long long)R - (long long)L;
    // output position in out[]: the output range starts len_bias bytes in, and the carry0
    // leading bytes covered by a match kept before this buffer are not emitted here
    // (kModeMulti: the look-back prefix is sum(R - L) over the earlier matches plus kMultiBias per
    // earlier super-tile)
    const long long dprefix = MODE == kModeMulti ? (long long)kexcl - (long long)t * (long long)kMultiBias
                                                 : (long long)kexcl * delta;
    unsigned long long O =
        p.len_bias + (unsigned long long)((long long)(tstart + cin) - (long long)carry0 + dprefix);
    const bool failed = s_fail != 0;

    // ================= pass B, table-driven: every warp region of this whole super-tile is a run of
    // replacements, empty, or (mode 2) a copy of its input. Mode 2: lane r stands for region
    // r % 8 of sub-tile r / 8: its output length from the tables, a scan over the 32 lanes
    // places it, and each warp writes its region of every sub-tile. The last kept start follows
    // from the regions (kept starts x0, x0 + L, ...).
    uint32_t noin_last1 = 0;
    if (noin) {
      // every region is a run of replacements: the super-tile's output is the replacement
      // repeated s_tcnt times from O, written in eight slices cut at 16-byte boundaries; its
      // last match ends s_cout bytes past the super-tile
      const uint32_t cnt = s_tcnt;
      const uint32_t total = cnt * R;
      noin_last1 = cnt ? m * (uint32_t)kTile + s_cout - L + 1u : 0u;
      const bool fits_t = (O + total <= p.out_cap) && (O <= p.out_cap);
      if (!fits_t && tid == 0) atomicExch(&p.res->overflow_epoch, p.epoch);
      if (fits_t && !failed && total) {
        const unsigned long long end = O + total;
        const unsigned long long s0 =
            warp == 0 ? O : (O + (((unsigned long long)total * warp) >> 3)) & ~15ull;
        const unsigned long long s1 =
            warp == kWarps - 1 ? end : (O + (((unsigned long long)total * (warp + 1u)) >> 3)) & ~15ull;
        const unsigned long long a = s0 > O ? s0 : O, b = s1 < end ? s1 : end;
        if (b > a)
          warp_emit_replace(p.out, reinterpret_cast<const uint4*>(smem + lay.tab16), rs, R, step512, rmag, a,
                            (uint32_t)(b - a), mod_small((uint32_t)(a - O), R, rmag));
      }
      O += total;
    } else if (pbm == 2u) {
      const uint32_t jr = lane >> 3, wr = lane & 7u;
      uint32_t wc = 0, x0 = 0, olen_r = 0, we = 0;
      if (kFreeLike && jr < m) {
        wc = wcnt_s[lane];  // index jr * kWarps + wr
        we = wcend_s[lane];
      }
      uint32_t pre = we;  // kModeFree: max cover end of the earlier regions of the same sub-tile
      if (kFreeLike) {
#pragma unroll
        for (int d = 1; d < 8; d <<= 1) {
          const uint32_t o = __shfl_up_sync(0xffffffffu, pre, d, 8);
          if (wr >= (uint32_t)d) pre = o > pre ? o : pre;
        }
        pre = __shfl_up_sync(0xffffffffu, pre, 1, 8);
      }
      if (jr < m) {
        if (kFreeLike) {
          // carry into sub-tile jr: cin, then the previous sub-tile's reach (L <= 64, so a cover
          // never spans a whole sub-tile)
          const uint32_t csj = jr == 0 ? cin : sublco_s[jr - 1];
          const uint32_t ex = wr == 0 ? 0u : pre;
          const uint32_t covs = csj > ex ? csj : ex;
          const uint32_t wlo = wr * 2048u;
          uint32_t wcov = covs > wlo ? covs - wlo : 0u;
          wcov = wcov < 2048u ? wcov : 2048u;
          const uint32_t over = we > wlo + 2048u ? we - (wlo + 2048u) : 0u;
          olen_r = 2048u - wcov - wc * L + over + wc * R;
          x0 = wcov;
        } else {
          const uint32_t cs = subrec_b[jr * L + cin];
          const uint32_t cw = wrec_b[(jr * kWarps + wr) * L + cs];
          const uint32_t e = (L <= 4u && s_dense[set][lane]) ? dense_region_entry(cw, L)
                                                               : reinterpret_cast<const uint32_t*>(wtab_b)[lane * L + cw];
          wc = e & 0xFFFFu;
          olen_r = 2048u - cw - wc * L + (e >> 16) + wc * R;
          x0 = cw;
        }
      }
      uint32_t incl = olen_r;
#pragma unroll
      for (int d = 1; d < 32; d <<= 1) {
        const uint32_t o = __shfl_up_sync(0xffffffffu, incl, d);
        if (lane >= (uint32_t)d) incl += o;
      }
      const uint32_t total = __shfl_sync(0xffffffffu, incl, 31);
      const uint32_t offr = incl - olen_r;
      // the last kept start: kModeFree, the region's last match ends at its cover end `we`
      // (from the sub-tile start); otherwise the region is a run x0, x0 + L, ...
      noin_last1 = __reduce_max_sync(
          0xffffffffu, wc ? (MODE == kModeFree ? jr * (uint32_t)kTile + we - L + 1u
                                               : jr * (uint32_t)kTile + wr * 2048u + x0 + (wc - 1u) * L + 1u)
                          : 0u);
      // a region not shown by the fold: literal bytes beside kept matches (kModeFree: beside
      // more than 16 of them; fewer are written as pieces)
      const bool odd = __any_sync(0xffffffffu, olen_r != wc * R && wc > (MODE == kModeFree ? 16u : 0u));
      const bool fits_t = (O + total <= p.out_cap) && (O <= p.out_cap);
      if (!fits_t && tid == 0) atomicExch(&p.res->overflow_epoch, p.epoch);
      if (odd && tid == 0) set_error(p);
      const bool write = fits_t && !odd && !failed;
#pragma unroll 1
      for (uint32_t j = 0; j < m; ++j) {
        const uint8_t* tb = ring.wait(p, smem, lay, s_bar, &s_fail);
        const uint32_t r = j * kWarps + warp;
        const uint32_t ol = __shfl_sync(0xffffffffu, olen_r, r);
        const uint32_t of = __shfl_sync(0xffffffffu, offr, r);
        const uint32_t cr = __shfl_sync(0xffffffffu, wc, r);
        const uint32_t xr = __shfl_sync(0xffffffffu, x0, r);
        if (write && ol) {
          if (cr == 0u) {
            warp_emit_literal(p.out, tb, O + of, ol, warp * 2048u + xr);
          } else if (ol == cr * R) {
            warp_emit_replace(p.out, reinterpret_cast<const uint4*>(smem + lay.tab16), rs, R, step512, rmag,
                              O + of, ol);
          } else if constexpr (MODE == kModeFree) {
            // matches beside literal bytes (at most 16, as the fold checked; all kept in free mode)
            emit_pieces(tb, masks_s[j * kThreads + tid], tstart + (unsigned long long)j * kTile + sb, xr, 2048u,
                        O + of, ol);
          }
        }
        __syncthreads();
        ring.release();
        if (tid == 0) ring.issue(p, smem, lay, s_bar, S, n16, want_a, n, nsub);
      }
      O += total;
    }

    // ================= pass B: exact kept starts and output, one warp region at a time
    uint32_t csub = cin;      // kModeFree: carry into sub-tile j
    long long last_abs = -1;  // last kept start seen by this thread
#pragma unroll 1
    for (uint32_t j = 0; j < (pbm != 0u ? 0u : m); ++j) {
      uint8_t* tb = ring.wait(p, smem, lay, s_bar, &s_fail);
      const unsigned long long sstart = tstart + (unsigned long long)j * kTile;
      const unsigned long long gseg = sstart + sb;
      const uint64_t mask = masks_s[j * kThreads + tid];
      // valid input bytes of warp region `lane` (lanes 0..7 stand for the 8 warps)
      const unsigned long long wrs = sstart + (unsigned long long)lane * 2048u;
      const uint32_t wbytes = wrs >= n ? 0u : ((n - wrs) < 2048ull ? (uint32_t)(n - wrs) : 2048u);
      uint32_t x_in = 0, cnt, wolen = 0;
      uint64_t kept;
      uint32_t csub_in = 0, covs_l = 0, ewc = 0, ewcov = 0;  // kModeFree: kept for x_in and the warp paths
      if (kFreeLike) {
        const uint32_t wc = lane < 8u ? wcnt_s[j * kWarps + lane] : 0u;
        const uint32_t we = lane < 8u ? wcend_s[j * kWarps + lane] : 0u;
        const uint32_t pre = lanes8_excl_max(we);  // max cover end of the earlier warps
        const uint32_t covs = csub > pre ? csub : pre;
        const uint32_t wlo = lane * 2048u, whi = wlo + 2048u;
        const uint32_t wcov = covs > wlo ? covs - wlo : 0u;
        const uint32_t over = we > whi ? we - whi : 0u;
        // the region's matches change its length by wc * (R - L), or (kModeMulti) by their sum of R - L
        const uint32_t grow = MODE == kModeMulti
                                  ? (lane < 8u ? (uint32_t)s_wd[set * (kMaxSub * kWarps) + j * kWarps + lane] : 0u)
                                  : wc * R - wc * L;
        wolen = wbytes - (wcov < wbytes ? wcov : wbytes) + over + grow;
        csub_in = csub;
        covs_l = covs;
        ewc = wc;
        ewcov = wcov < wbytes ? wcov : wbytes;
        kept = mask;
        cnt = (uint32_t)__popcll(mask);
        const long long sh = (long long)csub - (long long)kTile;
        const long long lco = (long long)sublco_s[j];
        const long long nx = sh > lco ? sh : lco;
        csub = nx > 0 ? (uint32_t)nx : 0u;
      } else {
        const uint32_t cs = (subrec_b)[j * L + cin];
        const uint8_t* wrec = wrec_b + (size_t)j * kWarps * L;
        const uint32_t* wt = reinterpret_cast<const uint32_t*>(wtab_b) + (size_t)j * kWarps * L;
        uint32_t cw = 0;
        if (lane < 8u) {
          cw = wrec[lane * L + cs];
          const uint32_t e = (L <= 4u && s_dense[set][j * kWarps + lane]) ? dense_region_entry(cw, L) : wt[lane * L + cw];
          const uint32_t wc = e & 0xFFFFu, co = e >> 16;
          wolen = wbytes - (cw < wbytes ? cw : wbytes) - wc * L + co + wc * R;
          ewc = wc;
          ewcov = cw < wbytes ? cw : wbytes;
        }
        covs_l = cw;  // kModeSmall: the carry into each warp region (lanes 0-7)
        kept = 0;
        cnt = 0;
      }
      // ---- L <= 64: a warp whose output is a copy of its input or a run of replacements is
      // written straight from the pass-A tables, with no per-thread walk or scan
      uint32_t wbase = 0, sub_total = 0;
      bool done = false;
      if (L <= 64u) {
        const uint32_t cut0 = __ballot_sync(0xffffffffu, lane < 8u && wbytes != 0u && wbytes < 2048u);
        if (!cut0) {
          lanes8_sum(wolen, &wbase, &sub_total);
          wbase = __shfl_sync(0xffffffffu, wbase, warp);
          sub_total = __shfl_sync(0xffffffffu, sub_total, 7);
          const bool fits0 = (O + sub_total <= p.out_cap) && (O <= p.out_cap);
          const bool stage0 =
              __reduce_max_sync(0xffffffffu, lane < 8u ? wolen : 0u) + 15u <= lay.wstage_cap;
          const uint32_t wcw = __shfl_sync(0xffffffffu, ewc, warp);
          const uint32_t wlw = __shfl_sync(0xffffffffu, wolen, warp);
          const uint32_t x0w = __shfl_sync(0xffffffffu, ewcov, warp);  // bytes covered at the region start
          // copy only (no kept start), nothing to write (all covered, R = 0), or replacements only
          const bool table_only = stage0 && (wcw == 0u || wlw == 0u || (rep_table && wlw == wcw * R));
          if (table_only) {
            // the last kept start, from the tables (also when nothing is written below)
            if (kFreeLike) {
              if (mask) last_abs = (long long)(gseg + (63u - (uint32_t)__clzll((long long)mask)));
            } else if (wcw != 0u && lane == 0) {
              // a region with no literal byte: its kept starts are cw, cw + L, ... (the block
              // maximum over threads of the last kept start needs only the warp's last one)
              last_abs = (long long)(sstart + warp * 2048u + x0w + (unsigned long long)(wcw - 1u) * L);
            }
          }
          if (fits0 && !failed && table_only) {
            done = true;  // the same in every lane of the warp
            if (wlw) {
              if (wcw == 0u)
                warp_emit_literal(p.out, tb, O + wbase, wlw, warp * 2048u + x0w);
              else
                warp_emit_replace(p.out, reinterpret_cast<const uint4*>(smem + lay.tab16), rs, R, step512,
                                  rmag, O + wbase, wlw);
            }
          }
        }
      }
      uint32_t tinf = 0;  // kModeMulti: this thread's (sum of R - L, last match end)
      if (!done) {
      if constexpr (MODE == kModeMulti) {
        // this thread's matches again (the pattern at each kept start): the sum of their R - L and
        // where the last one ends; the carry into the segment is the previous thread's last match
        // (L <= 32), or for a warp's first thread the carry into its region
        int dsum = 0;
        uint32_t le = 0;
        for (uint64_t km = kept; km; km &= km - 1ull) {
          const uint32_t b = (uint32_t)(__ffsll((long long)km) - 1);
          const int k = multi_identify(MT, tb + sb + b, n_all - (gseg + b));
          if (k >= 0) {
            dsum += (int)MT.R[k] - (int)MT.L[k];
            le = b + MT.L[k];
          }
        }
        tinf = ((uint32_t)dsum & 0xFFFFu) | (le << 16);
        const uint32_t prev_le = __shfl_up_sync(0xffffffffu, le, 1);
        const uint32_t pw = __shfl_sync(0xffffffffu, covs_l, warp);
        x_in = lane == 0 ? (pw > sb ? pw - sb : 0u) : (prev_le > 64u ? prev_le - 64u : 0u);
      } else if (MODE == kModeFree) {
        if (L <= 64u) {
          // only the previous segment's last match (or the sub-tile carry) can reach here
          uint32_t cov = tid == 0 ? csub_in : 0u;
          if (tid > 0) {
            const uint64_t pm = masks_s[j * kThreads + tid - 1];
            if (pm) {
              const uint32_t e = 63u - (uint32_t)__clzll((long long)pm) + L;
              if (e > 64u && e - 64u > cov) cov = e - 64u;
            }
          }
          x_in = cov;
        } else {
          uint32_t ce = mask ? sb + (63u - (uint32_t)__clzll((long long)mask)) + L : 0u;
#pragma unroll
          for (int d = 1; d < 32; d <<= 1) {
            const uint32_t o = __shfl_up_sync(0xffffffffu, ce, d);
            if (lane >= (uint32_t)d) ce = o > ce ? o : ce;
          }
          uint32_t prev = __shfl_up_sync(0xffffffffu, ce, 1);
          if (lane == 0) prev = 0;
          const uint32_t pw = __shfl_sync(0xffffffffu, covs_l, warp);
          const uint32_t cv = prev > pw ? prev : pw;
          x_in = cv > sb ? cv - sb : 0u;
        }
      } else {
        const uint32_t mycw = __shfl_sync(0xffffffffu, covs_l, warp);
        x_in = (L <= 4u && s_dense[set][j * kWarps + warp]) ? dense_seg_carry(mycw, lane * 64u, L)
                                                            : (srec_b)[((size_t)j * kThreads + tid) * L + mycw];
        if (x_in < 64u) {
          const Walk w = seg_walk(mask, x_in, L, p.inv_l, p.stride_mask);
          kept = w.kept;
          cnt = w.cnt;
        }
      }
      const uint32_t V = gseg >= n ? 0u : ((n - gseg) < 64ull ? (uint32_t)(n - gseg) : 64u);
      uint32_t covered = x_in < V ? x_in : V;
      uint32_t olen;
      if constexpr (MODE == kModeMulti) {
        // literal bytes V - x_in - sum(L) + (what the last match covers past V), plus sum(R)
        const int dthr = (int)(int16_t)(tinf & 0xFFFFu);
        const uint32_t le = tinf >> 16;
        const uint32_t over = (cnt && le > V) ? le - V : 0u;
        if (cnt) last_abs = (long long)(gseg + (63u - (uint32_t)__clzll((long long)kept)));
        olen = (uint32_t)((int)(V - covered + over) + dthr);
      } else {
        if (cnt) {
          const uint32_t lastk = 63u - (uint32_t)__clzll((long long)kept);
          const uint32_t over = (lastk + L > V) ? lastk + L - V : 0u;
          covered += cnt * L - over;
          last_abs = (long long)(gseg + lastk);
        }
        olen = V - covered + cnt * R;
      }
      uint32_t toff = warp_incl_scan(olen, OpSum());
      const uint32_t wtot = __shfl_sync(0xffffffffu, toff, 31);
      toff -= olen;  // exclusive offset inside the warp region

      // The warp region that holds the end n of the output range is cut short. When input is
      // held back past n, a match kept there may run beyond n, which the region functions
      // (built over whole 2048-byte regions) do not see; the region's exact length is the sum
      // over its threads. At most one sub-tile per launch has such a region; `cut` is the
      // same in every warp (all compute the eight regions' lengths), so the barrier is uniform.
      const uint32_t cut = __ballot_sync(0xffffffffu, lane < 8u && wbytes != 0u && wbytes < 2048u);
      if (cut) {
        const uint32_t cw = (uint32_t)__ffs(cut) - 1u;
        if (warp == cw && lane == 0) s_cutlen = wtot;
        __syncthreads();
        if (lane == cw) wolen = s_cutlen;
      }
      lanes8_sum(wolen, &wbase, &sub_total);
      wbase = __shfl_sync(0xffffffffu, wbase, warp);
      sub_total = __shfl_sync(0xffffffffu, sub_total, 7);

      const bool fits = (O + sub_total <= p.out_cap) && (O <= p.out_cap);
      // every warp's output of this sub-tile fits its staging area (with the up to 15 bytes of
      // alignment in front): the warp paths; otherwise the whole block writes windows. Lanes
      // 0-7 of every warp hold the eight lengths, so the choice is the same in every warp.
      const bool warp_stage = __reduce_max_sync(0xffffffffu, lane < 8u ? wolen : 0u) + 15u <= lay.wstage_cap;
      if (!fits && tid == 0) atomicExch(&p.res->overflow_epoch, p.epoch);
      // kModeMulti: the warp's own sum of its threads' lengths must equal the length its slot was
      // given from the pass-A sums, or it would write over its neighbour; a mismatch (which the
      // arithmetic rules out) is reported as an error and the warp writes nothing. The same in
      // every lane of the warp; the branches below keep their block-uniform choice regardless.
      bool len_ok = true;
      if (MODE == kModeMulti) {
        len_ok = __shfl_sync(0xffffffffu, wolen, warp) == wtot;
        if (!len_ok && lane == 0) set_error(p);
      }
      // warp output mode: no kept match in the warp (a copy of its input), or no literal byte
      // (a run of replacements), or mixed
      const uint32_t notlit = __ballot_sync(0xffffffffu, cnt != 0u || (lane > 0u && x_in != 0u));
      const uint32_t notrep = __ballot_sync(0xffffffffu, olen != cnt * R);
      if (fits && !failed && warp_stage && wtot != 0u && (notlit == 0u || (notrep == 0u && rep_table))) {
        if (!len_ok) {
        } else if (notlit == 0u) {
          // ---- LITERAL: output = input bytes [warp start + x0, ...)
          warp_emit_literal(p.out, tb, O + wbase, wtot, warp * 2048u + __shfl_sync(0xffffffffu, x_in, 0));
        } else {
          // ---- REPLACE: output = the replacement repeated
          warp_emit_replace(p.out, reinterpret_cast<const uint4*>(smem + lay.tab16), rs, R, step512, rmag, O + wbase,
                            wtot);
        }
      } else if (fits && !failed && warp_stage) {
        if (len_ok) {
        bool pieces_done = false;
        if constexpr (kFreeLike) {
          // few matches in the region: literal runs between replacements
          pieces_done = emit_pieces(tb, kept, gseg, __shfl_sync(0xffffffffu, x_in, 0),
                                    __reduce_add_sync(0xffffffffu, V), O + wbase, wtot);
        }
        if (!pieces_done) {
        uint32_t W[17];
        load_seg_words(tb + sb, W);
        // ---- this warp's output: assemble in its padded staging area, then copy out
        uint32_t* stg = reinterpret_cast<uint32_t*>(ob) + (size_t)warp * lay.wstage_words;
        uint8_t* sbytes = reinterpret_cast<uint8_t*>(stg);
        const unsigned long long g0 = O + wbase;
        const unsigned long long ga = g0 & ~15ull;
        const uint32_t cur = (uint32_t)(g0 - ga) + toff;
        if (olen && kept == 0 && x_in == 0 && V == 64u) {
          // literal-only segment: its 64 input bytes, shifted to the output word grid
          const uint32_t d = (4u - (cur & 3u)) & 3u;
          for (uint32_t i = 0; i < d; ++i) {
            const uint32_t b = cur + i;
            sbytes[stg_pad(b >> 2) * 4u + (b & 3u)] = (uint8_t)(W[0] >> (8u * i));
          }
          const uint32_t wb = (cur + d) >> 2;
          if (d == 0) {
#pragma unroll
            for (int k = 0; k < 16; ++k) stg[stg_pad(wb + k)] = W[k];
          } else {
#pragma unroll
            for (int k = 0; k < 15; ++k) stg[stg_pad(wb + k)] = __funnelshift_r(W[k], W[k + 1], 8u * d);
            for (uint32_t i = d + 60u; i < 64u; ++i) {
              const uint32_t b = cur + i;
              sbytes[stg_pad(b >> 2) * 4u + (b & 3u)] = (uint8_t)(W[15] >> (8u * (i & 3u)));
            }
          }
        } else if (olen) {
          Emitter e;
          e.init(stg, cur);
          const uint8_t* src = tb + sb;
          uint32_t pos = x_in < V ? x_in : V;
          while (pos < V) {
            const uint64_t km = pos < 64u ? (kept >> pos) : 0ull;
            uint32_t nk = km ? pos + (uint32_t)(__ffsll((long long)km) - 1) : V;
            if (nk > V) nk = V;
            if (nk > pos) emit_literal(e, src + pos, nk - pos);
            if (nk >= V) break;
            if constexpr (MODE == kModeMulti) {  // this match's own replacement
              const int k = multi_identify(MT, src + nk, n_all - (gseg + nk));
              if (k < 0) break;  // cannot happen: pass A found this pattern here
              emit_literal(e, MT.rep[k], MT.R[k]);
              pos = nk + MT.L[k];
              continue;
            }
            uint32_t r = 1;  // kept starts nk, nk+L, ... with nothing literal between them
            if (L < 64u) {
              const uint64_t holes = p.stride_mask & ~(kept >> nk);
              const uint32_t h = holes ? (uint32_t)(__ffsll((long long)holes) - 1) : 64u;
              r = ((h + L - 1) * p.inv_l) >> 16;
            }
            if (R) emit_repeat(e, rs, R, step4, r);
            pos = nk + r * L;
          }
          e.finish();
        }
        __syncwarp();
        // coalesced 16-byte stores for the whole chunks; the partial chunks at both ends of
        // the region one byte per lane (the neighbouring regions own their other bytes)
        const unsigned long long gend = g0 + wtot;
        const uint32_t c0 = (uint32_t)((g0 - ga + 15ull) >> 4);  // first whole chunk
        const uint32_t c1 = (uint32_t)((gend - ga) >> 4);        // end of the whole chunks
        for (uint32_t c = c0 + lane; c < c1; c += 32u) {
          const uint32_t w = c << 2;
          uint4 v;
          v.x = stg[stg_pad(w)];
          v.y = stg[stg_pad(w + 1)];
          v.z = stg[stg_pad(w + 2)];
          v.w = stg[stg_pad(w + 3)];
          st_out16(p.out + ga + ((unsigned long long)c << 4), v);
        }
        {
          // head bytes [g0, ga + 16*c0) on lanes 0-15, tail bytes [ga + 16*c1, gend) on 16-31;
          // with no whole chunk, the region (< 32 bytes) is covered by all 32 lanes
          unsigned long long b;
          bool ok;
          if (c0 < c1) {
            b = lane < 16u ? g0 + lane : ga + ((unsigned long long)c1 << 4) + (lane - 16u);
            ok = lane < 16u ? (b < ga + ((unsigned long long)c0 << 4)) : (b < gend);
          } else {
            b = g0 + lane;
            ok = b < gend;
          }
          if (ok) {
            const uint32_t sbi = (uint32_t)(b - ga);
            p.out[b] = sbytes[stg_pad(sbi >> 2) * 4u + (sbi & 3u)];
          }
        }
        }  // !pieces_done
        }  // len_ok
      } else if (fits && !failed) {
        // very large expansions: windows of the sub-tile output, byte by byte (the windows
        // share the staging area with the warps' own staging, which the block barrier at the
        // end of every sub-tile keeps apart)
        const uint32_t ooff = wbase + toff;
        const uint32_t sub_olen = sub_total;
        for (uint32_t w0 = 0; w0 < sub_olen; w0 += kOutWin) {
          const uint32_t w1 = (w0 + kOutWin) < sub_olen ? (w0 + kOutWin) : sub_olen;
          const unsigned long long g0 = O + w0;
          const uint32_t sh = (uint32_t)(g0 & 15ull);
          uint8_t* obw = ob + sh;
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
              if constexpr (MODE == kModeMulti) {  // this match's own replacement
                const int k = multi_identify(MT, src + nk, n_all - (gseg + nk));
                if (k < 0) break;  // cannot happen: pass A found this pattern here
                copy_clip(obw, o, MT.rep[k], MT.R[k], w0, w1);
                o += MT.R[k];
                pos = nk + MT.L[k];
                continue;
              }
              copy_clip(obw, o, rs, R, w0, w1);
              o += R;
              pos = nk + L;
            }
          }
          fence_proxy_async_smem();
          __syncthreads();
          const unsigned long long gend = O + w1;
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
      }  // !done
      O += sub_total;
      __syncthreads();
      ring.release();
      if (tid == 0) ring.issue(p, smem, lay, s_bar, S, n16, want_a, n, nsub);
    }

    // ================= per-super-tile records: last kept start, totals
    {
      const uint32_t last1 = last_abs >= 0 ? (uint32_t)((unsigned long long)last_abs - tstart + 1) : 0u;
      uint32_t tot_last1 = noin_last1;  // table-driven: the same in every thread already
      if (pbm == 0u) (void)block_excl_scan1(last1, 0u, OpMax(), s_scan2[nscan++ & 1u], &tot_last1);
      if (tid == 0) {
        const long long lastt = tot_last1 ? (long long)(tstart + tot_last1 - 1) : -1ll;
        __stcg(p.tile_last + t, lastt);
        if (lastt >= 0)
          atomicMax(&p.res->last_tagged, ((unsigned long long)p.epoch << 40) | (unsigned long long)(lastt + 1));
        if (t == NT - 1) {
          p.res->out_len = O - p.len_bias;
          // (kModeMulti: the look-back sums are not match counts; no count is reported)
          p.res->kept = MODE == kModeMulti ? 0ull : __ldcg(&p.incl[t].kept);
          if (p.len_out) *p.len_out = O;
          if (MODE != kModeMulti && p.carry_out) {
            // coverage past the output range n: by the last kept match, or by the carry into
            // this super-tile when no match starts in it
            unsigned long long e = tstart + cin;
            if (lastt >= 0 && (unsigned long long)lastt + L > e) e = (unsigned long long)lastt + L;
            *p.carry_out = e > n ? (unsigned int)(e - n) : 0u;
          }
        }
      }
    }
  };

  if (tid == 0) {
    for (int b = 0; b < kNBuf; ++b) mbar_init(&s_bar[b], 1);
    fence_mbar_init();
    s_fail = 0;
    if (SEG) {
      s_jobid = kNone;
      s_newjob = 0;
      s_q[0] = seg_claim(sl, s_job, &s_jobid, &s_newjob);
      if (s_q[0] != kNone) {
        const JobDims d = job_dims(p, S);
        ring.push(s_q[0], 0);
        ring.push(s_q[0], 1);
        ring.issue(p, smem, lay, s_bar, S, d.n16, d.want_a, d.n, nsub);
      }
    } else {
      const uint32_t first = atomicAdd(sched, 1u);
      s_q[0] = first < NT ? first : kNone;
      if (s_q[0] != kNone) {
        ring.push(s_q[0], 0);
        ring.issue(p, smem, lay, s_bar, S, n16, want_a, n, nsub);
      }
    }
  }

  if (SEG) {
    // segmented launch: one super-tile at a time (the job, and its pattern, may change)
    for (;;) {
      __syncthreads();
      const uint32_t t = s_q[0];
      if (t == kNone) break;
      if (s_newjob) {  // a super-tile of another job: its dimensions and pattern
        setup_job();
        __syncthreads();
        if (tid == 0) s_newjob = 0;
      }
      tile_front(t, 0);
      __syncthreads();  // the fold (warp 1) is done before this super-tile's look-back (warp 0)
      tile_back(t, 0, kNone, 0);
      // claim the next super-tile only now, when its pass A starts: a super-tile claimed
      // early but started late would hold up the look-back of every later super-tile
      if (tid == 0) {
        s_fail = 0;
        s_q[0] = seg_claim(sl, s_job, &s_jobid, &s_newjob);
        if (s_q[0] != kNone) {
          const JobDims d = job_dims(p, S);
          ring.push(s_q[0], 0);
          ring.push(s_q[0], 1);
          ring.issue(p, smem, lay, s_bar, S, d.n16, d.want_a, d.n, nsub);
        }
      }
    }
  } else {
    // one apply: pass A of super-tile k runs while super-tile k-1's predecessors publish
    // their records; then k-1 looks back (its wait mostly over) and writes its output. The
    // next super-tile is claimed right after that look-back, so its pass-A loads stream in
    // during k-1's pass B, and it still publishes its aggregate without waiting on another CTA.
    uint32_t tprev = kNone, k = 0;
    for (;;) {
      __syncthreads();
      const uint32_t tcur = s_q[0];
      if (tcur == kNone && tprev == kNone) break;
      if (tcur != kNone) tile_front(tcur, k & 1u);
      if (tprev != kNone) {
        tile_back(tprev, (k & 1u) ^ 1u, tcur, k & 1u);
      } else if (tcur != kNone) {
        __syncthreads();  // the fold's flags of tcur are visible to thread 0
        if (tid == 0) schedule(tcur, k & 1u);
      }
      tprev = tcur;
      ++k;
    }
  }

  if (tid == 0) {
    bulk_wait_all();
    __threadfence();
    const unsigned int d = atomicAdd(sched + 1, 1u);
    if (d == gridDim.x - 1) {
      atomicExch(sched, 0u);
      atomicExch(sched + 1, 0u);
      __threadfence();
    }
  }
}

// One CTA answers query_prefix for a super-tile layout: kept starts before limit and the
// last one, re-deriving the kept starts of the super-tile that holds limit from its exact
// carry-in (the predecessor's inclusive prefix) and searching earlier super-tiles' records.
template <int MODE>
__global__ void __launch_bounds__(kThreads) query_super_kernel(const __grid_constant__ ReplaceParams p) {
  extern __shared__ __align__(128) uint8_t smem[];
  __shared__ __align__(8) uint64_t s_bar;
  __shared__ uint32_t s_scan[kWarps];
  __shared__ uint32_t s_x;
  __shared__ unsigned long long s_k;
  __shared__ long long s_last;
  __shared__ uint32_t s_ok;
  const uint32_t L = p.L;
  const LayoutS lay = make_layout_s(kModeFree, L, p.R, 1);
  uint8_t* tb = smem + lay.in0;
  uint8_t* ps = smem + lay.pat;
  uint64_t* masks = reinterpret_cast<uint64_t*>(smem + lay.masks);
  const uint32_t tid = threadIdx.x, sb = tid * kSeg;
  const unsigned long long n = p.n, n16 = (n + 15ull) & ~15ull;
  const unsigned long long S = (unsigned long long)p.nsub * kTile;
  const unsigned long long limit = p.query_limit64;
  const uint32_t t = (uint32_t)(limit / S);
  const unsigned long long rel = limit - (unsigned long long)t * S;
  {
    const uint8_t* psrc = L <= (uint32_t)kInlineMax ? p.pat : p.pat_ext;
    for (uint32_t i = tid; i < L; i += kThreads) ps[i] = psrc[i];
  }
  if (tid == 0) {
    mbar_init(&s_bar, 1);
    fence_mbar_init();
    s_ok = 1;
    s_k = t > 0 ? __ldcg(&p.incl[t - 1].kept) : 0ull;
    s_x = t > 0 ? __ldcg(&p.incl[t - 1].carry) : 0u;
    s_last = -1;
  }
  __syncthreads();
  uint32_t phase = 0;
  for (uint32_t j = 0; (unsigned long long)j * kTile < rel; ++j) {
    const unsigned long long sstart = (unsigned long long)t * S + (unsigned long long)j * kTile;
    if (tid == 0) {
      const uint32_t want = align_up_u32(kTile + (L > 1 ? L - 1 : 0), 16);
      const unsigned long long avail = n16 - sstart;
      const uint32_t bytes = avail < want ? (uint32_t)avail : want;
      fence_proxy_async_smem();
      mbar_arrive_expect_tx(&s_bar, bytes);
      bulk_load(tb, p.in + sstart, bytes, &s_bar);
    }
    if (!wait_tile(&s_bar, phase) && tid == 0) s_ok = 0;
    phase ^= 1u;
    const unsigned long long gseg = sstart + sb;
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
      const unsigned long long lim = rel - (unsigned long long)j * kTile;  // limit relative to this sub-tile
      uint32_t x = s_x;
      unsigned long long K = s_k;
      long long last = s_last;
      for (uint32_t seg = 0; seg < (uint32_t)kThreads; ++seg) {
        const unsigned long long base = (unsigned long long)seg * 64u;
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
        if (base < lim) {
          const uint64_t kb = kept & low_bits(lim - base < 64ull ? (uint32_t)(lim - base) : 64u);
          K += (unsigned long long)__popcll(kb);
          if (kb) last = (long long)(sstart + base + 63u - (uint32_t)__clzll((long long)kb));
        }
        x = xn;
      }
      s_x = x;
      s_k = K;
      s_last = last;
    }
    __syncthreads();
  }
  // last kept start in earlier super-tiles when none was found in this one
  uint32_t best_hi = 0, best_lo = 0;
  if (s_last < 0) {
    for (uint32_t i = tid; i < t; i += kThreads) {
      const long long v = __ldcg(p.tile_last + i);
      const unsigned long long u = (unsigned long long)(v + 1);
      const uint32_t hi = (uint32_t)(u >> 32), lo = (uint32_t)u;
      if (hi > best_hi || (hi == best_hi && lo > best_lo)) {
        best_hi = hi;
        best_lo = lo;
      }
    }
  }
  uint32_t tot_hi;
  (void)block_excl_scan(best_hi, 0u, OpMax(), s_scan, &tot_hi);
  uint32_t tot_lo;
  (void)block_excl_scan(best_hi == tot_hi ? best_lo : 0u, 0u, OpMax(), s_scan, &tot_lo);
  if (tid == 0) {
    long long last = s_last;
    if (last < 0) last = (long long)(((unsigned long long)tot_hi << 32) | tot_lo) - 1;
    p.res->q_kept = s_k;
    p.res->q_last = last;
    if (!s_ok) set_error(p);
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
// A single apply holds two super-tiles' tables at once (pass A of one overlaps the previous
// one's look-back), so its super-tiles are 4 sub-tiles (64 KiB): three CTAs still fit an SM.
constexpr uint32_t kApplySub = 4;

uint32_t super_nsub(uint32_t mode, uint32_t L) {
  if (mode == kModeFree) return kApplySub;
  if (mode == kModeSmall && L >= 2 && L <= 32) {
    const uint32_t by_rec = 128u / L;  // keep the per-segment carry records within 32 KiB
    return by_rec < kApplySub ? (by_rec ? by_rec : 1u) : kApplySub;
  }
  return 0;
}

namespace {
template <int MODE>
cudaError_t launch_super_mode(const ReplaceParams& p, cudaStream_t st, int* grid_out) {
  static std::mutex mu;
  static unsigned long long attr_dev_mask = 0;
  const uint32_t smem = make_layout_s(MODE, p.L, p.R, p.nsub, 0u, 2u).total;  // two sets of tables
  int dev = 0;
  cudaGetDevice(&dev);
  {
    std::lock_guard<std::mutex> g(mu);
    if (!(attr_dev_mask & (1ull << (dev & 63)))) {
      cudaError_t e = cudaFuncSetAttribute(replace_super_kernel<MODE, false>,
                                           cudaFuncAttributeMaxDynamicSharedMemorySize, 220 * 1024);
      if (e != cudaSuccess) return e;
      e = cudaFuncSetAttribute(query_super_kernel<MODE>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                               200 * 1024);
      if (e != cudaSuccess) return e;
      attr_dev_mask |= 1ull << (dev & 63);
    }
  }
  int per_sm = 0;
  cudaError_t e = cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, replace_super_kernel<MODE, false>,
                                                                kThreads, smem);
  if (e != cudaSuccess) return e;
  if (per_sm < 1) per_sm = 1;
  long long grid = (long long)per_sm * device_sm_count();
  if (grid > (long long)p.num_tiles) grid = p.num_tiles;
  if (grid < 1) grid = 1;
  replace_super_kernel<MODE, false><<<(unsigned)grid, kThreads, smem, st>>>(p, SegLaunch{});
  if (grid_out) *grid_out = (int)grid;
  return cudaGetLastError();
}
}  // namespace

cudaError_t launch_replace_super(const ReplaceParams& p, cudaStream_t st, int* grid_ctas_out) {
  if (p.mode == kModeFree) return launch_super_mode<kModeFree>(p, st, grid_ctas_out);
  return launch_super_mode<kModeSmall>(p, st, grid_ctas_out);
}

cudaError_t launch_query_super(const ReplaceParams& p, cudaStream_t st) {
  const uint32_t smem = make_layout_s(kModeFree, p.L, p.R, 1).total;
  if (p.mode == kModeFree)
    query_super_kernel<kModeFree><<<1, kThreads, smem, st>>>(p);
  else
    query_super_kernel<kModeSmall><<<1, kThreads, smem, st>>>(p);
  return cudaGetLastError();
}


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

cudaError_t launch_move_tail(const uint8_t* buf, const unsigned long long* total, unsigned long long cap,
                             uint32_t P, uint8_t* dst, cudaStream_t st) {
  move_tail_kernel<<<1, 256, 0, st>>>(buf, total, cap, P, dst);
  return cudaGetLastError();
}

uint32_t seg_smem_bytes(const SegLaunch& sl) { return make_layout_s(sl.mode, sl.Lmax, sl.Rmax, sl.nsub, 3u).total; }

namespace {
template <int MODE>
int seg_occupancy(uint32_t smem) {
  static std::mutex mu;
  static unsigned long long attr_dev_mask = 0;
  int dev = 0;
  cudaGetDevice(&dev);
  {
    std::lock_guard<std::mutex> g(mu);
    if (!(attr_dev_mask & (1ull << (dev & 63)))) {
      if (cudaFuncSetAttribute(replace_super_kernel<MODE, true>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                               220 * 1024) != cudaSuccess)
        return -1;
      attr_dev_mask |= 1ull << (dev & 63);
    }
  }
  int per_sm = 0;
  if (cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, replace_super_kernel<MODE, true>, kThreads, smem) !=
      cudaSuccess)
    return -1;
  return per_sm < 1 ? 1 : per_sm;
}
}  // namespace

int seg_ctas_per_sm(const SegLaunch& sl) {
  const uint32_t smem = seg_smem_bytes(sl);
  return sl.mode == kModeFree ? seg_occupancy<kModeFree>(smem) : seg_occupancy<kModeSmall>(smem);
}

cudaError_t launch_seg(const SegLaunch& sl, cudaStream_t st, int grid_ctas) {
  if (sl.mode != kModeFree && sl.mode != kModeSmall) return cudaErrorInvalidValue;
  if (sl.Lmax > kSegMaxL || sl.Rmax > kSegMaxR || sl.nsub < 1 || sl.nsub > (uint32_t)kMaxSub)
    return cudaErrorInvalidValue;
  if (sl.mode == kModeSmall && sl.nsub * sl.Lmax > 128u) return cudaErrorInvalidValue;
  const uint32_t smem = seg_smem_bytes(sl);
  int grid = grid_ctas;
  if (grid <= 0) {  // (a caller that passes the grid has called seg_ctas_per_sm for this mode before)
    const int per_sm = seg_ctas_per_sm(sl);
    if (per_sm < 0) return cudaErrorUnknown;
    grid = per_sm * device_sm_count();
  }
  seg_plan_kernel<<<1, 1024, 0, st>>>(sl);
  cudaError_t e = cudaGetLastError();
  if (e != cudaSuccess) return e;
  if (sl.mode == kModeFree)
    replace_super_kernel<kModeFree, true><<<(unsigned)grid, kThreads, smem, st>>>(ReplaceParams{}, sl);
  else
    replace_super_kernel<kModeSmall, true><<<(unsigned)grid, kThreads, smem, st>>>(ReplaceParams{}, sl);
  return cudaGetLastError();
}

bool make_seg_pair(SegPair& q, const uint8_t* pat, uint32_t L, const uint8_t* rep, uint32_t R) {
  if (L < 1 || L > kSegMaxL || R > kSegMaxR) return false;
  ReplaceParams p;
  memset(&p, 0, sizeof(p));
  prepare_pattern_fields(p, pat, L);
  if (p.mode != kModeFree && p.mode != kModeSmall) return false;
  if (p.mode == kModeSmall && super_nsub(p.mode, L) == 0) return false;
  memset(&q, 0, sizeof(q));
  q.stride_mask = p.stride_mask;
  q.L = L;
  q.R = R;
  q.mode = p.mode;
  q.p4 = p.p4;
  q.m4 = p.m4;
  q.inv_l = p.inv_l;
  q.agg_entries = p.agg_entries;
  memcpy(q.pat, pat, L);
  if (R) memcpy(q.rep, rep, R);
  return true;
}

cudaError_t launch_presence(const uint8_t* in, unsigned long long n, uint32_t shift, uint32_t* masks,
                            cudaStream_t st) {
  if (n == 0) return cudaSuccess;
  const unsigned long long chunks = (n + (1ull << shift) - 1) >> shift;
  if (chunks > 0x7FFFFFFFull || shift < 14) return cudaErrorInvalidValue;
  presence_kernel<<<(unsigned)chunks, 256, 0, st>>>(in, n, shift, masks);
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

// ---------------------------------------------------------------- multi-pattern stages
namespace {

bool bytes_equal(const uint8_t* a, const uint8_t* b, uint32_t n) { return n == 0 || std::memcmp(a, b, n) == 0; }

// Can an occurrence of a and an occurrence of b (different pairs, or the same pattern at two
// positions) overlap in some text? Yes when they are equal (two pairs with one pattern), when
// one lies inside the other, or when a proper suffix of one is a proper prefix of the other
// (for a == b alone: a proper border).
bool may_overlap(const uint8_t* a, uint32_t La, const uint8_t* b, uint32_t Lb, bool same_pair) {
  if (!same_pair && La == Lb && bytes_equal(a, b, La)) return true;
  if (!same_pair) {
    if (Lb < La)
      for (uint32_t o = 0; o + Lb <= La; ++o)
        if (bytes_equal(a + o, b, Lb)) return true;
    if (La < Lb)
      for (uint32_t o = 0; o + La <= Lb; ++o)
        if (bytes_equal(b + o, a, La)) return true;
  }
  const uint32_t m = La < Lb ? La : Lb;
  for (uint32_t k = 1; k < m; ++k) {
    if (bytes_equal(a + (La - k), b, k)) return true;
    if (bytes_equal(b + (Lb - k), a, k)) return true;
  }
  return false;
}

// Can replacement r (of an earlier pair), with whatever bytes surround it, form an occurrence of
// pattern p (of a later pair) that overlaps it? An occurrence that includes no byte of r lay
// entirely before or after it, so it was there before the replacement; one that overlaps r
// must agree with r wherever they overlap. An empty r joins its two neighbours, which any
// pattern of two bytes or more may straddle.
bool may_create(const uint8_t* r, uint32_t R, const uint8_t* p, uint32_t L) {
  if (R == 0) return L >= 2;
  for (int d = -(int)L + 1; d < (int)R; ++d) {  // p starts d bytes after r starts
    bool ok = true;
    for (uint32_t k = 0; k < L && ok; ++k) {
      const int i = d + (int)k;
      if (i >= 0 && i < (int)R && p[k] != r[i]) ok = false;
    }
    if (ok) return true;
  }
  return false;
}

bool multi_eligible(const uint8_t* pat, int L, int R) {
  return L >= 1 && L <= (int)kMultiMaxL && R >= 0 && R <= (int)kMultiMaxR && pat != nullptr &&
         !may_overlap(pat, (uint32_t)L, pat, (uint32_t)L, true);
}

}  // namespace

int plan_stages(const uint8_t* const* pats, const int* pat_lens, const uint8_t* const* reps,
                const int* rep_lens, int count, bool keep_last_alone, int* stage_of) {
  int stage = -1, first = 0;  // current stage and its first pair
  uint32_t firsts[kMultiMaxFirst];
  uint32_t nfirst = 0;
  bool open = false;  // the current stage can take more pairs
  for (int k = 0; k < count; ++k) {
    const int L = pat_lens[k], R = rep_lens[k];
    const bool elig = multi_eligible(pats[k], L, R) && !(keep_last_alone && k == count - 1);
    bool join = open && elig && (k - first) < (int)kMultiMaxPairs;
    if (join) {
      const uint32_t b0 = pats[k][0];
      bool known = false;
      for (uint32_t f = 0; f < nfirst; ++f) known = known || firsts[f] == b0;
      if (!known && nfirst == kMultiMaxFirst) join = false;
      for (int i = first; i < k && join; ++i) {
        if (may_overlap(pats[i], (uint32_t)pat_lens[i], pats[k], (uint32_t)L, false) ||
            may_create(reps[i], (uint32_t)rep_lens[i], pats[k], (uint32_t)L))
          join = false;
      }
      if (join && !known) firsts[nfirst++] = b0;
    }
    if (!join) {
      ++stage;
      first = k;
      open = elig;
      nfirst = 0;
      if (elig) firsts[nfirst++] = pats[k][0];
    }
    stage_of[k] = stage;
  }
  return stage + 1;
}

void build_multi_table(MultiTable& T, const uint8_t* const* pats, const int* pat_lens, const uint8_t* const* reps,
                       const int* rep_lens, int count) {
  std::memset(&T, 0, sizeof(T));
  T.npairs = (uint32_t)count;
  T.Lmin = ~0u;
  uint32_t ratio = 1;
  for (int k = 0; k < count; ++k) {
    const uint32_t L = (uint32_t)pat_lens[k], R = (uint32_t)rep_lens[k];
    T.L[k] = (uint8_t)L;
    T.R[k] = (uint8_t)R;
    T.Lmin = L < T.Lmin ? L : T.Lmin;
    T.Lmax = L > T.Lmax ? L : T.Lmax;
    std::memcpy(T.pat[k], pats[k], L);
    if (R) std::memcpy(T.rep[k], reps[k], R);
    for (uint32_t i = 0; i < 4 && i < L; ++i) {
      T.p4[k] |= (uint32_t)pats[k][i] << (8 * i);
      T.m4[k] |= 0xFFu << (8 * i);
    }
    const uint32_t b0 = pats[k][0];
    bool known = false;
    for (uint32_t f = 0; f < T.nfirst; ++f) known = known || ((T.firsts >> (8 * f)) & 0xFFu) == b0;
    if (!known) T.firsts |= b0 << (8 * T.nfirst++);
    if (L == 1) {
      T.one[b0] = (uint8_t)(k + 1);
    } else {  // chained in pair order behind the hash of the first two bytes
      const uint32_t h = multi_hash(b0, pats[k][1]);
      if (!T.head[h]) {
        T.head[h] = (uint8_t)(k + 1);
      } else {
        uint32_t c = T.head[h] - 1u;
        while (T.next[c]) c = T.next[c] - 1u;
        T.next[c] = (uint8_t)(k + 1);
      }
    }
    const uint32_t r = R > L ? (R + L - 1) / L : 1u;
    ratio = r > ratio ? r : ratio;
  }
  T.ratio = ratio < 3u ? ratio : 3u;
}

unsigned long long multi_output_bound(const MultiTable& T, unsigned long long n) {
  unsigned __int128 grow = 0;
  for (uint32_t k = 0; k < T.npairs; ++k)
    if (T.R[k] > T.L[k]) {
      const unsigned __int128 g = (unsigned __int128)(n / T.L[k]) * (T.R[k] - T.L[k]);
      grow = g > grow ? g : grow;
    }
  const unsigned __int128 b = (unsigned __int128)n + grow;
  return b > (unsigned __int128)~0ull ? ~0ull : (unsigned long long)b;
}

cudaError_t launch_replace_multi(const ReplaceParams& p, cudaStream_t st, int* grid_out) {
  if (p.mode != kModeMulti || !p.multi || !p.nsub || p.hold || p.carry_out || p.carry0 || p.carry0_dev ||
      p.L > kMultiMaxL)
    return cudaErrorInvalidValue;
  static std::mutex mu;
  static unsigned long long attr_dev_mask = 0;
  const uint32_t smem = make_layout_s(kModeMulti, p.L, p.R, p.nsub, p.multi_ratio, 2u).total;
  int dev = 0;
  cudaGetDevice(&dev);
  {
    std::lock_guard<std::mutex> g(mu);
    if (!(attr_dev_mask & (1ull << (dev & 63)))) {
      cudaError_t e = cudaFuncSetAttribute(replace_super_kernel<kModeMulti, false>,
                                           cudaFuncAttributeMaxDynamicSharedMemorySize, 220 * 1024);
      if (e != cudaSuccess) return e;
      attr_dev_mask |= 1ull << (dev & 63);
    }
  }
  int per_sm = 0;
  cudaError_t e = cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, replace_super_kernel<kModeMulti, false>,
                                                                kThreads, smem);
  if (e != cudaSuccess) return e;
  if (per_sm < 1) per_sm = 1;
  long long grid = (long long)per_sm * device_sm_count();
  if (grid > (long long)p.num_tiles) grid = p.num_tiles;
  if (grid < 1) grid = 1;
  replace_super_kernel<kModeMulti, false><<<(unsigned)grid, kThreads, smem, st>>>(p, SegLaunch{});
  if (grid_out) *grid_out = (int)grid;
  return cudaGetLastError();
}

}  // namespace crb
