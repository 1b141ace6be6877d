// replace_kernels.h - launch interface between the session layer (capi.cu) and the
// sm_100a kernels (replace_kernels.cu).
//
// One apply of (pattern P of length L, replacement R) over an input of n bytes is ONE
// launch of replace_tiles_kernel. The input is cut into 16 KiB tiles; each CTA of a
// persistent grid takes tiles in increasing order from an atomic counter, stages the
// tile plus an (L-1)-byte halo in shared memory with a 1-D TMA bulk copy, finds the
// candidate positions, publishes the tile's carry function, resolves its exact
// carry-in with a decoupled look-back over the predecessors, and writes its output
// bytes at a 64-bit offset with TMA bulk stores. The leftmost, non-overlapping rule
// of bytes.replace is exact across every tile boundary; no second pass exists.
#pragma once

#include <cstdint>
#include <cuda_runtime.h>

namespace crb {

constexpr int kThreads = 256;               // threads per CTA
constexpr int kWarps = kThreads / 32;
constexpr int kSeg = 64;                    // input bytes owned by one thread
constexpr int kTile = kThreads * kSeg;      // 16384 input bytes per tile
constexpr int kOutWin = 16384;              // output staging window in shared memory
constexpr int kInlineMax = 256;             // pattern/replacement bytes carried in the launch parameters
constexpr uint32_t kMaxLen = 8192;          // longest pattern / replacement (CUDA_REPLACE_MAX_PATTERN)

// Carry modes. The carry between two tiles is "blocked until": how many leading bytes
// of the next tile are covered by a match kept earlier.
//  kModeFree:  P has no proper border (or L == 1), so two occurrences never overlap and
//              every occurrence is kept; the carry only tells which leading bytes are
//              covered. A tile's function is carry_out(c) = max(c - kTile, lco).
//  kModeSmall: P has a border and L <= 64: the tile function is a table over c in [0, L).
//  kModeLarge: P has a border and L > 64: same table, built without the warp level.
//  kModeMulti: several (pattern, replacement) pairs applied in one pass, with the result of
//              applying them one after the other (a "stage" of an apply_batch chain; see
//              MultiTable). No two occurrences of the stage's patterns can overlap, so, as in
//              kModeFree, every occurrence is kept and the carry only tells which leading bytes
//              are covered; the output offset advances by R_i - L_i per occurrence of pair i.
enum CarryMode : uint32_t { kModeFree = 0, kModeSmall = 1, kModeLarge = 2, kModeMulti = 3 };

// ---- Multi-pattern stages. A run of consecutive pairs of a chain is applied in ONE pass when
// the host has proved (plan_stages) that applying them one after the other gives the same
// bytes as replacing every occurrence of every pattern of the run in the run's input at once:
// no occurrence of one pattern can overlap an occurrence of another (or of itself), and no
// replacement of an earlier pair can form, with the bytes around it, an occurrence of a later
// pattern. The stage's pairs live in a table in device memory, staged into shared memory.
constexpr uint32_t kMultiMaxPairs = 32;
constexpr uint32_t kMultiMaxL = 32;
constexpr uint32_t kMultiMaxR = 64;
constexpr uint32_t kMultiMaxFirst = 4;             // distinct first pattern bytes of a stage
constexpr unsigned long long kMultiBias = 65536;   // look-back payload bias per super-tile (>= its bytes)

struct MultiTable {
  uint32_t npairs, nfirst, Lmin, Lmax;
  uint32_t firsts;                     // the nfirst distinct first bytes, one per byte lane
  uint32_t ratio;                      // output staging per input byte (1..3)
  uint32_t pad[2];
  uint32_t p4[kMultiMaxPairs], m4[kMultiMaxPairs];  // first min(L, 4) bytes and their mask
  uint8_t L[kMultiMaxPairs], R[kMultiMaxPairs];
  uint8_t next[kMultiMaxPairs];        // hash chain: next pair + 1 (0 = end)
  uint8_t pad2[kMultiMaxPairs];
  uint8_t one[256];                    // byte -> pair + 1 of a one-byte pattern (0 = none)
  uint8_t head[256];                   // hash of the first two bytes -> first pair + 1
  uint8_t pat[kMultiMaxPairs][kMultiMaxL];
  uint8_t rep[kMultiMaxPairs][kMultiMaxR + 16];  // padded: replacements are read four bytes at a time
};
static_assert(sizeof(MultiTable) % 16 == 0, "MultiTable is staged with 16-byte copies");

__host__ __device__ __forceinline__ uint32_t multi_hash(uint32_t b0, uint32_t b1) { return (b0 + 131u * b1) & 255u; }

// Look-back state of tile t: status[t] = (epoch << 2) | state.
enum TileState : uint32_t { kStAgg = 1, kStInc = 2 };

struct TileIncl {                 // inclusive prefix through tile t
  unsigned long long kept;        // matches kept in tiles [0, t]
  long long last;                 // start of the last of them (input position) or -1
  unsigned int carry;             // bytes of tile t+1 covered by a match kept in [0, t]
  unsigned int pad;
};

struct ApplyResult {              // device-side result block of one session
  unsigned long long out_len;     // written by the CTA that owns the last tile
  unsigned long long kept;
  long long last_kept;
  unsigned int error_epoch;       // == epoch: a bounded wait gave up; results invalid
  unsigned int overflow_epoch;    // == epoch: output did not fit in out_cap; nothing valid written
  unsigned int tile_counter;      // dynamic tile scheduler, reset by the last CTA to exit
  unsigned int done_ctas;
  unsigned long long q_kept;      // query_prefix answer
  long long q_last;
  unsigned long long last_tagged; // super-tile kernel: (epoch << 40) | (last kept start + 1), atomicMax
  unsigned long long pad;
};

struct ReplaceParams {
  const uint8_t* in;              // 16-byte aligned; readable up to round_up(n, 16)
  uint8_t* out;                   // 16-byte aligned, out_cap bytes
  unsigned long long n;
  unsigned long long out_cap;
  unsigned long long block_before;  // candidates starting before this position are not taken
  unsigned long long stride_mask; // bits 0, L, 2L, ... below 64 (1 when L >= 64)
  unsigned int L, R;
  unsigned int mode;              // CarryMode
  unsigned int num_tiles;
  unsigned int epoch;
  unsigned int agg_entries;       // entries per tile function (1 in kModeFree, min(L, kTile) otherwise)
  unsigned int p4, m4;            // first min(L, 4) pattern bytes (little endian) and their byte mask
  unsigned int inv_l;             // ceil(65536 / L), for L < 64
  unsigned int query_limit;       // query kernel: tile-relative limit
  unsigned int query_tile;        // query kernel: tile index
  unsigned int nsub;              // super-tile kernel: 16 KiB sub-tiles per super-tile (0 = tile kernel)
  unsigned long long query_limit64;  // super-tile query: absolute limit
  unsigned int* status;           // [num_tiles]
  TileIncl* incl;                 // [num_tiles]
  unsigned long long* agg;        // [num_tiles * agg_entries]
  ApplyResult* res;
  long long* tile_last;           // super-tile kernel: last kept start per super-tile or -1 [num_tiles]
  unsigned long long* rec;        // super-tile kernel: 16-byte look-back record per super-tile [2 * num_tiles]
  // Chaining (super-tile kernel). When n_dev is set the input length is read from device
  // memory (the previous launch's len_out), so launches chain without a host round trip;
  // num_tiles is then only an upper bound. `hold` trailing bytes are matched against but
  // produce no output (a streaming chunk keeps them for the next chunk). carry0 (or
  // *carry0_dev) leading bytes are covered by a match kept before this buffer; the last
  // tile writes the output length to *len_out and the coverage past the output range to
  // *carry_out.
  const unsigned long long* n_dev;
  unsigned long long* len_out;
  const unsigned int* carry0_dev;
  unsigned int* carry_out;
  unsigned long long hold;
  unsigned long long n_cap;       // with n_dev: the input buffer's capacity (a longer length is clamped)
  unsigned long long len_bias;    // output starts this many bytes into out (out stays 16-byte aligned);
                                  // *len_out receives len_bias + the output length
  unsigned int carry0;
  unsigned int multi_ratio;       // kModeMulti: output staging per input byte (1..3), as MultiTable::ratio
  const uint8_t* pat_ext;         // device copy when L > kInlineMax
  const uint8_t* rep_ext;         // device copy when R > kInlineMax
  const MultiTable* multi;        // kModeMulti: the stage's pairs (device memory); L = their longest
  // Presence index of the input (cuda_replace_build_index): 8 words (a 256-bit byte set) per
  // chunk of 2^presence_shift bytes (>= 16 KiB). A 16 KiB sub-tile whose chunk lacks the
  // pattern's first byte has no candidate and skips the search. nullptr: no index.
  const uint32_t* presence;
  unsigned int presence_shift;
  unsigned int pad2;
  uint8_t pat[kInlineMax];
  uint8_t rep[kInlineMax];
};

// ---- Segmented launch: many jobs in ONE launch of the super-tile kernel. Each job has its
// own input, output and (pattern, replacement); work is split by super-tiles across all jobs,
// not by jobs: super-tile g of the launch belongs to job tile_job[g], at local index
// g - jobs[tile_job[g]].tile_base. A plan kernel (one CTA) reads every job's input length
// from device memory, numbers the super-tiles and draws a fresh epoch, so a sequence of
// segmented launches chains on the device and can be replayed from a CUDA graph.
constexpr uint32_t kSegMaxL = 32;  // longest pattern of a segmented launch
constexpr uint32_t kSegMaxR = 64;  // longest replacement of a segmented launch

struct SegPair {                   // one (pattern, replacement) and its derived fields
  unsigned long long stride_mask;
  unsigned int L, R, mode, p4, m4, inv_l, agg_entries, pad;
  uint8_t pat[kSegMaxL];
  uint8_t rep[kSegMaxR];
};

struct SegJob {                    // one job of a segmented launch
  const uint8_t* in;               // 16-byte aligned, readable up to its length rounded up to 16
  uint8_t* out;                    // 16-byte aligned
  const unsigned long long* n_dev; // input length (device)
  unsigned long long* len_out;     // receives the output length (device)
  unsigned long long out_cap;
  unsigned int pair;               // index into SegLaunch::pairs
  unsigned int res;                // index of the job's result block
  unsigned int tile_base;          // written by the plan kernel
  unsigned int ntiles;             // written by the plan kernel
  unsigned int pad[2];
};

struct SegLaunch {
  SegJob* jobs;
  const unsigned int* njobs;       // device: jobs in this launch
  const SegPair* pairs;
  ApplyResult* res;                // per job; a nonzero error or overflow epoch marks the job failed
  unsigned int* total;             // device: super-tiles of this launch (plan kernel)
  unsigned int* tile_job;          // [max_tiles]: super-tile -> job (plan kernel)
  unsigned int* sched;             // [2]: claim counter, finished CTAs (reset by the last CTA)
  unsigned int* epoch;             // [2]: launch counter (plan kernel) and the current epoch
  uint32_t* status;                // look-back scratch shared by the launches of one stream
  TileIncl* incl;
  unsigned long long* agg;
  long long* tile_last;
  unsigned long long* rec;
  unsigned int max_tiles;          // capacity of the scratch arrays, in super-tiles
  unsigned int agg_stride;         // agg entries per super-tile (the largest L of the launch)
  unsigned int mode;               // CarryMode of every pair in the launch
  unsigned int Lmax, Rmax;         // largest pattern and replacement (shared-memory layout)
  unsigned int nsub;               // 16 KiB sub-tiles per super-tile
};

// Host helpers (replace_kernels.cu).
// Fills the pattern-derived fields of p (mode, p4, m4, inv_l, stride_mask, agg_entries).
void prepare_pattern_fields(ReplaceParams& p, const uint8_t* pat, uint32_t L);
// Dynamic shared memory bytes used by replace_tiles_kernel for (mode, L, R).
uint32_t tile_kernel_smem_bytes(uint32_t mode, uint32_t L, uint32_t R);
// Launch one apply. grid_ctas_out receives the number of CTAs launched.
cudaError_t launch_replace(const ReplaceParams& p, cudaStream_t st, int* grid_ctas_out);
// Sub-tiles per super-tile for the super-tile kernel, or 0 when (mode, L) needs the tile kernel.
uint32_t super_nsub(uint32_t mode, uint32_t L);
// Launch one apply with the super-tile kernel (p.nsub > 0, p.tile_last set).
cudaError_t launch_replace_super(const ReplaceParams& p, cudaStream_t st, int* grid_ctas_out);
// Query for an apply made by the super-tile kernel: p.query_limit64 = limit (< p.n).
cudaError_t launch_query_super(const ReplaceParams& p, cudaStream_t st);
// One CTA answers query_prefix for tile p.query_tile at tile-relative limit p.query_limit,
// using the tile records of the apply described by p; writes res->q_kept / res->q_last.
cudaError_t launch_query(const ReplaceParams& p, cudaStream_t st);
// Copy the last P bytes of buf[0, min(*total, cap)) to dst (streaming: a stage's held tail).
cudaError_t launch_move_tail(const uint8_t* buf, const unsigned long long* total, unsigned long long cap,
                             uint32_t P, uint8_t* dst, cudaStream_t st);
// Segmented launch (sl.mode free or small): the plan kernel, then the super-tile kernel over
// every job's super-tiles. grid_ctas = 0 picks the occupancy-limited persistent grid; a
// caller passing its own grid must have called seg_ctas_per_sm for the mode once (it sets the
// kernel's shared-memory limit), after which launch_seg makes no other runtime call than the
// two launches (so it can be captured in a CUDA graph).
cudaError_t launch_seg(const SegLaunch& sl, cudaStream_t st, int grid_ctas);
// Dynamic shared memory of a segmented launch, and its CTAs per SM.
uint32_t seg_smem_bytes(const SegLaunch& sl);
int seg_ctas_per_sm(const SegLaunch& sl);
// Fills a SegPair from (pat, L, rep, R); false when the pair does not fit a segmented launch.
bool make_seg_pair(SegPair& q, const uint8_t* pat, uint32_t L, const uint8_t* rep, uint32_t R);
// Partition of a chain of pairs into stages that each run as one pass (kModeMulti when a stage
// has two pairs or more, the pair's own mode otherwise). stage_of[k] receives the stage of pair
// k; returns the number of stages. keep_last_alone: the last pair gets a stage of its own.
int plan_stages(const uint8_t* const* pats, const int* pat_lens, const uint8_t* const* reps,
                const int* rep_lens, int count, bool keep_last_alone, int* stage_of);
// Fills a MultiTable from pairs [0, count) (count in [2, kMultiMaxPairs], as plan_stages formed).
void build_multi_table(MultiTable& T, const uint8_t* const* pats, const int* pat_lens,
                       const uint8_t* const* reps, const int* rep_lens, int count);
// Worst-case output length of one pass of a stage over n input bytes (saturating).
unsigned long long multi_output_bound(const MultiTable& T, unsigned long long n);
// Launch one stage (p.mode == kModeMulti, p.multi set, p.nsub > 0).
cudaError_t launch_replace_multi(const ReplaceParams& p, cudaStream_t st, int* grid_ctas_out);
// Presence index: for every chunk of 2^shift bytes of in[0, n), the set of byte values in it
// (8 words, bit b of word b / 32) into masks[8 * chunk ...].
cudaError_t launch_presence(const uint8_t* in, unsigned long long n, uint32_t shift, uint32_t* masks,
                            cudaStream_t st);
// bytes.replace with an empty pattern: rep before every byte and at the end.
cudaError_t launch_empty_pattern(const uint8_t* in, unsigned long long n, const uint8_t* rep_dev,
                                 uint32_t R, uint8_t* out, cudaStream_t st);

}  // namespace crb
