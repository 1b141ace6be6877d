/*
 * replace_oracle.c - TEST INFRASTRUCTURE ONLY. CPU restatement of the reference
 * algorithm used as the checker for the CUDA path; nothing in the product links it.
 *
 * Semantics restated (RAZZULLIX/cuda_replace):
 *   - leftmost, non-overlapping greedy: a candidate p is kept when p >= blocked, then
 *     blocked = p + L. This is the serial greedy of greedy_keep_on_indices_kernel_seeded
 *     (cuda_replace.cu:938-968: `if (p - last >= L) { keep; last = p; }`), applied to
 *     every occurrence in position order, i.e. Python's bytes.replace
 *     (the reference's own correctness check, test/test.py:102-112, 150-161).
 *   - carry-in (apply_seeded, cuda_replace.cu:2403-2450): `last` starts at the previous
 *     kept start prev_last_rel, so candidates before prev_last_rel + L are blocked; the
 *     scatter kernels (cuda_replace.cu:1391-1608) only treat bytes covered by matches kept
 *     inside the buffer as covered, so seed-covered leading bytes are emitted.
 *   - query_prefix (cuda_replace.cu:1825-1897): number of kept starts < limit and the last
 *     such start (or -1), over the kept set of the last apply.
 *   - empty pattern: Python bytes.replace inserts rep before every byte and at the end
 *     (the reference instead returns the input unchanged, cuda_replace.cu:2104-2109).
 * Build: gcc -O2 -shared -fPIC -o oracle/_build/libreplace_oracle.so oracle/replace_oracle.c
 */
#include <stdint.h>
#include <stdlib.h>
#include <string.h>

#define ORACLE_EXPORT __attribute__((visibility("default")))

static const uint8_t* find_at_or_after(const uint8_t* s, int64_t n, int64_t from, const uint8_t* pat,
                                       int64_t L) {
  if (from < 0) from = 0;
  if (L <= 0 || from + L > n) return NULL;
  /* memchr on the first byte, then memcmp: O(n * L) in the worst case, fine for tests */
  const uint8_t* p = s + from;
  const uint8_t* end = s + n - L + 1;
  while (p < end) {
    const uint8_t* q = (const uint8_t*)memchr(p, pat[0], (size_t)(end - p));
    if (!q) return NULL;
    if (memcmp(q, pat, (size_t)L) == 0) return q;
    p = q + 1;
  }
  return NULL;
}

/* Output length of one replace (same walk as oracle_replace, nothing written). */
ORACLE_EXPORT int64_t oracle_replace_len(const uint8_t* src, int64_t n, const uint8_t* pat, int64_t L,
                                         int64_t R, int64_t block_before, int64_t* kept_count,
                                         int64_t* last_kept) {
  int64_t kept = 0, last = -1;
  if (L == 0) {
    if (kept_count) *kept_count = n + 1;
    if (last_kept) *last_kept = n;
    return n * (R + 1) + R;
  }
  int64_t out = 0, pos = 0;
  int64_t search = block_before > 0 ? block_before : 0;
  for (;;) {
    const uint8_t* q = find_at_or_after(src, n, search > pos ? search : pos, pat, L);
    if (!q) break;
    const int64_t p = (int64_t)(q - src);
    out += (p - pos) + R;
    pos = p + L;
    ++kept;
    last = p;
  }
  out += n - pos;
  if (kept_count) *kept_count = kept;
  if (last_kept) *last_kept = last;
  return out;
}

/* One replace into out (capacity out_cap). Returns the output length, or -1 when it does
 * not fit. Candidates starting before block_before are not taken (carry-in). */
ORACLE_EXPORT int64_t oracle_replace(const uint8_t* src, int64_t n, const uint8_t* pat, int64_t L,
                                     const uint8_t* rep, int64_t R, int64_t block_before, uint8_t* out,
                                     int64_t out_cap, int64_t* kept_count, int64_t* last_kept) {
  int64_t kept = 0, last = -1, o = 0;
  if (L == 0) {
    const int64_t total = n * (R + 1) + R;
    if (total > out_cap) return -1;
    for (int64_t i = 0; i < n; ++i) {
      memcpy(out + o, rep, (size_t)R);
      o += R;
      out[o++] = src[i];
    }
    memcpy(out + o, rep, (size_t)R);
    o += R;
    if (kept_count) *kept_count = n + 1;
    if (last_kept) *last_kept = n;
    return o;
  }
  int64_t pos = 0;
  int64_t search = block_before > 0 ? block_before : 0;
  for (;;) {
    const uint8_t* q = find_at_or_after(src, n, search > pos ? search : pos, pat, L);
    if (!q) break;
    const int64_t p = (int64_t)(q - src);
    if (o + (p - pos) + R > out_cap) return -1;
    memcpy(out + o, src + pos, (size_t)(p - pos));
    o += p - pos;
    memcpy(out + o, rep, (size_t)R);
    o += R;
    pos = p + L;
    ++kept;
    last = p;
  }
  if (o + (n - pos) > out_cap) return -1;
  memcpy(out + o, src + pos, (size_t)(n - pos));
  o += n - pos;
  if (kept_count) *kept_count = kept;
  if (last_kept) *last_kept = last;
  return o;
}

/* Kept starts of one replace written to positions[0, cap); returns how many were kept
 * (may exceed cap: then only the first cap are written). */
ORACLE_EXPORT int64_t oracle_kept_positions(const uint8_t* src, int64_t n, const uint8_t* pat, int64_t L,
                                            int64_t block_before, int64_t* positions, int64_t cap) {
  int64_t kept = 0, pos = 0;
  if (L == 0) return 0;
  int64_t search = block_before > 0 ? block_before : 0;
  for (;;) {
    const uint8_t* q = find_at_or_after(src, n, search > pos ? search : pos, pat, L);
    if (!q) break;
    const int64_t p = (int64_t)(q - src);
    if (kept < cap) positions[kept] = p;
    ++kept;
    pos = p + L;
  }
  return kept;
}

/* query_prefix over the kept set of one replace: kept starts < limit and the last one. */
ORACLE_EXPORT void oracle_query_prefix(const uint8_t* src, int64_t n, const uint8_t* pat, int64_t L,
                                       int64_t block_before, int64_t limit, int64_t* kept_before,
                                       int64_t* last_before) {
  int64_t kept = 0, last = -1, pos = 0;
  if (limit > n) limit = n;
  if (L == 0) { /* an empty match at every position: those before limit */
    *kept_before = limit > 0 ? limit : 0;
    *last_before = limit > 0 ? limit - 1 : -1;
    return;
  }
  int64_t search = block_before > 0 ? block_before : 0;
  for (;;) {
    const uint8_t* q = find_at_or_after(src, n, search > pos ? search : pos, pat, L);
    if (!q) break;
    const int64_t p = (int64_t)(q - src);
    if (p >= limit) break;
    ++kept;
    last = p;
    pos = p + L;
  }
  *kept_before = kept;
  *last_before = last;
}
