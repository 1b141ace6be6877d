/*
 * fake_capi.c - TEST DOUBLE. A CPU implementation of the libcuda_replace C ABI built on
 * the oracle restatement (oracle/replace_oracle.c), so the Python host logic (ctypes
 * bindings, the chunked streaming helper, return-code handling) can be tested without a
 * GPU. It is never shipped and never loaded by the product.
 */
#include <stdint.h>
#include <stdlib.h>
#include <string.h>

#include "../oracle/replace_oracle.c"

#define FAKE_EXPORT __attribute__((visibility("default")))

typedef struct {
  int alive;
  uint8_t* buf;
  int64_t len;
  /* last apply, for query_prefix */
  uint8_t* prev;
  int64_t prev_len;
  uint8_t* pat;
  int64_t L;
  int64_t block_before;
  int valid;
  int64_t launches;
  int64_t kept;
} FakeSession;

static int apply_one(FakeSession* s, const uint8_t* pat, int pat_len, const uint8_t* rep, int rep_len,
                     int64_t block_before, long long* out_last, size_t* new_len) {
  if (pat_len < 0 || rep_len < 0) return -1;
  if (pat_len > 8192 || rep_len > 8192) return -4;
  int64_t kept = 0, last = -1;
  const int64_t out_n =
      oracle_replace_len(s->buf, s->len, pat, pat_len, rep_len, block_before, &kept, &last);
  uint8_t* out = (uint8_t*)malloc(out_n ? (size_t)out_n : 1);
  oracle_replace(s->buf, s->len, pat, pat_len, rep, rep_len, block_before, out, out_n, &kept, &last);
  free(s->prev);
  free(s->pat);
  s->prev = s->buf;
  s->prev_len = s->len;
  s->pat = (uint8_t*)malloc(pat_len ? (size_t)pat_len : 1);
  memcpy(s->pat, pat, (size_t)pat_len);
  s->L = pat_len;
  s->block_before = block_before;
  s->valid = 1;
  s->buf = out;
  s->len = out_n;
  s->launches += 1;
  s->kept = kept;
  if (out_last) *out_last = (pat_len == 0) ? (long long)s->prev_len : (long long)last;
  if (new_len) *new_len = (size_t)out_n;
  return 0;
}

FAKE_EXPORT const char* cuda_replace_version(void) { return "fake cpu capi (test double)"; }

FAKE_EXPORT void cuda_free_host(void* p) { free(p); }

FAKE_EXPORT int cuda_replace_open(void** ph, const uint8_t* src, size_t len) {
  if (!ph) return -1;
  FakeSession* s = (FakeSession*)calloc(1, sizeof(FakeSession));
  if (!s) return -2;
  s->alive = 1;
  s->buf = (uint8_t*)malloc(len ? len : 1);
  if (len) memcpy(s->buf, src, len);
  s->len = (int64_t)len;
  *ph = s;
  return 0;
}

FAKE_EXPORT int cuda_replace_reset(void* h, const uint8_t* src, size_t len) {
  FakeSession* s = (FakeSession*)h;
  if (!s) return -1;
  if (!s->alive) return -3;
  free(s->buf);
  s->buf = (uint8_t*)malloc(len ? len : 1);
  if (len) memcpy(s->buf, src, len);
  s->len = (int64_t)len;
  s->valid = 0;
  return 0;
}

FAKE_EXPORT int cuda_replace_build_index(void* h, size_t chunk) {
  (void)chunk;
  return h ? 0 : -1;
}

FAKE_EXPORT int cuda_replace_apply(void* h, const uint8_t* pat, int pat_len, const uint8_t* rep, int rep_len,
                                   size_t* new_len) {
  FakeSession* s = (FakeSession*)h;
  if (!s) return -1;
  if (!s->alive) return -3;
  return apply_one(s, pat, pat_len, rep, rep_len, 0, NULL, new_len);
}

FAKE_EXPORT int cuda_replace_apply_seeded(void* h, const uint8_t* pat, int pat_len, const uint8_t* rep,
                                          int rep_len, long long prev_last_rel, long long* out_last_rel,
                                          size_t* new_len) {
  FakeSession* s = (FakeSession*)h;
  if (!s) return -1;
  if (!s->alive) return -3;
  const long long b = pat_len > 0 ? prev_last_rel + pat_len : 0;
  return apply_one(s, pat, pat_len, rep, rep_len, b > 0 ? b : 0, out_last_rel, new_len);
}

FAKE_EXPORT int cuda_replace_query_prefix64(void* h, size_t limit, long long* kept, long long* last) {
  FakeSession* s = (FakeSession*)h;
  if (!s) return -1;
  if (!s->alive) return -3;
  int64_t k = 0, l = -1;
  if (s->valid)
    oracle_query_prefix(s->prev, s->prev_len, s->pat, s->L, s->block_before, (int64_t)limit, &k, &l);
  if (kept) *kept = k;
  if (last) *last = l;
  return 0;
}

FAKE_EXPORT int cuda_replace_query_prefix(void* h, size_t limit, int* kept, int* last) {
  long long k = 0, l = -1;
  const int rc = cuda_replace_query_prefix64(h, limit, &k, &l);
  if (rc) return rc;
  if (k > 0x7FFFFFFF || l > 0x7FFFFFFF) return -5;
  if (kept) *kept = (int)k;
  if (last) *last = (int)l;
  return 0;
}

FAKE_EXPORT int cuda_replace_apply_batch(void* h, const uint8_t** pats, const int* pat_lens,
                                         const uint8_t** reps, const int* rep_lens, int count,
                                         size_t* new_len) {
  FakeSession* s = (FakeSession*)h;
  if (!s) return -1;
  if (!s->alive) return -3;
  for (int i = 0; i < count; ++i) {
    const int rc = apply_one(s, pats[i], pat_lens[i], reps[i], rep_lens[i], 0, NULL, NULL);
    if (rc) return rc;
  }
  if (new_len) *new_len = (size_t)s->len;
  return 0;
}

FAKE_EXPORT int cuda_replace_result(void* h, uint8_t** out, size_t* len) {
  FakeSession* s = (FakeSession*)h;
  if (!s || !out || !len) return -1;
  if (!s->alive) return -3;
  *len = (size_t)s->len;
  *out = NULL;
  if (!s->len) return 0;
  *out = (uint8_t*)malloc((size_t)s->len);
  memcpy(*out, s->buf, (size_t)s->len);
  return 0;
}

FAKE_EXPORT int cuda_replace_result_into(void* h, uint8_t* dst, size_t cap, size_t* len) {
  FakeSession* s = (FakeSession*)h;
  if (!s) return -1;
  if (len) *len = (size_t)s->len;
  if ((size_t)s->len > cap) return 1;
  memcpy(dst, s->buf, (size_t)s->len);
  return 0;
}

FAKE_EXPORT int cuda_replace_length(void* h, size_t* len) {
  FakeSession* s = (FakeSession*)h;
  if (!s || !len) return -1;
  if (!s->alive) return -3;
  *len = (size_t)s->len;
  return 0;
}

FAKE_EXPORT int cuda_replace_stats(void* h, unsigned long long* kept, unsigned long long* launches) {
  FakeSession* s = (FakeSession*)h;
  if (!s) return -1;
  if (kept) *kept = (unsigned long long)s->kept;
  if (launches) *launches = (unsigned long long)s->launches;
  return 0;
}

FAKE_EXPORT void cuda_replace_close(void* h) {
  FakeSession* s = (FakeSession*)h;
  if (!s || !s->alive) return;
  s->alive = 0;
  free(s->buf);
  free(s->prev);
  free(s->pat);
  free(s);
}

FAKE_EXPORT int cuda_replace_unified(const uint8_t* src, size_t n, const uint8_t* pat, int pat_len,
                                     const uint8_t* rep, int rep_len, uint8_t** out, size_t* out_len) {
  void* h = NULL;
  int rc = cuda_replace_open(&h, src, n);
  if (rc) return rc;
  rc = cuda_replace_apply(h, pat, pat_len, rep, rep_len, NULL);
  if (!rc) rc = cuda_replace_result(h, out, out_len);
  cuda_replace_close(h);
  return rc;
}

FAKE_EXPORT int cuda_replace_output_bound(size_t n, int pat_len, int rep_len, size_t* bound) {
  if (!bound || pat_len < 0 || rep_len < 0) return -1;
  if (pat_len == 0)
    *bound = n * ((size_t)rep_len + 1) + (size_t)rep_len;
  else
    *bound = rep_len <= pat_len ? n : n + n / (size_t)pat_len * (size_t)(rep_len - pat_len);
  return 0;
}

FAKE_EXPORT int cuda_replace_unified_into(const uint8_t* src, size_t n, const uint8_t* pat, int pat_len,
                                          const uint8_t* rep, int rep_len, uint8_t* dst, size_t cap,
                                          size_t* out_len) {
  if (!out_len) return -1;
  uint8_t* out = NULL;
  size_t m = 0;
  const int rc = cuda_replace_unified(src, n, pat, pat_len, rep, rep_len, &out, &m);
  if (rc) return rc;
  *out_len = m;
  if (m > cap) {
    free(out);
    return 1; /* cudaErrorInvalidValue: *out_len holds the length needed */
  }
  if (m) memcpy(dst, out, m);
  free(out);
  return 0;
}
