/*
 * cuda_replace.h - C ABI of libcuda_replace.so (B200 / sm_100a build).
 *
 * Leftmost, non-overlapping byte-pattern replacement with the semantics of
 * Python's bytes.replace. The first twelve entry points keep the exact
 * signatures, ownership rules and return codes of the RAZZULLIX/cuda_replace
 * library (cuda_replace.cu), so the unchanged cuda_replace_wrapper.py binds this
 * library through ctypes. Each declaration cites the reference export it
 * replaces (cuda_replace.cu:<line>) and the ctypes binding that loads it
 * (cuda_replace_wrapper.py:<line>).
 *
 * Return codes (all int-returning calls):
 *    0   success
 *   -1   null handle or null output argument
 *   -2   the session object could not be allocated
 *   -3   the handle has been closed
 *   -4   pattern or replacement longer than CUDA_REPLACE_MAX_PATTERN
 *   -5   a 32-bit output of cuda_replace_query_prefix cannot hold the value
 *        (use cuda_replace_query_prefix64)
 *   -6   a size above the fixed limits of cuda_replace_apply_device_noalloc
 *   -7   cuda_replace_stream: a pair outside the limits of the chunk-major path
 *   >0   a cudaError_t; 999 (cudaErrorUnknown) for internal failures, including a
 *        bounded device-side wait that gave up
 *
 * Threading: calls on one handle are serialised by a per-handle mutex; different
 * handles may be used concurrently from different threads. A handle must not be
 * used after cuda_replace_close returns.
 *
 * Ownership: input buffers stay owned by the caller and are only read during the
 * call. *out_host buffers are page-locked host memory owned by the library and are
 * released with cuda_free_host. An empty result returns *out_host == NULL.
 */
#ifndef CUDA_REPLACE_H
#define CUDA_REPLACE_H

#include <stddef.h>
#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

/* Longest pattern and replacement accepted by every apply call. */
#define CUDA_REPLACE_MAX_PATTERN 8192

/* Library identification string.
 * Replaces cuda_replace_version (cuda_replace.cu:2251). Not bound by the wrapper. */
const char* cuda_replace_version(void);

/* One-shot replace: upload src, replace every leftmost non-overlapping pat with rep,
 * return the result in library-owned page-locked memory. A src of 256 MiB or more is uploaded,
 * replaced and downloaded chunk by chunk, the directions overlapped (a pageable src is copied
 * chunk by chunk into page-locked staging buffers by a second host thread meanwhile).
 * Replaces cuda_replace_unified (cuda_replace.cu:2579);
 * bound at cuda_replace_wrapper.py:48-54, called at cuda_replace_wrapper.py:124-141. */
int cuda_replace_unified(const uint8_t* src, size_t src_len,
                         const uint8_t* pat, int pat_len,
                         const uint8_t* rep, int rep_len,
                         uint8_t** out_host, size_t* out_len);

/* cuda_replace_unified into caller memory dst[0, dst_cap) (pageable or page-locked): *out_len
 * receives the result length. With dst_cap at least cuda_replace_output_bound's worst case, a
 * src of 256 MiB or more is replaced chunk by chunk; each chunk's output is downloaded into a
 * pooled page-locked block and copied into dst on the host copy threads as soon as it lands,
 * while later chunks upload, replace and download (a result of 32 MiB or more from the
 * single-launch path is downloaded and copied the same way in pieces), so the copy into dst
 * overlaps the transfers. Returns cudaErrorInvalidValue (1) when dst_cap is below the
 * result length (*out_len then holds that length; dst is unspecified); -1 for NULL arguments
 * or negative lengths, -4 for a pattern or replacement above CUDA_REPLACE_MAX_PATTERN.
 * An addition to the reference's API (its wrapper returns bytes built from the unified result,
 * cuda_replace_wrapper.py:124-141; this call lets a binding fill its bytes object directly). */
int cuda_replace_unified_into(const uint8_t* src, size_t src_len,
                              const uint8_t* pat, int pat_len,
                              const uint8_t* rep, int rep_len,
                              uint8_t* dst, size_t dst_cap, size_t* out_len);

/* Worst-case output length of one replace of pat_len bytes by rep_len bytes over src_len bytes
 * (src_len when rep_len <= pat_len; saturates at SIZE_MAX). -1 for a NULL bound or a negative
 * length. */
int cuda_replace_output_bound(size_t src_len, int pat_len, int rep_len, size_t* bound);

/* Release a buffer returned through *out_host.
 * Replaces cuda_free_host (cuda_replace.cu:2559); bound at cuda_replace_wrapper.py:57-58. */
void cuda_free_host(void* p);

/* Open a session whose device-resident buffer holds a copy of src[0, len).
 * Replaces cuda_replace_open (cuda_replace.cu:2256); bound at cuda_replace_wrapper.py:61-62. */
int cuda_replace_open(void** ph, const uint8_t* src, size_t len);

/* Replace the session buffer with a copy of src[0, len), reusing device capacity.
 * Replaces cuda_replace_reset (cuda_replace.cu:2295); bound at cuda_replace_wrapper.py:97-101. */
int cuda_replace_reset(void* h, const uint8_t* src, size_t len);

/* Build a presence index of the session buffer: for every chunk of chunk_size bytes (0: 1 MiB,
 * the reference's default; otherwise rounded up to a power of two of at least 16 KiB) the set of
 * byte values it holds. The next apply, apply_seeded or apply_batch (its first pair) of this
 * buffer skips the candidate search in every 16 KiB sub-tile whose chunk lacks the pattern's
 * first byte; results are unchanged. Any change of the buffer (reset, apply) retires the index.
 * The reference builds the same kind of index but no apply path consults it (cu:1249, 1904, 2006).
 * Replaces cuda_replace_build_index (cuda_replace.cu:2320); bound at cuda_replace_wrapper.py:65-69. */
int cuda_replace_build_index(void* h, size_t chunk_size);

/* Replace every leftmost non-overlapping occurrence of pat in the session buffer.
 * *new_len receives the new buffer length.
 * Replaces cuda_replace_apply (cuda_replace.cu:2356); bound at cuda_replace_wrapper.py:73-76. */
int cuda_replace_apply(void* h, const uint8_t* pat, int pat_len,
                       const uint8_t* rep, int rep_len, size_t* new_len);

/* As cuda_replace_apply, with a carry-in: prev_last_rel is the start of the previous
 * kept match relative to byte 0 of this buffer (negative when it lies in an earlier
 * chunk), so candidates starting before prev_last_rel + pat_len are not taken. The
 * bytes that match covers inside this buffer are still emitted as literals (the
 * previous chunk already emitted its replacement). *out_last_rel receives the start of
 * the last match kept in this buffer, or -1.
 * Replaces cuda_replace_apply_seeded (cuda_replace.cu:2403); bound at cuda_replace_wrapper.py:104-114. */
int cuda_replace_apply_seeded(void* h, const uint8_t* pat, int pat_len,
                              const uint8_t* rep, int rep_len,
                              long long prev_last_rel, long long* out_last_rel,
                              size_t* new_len);

/* Over the matches kept by the most recent apply (positions in that apply's input):
 * *kept_before_limit = how many start before limit, *last_kept_before_limit = the
 * last such start or -1. limit is clamped to that input's length.
 * Replaces cuda_replace_query_prefix (cuda_replace.cu:2452); bound at cuda_replace_wrapper.py:117-121. */
int cuda_replace_query_prefix(void* h, size_t limit, int* kept_before_limit,
                              int* last_kept_before_limit);

/* Apply count (pattern, replacement) pairs in order, each to the output of the previous.
 * Replaces cuda_replace_apply_batch (cuda_replace.cu:2465); bound at cuda_replace_wrapper.py:79-87. */
int cuda_replace_apply_batch(void* h, const uint8_t** pats, const int* pat_lens,
                             const uint8_t** reps, const int* rep_lens,
                             int count, size_t* new_len);

/* Copy the session buffer to library-owned page-locked memory (free with cuda_free_host).
 * Replaces cuda_replace_result (cuda_replace.cu:2528); bound at cuda_replace_wrapper.py:90-91. */
int cuda_replace_result(void* h, uint8_t** out_host, size_t* outlen_host);

/* Close the session and free its device memory.
 * Replaces cuda_replace_close (cuda_replace.cu:2565); bound at cuda_replace_wrapper.py:94-95. */
void cuda_replace_close(void* h);

/* ---- Additive entry points (no counterpart in the reference; optional for callers) ---- */

/* Current length of the session buffer, without copying it to the host. */
int cuda_replace_length(void* h, size_t* len);

/* 64-bit form of cuda_replace_query_prefix. */
int cuda_replace_query_prefix64(void* h, size_t limit, long long* kept_before_limit,
                                long long* last_kept_before_limit);

/* Copy the session buffer into caller memory dst[0, cap). *len receives the length;
 * returns cudaErrorInvalidValue (1) when cap is too small (nothing is copied). */
int cuda_replace_result_into(void* h, uint8_t* dst, size_t cap, size_t* len);

/* Device-side counters of the most recent apply on this handle: number of matches kept
 * and the number of kernel launches issued by this library since the handle was opened. */
int cuda_replace_stats(void* h, unsigned long long* kept_last_apply,
                       unsigned long long* kernel_launches);

/* Replace in device memory: d_in[0, n) -> d_out, enqueued on `stream` (a cudaStream_t;
 * NULL = the session's own stream) without waiting for it. d_in and d_out must be 16-byte
 * aligned device pointers, d_in readable up to n rounded up to 16, and out_cap at least
 * the worst-case output n + (n / pat_len) * max(0, rep_len - pat_len). pat_len must be in
 * [1, 256] and rep_len in [0, 256]. When n < pat_len no occurrence is possible and d_in is
 * copied to d_out unchanged (as bytes.replace returns its input). Calls on one handle must use
 * one stream (they share the handle's look-back scratch); the handle's own stream is ordered
 * around the launch by events, so its scratch clears never overlap the kernel. The session
 * buffer is not touched. */
int cuda_replace_apply_device_async(void* h, const uint8_t* d_in, size_t n,
                                    const uint8_t* pat, int pat_len,
                                    const uint8_t* rep, int rep_len,
                                    uint8_t* d_out, size_t out_cap, void* stream);

/* Wait for the last cuda_replace_apply_device_async of this handle and report its output
 * length and number of matches kept. */
int cuda_replace_device_result(void* h, size_t* out_len, unsigned long long* kept);

/* No counterpart in the reference. For callers that must not allocate memory at call time
 * (an arena or pool owns the device budget, a host forbids cudaMalloc/cudaFree because they
 * can synchronise the device, or the path must not fail on out-of-memory): replace
 * d_in[0, n) into d_out with no allocation at all. The kernel's scratch is a fixed
 * __device__ array of about 2.1 MiB that every GPU loading this library keeps until exit.
 * Limits: n <= CUDA_REPLACE_NOALLOC_MAX_INPUT, pat_len in [1, 64], rep_len in [0, 256]
 * (else -6); d_in and d_out 16-byte aligned, d_in readable up to n rounded up to 16, and
 * out_cap >= n + (n / pat_len) * max(0, rep_len - pat_len) (else 1). Runs on `stream`
 * (a cudaStream_t, NULL = default stream) and waits for it; *out_len gets the output length.
 * The first call on a device looks up the array's device address (cudaGetSymbolAddress)
 * with that device current; make that first call before any stream capture. All calls on
 * a device share the array: calls whose work overlaps on the GPU race and must not be made. */
#define CUDA_REPLACE_NOALLOC_MAX_INPUT (64u << 20)
int cuda_replace_apply_device_noalloc(const uint8_t* d_in, size_t n,
                                      const uint8_t* pat, int pat_len,
                                      const uint8_t* rep, int rep_len,
                                      uint8_t* d_out, size_t out_cap, size_t* out_len,
                                      void* stream);

/* Chunk-major streaming: apply every (pats[k], reps[k]) in order, as chained bytes.replace,
 * to src[0, n), read chunk_bytes at a time (0 = 256 MiB), so n may exceed device memory.
 * Replaces the pair-major helper gpu_replace_streaming (cuda_replace_wrapper.py:305-366),
 * which crosses the host link twice per pair and drops the replacement of a match that
 * straddles a chunk boundary (py:356); here the result equals chained bytes.replace for any
 * chunk size. Each chunk passes through all pairs on the device before the next chunk is
 * needed: each pair holds its last pat_len - 1 bytes back for the next chunk, the coverage of
 * a match kept before a chunk is carried into it, lengths between pairs stay on the device,
 * and the next chunk's upload and the previous chunk's download overlap the compute.
 * *out_host receives page-locked memory to release with cuda_free_host (NULL when the result
 * is empty). Limits: pat_lens in [1, 256], rep_lens in [0, 256], and a pattern with a proper
 * border (a prefix that is also a suffix) at most 32 bytes long; -7 when a pair is outside
 * them (stream such pairs pair-major); -1 for NULL arguments or a negative length;
 * >0 a cudaError_t. */
int cuda_replace_stream(const uint8_t* src, size_t n, const uint8_t** pats, const int* pat_lens,
                        const uint8_t** reps, const int* rep_lens, int count, size_t chunk_bytes,
                        uint8_t** out_host, size_t* out_len);

/* How cuda_replace_apply_batch groups a chain of pairs into passes (no counterpart in the
 * reference, whose apply_batch makes one full pass per pair, cuda_replace.cu:2480-2519). A run of
 * consecutive pairs is one pass (a "stage") when applying them one after the other provably gives
 * the same bytes as replacing, in the run's input, every occurrence of every pattern of the run at
 * once: every pattern has no proper border, no two patterns of the run can overlap (none inside
 * another, no suffix of one equal to a prefix of another, no pattern twice), no replacement of an
 * earlier pair of the run can form an occurrence of a later pattern with the bytes around it (an
 * empty replacement joins two bytes, so it ends the run unless the later patterns are one byte
 * long), and the run has at most 32 pairs, patterns of 1-32 bytes with at most 4 distinct first
 * bytes, replacements of at most 64 bytes. stage_of[k] receives the pass of pair k; returns the
 * number of passes, or -1 for invalid arguments. keep_last_alone: the last pair gets a pass of its
 * own (apply_batch does this, so query_prefix afterwards describes the last pair). Host code only:
 * needs no GPU. The environment variable CUDA_REPLACE_STAGES=0 makes apply_batch use one pass
 * per pair. */
int cuda_replace_plan_stages(const uint8_t** pats, const int* pat_lens, const uint8_t** reps,
                             const int* rep_lens, int count, int keep_last_alone, int* stage_of);

/* As cuda_replace_stream, between two open file descriptors (no counterpart in the reference,
 * whose streaming helper takes and returns Python bytes, cuda_replace_wrapper.py:305-366): the
 * input is read from in_fd until it ends (a regular file or a pipe) in chunk_bytes pieces (0 =
 * 256 MiB) into two page-locked buffers, the next piece while the current one is on the
 * device; each piece's output is written to out_fd while the next piece computes. Neither the
 * input nor the output is ever held whole in host or device memory. *in_bytes / *out_bytes
 * (may be NULL) receive the bytes read and written. Same pair limits as cuda_replace_stream
 * (-7 outside them); -10 when reading or writing failed (errno tells why); -1 for invalid
 * arguments; >0 a cudaError_t. On an error the output file holds a prefix of the result. */
int cuda_replace_stream_fd(int in_fd, int out_fd, const uint8_t** pats, const int* pat_lens,
                           const uint8_t** reps, const int* rep_lens, int count, size_t chunk_bytes,
                           unsigned long long* in_bytes, unsigned long long* out_bytes);

/* Host memcpy on up to 16 threads (large copies): moves a result out of the page-locked
 * block the library returned into memory the caller allocated (in Python: a bytes object
 * created uninitialised), whose first-touch page faults bound a single-threaded copy. No
 * counterpart in the reference. */
void cuda_replace_host_copy(void* dst, const void* src, size_t n);

/* ---- Batched jobs and serving. No counterpart in the reference, whose only batch is the
 * sequential pair chain of one buffer (cuda_replace_apply_batch, cu:2465); a caller with many
 * independent buffers there makes one unified() call per buffer and pair
 * (cuda_replace_wrapper.py:124-141). Here many jobs (each an input and its own sequence of
 * pairs) run together: round r applies every job's r-th pair in one segmented launch per
 * carry class, work split by 16 KiB super-tiles across all jobs, with the rounds replayed from
 * a CUDA graph and lengths passed between rounds on the device. Results equal, per job, the
 * chained bytes.replace. Pairs outside the segmented limits (pattern 1-32 B, replacement up
 * to 64 B, at most 16 pairs per job), and jobs whose output outgrows the buffers planned for
 * them, run through a Session instead; the result is the same. */

/* A server keeps its device memory (an arena of hbm_budget bytes; 0 = 40% of the free
 * memory) for its lifetime. submit() copies the input and pairs, so the caller's buffers may
 * be released when it returns. A dispatcher thread forms a batch whenever one of two batch
 * slots is free, admitting queued requests in arrival order while their device footprint
 * (input + two ping-pong buffers of up to 4x input + 1 MiB) fits the arena; requests that
 * arrive while a batch runs form the next one, which runs beside it. max_jobs_per_batch: 0 =
 * 4096. All calls are thread-safe. */
typedef struct CudaReplaceServerStats {
  unsigned long long jobs_done;         /* since open or the last reset_stats */
  unsigned long long jobs_via_session;  /* of those, run through a Session */
  unsigned long long batches;
  unsigned long long bytes_in, bytes_out;
  unsigned long long kernel_launches;   /* plan + segmented kernels enqueued (in graphs) */
  unsigned long long graph_launches;
  unsigned long long pending;           /* requests queued, not yet on the device */
  unsigned long long arena_bytes, arena_peak_bytes;
  double p50_us, p99_us, max_us;        /* latency: submit() to result ready */
  double gpu_us;                        /* batches on the device: uploads and rounds (CUDA events) */
  double download_us;                   /* result downloads, host wall time */
  double session_us;                    /* jobs run through a Session, host wall time */
  unsigned int tile_bytes[3];           /* autotuned super-tile bytes: free, bordered L<=4, bordered L<=32 */
  int grid_ctas[3];
  unsigned long long cancelled;         /* requests cancelled before they reached the device */
} CudaReplaceServerStats;

int cuda_replace_server_open(void** srv, size_t hbm_budget, int max_jobs_per_batch);
/* -1 NULL arguments or a negative length, -4 a pattern or replacement longer than
 * CUDA_REPLACE_MAX_PATTERN, >0 a cudaError_t. *ticket identifies the request. */
int cuda_replace_server_submit(void* srv, const uint8_t* src, size_t n,
                               const uint8_t** pats, const int* pat_lens,
                               const uint8_t** reps, const int* rep_lens, int count,
                               unsigned long long* ticket);
/* As cuda_replace_server_submit, for a tenant (tenant 0: none). While the tenant's budget (see
 * cuda_replace_server_set_tenant_budget) is in use by its requests on the device, its further
 * requests wait in the queue without holding back other tenants' requests. -9: the request alone
 * needs more device memory than its tenant's budget. */
int cuda_replace_server_submit_tenant(void* srv, unsigned int tenant, const uint8_t* src, size_t n,
                                      const uint8_t** pats, const int* pat_lens,
                                      const uint8_t** reps, const int* rep_lens, int count,
                                      unsigned long long* ticket);
/* Cancel a request that is still queued: returns 0 and its wait then returns -8 (cancelled)
 * with no result; 1 when the request is already on the device, running or done (it completes
 * normally); -1 for an unknown ticket. */
int cuda_replace_server_cancel(void* srv, unsigned long long ticket);
/* Device memory (bytes of the server's arena) that requests of tenant (>= 1) may hold at once;
 * 0 removes the limit. Requests of a tenant without a budget share the whole arena. Requests
 * that run through a Session instead of a batch use no arena memory and are not counted. */
int cuda_replace_server_set_tenant_budget(void* srv, unsigned int tenant, size_t bytes);
/* Arena bytes held by a tenant's requests now and at most since the server opened. */
int cuda_replace_server_tenant_usage(void* srv, unsigned int tenant, unsigned long long* in_use,
                                     unsigned long long* peak);
/* 0: done; *out_host (page-locked, release with cuda_free_host; NULL when empty) and
 * *out_len receive the result and the ticket is retired. 1: not done within timeout_ms
 * (negative: wait without limit). -1: unknown ticket. -8: cancelled (retired, no result).
 * Other: the request's error code. */
int cuda_replace_server_wait(void* srv, unsigned long long ticket, int timeout_ms,
                             uint8_t** out_host, size_t* out_len);
int cuda_replace_server_stats(void* srv, CudaReplaceServerStats* stats);
int cuda_replace_server_reset_stats(void* srv);
/* Finishes every submitted request, then releases the server. */
void cuda_replace_server_close(void* srv);

/* One call for many jobs: job i is srcs[i][0, src_lens[i]) with pair_counts[i] pairs, the
 * pairs of all jobs concatenated in pats/pat_lens/reps/rep_lens. out_hosts[i] / out_lens[i]
 * receive job i's result (release each with cuda_free_host). Runs on one server per device that
 * every call shares: opened by the first call with device memory for its inputs (about nine
 * bytes per input byte, at least 256 MiB, at most 40% of the free memory) and reopened larger
 * when a later call needs more; calls are serialised. On an error no result is returned. */
int cuda_replace_jobs(int njobs, const uint8_t** srcs, const size_t* src_lens, const int* pair_counts,
                      const uint8_t** pats, const int* pat_lens, const uint8_t** reps, const int* rep_lens,
                      uint8_t** out_hosts, size_t* out_lens);
/* Close the server that cuda_replace_jobs keeps and release its device and page-locked memory
 * (the next call opens a new one). */
void cuda_replace_jobs_release(void);

#ifdef __cplusplus
}
#endif

#endif /* CUDA_REPLACE_H */
