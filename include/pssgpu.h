/*
 * pssgpu.h -- C ABI of the B200 string sample sort (libpssgpu.so).
 *
 * The library sorts NUL-terminated byte strings on one NVIDIA B200 and
 * optionally emits the LCP array. Its results equal those of the reference
 * pS5 (bingmann/parallel-string-sorting, "pS5-Unroll",
 * src/parallel/bingmann-parallel_sample_sort.cpp:31-42): the same sorted
 * string sequence and the same LCP array; only the order of pointers to
 * equal strings may differ.
 *
 * String model (the reference's UCharStringSet, src/tools/stringset.hpp):
 * a string is the bytes from its start up to its first NUL; comparison is
 * unsigned bytewise (strcmp). LCP convention (src/tools/stringptr.hpp:
 * 977-1046): lcp[i] = number of chars shared by sorted strings i-1 and i,
 * for i >= 1; lcp[0] is never written.
 *
 * All entry points are thread-safe. Errors are returned as a status code;
 * pssgpu_last_error() gives the message of the calling thread's last error.
 * The drop-in pointer-array entry points (the psstest contestant signatures)
 * have no error channel in the reference, so they abort() with the message on
 * stderr, which psstest --fork reports as status=aborted
 * (src/psstest.cpp:341-369).
 */
#ifndef PSSGPU_H
#define PSSGPU_H

#include <stddef.h>
#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

/* ---- status codes ------------------------------------------------------ */
#define PSSGPU_OK 0
#define PSSGPU_EINVAL 1   /* bad argument: sizes, alignment, unterminated arena */
#define PSSGPU_ENOMEM 2   /* device or host allocation failed */
#define PSSGPU_ECUDA 3    /* a CUDA runtime call failed */
#define PSSGPU_ETIMEOUT 4 /* a bounded wait or the pass limit of a sort gave up */
#define PSSGPU_ENODEV 5   /* no usable CUDA device */
#define PSSGPU_EBUDGET 6  /* request exceeds the configured memory budget */

/* Device arenas must stay readable this many bytes past their last char. */
#define PSSGPU_ARENA_PAD 16

/* Largest string count one call accepts (ids are 32-bit). */
#define PSSGPU_MAX_STRINGS 0xFFFFFFF0u

const char* pssgpu_last_error(void);
const char* pssgpu_version(void);

/* ---- contexts ------------------------------------------------------------
 * A context owns a CUDA stream and a device workspace that grows to the
 * largest sort seen and is reused. Calls on one context are serialised by
 * its mutex; separate contexts run concurrently. */
typedef struct pssgpu_ctx pssgpu_ctx;

int pssgpu_ctx_create(int device, pssgpu_ctx** out);
void pssgpu_ctx_destroy(pssgpu_ctx* ctx);
/* Bytes of device workspace a sort of n strings needs (excluding inputs and
 * outputs). */
uint64_t pssgpu_workspace_bytes(uint64_t n);

/* Statistics of the last sort on a context (all counts, device ms). */
typedef struct pssgpu_stats {
    uint32_t passes;          /* big-segment sample-sort passes */
    uint32_t kernel_launches; /* kernels launched by the last sort */
    uint64_t big_elements;    /* sum over passes of strings in big segments */
    uint64_t small_segments;  /* segments finished by the small-sort kernel */
    uint64_t boundaries;      /* split boundaries whose LCP was set at the end */
    float device_ms;          /* device time of the last sort (events) */
} pssgpu_stats;
int pssgpu_ctx_stats(pssgpu_ctx* ctx, pssgpu_stats* out);

/* Per-kernel-class figures of the last sort: launches, strings processed,
 * algorithmic bytes (per-string model: key gather 4 id + 8 chars + 8 key,
 * classify 8 key, scatter 12 + 12, base case 12 + output) and, in profile
 * mode, summed device time from CUDA events around each class. Returns the
 * number of entries written (at most max), or a negative status. */
typedef struct pssgpu_kernel_stats {
    char name[16];
    uint32_t launches;
    uint64_t strings;
    uint64_t alg_bytes;
    double ms;
} pssgpu_kernel_stats;
int pssgpu_ctx_set_profile(pssgpu_ctx* ctx, int on);
int pssgpu_ctx_kernel_stats(pssgpu_ctx* ctx, pssgpu_kernel_stats* out, int max);

/* Context options. PSSGPU_OPT_PROFILE: as pssgpu_ctx_set_profile.
 * PSSGPU_OPT_INDIRECT_HANDLES: carry bare string ids through the sort and
 * read offsets from the offset array at every gather -- the path a sort takes
 * on its own when an id and an arena offset do not fit one 64-bit handle,
 * and a merge when the arena exceeds 4 GiB; for testing those paths on small
 * inputs.
 * PSSGPU_OPT_SINGLE_LAUNCH (default 1): a single-instance sort whose strings
 * fit one wave of resident blocks (about 1.2 M strings on a B200) runs as one
 * cooperative kernel launch, with no host round trip between its steps;
 * 0 sends every sort through the multi-launch pass loop.
 * PSSGPU_OPT_WAIT_LIMIT (default 4,194,304): polls of a grid-barrier wait in
 * that kernel before it gives up and the sort returns PSSGPU_ETIMEOUT.
 * PSSGPU_OPT_MERGE_PIECE (1..4096; by default chosen per merge, 64..256,
 * so that the pieces fill whole waves of the GPU's resident merge threads):
 * outputs one GPU thread merges in each round of pssgpu_merge_lcp_device.
 * PSSGPU_OPT_SUFFIX_DOUBLING (default 1): when the strings of a sort are all
 * suffixes of one text (n == nchars, offs[i] == i, no NUL before the last
 * char: psstest --suffix, src/psstest.cpp:502-518), groups that share 8 or
 * more chars are finished by prefix doubling on suffix ranks instead of
 * deeper string passes; the output is the same. 0: sort them as strings. */
#define PSSGPU_OPT_PROFILE 1
#define PSSGPU_OPT_INDIRECT_HANDLES 2
#define PSSGPU_OPT_SINGLE_LAUNCH 3
#define PSSGPU_OPT_WAIT_LIMIT 4
#define PSSGPU_OPT_MERGE_PIECE 5
#define PSSGPU_OPT_SUFFIX_DOUBLING 6
int pssgpu_ctx_set_option(pssgpu_ctx* ctx, int option, int64_t value);

/* ---- arena sorts ---------------------------------------------------------
 * chars[0, nchars) holds the strings; string i starts at chars + offs[i] and
 * ends at its first NUL, which must lie inside the arena (chars[nchars-1]
 * must be 0). Outputs: perm[r] = id of the r-th smallest string; lcp (may be
 * NULL) as in the LCP convention above (lcp[0] untouched).
 *
 * pssgpu_sort_host: host buffers; the call copies the arena and offsets to
 * the device, sorts, and copies perm/lcp back. Replaces the body of a
 * psstest contestant run (src/psstest.cpp:387-403) for an arena input.
 * Offsets of 2^20 or more strings that never decrease, with every gap below
 * 65536 (strings laid out in order), cross PCIe as 1- or 2-byte gaps,
 * computed by host threads while the arena is copied, and are rebuilt on the
 * device; other offset arrays are copied as they are. The result is the same
 * either way. Pinned host buffers let the copies overlap the host work.
 *
 * pssgpu_sort_device: device buffers on the context's device. d_chars must
 * be 8-byte aligned and readable for nchars + PSSGPU_ARENA_PAD bytes (the
 * kernels read whole 16-byte blocks, so the block holding d_chars[0] is read
 * from its start: any device allocation satisfies this);
 * `stream` is a cudaStream_t or NULL for the context's stream, which orders
 * with the legacy default stream (work the caller queued there before the
 * call is done before the sort starts). The call returns after the sort has
 * completed. */
int pssgpu_sort_host(pssgpu_ctx* ctx, const uint8_t* chars, uint64_t nchars,
                     const uint64_t* offs, uint64_t n, uint32_t* perm,
                     uint32_t* lcp);
int pssgpu_sort_device(pssgpu_ctx* ctx, const uint8_t* d_chars,
                       uint64_t nchars, const uint64_t* d_offs, uint64_t n,
                       uint32_t* d_perm, uint32_t* d_lcp, void* stream);

/* ---- device-side input preparation ---------------------------------------
 * A text becomes an arena and its offset array on the device, as psstest's
 * plain-file loader and pointer-array build do it on the host
 * (src/tools/input.hpp:255-297, src/psstest.cpp:479-518):
 *   PSSGPU_TEXT_LINES     every '\n' and NUL byte ends a string and becomes
 *                         NUL; n = 1 + such bytes in text[0, size - 1)
 *   PSSGPU_TEXT_SUFFIXES  every position starts a string; n = size
 * Both force the last byte, text[size - 1], to NUL.
 *
 * pssgpu_prepare_text_device: in place on device buffers. d_text must be
 * 8-byte aligned, readable and writable for size + PSSGPU_ARENA_PAD bytes,
 * the pad bytes zero. d_offs receives the n offsets. *n_out is set to n; if
 * n exceeds offs_cap the call returns PSSGPU_EINVAL and changes nothing. The
 * result sorts with pssgpu_sort_device(ctx, d_text, size, d_offs, n, ...).
 *
 * pssgpu_sort_text_host: copies the host text (size bytes, left unchanged)
 * to the device, prepares it there and sorts it: perm receives the string
 * ids (their order in the text), lcp (may be NULL) the LCP array, both for
 * the n strings; cap is their capacity (n > cap: PSSGPU_EINVAL with *n_out =
 * n, nothing written). No counterpart in the reference's sorter interface:
 * it replaces psstest's loading and pointer-array steps before a run. */
#define PSSGPU_TEXT_LINES 0
#define PSSGPU_TEXT_SUFFIXES 1
int pssgpu_prepare_text_device(pssgpu_ctx* ctx, uint8_t* d_text, uint64_t size,
                               int mode, uint64_t* d_offs, uint64_t offs_cap,
                               uint64_t* n_out, void* stream);
int pssgpu_sort_text_host(pssgpu_ctx* ctx, const uint8_t* text, uint64_t size,
                          int mode, uint32_t* perm, uint32_t* lcp, uint64_t cap,
                          uint64_t* n_out);

/* ---- merge of sorted runs ---------------------------------------------------
 * pssgpu_merge_lcp_device merges nruns sorted runs of one arena into one
 * sorted sequence with its LCP array: the step after per-shard sorts that
 * the reference takes in its top-level merge of per-NUMA-node pS5 outputs
 * (src/parallel/eberle-ps5-parallel-toplevel-merge.hpp:56-175 with the
 * LCP-aware K-way merge of src/parallel/eberle-parallel-lcp-merge*.hpp).
 * runs: host array of nruns + 1 boundaries into d_ids / d_lcp (runs[0] = 0,
 * non-decreasing, runs[nruns] = n); run k is d_ids[runs[k], runs[k+1]),
 * sorted, with d_lcp[q] the LCP of d_ids[q - 1] and d_ids[q] inside the run
 * (the entry at a run's first position is ignored). d_ids_out receives the
 * merged ids (equal strings keep the order of their runs), d_lcp_out (may be
 * NULL; then d_lcp may be NULL too) its LCP array with d_lcp_out[0] left
 * unchanged. Outputs must not overlap the inputs. All device buffers are on
 * the context's device; the arena rules of pssgpu_sort_device apply. Every
 * id in d_ids must index d_offs (the call cannot check that: it does not
 * know the length of d_offs); an offset outside the arena returns
 * PSSGPU_EINVAL, with d_ids_out / d_lcp_out unspecified. With d_lcp the
 * merge is LCP-aware (compares start at the known common prefix, and each
 * run head carries the next 7 chars from there). The context keeps about
 * 40 bytes per string of merge scratch (entries, LCPs and char caches, two
 * of each) between calls. */
int pssgpu_merge_lcp_device(pssgpu_ctx* ctx, const uint8_t* d_chars, uint64_t nchars,
                            const uint64_t* d_offs, const uint64_t* runs, uint32_t nruns,
                            const uint32_t* d_ids, const uint32_t* d_lcp,
                            uint32_t* d_ids_out, uint32_t* d_lcp_out, void* stream);

/* ---- batched sorts ---------------------------------------------------------
 * Many independent sort instances in one call: every instance becomes a
 * root segment of the same device passes, so instances of any size share
 * the kernel launches. Instance k owns strings [inst[k], inst[k+1]) of the
 * offset array (inst is a host array of ninst + 1 entries, inst[0] = 0,
 * non-decreasing, inst[ninst] = n). On return perm[p] for p in
 * [inst[k], inst[k+1]) is a string id of instance k counted from 0, i.e. the
 * instance's own permutation; lcp (may be NULL) holds each instance's LCP
 * array with its first entry written as 0. No counterpart in the reference,
 * which sorts one string set per call. */
int pssgpu_sort_batch_host(pssgpu_ctx* ctx, const uint8_t* chars, uint64_t nchars,
                           const uint64_t* offs, const uint64_t* inst, uint32_t ninst,
                           uint32_t* perm, uint32_t* lcp);
int pssgpu_sort_batch_device(pssgpu_ctx* ctx, const uint8_t* d_chars, uint64_t nchars,
                             const uint64_t* d_offs, const uint64_t* inst, uint32_t ninst,
                             uint32_t* d_perm, uint32_t* d_lcp, void* stream);

/* Tuning table: splitter-tree levels (1..10) for big segments of
 * 2^k .. 2^(k+1)-1 strings, k < count <= 33; 0 keeps the default rule
 * (about 8 strings per bucket). Written by the autotuner. */
int pssgpu_ctx_set_tree_bits(pssgpu_ctx* ctx, const uint8_t* tree_bits, int count);

/* ---- serving ---------------------------------------------------------------
 * A request server with continuous batching; no counterpart in the
 * reference. hbm_budget bounds all device memory the server holds: every
 * worker reserves a workspace for max_batch_strings strings, the rest is a
 * slab that keeps admitted requests' arenas and offsets resident. submit()
 * only queues the request and returns a ticket; an admission thread admits
 * requests in arrival order as slab space frees up, and each worker sorts
 * all admitted requests it can take (up to max_batch_strings strings and
 * max_batch_requests requests, 0 = 4096) as one batch on its own stream, so
 * requests arriving while others run join the next batch and the workers'
 * batches overlap on the device. Results are written to the caller's perm
 * and lcp (may be NULL; lcp[0] untouched) before wait() returns; the caller
 * keeps chars, offs and the outputs alive until then. String i of a request
 * starts at chars + (offs[i] - offs_base). */
typedef struct pssgpu_server pssgpu_server;
typedef struct pssgpu_server_config {
    uint64_t hbm_budget;
    uint64_t max_batch_strings;
    uint32_t workers;
    uint32_t max_batch_requests;
} pssgpu_server_config;
typedef struct pssgpu_request_info {
    int status;
    uint32_t batch_requests;  /* requests sorted in the same batch */
    uint64_t batch_strings;   /* strings in that batch */
    uint64_t t_submit_ns, t_admit_ns, t_start_ns, t_done_ns;  /* steady clock */
} pssgpu_request_info;
typedef struct pssgpu_server_stats {
    uint64_t slab_bytes, slab_peak_bytes;
    uint64_t batches, batched_requests;
    uint64_t pending, ready;
} pssgpu_server_stats;
int pssgpu_server_create(int device, const pssgpu_server_config* cfg, pssgpu_server** out);
void pssgpu_server_destroy(pssgpu_server* srv);
int pssgpu_server_submit(pssgpu_server* srv, const uint8_t* chars, uint64_t nchars,
                         const uint64_t* offs, uint64_t offs_base, uint64_t n,
                         uint32_t* perm, uint32_t* lcp, uint64_t* ticket);
int pssgpu_server_wait(pssgpu_server* srv, uint64_t ticket, pssgpu_request_info* info);
int pssgpu_server_get_stats(pssgpu_server* srv, pssgpu_server_stats* out);

/* ---- psstest Contest drop-ins --------------------------------------------
 * The three contestant signatures of Contestant_UCArray
 * (src/tools/contest.hpp:88-91). Each permutes `strings` in place into
 * sorted order exactly as the reference's
 * parallel_sample_sortBTCUI (bingmann-parallel_sample_sort.cpp:31-37) and
 * parallel_sample_sort_lcp_base (bingmann-parallel_sample_sort.hpp:1733-1748)
 * do, never writes the characters, and uses the default context of device 0.
 * lcp[0] is left untouched; cache[i] = strings[i][lcp[i]] for i >= 1
 * (verify_lcp_cache, src/tools/stringptr.hpp:977-1033). On failure they
 * abort(). The _status variants return the status code instead.
 * These entry points read each string from its own pointer (strlen, then a
 * copy of its bytes), so the strings may live in separate allocations. */
void pssgpu_sort_strings(unsigned char** strings, size_t n);
void pssgpu_sort_strings_lcp(unsigned char** strings, uintptr_t* lcp, size_t n);
void pssgpu_sort_strings_lcp_cache(uint8_t** strings, uintptr_t* lcp,
                                   uint8_t* cache, size_t n);
int pssgpu_sort_strings_status(unsigned char** strings, uintptr_t* lcp,
                               uint8_t* cache, size_t n);

/* Separate-output variant: the sorted pointers go to output[0, n) and
 * strings[] is left unchanged. Replaces parallel_sample_sort_out_base
 * (bingmann-parallel_sample_sort.hpp:1704-1714) behind the reference's
 * parallel_sample_sortBTCUI_out contestant
 * (bingmann-parallel_sample_sort.cpp:44-62), whose input array serves as
 * scratch. output must not overlap strings (output == strings sorts in
 * place). */
void pssgpu_sort_strings_out(unsigned char** strings, unsigned char** output, size_t n);
int pssgpu_sort_strings_out_status(unsigned char** strings, unsigned char** output,
                                   size_t n);

/* The pointer-array sort for strings that all lie in one caller-owned buffer,
 * as psstest's string data does (g_string_data / g_string_datasize,
 * src/psstest.cpp:87-88, which the reference's own contestants declare extern,
 * src/sinha-copy-burstsort/glue.cpp:33-34). The caller vouches that every
 * strings[i] and the NUL ending it lie in arena[0, arena_size); a pointer
 * outside returns PSSGPU_EINVAL. Only the span from the lowest string pointer
 * to the end of the highest string is read, and it is copied to the device
 * in one piece, with no per-string host work. output: NULL sorts strings in
 * place; otherwise as pssgpu_sort_strings_out. lcp and cache (both may be
 * NULL) as for pssgpu_sort_strings_lcp_cache, indexed by sorted position.
 * Returns a status code. */
int pssgpu_sort_strings_arena(const uint8_t* arena, uint64_t arena_size,
                              unsigned char** strings, unsigned char** output,
                              uintptr_t* lcp, uint8_t* cache, size_t n);

/* ---- allocation-free sort --------------------------------------------------
 * No counterpart in the reference. Sorts at most PSSGPU_NOALLOC_MAX_STRINGS
 * strings on the current device and allocates nothing: no cudaMalloc, no
 * cudaFree, no allocating library call, no context. It exists for callers
 * that cannot allocate device memory: a plugin inside a host application
 * that owns all device memory through its own pool and forbids other
 * allocations, a latency-critical path that cannot afford cudaMalloc's
 * implicit device synchronisation, or a process whose device memory is
 * already fully reserved. Inputs and outputs are caller-owned device buffers
 * exactly as for pssgpu_sort_device; `stream` is a cudaStream_t (NULL: the
 * default stream); the call returns after the sort has completed.
 * Scratch is one file-scope device array of 16,528 bytes inside the library,
 * held by every device that loads the library until the process exits. All
 * calls share it: calls whose GPU work overlaps (other streams, other host
 * threads) race on it, so the caller must serialise them. The first call on
 * a device looks up the array's device address and raises the kernel's
 * shared-memory limit; make that first call before any stream capture. Both
 * are kept for the life of the process, so calls after a cudaDeviceReset of
 * that device are not supported.
 * More than PSSGPU_NOALLOC_MAX_STRINGS strings returns PSSGPU_EINVAL. When a
 * call fails (an offset outside the arena: PSSGPU_EINVAL), d_perm and d_lcp
 * hold unspecified values. */
#define PSSGPU_NOALLOC_MAX_STRINGS 2048
int pssgpu_sort_device_noalloc(const uint8_t* d_chars, uint64_t nchars,
                               const uint64_t* d_offs, uint64_t n,
                               uint32_t* d_perm, uint32_t* d_lcp, void* stream);

#ifdef __cplusplus
}
#endif

#endif /* PSSGPU_H */
