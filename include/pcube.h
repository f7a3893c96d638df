/*
 * libpcube: B200 (sm_100a) kernels for the doubly-focused pseudocube sieve, behind a plain C ABI.
 *
 * Every integer is uint64_t unless stated; every pointer argument is host memory owned by the
 * caller unless the name says "device".  Device memory is owned by the library and reached
 * through opaque handles.  One host thread per context; every context owns one CUDA stream and
 * all of its work is ordered on it.  Calls block until their results are on the host.
 *
 * The reference project reaches the same path through CuPy objects; each entry point below
 * names the reference interface it replaces (file:line inside the reference project).
 *
 * Return codes (the Python layer maps them to the reference's exception types):
 */
#ifndef PCUBE_H
#define PCUBE_H
#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

#define PC_OK 0          /* success */
#define PC_OVERFLOW 1    /* output or window capacity exceeded -> OverflowError; no partial results */
#define PC_INVALID 2     /* invalid arguments -> ValueError */
#define PC_ARITHMETIC 3  /* underflow flag or an inconsistent device result -> ArithmeticError */
#define PC_TIMEOUT 4     /* deadline passed -> TimeoutError('BUDGET_EXHAUSTED') */
#define PC_NOMEM 5       /* device memory cap exceeded -> MemoryError */
#define PC_CUDA 6        /* CUDA runtime error (message in pc_last_error) -> RuntimeError */

typedef struct pc_ctx pc_ctx;         /* device, stream, memory accounting */
typedef struct pc_focus pc_focus;     /* device-resident wheel tables of one focus modulus */
typedef struct pc_filters pc_filters; /* residual filter tables of one (p, A, B) */
typedef struct pc_buf pc_buf;         /* device array of uint64 (a sorted focus window) */

/* Library / device queries. */
int pc_version(void);
int pc_device_count(int *count);
const char *pc_last_error(const pc_ctx *ctx);

/* Context: replaces Runtime.__init__/check (pseudocube/gpu.py:38-52).  The cap is
 * min(mem_cap, fraction * total, free - 256 MiB) as the reference computes it. */
int pc_init(int device, uint64_t mem_cap, double fraction, pc_ctx **out);
int pc_free(pc_ctx *ctx);
int pc_mem_info(const pc_ctx *ctx, uint64_t *in_use, uint64_t *peak, uint64_t *cap);
/* Bytes the library has copied from the host to the device and back on this context so far
 * (the reference's Runtime keeps no such count; a caller takes differences around any sequence
 * of calls, e.g. a window plan and its run). */
int pc_copy_info(const pc_ctx *ctx, uint64_t *h2d, uint64_t *d2h);
int pc_device_info(const pc_ctx *ctx, int *sm_count, int *cc_major, int *cc_minor, char *name, int name_len);

/* Page-locked host memory for result buffers (counts, geometry, outputs): device-to-host copies
 * into it run at full link speed instead of through the driver's staging.  PC_NOMEM when it cannot
 * be had; free with pc_host_free (which waits for the device). */
int pc_host_alloc(uint64_t bytes, void **out);
int pc_host_free(void *p);
int pc_sync(pc_ctx *ctx);
/* Device timestamps on the context's stream (slot 0..7) and the milliseconds between two. */
int pc_mark(pc_ctx *ctx, int slot);
int pc_elapsed(pc_ctx *ctx, int from_slot, int to_slot, double *ms);

/* Device buffers of uint64. */
int pc_buf_upload(pc_ctx *ctx, const uint64_t *host, uint64_t n, pc_buf **out);
int pc_buf_download(pc_ctx *ctx, const pc_buf *buf, uint64_t offset, uint64_t n, uint64_t *host);
int pc_buf_size(const pc_buf *buf, uint64_t *n);
int pc_buf_free(pc_ctx *ctx, pc_buf *buf);
/* searchsorted(left) of n sorted host queries in a sorted device buffer
 * (replaces cp.searchsorted, pseudocube/batch_experiment.py:41-42). */
int pc_buf_searchsorted(pc_ctx *ctx, const pc_buf *buf, const uint64_t *queries, uint64_t n, uint64_t *positions);

/* Focus wheel tables: replaces GPUFocus.__init__ + partial (pseudocube/gpu.py:70-92).
 * rings: nrings prime-power moduli q[k] with counts[k] coefficient-adjusted allowed residues,
 * concatenated in residues[].  M = product of q[k] < 2^63.  table_budget bounds the bytes of the
 * device tables (0 = library default). */
int pc_focus_create(pc_ctx *ctx, uint64_t M, uint32_t nrings, const uint32_t *q, const uint32_t *counts,
                    const uint32_t *residues, uint64_t table_budget, pc_focus **out);
int pc_focus_free(pc_ctx *ctx, pc_focus *focus);
/* info[0..7]: M, M1 (wheel modulus), wheel entries, number of bitset rings, table bytes,
 * focus count low 64 bits, focus count high 64 bits, wheel build milliseconds */
int pc_focus_info(const pc_focus *focus, uint64_t *info);

/* Sorted focus values in [low, high): replaces GPUFocus.window (pseudocube/gpu.py:94-114).
 * PC_OVERFLOW if more than cap values or more than 4096 periods of M. */
int pc_focus_window(pc_ctx *ctx, const pc_focus *focus, uint64_t low, uint64_t high, uint64_t cap,
                    pc_buf **out, uint64_t *count);

/* Residual filters of one (p, A, B): replaces the generated tables of match_source and the
 * mask_build sources (pseudocube/gpu.py:129-146, pseudocube/batch_experiment.py:175-196).
 * primes: the residual filters in the reference order (9, then q = 1 mod 3, then the rest, each
 * ascending); allowed: concatenated byte tables (q bytes each, 1 = allowed residue). */
int pc_filters_create(pc_ctx *ctx, uint64_t A, uint64_t B, const uint32_t *primes, uint32_t nres,
                      const uint8_t *allowed, pc_filters **out);
int pc_filters_free(pc_ctx *ctx, pc_filters *filters);

/* Tunables of the batch kernel (all optional: 0 selects the library default). */
typedef struct pc_tuning {
    uint32_t bitset_filters;   /* residual filters intersected as bitsets (1..8, >= min(4, nres)) */
    uint32_t block_words;      /* u words (32 u each) staged per CTA: 16, 32 or 64 */
    uint32_t words_per_thread; /* ignored: a lane walks all block_words words of its (v row, block) piece */
    uint32_t v_chunk;          /* v rows per work item (0 = total pieces / (32 x SMs), at least 4 x threads) */
    uint32_t threads;          /* threads per CTA: 512, 768, 896 or 1024 (0: 896, stepping down to fit) */
    uint32_t deep_records;     /* survivor buffer: deep records per CTA slice (0 = 32768); a run that
                                  needs more reruns once with room for every record */
    uint32_t reserved[2];
} pc_tuning;

/* Per-call statistics. */
typedef struct pc_stats {
    double kernel_ms;          /* batch kernel (stages 2+3) device time */
    double bounds_ms;          /* per-v bounds + residues */
    double window_ms;          /* stage-1 windows (lease calls only) */
    double total_ms;           /* device time of the whole call */
    uint64_t work_items;
    uint64_t outputs;
    uint64_t launches;         /* kernels launched by the call */
    uint64_t reserved[5];      /* [0..3]: bitset filters, block words, threads and cheap-tier
                                  filters the call used; [4]: 1 when a recorded graph ran */
    uint64_t h2d_bytes;        /* bytes the call copied from the host to the device */
    uint64_t d2h_bytes;        /* bytes the call copied from the device to the host */
} pc_stats;

/*
 * One fused batch over the sorted focus lists us[u_off, u_off+nu) and vs[v_off, v_off+nv):
 * replaces MaskedMatcher.run's device half (pseudocube/batch_experiment.py:104-135, 239-248).
 * Subtile of v = (v - v_first) / width; ntiles subtiles.  lo/hi: the 128-bit interval (lo, hi]
 * as two limbs.
 * counts   [ntiles x (ng+3)] out: focused positions, ng group survivors, outputs, underflows
 * geometry [ntiles x 2]      out: u count and v count of each subtile's envelope (the
 *                            reference's searchsorted bounds, batch_experiment.py:37-43)
 * out      [out_cap x 2]     out: emitted x (limb 0, limb 1 | subtile << 32), unordered
 * PC_OVERFLOW if more than out_cap values were emitted (counts are still complete).
 */
int pc_run_batch(pc_ctx *ctx, const pc_filters *filters, const pc_tuning *tuning,
                 const pc_buf *us, uint64_t u_off, uint64_t nu, const pc_buf *vs, uint64_t v_off, uint64_t nv,
                 uint64_t lo0, uint64_t lo1, uint64_t hi0, uint64_t hi1,
                 uint64_t v_first, uint64_t width, uint32_t ntiles, uint64_t v_end,
                 uint64_t *counts, uint64_t *geometry, uint64_t *out, uint64_t out_cap, uint64_t *n_out,
                 pc_stats *stats);

/*
 * Whole lease [first, end) in one call: windows of both focuses from the device-resident
 * wheels, then the fused kernel over every subtile of width `width`; replaces the device side
 * of compute_lease (pseudocube/optimized.py:81-90) for MaskedMatcher.  Same output layouts
 * as pc_run_batch with ntiles = ceil((end-first)/width).
 */
int pc_run_lease(pc_ctx *ctx, const pc_focus *fa, const pc_focus *fb, const pc_filters *filters,
                 const pc_tuning *tuning, uint64_t first, uint64_t end, uint64_t width,
                 uint64_t lo0, uint64_t lo1, uint64_t hi0, uint64_t hi1,
                 uint64_t *counts, uint64_t *geometry, uint64_t *out, uint64_t out_cap, uint64_t *n_out,
                 pc_stats *stats);

/*
 * pc_run_lease over leases [first[i], end[i]), i < n, one after another on the calling thread,
 * each with its own counts[i], geometry[i] and out[i] (out_cap records) as pc_run_lease.  status[i]
 * is set to 1 + the lease's return code once its results are on the host (a release store), so a
 * second host thread may consume lease i while later leases run; the call stops at, and returns the
 * code of, the first lease that fails.  stats may be NULL.  A worker that commits lease after lease
 * (pseudocube/multi.py:197-272) calls this from a helper thread instead of compute_lease per lease.
 */
int pc_run_leases(pc_ctx *ctx, const pc_focus *fa, const pc_focus *fb, const pc_filters *filters,
                  const pc_tuning *tuning, uint32_t n, const uint64_t *first, const uint64_t *end, uint64_t width,
                  uint64_t lo0, uint64_t lo1, uint64_t hi0, uint64_t hi1, uint64_t *const *counts,
                  uint64_t *const *geometry, uint64_t *const *out, uint64_t out_cap, uint64_t *n_out,
                  pc_stats *stats, int32_t *status);

/* Flags of pc_multi_run. */
#define PC_RUN_GRAPH 1u   /* record the run into a CUDA graph once, then replay it on every call */

/* One window of a multi-window launch. */
typedef struct pc_window {
    uint64_t first, end;          /* canonical v range [first, end) */
    uint64_t width;               /* subtile width in v */
    uint64_t lo0, lo1, hi0, hi1;  /* interval (lo, hi] as two limbs each, hi < 2^96 */
    uint32_t focus_a, focus_b;    /* indices into the focus array (moduli A and B of the family) */
    uint32_t family;              /* index into the filter-family array */
    uint32_t reserved;
} pc_window;

typedef struct pc_multi pc_multi;   /* planned multi-window launch with its device buffers */

/*
 * Many windows in one launch sequence, each with its own interval, v range, subtile width, focus
 * pair and filter family (prime bound): the batched form of compute_lease and of Matcher.tile
 * over many tiles (pseudocube/optimized.py:81-90, pseudocube/gpu.py:212-234), for which the
 * reference has no single call.  pc_multi_create plans the u and v windows of every window and
 * sizes every device buffer (out_cap output records in all); pc_multi_run regenerates the windows
 * on the device and runs stages 2 and 3 over all of them.  With PC_RUN_GRAPH the first call runs
 * eagerly, records the whole sequence into a CUDA graph and replays it; later calls replay only.
 * Families sharing a launch must admit one bitset filter count (every family's first four
 * filters fit bitset rows).  Results are bit-identical to one pc_run_lease per window.
 */
int pc_multi_create(pc_ctx *ctx, const pc_focus *const *foci, uint32_t nfoci, const pc_filters *const *families,
                    uint32_t nfam, const pc_window *windows, uint32_t nwin, const pc_tuning *tuning,
                    uint64_t out_cap, pc_multi **out);
int pc_multi_run(pc_ctx *ctx, pc_multi *m, uint32_t flags, pc_stats *stats);
/* tile_base [nwin+1]: first subtile of each window; sizes [nwin x 2]: u and v list lengths;
 * info[0..7]: subtiles, counters per subtile (stride), padded u entries, v entries, deep slice
 * capacity, bitset filters, block words, threads. */
int pc_multi_layout(const pc_multi *m, uint32_t *tile_base, uint64_t *sizes, uint64_t *info);
/* Results of the last run: counts [subtiles x stride] (focused positions, the ng group survivors
 * of the window's family, outputs, underflows), geometry [subtiles x 2], out [min(n_out, out_cap)
 * x 2] with the global subtile in the high half of limb 1, as pc_run_batch. */
int pc_multi_results(pc_ctx *ctx, const pc_multi *m, uint64_t *counts, uint64_t *geometry, uint64_t *out,
                     uint64_t out_cap, uint64_t *n_out);
int pc_multi_free(pc_ctx *ctx, pc_multi *m);

/*
 * Plain per-position matcher over one tile: replaces Matcher.arrays' kernel (pseudocube/gpu.py:
 * 147-182, 199-210).  Every residual filter is tested per position; counts [ng+3]; out [out_cap x 2].
 */
int pc_run_plain(pc_ctx *ctx, const pc_filters *filters, const pc_buf *us, uint64_t u_off, uint64_t nu,
                 const pc_buf *vs, uint64_t v_off, uint64_t nv, uint64_t lo0, uint64_t lo1, uint64_t hi0,
                 uint64_t hi1, uint64_t *counts, uint64_t *out, uint64_t out_cap, pc_stats *stats);

/*
 * Plain per-tile matcher that allocates no device memory (no counterpart in the reference).
 * For callers that cannot call cudaMalloc: code embedded in a process whose own allocator has
 * already taken the device's memory (a pool sized to the whole GPU leaves nothing for a library
 * to allocate), and code that must not pay cudaMalloc's implicit device synchronisation in the
 * middle of other work.  Same result as pc_run_plain with host inputs: us[nu], vs[nv] (sorted
 * focus values of one tile), the residual filters as for pc_filters_create (primes and allowed
 * must not be NULL), counts [ng+3] and out [out_cap x 2] on the host (out may be NULL only when
 * out_cap is 0).  Its scratch is a 16 MiB static device array inside the library, held by every
 * GPU that loads it until the process exits: inputs, filter tables and outputs must fit in it
 * (at most 2^21 u or v entries, 2^20 output records, and their sum with the tables within
 * 16 MiB), or the call returns PC_INVALID with the reason in err before touching the device.
 * The first call on a device looks up the array's device address (cudaGetSymbolAddress) with
 * that device current and caches it; make that first call before any stream capture, and do not
 * call the entry point again on a device the process has reset.  The call selects `device` for
 * its own work and restores the caller's current device before it returns.  It works on the
 * legacy default stream and clears the counters it reads; every call reuses the same array, so
 * calls that overlap on one GPU race with each other.  err (err_len bytes, may be NULL) receives
 * a message on failure.
 */
int pc_run_plain_static(int device, const uint64_t *us, uint64_t nu, const uint64_t *vs, uint64_t nv,
                        uint64_t A, uint64_t B, uint64_t lo0, uint64_t lo1, uint64_t hi0, uint64_t hi1,
                        const uint32_t *primes, uint32_t nres, const uint8_t *allowed, uint64_t *counts,
                        uint64_t *out, uint64_t out_cap, char *err, int err_len);

/*
 * Canonical JSON of the subtile scopes of consecutive batches, concatenated in batch order: the
 * bytes a lease transcript hashes (encoded(subtile_scopes) per batch, pseudocube/accounting.py:17-28,
 * scopes as built at pseudocube/batch_experiment.py:145-157, hashed at pseudocube/optimized.py:61).
 * Subtiles [first + k width, ...) of [first, end), tiles_per_batch per batch; counts [ntiles x
 * stride] as pc_run_lease writes them; digests [ntiles x 64] the hex output_sha256 of each subtile.
 * Host-only; PC_OVERFLOW if cap bytes are too few.
 */
int pc_scopes_json(const uint64_t *counts, uint32_t stride, uint32_t ng, uint64_t ntiles, uint64_t first,
                   uint64_t end, uint64_t width, uint32_t tiles_per_batch, const char *digests, char *out,
                   uint64_t cap, uint64_t *len);

/*
 * Genuine-cube control: the number of integers a in [first, last] coprime to every prime <= p,
 * i.e. the cube roots whose cubes a correct sieve of bound p must emit.  Replaces the reference's
 * host checkers review/cube_count.c:12-37 and review/cube_count_independent.c:9-34 (same inclusive
 * root bounds and limits: 1 <= first <= last < 2^32, 2 <= p <= 2000, else PC_INVALID).  With
 * roots == NULL only *count is written; otherwise the roots are also written to roots[cap] on the
 * host in ascending order (their --list form), or PC_OVERFLOW is returned with *count set when
 * more than cap exist.  kernel_ms (may be NULL) receives the device time of the sieve launches.
 */
int pc_cube_roots(pc_ctx *ctx, uint64_t first, uint64_t last, uint32_t p, uint32_t *roots, uint64_t cap,
                  uint64_t *count, double *kernel_ms);

/* 128-bit limb self-test: for each of n cases (a, b, c, d) in in4, out3 = low, high limb of
 * a*b - c*d mod 2^128 and the borrow flag; replaces the `arithmetic` kernel
 * (kernels/pseudocube.cuh:7-11). */
int pc_selftest_wide(pc_ctx *ctx, const uint64_t *in4, uint64_t *out3, uint64_t n);

#ifdef __cplusplus
}
#endif
#endif
