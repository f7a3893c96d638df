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
int pc_device_info(const pc_ctx *ctx, int *sm_count, int *cc_major, int *cc_minor, char *name, int name_len);
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
    uint32_t words_per_thread; /* bitset words per thread per v row: 1, 2 or 4 */
    uint32_t v_chunk;          /* v rows per work item (0 = whole block) */
    uint32_t threads;          /* threads per CTA: 256, 512 or 1024 */
    uint32_t reserved[3];
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
    uint64_t reserved[5];      /* [0..2]: bitset filters, block words and threads the call used */
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
 * Plain per-position matcher over one tile: replaces Matcher.arrays' kernel (pseudocube/gpu.py:
 * 147-182, 199-210).  Every residual filter is tested per position; counts [ng+3]; out [out_cap x 2].
 */
int pc_run_plain(pc_ctx *ctx, const pc_filters *filters, const pc_buf *us, uint64_t u_off, uint64_t nu,
                 const pc_buf *vs, uint64_t v_off, uint64_t nv, uint64_t lo0, uint64_t lo1, uint64_t hi0,
                 uint64_t hi1, uint64_t *counts, uint64_t *out, uint64_t out_cap, pc_stats *stats);

/*
 * Plain per-tile matcher that allocates no device memory (no counterpart in the reference).
 * For callers that cannot call cudaMalloc: code that runs while a stream is being captured into
 * a CUDA graph (allocation is refused there), code embedded in a process whose allocator already
 * owns the device's memory, and code that must not pay cudaMalloc's implicit device
 * synchronisation.  Same result as pc_run_plain with host inputs: us[nu], vs[nv] (sorted focus
 * values of one tile), the residual filters as for pc_filters_create, counts [ng+3] and
 * out [out_cap x 2] on the host.  Its scratch is a 16 MiB static device array inside the
 * library: inputs, filter tables and outputs must fit in it, or the call returns PC_INVALID with
 * the reason in err.  The first call on a device looks up the array's address (make that first
 * call before any stream capture).  It works on the legacy default stream; every call reuses the
 * same array, so calls that overlap on one GPU race with each other.  err (err_len bytes, may be
 * NULL) receives a message on failure.
 */
int pc_run_plain_static(int device, const uint64_t *us, uint64_t nu, const uint64_t *vs, uint64_t nv,
                        uint64_t A, uint64_t B, uint64_t lo0, uint64_t lo1, uint64_t hi0, uint64_t hi1,
                        const uint32_t *primes, uint32_t nres, const uint8_t *allowed, uint64_t *counts,
                        uint64_t *out, uint64_t out_cap, char *err, int err_len);

/* 128-bit limb self-test: for each of n cases (a, b, c, d) in in4, out3 = low, high limb of
 * a*b - c*d mod 2^128 and the borrow flag; replaces the `arithmetic` kernel
 * (kernels/pseudocube.cuh:7-11). */
int pc_selftest_wide(pc_ctx *ctx, const uint64_t *in4, uint64_t *out3, uint64_t n);

#ifdef __cplusplus
}
#endif
#endif
