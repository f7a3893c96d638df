/*
 * CPU restatement of the reference's doubly-focused pseudocube sieve.
 *
 * TEST INFRASTRUCTURE ONLY.  Nothing in the product (psuedocubes_b200/) links,
 * loads or calls this file; only tests/, __graft_entry__.smoke() and the CPU
 * baseline leg of bench.py use it, and only as the checker.
 *
 * What it restates (file:line refer to the reference project):
 *   oc_partial      pseudocube/gpu.py:82-92        mixed-radix CRT partial sums of one ring half
 *   oc_window       review/focus_window_cpu.cpp:4-25 two monotone pointers over sorted C for each
 *                   sorted d, two wraps; periods as in pseudocube/gpu.py:94-114; output sorted.
 *   oc_masked_batch pseudocube/batch_experiment.py:184-234 (MaskedMatcher): per v row the two
 *                   128-bit lower bounds (:210-215), residue rows of the first four residual
 *                   filters (:185-193), AND + popcount (:217-221), 128-bit x, underflow flag,
 *                   later filters with group counters every four filters (:222-228), per-subtile
 *                   counters and output slots (:206-207, :229-230).
 *   oc_wide         review/wide.c:3-7 (a*b - c*d mod 2^128 and the borrow flag).
 *   oc_cube_roots   review/cube_count.c:12-37: the roots in [first, last] coprime to every prime
 *                   <= p, by a segmented byte sieve (count, and the ascending list up to cap).
 *
 * Per-subtile counter layout (as the reference's fused kernel): ng+3 uint64 per subtile,
 * [0] focused positions, [1..ng] group survivors, [ng+1] outputs, [ng+2] underflows.
 */
#include <stdint.h>
#include <stdlib.h>
#include <string.h>
#include <pthread.h>

typedef unsigned __int128 u128;

static int cmp_u64(const void *a, const void *b) {
    uint64_t x = *(const uint64_t *)a, y = *(const uint64_t *)b;
    return x < y ? -1 : x > y;
}

/* All partial CRT sums of one half (ring 0 is the fastest digit).  gpu.py:82-92 */
int oc_partial(const uint64_t *terms, const uint32_t *sizes, uint32_t nrings, uint64_t M,
               uint64_t *out, uint64_t count) {
    if (M == 0 || M >= ((uint64_t)1 << 63)) return 2;
    for (uint64_t i = 0; i < count; ++i) {
        uint64_t r = 0, rem = i, off = 0;
        for (uint32_t k = 0; k < nrings; ++k) {
            r += terms[off + rem % sizes[k]];
            rem /= sizes[k];
            if (r >= M) r -= M;
            off += sizes[k];
        }
        out[i] = r;
    }
    return 0;
}

void oc_sort_u64(uint64_t *a, uint64_t n) { qsort(a, n, sizeof(uint64_t), cmp_u64); }

/* One within-period window [lo, hi) with offset; sorted C and sorted D.
 * focus_window_cpu.cpp:4-25.  Returns 0 ok, 1 overflow (count = written + 1), 2 bad args. */
static int window_period(const uint64_t *C, uint64_t nc, const uint64_t *D, uint64_t nd,
                         uint64_t M, uint64_t lo, uint64_t hi, uint64_t offset,
                         uint64_t *out, uint64_t cap, uint64_t *written_io) {
    if (lo > hi || hi > M || M >= ((uint64_t)1 << 63)) return 2;
    uint64_t written = *written_io;
    for (unsigned wrap = 0; wrap < 2; ++wrap) {
        uint64_t a = lo + (wrap ? M : 0), b = hi + (wrap ? M : 0), left = nc, right = nc;
        for (uint64_t j = 0; j < nd; ++j) {
            uint64_t d = D[j];
            if (d >= b) break;
            uint64_t lower = a > d ? a - d : 0, upper = b - d;
            while (left && C[left - 1] >= lower) --left;
            while (right && C[right - 1] >= upper) --right;
            for (uint64_t i = left; i < right; ++i) {
                if (written >= cap) { *written_io = written + 1; return 1; }
                out[written++] = C[i] + d - (wrap ? M : 0) + offset;
            }
        }
    }
    *written_io = written;
    return 0;
}

/* Sorted focus values in [low, high): periods as gpu.py:97-113 (at most 4096 periods). */
int oc_window(const uint64_t *C, uint64_t nc, const uint64_t *D, uint64_t nd, uint64_t M,
              uint64_t low, uint64_t high, uint64_t *out, uint64_t cap, uint64_t *count) {
    *count = 0;
    if (high < low || M == 0) return 2;
    if (high == low) return 0;
    uint64_t p0 = low / M, p1 = (high - 1) / M;
    if (p1 - p0 + 1 > 4096) return 1;
    uint64_t written = 0;
    for (uint64_t period = p0; period <= p1; ++period) {
        uint64_t base = period * M;
        uint64_t a = low > base ? low - base : 0;
        uint64_t b = high - base < M ? high - base : M;
        int rc = window_period(C, nc, D, nd, M, a, b, base, out, cap, &written);
        if (rc) { *count = written; return rc; }
    }
    qsort(out, written, sizeof(uint64_t), cmp_u64);
    *count = written;
    return 0;
}

/* a*b - c*d mod 2^128 and borrow; review/wide.c:3-7 */
void oc_wide(const uint64_t *in4, uint64_t *out3, uint64_t n) {
    for (uint64_t i = 0; i < n; ++i) {
        u128 l = (u128)in4[4 * i] * in4[4 * i + 1], r = (u128)in4[4 * i + 2] * in4[4 * i + 3];
        u128 d = l - r;
        out3[3 * i] = (uint64_t)d;
        out3[3 * i + 1] = (uint64_t)(d >> 64);
        out3[3 * i + 2] = l < r;
    }
}

/* ------------------------------------------------------------------------------------------ */
/* Masked batch matcher (batch_experiment.py:170-254)                                          */

typedef struct {
    /* inputs */
    const uint64_t *us; uint64_t nu;
    const uint64_t *vs; uint64_t nv;
    uint64_t A, B;
    u128 lo, hi;
    const uint32_t *primes; uint32_t nres;      /* residual filters in reference order */
    const uint8_t *allowed;                     /* concatenated byte tables, q bytes each */
    const uint64_t *offsets;                    /* table offset of each residual */
    uint64_t v_first, width; uint32_t ntiles;
    uint64_t cap;
    uint32_t ng, nfirst;
    const uint32_t *rows;                       /* nfirst filters: q rows x words each */
    const uint64_t *row_offset;                 /* first row index of each first filter */
    uint64_t words;
    /* per-thread outputs */
    uint64_t j0, j1;
    uint64_t *counts;                           /* ntiles x (ng+3) */
    uint64_t *vals; uint32_t *val_tile; uint64_t nvals, capvals;
    int err;
} job_t;

static uint64_t lower_bound_u(const uint64_t *us, uint64_t nu, uint64_t B, u128 key) {
    /* first i with us[i]*B > key; batch_experiment.py:210-215 */
    uint64_t left = 0, h = nu;
    while (left < h) {
        uint64_t mid = left + (h - left) / 2;
        if (!(key < (u128)us[mid] * B)) left = mid + 1; else h = mid;
    }
    return left;
}

static void push_value(job_t *jb, uint64_t tile, u128 x) {
    if (jb->nvals == jb->capvals) {
        uint64_t nc = jb->capvals ? 2 * jb->capvals : 1024;
        uint64_t *nv = realloc(jb->vals, nc * 2 * sizeof(uint64_t));
        uint32_t *nt = realloc(jb->val_tile, nc * sizeof(uint32_t));
        if (!nv || !nt) { jb->err = 1; if (nv) jb->vals = nv; if (nt) jb->val_tile = nt; return; }
        jb->vals = nv; jb->val_tile = nt; jb->capvals = nc;
    }
    jb->vals[2 * jb->nvals] = (uint64_t)x;
    jb->vals[2 * jb->nvals + 1] = (uint64_t)(x >> 64);
    jb->val_tile[jb->nvals] = (uint32_t)tile;
    jb->nvals++;
}

static void *match_rows(void *arg) {
    job_t *jb = (job_t *)arg;
    const uint32_t stride = jb->ng + 3;
    for (uint64_t j = jb->j0; j < jb->j1; ++j) {
        uint64_t v = jb->vs[j];
        uint64_t tile = (v - jb->v_first) / jb->width;
        uint64_t *cnt = jb->counts + tile * stride;
        u128 shift = (u128)v * jb->A;
        uint64_t left = lower_bound_u(jb->us, jb->nu, jb->B, shift + jb->lo);
        uint64_t right = lower_bound_u(jb->us, jb->nu, jb->B, shift + jb->hi);
        if (right < left) right = left;
        const uint32_t *m[8];
        for (uint32_t f = 0; f < jb->nfirst; ++f)
            m[f] = jb->rows + (jb->row_offset[f] + v % jb->primes[f]) * jb->words;
        for (uint64_t word = left / 32; word < (right + 31) / 32; ++word) {
            uint64_t base = word * 32;
            uint32_t bits = 0xffffffffu;
            if (base < left) bits &= 0xffffffffu << (left - base);
            if (right < base + 32) bits &= (uint32_t)((1ull << (right - base)) - 1u);
            cnt[0] += (uint64_t)__builtin_popcount(bits);
            for (uint32_t f = 0; f < jb->nfirst; ++f) bits &= m[f][word];
            while (bits) {
                unsigned bit = (unsigned)__builtin_ctz(bits);
                bits &= bits - 1;
                u128 positive = (u128)jb->us[base + bit] * jb->B;
                if (positive < shift) { cnt[jb->ng + 2]++; continue; }
                u128 x = positive - shift;
                cnt[1]++;
                int ok = 1;
                for (uint32_t idx = 4; idx < jb->nres; ++idx) {
                    uint32_t q = jb->primes[idx];
                    uint32_t r = (uint32_t)(x % q);
                    if (!jb->allowed[jb->offsets[idx] + r]) { ok = 0; break; }
                    if (idx % 4 == 3 || idx + 1 == jb->nres) cnt[idx / 4 + 1]++;
                }
                if (!ok) continue;
                cnt[jb->ng + 1]++;
                push_value(jb, tile, x);
            }
        }
    }
    return NULL;
}

typedef struct {
    const uint64_t *us; uint64_t nu; uint64_t B;
    const uint32_t *primes; const uint8_t *allowed; const uint64_t *offsets;
    uint64_t A; uint32_t *rows; const uint64_t *row_offset; uint64_t words;
    uint32_t f0, f1;
} rowjob_t;

/* mask_build: row r of filter q, bit i of word w <=> allowed[((u%q)(B%q) + q - (r(A%q))%q) % q]
 * batch_experiment.py:185-193 */
static void *build_rows(void *arg) {
    rowjob_t *rj = (rowjob_t *)arg;
    for (uint32_t f = rj->f0; f < rj->f1; ++f) {
        uint64_t q = rj->primes[f];
        const uint8_t *tab = rj->allowed + rj->offsets[f];
        uint16_t *ub = malloc((rj->nu ? rj->nu : 1) * sizeof(uint16_t));
        for (uint64_t i = 0; i < rj->nu; ++i) ub[i] = (uint16_t)((rj->us[i] % q) * (rj->B % q) % q);
        for (uint64_t r = 0; r < q; ++r) {
            uint64_t sub = (r * (rj->A % q)) % q;
            uint32_t *row = rj->rows + (rj->row_offset[f] + r) * rj->words;
            for (uint64_t w = 0; w < rj->words; ++w) {
                uint32_t bits = 0;
                for (uint32_t l = 0; l < 32; ++l) {
                    uint64_t i = w * 32 + l;
                    if (i < rj->nu && tab[(ub[i] + q - sub) % q]) bits |= 1u << l;
                }
                row[w] = bits;
            }
        }
        free(ub);
    }
    return NULL;
}

/*
 * One fused batch (FusedMatcher.run + MaskedMatcher).  lo/hi are 128-bit (two limbs).
 * primes/allowed/offsets: residual filters in the reference order (batch_experiment.py:84-86).
 * counts: ntiles x (ng+3), zeroed here.  out: ntiles x 2 x cap limbs (only the first cap values
 * per subtile are stored; counts[ng+1] holds the true number, as the reference).
 * Returns 0, 2 (bad arguments) or 5 (host memory).
 */
int oc_masked_batch(const uint64_t *us, uint64_t nu, const uint64_t *vs, uint64_t nv,
                    uint64_t A, uint64_t B, uint64_t lo0, uint64_t lo1, uint64_t hi0, uint64_t hi1,
                    const uint32_t *primes, uint32_t nres, const uint8_t *allowed,
                    uint64_t v_first, uint64_t width, uint32_t ntiles, uint64_t cap,
                    uint64_t *counts, uint64_t *out, int threads) {
    if (nres == 0 || width == 0 || ntiles == 0 || threads < 1) return 2;
    uint32_t ng = (nres + 3) / 4, nfirst = nres < 4 ? nres : 4;
    uint32_t stride = ng + 3;
    memset(counts, 0, (size_t)ntiles * stride * sizeof(uint64_t));
    if (nu == 0 || nv == 0) return 0;
    for (uint64_t j = 0; j < nv; ++j)
        if (vs[j] < v_first || (vs[j] - v_first) / width >= ntiles) return 2;
    uint64_t *offsets = malloc(nres * sizeof(uint64_t));
    uint64_t off = 0;
    for (uint32_t i = 0; i < nres; ++i) { offsets[i] = off; off += primes[i]; }
    uint64_t words = (nu + 31) / 32;
    uint64_t row_offset[8], nrows = 0;
    for (uint32_t f = 0; f < nfirst; ++f) { row_offset[f] = nrows; nrows += primes[f]; }
    uint32_t *rows = malloc(nrows * words * sizeof(uint32_t));
    if (!rows) { free(offsets); return 5; }
    {
        pthread_t th[8]; rowjob_t rj[8];
        for (uint32_t f = 0; f < nfirst; ++f) {
            rj[f] = (rowjob_t){us, nu, B, primes, allowed, offsets, A, rows, row_offset, words, f, f + 1};
            pthread_create(&th[f], NULL, build_rows, &rj[f]);
        }
        for (uint32_t f = 0; f < nfirst; ++f) pthread_join(th[f], NULL);
    }
    int T = threads;
    job_t *jobs = calloc((size_t)T, sizeof(job_t));
    pthread_t *th = calloc((size_t)T, sizeof(pthread_t));
    for (int t = 0; t < T; ++t) {
        job_t *jb = &jobs[t];
        jb->us = us; jb->nu = nu; jb->vs = vs; jb->nv = nv; jb->A = A; jb->B = B;
        jb->lo = ((u128)lo1 << 64) | lo0; jb->hi = ((u128)hi1 << 64) | hi0;
        jb->primes = primes; jb->nres = nres; jb->allowed = allowed; jb->offsets = offsets;
        jb->v_first = v_first; jb->width = width; jb->ntiles = ntiles; jb->cap = cap;
        jb->ng = ng; jb->nfirst = nfirst; jb->rows = rows; jb->row_offset = row_offset; jb->words = words;
        jb->j0 = nv * (uint64_t)t / T; jb->j1 = nv * (uint64_t)(t + 1) / T;
        jb->counts = calloc((size_t)ntiles * stride, sizeof(uint64_t));
        pthread_create(&th[t], NULL, match_rows, jb);
    }
    int err = 0;
    uint64_t *filled = calloc(ntiles, sizeof(uint64_t));
    for (int t = 0; t < T; ++t) {
        pthread_join(th[t], NULL);
        job_t *jb = &jobs[t];
        err |= jb->err;
        for (uint64_t k = 0; k < (uint64_t)ntiles * stride; ++k) counts[k] += jb->counts[k];
        for (uint64_t k = 0; k < jb->nvals; ++k) {
            uint32_t tile = jb->val_tile[k];
            if (filled[tile] < cap) {
                out[(uint64_t)tile * 2 * cap + 2 * filled[tile]] = jb->vals[2 * k];
                out[(uint64_t)tile * 2 * cap + 2 * filled[tile] + 1] = jb->vals[2 * k + 1];
            }
            filled[tile]++;
        }
        free(jb->counts); free(jb->vals); free(jb->val_tile);
    }
    free(filled); free(jobs); free(th); free(rows); free(offsets);
    return err ? 5 : 0;
}

/*
 * Plain per-position matcher (gpu.py:129-182, 'byte' variant): every residual filter is tested
 * per position, group counters after each fourth filter, underflow checked before pop[0].
 * Single tile.  counts: ng+3.  out: 2*cap limbs.
 */
int oc_plain_tile(const uint64_t *us, uint64_t nu, const uint64_t *vs, uint64_t nv,
                  uint64_t A, uint64_t B, uint64_t lo0, uint64_t lo1, uint64_t hi0, uint64_t hi1,
                  const uint32_t *primes, uint32_t nres, const uint8_t *allowed,
                  uint64_t cap, uint64_t *counts, uint64_t *out) {
    uint32_t ng = (nres + 3) / 4;
    memset(counts, 0, (size_t)(ng + 3) * sizeof(uint64_t));
    u128 lo = ((u128)lo1 << 64) | lo0, hi = ((u128)hi1 << 64) | hi0;
    uint64_t *offsets = malloc((nres ? nres : 1) * sizeof(uint64_t));
    uint64_t off = 0;
    for (uint32_t i = 0; i < nres; ++i) { offsets[i] = off; off += primes[i]; }
    for (uint64_t j = 0; j < nv; ++j) {
        u128 shift = (u128)vs[j] * A, upper = shift + hi;
        uint64_t i = lower_bound_u(us, nu, B, shift + lo);
        for (; i < nu; ++i) {
            u128 positive = (u128)us[i] * B;
            if (upper < positive) break;
            if (positive < shift) { counts[ng + 2]++; continue; }
            u128 x = positive - shift;
            counts[0]++;
            int ok = 1;
            for (uint32_t idx = 0; idx < nres; ++idx) {
                uint32_t q = primes[idx];
                if (!allowed[offsets[idx] + (uint32_t)(x % q)]) { ok = 0; break; }
                if (idx % 4 == 3 || idx + 1 == nres) counts[idx / 4 + 1]++;
            }
            if (!ok) continue;
            uint64_t slot = counts[ng + 1]++;
            if (slot < cap) { out[2 * slot] = (uint64_t)x; out[2 * slot + 1] = (uint64_t)(x >> 64); }
        }
    }
    free(offsets);
    return 0;
}

/* Decimal JSON list of sorted 64-bit values, e.g. ["1","7"]\n, as accounting.encoded() writes a
 * list of str; used only to hash very long output lists.  Returns bytes written or 0 if the
 * buffer is too small. */
uint64_t oc_json_strings_u64(const uint64_t *vals, uint64_t n, char *buf, uint64_t cap) {
    uint64_t pos = 0;
    if (cap < 3) return 0;
    buf[pos++] = '[';
    for (uint64_t i = 0; i < n; ++i) {
        char tmp[24]; int len = 0; uint64_t v = vals[i];
        do { tmp[len++] = (char)('0' + v % 10); v /= 10; } while (v);
        if (pos + (uint64_t)len + 4 > cap) return 0;
        if (i) buf[pos++] = ',';
        buf[pos++] = '"';
        while (len) buf[pos++] = tmp[--len];
        buf[pos++] = '"';
    }
    buf[pos++] = ']';
    buf[pos++] = '\n';
    return pos;
}

/* ---- genuine-cube control (review/cube_count.c:12-37) ---------------------------------- */

typedef struct {
    uint64_t first, last, count;
    const uint32_t *primes;
    uint32_t np;
    uint32_t *roots;      /* NULL: count only */
    uint64_t cap;
} roots_job;

static void *roots_slice(void *arg) {
    roots_job *j = (roots_job *)arg;
    enum { SEGMENT = 1 << 20 };
    unsigned char *keep = malloc(SEGMENT);
    if (!keep) { j->count = UINT64_MAX; return NULL; }
    for (uint64_t start = j->first; start <= j->last;) {
        uint64_t n = j->last - start + 1;
        if (n > SEGMENT) n = SEGMENT;
        memset(keep, 1, n);
        for (uint32_t i = 0; i < j->np; ++i) {
            uint64_t q = j->primes[i], m = (start + q - 1) / q * q;   /* first multiple >= start */
            for (; m < start + n; m += q) keep[m - start] = 0;
        }
        for (uint64_t i = 0; i < n; ++i)
            if (keep[i]) {
                if (j->roots && j->count < j->cap) j->roots[j->count] = (uint32_t)(start + i);
                j->count++;
            }
        start += n;
    }
    free(keep);
    return NULL;
}

/* Returns 2 on invalid bounds (as the reference checker's exit status), 1 when a list was asked
 * for and more than cap roots exist (count still set), else 0.  threads > 1 splits a count-only
 * range into contiguous slices. */
int oc_cube_roots(uint64_t first, uint64_t last, uint32_t p, uint32_t *roots, uint64_t cap, uint64_t *count,
                  int threads) {
    if (first < 1 || last < first || last > UINT32_MAX || p < 2 || p > 2000) return 2;
    uint32_t primes[400], np = 0;
    for (uint32_t q = 2; q <= p; ++q) {
        int prime = 1;
        for (uint32_t d = 2; d * d <= q; ++d)
            if (q % d == 0) { prime = 0; break; }
        if (prime) primes[np++] = q;
    }
    if (roots || threads < 1) threads = 1;
    if (threads > 64) threads = 64;
    roots_job jobs[64];
    pthread_t tid[64];
    const uint64_t n = last - first + 1, per = (n + threads - 1) / threads;
    int started = 0;
    for (int t = 0; t < threads; ++t) {
        const uint64_t a = first + (uint64_t)t * per;
        if (a > last) break;
        jobs[t] = (roots_job){a, (last - a < per ? last : a + per - 1), 0, primes, np, roots, cap};
        if (threads == 1) roots_slice(&jobs[t]);
        else pthread_create(&tid[t], NULL, roots_slice, &jobs[t]);
        started++;
    }
    uint64_t total = 0;
    int failed = 0;
    for (int t = 0; t < started; ++t) {
        if (threads > 1) pthread_join(tid[t], NULL);
        if (jobs[t].count == UINT64_MAX) failed = 1;
        else total += jobs[t].count;
    }
    if (failed) return 3;
    *count = total;
    return roots && total > cap ? 1 : 0;
}
