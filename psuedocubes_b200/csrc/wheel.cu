// Stage 1: CRT focus-wheel tables and sorted focus windows.
//
// A focus of modulus M is the set of y >= 0 whose residue mod every ring modulus q | M lies in
// the ring's (coefficient-adjusted) allowed set R_q.  Split the rings into S (small moduli) and
// T (the largest few).  With M1 = prod(S), the sorted wheel W1 = {w in [0, M1): w mod q in R_q
// for q in S} is built once by a bitset sieve over [0, M1).  Every y = K*M1 + w (w in W1)
// satisfies the S rings; it is in the focus iff (K*M1 + w) mod q in R_q for the T rings.  For
// each T ring and each s in [0, q), a bitset row over W1's index space marks the w with
// (s + w) mod q in R_q; the window for period K is the AND of the rows s = K*M1 mod q.
//
// A window [low, high) is therefore walked in (period, wheel index) order, which is ascending
// value order: a count pass, an exclusive scan and an emit pass produce the sorted values with
// no sort and no residue set materialised.  Tables are p-independent for p above the largest
// focus prime.
#include "common.cuh"
#include <algorithm>
#include <chrono>
#include <numeric>

struct pc_focus {
    uint64_t M = 0, M1 = 1, count1 = 0, words1 = 0;
    uint32_t nT = 0;
    uint32_t tq[PC_MAX_WHEEL_T] = {};
    uint32_t t_m1mod[PC_MAX_WHEEL_T] = {};
    uint32_t t_row0[PC_MAX_WHEEL_T] = {};
    uint32_t total_rows = 0;
    uint64_t *W1 = nullptr;      // device, sorted wheel
    uint32_t *rows = nullptr;    // device, total_rows x words1
    uint64_t W1_bytes = 0, rows_bytes = 0;
    std::vector<uint64_t> W1_host;
    uint64_t count_lo = 0, count_hi = 0;
    double build_ms = 0;
};

namespace {

constexpr int WT = 256;          // threads per CTA of the window kernels
constexpr int SIEVE_WORDS = 64;  // sieve words per thread
constexpr int WIN_WORDS = 32;    // wheel words per window unit
constexpr uint64_t WIN_WORDS_BUDGET = UINT64_C(512) << 20;   // kept count-pass words, bytes

// Periodic bit patterns of the S rings, replicated so any 32-bit window at offset < q is one
// funnel shift of two consecutive words.
struct SieveRings {
    uint32_t n;
    uint32_t q[16];
    uint32_t off[16];            // word offset of each ring's pattern in the pattern array
    uint32_t step[16];           // 32 mod q
    ModQ mq[16];
};

__global__ void k_sieve(const SieveRings rings, const uint32_t *__restrict__ patterns, uint64_t M1,
                        uint64_t nwords, uint64_t *__restrict__ counts, const uint64_t *__restrict__ offsets,
                        uint64_t *__restrict__ out) {
    uint64_t t = blockIdx.x * (uint64_t)blockDim.x + threadIdx.x;
    uint64_t w0 = t * SIEVE_WORDS;
    if (w0 >= nwords) return;
    uint64_t w1 = min(nwords, w0 + SIEVE_WORDS);
    uint32_t s[16];
    for (uint32_t r = 0; r < rings.n; ++r) s[r] = mod64(w0 * 32, rings.mq[r]);
    uint64_t total = 0, pos = offsets ? offsets[t] : 0;
    for (uint64_t w = w0; w < w1; ++w) {
        uint32_t bits = 0xffffffffu;
        for (uint32_t r = 0; r < rings.n; ++r) {
            const uint32_t *p = patterns + rings.off[r];
            uint32_t lo = p[s[r] >> 5], hi = p[(s[r] >> 5) + 1];
            bits &= __funnelshift_r(lo, hi, s[r] & 31);
            s[r] += rings.step[r];
            if (s[r] >= rings.q[r]) s[r] -= rings.q[r];
        }
        uint64_t base = w * 32;
        if (base + 32 > M1) bits &= low_bits((uint32_t)(M1 - base));
        if (offsets) {
            while (bits) {
                uint32_t b = __ffs(bits) - 1;
                bits &= bits - 1;
                out[pos++] = base + b;
            }
        } else {
            total += __popc(bits);
        }
    }
    if (!offsets) counts[t] = total;
}

// rows[row0 + s][w] bit l = R[(s + W1[32w + l] mod q) mod q], via the rotation of the pattern
// RR (R repeated) by m = W1 mod q and a warp transpose.
__global__ void k_wheel_rows(const uint64_t *__restrict__ W1, uint64_t count1, uint64_t words1,
                             const uint32_t *__restrict__ pattern, uint32_t q, ModQ mq,
                             uint32_t *__restrict__ rows) {
    const uint32_t lane = threadIdx.x & 31;
    uint64_t w = (blockIdx.x * (uint64_t)blockDim.x + threadIdx.x) >> 5;
    if (w >= words1) return;
    uint64_t j = w * 32 + lane;
    bool valid = j < count1;
    uint32_t m = valid ? mod64(W1[j], mq) : 0;
    for (uint32_t k = 0; k * 32 < q; ++k) {
        uint32_t st = 32 * k + m;
        uint32_t col = __funnelshift_r(pattern[st >> 5], pattern[(st >> 5) + 1], st & 31);
        col = valid ? col : 0u;
        uint32_t row = transpose32(col, lane);
        uint32_t s = 32 * k + lane;
        if (s < q) rows[(uint64_t)s * words1 + w] = row;
    }
}

struct WindowPlan {
    uint64_t K0, K1, j_lo, j_hi;
    uint64_t wa0, wb0, wa1, wb1;       // word ranges of the first and last period
    uint64_t units_first, units_mid, units_last, units;
};

// Device view of one focus: the sorted wheel and the bitset rows of its T rings.
struct FocusDev {
    const uint64_t *W1;
    const uint32_t *rows;
    uint64_t M1, count1, words1;
    uint32_t nT, pad;
    uint32_t tq[PC_MAX_WHEEL_T];
    uint32_t t_m1mod[PC_MAX_WHEEL_T];
    uint32_t t_row0[PC_MAX_WHEEL_T];
    ModQ tmq[PC_MAX_WHEEL_T];
};

// One window of a batch: its plan, its first unit in the batch-wide unit numbering and its focus.
struct WinDesc {
    WindowPlan plan;
    uint64_t unit_base;
    uint32_t focus, pad;
};

__device__ __forceinline__ void unit_of(const WindowPlan &p, uint64_t words1, uint64_t u, uint64_t &K,
                                        uint64_t &wa, uint64_t &wb) {
    if (u < p.units_first) {
        K = p.K0;
        wa = p.wa0 + u * WIN_WORDS;
        wb = min(p.wb0, wa + WIN_WORDS);
        return;
    }
    u -= p.units_first;
    uint64_t mid_periods = p.K1 > p.K0 + 1 ? p.K1 - p.K0 - 1 : 0;
    if (u < mid_periods * p.units_mid) {
        const uint32_t um = (uint32_t)p.units_mid, uu = (uint32_t)u;     // unit counts < 2^32
        const uint32_t period = uu / um;
        K = p.K0 + 1 + period;
        wa = (uint64_t)(uu - period * um) * WIN_WORDS;
        wb = min(words1, wa + WIN_WORDS);
        return;
    }
    u -= mid_periods * p.units_mid;
    K = p.K1;
    wa = p.wa1 + u * WIN_WORDS;
    wb = min(p.wb1, wa + WIN_WORDS);
}

constexpr int WIN_UNITS_PER_WARP = 16;

// One warp per WIN_UNITS_PER_WARP consecutive window units of WIN_WORDS = 32 wheel words each, one
// word per lane, so every row load of the warp is one coalesced 128-byte request.  The warp finds
// the window of its first unit by a binary search over the windows' first units and steps to the
// next window when its units cross into it.  The row addresses of a period are computed once and
// reused while its units stay in that period (a period spans hundreds of units), and the rows of a
// unit are loaded together before they are combined.  Count pass: per-unit totals, and (words
// not null) each unit's 32 words kept for the emit pass, which then reads them instead of the
// rows.  Emit pass: the lane's exclusive prefix inside the warp, plus the unit's offset inside
// its window, plus the window's base gives ascending output slots.  Both passes wait on L2 (row
// words, wheel entries), so the kernel is held to 32 registers for 64 resident warps per SM; the
// few spills sit on the once-per-period row-address path.
__global__ void __launch_bounds__(WT, 8) k_windows(const WinDesc *__restrict__ desc, uint32_t ndesc, const FocusDev *__restrict__ foci,
                          uint64_t units, uint64_t *__restrict__ counts, const uint64_t *__restrict__ offsets,
                          const uint64_t *__restrict__ bases, uint64_t *__restrict__ out, uint32_t *__restrict__ words) {
    const uint32_t lane = threadIdx.x & 31;
    const uint64_t u0 = ((blockIdx.x * (uint64_t)blockDim.x + threadIdx.x) >> 5) * WIN_UNITS_PER_WARP;
    if (u0 >= units) return;                            // warp-uniform
    const uint64_t u1 = umin64(units, u0 + WIN_UNITS_PER_WARP);
    uint32_t lo = 0, hi = ndesc;                        // last window with unit_base <= u0
    while (hi - lo > 1) {
        const uint32_t mid = (lo + hi) / 2;
        if (desc[mid].unit_base <= u0) lo = mid;
        else hi = mid;
    }
    uint64_t next_base = lo + 1 < ndesc ? desc[lo + 1].unit_base : UINT64_MAX;
    // The rows of period K, kept while consecutive units stay in the same period and window.
    const uint32_t *row[PC_MAX_WHEEL_T];
    uint64_t row_K = UINT64_MAX;
    uint32_t row_win = UINT32_MAX;
    for (uint64_t gu = u0; gu < u1; ++gu) {
        while (gu >= next_base) {                       // the units crossed into the next window
            ++lo;
            next_base = lo + 1 < ndesc ? desc[lo + 1].unit_base : UINT64_MAX;
        }
        const WindowPlan &p = desc[lo].plan;
        const uint64_t ubase = desc[lo].unit_base;
        const FocusDev &f = foci[desc[lo].focus];
        uint64_t K, wa, wb;
        unit_of(p, f.words1, gu - ubase, K, wa, wb);
        const uint64_t w = wa + lane;
        uint32_t bits = 0;
        if (offsets && words) {                         // emit pass: the count pass kept the words
            bits = words[gu * 32 + lane];
        } else {
            if (K != row_K || lo != row_win) {             // warp-uniform
                row_K = K;
                row_win = lo;
#pragma unroll
                for (uint32_t t = 0; t < PC_MAX_WHEEL_T; ++t) {
                    row[t] = f.rows;                        // rows past nT: a valid address, never read
                    if (t < f.nT) {
                        const uint32_t s = fastmod32(mod64(K, f.tmq[t]) * f.t_m1mod[t], f.tmq[t].c, f.tq[t]);   // < q^2 < 2^32
                        row[t] += (uint64_t)(f.t_row0[t] + s) * f.words1;
                    }
                }
            }
            if (w < wb) {
                bits = 0xffffffffu;
                if (f.nT) {                                 // all row loads in flight before the first use
                    uint32_t r[PC_MAX_WHEEL_T];
#pragma unroll
                    for (uint32_t t = 0; t < PC_MAX_WHEEL_T; ++t) r[t] = t < f.nT ? __ldg(row[t] + w) : 0xffffffffu;
#pragma unroll
                    for (uint32_t t = 0; t < PC_MAX_WHEEL_T; ++t) bits &= r[t];
                }
                const uint64_t jmin = K == p.K0 ? p.j_lo : 0;
                const uint64_t jmax = K == p.K1 ? p.j_hi : f.count1;
                const uint64_t j0 = w * 32;
                if (j0 < jmin) bits &= ~low_bits((uint32_t)(jmin - j0 < 32 ? jmin - j0 : 32));
                if (j0 + 32 > jmax) bits &= jmax > j0 ? low_bits((uint32_t)(jmax - j0)) : 0u;
            }
            if (words) words[gu * 32 + lane] = bits;
        }
        const uint32_t n = __popc(bits);
        if (!offsets) {
            const uint32_t total = __reduce_add_sync(0xffffffffu, n);
            if (lane == 0) counts[gu] = total;
            continue;
        }
        uint32_t incl = n;
#pragma unroll
        for (int d = 1; d < 32; d <<= 1) {
            const uint32_t y = __shfl_up_sync(0xffffffffu, incl, d);
            if (lane >= (uint32_t)d) incl += y;
        }
        uint64_t pos = bases[lo] + (offsets[gu] - offsets[ubase]) + incl - n;
        const uint64_t base = K * f.M1, j0 = w * 32;
        while (bits) {
            const uint32_t b = __ffs(bits) - 1;
            bits &= bits - 1;
            out[pos++] = base + __ldg(f.W1 + j0 + b);
        }
    }
}

// Per window: its value count (offsets hold units + 1 entries, the total last).
__global__ void k_window_totals(const WinDesc *__restrict__ desc, uint32_t ndesc, const uint64_t *__restrict__ offsets,
                                uint64_t *__restrict__ totals) {
    const uint32_t w = blockIdx.x * blockDim.x + threadIdx.x;
    if (w >= ndesc) return;
    const uint64_t b = desc[w].unit_base;
    totals[w] = offsets[b + desc[w].plan.units] - offsets[b];
}

// 128-bit product of 64-bit counts, host side.
void mul_acc(uint64_t &lo, uint64_t &hi, uint64_t f) {
    unsigned __int128 v = ((unsigned __int128)hi << 64 | lo) * f;
    lo = (uint64_t)v;
    hi = (uint64_t)(v >> 64);
}

uint64_t gcd64(uint64_t a, uint64_t b) {
    while (b) {
        uint64_t t = a % b;
        a = b;
        b = t;
    }
    return a;
}

}  // namespace

extern "C" int pc_focus_create(pc_ctx *ctx, uint64_t M, uint32_t nrings, const uint32_t *q, const uint32_t *counts,
                               const uint32_t *residues, uint64_t table_budget, pc_focus **out) {
    *out = nullptr;
    if (M == 0 || M >= (UINT64_C(1) << 63) || nrings > 16) return pc_fail(ctx, PC_INVALID, "invalid focus modulus");
    auto t_start = std::chrono::steady_clock::now();
    if (!table_budget) table_budget = UINT64_C(256) << 20;
    struct Ring {
        uint32_t q, n;
        std::vector<uint32_t> res;
    };
    std::vector<Ring> rings;
    uint64_t prodq = 1, off = 0;
    for (uint32_t k = 0; k < nrings; ++k) {
        Ring r{q[k], counts[k], std::vector<uint32_t>(residues + off, residues + off + counts[k])};
        off += counts[k];
        if (r.q < 2 || r.q > 65535 || r.n == 0 || r.n > r.q) return pc_fail(ctx, PC_INVALID, "invalid ring");
        for (uint32_t a : r.res)
            if (a >= r.q) return pc_fail(ctx, PC_INVALID, "ring residue out of range");
        if (M % r.q || gcd64(M / r.q, r.q) != 1) return pc_fail(ctx, PC_INVALID, "ring moduli must be coprime factors of M");
        prodq *= r.q;
        rings.push_back(std::move(r));
    }
    if (prodq != M) return pc_fail(ctx, PC_INVALID, "ring moduli do not multiply to M");
    std::sort(rings.begin(), rings.end(), [](const Ring &a, const Ring &b) { return a.q < b.q; });

    pc_focus *f = new pc_focus();
    f->M = M;
    f->count_lo = 1;
    for (auto &r : rings) mul_acc(f->count_lo, f->count_hi, r.n);
    // Choose the T rings: the fewest largest rings whose removal makes the sieve over M1 and
    // the tables fit; among the feasible, the smallest table budget use wins ties.
    uint32_t chosen = UINT32_MAX;
    for (uint32_t nT = 0; nT <= std::min<uint32_t>(PC_MAX_WHEEL_T, nrings); ++nT) {
        uint64_t M1 = M, count1_lo = f->count_lo, count1_hi = f->count_hi, rowsum = 0;
        for (uint32_t k = nrings - nT; k < nrings; ++k) {
            M1 /= rings[k].q;
            rowsum += rings[k].q;
            unsigned __int128 c = ((unsigned __int128)count1_hi << 64 | count1_lo) / rings[k].n;
            count1_lo = (uint64_t)c;
            count1_hi = (uint64_t)(c >> 64);
        }
        if (count1_hi || M1 > (UINT64_C(1) << 36)) continue;
        uint64_t words1 = (count1_lo + 31) / 32;
        uint64_t bytes = count1_lo * 8 + rowsum * words1 * 4;
        if (bytes <= table_budget) {
            chosen = nT;
            break;
        }
    }
    if (chosen == UINT32_MAX) {
        delete f;
        return pc_fail(ctx, PC_INVALID, "focus wheel does not fit the table budget");
    }
    f->nT = chosen;
    uint32_t nS = nrings - chosen;
    f->M1 = 1;
    for (uint32_t k = 0; k < nS; ++k) f->M1 *= rings[k].q;

    // --- W1: sieve over [0, M1) with the S rings
    SieveRings sr{};
    sr.n = nS;
    std::vector<uint32_t> pat;
    for (uint32_t k = 0; k < nS; ++k) {
        const Ring &r = rings[k];
        sr.q[k] = r.q;
        sr.off[k] = (uint32_t)pat.size();
        sr.step[k] = 32 % r.q;
        sr.mq[k] = make_modq(r.q);
        uint32_t nbits = r.q + 64;
        std::vector<uint32_t> words((nbits + 31) / 32 + 1, 0);
        std::vector<char> ok(r.q, 0);
        for (uint32_t a : r.res) ok[a] = 1;
        for (uint32_t b = 0; b < nbits; ++b)
            if (ok[b % r.q]) words[b / 32] |= 1u << (b % 32);
        pat.insert(pat.end(), words.begin(), words.end());
    }
    Scratch s(ctx);
    uint32_t *d_pat;
    int rc = s.get(&d_pat, pat.size() + 1);
    if (rc) {
        delete f;
        return rc;
    }
    if (!pat.empty()) pc_copy(ctx, d_pat, pat.data(), pat.size() * 4, cudaMemcpyHostToDevice);
    uint64_t nwords = (f->M1 + 31) / 32;
    uint64_t nthreads = (nwords + SIEVE_WORDS - 1) / SIEVE_WORDS;
    uint64_t *d_cnt, *d_off, *d_total;
    rc = s.get(&d_cnt, nthreads);
    if (!rc) rc = s.get(&d_off, nthreads);
    if (!rc) rc = s.get(&d_total, 1);
    if (rc) {
        delete f;
        return rc;
    }
    unsigned grid = (unsigned)((nthreads + WT - 1) / WT);
    k_sieve<<<grid, WT, 0, ctx->stream>>>(sr, d_pat, f->M1, nwords, d_cnt, nullptr, nullptr);
    rc = pc_exclusive_scan_u64(ctx, d_cnt, d_off, nthreads, d_total);
    uint64_t total = 0;
    if (!rc && pc_copy(ctx, &total, d_total, 8, cudaMemcpyDeviceToHost) == cudaSuccess &&
        cudaStreamSynchronize(ctx->stream) == cudaSuccess) {
    } else if (!rc) {
        rc = pc_cuda_fail(ctx, cudaGetLastError(), "wheel count");
    }
    if (rc) {
        delete f;
        return rc;
    }
    uint64_t expect_lo = f->count_lo, expect_hi = f->count_hi;
    for (uint32_t k = nS; k < nrings; ++k) {
        unsigned __int128 c = ((unsigned __int128)expect_hi << 64 | expect_lo) / rings[k].n;
        expect_lo = (uint64_t)c;
        expect_hi = (uint64_t)(c >> 64);
    }
    if (total != expect_lo || expect_hi) {
        delete f;
        return pc_fail(ctx, PC_ARITHMETIC, "wheel size disagrees with the ring counts");
    }
    f->count1 = total;
    f->words1 = (total + 31) / 32;
    f->W1_bytes = std::max<uint64_t>(16, total * 8);
    rc = pc_alloc(ctx, (void **)&f->W1, f->W1_bytes);
    if (rc) {
        delete f;
        return rc;
    }
    k_sieve<<<grid, WT, 0, ctx->stream>>>(sr, d_pat, f->M1, nwords, nullptr, d_off, f->W1);
    PC_LAUNCHED(ctx, "wheel sieve");

    // --- rows of the T rings
    f->total_rows = 0;
    for (uint32_t t = 0; t < chosen; ++t) {
        f->tq[t] = rings[nS + t].q;
        f->t_m1mod[t] = (uint32_t)(f->M1 % f->tq[t]);
        f->t_row0[t] = f->total_rows;
        f->total_rows += f->tq[t];
    }
    f->rows_bytes = std::max<uint64_t>(16, (uint64_t)f->total_rows * f->words1 * 4);
    rc = pc_alloc(ctx, (void **)&f->rows, f->rows_bytes);
    if (rc) {
        pc_release(ctx, f->W1, f->W1_bytes);
        delete f;
        return rc;
    }
    for (uint32_t t = 0; t < chosen; ++t) {
        const Ring &r = rings[nS + t];
        uint32_t nbits = 2 * r.q + 64;
        std::vector<uint32_t> words((nbits + 31) / 32 + 1, 0);
        std::vector<char> ok(r.q, 0);
        for (uint32_t a : r.res) ok[a] = 1;
        for (uint32_t b = 0; b < nbits; ++b)
            if (ok[b % r.q]) words[b / 32] |= 1u << (b % 32);
        uint32_t *d_rp;
        rc = s.get(&d_rp, words.size());
        if (rc) break;
        pc_copy(ctx, d_rp, words.data(), words.size() * 4, cudaMemcpyHostToDevice);
        uint64_t threads = f->words1 * 32;
        k_wheel_rows<<<(unsigned)((threads + WT - 1) / WT), WT, 0, ctx->stream>>>(
            f->W1, f->count1, f->words1, d_rp, r.q, make_modq(r.q), f->rows + (uint64_t)f->t_row0[t] * f->words1);
        cudaError_t e = cudaGetLastError();
        if (e != cudaSuccess) {
            rc = pc_cuda_fail(ctx, e, "wheel rows");
            break;
        }
    }
    if (!rc) {
        f->W1_host.resize(f->count1);
        cudaError_t e = pc_copy(ctx, f->W1_host.data(), f->W1, f->count1 * 8, cudaMemcpyDeviceToHost);
        if (e == cudaSuccess) e = cudaStreamSynchronize(ctx->stream);
        if (e != cudaSuccess) rc = pc_cuda_fail(ctx, e, "wheel download");
    }
    if (rc) {
        pc_release(ctx, f->W1, f->W1_bytes);
        pc_release(ctx, f->rows, f->rows_bytes);
        delete f;
        return rc;
    }
    f->build_ms = std::chrono::duration<double, std::milli>(std::chrono::steady_clock::now() - t_start).count();
    *out = f;
    return PC_OK;
}

uint64_t pc_focus_modulus(const pc_focus *f) { return f->M; }

extern "C" int pc_focus_free(pc_ctx *ctx, pc_focus *f) {
    if (!f) return PC_OK;
    pc_release(ctx, f->W1, f->W1_bytes);
    pc_release(ctx, f->rows, f->rows_bytes);
    delete f;
    return PC_OK;
}

extern "C" int pc_focus_info(const pc_focus *f, uint64_t *info) {
    info[0] = f->M;
    info[1] = f->M1;
    info[2] = f->count1;
    info[3] = f->nT;
    info[4] = f->W1_bytes + f->rows_bytes;
    info[5] = f->count_lo;
    info[6] = f->count_hi;
    info[7] = (uint64_t)f->build_ms;
    return PC_OK;
}

namespace {

// Host plan of the window [low, high) of focus f: period and wheel-index range, units per part.
int plan_window(pc_ctx *ctx, const pc_focus *f, uint64_t low, uint64_t high, WindowPlan &p) {
    p = WindowPlan{};
    if (high < low) return pc_fail(ctx, PC_INVALID, "invalid bounded focus window");
    if (high == low) return PC_OK;
    if ((high - 1) / f->M - low / f->M + 1 > 4096) return pc_fail(ctx, PC_OVERFLOW, "focus window exceeds bounded period count");
    p.K0 = low / f->M1;
    p.K1 = (high - 1) / f->M1;
    const std::vector<uint64_t> &W = f->W1_host;
    p.j_lo = std::lower_bound(W.begin(), W.end(), low - p.K0 * f->M1) - W.begin();
    p.j_hi = std::lower_bound(W.begin(), W.end(), high - p.K1 * f->M1) - W.begin();
    if (p.K0 == p.K1) {
        p.wa0 = p.j_lo / 32;
        p.wb0 = std::max(p.wa0, (p.j_hi + 31) / 32);
        p.wa1 = p.wb1 = 0;
    } else {
        p.wa0 = p.j_lo / 32;
        p.wb0 = f->words1;
        p.wa1 = 0;
        p.wb1 = (p.j_hi + 31) / 32;
    }
    p.units_first = (p.wb0 - p.wa0 + WIN_WORDS - 1) / WIN_WORDS;
    p.units_mid = (f->words1 + WIN_WORDS - 1) / WIN_WORDS;
    p.units_last = p.K1 > p.K0 ? (p.wb1 - p.wa1 + WIN_WORDS - 1) / WIN_WORDS : 0;
    uint64_t mid_periods = p.K1 > p.K0 + 1 ? p.K1 - p.K0 - 1 : 0;
    p.units = p.units_first + mid_periods * p.units_mid + p.units_last;
    if (p.units >= (UINT64_C(1) << 31)) return pc_fail(ctx, PC_OVERFLOW, "focus window too long");
    return PC_OK;
}

FocusDev focus_dev(const pc_focus *f) {
    FocusDev d{};
    d.W1 = f->W1;
    d.rows = f->rows;
    d.M1 = f->M1;
    d.count1 = f->count1;
    d.words1 = f->words1;
    d.nT = f->nT;
    for (uint32_t t = 0; t < f->nT; ++t) {
        d.tq[t] = f->tq[t];
        d.t_m1mod[t] = f->t_m1mod[t];
        d.t_row0[t] = f->t_row0[t];
        d.tmq[t] = make_modq(f->tq[t]);
    }
    return d;
}

}  // namespace

int winbatch_count(pc_ctx *ctx, const WinBatch &wb) {
    if (wb.units) {
        const uint64_t warps = (wb.units + WIN_UNITS_PER_WARP - 1) / WIN_UNITS_PER_WARP;
        const unsigned grid = (unsigned)((warps * 32 + WT - 1) / WT);
        k_windows<<<grid, WT, 0, ctx->stream>>>((const WinDesc *)wb.d_desc, wb.n, (const FocusDev *)wb.d_foci, wb.units,
                                                wb.d_cnt, nullptr, nullptr, nullptr, wb.d_bits);
        PC_LAUNCHED(ctx, "window count");
    }
    return pc_exclusive_scan_ws(ctx, wb.d_cnt, wb.d_off, wb.units, wb.d_off + wb.units, wb.d_ws);
}

int winbatch_emit(pc_ctx *ctx, const WinBatch &wb, uint64_t *out) {
    if (!wb.out_len) return PC_OK;
    PC_CHECK(ctx, cudaMemsetAsync(out, 0, wb.out_len * 8, ctx->stream));   // padding slots read as 0
    if (wb.units) {
        const uint64_t warps = (wb.units + WIN_UNITS_PER_WARP - 1) / WIN_UNITS_PER_WARP;
        const unsigned grid = (unsigned)((warps * 32 + WT - 1) / WT);
        k_windows<<<grid, WT, 0, ctx->stream>>>((const WinDesc *)wb.d_desc, wb.n, (const FocusDev *)wb.d_foci, wb.units,
                                                nullptr, wb.d_off, wb.d_base, out, wb.d_bits);
        PC_LAUNCHED(ctx, "window emit");
    }
    return PC_OK;
}

int winbatch_plan(pc_ctx *ctx, Scratch &hold, const pc_focus *const *focus, const uint64_t *low, const uint64_t *high,
                  const uint64_t *pad, uint32_t n, uint64_t cap, WinBatch &wb, int *launches) {
    wb = WinBatch{};
    wb.n = n;
    if (!n) return PC_OK;
    std::vector<WinDesc> desc(n);
    std::vector<FocusDev> foci;
    std::vector<const pc_focus *> seen;
    for (uint32_t i = 0; i < n; ++i) {
        int rc = plan_window(ctx, focus[i], low[i], high[i], desc[i].plan);
        if (rc) return rc;
        desc[i].unit_base = wb.units;
        wb.units += desc[i].plan.units;
        uint32_t k = 0;
        while (k < seen.size() && seen[k] != focus[i]) ++k;
        if (k == seen.size()) {
            seen.push_back(focus[i]);
            foci.push_back(focus_dev(focus[i]));
        }
        desc[i].focus = k;
    }
    if (wb.units >= (UINT64_C(1) << 34)) return pc_fail(ctx, PC_OVERFLOW, "focus windows too long");
    WinDesc *d_desc;
    FocusDev *d_foci;
    int rc = hold.get(&d_desc, n);
    if (!rc) rc = hold.get(&d_foci, foci.size());
    if (!rc) rc = hold.get(&wb.d_cnt, std::max<uint64_t>(1, wb.units));
    if (!rc) rc = hold.get(&wb.d_off, wb.units + 1);
    if (!rc) rc = hold.get(&wb.d_ws, pc_scan_workspace(wb.units));
    if (!rc) rc = hold.get(&wb.d_tot, n);
    if (!rc) rc = hold.get(&wb.d_base, n);
    // keep the count pass's unit words for the emit pass when they fit WIN_WORDS_BUDGET bytes
    if (!rc && wb.units * WIN_WORDS * 4 <= WIN_WORDS_BUDGET && ctx->in_use + wb.units * WIN_WORDS * 4 <= ctx->cap / 2)
        rc = hold.get(&wb.d_bits, wb.units * WIN_WORDS);
    if (rc) return rc;
    wb.d_desc = d_desc;
    wb.d_foci = d_foci;
    PC_CHECK(ctx, pc_copy(ctx, d_desc, desc.data(), n * sizeof(WinDesc), cudaMemcpyHostToDevice));
    PC_CHECK(ctx, pc_copy(ctx, d_foci, foci.data(), foci.size() * sizeof(FocusDev), cudaMemcpyHostToDevice));
    rc = winbatch_count(ctx, wb);
    if (rc) return rc;
    k_window_totals<<<(n + 255) / 256, 256, 0, ctx->stream>>>(d_desc, n, wb.d_off, wb.d_tot);
    PC_LAUNCHED(ctx, "window totals");
    wb.total.assign(n, 0);
    PC_CHECK(ctx, pc_copy(ctx, wb.total.data(), wb.d_tot, n * 8, cudaMemcpyDeviceToHost));
    PC_CHECK(ctx, cudaStreamSynchronize(ctx->stream));
    wb.base.assign(n, 0);
    for (uint32_t i = 0; i < n; ++i) {
        if (wb.total[i] > cap) return pc_fail(ctx, PC_OVERFLOW, "focus buffer overflow; tile invalid");
        const uint64_t pd = pad && pad[i] ? pad[i] : 1;
        wb.base[i] = (wb.out_len + pd - 1) / pd * pd;
        wb.out_len = wb.base[i] + wb.total[i];
    }
    PC_CHECK(ctx, pc_copy(ctx, wb.d_base, wb.base.data(), n * 8, cudaMemcpyHostToDevice));
    PC_CHECK(ctx, cudaStreamSynchronize(ctx->stream));   // the host vectors above go out of scope
    if (launches) *launches += 4;
    return PC_OK;
}

// Plan and run one window; out is allocated by the call (out_bytes returned for release).
// total_host receives the count.
int pc_window_into(pc_ctx *ctx, const pc_focus *f, uint64_t low, uint64_t high, uint64_t cap,
                   uint64_t **out, uint64_t *out_bytes, uint64_t *total_host, int *launches) {
    *out = nullptr;
    *out_bytes = 0;
    *total_host = 0;
    if (high < low) return pc_fail(ctx, PC_INVALID, "invalid bounded focus window");
    if (high == low) return PC_OK;
    Scratch s(ctx);
    WinBatch wb;
    int rc = winbatch_plan(ctx, s, &f, &low, &high, nullptr, 1, UINT64_MAX, wb, launches);
    if (rc) return rc;
    *total_host = wb.total[0];
    if (wb.total[0] > cap) return pc_fail(ctx, PC_OVERFLOW, "focus buffer overflow; tile invalid");
    if (!wb.out_len) return PC_OK;
    const uint64_t bytes = std::max<uint64_t>(16, wb.out_len * 8);
    rc = pc_alloc(ctx, (void **)out, bytes);
    if (rc) return rc;
    *out_bytes = bytes;
    rc = winbatch_emit(ctx, wb, *out);
    if (launches) *launches += 1;
    return rc;
}

extern "C" int pc_focus_window(pc_ctx *ctx, const pc_focus *f, uint64_t low, uint64_t high, uint64_t cap,
                               pc_buf **out, uint64_t *count) {
    *out = nullptr;
    *count = 0;
    uint64_t *d = nullptr, bytes = 0, total = 0;
    int rc = pc_window_into(ctx, f, low, high, cap, &d, &bytes, &total, nullptr);
    *count = total;
    if (rc) {
        pc_release(ctx, d, bytes);
        return rc;
    }
    pc_buf *b = new pc_buf();
    b->d = d;
    b->n = total;
    b->bytes = bytes;
    if (!d) {
        rc = pc_alloc(ctx, (void **)&b->d, 16);
        if (rc) {
            delete b;
            return rc;
        }
        b->bytes = 16;
    }
    PC_CHECK(ctx, cudaStreamSynchronize(ctx->stream));
    *out = b;
    return PC_OK;
}
