// Shared device/host definitions of libpcube (sm_100a).
#pragma once
#include <cuda_runtime.h>
#include <stdint.h>
#include <string>
#include <vector>
#include "../../include/pcube.h"

#define PC_MAX_BITSET 8        // residual filters intersected as bitsets
#define PC_MAX_RES 1024        // residual filters per (p, A, B)
#define PC_MAX_WHEEL_T 6       // focus rings handled as wheel bitset rows
#define PC_MAX_CHEAP 4         // residual filters tested per survivor from u and v residues

// ------------------------------------------------------------------------------------------
// context, errors, memory accounting

struct pc_ctx {
    int device = 0;
    cudaStream_t stream = nullptr;
    cudaEvent_t ev[8] = {};
    cudaEvent_t marks[8] = {};
    uint64_t cap = 0, in_use = 0, peak = 0;
    uint64_t h2d = 0, d2h = 0;       // bytes the library has copied to and from the host
    int sm_count = 0, cc_major = 0, cc_minor = 0;
    char name[256] = {};
    std::string err;
};

struct pc_buf {
    uint64_t *d = nullptr;
    uint64_t n = 0;
    uint64_t bytes = 0;
};

int pc_fail(pc_ctx *ctx, int code, const std::string &msg);
int pc_cuda_fail(pc_ctx *ctx, cudaError_t e, const char *what);
int pc_alloc(pc_ctx *ctx, void **ptr, uint64_t bytes);
void pc_release(pc_ctx *ctx, void *ptr, uint64_t bytes);

#define PC_CHECK(ctx, call)                                                   \
    do {                                                                      \
        cudaError_t e_ = (call);                                              \
        if (e_ != cudaSuccess) return pc_cuda_fail((ctx), e_, #call);         \
    } while (0)

// An asynchronous copy on the context's stream, counted in ctx->h2d / ctx->d2h.
inline cudaError_t pc_copy(pc_ctx *ctx, void *dst, const void *src, size_t bytes, cudaMemcpyKind kind) {
    if (kind == cudaMemcpyHostToDevice) ctx->h2d += bytes;
    else if (kind == cudaMemcpyDeviceToHost) ctx->d2h += bytes;
    return cudaMemcpyAsync(dst, src, bytes, kind, ctx->stream);
}

inline int pc_cuda_status(pc_ctx *ctx, cudaError_t e, const char *what) {
    return e == cudaSuccess ? PC_OK : pc_cuda_fail(ctx, e, what);
}

#define PC_LAUNCHED(ctx, what)                                                \
    do {                                                                      \
        cudaError_t e_ = cudaGetLastError();                                  \
        if (e_ != cudaSuccess) return pc_cuda_fail((ctx), e_, what);          \
    } while (0)

// RAII holder for device scratch owned by one call.
struct Scratch {
    pc_ctx *ctx;
    std::vector<std::pair<void *, uint64_t>> items;
    explicit Scratch(pc_ctx *c) : ctx(c) {}
    ~Scratch() {
        for (auto &it : items) pc_release(ctx, it.first, it.second);
    }
    template <class T>
    int get(T **p, uint64_t count) {
        uint64_t bytes = count * sizeof(T);
        if (bytes == 0) bytes = 16;
        void *q = nullptr;
        int rc = pc_alloc(ctx, &q, bytes);
        if (rc) return rc;
        items.emplace_back(q, bytes);
        *p = (T *)q;
        return PC_OK;
    }
};

__host__ __device__ __forceinline__ uint64_t umin64(uint64_t a, uint64_t b) { return a < b ? a : b; }
__host__ __device__ __forceinline__ uint64_t umax64(uint64_t a, uint64_t b) { return a > b ? a : b; }
__host__ __device__ __forceinline__ int64_t imin64(int64_t a, int64_t b) { return a < b ? a : b; }
__host__ __device__ __forceinline__ int64_t imax64(int64_t a, int64_t b) { return a > b ? a : b; }

// ------------------------------------------------------------------------------------------
// 128-bit unsigned arithmetic in two 64-bit limbs (add.cc/addc and sub.cc/subc carry chains)

struct u128 {
    uint64_t lo, hi;
};

__device__ __forceinline__ u128 mul_wide(uint64_t a, uint64_t b) {
    u128 r;
    r.lo = a * b;
    r.hi = __umul64hi(a, b);
    return r;
}

__device__ __forceinline__ u128 add128(u128 a, u128 b) {
    u128 r;
    asm("add.cc.u64 %0, %2, %4;\n\taddc.u64 %1, %3, %5;"
        : "=l"(r.lo), "=l"(r.hi)
        : "l"(a.lo), "l"(a.hi), "l"(b.lo), "l"(b.hi));
    return r;
}

__device__ __forceinline__ u128 sub128(u128 a, u128 b) {
    u128 r;
    asm("sub.cc.u64 %0, %2, %4;\n\tsubc.u64 %1, %3, %5;"
        : "=l"(r.lo), "=l"(r.hi)
        : "l"(a.lo), "l"(a.hi), "l"(b.lo), "l"(b.hi));
    return r;
}

__device__ __forceinline__ bool less128(u128 a, u128 b) {
    return a.hi < b.hi || (a.hi == b.hi && a.lo < b.lo);
}

// ------------------------------------------------------------------------------------------
// Remainders by small odd or even moduli q < 2^16 without a hardware divide.
//
// fastmod32: Lemire, Kaser and Kurz, "Faster Remainder by Direct Computation" (2019): with
// c = floor((2^64 - 1) / q) + 1, x mod q = floor(((c * x) mod 2^64) * q / 2^64) for every 32-bit x.
//
// A 128-bit value is folded first: with 16-bit limbs h_k and r_k = 2^(16k) mod q,
// sum h_k r_k < 8 * 2^16 * 2^16 = 2^35 when q < 2^16; limbs are folded in two halves so each
// partial sum stays below 2^32 for q < 2^13 (residual primes are far smaller).

struct ModQ {
    uint32_t q;
    uint32_t r16[7];   // 2^(16k) mod q, k = 1..7
    uint64_t c;        // fastmod constant
};

__host__ __device__ __forceinline__ uint64_t fastmod_constant(uint32_t q) {
    return UINT64_C(0xFFFFFFFFFFFFFFFF) / q + 1;
}

__device__ __forceinline__ uint32_t fastmod32(uint32_t x, uint64_t c, uint32_t q) {
    uint64_t low = c * x;
    return (uint32_t)__umul64hi(low, q);
}

// x mod q for 64-bit x, q < 2^13 (r16 from a ModQ).
__device__ __forceinline__ uint32_t mod64(uint64_t x, const ModQ &m) {
    uint32_t w0 = (uint32_t)x, w1 = (uint32_t)(x >> 32);
    uint32_t t = (w0 & 0xffffu) + (w0 >> 16) * m.r16[0] + (w1 & 0xffffu) * m.r16[1] + (w1 >> 16) * m.r16[2];
    return fastmod32(t, m.c, m.q);
}

// x mod q for 128-bit x, q < 2^13.
__device__ __forceinline__ uint32_t mod128(u128 x, const ModQ &m) {
    uint32_t w0 = (uint32_t)x.lo, w1 = (uint32_t)(x.lo >> 32), w2 = (uint32_t)x.hi, w3 = (uint32_t)(x.hi >> 32);
    uint32_t t0 = (w0 & 0xffffu) + (w0 >> 16) * m.r16[0] + (w1 & 0xffffu) * m.r16[1] + (w1 >> 16) * m.r16[2];
    uint32_t t1 = (w2 & 0xffffu) * m.r16[3] + (w2 >> 16) * m.r16[4] + (w3 & 0xffffu) * m.r16[5] + (w3 >> 16) * m.r16[6];
    return fastmod32(fastmod32(t0, m.c, m.q) + fastmod32(t1, m.c, m.q), m.c, m.q);
}

inline ModQ make_modq(uint32_t q) {
    ModQ m{};
    m.q = q;
    uint64_t r = 1;
    for (int k = 0; k < 7; ++k) {
        r = (r << 16) % q;
        m.r16[k] = (uint32_t)r;
    }
    m.c = fastmod_constant(q);
    return m;
}

// Bits [n, 32) cleared for n in [0, 32]; PTX shl clamps shift counts >= 32 to a zero result.
__device__ __forceinline__ uint32_t low_bits(uint32_t n) {
    uint32_t r;
    asm("shl.b32 %0, %1, %2;" : "=r"(r) : "r"(0xffffffffu), "r"(n));
    return ~r;
}

// ------------------------------------------------------------------------------------------
// 32x32 bit-matrix transpose across a warp: lane l holds row l (bit i = column i) on entry and
// column l on exit.  Five exchange rounds of the off-diagonal blocks.
__device__ __forceinline__ uint32_t transpose32(uint32_t x, uint32_t lane) {
#pragma unroll
    for (int j = 16; j >= 1; j >>= 1) {
        const uint32_t hm = j == 16 ? 0xffff0000u : j == 8 ? 0xff00ff00u : j == 4 ? 0xf0f0f0f0u
                          : j == 2 ? 0xccccccccu : 0xaaaaaaaau;
        uint32_t p = __shfl_xor_sync(0xffffffffu, x, j);
        bool upper = lane & j;
        uint32_t keep = upper ? hm : ~hm;
        uint32_t moved = upper ? (p >> j) : (p << j);
        x = (x & keep) | (moved & ~keep);
    }
    return x;
}

// The same transpose with its per-lane constants computed once: in exchange round r (block size
// j = 16 >> r) a lane rotates its partner's word by sh[r] (left by j for the lower lane of a pair,
// right by j for the upper one) and keeps its own bits where keep[r] is set, one funnel shift and
// one bit-select per round.
__device__ __forceinline__ void transpose_consts(uint32_t lane, uint32_t (&sh)[5], uint32_t (&keep)[5]) {
#pragma unroll
    for (int r = 0; r < 5; ++r) {
        const uint32_t j = 16u >> r;
        const uint32_t hm = r == 0 ? 0xffff0000u : r == 1 ? 0xff00ff00u : r == 2 ? 0xf0f0f0f0u
                          : r == 3 ? 0xccccccccu : 0xaaaaaaaau;
        const bool upper = lane & j;
        sh[r] = upper ? 32u - j : j;
        keep[r] = upper ? hm : ~hm;
    }
}

__device__ __forceinline__ uint32_t transpose32c(uint32_t x, const uint32_t (&sh)[5], const uint32_t (&keep)[5]) {
#pragma unroll
    for (int r = 0; r < 5; ++r) {
        const uint32_t p = __shfl_xor_sync(0xffffffffu, x, 16u >> r);
        const uint32_t moved = __funnelshift_l(p, p, sh[r]);
        x = (x & keep[r]) | (moved & ~keep[r]);
    }
    return x;
}

// ------------------------------------------------------------------------------------------
// internal host helpers shared across translation units

int pc_exclusive_scan_u64(pc_ctx *ctx, const uint64_t *in, uint64_t *out, uint64_t n, uint64_t *total_dev);
uint64_t pc_scan_workspace(uint64_t n);
int pc_exclusive_scan_ws(pc_ctx *ctx, const uint64_t *in, uint64_t *out, uint64_t n, uint64_t *total_dev,
                         uint64_t *ws);

// Many sorted focus windows generated together: one count launch, one scan and one emit launch.
// Window i is written at base[i] of the shared output; each base is rounded up to a multiple of
// the window's padding (so a u list can start on a block boundary of the matcher).
struct WinBatch {
    uint32_t n = 0;
    uint64_t units = 0;
    void *d_desc = nullptr, *d_foci = nullptr;
    uint64_t *d_cnt = nullptr, *d_off = nullptr, *d_ws = nullptr, *d_tot = nullptr, *d_base = nullptr;
    uint32_t *d_bits = nullptr;      // the count pass's unit words for the emit pass (null: recompute)
    std::vector<uint64_t> total, base;
    uint64_t out_len = 0;
};
struct pc_focus;
uint64_t pc_focus_modulus(const pc_focus *f);
int winbatch_plan(pc_ctx *ctx, Scratch &hold, const pc_focus *const *focus, const uint64_t *low, const uint64_t *high,
                  const uint64_t *pad, uint32_t n, uint64_t cap, WinBatch &wb, int *launches);
int winbatch_count(pc_ctx *ctx, const WinBatch &wb);
int winbatch_emit(pc_ctx *ctx, const WinBatch &wb, uint64_t *out);
int pc_window_into(pc_ctx *ctx, const pc_focus *f, uint64_t low, uint64_t high, uint64_t cap, uint64_t **out,
                   uint64_t *out_bytes, uint64_t *total_host, int *launches);
