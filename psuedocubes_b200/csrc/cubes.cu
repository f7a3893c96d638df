// Genuine-cube control: the integers a in [first, last] coprime to every prime <= p.
//
// Every such a gives a cube a^3 that is a pseudocube candidate of bound p (it is +-1 mod 9 when
// 3 does not divide a, and a cubic residue and a unit modulo every other prime <= p), so the
// count over the cube roots of (lo, hi] is the number of genuine cubes a correct sieve of (lo, hi]
// must emit.  The reference counts them on the host with a byte-segment sieve
// (review/cube_count.c:12-37) and an odd-only bit sieve (review/cube_count_independent.c:9-34)
// over inclusive root bounds 1 <= first <= last < 2^32, 2 <= p <= 2000.
//
// Device form: the primes <= p are packed into groups whose product P stays <= 2^16; for each
// group a bit pattern marks the residues r mod P that share a factor with P, stored for r up to
// P + 33 * 32 so that 33 consecutive words starting at any offset r < P are read without a wrap.
// A warp owns 32 x 33 consecutive words of the root bitmap (bit i <-> root first + i); lane l
// holds the 33 words from 33 l on, so its window for word k + 1 shares a pattern word with the
// window for word k: one shared-memory load, one funnel shift and one OR per group and word.  The
// lanes start 33 words apart, so (away from the pattern's end) their loads fall in 32 different
// banks.  The OR over all groups marks the roots with a prime factor <= p; the rest are counted,
// or, after a scan of per-warp counts, written out in ascending order (lane order is root order).
#include "common.cuh"
#include <algorithm>
#include <vector>

namespace {

constexpr uint32_t ROOT_GROUP_MAX = 1u << 16;   // largest product of one prime group
constexpr int ROOT_LANE_WORDS = 33;             // consecutive words per lane of one warp chunk
constexpr uint64_t ROOT_CHUNK_WORDS = 32 * ROOT_LANE_WORDS;
constexpr int ROOT_THREADS = 256;

struct RootGroup {
    uint64_t c;                      // fastmod constant of P
    uint32_t P, P2, two32, off;      // period, 2P, 2^32 mod P, pattern word offset
};

struct RootTables {
    std::vector<RootGroup> groups;
    std::vector<uint32_t> pattern;
};

RootTables root_tables(uint32_t p) {
    std::vector<uint32_t> primes;
    std::vector<char> composite(p + 1, 0);
    for (uint32_t q = 2; q <= p; ++q) {
        if (composite[q]) continue;
        primes.push_back(q);
        for (uint32_t m = q * q; m <= p; m += q) composite[m] = 1;
    }
    RootTables t;
    for (size_t i = 0; i < primes.size();) {
        uint32_t P = 1;
        size_t j = i;
        while (j < primes.size() && (uint64_t)P * primes[j] <= ROOT_GROUP_MAX) P *= primes[j++];
        RootGroup g{};
        g.P = P;
        g.c = fastmod_constant(P);
        g.P2 = 2 * P;
        g.two32 = (uint32_t)((UINT64_C(1) << 32) % P);
        g.off = (uint32_t)t.pattern.size();
        const uint32_t words = (P - 1) / 32 + ROOT_LANE_WORDS + 1;   // 33 windows from any r < P
        t.pattern.resize(t.pattern.size() + words, 0);
        uint32_t *w = t.pattern.data() + g.off;
        for (size_t k = i; k < j; ++k)                 // q | P, so q | r iff q | (r mod P)
            for (uint32_t r = 0; r < words * 32; r += primes[k]) w[r >> 5] |= 1u << (r & 31);
        t.groups.push_back(g);
        i = j;
    }
    return t;
}

// Counts (offsets == nullptr) or writes (offsets != nullptr) the roots of each warp chunk.
// Count mode adds into *total, or stores per-chunk counts when chunk_counts is given.
__global__ void __launch_bounds__(ROOT_THREADS) k_roots(const uint4 *__restrict__ tables, uint32_t table_words,
                                                        uint32_t ngroups, uint64_t first, uint64_t n, uint64_t nchunks,
                                                        unsigned long long *__restrict__ total,
                                                        uint64_t *__restrict__ chunk_counts,
                                                        const uint64_t *__restrict__ offsets, uint32_t *__restrict__ out) {
    extern __shared__ uint4 smem4[];
    for (uint32_t i = threadIdx.x; i < table_words / 4; i += blockDim.x) smem4[i] = tables[i];
    __syncthreads();
    const RootGroup *groups = (const RootGroup *)smem4;
    const uint32_t *pattern = (const uint32_t *)(groups + ngroups);
    const uint32_t lane = threadIdx.x & 31, warps = blockDim.x >> 5;
    for (uint64_t chunk = blockIdx.x * (uint64_t)warps + (threadIdx.x >> 5); chunk < nchunks;
         chunk += (uint64_t)gridDim.x * warps) {          // warp-uniform
        const uint64_t w0 = chunk * ROOT_CHUNK_WORDS + ROOT_LANE_WORDS * lane;   // the lane's first word
        const uint64_t x0 = first + 32 * w0;                                     // < 2^34
        const uint32_t xlo = (uint32_t)x0, xhi = (uint32_t)(x0 >> 32);
        uint32_t acc[ROOT_LANE_WORDS];
#pragma unroll
        for (int k = 0; k < ROOT_LANE_WORDS; ++k) acc[k] = 0;
        for (uint32_t g = 0; g < ngroups; ++g) {
            const RootGroup G = groups[g];
            uint32_t s = fastmod32(xlo, G.c, G.P) + xhi * G.two32;   // < 3P, as x0 < 2^34
            s -= s >= G.P2 ? G.P2 : 0;
            s -= s >= G.P ? G.P : 0;
            const uint32_t *pat = pattern + G.off + (s >> 5), sh = s & 31;
            uint32_t lo = pat[0];
#pragma unroll
            for (int k = 0; k < ROOT_LANE_WORDS; ++k) {
                const uint32_t hi = pat[k + 1];
                acc[k] |= __funnelshift_r(lo, hi, sh);
                lo = hi;
            }
        }
        uint32_t count = 0;
#pragma unroll
        for (int k = 0; k < ROOT_LANE_WORDS; ++k) {
            const uint64_t bit0 = 32 * (w0 + k);
            const uint32_t valid = bit0 >= n ? 0u : (n - bit0 >= 32 ? 0xffffffffu : low_bits((uint32_t)(n - bit0)));
            acc[k] = ~acc[k] & valid;
            count += __popc(acc[k]);
        }
        if (!offsets) {
            const uint32_t sum = __reduce_add_sync(0xffffffffu, count);
            if (lane == 0) {
                if (chunk_counts) chunk_counts[chunk] = sum;
                else atomicAdd(total, (unsigned long long)sum);
            }
            continue;
        }
        uint32_t incl = count;                            // lanes hold ascending root ranges
#pragma unroll
        for (int d = 1; d < 32; d <<= 1) {
            const uint32_t y = __shfl_up_sync(0xffffffffu, incl, d);
            if (lane >= (uint32_t)d) incl += y;
        }
        uint64_t slot = offsets[chunk] + incl - count;
#pragma unroll
        for (int k = 0; k < ROOT_LANE_WORDS; ++k) {
            const uint64_t root0 = x0 + 32 * (uint64_t)k;
            uint32_t bits = acc[k];
            while (bits) {
                const uint32_t b = __ffs(bits) - 1;
                bits &= bits - 1;
                out[slot++] = (uint32_t)(root0 + b);
            }
        }
    }
}

}  // namespace

extern "C" int pc_cube_roots(pc_ctx *ctx, uint64_t first, uint64_t last, uint32_t p, uint32_t *roots, uint64_t cap,
                             uint64_t *count, double *kernel_ms) {
    if (!ctx || !count) return pc_fail(ctx, PC_INVALID, "null argument");
    if (kernel_ms) *kernel_ms = 0;
    if (first < 1 || last < first || last > UINT32_MAX || p < 2 || p > 2000)
        return pc_fail(ctx, PC_INVALID, "cube roots need 1 <= first <= last < 2^32 and 2 <= p <= 2000");
    const RootTables t = root_tables(p);
    const uint32_t ngroups = (uint32_t)t.groups.size();
    std::vector<uint32_t> host(ngroups * sizeof(RootGroup) / 4 + t.pattern.size());
    std::copy(t.pattern.begin(), t.pattern.end(),
              std::copy((const uint32_t *)t.groups.data(), (const uint32_t *)(t.groups.data() + ngroups), host.begin()));
    host.resize((host.size() + 3) & ~size_t(3), 0);
    const uint32_t table_words = (uint32_t)host.size();
    const size_t smem = table_words * 4;

    const uint64_t n = last - first + 1;
    const uint64_t nchunks = (n + 32 * ROOT_CHUNK_WORDS - 1) / (32 * ROOT_CHUNK_WORDS);   // bits per chunk
    Scratch hold(ctx);
    uint32_t *d_tables = nullptr;
    unsigned long long *d_total = nullptr;
    int rc = hold.get(&d_tables, table_words);
    if (!rc) rc = hold.get(&d_total, 1);
    if (rc) return rc;
    PC_CHECK(ctx, cudaFuncSetAttribute(k_roots, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem));
    int per_sm = 0;
    PC_CHECK(ctx, cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, k_roots, ROOT_THREADS, smem));
    const uint64_t warps = ROOT_THREADS / 32;
    const unsigned grid = (unsigned)std::max<uint64_t>(
        1, std::min<uint64_t>((nchunks + warps - 1) / warps, (uint64_t)ctx->sm_count * std::max(1, per_sm)));
    PC_CHECK(ctx, pc_copy(ctx, d_tables, host.data(), smem, cudaMemcpyHostToDevice));
    PC_CHECK(ctx, cudaMemsetAsync(d_total, 0, 8, ctx->stream));
    auto elapsed = [&](float &ms) { return cudaEventElapsedTime(&ms, ctx->ev[0], ctx->ev[1]); };
    if (!roots) {
        PC_CHECK(ctx, cudaEventRecord(ctx->ev[0], ctx->stream));
        k_roots<<<grid, ROOT_THREADS, smem, ctx->stream>>>((const uint4 *)d_tables, table_words, ngroups, first, n, nchunks,
                                                           d_total, nullptr, nullptr, nullptr);
        PC_LAUNCHED(ctx, "cube roots count");
        PC_CHECK(ctx, cudaEventRecord(ctx->ev[1], ctx->stream));
        unsigned long long total = 0;
        PC_CHECK(ctx, pc_copy(ctx, &total, d_total, 8, cudaMemcpyDeviceToHost));
        PC_CHECK(ctx, cudaStreamSynchronize(ctx->stream));
        float ms = 0;
        PC_CHECK(ctx, elapsed(ms));
        if (kernel_ms) *kernel_ms = ms;
        *count = total;
        return PC_OK;
    }
    uint64_t *d_counts = nullptr, *d_offsets = nullptr, *d_ws = nullptr;
    rc = hold.get(&d_counts, nchunks + 1);
    if (!rc) rc = hold.get(&d_offsets, nchunks + 1);
    if (!rc) rc = hold.get(&d_ws, pc_scan_workspace(nchunks));
    if (rc) return rc;
    PC_CHECK(ctx, cudaEventRecord(ctx->ev[0], ctx->stream));
    k_roots<<<grid, ROOT_THREADS, smem, ctx->stream>>>((const uint4 *)d_tables, table_words, ngroups, first, n, nchunks,
                                                       nullptr, d_counts, nullptr, nullptr);
    PC_LAUNCHED(ctx, "cube roots chunk counts");
    PC_CHECK(ctx, cudaEventRecord(ctx->ev[1], ctx->stream));
    rc = pc_exclusive_scan_ws(ctx, d_counts, d_offsets, nchunks, d_offsets + nchunks, d_ws);
    if (rc) return rc;
    uint64_t total = 0;
    PC_CHECK(ctx, pc_copy(ctx, &total, d_offsets + nchunks, 8, cudaMemcpyDeviceToHost));
    PC_CHECK(ctx, cudaStreamSynchronize(ctx->stream));
    float ms = 0;
    PC_CHECK(ctx, elapsed(ms));
    if (kernel_ms) *kernel_ms = ms;
    *count = total;
    if (total > cap) return pc_fail(ctx, PC_OVERFLOW, "more cube roots than the output capacity");
    if (!total) return PC_OK;
    uint32_t *d_out = nullptr;
    rc = hold.get(&d_out, total);
    if (rc) return rc;
    PC_CHECK(ctx, cudaEventRecord(ctx->ev[0], ctx->stream));
    k_roots<<<grid, ROOT_THREADS, smem, ctx->stream>>>((const uint4 *)d_tables, table_words, ngroups, first, n, nchunks,
                                                       nullptr, nullptr, d_offsets, d_out);
    PC_LAUNCHED(ctx, "cube roots emit");
    PC_CHECK(ctx, cudaEventRecord(ctx->ev[1], ctx->stream));
    PC_CHECK(ctx, pc_copy(ctx, roots, d_out, total * 4, cudaMemcpyDeviceToHost));
    PC_CHECK(ctx, cudaStreamSynchronize(ctx->stream));
    float emit_ms = 0;
    PC_CHECK(ctx, elapsed(emit_ms));
    if (kernel_ms) *kernel_ms += emit_ms;
    return PC_OK;
}
