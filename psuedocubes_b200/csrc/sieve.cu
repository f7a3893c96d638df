// Stages 2 and 3: residue-bitset intersection and exact 128-bit later filters.
//
// Layout.  The sorted u list is cut into blocks of K words (32 u per word).  A work item is one
// u block and a run of consecutive v rows whose exact u interval meets the block.  The CTA that
// owns an item builds, in shared memory, the residue rows of the first NB residual filters for
// its block (row r of filter q, bit i <=> allowed_q[(u_i B - r A) mod q]) and then streams its v
// rows: each v reads the K-word rows selected by v mod q with 128-bit loads, ANDs them, counts
// the group survivors by popcount, and constructs x = uB - vA only for the bits that survive
// every bitset filter.  Those are tested exactly against the remaining filters in 128-bit
// arithmetic.
//
// Rows are stored as 16-byte units with the unit index XOR-swizzled by the row index, so the
// transposing writer (32 rows, one unit each) and the readers (one row, consecutive units) both
// touch all banks once per wavefront.
#include "common.cuh"
#include <algorithm>
#include <chrono>
#include <cstring>
#include <cstdio>

struct FiltConst {
    ModQ m;
    uint32_t tab_off;   // word offset of the packed allowed bitmap
    uint32_t pad;
};

// Compact filter constants passed inside the kernel parameters (constant bank): fast remainder
// constant, modulus, bitmap offset and 2^(16k) mod q for k = 1..5 (x < 2^96).
struct FiltC {
    uint64_t c;
    uint32_t q, tab_off;
    uint16_t r16[5];
    uint16_t pad[3];
};
constexpr int FC_INLINE = 128;

struct pc_filters {
    uint64_t A = 0, B = 0;
    uint32_t nres = 0, ng = 0;
    std::vector<uint32_t> primes;
    FiltConst *d_fc = nullptr;
    uint32_t *d_bits = nullptr;
    uint32_t *d_pat = nullptr;       // swizzle-free RR patterns of the first filters (PATW words each)
    uint64_t fc_bytes = 0, bits_bytes = 0, pat_bytes = 0;
    uint32_t nbmax = 0;              // filters usable as bitset rows
    uint32_t ainvb[PC_MAX_BITSET] = {};
    uint32_t rows_sum[PC_MAX_BITSET + 1] = {};   // prefix sums of q over the first filters
    std::vector<FiltC> fcs;
};

namespace {

constexpr int PATW = 136;            // pattern words per bitset filter (q <= 2047)
constexpr int TMAX_DEFAULT = 64;     // subtile counter slots per CTA

struct __align__(16) VRec {
    uint32_t left, right;            // exact u interval as indices into the sorted u list
    uint64_t v;
    uint16_t row[8];                 // row index (row0 + v mod q) of each bitset filter
};

struct MatchArgs {
    const uint64_t *us;
    const uint64_t *vs;
    const VRec *rec;
    uint64_t nu, nv;
    uint64_t A, B;
    u128 lo, hi;
    uint32_t nres, ng, nb;
    uint32_t tmax;
    const FiltConst *fc;
    const uint32_t *bits;
    const uint32_t *pat;
    uint32_t q[PC_MAX_BITSET];
    uint32_t row0[PC_MAX_BITSET];
    uint32_t ainvb[PC_MAX_BITSET];
    ModQ mq[PC_MAX_BITSET];
    uint32_t total_rows;
    uint64_t *counts;                // ntiles x (ng+3)
    uint64_t *out;
    uint64_t out_cap;
    unsigned long long *n_out;
    uint32_t ntiles;
    const uint4 *bv;                 // per u block: v rows meeting it, v rows covering it
    const uint64_t *item_prefix;     // nblocks + 1
    uint64_t nblocks;
    const uint64_t *vchunk;          // device scalar
    uint64_t v_first, width;         // subtile of v = (v - v_first) / width
    // cheap tier: residual filters nb .. nb+nch-1 tested per survivor from residues of u and v
    uint32_t nch;
    uint32_t cq[PC_MAX_CHEAP], caq[PC_MAX_CHEAP], cbq[PC_MAX_CHEAP], cbits_off[PC_MAX_CHEAP];
    ModQ cmq[PC_MAX_CHEAP];
    uint8_t bgroup[16];              // group ended by filter idx (0 = none), idx < nb + nch
    // deep tier: survivors of every cheap filter, appended to this CTA's slice
    uint4 *deep;                     // (v lo, v hi, u index, subtile) records
    uint32_t deep_cap;               // records per CTA slice
    uint32_t *deep_count;            // per CTA (may exceed deep_cap: the caller retries larger)
};

struct DeepArgs {
    const uint64_t *us;
    const uint4 *deep;
    const uint32_t *deep_count;
    uint32_t deep_cap, slices;
    uint64_t A, B;
    uint32_t first, nres, ng, ntiles;          // filters first .. nres-1 remain
    const uint32_t *bits;
    uint64_t *counts;
    uint64_t *out;
    uint64_t out_cap;
    unsigned long long *n_out;
    FiltC fcs[FC_INLINE];
};

// first j with us[j] * B > key
__device__ __forceinline__ uint64_t count_le(const uint64_t *__restrict__ us, uint64_t n, uint64_t B, u128 key) {
    uint64_t lo = 0, hi = n;
    while (lo < hi) {
        uint64_t mid = lo + (hi - lo) / 2;
        if (less128(key, mul_wide(__ldg(us + mid), B))) hi = mid;
        else lo = mid + 1;
    }
    return lo;
}

__device__ __forceinline__ uint64_t lower_bound64(const uint64_t *__restrict__ a, uint64_t n, uint64_t key) {
    uint64_t lo = 0, hi = n;
    while (lo < hi) {
        uint64_t mid = lo + (hi - lo) / 2;
        if (__ldg(a + mid) < key) lo = mid + 1;
        else hi = mid;
    }
    return lo;
}

__device__ __forceinline__ uint64_t tile_of(uint64_t v, uint64_t v_first, uint64_t width) {
    uint64_t d = v - v_first;
    uint64_t t = (uint64_t)((double)d / (double)width);
    while (t * width > d) --t;
    while ((t + 1) * width <= d) ++t;
    return t;
}

struct PrepArgs {
    const uint64_t *us;
    const uint64_t *vs;
    uint64_t nu, nv, A, B;
    u128 lo, hi;
    uint64_t v_first, width;
    uint32_t ntiles, nb, ng;
    uint32_t q[PC_MAX_BITSET];
    uint32_t row0[PC_MAX_BITSET];
    ModQ mq[PC_MAX_BITSET];
    VRec *rec;
    uint64_t *counts;
    unsigned long long *bad;
};

// Per v row: exact u interval as list indices (batch_experiment.py:209-215), bitset row
// indices, and the focused-position count of its subtile.  A thread owns PREP_RUN consecutive v
// rows: one binary search per bound for the first, then the monotone bounds advance linearly
// (about N_u/N_v < 1 step per row).
constexpr int PREP_RUN = 16;

__device__ __forceinline__ uint64_t advance_le(const uint64_t *__restrict__ us, uint64_t n, uint64_t B, u128 key,
                                               uint64_t from) {
    for (int step = 0; step < 16; ++step) {
        if (from >= n || less128(key, mul_wide(__ldg(us + from), B))) return from;
        ++from;
    }
    return from + count_le(us + from, n - from, B, key);   // long gap: binary search the rest
}

__global__ void k_vprep(const PrepArgs a) {
    const uint64_t t = blockIdx.x * (uint64_t)blockDim.x + threadIdx.x;
    const uint64_t j0 = t * PREP_RUN;
    if (j0 >= a.nv) return;
    const uint64_t j1 = umin64(a.nv, j0 + PREP_RUN);
    uint64_t left = 0, right = 0, tile = UINT64_MAX, t_lo = 1, t_hi = 0, pop = 0;
    for (uint64_t j = j0; j < j1; ++j) {
        const uint64_t v = a.vs[j];
        const u128 shift = mul_wide(v, a.A);
        const u128 klo = add128(shift, a.lo), khi = add128(shift, a.hi);
        if (j == j0) {
            left = count_le(a.us, a.nu, a.B, klo);
            right = umax64(left, count_le(a.us, a.nu, a.B, khi));
        } else {
            left = advance_le(a.us, a.nu, a.B, klo, left);
            right = advance_le(a.us, a.nu, a.B, khi, umax64(left, right));
        }
        if (v < t_lo || v >= t_hi) {
            if (tile != UINT64_MAX && pop)
                atomicAdd((unsigned long long *)&a.counts[tile * (a.ng + 3)], (unsigned long long)pop);
            pop = 0;
            if (v < a.v_first) {
                atomicAdd(a.bad, 1ull);
                tile = UINT64_MAX, t_lo = 1, t_hi = 0;
            } else {
                tile = tile_of(v, a.v_first, a.width);
                t_lo = a.v_first + tile * a.width;
                t_hi = t_lo + a.width;
                if (tile >= a.ntiles) {
                    atomicAdd(a.bad, 1ull);
                    tile = UINT64_MAX, t_lo = 1, t_hi = 0;
                }
            }
        }
        VRec r;
        r.left = (uint32_t)left;
        r.right = (uint32_t)right;
        r.v = v;
#pragma unroll
        for (int f = 0; f < PC_MAX_BITSET; ++f)
            r.row[f] = f < (int)a.nb ? (uint16_t)(a.row0[f] + mod64(v, a.mq[f])) : (uint16_t)0;
        a.rec[j] = r;
        pop += right - left;
    }
    if (tile != UINT64_MAX && pop) atomicAdd((unsigned long long *)&a.counts[tile * (a.ng + 3)], (unsigned long long)pop);
}

// Per subtile: u count and v count of its envelope (searchsorted bounds of
// batch_experiment.py:37-43, as list-independent differences).
__global__ void k_geometry(const uint64_t *__restrict__ us, uint64_t nu, const uint64_t *__restrict__ vs, uint64_t nv,
                           uint64_t A, uint64_t B, u128 lo, u128 hi, uint64_t v_first, uint64_t width,
                           uint64_t v_end, uint32_t ntiles, uint64_t *__restrict__ geometry) {
    uint64_t s = blockIdx.x * (uint64_t)blockDim.x + threadIdx.x;
    if (s >= ntiles) return;
    uint64_t first = v_first + s * width;
    uint64_t end = min(first + width, v_end);
    uint64_t ua = count_le(us, nu, B, add128(mul_wide(first, A), lo));
    uint64_t ub = count_le(us, nu, B, add128(mul_wide(end - 1, A), hi));
    uint64_t va = lower_bound64(vs, nv, first), vb = lower_bound64(vs, nv, end);
    geometry[2 * s] = ub > ua ? ub - ua : 0;
    geometry[2 * s + 1] = vb - va;
}

// Per u block of UB entries: [va, vb) of v rows whose [left, right) meets the block, and the
// sub-range [f0, f1) of rows covering the whole block (left <= start and right >= stop); left and
// right are monotone in the row index, so all four are binary searches.
__device__ __forceinline__ uint64_t first_right_ge(const VRec *__restrict__ rec, uint64_t lo, uint64_t hi, uint64_t x) {
    while (lo < hi) {
        uint64_t mid = lo + (hi - lo) / 2;
        if (rec[mid].right >= x) hi = mid;
        else lo = mid + 1;
    }
    return lo;
}

__device__ __forceinline__ uint64_t first_left_ge(const VRec *__restrict__ rec, uint64_t lo, uint64_t hi, uint64_t x) {
    while (lo < hi) {
        uint64_t mid = lo + (hi - lo) / 2;
        if (rec[mid].left >= x) hi = mid;
        else lo = mid + 1;
    }
    return lo;
}

__global__ void k_blocks(const VRec *__restrict__ rec, uint64_t nv, uint64_t nu, uint32_t UB, uint64_t nblocks,
                         uint4 *__restrict__ bv, uint64_t *__restrict__ pieces) {
    uint64_t b = blockIdx.x * (uint64_t)blockDim.x + threadIdx.x;
    if (b >= nblocks) return;
    const uint64_t start = b * UB, stop = umin64(nu, start + UB);
    const uint64_t va = first_right_ge(rec, 0, nv, start + 1);
    const uint64_t vb = first_left_ge(rec, va, nv, stop);
    uint64_t f0 = umax64(va, first_right_ge(rec, va, vb, stop));
    uint64_t f1 = umin64(vb, first_left_ge(rec, va, vb, start + 1));
    if (f1 < f0) f1 = f0;
    bv[b] = make_uint4((uint32_t)va, (uint32_t)vb, (uint32_t)f0, (uint32_t)f1);
    pieces[b] = vb > va ? vb - va : 0;
}

// v chunk per work item: fixed, or total pieces / target items (at least 64, at most 2^20).
__global__ void k_chunk(const uint64_t *__restrict__ total_pieces, uint64_t fixed_chunk, uint64_t target_items,
                        uint64_t *__restrict__ vchunk) {
    uint64_t c = fixed_chunk;
    if (!c) c = umax64((*total_pieces + target_items - 1) / umax64(1, target_items), 64);
    *vchunk = umin64(c, UINT64_C(1) << 20);
}

__global__ void k_item_counts(const uint64_t *__restrict__ pieces, uint64_t nblocks,
                              const uint64_t *__restrict__ vchunk, uint64_t *__restrict__ items) {
    uint64_t b = blockIdx.x * (uint64_t)blockDim.x + threadIdx.x;
    if (b >= nblocks) return;
    uint64_t c = *vchunk;
    items[b] = (pieces[b] + c - 1) / c;
}

// ------------------------------------------------------------------------------------------
// the fused kernel

template <int K>
struct Geo {
    static constexpr int U = K / 4;                      // 16-byte units per row
    static constexpr int UB = K * 32;                    // u entries per block
    __device__ static __forceinline__ uint32_t unit(uint32_t row, uint32_t c) { return row * U + c; }
};

template <int NB, int K>
__device__ void build_rows(const MatchArgs &a, uint4 *__restrict__ rows, uint16_t *__restrict__ ures,
                           const uint32_t *__restrict__ pat_s, uint32_t block_u0, uint32_t lane, uint32_t warp,
                           uint32_t nwarps) {
    using G = Geo<K>;
    const uint64_t *ub = a.us + block_u0;
    // residues u*B mod q of the cheap-tier filters, one per block entry
    for (uint32_t k = threadIdx.x; k < G::UB; k += blockDim.x) {
        const bool valid = block_u0 + k < a.nu;
        const uint64_t u = valid ? __ldg(ub + k) : 0;
        for (uint32_t t = 0; t < a.nch; ++t)
            ures[t * G::UB + k] = (uint16_t)fastmod32(mod64(u, a.cmq[t]) * a.cbq[t], a.cmq[t].c, a.cq[t]);
    }
    // a warp builds all q rows of one filter for one 16-byte unit (4 words = 128 u)
    for (uint32_t pair = warp; pair < NB * G::U; pair += nwarps) {
        uint32_t f = pair / G::U, c = pair % G::U;
        const uint32_t q = a.q[f];
        uint32_t t[4];
        bool valid[4];
#pragma unroll
        for (int k = 0; k < 4; ++k) {
            uint32_t local = (c * 4 + k) * 32 + lane;
            valid[k] = block_u0 + local < a.nu;
            uint32_t um = valid[k] ? mod64(__ldg(ub + local), a.mq[f]) : 0;
            t[k] = fastmod32(um * a.ainvb[f], a.mq[f].c, q);
        }
        const uint32_t *p = pat_s + f * PATW;
        for (uint32_t g = 0; g * 32 < q; ++g) {
            uint32_t w[4];
#pragma unroll
            for (int k = 0; k < 4; ++k) {
                uint32_t st = 32 * g + q - t[k];
                uint32_t col = __funnelshift_r(p[st >> 5], p[(st >> 5) + 1], st & 31);
                w[k] = transpose32(valid[k] ? col : 0u, lane);
            }
            uint32_t r = 32 * g + lane;
            if (r < q) {
                uint32_t row = a.row0[f] + r;
                rows[G::unit(row, c)] = make_uint4(w[0], w[1], w[2], w[3]);
            }
        }
    }
}

constexpr int CBW = 64;   // bitmap words per cheap-tier filter (q <= 2047)

// Shared-memory layout of k_match (byte offsets); every region starts 16-byte aligned.
constexpr int QCAP = 64;              // survivor ring per warp (pending < 64 by construction)
constexpr uint32_t SLOT_FAR = 0xFFFFF;  // queued slot too large to encode: the drain recomputes it

// Shared-memory layout of k_match (byte offsets); every region starts 16-byte aligned.  The
// residue-row patterns are only read while rows are built, when every survivor ring is empty,
// so they share the rings' space.
struct MatchSmem {
    uint32_t rows, ures, qv, qm, pat, cbits, cnt, misc, total;
    __host__ __device__ MatchSmem(uint32_t total_rows, uint32_t K, uint32_t nb, uint32_t nch, uint32_t tmax,
                                  uint32_t ng, uint32_t warps) {
        rows = 0;
        ures = rows + total_rows * (K / 4) * 16;
        qv = ures + ((nch * K * 32 * 2 + 15) & ~15u);
        qm = qv + warps * QCAP * 8;
        pat = qv;
        const uint32_t ring_end = qm + warps * QCAP * 4, pat_end = pat + nb * PATW * 4;
        cbits = ((ring_end > pat_end ? ring_end : pat_end) + 15) & ~15u;
        cnt = cbits + nch * CBW * 4;
        misc = cnt + ((tmax * (ng + 2) * 4 + 15) & ~15u);
        total = misc + 16;
    }
};

__device__ __forceinline__ uint32_t unit_mask(int32_t lo, int32_t hi) {   // bits [lo, hi) of one 32-bit word
    return low_bits((uint32_t)min(max(hi, 0), 32)) & ~low_bits((uint32_t)min(max(lo, 0), 32));
}

// One lane owns one (v row, u block) piece: it walks the block's K/4 16-byte units in the order
// (lane + p) mod (K/4), so at every step the 32 lanes of a warp hit each 16-byte bank group
// exactly 32/(K/4) times whatever rows they read.  Group counters of groups 1..3 live in
// registers (c[0..2]) and are reduced per subtile when a lane's subtile changes.
template <int NB, int K, int NT>
__global__ void __launch_bounds__(NT, 1) k_match(const MatchArgs a) {
    using G = Geo<K>;
    constexpr uint32_t U = G::U;
    extern __shared__ uint4 smem[];
    const uint32_t lane = threadIdx.x & 31, warp = threadIdx.x >> 5, nwarps = blockDim.x >> 5;
    const MatchSmem L(a.total_rows, K, NB, a.nch, a.tmax, a.ng, nwarps);
    char *base = (char *)smem;
    const uint4 *rows = (const uint4 *)(base + L.rows);
    uint16_t *ures = (uint16_t *)(base + L.ures);
    uint64_t *qv = (uint64_t *)(base + L.qv) + warp * QCAP;
    uint32_t *qm = (uint32_t *)(base + L.qm) + warp * QCAP;
    uint32_t *pat_s = (uint32_t *)(base + L.pat);
    uint32_t *cbits = (uint32_t *)(base + L.cbits);
    uint32_t *cnt_s = (uint32_t *)(base + L.cnt);      // tmax x (ng+2): groups 1..ng, outputs
    uint32_t *deep_ctr = (uint32_t *)(base + L.misc);
    const uint32_t stride = a.ng + 2;

    const uint32_t lanes_below = (1u << lane) - 1u;
    for (uint32_t i = threadIdx.x; i < a.nch * CBW; i += blockDim.x) {
        const uint32_t t = i / CBW, w = i % CBW;
        cbits[i] = w * 32 < a.cq[t] ? a.bits[a.cbits_off[t] + w] : 0u;
    }
    if (threadIdx.x == 0) *deep_ctr = 0;
    uint4 *deep_slice = a.deep + (size_t)blockIdx.x * a.deep_cap;

    const uint64_t n_items = a.item_prefix[a.nblocks];
    const uint64_t vch = *a.vchunk;
    const uint64_t i0 = n_items * blockIdx.x / gridDim.x, i1 = n_items * (blockIdx.x + 1) / gridDim.x;
    uint64_t cur = UINT64_MAX, bsearch = 0;
    if (i0 < i1) {                                        // block of the first item: last b with prefix[b] <= i0
        uint64_t lo = 0, hi = a.nblocks;
        while (hi - lo > 1) {
            uint64_t mid = (lo + hi) / 2;
            if (a.item_prefix[mid] <= i0) lo = mid;
            else hi = mid;
        }
        bsearch = lo;
    }
    const bool c2_live = NB == 8 || (NB > 4 && NB == (int)a.nres);
    const uint32_t nch = a.nch;

    for (uint64_t it = i0; it < i1; ++it) {
        while (a.item_prefix[bsearch + 1] <= it) ++bsearch;  // items are visited in order
        const uint64_t b = bsearch;
        const uint4 range = a.bv[b];
        const uint64_t va = range.x + (it - a.item_prefix[b]) * vch;
        const uint32_t nv_item = (uint32_t)(umin64(range.y, va + vch) - va);   // <= 2^20
        // rows of this item covering the whole block, relative to va
        const uint32_t full_lo = (uint32_t)(range.z > va ? umin64(range.z - va, nv_item) : 0);
        const uint32_t full_hi = (uint32_t)(range.w > va ? umin64(range.w - va, nv_item) : 0);
        const uint32_t block_u0 = (uint32_t)(b * G::UB);
        __syncthreads();                                  // previous item finished with shared memory
        if (b != cur) {
            for (uint32_t i = threadIdx.x; i < NB * PATW; i += blockDim.x) pat_s[i] = a.pat[i];
            __syncthreads();
            build_rows<NB, K>(a, (uint4 *)rows, ures, pat_s, block_u0, lane, warp, nwarps);
            cur = b;
        }
        for (uint32_t k = threadIdx.x; k < a.tmax * stride; k += blockDim.x) cnt_s[k] = 0;
        __syncthreads();
        const uint64_t tile_base = tile_of(a.rec[va].v, a.v_first, a.width);

        uint32_t c[3] = {0, 0, 0};
        uint64_t ctile = UINT64_MAX, t_lo = 1, t_hi = 0;  // this lane's subtile and its v range

        auto flush = [&]() {                              // populations reduced over lanes of a subtile
            const uint64_t key = (c[0] | c[1] | c[2]) ? ctile : UINT64_MAX - 1 - lane;
            const uint32_t same = __match_any_sync(0xffffffffu, key);
            const uint32_t leader = __ffs(same) - 1;
#pragma unroll
            for (int g = 0; g < 3; ++g) {
                const uint32_t sum = __reduce_add_sync(same, c[g]);
                if (key == ctile && lane == leader && sum) {
                    const uint64_t slot = ctile - tile_base;
                    if (slot < a.tmax) atomicAdd(cnt_s + slot * stride + 1 + g, sum);
                    else if (ctile < a.ntiles)
                        atomicAdd((unsigned long long *)&a.counts[ctile * (a.ng + 3) + 1 + g], (unsigned long long)sum);
                }
                c[g] = 0;
            }
        };

        uint32_t qhead = 0, qtail = 0;                    // warp-uniform ring positions

        // Cheap-tier filters on up to 32 queued survivors, one per lane; survivors of all of them
        // go to this CTA's deep slice.
        auto drain = [&](uint32_t n) {
            __syncwarp();
            const bool mine = lane < n;
            uint64_t v = 0;
            uint32_t meta = 0;
            if (mine) {
                v = qv[(qhead + lane) & (QCAP - 1)];
                meta = qm[(qhead + lane) & (QCAP - 1)];
            }
            __syncwarp();
            qhead += n;
            if (!mine) return;
            const uint32_t uidx = meta & 0xfff, slot = meta >> 12;
            const uint64_t tile = slot == SLOT_FAR ? tile_of(v, a.v_first, a.width) : tile_base + slot;
            for (uint32_t t = 0; t < nch; ++t) {
                const uint32_t vr = fastmod32(mod64(v, a.cmq[t]) * a.caq[t], a.cmq[t].c, a.cq[t]);
                int32_t m = (int32_t)ures[t * G::UB + uidx] - (int32_t)vr;
                if (m < 0) m += (int32_t)a.cq[t];
                if (!((cbits[t * CBW + (m >> 5)] >> (m & 31)) & 1u)) return;
                const uint32_t g = a.bgroup[NB + t];
                if (g) {
                    if (slot < a.tmax) atomicAdd(cnt_s + slot * stride + g, 1u);
                    else if (tile < a.ntiles)
                        atomicAdd((unsigned long long *)&a.counts[tile * (a.ng + 3) + g], 1ull);
                }
            }
            const uint32_t at = atomicAdd(deep_ctr, 1u);
            if (at < a.deep_cap)
                deep_slice[at] = make_uint4((uint32_t)v, (uint32_t)(v >> 32), block_u0 + uidx, (uint32_t)tile);
        };

        const uint32_t nrounds = (nv_item + 31) / 32;
        VRec next;
        if (warp < nrounds && warp * 32 + lane < nv_item) next = a.rec[va + warp * 32 + lane];
        for (uint32_t r = warp; r < nrounds; r += nwarps) {
            const uint32_t rel = r * 32 + lane;
            const bool active = rel < nv_item;
            const VRec rec = next;
            if (r + nwarps < nrounds && rel + nwarps * 32 < nv_item)
                next = a.rec[va + rel + nwarps * 32];     // prefetch one round ahead
            // warp-uniform: all 32 rows exist and cover the whole block
            const bool full = r * 32 >= full_lo && r * 32 + 32 <= full_hi;
            int32_t s = 0, e = 0;                         // piece as bits of the block
            if (active) {
                s = max((int32_t)(rec.left - block_u0), 0);
                e = min((int32_t)(rec.right - block_u0), (int32_t)G::UB);
                e = max(e, s);
            }
            const bool moved = active && (rec.v < t_lo || rec.v >= t_hi);
            if (__any_sync(0xffffffffu, moved)) {
                flush();
                if (moved) {
                    ctile = tile_of(rec.v, a.v_first, a.width);
                    t_lo = a.v_first + ctile * a.width;
                    t_hi = t_lo + a.width;
                }
            }
            uint32_t ro[NB];                              // unit offset of each filter's row
#pragma unroll
            for (int f = 0; f < NB; ++f) ro[f] = (uint32_t)(active ? rec.row[f] : a.row0[f]) * U;
            const uint64_t slot64 = ctile - tile_base;
            const uint32_t meta_hi = (slot64 < SLOT_FAR ? (uint32_t)slot64 : SLOT_FAR) << 12;

#pragma unroll 1
            for (uint32_t p = 0; p < U; ++p) {
                const uint32_t u = (lane + p) & (U - 1);
                uint4 acc = rows[ro[0] + u];
                uint4 acc4;
#pragma unroll
                for (int f = 1; f < NB; ++f) {
                    if (f == 4) acc4 = acc;
                    const uint4 w = rows[ro[f] + u];
                    acc.x &= w.x;
                    acc.y &= w.y;
                    acc.z &= w.z;
                    acc.w &= w.w;
                }
                if (NB <= 4) acc4 = acc;
                if (!full) {
                    const int32_t lo = s - (int32_t)u * 128, hi = e - (int32_t)u * 128;
                    const uint32_t m0 = unit_mask(lo, hi), m1 = unit_mask(lo - 32, hi - 32);
                    const uint32_t m2 = unit_mask(lo - 64, hi - 64), m3 = unit_mask(lo - 96, hi - 96);
                    acc.x &= m0, acc.y &= m1, acc.z &= m2, acc.w &= m3;
                    acc4.x &= m0, acc4.y &= m1, acc4.z &= m2, acc4.w &= m3;
                }
                c[0] += __popc(acc4.x) + __popc(acc4.y) + __popc(acc4.z) + __popc(acc4.w);
                if (c2_live) c[1] += __popc(acc.x) + __popc(acc.y) + __popc(acc.z) + __popc(acc.w);
                while (__any_sync(0xffffffffu, (acc.x | acc.y | acc.z | acc.w) != 0)) {
                    const bool has = (acc.x | acc.y | acc.z | acc.w) != 0;
                    const uint32_t bal = __ballot_sync(0xffffffffu, has);
                    if (has) {
                        uint32_t bit;
                        if (acc.x) {
                            bit = __ffs(acc.x) - 1;
                            acc.x &= acc.x - 1;
                        } else if (acc.y) {
                            bit = 32 + __ffs(acc.y) - 1;
                            acc.y &= acc.y - 1;
                        } else if (acc.z) {
                            bit = 64 + __ffs(acc.z) - 1;
                            acc.z &= acc.z - 1;
                        } else {
                            bit = 96 + __ffs(acc.w) - 1;
                            acc.w &= acc.w - 1;
                        }
                        const uint32_t at = (qtail + __popc(bal & lanes_below)) & (QCAP - 1);
                        qv[at] = rec.v;
                        qm[at] = (u * 128 + bit) | meta_hi;
                    }
                    qtail += __popc(bal);
                    if (qtail - qhead >= 32) drain(32);
                }
            }
        }
        if (qtail != qhead) drain(qtail - qhead);
        flush();
        __syncthreads();
        for (uint32_t k = threadIdx.x; k < a.tmax * stride; k += blockDim.x) {
            uint32_t cv = cnt_s[k];
            if (cv) {
                uint32_t slot = k / stride, g = k % stride;
                uint64_t tile = tile_base + slot;
                if (tile < a.ntiles)
                    atomicAdd((unsigned long long *)&a.counts[tile * (a.ng + 3) + g], (unsigned long long)cv);
            }
        }
    }
    __syncthreads();
    if (threadIdx.x == 0) a.deep_count[blockIdx.x] = *deep_ctr;
}

// x mod q for x < 2^96 from its six 16-bit limbs h (h[0] + sum h[k] (2^16k mod q), then one
// fast remainder; every partial sum stays below 2^32 because q < 2^13).
__device__ __forceinline__ uint32_t mod_limbs(const uint32_t h[6], const FiltC &f) {
    uint32_t t = h[0] + h[1] * f.r16[0] + h[2] * f.r16[1] + h[3] * f.r16[2] + h[4] * f.r16[3] + h[5] * f.r16[4];
    return fastmod32(t, f.c, f.q);
}

// Exact later filters on every deep record: x = uB - vA in two 64-bit limbs, filters first..nres-1
// with group counters, then the output record.  One record per thread; outputs are appended with
// one atomic per warp.
__global__ void __launch_bounds__(256) k_deep(const DeepArgs a) {
    const uint32_t lane = threadIdx.x & 31;
    const uint32_t lanes_below = (1u << lane) - 1u;
    const uint32_t slice = blockIdx.y;
    const uint32_t count = min(a.deep_count[slice], a.deep_cap);
    for (uint32_t base = blockIdx.x * blockDim.x; base < count; base += gridDim.x * blockDim.x) {
        const uint32_t at = base + threadIdx.x;
        const uint64_t i = (uint64_t)slice * a.deep_cap + at;
        const bool mine = at < count;
        bool pass = false;
        u128 x{0, 0};
        uint64_t tile = 0;
        if (mine) {
            const uint4 r = a.deep[i];
            const uint64_t v = (uint64_t)r.y << 32 | r.x;
            tile = r.w;
            const u128 pos = mul_wide(__ldg(a.us + r.z), a.B), shift = mul_wide(v, a.A);
            if (tile >= a.ntiles) {
            } else if (less128(pos, shift)) {
                atomicAdd((unsigned long long *)&a.counts[tile * (a.ng + 3) + a.ng + 2], 1ull);
            } else {
                x = sub128(pos, shift);
                const uint32_t h[6] = {(uint32_t)x.lo & 0xffffu, (uint32_t)(x.lo >> 16) & 0xffffu,
                                       (uint32_t)(x.lo >> 32) & 0xffffu, (uint32_t)(x.lo >> 48),
                                       (uint32_t)x.hi & 0xffffu, (uint32_t)(x.hi >> 16) & 0xffffu};
                pass = true;
                for (uint32_t idx = a.first; idx < a.nres; ++idx) {
                    const FiltC f = a.fcs[idx];
                    const uint32_t m = mod_limbs(h, f);
                    if (!((__ldg(a.bits + f.tab_off + (m >> 5)) >> (m & 31)) & 1u)) {
                        pass = false;
                        break;
                    }
                    if ((idx & 3) == 3 || idx + 1 == a.nres)
                        atomicAdd((unsigned long long *)&a.counts[tile * (a.ng + 3) + idx / 4 + 1], 1ull);
                }
            }
        }
        const uint32_t won = __ballot_sync(0xffffffffu, pass);
        if (won) {
            const uint32_t leader = __ffs(won) - 1;
            unsigned long long first = 0;
            if (lane == leader) first = atomicAdd(a.n_out, (unsigned long long)__popc(won));
            first = __shfl_sync(0xffffffffu, first, leader);
            if (pass) {
                const uint32_t same = __match_any_sync(won, tile);
                if (lane == (uint32_t)(__ffs(same) - 1))
                    atomicAdd((unsigned long long *)&a.counts[tile * (a.ng + 3) + a.ng + 1],
                              (unsigned long long)__popc(same));
                const unsigned long long o = first + __popc(won & lanes_below);
                if (o < a.out_cap) {
                    a.out[2 * o] = x.lo;
                    a.out[2 * o + 1] = x.hi | (tile << 32);
                }
            }
        }
    }
}

// ------------------------------------------------------------------------------------------
// plain per-position matcher (pseudocube/gpu.py:147-182): warp per v row, lanes over u

struct PlainArgs {
    const uint64_t *us;
    const uint64_t *vs;
    uint64_t nu, nv, A, B;
    u128 lo, hi;
    uint32_t nres, ng;
    const FiltConst *fc;
    const uint32_t *bits;
    uint64_t *counts;
    uint64_t *out;
    uint64_t out_cap;
};

__global__ void __launch_bounds__(256) k_plain(const PlainArgs a) {
    __shared__ unsigned long long cnt[PC_MAX_RES / 4 + 4];
    for (uint32_t k = threadIdx.x; k < a.ng + 3; k += blockDim.x) cnt[k] = 0;
    __syncthreads();
    const uint32_t lane = threadIdx.x & 31;
    const uint64_t warps = (uint64_t)gridDim.x * (blockDim.x >> 5);
    unsigned long long c0 = 0;
    for (uint64_t j = (blockIdx.x * (uint64_t)blockDim.x + threadIdx.x) >> 5; j < a.nv; j += warps) {
        const u128 shift = mul_wide(a.vs[j], a.A), upper = add128(shift, a.hi);
        const uint64_t left = count_le(a.us, a.nu, a.B, add128(shift, a.lo));
        for (uint64_t i = left + lane; i < a.nu; i += 32) {
            const u128 pos = mul_wide(a.us[i], a.B);
            if (less128(upper, pos)) break;
            if (less128(pos, shift)) {
                atomicAdd(&cnt[a.ng + 2], 1ull);
                continue;
            }
            const u128 x = sub128(pos, shift);
            ++c0;
            bool ok = true;
            for (uint32_t idx = 0; idx < a.nres; ++idx) {
                const FiltConst fc = a.fc[idx];
                uint32_t m = mod128(x, fc.m);
                if (!((__ldg(a.bits + fc.tab_off + (m >> 5)) >> (m & 31)) & 1u)) {
                    ok = false;
                    break;
                }
                if ((idx & 3) == 3 || idx + 1 == a.nres) atomicAdd(&cnt[idx / 4 + 1], 1ull);
            }
            if (!ok) continue;
            unsigned long long slot = atomicAdd((unsigned long long *)&a.counts[a.ng + 1], 1ull);
            if (slot < a.out_cap) {
                a.out[2 * slot] = x.lo;
                a.out[2 * slot + 1] = x.hi;
            }
        }
    }
    atomicAdd(&cnt[0], c0);
    __syncthreads();
    for (uint32_t k = threadIdx.x; k < a.ng + 3; k += blockDim.x)
        if (k != a.ng + 1 && cnt[k]) atomicAdd((unsigned long long *)&a.counts[k], cnt[k]);
}

template <int NB, int K, int NT>
int launch_match_t(pc_ctx *ctx, const MatchArgs &a, size_t smem, int grid) {
    auto kern = k_match<NB, K, NT>;
    cudaError_t e = cudaFuncSetAttribute(kern, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem);
    if (e != cudaSuccess) return pc_cuda_fail(ctx, e, "match smem attribute");
    kern<<<grid, NT, smem, ctx->stream>>>(a);
    PC_LAUNCHED(ctx, "match");
    return PC_OK;
}

template <int K, int NT>
int launch_match_k(pc_ctx *ctx, const MatchArgs &a, size_t smem, int grid) {
    switch (a.nb) {
        case 1: return launch_match_t<1, K, NT>(ctx, a, smem, grid);
        case 2: return launch_match_t<2, K, NT>(ctx, a, smem, grid);
        case 3: return launch_match_t<3, K, NT>(ctx, a, smem, grid);
        case 4: return launch_match_t<4, K, NT>(ctx, a, smem, grid);
        case 5: return launch_match_t<5, K, NT>(ctx, a, smem, grid);
        case 6: return launch_match_t<6, K, NT>(ctx, a, smem, grid);
        case 7: return launch_match_t<7, K, NT>(ctx, a, smem, grid);
        case 8: return launch_match_t<8, K, NT>(ctx, a, smem, grid);
    }
    return pc_fail(ctx, PC_INVALID, "unsupported bitset filter count");
}

template <int NT>
int launch_match_n(pc_ctx *ctx, const MatchArgs &a, uint32_t K, size_t smem, int grid) {
    if (K == 16) return launch_match_k<16, NT>(ctx, a, smem, grid);
    if (K == 32) return launch_match_k<32, NT>(ctx, a, smem, grid);
    return launch_match_k<64, NT>(ctx, a, smem, grid);
}

uint32_t inv_mod(uint32_t a, uint32_t q) {
    int64_t t = 0, nt = 1, r = q, nr = a % q;
    while (nr) {
        int64_t quo = r / nr, tmp;
        tmp = t - quo * nt; t = nt; nt = tmp;
        tmp = r - quo * nr; r = nr; nr = tmp;
    }
    if (r != 1) return 0;
    return (uint32_t)(t < 0 ? t + q : t);
}

double elapsed_ms(cudaEvent_t a, cudaEvent_t b) {
    float ms = 0;
    cudaEventElapsedTime(&ms, a, b);
    return ms;
}

}  // namespace

extern "C" int pc_filters_create(pc_ctx *ctx, uint64_t A, uint64_t B, const uint32_t *primes, uint32_t nres,
                                 const uint8_t *allowed, pc_filters **out) {
    *out = nullptr;
    if (nres == 0) return pc_fail(ctx, PC_INVALID, "bitset experiment requires at least one residual filter");
    if (nres > PC_MAX_RES || A == 0 || B == 0) return pc_fail(ctx, PC_INVALID, "invalid residual filters");
    pc_filters *f = new pc_filters();
    f->A = A;
    f->B = B;
    f->nres = nres;
    f->ng = (nres + 3) / 4;
    f->primes.assign(primes, primes + nres);
    std::vector<FiltConst> fc(nres);
    std::vector<uint32_t> bits;
    uint64_t off = 0;
    for (uint32_t i = 0; i < nres; ++i) {
        uint32_t q = primes[i];
        if (q < 2 || q >= 8192 || A % q == 0 || B % q == 0) {
            delete f;
            return pc_fail(ctx, PC_INVALID, "residual modulus must be in [2, 8192) and coprime to A and B");
        }
        fc[i].m = make_modq(q);
        fc[i].tab_off = (uint32_t)bits.size();
        FiltC c{};
        c.c = fc[i].m.c;
        c.q = q;
        c.tab_off = fc[i].tab_off;
        for (int k = 0; k < 5; ++k) c.r16[k] = (uint16_t)fc[i].m.r16[k];
        f->fcs.push_back(c);
        std::vector<uint32_t> w((q + 31) / 32, 0);
        for (uint32_t r = 0; r < q; ++r)
            if (allowed[off + r]) w[r / 32] |= 1u << (r % 32);
        bits.insert(bits.end(), w.begin(), w.end());
        off += q;
    }
    // patterns of the first filters: RR[j] = S'[(-j) mod q] with S'[k] = allowed[(A k) mod q]
    f->nbmax = std::min<uint32_t>(nres, PC_MAX_BITSET);
    std::vector<uint32_t> pat((size_t)PC_MAX_BITSET * PATW, 0);
    uint64_t aoff = 0;
    for (uint32_t i = 0; i < f->nbmax; ++i) {
        uint32_t q = primes[i];
        if (q > 2047) {
            f->nbmax = i;
            break;
        }
        uint32_t a = (uint32_t)(A % q), b = (uint32_t)(B % q);
        f->ainvb[i] = (uint32_t)((uint64_t)b * inv_mod(a, q) % q);
        for (uint32_t j = 0; j < 2 * q + 64; ++j) {
            uint32_t k = (q - j % q) % q;
            uint32_t m = (uint32_t)((uint64_t)a * k % q);
            if (allowed[aoff + m]) pat[(size_t)i * PATW + j / 32] |= 1u << (j % 32);
        }
        aoff += q;
        f->rows_sum[i + 1] = f->rows_sum[i] + q;
    }
    if (f->nbmax < std::min<uint32_t>(nres, 4)) {
        delete f;
        return pc_fail(ctx, PC_INVALID, "first residual filters too large for bitset rows");
    }
    f->fc_bytes = nres * sizeof(FiltConst);
    f->bits_bytes = bits.size() * 4;
    f->pat_bytes = pat.size() * 4;
    int rc = pc_alloc(ctx, (void **)&f->d_fc, f->fc_bytes);
    if (!rc) rc = pc_alloc(ctx, (void **)&f->d_bits, f->bits_bytes);
    if (!rc) rc = pc_alloc(ctx, (void **)&f->d_pat, f->pat_bytes);
    if (rc) {
        pc_filters_free(ctx, f);
        return rc;
    }
    cudaMemcpyAsync(f->d_fc, fc.data(), f->fc_bytes, cudaMemcpyHostToDevice, ctx->stream);
    cudaMemcpyAsync(f->d_bits, bits.data(), f->bits_bytes, cudaMemcpyHostToDevice, ctx->stream);
    cudaMemcpyAsync(f->d_pat, pat.data(), f->pat_bytes, cudaMemcpyHostToDevice, ctx->stream);
    cudaError_t e = cudaStreamSynchronize(ctx->stream);
    if (e != cudaSuccess) {
        pc_filters_free(ctx, f);
        return pc_cuda_fail(ctx, e, "filters upload");
    }
    *out = f;
    return PC_OK;
}

extern "C" int pc_filters_free(pc_ctx *ctx, pc_filters *f) {
    if (!f) return PC_OK;
    pc_release(ctx, f->d_fc, f->fc_bytes);
    pc_release(ctx, f->d_bits, f->bits_bytes);
    pc_release(ctx, f->d_pat, f->pat_bytes);
    delete f;
    return PC_OK;
}

namespace {

struct Tuned {
    uint32_t nb, K, threads, nch;
    uint64_t v_chunk;
};

// Residual filters after the bitset tier that the cheap tier can test (bitmap of <= 64 words).
uint32_t cheap_count(const pc_filters *f, uint32_t nb) {
    uint32_t n = 0;
    while (n < PC_MAX_CHEAP && nb + n < f->nres && f->primes[nb + n] <= 2047) ++n;
    return n;
}

Tuned resolve_tuning(pc_ctx *ctx, const pc_filters *f, const pc_tuning *t, size_t *smem_out, uint32_t *tmax_out) {
    Tuned r{};
    uint32_t nb_min = std::min<uint32_t>(f->nres, 4);
    r.nb = t && t->bitset_filters ? t->bitset_filters : std::min<uint32_t>(f->nbmax, 7);
    r.nb = std::max(nb_min, std::min(r.nb, f->nbmax));
    r.K = t && t->block_words ? t->block_words : 32;
    if (r.K != 16 && r.K != 32 && r.K != 64) r.K = 32;
    const bool fixed_threads = t && t->threads;
    r.threads = fixed_threads ? t->threads : 1024;
    if (r.threads != 512 && r.threads != 768 && r.threads != 1024) r.threads = 512;
    r.v_chunk = t ? t->v_chunk : 0;
    int optin = 0;
    cudaDeviceGetAttribute(&optin, cudaDevAttrMaxSharedMemoryPerBlockOptin, ctx->device);
    if (optin <= 0) optin = 227 * 1024;
    for (;;) {
        r.nch = cheap_count(f, r.nb);
        for (uint32_t tmax = TMAX_DEFAULT; tmax >= 4; tmax /= 2) {
            MatchSmem L(f->rows_sum[r.nb], r.K, r.nb, r.nch, tmax, f->ng, r.threads / 32);
            if (L.total <= (uint32_t)optin) {
                *tmax_out = tmax;
                *smem_out = L.total;
                return r;
            }
        }
        if (!fixed_threads && r.threads > 512) r.threads = r.threads == 1024 ? 768 : 512;
        else if (r.K > 16) r.K /= 2;
        else if (r.nb > nb_min) r.nb--;
        else {
            *smem_out = 0;
            return r;
        }
    }
}

struct BatchIO {
    uint64_t *counts, *geometry, *out;
    uint64_t out_cap, *n_out;
    pc_stats *stats;
};

// Device part shared by pc_run_batch and pc_run_lease.
int run_device(pc_ctx *ctx, const pc_filters *f, const pc_tuning *tuning, const uint64_t *d_us, uint64_t nu,
               const uint64_t *d_vs, uint64_t nv, u128 lo, u128 hi, uint64_t v_first, uint64_t width,
               uint32_t ntiles, uint64_t v_end, const BatchIO &io, int launches0) {
    if (nu >= (UINT64_C(1) << 31) || nv >= (UINT64_C(1) << 32)) return pc_fail(ctx, PC_INVALID, "focus list too long");
    if (hi.hi >= (UINT64_C(1) << 32)) return pc_fail(ctx, PC_INVALID, "interval bound must be below 2^96");
    if (f->nres > (uint32_t)FC_INLINE) return pc_fail(ctx, PC_INVALID, "more residual filters than the fused kernel holds");
    const uint32_t ng = f->ng, stride = ng + 3;
    size_t smem = 0;
    uint32_t tmax = 0;
    Tuned tn = resolve_tuning(ctx, f, tuning, &smem, &tmax);
    if (!smem) return pc_fail(ctx, PC_INVALID, "residual rows do not fit shared memory");
    const int grid = ctx->sm_count;
    uint32_t deep_cap = 1u << 15;
    for (int attempt = 0;; ++attempt) {
        Scratch s(ctx);
        uint64_t *d_counts, *d_geo, *d_out, *d_prefix, *d_vchunk, *d_pieces;
        unsigned long long *d_nout, *d_bad;
        VRec *d_rec;
        uint4 *d_bv, *d_deep;
        uint32_t *d_deep_count;
        const uint32_t UB = tn.K * 32;
        const uint64_t nblocks = (nu + UB - 1) / UB;
        int rc = s.get(&d_counts, (uint64_t)ntiles * stride);
        if (!rc) rc = s.get(&d_geo, 2 * (uint64_t)ntiles);
        if (!rc) rc = s.get(&d_out, 2 * std::max<uint64_t>(1, io.out_cap));
        if (!rc) rc = s.get(&d_nout, 2);
        if (!rc) rc = s.get(&d_rec, std::max<uint64_t>(1, nv));
        if (!rc) rc = s.get(&d_bv, std::max<uint64_t>(1, nblocks));
        if (!rc) rc = s.get(&d_pieces, std::max<uint64_t>(1, nblocks));
        if (!rc) rc = s.get(&d_prefix, nblocks + 1);
        if (!rc) rc = s.get(&d_vchunk, 1);
        if (!rc) rc = s.get(&d_deep, (uint64_t)grid * deep_cap);
        if (!rc) rc = s.get(&d_deep_count, grid);
        if (rc) return rc;
        d_bad = d_nout + 1;
        cudaStream_t st = ctx->stream;
        PC_CHECK(ctx, cudaMemsetAsync(d_counts, 0, (uint64_t)ntiles * stride * 8, st));
        PC_CHECK(ctx, cudaMemsetAsync(d_nout, 0, 16, st));
        PC_CHECK(ctx, cudaMemsetAsync(d_deep_count, 0, (uint64_t)grid * 4, st));
        PC_CHECK(ctx, cudaEventRecord(ctx->ev[0], st));
        int launches = launches0;

        PrepArgs pa{};
        pa.us = d_us;
        pa.vs = d_vs;
        pa.nu = nu;
        pa.nv = nv;
        pa.A = f->A;
        pa.B = f->B;
        pa.lo = lo;
        pa.hi = hi;
        pa.v_first = v_first;
        pa.width = width;
        pa.ntiles = ntiles;
        pa.nb = tn.nb;
        pa.ng = ng;
        for (uint32_t i = 0; i < tn.nb; ++i) {
            pa.q[i] = f->primes[i];
            pa.row0[i] = f->rows_sum[i];
            pa.mq[i] = make_modq(f->primes[i]);
        }
        pa.rec = d_rec;
        pa.counts = d_counts;
        pa.bad = d_bad;
        if (nv) {
            uint64_t runs = (nv + PREP_RUN - 1) / PREP_RUN;
            k_vprep<<<(unsigned)((runs + 127) / 128), 128, 0, st>>>(pa);
            PC_LAUNCHED(ctx, "vprep");
            ++launches;
        }
        k_geometry<<<(ntiles + 127) / 128, 128, 0, st>>>(d_us, nu, d_vs, nv, f->A, f->B, lo, hi, v_first, width,
                                                          v_end, ntiles, d_geo);
        PC_LAUNCHED(ctx, "geometry");
        ++launches;
        PC_CHECK(ctx, cudaEventRecord(ctx->ev[1], st));
        const bool run_match = nu && nv;
        uint32_t deep_max = 0;
        if (run_match) {
            k_blocks<<<(unsigned)((nblocks + 255) / 256), 256, 0, st>>>(d_rec, nv, nu, UB, nblocks, d_bv, d_pieces);
            PC_LAUNCHED(ctx, "blocks");
            uint64_t *d_items, *d_tmp;
            rc = s.get(&d_items, nblocks);
            if (!rc) rc = s.get(&d_tmp, nblocks + 1);
            if (!rc) rc = pc_exclusive_scan_u64(ctx, d_pieces, d_tmp, nblocks, d_tmp + nblocks);
            if (rc) return rc;
            k_chunk<<<1, 1, 0, st>>>(d_tmp + nblocks, tn.v_chunk, (uint64_t)grid * 32, d_vchunk);
            PC_LAUNCHED(ctx, "chunk");
            k_item_counts<<<(unsigned)((nblocks + 255) / 256), 256, 0, st>>>(d_pieces, nblocks, d_vchunk, d_items);
            PC_LAUNCHED(ctx, "item counts");
            rc = pc_exclusive_scan_u64(ctx, d_items, d_prefix, nblocks, d_prefix + nblocks);
            if (rc) return rc;
            launches += 7;
            MatchArgs ma{};
            ma.us = d_us;
            ma.vs = d_vs;
            ma.rec = d_rec;
            ma.nu = nu;
            ma.nv = nv;
            ma.A = f->A;
            ma.B = f->B;
            ma.lo = lo;
            ma.hi = hi;
            ma.nres = f->nres;
            ma.ng = ng;
            ma.nb = tn.nb;
            ma.tmax = tmax;
            ma.fc = f->d_fc;
            ma.bits = f->d_bits;
            ma.pat = f->d_pat;
            for (uint32_t i = 0; i < tn.nb; ++i) {
                ma.q[i] = f->primes[i];
                ma.row0[i] = f->rows_sum[i];
                ma.ainvb[i] = f->ainvb[i];
                ma.mq[i] = make_modq(f->primes[i]);
            }
            ma.total_rows = f->rows_sum[tn.nb];
            ma.counts = d_counts;
            ma.out = d_out;
            ma.out_cap = io.out_cap;
            ma.n_out = d_nout;
            ma.ntiles = ntiles;
            ma.bv = d_bv;
            ma.item_prefix = d_prefix;
            ma.nblocks = nblocks;
            ma.vchunk = d_vchunk;
            ma.v_first = v_first;
            ma.width = width;
            ma.nch = tn.nch;
            for (uint32_t t = 0; t < tn.nch; ++t) {
                const uint32_t q = f->primes[tn.nb + t];
                ma.cq[t] = q;
                ma.caq[t] = (uint32_t)(f->A % q);
                ma.cbq[t] = (uint32_t)(f->B % q);
                ma.cmq[t] = make_modq(q);
                ma.cbits_off[t] = f->fcs[tn.nb + t].tab_off;
            }
            for (uint32_t idx = 0; idx < 16; ++idx)
                ma.bgroup[idx] = (uint8_t)(idx < f->nres && ((idx & 3) == 3 || idx + 1 == f->nres) ? idx / 4 + 1 : 0);
            ma.deep = d_deep;
            ma.deep_cap = deep_cap;
            ma.deep_count = d_deep_count;
            PC_CHECK(ctx, cudaEventRecord(ctx->ev[2], st));
            if (tn.threads == 1024) rc = launch_match_n<1024>(ctx, ma, tn.K, smem, grid);
            else if (tn.threads == 768) rc = launch_match_n<768>(ctx, ma, tn.K, smem, grid);
            else rc = launch_match_n<512>(ctx, ma, tn.K, smem, grid);
            if (rc) return rc;
            ++launches;
            std::vector<uint32_t> deep_counts(grid);
            PC_CHECK(ctx, cudaMemcpyAsync(deep_counts.data(), d_deep_count, (uint64_t)grid * 4, cudaMemcpyDeviceToHost, st));
            PC_CHECK(ctx, cudaStreamSynchronize(st));
            for (uint32_t c : deep_counts) deep_max = std::max(deep_max, c);
            if (deep_max > deep_cap) {
                if (attempt) return pc_fail(ctx, PC_ARITHMETIC, "deep survivor count changed between attempts");
                deep_cap = deep_max + 1024;
                continue;                                  // rerun with room for every deep survivor
            }
            DeepArgs da{};
            da.us = d_us;
            da.deep = d_deep;
            da.deep_count = d_deep_count;
            da.deep_cap = deep_cap;
            da.slices = grid;
            da.A = f->A;
            da.B = f->B;
            da.first = tn.nb + tn.nch;
            da.nres = f->nres;
            da.ng = ng;
            da.ntiles = ntiles;
            da.bits = f->d_bits;
            da.counts = d_counts;
            da.out = d_out;
            da.out_cap = io.out_cap;
            da.n_out = d_nout;
            for (uint32_t i = 0; i < f->nres && i < (uint32_t)FC_INLINE; ++i) da.fcs[i] = f->fcs[i];
            if (deep_max) {
                dim3 dg((unsigned)std::min<uint64_t>((deep_max + 255) / 256, 64), (unsigned)grid);
                k_deep<<<dg, 256, 0, st>>>(da);
                PC_LAUNCHED(ctx, "deep");
                ++launches;
            }
            PC_CHECK(ctx, cudaEventRecord(ctx->ev[3], st));
        }
        unsigned long long host_nout[2] = {0, 0};
        PC_CHECK(ctx, cudaMemcpyAsync(host_nout, d_nout, 16, cudaMemcpyDeviceToHost, st));
        PC_CHECK(ctx, cudaMemcpyAsync(io.counts, d_counts, (uint64_t)ntiles * stride * 8, cudaMemcpyDeviceToHost, st));
        PC_CHECK(ctx, cudaMemcpyAsync(io.geometry, d_geo, 2 * (uint64_t)ntiles * 8, cudaMemcpyDeviceToHost, st));
        PC_CHECK(ctx, cudaStreamSynchronize(st));
        uint64_t n = host_nout[0];
        *io.n_out = n;
        if (io.stats) {
            io.stats->bounds_ms = elapsed_ms(ctx->ev[0], ctx->ev[1]);
            io.stats->kernel_ms = run_match ? elapsed_ms(ctx->ev[2], ctx->ev[3]) : 0.0;
            io.stats->outputs = n;
            io.stats->launches = launches;
            io.stats->work_items = deep_max;
            io.stats->reserved[0] = tn.nb;
            io.stats->reserved[1] = tn.K;
            io.stats->reserved[2] = tn.threads;
            io.stats->reserved[3] = tn.nch;
        }
        if (host_nout[1]) return pc_fail(ctx, PC_INVALID, "v row outside the subtile geometry");
        if (n > io.out_cap) return pc_fail(ctx, PC_OVERFLOW, "output overflow; attempt cannot commit");
        if (n) {
            PC_CHECK(ctx, cudaMemcpyAsync(io.out, d_out, 2 * n * 8, cudaMemcpyDeviceToHost, st));
            PC_CHECK(ctx, cudaStreamSynchronize(st));
        }
        for (uint32_t t = 0; t < ntiles; ++t)
            if (io.counts[(uint64_t)t * stride + ng + 2]) return pc_fail(ctx, PC_ARITHMETIC, "unsigned underflow flagged");
        return PC_OK;
    }
}

}  // namespace

int pc_window_into(pc_ctx *ctx, const pc_focus *f, uint64_t low, uint64_t high, uint64_t cap, uint64_t **out,
                   uint64_t *out_bytes, uint64_t *total_host, int *launches);

extern "C" int pc_run_batch(pc_ctx *ctx, const pc_filters *f, const pc_tuning *tuning, const pc_buf *us, uint64_t u_off,
                            uint64_t nu, const pc_buf *vs, uint64_t v_off, uint64_t nv, uint64_t lo0, uint64_t lo1,
                            uint64_t hi0, uint64_t hi1, uint64_t v_first, uint64_t width, uint32_t ntiles,
                            uint64_t v_end, uint64_t *counts, uint64_t *geometry, uint64_t *out, uint64_t out_cap,
                            uint64_t *n_out, pc_stats *stats) {
    if (!f || !us || !vs || width == 0 || ntiles == 0) return pc_fail(ctx, PC_INVALID, "invalid batch arguments");
    if (u_off > us->n || nu > us->n - u_off || v_off > vs->n || nv > vs->n - v_off)
        return pc_fail(ctx, PC_INVALID, "focus list slice out of range");
    if (v_end <= v_first || (v_end - v_first + width - 1) / width != ntiles)
        return pc_fail(ctx, PC_INVALID, "inconsistent subtile geometry");
    if (stats) memset(stats, 0, sizeof(*stats));
    auto t0 = std::chrono::steady_clock::now();
    BatchIO io{counts, geometry, out, out_cap, n_out, stats};
    int rc = run_device(ctx, f, tuning, us->d + u_off, nu, vs->d + v_off, nv, u128{lo0, lo1}, u128{hi0, hi1}, v_first,
                        width, ntiles, v_end, io, 0);
    if (stats) stats->total_ms = std::chrono::duration<double, std::milli>(std::chrono::steady_clock::now() - t0).count();
    return rc;
}

extern "C" int pc_run_lease(pc_ctx *ctx, const pc_focus *fa, const pc_focus *fb, const pc_filters *f,
                            const pc_tuning *tuning, uint64_t first, uint64_t end, uint64_t width, uint64_t lo0,
                            uint64_t lo1, uint64_t hi0, uint64_t hi1, uint64_t *counts, uint64_t *geometry,
                            uint64_t *out, uint64_t out_cap, uint64_t *n_out, pc_stats *stats) {
    if (!fa || !fb || !f || width == 0 || end <= first) return pc_fail(ctx, PC_INVALID, "invalid lease arguments");
    if (stats) memset(stats, 0, sizeof(*stats));
    auto t0 = std::chrono::steady_clock::now();
    typedef unsigned __int128 w128;
    w128 lo = (w128)lo1 << 64 | lo0, hi = (w128)hi1 << 64 | hi0;
    w128 ulo = (lo + (w128)first * f->A) / f->B + 1, uhi = (hi + (w128)(end - 1) * f->A) / f->B + 1;
    if (uhi >> 64) return pc_fail(ctx, PC_INVALID, "u window exceeds 64 bits");
    uint64_t ntiles64 = (end - first + width - 1) / width;
    if (ntiles64 >= (UINT64_C(1) << 31)) return pc_fail(ctx, PC_INVALID, "too many subtiles");
    int launches = 0;
    PC_CHECK(ctx, cudaEventRecord(ctx->ev[4], ctx->stream));
    uint64_t *d_us = nullptr, *d_vs = nullptr, us_bytes = 0, vs_bytes = 0, nu = 0, nv = 0;
    const uint64_t cap = (UINT64_C(1) << 32) - 1;
    int rc = pc_window_into(ctx, fa, (uint64_t)ulo, (uint64_t)uhi, cap, &d_us, &us_bytes, &nu, &launches);
    if (!rc) rc = pc_window_into(ctx, fb, first, end, cap, &d_vs, &vs_bytes, &nv, &launches);
    if (!rc) {
        cudaEventRecord(ctx->ev[5], ctx->stream);
        BatchIO io{counts, geometry, out, out_cap, n_out, stats};
        rc = run_device(ctx, f, tuning, d_us ? d_us : (const uint64_t *)nullptr, nu, d_vs, nv, u128{lo0, lo1},
                        u128{hi0, hi1}, first, width, (uint32_t)ntiles64, end, io, launches);
        if (stats) stats->window_ms = elapsed_ms(ctx->ev[4], ctx->ev[5]);
    }
    pc_release(ctx, d_us, us_bytes);
    pc_release(ctx, d_vs, vs_bytes);
    if (stats) stats->total_ms = std::chrono::duration<double, std::milli>(std::chrono::steady_clock::now() - t0).count();
    return rc;
}

extern "C" int pc_run_plain(pc_ctx *ctx, const pc_filters *f, const pc_buf *us, uint64_t u_off, uint64_t nu,
                            const pc_buf *vs, uint64_t v_off, uint64_t nv, uint64_t lo0, uint64_t lo1, uint64_t hi0,
                            uint64_t hi1, uint64_t *counts, uint64_t *out, uint64_t out_cap, pc_stats *stats) {
    if (!f || !us || !vs) return pc_fail(ctx, PC_INVALID, "invalid plain arguments");
    if (u_off > us->n || nu > us->n - u_off || v_off > vs->n || nv > vs->n - v_off)
        return pc_fail(ctx, PC_INVALID, "focus list slice out of range");
    if (stats) memset(stats, 0, sizeof(*stats));
    const uint32_t ng = f->ng;
    Scratch s(ctx);
    uint64_t *d_counts, *d_out;
    int rc = s.get(&d_counts, ng + 3);
    if (!rc) rc = s.get(&d_out, 2 * std::max<uint64_t>(1, out_cap));
    if (rc) return rc;
    cudaStream_t st = ctx->stream;
    PC_CHECK(ctx, cudaMemsetAsync(d_counts, 0, (ng + 3) * 8, st));
    PC_CHECK(ctx, cudaEventRecord(ctx->ev[6], st));
    if (nu && nv) {
        PlainArgs a{};
        a.us = us->d + u_off;
        a.vs = vs->d + v_off;
        a.nu = nu;
        a.nv = nv;
        a.A = f->A;
        a.B = f->B;
        a.lo = u128{lo0, lo1};
        a.hi = u128{hi0, hi1};
        a.nres = f->nres;
        a.ng = ng;
        a.fc = f->d_fc;
        a.bits = f->d_bits;
        a.counts = d_counts;
        a.out = d_out;
        a.out_cap = out_cap;
        uint64_t blocks = std::min<uint64_t>((nv + 7) / 8, (uint64_t)ctx->sm_count * 8);
        k_plain<<<(unsigned)blocks, 256, 0, st>>>(a);
        PC_LAUNCHED(ctx, "plain match");
    }
    PC_CHECK(ctx, cudaEventRecord(ctx->ev[7], st));
    PC_CHECK(ctx, cudaMemcpyAsync(counts, d_counts, (ng + 3) * 8, cudaMemcpyDeviceToHost, st));
    PC_CHECK(ctx, cudaStreamSynchronize(st));
    uint64_t n = counts[ng + 1];
    if (stats) {
        stats->kernel_ms = elapsed_ms(ctx->ev[6], ctx->ev[7]);
        stats->outputs = n;
        stats->launches = nu && nv ? 1 : 0;
    }
    uint64_t copy = std::min(n, out_cap);
    if (copy) {
        PC_CHECK(ctx, cudaMemcpyAsync(out, d_out, 2 * copy * 8, cudaMemcpyDeviceToHost, st));
        PC_CHECK(ctx, cudaStreamSynchronize(st));
    }
    return PC_OK;
}

// ------------------------------------------------------------------------------------------
// Plain per-tile matcher with no device allocation (pc_run_plain_static).
//
// Its scratch is this file-scope device array, reserved when the library loads and held by every
// GPU that loads it until the process exits.  Host code must not pass the array's name to a
// kernel (on the host the name is only a stand-in, not a device address): the device address is
// looked up once per device with cudaGetSymbolAddress and cached.  Every call reuses the same
// bytes, so calls that overlap on one GPU race with each other.

constexpr uint64_t STATIC_SCRATCH_BYTES = UINT64_C(16) << 20;   // 16 MiB
static __device__ __align__(256) unsigned char g_static_scratch[STATIC_SCRATCH_BYTES];

namespace {
constexpr int STATIC_MAX_DEVICES = 64;
unsigned char *g_static_ptr[STATIC_MAX_DEVICES] = {};

inline uint64_t align256(uint64_t x) { return (x + 255) & ~UINT64_C(255); }

int static_fail(char *err, int err_len, int code, const char *msg) {
    if (err && err_len > 0) {
        strncpy(err, msg, (size_t)err_len - 1);
        err[err_len - 1] = 0;
    }
    return code;
}

int static_cuda(char *err, int err_len, cudaError_t e, const char *what) {
    char buf[256];
    snprintf(buf, sizeof(buf), "%s: %s", what, cudaGetErrorString(e));
    return static_fail(err, err_len, PC_CUDA, buf);
}
}  // namespace

extern "C" int pc_run_plain_static(int device, const uint64_t *us, uint64_t nu, const uint64_t *vs, uint64_t nv,
                                   uint64_t A, uint64_t B, uint64_t lo0, uint64_t lo1, uint64_t hi0, uint64_t hi1,
                                   const uint32_t *primes, uint32_t nres, const uint8_t *allowed, uint64_t *counts,
                                   uint64_t *out, uint64_t out_cap, char *err, int err_len) {
    if (device < 0 || device >= STATIC_MAX_DEVICES) return static_fail(err, err_len, PC_INVALID, "device index out of range");
    if (nres == 0 || nres > PC_MAX_RES || A == 0 || B == 0 || !counts || (nu && !us) || (nv && !vs))
        return static_fail(err, err_len, PC_INVALID, "invalid plain tile arguments");
    uint64_t words = 0;
    for (uint32_t i = 0; i < nres; ++i) {
        const uint32_t q = primes[i];
        if (q < 2 || q >= 8192 || A % q == 0 || B % q == 0)
            return static_fail(err, err_len, PC_INVALID, "residual modulus must be in [2, 8192) and coprime to A and B");
        words += (q + 31) / 32;
    }
    const uint32_t ng = (nres + 3) / 4;
    // layout of the static scratch: counters | filter constants | bitmaps | us | vs | outputs
    const uint64_t o_counts = 0, o_fc = align256(o_counts + (ng + 3) * 8), o_bits = align256(o_fc + nres * sizeof(FiltConst));
    const uint64_t o_us = align256(o_bits + words * 4), o_vs = align256(o_us + nu * 8), o_out = align256(o_vs + nv * 8);
    const uint64_t need = o_out + 2 * (out_cap ? out_cap : 1) * 8;
    if (need > STATIC_SCRATCH_BYTES)
        return static_fail(err, err_len, PC_INVALID, "tile exceeds the 16 MiB static scratch of pc_run_plain_static");

    cudaError_t e = cudaSetDevice(device);
    if (e != cudaSuccess) return static_cuda(err, err_len, e, "cudaSetDevice");
    if (!g_static_ptr[device]) {          // set-up, once per device, with that device current
        void *ptr = nullptr;
        e = cudaGetSymbolAddress(&ptr, g_static_scratch);
        if (e != cudaSuccess) return static_cuda(err, err_len, e, "cudaGetSymbolAddress");
        g_static_ptr[device] = (unsigned char *)ptr;
    }
    unsigned char *base = g_static_ptr[device];
    cudaStream_t st = 0;
    // filter constants and packed bitmaps, staged through fixed host buffers
    {
        FiltConst fc[32];
        uint32_t bits[1024];
        uint64_t word_at = 0, nbits = 0, off = 0;
        uint32_t nfc = 0, fc_at = 0;
        for (uint32_t i = 0; i < nres; ++i) {
            const uint32_t q = primes[i];
            FiltConst &c = fc[nfc++];
            c.m = make_modq(q);
            c.tab_off = (uint32_t)(word_at + nbits);
            c.pad = 0;
            for (uint32_t w = 0; w < (q + 31) / 32; ++w) {
                uint32_t v = 0;
                for (uint32_t r = w * 32; r < q && r < w * 32 + 32; ++r)
                    if (allowed[off + r]) v |= 1u << (r - w * 32);
                bits[nbits++] = v;
                if (nbits == 1024) {
                    e = cudaMemcpyAsync(base + o_bits + word_at * 4, bits, nbits * 4, cudaMemcpyHostToDevice, st);
                    if (e == cudaSuccess) e = cudaStreamSynchronize(st);
                    if (e != cudaSuccess) return static_cuda(err, err_len, e, "bitmap upload");
                    word_at += nbits;
                    nbits = 0;
                }
            }
            off += q;
            if (nfc == 32 || i + 1 == nres) {
                e = cudaMemcpyAsync(base + o_fc + (uint64_t)fc_at * sizeof(FiltConst), fc, nfc * sizeof(FiltConst),
                                    cudaMemcpyHostToDevice, st);
                if (e == cudaSuccess) e = cudaStreamSynchronize(st);
                if (e != cudaSuccess) return static_cuda(err, err_len, e, "filter upload");
                fc_at += nfc;
                nfc = 0;
            }
        }
        if (nbits) {
            e = cudaMemcpyAsync(base + o_bits + word_at * 4, bits, nbits * 4, cudaMemcpyHostToDevice, st);
            if (e == cudaSuccess) e = cudaStreamSynchronize(st);
            if (e != cudaSuccess) return static_cuda(err, err_len, e, "bitmap upload");
        }
    }
    e = cudaMemsetAsync(base + o_counts, 0, (ng + 3) * 8, st);   // the array keeps the previous call's counts
    if (e == cudaSuccess && nu) e = cudaMemcpyAsync(base + o_us, us, nu * 8, cudaMemcpyHostToDevice, st);
    if (e == cudaSuccess && nv) e = cudaMemcpyAsync(base + o_vs, vs, nv * 8, cudaMemcpyHostToDevice, st);
    if (e != cudaSuccess) return static_cuda(err, err_len, e, "input upload");
    if (nu && nv) {
        int sm = 0;
        cudaDeviceGetAttribute(&sm, cudaDevAttrMultiProcessorCount, device);
        PlainArgs a{};
        a.us = (const uint64_t *)(base + o_us);
        a.vs = (const uint64_t *)(base + o_vs);
        a.nu = nu;
        a.nv = nv;
        a.A = A;
        a.B = B;
        a.lo = u128{lo0, lo1};
        a.hi = u128{hi0, hi1};
        a.nres = nres;
        a.ng = ng;
        a.fc = (const FiltConst *)(base + o_fc);
        a.bits = (const uint32_t *)(base + o_bits);
        a.counts = (uint64_t *)(base + o_counts);
        a.out = (uint64_t *)(base + o_out);
        a.out_cap = out_cap;
        uint64_t blocks = std::min<uint64_t>((nv + 7) / 8, (uint64_t)std::max(sm, 1) * 8);
        k_plain<<<(unsigned)blocks, 256, 0, st>>>(a);
        e = cudaGetLastError();
        if (e != cudaSuccess) return static_cuda(err, err_len, e, "plain match launch");
    }
    e = cudaMemcpyAsync(counts, base + o_counts, (ng + 3) * 8, cudaMemcpyDeviceToHost, st);
    if (e == cudaSuccess) e = cudaStreamSynchronize(st);
    if (e != cudaSuccess) return static_cuda(err, err_len, e, "counter download");
    const uint64_t copy = std::min(counts[ng + 1], out_cap);
    if (copy && out) {
        e = cudaMemcpyAsync(out, base + o_out, 2 * copy * 8, cudaMemcpyDeviceToHost, st);
        if (e == cudaSuccess) e = cudaStreamSynchronize(st);
        if (e != cudaSuccess) return static_cuda(err, err_len, e, "output download");
    }
    return PC_OK;
}
