// Stages 2 and 3: residue-bitset intersection and exact 128-bit later filters, over one or many
// windows ("segments") in one launch sequence.
//
// Layout.  The sorted u lists of all segments are concatenated, each starting on a 2048-entry
// boundary, and cut into blocks of K words (32 u per word); a block therefore belongs to exactly
// one segment.  The v lists are concatenated unpadded.  A work item is one u block and a run of
// consecutive v rows (of the block's segment) whose exact u interval meets the block.  The CTA
// that owns an item builds, in shared memory, the residue rows of the first NB residual filters
// of the segment's filter family for its block (row r of filter q, bit i <=> allowed_q[(u_i B -
// r A) mod q]) and then streams its v rows: one lane per (v row, block) piece reads the K-word
// rows selected by v mod q with 128-bit loads, ANDs them, counts the group survivors by
// popcount, and queues the bits that survive every bitset filter.  Queued survivors are tested
// by a warp against the next few filters from residues of u and v (the cheap tier); the rest go
// to a per-CTA slice that k_deep finishes in exact 128-bit arithmetic.
//
// Rows are stored unswizzled, K/4 16-byte units per row; lane l reads unit (l + p) mod (K/4) at
// step p, so the 32 lanes of a warp spread evenly over the bank groups whatever rows they read.
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

// Compact filter constants: fast remainder constant, modulus, bitmap offset and 2^(16k) mod q for
// k = 1..5 (x < 2^96).
struct FiltC {
    uint64_t c;
    uint32_t q, tab_off;
    uint16_t r16[5];
    uint16_t pad[3];
};

struct pc_filters {
    uint64_t A = 0, B = 0;
    uint32_t nres = 0, ng = 0;
    std::vector<uint32_t> primes;
    FiltConst *d_fc = nullptr;
    FiltC *d_fcs = nullptr;
    uint32_t *d_bits = nullptr;
    uint32_t *d_pat = nullptr;       // rotation patterns of the first filters (PATW words each)
    uint64_t fc_bytes = 0, fcs_bytes = 0, bits_bytes = 0, pat_bytes = 0;
    uint32_t nbmax = 0;              // filters usable as bitset rows
    uint32_t ainvb[PC_MAX_BITSET] = {};
    uint32_t rows_sum[PC_MAX_BITSET + 1] = {};   // prefix sums of q over the first filters
    std::vector<FiltC> fcs;
};

namespace {

constexpr int PATW = 136;            // pattern words per bitset filter (q <= 2047)
constexpr int TMAX_DEFAULT = 64;     // subtile counter slots per CTA
constexpr uint64_t SEG_ALIGN = 2048; // u entries: every segment's u list starts on a block boundary

struct __align__(16) VRec {
    uint32_t left, right;            // exact u interval as indices into the concatenated u list
    uint64_t v;
    uint16_t row[8];                 // row index (row0 + v mod q) of each bitset filter
};

// One window: its focus moduli, interval, subtile geometry and slices of the concatenated lists.
struct SegDev {
    uint64_t A, B;
    u128 lo, hi;
    uint64_t v_first, width, v_end;
    uint32_t u_off, nu, v_off, nv;
    uint32_t tile_base, ntiles, fam, pad;
};

// One residual filter family (the filter list of one (p, A, B)) as the launch uses it: bitset
// filters 0..NB-1, cheap-tier filters NB..NB+nch-1, the rest in k_deep.
struct FamDev {
    uint32_t nres, ng, total_rows, c2_live;   // c2_live: group 2 ends at the last bitset filter
    uint32_t q[PC_MAX_BITSET], row0[PC_MAX_BITSET], ainvb[PC_MAX_BITSET];
    ModQ mq[PC_MAX_BITSET];
    uint32_t cq[PC_MAX_CHEAP], caq[PC_MAX_CHEAP], cbq[PC_MAX_CHEAP], cbits_off[PC_MAX_CHEAP];
    ModQ cmq[PC_MAX_CHEAP];
    uint8_t bgroup[16];              // group ended by filter idx (0 = none), idx < NB + nch
    uint32_t cqg[PC_MAX_CHEAP];      // cheap-tier filter t: q | the group it ends (bgroup[NB + t]) << 16
    const uint32_t *pat;
    const uint32_t *bits;
    const FiltC *fcs;
};

struct MatchArgs {
    const uint64_t *us;
    const VRec *rec;
    const uint64_t *cres;            // per v: cheap-tier residues v*A mod q, 16 bits each
    const SegDev *seg;
    const FamDev *fam;
    const uint32_t *blk_seg;         // per u block: its segment
    uint32_t nch, tmax, stride;      // stride: counters per subtile (largest ng + 3)
    uint32_t total_rows;             // largest over the families
    uint64_t *counts;                // ntiles x stride
    const uint4 *bv;                 // per u block: v rows meeting it, v rows covering it
    const uint64_t *item_prefix;     // nblocks + 1
    uint64_t nblocks;
    const uint64_t *vchunk;          // device scalar
    uint4 *deep;                     // (v lo, v hi, u index, subtile) records
    uint32_t deep_cap;               // records per CTA slice
    uint32_t *deep_count;            // per CTA (may exceed deep_cap: the caller retries larger)
    unsigned long long *item_next;   // next unclaimed work item (zeroed before the launch)
};

struct DeepArgs {
    const uint64_t *us;
    const uint4 *deep;
    const uint32_t *deep_count;
    uint32_t deep_cap, first, stride;        // filters first .. nres-1 remain
    uint64_t ntiles;
    const SegDev *seg;
    const FamDev *fam;
    const uint32_t *tile_seg;
    uint64_t *counts;
    uint64_t *out;
    uint64_t out_cap;
    unsigned long long *n_out;
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

// Subtile of v inside a segment, floor((v - v_first) / width), or ntiles when v lies outside.
// The double estimate is within one of the quotient (quotients are below 2^31), and the host
// guarantees ntiles * width < 2^64.
__device__ __forceinline__ uint64_t local_tile(uint64_t v, uint64_t v_first, uint64_t width, uint64_t ntiles) {
    if (v < v_first) return ntiles;
    const uint64_t d = v - v_first;
    uint64_t t = (uint64_t)((double)d / (double)width);
    if (t > ntiles) return ntiles;
    if (t && t * width > d) --t;
    if (t < ntiles && (t + 1) * width <= d) ++t;
    return t;
}

// Last segment whose list starts at or before index j (an empty segment shares its start with the
// next one, so the search lands on the segment that holds j).
__device__ __forceinline__ uint32_t seg_of_v(const SegDev *__restrict__ seg, uint32_t nseg, uint64_t j) {
    uint32_t lo = 0, hi = nseg;
    while (hi - lo > 1) {
        const uint32_t mid = (lo + hi) / 2;
        if (seg[mid].v_off <= j) lo = mid;
        else hi = mid;
    }
    return lo;
}

__device__ __forceinline__ uint32_t seg_of_u(const SegDev *__restrict__ seg, uint32_t nseg, uint64_t j) {
    uint32_t lo = 0, hi = nseg;
    while (hi - lo > 1) {
        const uint32_t mid = (lo + hi) / 2;
        if (seg[mid].u_off <= j) lo = mid;
        else hi = mid;
    }
    return lo;
}

struct PrepArgs {
    const uint64_t *us;
    const uint64_t *vs;
    uint64_t nv;
    const SegDev *seg;
    uint32_t nseg;
    const FamDev *fam;
    uint32_t nb, stride;
    VRec *rec;
    uint64_t *cres;                  // per v: v*A mod q of the cheap-tier filters, 16 bits each
    uint32_t nch;
    uint64_t *counts;
    unsigned long long *bad;
};

// Per v row: exact u interval as list indices (batch_experiment.py:209-215), bitset row
// indices, the residues v*A mod q of the cheap-tier filters, and the focused-position count of
// its subtile.  A thread owns PREP_RUN consecutive v
// rows: one binary search per bound for the first row of each segment, then the monotone bounds
// advance linearly (about N_u/N_v < 1 step per row).
constexpr int PREP_RUN = 16;

// Monotone advance of a bound from its previous position: a few linear steps, then a galloping
// search (strides 8, 16, 32, ...) that brackets the answer, then a binary search inside the
// bracket, so a row whose bound moved by g entries costs O(log g) loads near the previous bound.
__device__ __forceinline__ uint64_t advance_le(const uint64_t *__restrict__ us, uint64_t n, uint64_t B, u128 key,
                                               uint64_t from) {
    for (int step = 0; step < 4; ++step) {
        if (from >= n || less128(key, mul_wide(__ldg(us + from), B))) return from;
        ++from;
    }
    uint64_t lo = from, stride = 8;                      // us[lo - 1] * B <= key
    for (;;) {
        const uint64_t probe = lo + stride;
        if (probe >= n) return lo + count_le(us + lo, n - lo, B, key);
        if (less128(key, mul_wide(__ldg(us + probe), B))) return lo + count_le(us + lo, probe - lo, B, key);
        lo = probe + 1;
        stride *= 2;
    }
}

__global__ void k_vprep(const PrepArgs a) {
    const uint64_t t = blockIdx.x * (uint64_t)blockDim.x + threadIdx.x;
    const uint64_t j0 = t * PREP_RUN;
    if (j0 >= a.nv) return;
    const uint64_t j1 = umin64(a.nv, j0 + PREP_RUN);
    uint32_t s = seg_of_v(a.seg, a.nseg, j0);
    uint64_t left = 0, right = 0, tile = UINT64_MAX, t_lo = 1, t_hi = 0, pop = 0;
    bool fresh = true;
    for (uint64_t j = j0; j < j1; ++j) {
        while (s + 1 < a.nseg && j >= (uint64_t)a.seg[s].v_off + a.seg[s].nv) {
            ++s;
            fresh = true;
        }
        const SegDev &g = a.seg[s];
        const FamDev &F = a.fam[g.fam];
        const uint64_t u0 = g.u_off, u1 = u0 + g.nu;
        const uint64_t v = a.vs[j];
        const u128 shift = mul_wide(v, g.A);
        const u128 klo = add128(shift, g.lo), khi = add128(shift, g.hi);
        if (fresh) {
            left = u0 + count_le(a.us + u0, g.nu, g.B, klo);
            right = umax64(left, u0 + count_le(a.us + u0, g.nu, g.B, khi));
            t_lo = 1, t_hi = 0;                           // force a subtile lookup
            fresh = false;
        } else {
            left = advance_le(a.us, u1, g.B, klo, left);
            right = advance_le(a.us, u1, g.B, khi, umax64(left, right));
        }
        if (v < t_lo || v >= t_hi) {
            if (tile != UINT64_MAX && pop) atomicAdd((unsigned long long *)&a.counts[tile * a.stride], (unsigned long long)pop);
            pop = 0;
            const uint64_t lt = local_tile(v, g.v_first, g.width, g.ntiles);
            if (lt >= g.ntiles) {
                atomicAdd(a.bad, 1ull);
                tile = UINT64_MAX, t_lo = 1, t_hi = 0;
            } else {
                tile = g.tile_base + lt;
                t_lo = g.v_first + lt * g.width;
                t_hi = t_lo + g.width;
            }
        }
        VRec r;
        r.left = (uint32_t)left;
        r.right = (uint32_t)right;
        r.v = v;
#pragma unroll
        for (int f = 0; f < PC_MAX_BITSET; ++f)
            r.row[f] = f < (int)a.nb ? (uint16_t)(F.row0[f] + mod64(v, F.mq[f])) : (uint16_t)0;
        a.rec[j] = r;
        uint64_t cr = 0;
#pragma unroll
        for (int t = 0; t < PC_MAX_CHEAP; ++t)
            if (t < (int)a.nch) cr |= (uint64_t)fastmod32(mod64(v, F.cmq[t]) * F.caq[t], F.cmq[t].c, F.cq[t]) << (16 * t);
        a.cres[j] = cr;
        pop += right - left;
    }
    if (tile != UINT64_MAX && pop) atomicAdd((unsigned long long *)&a.counts[tile * a.stride], (unsigned long long)pop);
}

// Per subtile: u count and v count of its envelope (searchsorted bounds of
// batch_experiment.py:37-43, as list-independent differences).
__global__ void k_geometry(const uint64_t *__restrict__ us, const uint64_t *__restrict__ vs, const SegDev *__restrict__ seg,
                           const uint32_t *__restrict__ tile_seg, uint64_t ntiles, uint64_t *__restrict__ geometry) {
    const uint64_t t = blockIdx.x * (uint64_t)blockDim.x + threadIdx.x;
    if (t >= ntiles) return;
    const SegDev &g = seg[tile_seg[t]];
    const uint64_t first = g.v_first + (t - g.tile_base) * g.width;
    const uint64_t end = umin64(first + g.width, g.v_end);
    const uint64_t *su = us + g.u_off, *sv = vs + g.v_off;
    const uint64_t ua = count_le(su, g.nu, g.B, add128(mul_wide(first, g.A), g.lo));
    const uint64_t ub = count_le(su, g.nu, g.B, add128(mul_wide(end - 1, g.A), g.hi));
    const uint64_t va = lower_bound64(sv, g.nv, first), vb = lower_bound64(sv, g.nv, end);
    geometry[2 * t] = ub > ua ? ub - ua : 0;
    geometry[2 * t + 1] = vb - va;
}

// Per u block of UB entries: [va, vb) of v rows whose [left, right) meets the block, and the
// sub-range [f0, f1) of rows covering the whole block (left <= start and right >= stop); left and
// right are monotone in the row index within a segment, so all four are binary searches.
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

__global__ void k_blocks(const VRec *__restrict__ rec, const SegDev *__restrict__ seg, uint32_t nseg, uint32_t UB,
                         uint64_t nblocks, uint4 *__restrict__ bv, uint32_t *__restrict__ blk_seg,
                         uint64_t *__restrict__ pieces) {
    const uint64_t b = blockIdx.x * (uint64_t)blockDim.x + threadIdx.x;
    if (b >= nblocks) return;
    const uint64_t start = b * UB;
    const uint32_t s = seg_of_u(seg, nseg, start);
    const SegDev &g = seg[s];
    const uint64_t u_end = (uint64_t)g.u_off + g.nu;
    blk_seg[b] = s;
    if (start >= u_end) {                                 // padding between segments
        bv[b] = make_uint4(0, 0, 0, 0);
        pieces[b] = 0;
        return;
    }
    const uint64_t stop = umin64(u_end, start + UB);
    const uint64_t r0 = g.v_off, r1 = r0 + g.nv;
    const uint64_t va = first_right_ge(rec, r0, r1, start + 1);
    const uint64_t vb = first_left_ge(rec, va, r1, stop);
    uint64_t f0 = umax64(va, first_right_ge(rec, va, vb, stop));
    uint64_t f1 = umin64(vb, first_left_ge(rec, va, vb, start + 1));
    if (f1 < f0) f1 = f0;
    bv[b] = make_uint4((uint32_t)va, (uint32_t)vb, (uint32_t)f0, (uint32_t)f1);
    pieces[b] = vb > va ? vb - va : 0;
}

// v chunk per work item: fixed, or total pieces / target items, at least min_chunk (four rounds of
// 32 rows for every warp of a k_match CTA, so a small launch keeps every warp busy and pays the
// per-item set-up over enough rows) and at most 2^20.
__global__ void k_chunk(const uint64_t *__restrict__ total_pieces, uint64_t fixed_chunk, uint64_t target_items,
                        uint64_t min_chunk, uint64_t *__restrict__ vchunk) {
    uint64_t c = fixed_chunk;
    if (!c) c = umax64((*total_pieces + target_items - 1) / umax64(1, target_items), min_chunk);
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

// Residue rows of the family's first NB filters for one block (entries >= n_valid are zero), and
// the residues u*B mod q of its cheap-tier filters.
template <int NB, int K>
__device__ void build_rows(const uint64_t *__restrict__ us, const FamDev &F, uint32_t nch, uint4 *__restrict__ rows,
                           uint16_t *__restrict__ ures, const uint32_t *__restrict__ pat_s, uint32_t block_u0,
                           uint32_t n_valid, uint32_t lane, uint32_t warp, uint32_t nwarps) {
    using G = Geo<K>;
    const uint64_t *ub = us + block_u0;
    for (uint32_t k = threadIdx.x; k < G::UB; k += blockDim.x) {
        const uint64_t u = k < n_valid ? __ldg(ub + k) : 0;
        for (uint32_t t = 0; t < nch; ++t)
            ures[t * G::UB + k] = (uint16_t)fastmod32(mod64(u, F.cmq[t]) * F.cbq[t], F.cmq[t].c, F.cq[t]);
    }
    // A warp builds all q rows of one filter for two 16-byte units, c and c + U/2 (4 words = 128 u
    // each).  Its lanes store the two units in two steps, half the lanes writing each unit, so a
    // quarter-warp store meets two bank groups instead of one.
    uint32_t sh[5], keep[5];                              // per-lane transpose constants
    transpose_consts(lane, sh, keep);
    constexpr uint32_t HU = G::U / 2;
    const bool hi_first = lane & 4;
    for (uint32_t item = warp; item < NB * HU; item += nwarps) {
        const uint32_t f = item / HU, c = item % HU;
        const uint32_t q = F.q[f];
        uint32_t t[8];
        bool valid[8];
#pragma unroll
        for (int k = 0; k < 8; ++k) {
            const uint32_t local = ((c + (k >> 2) * HU) * 4 + (k & 3)) * 32 + lane;
            valid[k] = local < n_valid;
            const uint32_t um = valid[k] ? mod64(__ldg(ub + local), F.mq[f]) : 0;
            t[k] = fastmod32(um * F.ainvb[f], F.mq[f].c, q);
        }
        const uint32_t *p = pat_s + f * PATW;
        const uint32_t row0 = F.row0[f];
        for (uint32_t g = 0; g * 32 < q; ++g) {
            uint32_t w[8];
#pragma unroll
            for (int k = 0; k < 8; ++k) {
                const uint32_t st = 32 * g + q - t[k];
                const uint32_t col = __funnelshift_r(p[st >> 5], p[(st >> 5) + 1], st & 31);
                w[k] = transpose32c(valid[k] ? col : 0u, sh, keep);
            }
            const uint32_t r = 32 * g + lane;
            if (r < q) {
                const uint4 lo = make_uint4(w[0], w[1], w[2], w[3]), hi = make_uint4(w[4], w[5], w[6], w[7]);
                rows[G::unit(row0 + r, hi_first ? c + HU : c)] = hi_first ? hi : lo;
                rows[G::unit(row0 + r, hi_first ? c : c + HU)] = hi_first ? lo : hi;
            }
        }
    }
}

constexpr int CBW = 64;                 // bitmap words per cheap-tier filter (q <= 2047)
constexpr uint64_t ITEM_GRAB = 2;       // fewest work items a CTA claims at a time
// Survivor ring per warp (pending < 64 by construction).  An entry is one word pair: the record's
// index in the work item (< 2^20) | the bit's position in the block (< 2^12) << 20, and the
// survivor's subtile slot; the drain reads the v row's cheap-tier residues by the record index.
constexpr int QCAP = 64;
// Leftover list per warp: a piece's marked units after its first, as the record's index in the
// work item | the unit << 20 | the subtile slot << 24 (255: recomputed from v), recomputed 32 at a
// time so the round loop does not wait on a few lanes.
constexpr int LCAP = 32;

__host__ __device__ constexpr uint32_t round16(uint32_t x) { return (x + 15) & ~15u; }

// Shared-memory layout of k_match (byte offsets); every region starts 16-byte aligned.  The
// residue-row patterns are only read while rows are built, when every survivor ring is empty,
// so they share the rings' space.
struct MatchSmem {
    uint32_t rows, ures, ring, lq, pat, cbits, cnt, fam, seg, misc, total;
    __host__ __device__ MatchSmem(uint32_t total_rows, uint32_t K, uint32_t nb, uint32_t nch, uint32_t tmax,
                                  uint32_t ng, uint32_t warps) {
        rows = 0;
        ures = rows + total_rows * (K / 4) * 16;
        ring = ures + round16(nch * K * 32 * 2);
        lq = ring + warps * QCAP * 8;
        pat = ring;
        const uint32_t ring_end = lq + warps * LCAP * 4, pat_end = pat + nb * PATW * 4;
        cbits = round16(ring_end > pat_end ? ring_end : pat_end);
        cnt = cbits + nch * CBW * 4;
        fam = cnt + round16(tmax * (ng + 2) * 4);
        seg = fam + round16(sizeof(FamDev));
        misc = seg + round16(sizeof(SegDev));
        total = misc + 32;   // deep counter (4 B), the item grab (8 B at +8), the item's first subtile and
                             // its segment's subtile end (8 B each at +16 and +24)
    }
};

__device__ __forceinline__ uint32_t unit_mask(int32_t lo, int32_t hi) {   // bits [lo, hi) of one 32-bit word
    return low_bits((uint32_t)min(max(hi, 0), 32)) & ~low_bits((uint32_t)min(max(lo, 0), 32));
}

__device__ __forceinline__ uint4 lds128(uint32_t addr) {      // 16-byte shared-memory load
    uint4 v;
    asm volatile("ld.shared.v4.u32 {%0, %1, %2, %3}, [%4];" : "=r"(v.x), "=r"(v.y), "=r"(v.z), "=r"(v.w) : "r"(addr));
    return v;
}

// The unit loop of one (v row, block) piece, from the shared address of each filter's row: AND of
// the NB rows per 16-byte unit, range masks unless the row covers the whole block (FULL), the
// group-1 popcount (first four filters) and, when group 2 ends at the last bitset filter (C2), the
// group-2 popcount.  Returns the mask of units that keep a bit after every bitset filter; save
// receives the bits of the last of them.
template <int NB, int U, bool FULL, bool C2>
__device__ __forceinline__ uint32_t piece_units(const uint32_t (&rb)[NB], uint32_t lane, int32_t s, int32_t e,
                                                uint32_t (&c)[2], uint4 &save) {
    uint32_t pend = 0;
#pragma unroll
    for (uint32_t p = 0; p < U; ++p) {
        const uint32_t u = (lane + p) & (U - 1), uo = u * 16;
        uint4 acc = lds128(rb[0] + uo);
        uint4 acc4;
#pragma unroll
        for (int f = 1; f < NB; ++f) {
            if (f == 4) acc4 = acc;
            const uint4 w = lds128(rb[f] + uo);
            acc.x &= w.x;
            acc.y &= w.y;
            acc.z &= w.z;
            acc.w &= w.w;
        }
        if (NB <= 4) acc4 = acc;
        if (!FULL) {
            const int32_t lo = s - (int32_t)u * 128, hi = e - (int32_t)u * 128;
            const uint32_t m0 = unit_mask(lo, hi), m1 = unit_mask(lo - 32, hi - 32);
            const uint32_t m2 = unit_mask(lo - 64, hi - 64), m3 = unit_mask(lo - 96, hi - 96);
            acc.x &= m0, acc.y &= m1, acc.z &= m2, acc.w &= m3;
            acc4.x &= m0, acc4.y &= m1, acc4.z &= m2, acc4.w &= m3;
        }
        c[0] += __popc(acc4.x) + __popc(acc4.y) + __popc(acc4.z) + __popc(acc4.w);
        if (C2) c[1] += __popc(acc.x) + __popc(acc.y) + __popc(acc.z) + __popc(acc.w);
        const bool live = (acc.x | acc.y | acc.z | acc.w) != 0;
        if (live) save = acc;                         // the last marked unit is not read again
        pend |= (uint32_t)live << p;
    }
    return pend;
}

__device__ __forceinline__ void copy_words(void *dst, const void *src, uint32_t bytes) {
    for (uint32_t i = threadIdx.x; i < bytes / 4; i += blockDim.x) ((uint32_t *)dst)[i] = ((const uint32_t *)src)[i];
}

// One lane owns one (v row, u block) piece: it walks the block's K/4 16-byte units in the order
// (lane + p) mod (K/4), so at every step the 32 lanes of a warp hit each 16-byte bank group
// exactly 32/(K/4) times whatever rows they read.  The group-1 and group-2 counters live in
// registers (c[0..1]) and are reduced per subtile when a lane's subtile changes.  The unit loop
// only marks the units that keep a bit after every bitset filter (and keeps the bits of the last
// one in registers); once the piece is done, each lane queues that unit's bits and puts its other
// marked units on a per-warp leftover list, recomputed 32 at a time, so the warp votes and
// diverges once per piece instead of after every unit, and never waits on a few lanes' units.
template <int NB, int K, int NT>
__global__ void __launch_bounds__(NT, 1) k_match(const MatchArgs a) {
    using G = Geo<K>;
    constexpr uint32_t U = G::U;
    extern __shared__ uint4 smem[];
    const uint32_t lane = threadIdx.x & 31, warp = threadIdx.x >> 5, nwarps = blockDim.x >> 5;
    const uint32_t ngmax = a.stride - 3;
    const MatchSmem L(a.total_rows, K, NB, a.nch, a.tmax, ngmax, nwarps);
    char *base = (char *)smem;
    const uint4 *rows = (const uint4 *)(base + L.rows);
    const uint32_t rows_addr = (uint32_t)__cvta_generic_to_shared(rows);
    uint16_t *ures = (uint16_t *)(base + L.ures);
    uint2 *qv = (uint2 *)(base + L.ring) + warp * QCAP;
    uint32_t *lq = (uint32_t *)(base + L.lq) + warp * LCAP;
    uint32_t *pat_s = (uint32_t *)(base + L.pat);
    uint32_t *cbits = (uint32_t *)(base + L.cbits);
    uint32_t *cnt_s = (uint32_t *)(base + L.cnt);      // tmax x (ngmax+2): groups 1..ng
    FamDev &F = *(FamDev *)(base + L.fam);
    SegDev &S = *(SegDev *)(base + L.seg);
    uint32_t *deep_ctr = (uint32_t *)(base + L.misc);
    volatile uint64_t *item_s = (volatile uint64_t *)(base + L.misc + 16);
    const uint32_t cstride = ngmax + 2;

    const uint32_t lanes_below = (1u << lane) - 1u;
    if (threadIdx.x == 0) *deep_ctr = 0;
    uint4 *deep_slice = a.deep + (size_t)blockIdx.x * a.deep_cap;

    const uint64_t n_items = a.item_prefix[a.nblocks];
    const uint64_t vch = *a.vchunk;
    uint64_t cur = UINT64_MAX, bsearch = 0;
    uint32_t cur_seg = UINT32_MAX, cur_fam = UINT32_MAX;
    const uint32_t nch = a.nch;
    unsigned long long *grab_s = (unsigned long long *)(base + L.misc + 8);

    // Items are handed out in ascending order from one device counter, so the CTAs work on
    // neighbouring blocks together: the per-v records of those blocks stay in L2, and the CTAs
    // finish within one grab of each other.  A grab takes as many items as a block averages (at
    // least ITEM_GRAB), so a block cut into several items is mostly built by one CTA once, but
    // never more than a quarter of an even share, so every CTA gets work.  A launch of fewer than
    // eight items per CTA (one batch) gives each CTA one even share of consecutive items, which
    // mostly lie in one block, so the rows of a block are built about once per CTA that meets it.
    const uint64_t ncta = gridDim.x;
    const uint64_t grab = n_items >= 8 * ncta
                              ? umax64(ITEM_GRAB, umin64(n_items / umax64(1, a.nblocks), n_items / (4 * ncta)))
                              : umax64(1, (n_items + ncta - 1) / ncta);
    uint64_t it = 0, it_end = 0;
    for (;;) {
        if (it == it_end) {
            __syncthreads();                              // every thread has read the previous grab
            if (threadIdx.x == 0) *grab_s = atomicAdd(a.item_next, (unsigned long long)grab);
            __syncthreads();
            it = *grab_s;
            if (it >= n_items) break;
            it_end = umin64(it + grab, n_items);
            uint64_t lo = 0, hi = a.nblocks;              // block of item it: last b with prefix[b] <= it
            while (hi - lo > 1) {
                const uint64_t mid = (lo + hi) / 2;
                if (a.item_prefix[mid] <= it) lo = mid;
                else hi = mid;
            }
            bsearch = lo;
        }
        while (a.item_prefix[bsearch + 1] <= it) ++bsearch;  // items of one grab are consecutive
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
            const uint32_t sg = a.blk_seg[b];
            if (sg != cur_seg) {
                const uint32_t fm = a.seg[sg].fam;
                copy_words(&S, a.seg + sg, sizeof(SegDev));
                if (fm != cur_fam) copy_words(&F, a.fam + fm, sizeof(FamDev));
                __syncthreads();
                if (fm != cur_fam) {
                    for (uint32_t i = threadIdx.x; i < nch * CBW; i += blockDim.x) {
                        const uint32_t t = i / CBW, w = i % CBW;
                        cbits[i] = w * 32 < F.cq[t] ? F.bits[F.cbits_off[t] + w] : 0u;
                    }
                }
                cur_seg = sg;
                cur_fam = fm;
            }
            for (uint32_t i = threadIdx.x; i < NB * PATW; i += blockDim.x) pat_s[i] = F.pat[i];
            __syncthreads();
            const uint32_t u_end = S.u_off + S.nu;
            const uint32_t n_valid = u_end > block_u0 ? min(u_end - block_u0, (uint32_t)G::UB) : 0u;
            build_rows<NB, K>(a.us, F, nch, (uint4 *)rows, ures, pat_s, block_u0, n_valid, lane, warp, nwarps);
            cur = b;
        }
        for (uint32_t k = threadIdx.x; k < a.tmax * cstride; k += blockDim.x) cnt_s[k] = 0;
        if (threadIdx.x == 0) {                           // the item's first subtile, once per CTA
            item_s[0] = S.tile_base + local_tile(a.rec[va].v, S.v_first, S.width, S.ntiles);
            item_s[1] = (uint64_t)S.tile_base + S.ntiles;
        }
        __syncthreads();
        // subtile geometry of the segment and of the item stays in shared memory (S, item_s): it is
        // read when a lane's subtile changes, once per round for the survivor slots, and when a
        // queued survivor needs its subtile, so no register holds it through the unit loop
        const bool c2_live = F.c2_live != 0;
        volatile uint64_t &tile_base = item_s[0], &seg_tiles_end = item_s[1];

        uint32_t c[2] = {0, 0};                           // group 1 and (C2) group 2 survivors of the lane
        // this lane's subtile as a slot from the item's first one (NO_SLOT: none), and the end of its
        // v range (a lane's rows rise in v within an item)
        constexpr uint32_t NO_SLOT = 0xFFFFFFFFu;
        uint32_t cslot = NO_SLOT;
        uint64_t t_hi = 0;

        auto flush = [&]() {                              // populations reduced over lanes of a subtile
            const uint32_t key = (c[0] | c[1]) ? cslot : NO_SLOT - 1 - lane;
            const uint32_t same = __match_any_sync(0xffffffffu, key);
            const uint32_t leader = __ffs(same) - 1;
#pragma unroll
            for (int g = 0; g < 2; ++g) {
                const uint32_t sum = __reduce_add_sync(same, c[g]);
                if (key == cslot && lane == leader && sum) {
                    if (cslot < a.tmax) atomicAdd(cnt_s + cslot * cstride + 1 + g, sum);
                    else {
                        const uint64_t tile = tile_base + cslot;
                        if (tile < seg_tiles_end)
                            atomicAdd((unsigned long long *)&a.counts[tile * a.stride + 1 + g], (unsigned long long)sum);
                    }
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
            uint32_t ent = 0, slot = 0;
            if (mine) {
                const uint2 q = qv[(qhead + lane) & (QCAP - 1)];
                ent = q.x, slot = q.y;
            }
            __syncwarp();
            qhead += n;
            if (!mine) return;
            const uint64_t tile = tile_base + slot;
            if (tile >= seg_tiles_end) return;            // v outside the subtile geometry (reported by k_vprep)
            const uint32_t uidx = ent >> 20;
            const uint64_t cr = __ldcg(a.cres + va + (ent & 0xFFFFFu));
            for (uint32_t t = 0; t < nch; ++t) {
                const uint32_t vr = (uint32_t)(cr >> (16 * t)) & 0xFFFFu, qg = F.cqg[t];
                int32_t m = (int32_t)ures[t * G::UB + uidx] - (int32_t)vr;
                if (m < 0) m += (int32_t)(qg & 0xFFFFu);
                if (!((cbits[t * CBW + (m >> 5)] >> (m & 31)) & 1u)) return;
                const uint32_t g = qg >> 16;
                if (g) {
                    if (slot < a.tmax) atomicAdd(cnt_s + slot * cstride + g, 1u);
                    else atomicAdd((unsigned long long *)&a.counts[tile * a.stride + g], 1ull);
                }
            }
            const uint32_t at = atomicAdd(deep_ctr, 1u);
            if (at < a.deep_cap) {
                const uint64_t v = a.rec[va + (ent & 0xFFFFFu)].v;
                deep_slice[at] = make_uint4((uint32_t)v, (uint32_t)(v >> 32), block_u0 + uidx, (uint32_t)tile);
            }
        };

        // The bits of one unit per lane go to the ring, one bit per lane per step (warp-uniform call).
        auto queue_bits = [&](uint4 acc, uint32_t u, uint32_t rel, uint32_t slot) {
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
                    qv[at] = make_uint2(rel | ((u * 128 + bit) << 20), slot);
                }
                qtail += __popc(bal);
                if (qtail - qhead >= 32) drain(32);
            }
        };

        uint32_t nl = 0;                                  // warp-uniform leftover count
        // Up to 32 leftover units, one per lane: recomputed from the record, bits queued.
        auto leftovers = [&]() {
            __syncwarp();
            const bool mine = lane < nl;
            const uint32_t ent = mine ? lq[lane] : 0u;
            __syncwarp();
            nl = 0;
            uint4 acc = make_uint4(0, 0, 0, 0);
            const uint32_t rel = ent & 0xFFFFFu, u = (ent >> 20) & 0xFu;
            uint32_t slot = ent >> 24;
            if (mine) {
                VRec rr;                                  // from L2, like the round's record
                const uint4 *src = (const uint4 *)(a.rec + va + rel);
                const uint4 h0 = __ldcg(src), h1 = __ldcg(src + 1);
                memcpy(&rr, &h0, 16);
                memcpy((char *)&rr + 16, &h1, 16);
                if (slot == 255u) {
                    const uint64_t lt = local_tile(rr.v, S.v_first, S.width, S.ntiles);
                    slot = lt < S.ntiles ? (uint32_t)(S.tile_base + lt - tile_base) : NO_SLOT;
                }
                acc = lds128(rows_addr + ((uint32_t)rr.row[0] * U + u) * 16);
#pragma unroll
                for (int f = 1; f < NB; ++f) {
                    const uint4 w = lds128(rows_addr + ((uint32_t)rr.row[f] * U + u) * 16);
                    acc.x &= w.x;
                    acc.y &= w.y;
                    acc.z &= w.z;
                    acc.w &= w.w;
                }
                const int32_t s = max((int32_t)(rr.left - block_u0), 0);
                const int32_t e = max(min((int32_t)(rr.right - block_u0), (int32_t)G::UB), s);
                const int32_t lo = s - (int32_t)u * 128, hi = e - (int32_t)u * 128;
                acc.x &= unit_mask(lo, hi), acc.y &= unit_mask(lo - 32, hi - 32);
                acc.z &= unit_mask(lo - 64, hi - 64), acc.w &= unit_mask(lo - 96, hi - 96);
            }
            queue_bits(acc, u, rel, slot);
        };

        // a warp takes consecutive rounds, so its lanes stay in one subtile for many rounds
        const uint32_t nrounds = (nv_item + 31) / 32, per_warp = (nrounds + nwarps - 1) / nwarps;
        const uint32_t r_end = min(nrounds, (warp + 1) * per_warp);
        for (uint32_t r = warp * per_warp; r < r_end; ++r) {
            const uint32_t rel = r * 32 + lane;
            const bool active = rel < nv_item;
            VRec rec{};
            if (active) {                                 // read once per block: cached in L2 only
                const uint4 *src = (const uint4 *)(a.rec + va + rel);
                const uint4 h0 = __ldcg(src), h1 = __ldcg(src + 1);
                memcpy(&rec, &h0, 16);
                memcpy((char *)&rec + 16, &h1, 16);
            }
            // warp-uniform: all 32 rows exist and cover the whole block
            const bool full = r * 32 >= full_lo && r * 32 + 32 <= full_hi;
            // piece as bits of the block, needed only where a row of the round covers part of it
            // (an inactive lane's zeroed record gives an empty piece)
            int32_t s = 0, e = (int32_t)G::UB;
            if (!full) {
                s = active ? max((int32_t)(rec.left - block_u0), 0) : 0;
                e = max(min((int32_t)(rec.right - block_u0), (int32_t)G::UB), s);
            }
            const bool moved = active && rec.v >= t_hi;
            if (__any_sync(0xffffffffu, moved)) {
                flush();
                if (moved) {
                    const uint64_t swidth = S.width;
                    if (cslot != NO_SLOT && rec.v - t_hi < 2 * swidth) {
                        // the next subtile or the one after it (the common step between rounds)
                        const bool two = rec.v - t_hi >= swidth;
                        cslot += two ? 2 : 1;
                        t_hi += two ? 2 * swidth : swidth;
                        if ((uint64_t)(tile_base + cslot) >= seg_tiles_end) cslot = NO_SLOT, t_hi = 0;
                    } else {
                        const uint64_t stn = S.ntiles;
                        const uint64_t lt = local_tile(rec.v, S.v_first, swidth, stn);
                        // slots fit 32 bits (an item's v rows lie in fewer than 2^31 subtiles)
                        cslot = lt < stn ? (uint32_t)(S.tile_base + lt - tile_base) : NO_SLOT;
                        const uint64_t t_lo = S.v_first + lt * swidth;
                        t_hi = lt < stn ? t_lo + swidth : t_lo;
                    }
                }
            }
            uint32_t rb[NB];                              // shared address of each filter's row
#pragma unroll
            for (int f = 0; f < NB; ++f) rb[f] = rows_addr + (uint32_t)rec.row[f] * (U * 16);   // row 0 if inactive

            // warp-uniform FULL and block-uniform C2 select the loop body, so the range masks and the
            // group-2 popcounts are not issued (as predicated code) where they cannot apply
            uint32_t pend;                                // units of this piece with survivors
            uint4 save;                                   // bits of the last one
            if (full)
                pend = c2_live ? piece_units<NB, U, true, true>(rb, lane, s, e, c, save)
                               : piece_units<NB, U, true, false>(rb, lane, s, e, c, save);
            else
                pend = c2_live ? piece_units<NB, U, false, true>(rb, lane, s, e, c, save)
                               : piece_units<NB, U, false, false>(rb, lane, s, e, c, save);
            // the last marked unit (its bits kept in registers) is queued now; the piece's other
            // marked units go to the leftover list
            uint4 acc = make_uint4(0, 0, 0, 0);
            uint32_t u = 0;
            if (pend) {
                const uint32_t pl = 31 - __clz(pend);
                u = (lane + pl) & (U - 1);
                acc = save;
                pend &= ~(1u << pl);
            }
            queue_bits(acc, u, rel, cslot);
            while (__any_sync(0xffffffffu, pend != 0)) {
                const bool has = pend != 0;
                const uint32_t bal = __ballot_sync(0xffffffffu, has);
                if (nl + __popc(bal) > LCAP) leftovers();
                if (has) {
                    lq[nl + __popc(bal & lanes_below)] =
                        rel | (((lane + __ffs(pend) - 1) & (U - 1)) << 20) | (min(cslot, 255u) << 24);
                    pend &= pend - 1;
                }
                nl += __popc(bal);
            }
        }
        if (nl) leftovers();
        if (qtail != qhead) drain(qtail - qhead);
        flush();
        __syncthreads();
        for (uint32_t k = threadIdx.x; k < a.tmax * cstride; k += blockDim.x) {
            const uint32_t cv = cnt_s[k];
            if (cv) {
                const uint32_t slot = k / cstride, g = k % cstride;
                const uint64_t tile = tile_base + slot;
                if (tile < seg_tiles_end)
                    atomicAdd((unsigned long long *)&a.counts[tile * a.stride + g], (unsigned long long)cv);
            }
        }
        ++it;
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
// of the record's family with group counters, then the output record.  One record per thread;
// outputs are appended with one atomic per warp.
__global__ void __launch_bounds__(256) k_deep(const DeepArgs a) {
    const uint32_t lane = threadIdx.x & 31;
    const uint32_t lanes_below = (1u << lane) - 1u;
    const uint32_t slice = blockIdx.y;
    const uint32_t count = min(a.deep_count[slice], a.deep_cap);
    for (uint32_t base = blockIdx.x * blockDim.x; base < count; base += gridDim.x * blockDim.x) {
        const uint32_t at = base + threadIdx.x;
        const uint64_t i = (uint64_t)slice * a.deep_cap + at;
        bool pass = false;
        u128 x{0, 0};
        uint64_t tile = 0;
        uint32_t ng = 0;
        if (at < count) {
            const uint4 r = a.deep[i];
            const uint64_t v = (uint64_t)r.y << 32 | r.x;
            tile = r.w;
            if (tile < a.ntiles) {
                const SegDev &g = a.seg[a.tile_seg[tile]];
                const FamDev &F = a.fam[g.fam];
                ng = F.ng;
                const u128 pos = mul_wide(__ldg(a.us + r.z), g.B), shift = mul_wide(v, g.A);
                if (less128(pos, shift)) {
                    atomicAdd((unsigned long long *)&a.counts[tile * a.stride + ng + 2], 1ull);
                } else {
                    x = sub128(pos, shift);
                    const uint32_t h[6] = {(uint32_t)x.lo & 0xffffu, (uint32_t)(x.lo >> 16) & 0xffffu,
                                           (uint32_t)(x.lo >> 32) & 0xffffu, (uint32_t)(x.lo >> 48),
                                           (uint32_t)x.hi & 0xffffu, (uint32_t)(x.hi >> 16) & 0xffffu};
                    pass = true;
                    const uint32_t nres = F.nres;
                    const FiltC *fcs = F.fcs;
                    const uint32_t *bits = F.bits;
                    for (uint32_t idx = a.first; idx < nres; ++idx) {
                        const FiltC f = fcs[idx];
                        const uint32_t m = mod_limbs(h, f);
                        if (!((__ldg(bits + f.tab_off + (m >> 5)) >> (m & 31)) & 1u)) {
                            pass = false;
                            break;
                        }
                        if ((idx & 3) == 3 || idx + 1 == nres)
                            atomicAdd((unsigned long long *)&a.counts[tile * a.stride + idx / 4 + 1], 1ull);
                    }
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
                    atomicAdd((unsigned long long *)&a.counts[tile * a.stride + ng + 1], (unsigned long long)__popc(same));
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
int launch_match_t(pc_ctx *ctx, const MatchArgs &a, size_t smem, int grid, int mode) {
    auto kern = k_match<NB, K, NT>;
    if (mode != 1) {       // 0: attribute and launch, 1: launch only (inside a capture), 2: attribute only
        cudaError_t e = cudaFuncSetAttribute(kern, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem);
        if (e != cudaSuccess) return pc_cuda_fail(ctx, e, "match smem attribute");
        if (mode == 2) return PC_OK;
    }
    kern<<<grid, NT, smem, ctx->stream>>>(a);
    PC_LAUNCHED(ctx, "match");
    return PC_OK;
}

template <int K, int NT>
int launch_match_k(pc_ctx *ctx, const MatchArgs &a, uint32_t nb, size_t smem, int grid, int mode) {
    switch (nb) {
        case 1: return launch_match_t<1, K, NT>(ctx, a, smem, grid, mode);
        case 2: return launch_match_t<2, K, NT>(ctx, a, smem, grid, mode);
        case 3: return launch_match_t<3, K, NT>(ctx, a, smem, grid, mode);
        case 4: return launch_match_t<4, K, NT>(ctx, a, smem, grid, mode);
        case 5: return launch_match_t<5, K, NT>(ctx, a, smem, grid, mode);
        case 6: return launch_match_t<6, K, NT>(ctx, a, smem, grid, mode);
        case 7: return launch_match_t<7, K, NT>(ctx, a, smem, grid, mode);
        case 8: return launch_match_t<8, K, NT>(ctx, a, smem, grid, mode);
    }
    return pc_fail(ctx, PC_INVALID, "unsupported bitset filter count");
}

template <int NT>
int launch_match_n(pc_ctx *ctx, const MatchArgs &a, uint32_t nb, uint32_t K, size_t smem, int grid, int mode) {
    if (K == 16) return launch_match_k<16, NT>(ctx, a, nb, smem, grid, mode);
    if (K == 32) return launch_match_k<32, NT>(ctx, a, nb, smem, grid, mode);
    return launch_match_k<64, NT>(ctx, a, nb, smem, grid, mode);
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
    f->fcs_bytes = nres * sizeof(FiltC);
    f->bits_bytes = bits.size() * 4;
    f->pat_bytes = pat.size() * 4;
    int rc = pc_alloc(ctx, (void **)&f->d_fc, f->fc_bytes);
    if (!rc) rc = pc_alloc(ctx, (void **)&f->d_fcs, f->fcs_bytes);
    if (!rc) rc = pc_alloc(ctx, (void **)&f->d_bits, f->bits_bytes);
    if (!rc) rc = pc_alloc(ctx, (void **)&f->d_pat, f->pat_bytes);
    if (rc) {
        pc_filters_free(ctx, f);
        return rc;
    }
    pc_copy(ctx, f->d_fc, fc.data(), f->fc_bytes, cudaMemcpyHostToDevice);
    pc_copy(ctx, f->d_fcs, f->fcs.data(), f->fcs_bytes, cudaMemcpyHostToDevice);
    pc_copy(ctx, f->d_bits, bits.data(), f->bits_bytes, cudaMemcpyHostToDevice);
    pc_copy(ctx, f->d_pat, pat.data(), f->pat_bytes, cudaMemcpyHostToDevice);
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
    pc_release(ctx, f->d_fcs, f->fcs_bytes);
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

// One launch shape for every family of a launch: NB inside every family's bitset range, the cheap
// tier as deep as the shallowest family allows, shared memory sized by the largest rows and
// counters.  Defaults: seven bitset filters, 32-word blocks, 896 threads, stepping down (threads,
// then block words, then bitset filters) until the layout fits the opt-in shared memory.
int resolve_tuning(pc_ctx *ctx, const std::vector<const pc_filters *> &fams, const pc_tuning *t, Tuned &r,
                   size_t &smem, uint32_t &tmax) {
    uint32_t nb_lo = 1, nb_hi = PC_MAX_BITSET, ngmax = 0;
    for (const pc_filters *f : fams) {
        nb_lo = std::max(nb_lo, std::min<uint32_t>(f->nres, 4));
        nb_hi = std::min(nb_hi, f->nbmax);
        ngmax = std::max(ngmax, f->ng);
    }
    if (nb_lo > nb_hi) return pc_fail(ctx, PC_INVALID, "filter families cannot share one bitset launch");
    r = Tuned{};
    r.nb = t && t->bitset_filters ? t->bitset_filters : std::min<uint32_t>(nb_hi, 7);
    r.nb = std::max(nb_lo, std::min(r.nb, nb_hi));
    r.K = t && t->block_words ? t->block_words : 32;
    if (r.K != 16 && r.K != 32 && r.K != 64) r.K = 32;
    const bool fixed_threads = t && t->threads;
    r.threads = fixed_threads ? t->threads : 896;
    if (r.threads != 512 && r.threads != 768 && r.threads != 896 && r.threads != 1024) r.threads = 512;
    r.v_chunk = t ? t->v_chunk : 0;
    int optin = 0;
    cudaDeviceGetAttribute(&optin, cudaDevAttrMaxSharedMemoryPerBlockOptin, ctx->device);
    if (optin <= 0) optin = 227 * 1024;
    for (;;) {
        r.nch = PC_MAX_CHEAP;
        uint32_t rows = 0;
        for (const pc_filters *f : fams) {
            r.nch = std::min(r.nch, cheap_count(f, r.nb));
            rows = std::max(rows, f->rows_sum[r.nb]);
        }
        for (uint32_t tm = TMAX_DEFAULT; tm >= 4; tm /= 2) {
            MatchSmem L(rows, r.K, r.nb, r.nch, tm, ngmax, r.threads / 32);
            if (L.total <= (uint32_t)optin) {
                tmax = tm;
                smem = L.total;
                return PC_OK;
            }
        }
        if (!fixed_threads && r.threads > 512) r.threads = r.threads > 896 ? 896 : r.threads == 896 ? 768 : 512;
        else if (r.K > 16) r.K /= 2;
        else if (r.nb > nb_lo) r.nb--;
        else return pc_fail(ctx, PC_INVALID, "residual rows do not fit shared memory");
    }
}

FamDev fam_dev(const pc_filters *f, uint32_t nb, uint32_t nch) {
    FamDev d{};
    d.nres = f->nres;
    d.ng = f->ng;
    d.total_rows = f->rows_sum[nb];
    d.c2_live = nb == 8 || (nb > 4 && nb == f->nres);
    for (uint32_t i = 0; i < nb; ++i) {
        d.q[i] = f->primes[i];
        d.row0[i] = f->rows_sum[i];
        d.ainvb[i] = f->ainvb[i];
        d.mq[i] = make_modq(f->primes[i]);
    }
    for (uint32_t t = 0; t < nch; ++t) {
        const uint32_t q = f->primes[nb + t];
        d.cq[t] = q;
        d.caq[t] = (uint32_t)(f->A % q);
        d.cbq[t] = (uint32_t)(f->B % q);
        d.cmq[t] = make_modq(q);
        d.cbits_off[t] = f->fcs[nb + t].tab_off;
    }
    for (uint32_t idx = 0; idx < 16; ++idx)
        d.bgroup[idx] = (uint8_t)(idx < f->nres && ((idx & 3) == 3 || idx + 1 == f->nres) ? idx / 4 + 1 : 0);
    for (uint32_t t = 0; t < nch; ++t) d.cqg[t] = d.cq[t] | (uint32_t)d.bgroup[nb + t] << 16;
    d.pat = f->d_pat;
    d.bits = f->d_bits;
    d.fcs = f->d_fcs;
    return d;
}

// The device half of stages 2 and 3 over a set of segments whose u and v lists are already on
// the device.  Every buffer is sized once by engine_prepare, so the launch sequence (front + back)
// can be recorded into a CUDA graph and replayed.
struct Engine {
    pc_ctx *ctx = nullptr;
    const uint64_t *us = nullptr, *vs = nullptr;
    uint64_t nu = 0, nv = 0;
    std::vector<SegDev> segs;
    std::vector<const pc_filters *> fams;
    std::vector<FamDev> famdev;
    std::vector<uint32_t> tile_seg;
    uint64_t ntiles = 0, out_cap = 0;
    Tuned tn{};
    size_t smem = 0;
    uint32_t tmax = 0, stride = 0, ngmax = 0;
    uint64_t nblocks = 0;
    int grid = 0;
    uint32_t deep_cap = 1u << 15, deep_max = 0;
    SegDev *d_seg = nullptr;
    FamDev *d_fam = nullptr;
    uint32_t *d_tile_seg = nullptr, *d_blk_seg = nullptr, *d_deep_count = nullptr;
    unsigned long long *d_item_next = nullptr;
    uint64_t *d_counts = nullptr, *d_geo = nullptr, *d_out = nullptr;
    unsigned long long *d_nout = nullptr;                 // [0] outputs, [1] rows outside the geometry
    VRec *d_rec = nullptr;
    uint64_t *d_cres = nullptr;
    uint4 *d_bv = nullptr;
    uint64_t *d_pieces = nullptr, *d_tmp = nullptr, *d_items = nullptr, *d_prefix = nullptr, *d_vchunk = nullptr;
    uint64_t *d_ws = nullptr;
    uint4 *d_deep = nullptr;
    uint64_t deep_bytes = 0;
    ~Engine() {
        if (ctx && d_deep) pc_release(ctx, d_deep, deep_bytes);
    }
};

int engine_deep_alloc(Engine &E, uint32_t cap) {
    if (E.d_deep) pc_release(E.ctx, E.d_deep, E.deep_bytes);
    E.d_deep = nullptr;
    E.deep_cap = cap;
    E.deep_bytes = (uint64_t)E.grid * cap * sizeof(uint4);
    return pc_alloc(E.ctx, (void **)&E.d_deep, E.deep_bytes);
}

int engine_prepare(Engine &E, const pc_tuning *tuning, Scratch &hold) {
    pc_ctx *ctx = E.ctx;
    if (E.nu >= (UINT64_C(1) << 31) || E.nv >= (UINT64_C(1) << 32)) return pc_fail(ctx, PC_INVALID, "focus list too long");
    if (E.segs.empty() || E.fams.empty()) return pc_fail(ctx, PC_INVALID, "no segments");
    for (const SegDev &g : E.segs)
        if (g.hi.hi >= (UINT64_C(1) << 32)) return pc_fail(ctx, PC_INVALID, "interval bound must be below 2^96");
    int rc = resolve_tuning(ctx, E.fams, tuning, E.tn, E.smem, E.tmax);
    if (rc) return rc;
    E.ngmax = 0;
    for (const pc_filters *f : E.fams) E.ngmax = std::max(E.ngmax, f->ng);
    E.stride = E.ngmax + 3;
    E.famdev.clear();
    for (const pc_filters *f : E.fams) E.famdev.push_back(fam_dev(f, E.tn.nb, E.tn.nch));
    E.grid = ctx->sm_count;
    if (tuning && tuning->deep_records) E.deep_cap = tuning->deep_records;
    const uint32_t UB = E.tn.K * 32;
    E.nblocks = (E.nu + UB - 1) / UB;
    const uint64_t nb1 = std::max<uint64_t>(1, E.nblocks);
    rc = hold.get(&E.d_seg, E.segs.size());
    if (!rc) rc = hold.get(&E.d_fam, E.famdev.size());
    if (!rc) rc = hold.get(&E.d_tile_seg, std::max<uint64_t>(1, E.ntiles));
    if (!rc) rc = hold.get(&E.d_counts, std::max<uint64_t>(1, E.ntiles * E.stride));
    if (!rc) rc = hold.get(&E.d_geo, std::max<uint64_t>(1, 2 * E.ntiles));
    if (!rc) rc = hold.get(&E.d_out, 2 * std::max<uint64_t>(1, E.out_cap));
    if (!rc) rc = hold.get(&E.d_nout, 2);
    if (!rc) rc = hold.get(&E.d_rec, std::max<uint64_t>(1, E.nv));
    if (!rc) rc = hold.get(&E.d_cres, std::max<uint64_t>(1, E.nv));
    if (!rc) rc = hold.get(&E.d_bv, nb1);
    if (!rc) rc = hold.get(&E.d_blk_seg, nb1);
    if (!rc) rc = hold.get(&E.d_pieces, nb1);
    if (!rc) rc = hold.get(&E.d_tmp, E.nblocks + 1);
    if (!rc) rc = hold.get(&E.d_items, nb1);
    if (!rc) rc = hold.get(&E.d_prefix, E.nblocks + 1);
    if (!rc) rc = hold.get(&E.d_vchunk, 1);
    if (!rc) rc = hold.get(&E.d_ws, pc_scan_workspace(E.nblocks));
    if (!rc) rc = hold.get(&E.d_deep_count, E.grid);
    if (!rc) rc = hold.get(&E.d_item_next, 1);
    if (!rc) rc = engine_deep_alloc(E, E.deep_cap);
    if (rc) return rc;
    PC_CHECK(ctx, pc_copy(ctx, E.d_seg, E.segs.data(), E.segs.size() * sizeof(SegDev), cudaMemcpyHostToDevice));
    PC_CHECK(ctx, pc_copy(ctx, E.d_fam, E.famdev.data(), E.famdev.size() * sizeof(FamDev), cudaMemcpyHostToDevice));
    if (E.ntiles)
        PC_CHECK(ctx, pc_copy(ctx, E.d_tile_seg, E.tile_seg.data(), E.ntiles * 4, cudaMemcpyHostToDevice));
    return PC_OK;
}

// mode 0: set the shared-memory attribute and launch; 1: launch only (inside a capture);
// 2: set the attribute only.
int engine_match(Engine &E, int mode) {
    MatchArgs ma{};
    ma.us = E.us;
    ma.rec = E.d_rec;
    ma.cres = E.d_cres;
    ma.seg = E.d_seg;
    ma.fam = E.d_fam;
    ma.blk_seg = E.d_blk_seg;
    ma.nch = E.tn.nch;
    ma.tmax = E.tmax;
    ma.stride = E.stride;
    ma.total_rows = 0;
    for (const FamDev &d : E.famdev) ma.total_rows = std::max(ma.total_rows, d.total_rows);
    ma.counts = E.d_counts;
    ma.bv = E.d_bv;
    ma.item_prefix = E.d_prefix;
    ma.nblocks = E.nblocks;
    ma.vchunk = E.d_vchunk;
    ma.deep = E.d_deep;
    ma.deep_cap = E.deep_cap;
    ma.deep_count = E.d_deep_count;
    ma.item_next = E.d_item_next;
    if (E.tn.threads == 1024) return launch_match_n<1024>(E.ctx, ma, E.tn.nb, E.tn.K, E.smem, E.grid, mode);
    if (E.tn.threads == 896) return launch_match_n<896>(E.ctx, ma, E.tn.nb, E.tn.K, E.smem, E.grid, mode);
    if (E.tn.threads == 768) return launch_match_n<768>(E.ctx, ma, E.tn.nb, E.tn.K, E.smem, E.grid, mode);
    return launch_match_n<512>(E.ctx, ma, E.tn.nb, E.tn.K, E.smem, E.grid, mode);
}

// Counters reset, per-v bounds, subtile envelopes, block ranges, work items and the fused match.
int engine_front(Engine &E, bool events, bool capturing, int *launches) {
    pc_ctx *ctx = E.ctx;
    cudaStream_t st = ctx->stream;
    if (E.ntiles) PC_CHECK(ctx, cudaMemsetAsync(E.d_counts, 0, E.ntiles * E.stride * 8, st));
    PC_CHECK(ctx, cudaMemsetAsync(E.d_nout, 0, 16, st));
    PC_CHECK(ctx, cudaMemsetAsync(E.d_deep_count, 0, (uint64_t)E.grid * 4, st));
    PC_CHECK(ctx, cudaMemsetAsync(E.d_item_next, 0, 8, st));
    if (events) PC_CHECK(ctx, cudaEventRecord(ctx->ev[0], st));
    if (E.nv) {
        PrepArgs pa{};
        pa.us = E.us;
        pa.vs = E.vs;
        pa.nv = E.nv;
        pa.seg = E.d_seg;
        pa.nseg = (uint32_t)E.segs.size();
        pa.fam = E.d_fam;
        pa.nb = E.tn.nb;
        pa.stride = E.stride;
        pa.rec = E.d_rec;
        pa.cres = E.d_cres;
        pa.nch = E.tn.nch;
        pa.counts = E.d_counts;
        pa.bad = E.d_nout + 1;
        const uint64_t runs = (E.nv + PREP_RUN - 1) / PREP_RUN;
        k_vprep<<<(unsigned)((runs + 127) / 128), 128, 0, st>>>(pa);
        PC_LAUNCHED(ctx, "vprep");
        ++*launches;
    }
    if (E.ntiles) {
        k_geometry<<<(unsigned)((E.ntiles + 127) / 128), 128, 0, st>>>(E.us, E.vs, E.d_seg, E.d_tile_seg, E.ntiles, E.d_geo);
        PC_LAUNCHED(ctx, "geometry");
        ++*launches;
    }
    if (events) PC_CHECK(ctx, cudaEventRecord(ctx->ev[1], st));
    if (!E.nu || !E.nv) return PC_OK;
    const uint32_t UB = E.tn.K * 32;
    k_blocks<<<(unsigned)((E.nblocks + 255) / 256), 256, 0, st>>>(E.d_rec, E.d_seg, (uint32_t)E.segs.size(), UB,
                                                                 E.nblocks, E.d_bv, E.d_blk_seg, E.d_pieces);
    PC_LAUNCHED(ctx, "blocks");
    int rc = pc_exclusive_scan_ws(ctx, E.d_pieces, E.d_tmp, E.nblocks, E.d_tmp + E.nblocks, E.d_ws);
    if (rc) return rc;
    k_chunk<<<1, 1, 0, st>>>(E.d_tmp + E.nblocks, E.tn.v_chunk, (uint64_t)E.grid * 32, 4 * (uint64_t)E.tn.threads,
                             E.d_vchunk);
    PC_LAUNCHED(ctx, "chunk");
    k_item_counts<<<(unsigned)((E.nblocks + 255) / 256), 256, 0, st>>>(E.d_pieces, E.nblocks, E.d_vchunk, E.d_items);
    PC_LAUNCHED(ctx, "item counts");
    rc = pc_exclusive_scan_ws(ctx, E.d_items, E.d_prefix, E.nblocks, E.d_prefix + E.nblocks, E.d_ws);
    if (rc) return rc;
    *launches += 7;
    if (events) PC_CHECK(ctx, cudaEventRecord(ctx->ev[2], st));
    rc = engine_match(E, capturing ? 1 : 0);
    if (rc) return rc;
    ++*launches;
    return PC_OK;
}

// The exact later filters on the deep survivors.
int engine_back(Engine &E, bool events, int *launches) {
    pc_ctx *ctx = E.ctx;
    if (E.nu && E.nv && E.deep_max) {
        DeepArgs da{};
        da.us = E.us;
        da.deep = E.d_deep;
        da.deep_count = E.d_deep_count;
        da.deep_cap = E.deep_cap;
        da.first = E.tn.nb + E.tn.nch;
        da.stride = E.stride;
        da.ntiles = E.ntiles;
        da.seg = E.d_seg;
        da.fam = E.d_fam;
        da.tile_seg = E.d_tile_seg;
        da.counts = E.d_counts;
        da.out = E.d_out;
        da.out_cap = E.out_cap;
        da.n_out = E.d_nout;
        dim3 dg((unsigned)std::min<uint64_t>((E.deep_max + 255) / 256, 64), (unsigned)E.grid);
        k_deep<<<dg, 256, 0, ctx->stream>>>(da);
        PC_LAUNCHED(ctx, "deep");
        ++*launches;
    }
    if (events) PC_CHECK(ctx, cudaEventRecord(ctx->ev[3], ctx->stream));
    return PC_OK;
}

// Eager run: the match, the deep-survivor counts on the host (a rerun with room for every deep
// survivor when a slice overflowed), then the deep tier.
int engine_eager(Engine &E, int *launches) {
    pc_ctx *ctx = E.ctx;
    for (int attempt = 0;; ++attempt) {
        int rc = engine_front(E, true, false, launches);
        if (rc) return rc;
        E.deep_max = 0;
        if (E.nu && E.nv) {
            std::vector<uint32_t> deep_counts(E.grid);
            PC_CHECK(ctx, pc_copy(ctx, deep_counts.data(), E.d_deep_count, (uint64_t)E.grid * 4, cudaMemcpyDeviceToHost));
            PC_CHECK(ctx, cudaStreamSynchronize(ctx->stream));
            for (uint32_t c : deep_counts) E.deep_max = std::max(E.deep_max, c);
            if (E.deep_max > E.deep_cap) {
                if (attempt) return pc_fail(ctx, PC_ARITHMETIC, "deep survivor count changed between attempts");
                rc = engine_deep_alloc(E, E.deep_max + 1024);
                if (rc) return rc;
                continue;
            }
        }
        return engine_back(E, true, launches);
    }
}

// Results of a finished run already copied to the host: output count, rows outside the subtile
// geometry, and the underflow counters of every subtile.
int engine_check(Engine &E, const unsigned long long nout[2], const uint64_t *counts) {
    if (nout[1]) return pc_fail(E.ctx, PC_INVALID, "v row outside the subtile geometry");
    if (nout[0] > E.out_cap) return pc_fail(E.ctx, PC_OVERFLOW, "output overflow; attempt cannot commit");
    for (uint64_t t = 0; t < E.ntiles; ++t) {
        const uint32_t ng = E.fams[E.segs[E.tile_seg[t]].fam]->ng;
        if (counts[t * E.stride + ng + 2]) return pc_fail(E.ctx, PC_ARITHMETIC, "unsigned underflow flagged");
    }
    return PC_OK;
}

int engine_collect(Engine &E, uint64_t *counts, uint64_t *geometry, uint64_t *out, uint64_t *n_out) {
    pc_ctx *ctx = E.ctx;
    cudaStream_t st = ctx->stream;
    unsigned long long nout[2] = {0, 0};
    PC_CHECK(ctx, pc_copy(ctx, nout, E.d_nout, 16, cudaMemcpyDeviceToHost));
    if (E.ntiles) {
        PC_CHECK(ctx, pc_copy(ctx, counts, E.d_counts, E.ntiles * E.stride * 8, cudaMemcpyDeviceToHost));
        PC_CHECK(ctx, pc_copy(ctx, geometry, E.d_geo, 2 * E.ntiles * 8, cudaMemcpyDeviceToHost));
    }
    PC_CHECK(ctx, cudaStreamSynchronize(st));
    *n_out = nout[0];
    int rc = engine_check(E, nout, counts);
    if (rc) return rc;
    if (nout[0]) {
        PC_CHECK(ctx, pc_copy(ctx, out, E.d_out, 2 * nout[0] * 8, cudaMemcpyDeviceToHost));
        PC_CHECK(ctx, cudaStreamSynchronize(st));
    }
    return PC_OK;
}

void engine_stats(Engine &E, pc_stats *stats, int launches, uint64_t n_out) {
    if (!stats) return;
    pc_ctx *ctx = E.ctx;
    const bool matched = E.nu && E.nv;
    stats->bounds_ms = elapsed_ms(ctx->ev[0], ctx->ev[1]);
    stats->kernel_ms = matched ? elapsed_ms(ctx->ev[2], ctx->ev[3]) : 0.0;
    stats->outputs = n_out;
    stats->launches = launches;
    stats->work_items = E.deep_max;
    stats->reserved[0] = E.tn.nb;
    stats->reserved[1] = E.tn.K;
    stats->reserved[2] = E.tn.threads;
    stats->reserved[3] = E.tn.nch;
}

// True when ntiles subtiles of width v fit below 2^64 and match the [first, end) span.
bool tiles_fit(uint64_t first, uint64_t end, uint64_t width, uint64_t ntiles) {
    typedef unsigned __int128 w128;
    if (!width || end <= first) return false;
    if (((w128)ntiles * width) >> 64) return false;
    return (end - first + width - 1) / width == ntiles;
}

SegDev one_segment(const pc_filters *f, uint64_t nu, uint64_t nv, u128 lo, u128 hi, uint64_t v_first,
                   uint64_t width, uint64_t v_end, uint32_t ntiles) {
    SegDev g{};
    g.A = f->A;
    g.B = f->B;
    g.lo = lo;
    g.hi = hi;
    g.v_first = v_first;
    g.width = width;
    g.v_end = v_end;
    g.u_off = 0;
    g.nu = (uint32_t)nu;
    g.v_off = 0;
    g.nv = (uint32_t)nv;
    g.tile_base = 0;
    g.ntiles = ntiles;
    g.fam = 0;
    return g;
}

}  // namespace

extern "C" int pc_run_batch(pc_ctx *ctx, const pc_filters *f, const pc_tuning *tuning, const pc_buf *us, uint64_t u_off,
                            uint64_t nu, const pc_buf *vs, uint64_t v_off, uint64_t nv, uint64_t lo0, uint64_t lo1,
                            uint64_t hi0, uint64_t hi1, uint64_t v_first, uint64_t width, uint32_t ntiles,
                            uint64_t v_end, uint64_t *counts, uint64_t *geometry, uint64_t *out, uint64_t out_cap,
                            uint64_t *n_out, pc_stats *stats) {
    if (!f || !us || !vs || width == 0 || ntiles == 0) return pc_fail(ctx, PC_INVALID, "invalid batch arguments");
    if (u_off > us->n || nu > us->n - u_off || v_off > vs->n || nv > vs->n - v_off)
        return pc_fail(ctx, PC_INVALID, "focus list slice out of range");
    if (!tiles_fit(v_first, v_end, width, ntiles) || ntiles >= (UINT32_C(1) << 31))
        return pc_fail(ctx, PC_INVALID, "inconsistent subtile geometry");
    if (stats) memset(stats, 0, sizeof(*stats));
    *n_out = 0;
    auto t0 = std::chrono::steady_clock::now();
    const uint64_t h2d0 = ctx->h2d, d2h0 = ctx->d2h;
    Engine E;
    E.ctx = ctx;
    E.us = us->d + u_off;
    E.vs = vs->d + v_off;
    E.nu = nu;
    E.nv = nv;
    if (nu >= (UINT64_C(1) << 31) || nv >= (UINT64_C(1) << 32)) return pc_fail(ctx, PC_INVALID, "focus list too long");
    E.segs.push_back(one_segment(f, nu, nv, u128{lo0, lo1}, u128{hi0, hi1}, v_first, width, v_end, ntiles));
    E.fams.push_back(f);
    E.tile_seg.assign(ntiles, 0);
    E.ntiles = ntiles;
    E.out_cap = out_cap;
    Scratch hold(ctx);
    int launches = 0;
    int rc = engine_prepare(E, tuning, hold);
    if (!rc) rc = engine_eager(E, &launches);
    if (!rc) rc = engine_collect(E, counts, geometry, out, n_out);
    if (!rc || rc == PC_OVERFLOW || rc == PC_ARITHMETIC) engine_stats(E, stats, launches, *n_out);
    if (stats) {
        stats->total_ms = std::chrono::duration<double, std::milli>(std::chrono::steady_clock::now() - t0).count();
        stats->h2d_bytes = ctx->h2d - h2d0;
        stats->d2h_bytes = ctx->d2h - d2h0;
    }
    return rc;
}

extern "C" int pc_run_lease(pc_ctx *ctx, const pc_focus *fa, const pc_focus *fb, const pc_filters *f,
                            const pc_tuning *tuning, uint64_t first, uint64_t end, uint64_t width, uint64_t lo0,
                            uint64_t lo1, uint64_t hi0, uint64_t hi1, uint64_t *counts, uint64_t *geometry,
                            uint64_t *out, uint64_t out_cap, uint64_t *n_out, pc_stats *stats) {
    if (!fa || !fb || !f || width == 0 || end <= first) return pc_fail(ctx, PC_INVALID, "invalid lease arguments");
    if (stats) memset(stats, 0, sizeof(*stats));
    *n_out = 0;
    auto t0 = std::chrono::steady_clock::now();
    const uint64_t h2d0 = ctx->h2d, d2h0 = ctx->d2h;
    typedef unsigned __int128 w128;
    const w128 lo = (w128)lo1 << 64 | lo0, hi = (w128)hi1 << 64 | hi0;
    const w128 ulo = (lo + (w128)first * f->A) / f->B + 1, uhi = (hi + (w128)(end - 1) * f->A) / f->B + 1;
    if (uhi >> 64) return pc_fail(ctx, PC_INVALID, "u window exceeds 64 bits");
    const uint64_t ntiles64 = (end - first + width - 1) / width;
    if (ntiles64 >= (UINT64_C(1) << 31) || !tiles_fit(first, end, width, ntiles64))
        return pc_fail(ctx, PC_INVALID, "too many subtiles");
    int launches = 0;
    Scratch hold(ctx);
    PC_CHECK(ctx, cudaEventRecord(ctx->ev[4], ctx->stream));
    const pc_focus *foc[2] = {fa, fb};
    const uint64_t lows[2] = {(uint64_t)ulo, first}, highs[2] = {(uint64_t)uhi, end};
    WinBatch wb;
    int rc = winbatch_plan(ctx, hold, foc, lows, highs, nullptr, 2, (UINT64_C(1) << 32) - 1, wb, &launches);
    uint64_t *d_lists = nullptr;
    if (!rc) rc = hold.get(&d_lists, std::max<uint64_t>(1, wb.out_len));
    if (!rc) rc = winbatch_emit(ctx, wb, d_lists);
    if (rc) return rc;
    ++launches;
    PC_CHECK(ctx, cudaEventRecord(ctx->ev[5], ctx->stream));
    Engine E;
    E.ctx = ctx;
    E.us = d_lists + wb.base[0];
    E.nu = wb.total[0];
    E.vs = d_lists + wb.base[1];
    E.nv = wb.total[1];
    E.segs.push_back(one_segment(f, E.nu, E.nv, u128{lo0, lo1}, u128{hi0, hi1}, first, width, end, (uint32_t)ntiles64));
    E.fams.push_back(f);
    E.tile_seg.assign(ntiles64, 0);
    E.ntiles = ntiles64;
    E.out_cap = out_cap;
    rc = engine_prepare(E, tuning, hold);
    if (!rc) rc = engine_eager(E, &launches);
    if (!rc) rc = engine_collect(E, counts, geometry, out, n_out);
    if (!rc || rc == PC_OVERFLOW || rc == PC_ARITHMETIC) {
        engine_stats(E, stats, launches, *n_out);
        if (stats) stats->window_ms = elapsed_ms(ctx->ev[4], ctx->ev[5]);
    }
    if (stats) {
        stats->total_ms = std::chrono::duration<double, std::milli>(std::chrono::steady_clock::now() - t0).count();
        stats->h2d_bytes = ctx->h2d - h2d0;
        stats->d2h_bytes = ctx->d2h - d2h0;
    }
    return rc;
}

// Leases one after another on the calling thread, so a host runtime that holds a lock while it
// builds receipts (an interpreter) never sits between two device calls.  status[i] becomes
// 1 + the return code of lease i once its outputs are on the host (release order), so another
// thread can consume lease i while later leases run; the loop stops at the first failing lease.
extern "C" int pc_run_leases(pc_ctx *ctx, const pc_focus *fa, const pc_focus *fb, const pc_filters *f,
                             const pc_tuning *tuning, uint32_t n, const uint64_t *first, const uint64_t *end,
                             uint64_t width, uint64_t lo0, uint64_t lo1, uint64_t hi0, uint64_t hi1,
                             uint64_t *const *counts, uint64_t *const *geometry, uint64_t *const *out, uint64_t out_cap,
                             uint64_t *n_out, pc_stats *stats, int32_t *status) {
    if (!ctx || (n && (!first || !end || !counts || !geometry || !out || !n_out || !status)))
        return pc_fail(ctx, PC_INVALID, "invalid lease list");
    for (uint32_t i = 0; i < n; ++i) {
        const int rc = pc_run_lease(ctx, fa, fb, f, tuning, first[i], end[i], width, lo0, lo1, hi0, hi1, counts[i],
                                    geometry[i], out[i], out_cap, n_out + i, stats ? stats + i : nullptr);
        __atomic_store_n(status + i, rc + 1, __ATOMIC_RELEASE);
        if (rc) return rc;
    }
    return PC_OK;
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
    PC_CHECK(ctx, pc_copy(ctx, counts, d_counts, (ng + 3) * 8, cudaMemcpyDeviceToHost));
    PC_CHECK(ctx, cudaStreamSynchronize(st));
    uint64_t n = counts[ng + 1];
    if (stats) {
        stats->kernel_ms = elapsed_ms(ctx->ev[6], ctx->ev[7]);
        stats->outputs = n;
        stats->launches = nu && nv ? 1 : 0;
    }
    uint64_t copy = std::min(n, out_cap);
    if (copy) {
        PC_CHECK(ctx, pc_copy(ctx, out, d_out, 2 * copy * 8, cudaMemcpyDeviceToHost));
        PC_CHECK(ctx, cudaStreamSynchronize(st));
    }
    return PC_OK;
}

// ------------------------------------------------------------------------------------------
// Many windows in one launch sequence (pc_multi_*).
//
// Every window carries its own interval, v range, subtile width, focus pair and filter family.
// Creation plans all u windows (on each window's A focus) and v windows (on its B focus), sizes
// every buffer and keeps them; a run regenerates the windows on the device and runs stages 2 and
// 3 over all of them as segments of one launch sequence.  With PC_RUN_GRAPH the sequence after
// the first eager run is recorded once into a CUDA graph and replayed.

struct pc_multi {
    pc_ctx *ctx;
    Scratch hold;                        // device buffers kept for the object's lifetime
    WinBatch wb;
    uint64_t *d_lists = nullptr;         // u windows (each on a 2048-entry boundary), then v windows
    Engine E;
    uint32_t nwin = 0;
    std::vector<uint32_t> tile_base;     // nwin + 1
    std::vector<uint64_t> sizes;         // per window: u count, v count
    std::vector<uint64_t> counts, geometry, out;
    uint64_t n_out = 0;
    int launches = 0;
    uint64_t graph_d2h = 0;          // bytes the recorded graph copies to the host per replay
    bool ran = false;
    cudaGraph_t graph = nullptr;
    cudaGraphExec_t exec = nullptr;
    uint64_t *h_counts = nullptr, *h_geo = nullptr;   // pinned copies written by the graph
    unsigned long long *h_nout = nullptr;
    uint32_t *h_deep = nullptr;
    explicit pc_multi(pc_ctx *c) : ctx(c), hold(c) { E.ctx = c; }
    ~pc_multi() {
        if (exec) cudaGraphExecDestroy(exec);
        if (graph) cudaGraphDestroy(graph);
        if (h_counts) cudaFreeHost(h_counts);
        if (h_geo) cudaFreeHost(h_geo);
        if (h_nout) cudaFreeHost(h_nout);
        if (h_deep) cudaFreeHost(h_deep);
    }
};

extern "C" int pc_multi_create(pc_ctx *ctx, const pc_focus *const *foci, uint32_t nfoci,
                               const pc_filters *const *families, uint32_t nfam, const pc_window *windows,
                               uint32_t nwin, const pc_tuning *tuning, uint64_t out_cap, pc_multi **out) {
    *out = nullptr;
    if (!foci || !families || !windows || nwin == 0) return pc_fail(ctx, PC_INVALID, "invalid window batch arguments");
    typedef unsigned __int128 w128;
    std::vector<const pc_focus *> focs(2 * (size_t)nwin);
    std::vector<uint64_t> lows(2 * (size_t)nwin), highs(2 * (size_t)nwin), pads(2 * (size_t)nwin);
    std::vector<uint32_t> fam_map(nfam, UINT32_MAX), tile_base(nwin + 1, 0);
    std::vector<const pc_filters *> used;
    uint64_t ntiles = 0;
    for (uint32_t i = 0; i < nwin; ++i) {
        const pc_window &w = windows[i];
        if (w.focus_a >= nfoci || w.focus_b >= nfoci || w.family >= nfam)
            return pc_fail(ctx, PC_INVALID, "window refers to a missing focus or filter family");
        const pc_filters *f = families[w.family];
        const pc_focus *fa = foci[w.focus_a], *fb = foci[w.focus_b];
        if (!f || !fa || !fb) return pc_fail(ctx, PC_INVALID, "null focus or filter family");
        if (pc_focus_modulus(fa) != f->A || pc_focus_modulus(fb) != f->B)
            return pc_fail(ctx, PC_INVALID, "focus moduli differ from the filter family's A and B");
        const w128 lo = (w128)w.lo1 << 64 | w.lo0, hi = (w128)w.hi1 << 64 | w.hi0;
        if (hi <= lo || (hi >> 96)) return pc_fail(ctx, PC_INVALID, "invalid window interval");
        if (w.width == 0 || w.end <= w.first) return pc_fail(ctx, PC_INVALID, "invalid window v range");
        const w128 ulo = (lo + (w128)w.first * f->A) / f->B + 1, uhi = (hi + (w128)(w.end - 1) * f->A) / f->B + 1;
        if (uhi >> 64) return pc_fail(ctx, PC_INVALID, "u window exceeds 64 bits");
        const uint64_t nt = (w.end - w.first + w.width - 1) / w.width;
        if (!tiles_fit(w.first, w.end, w.width, nt)) return pc_fail(ctx, PC_INVALID, "inconsistent subtile geometry");
        tile_base[i] = (uint32_t)ntiles;
        ntiles += nt;
        if (ntiles >= (UINT64_C(1) << 31)) return pc_fail(ctx, PC_INVALID, "too many subtiles");
        focs[i] = fa;
        lows[i] = (uint64_t)ulo;
        highs[i] = (uint64_t)uhi;
        pads[i] = SEG_ALIGN;
        focs[nwin + i] = fb;
        lows[nwin + i] = w.first;
        highs[nwin + i] = w.end;
        pads[nwin + i] = 1;
        if (fam_map[w.family] == UINT32_MAX) {
            fam_map[w.family] = (uint32_t)used.size();
            used.push_back(f);
        }
    }
    tile_base[nwin] = (uint32_t)ntiles;
    pc_multi *m = new pc_multi(ctx);
    m->nwin = nwin;
    m->tile_base = tile_base;
    int rc = winbatch_plan(ctx, m->hold, focs.data(), lows.data(), highs.data(), pads.data(), 2 * nwin,
                           (UINT64_C(1) << 32) - 1, m->wb, nullptr);
    if (!rc) rc = m->hold.get(&m->d_lists, std::max<uint64_t>(1, m->wb.out_len));
    if (rc) {
        delete m;
        return rc;
    }
    const uint64_t vstart = m->wb.base[nwin];
    Engine &E = m->E;
    E.us = m->d_lists;
    E.nu = vstart;
    E.vs = m->d_lists + vstart;
    E.nv = m->wb.out_len - vstart;
    E.fams = used;
    E.ntiles = ntiles;
    E.out_cap = out_cap;
    E.tile_seg.resize(ntiles);
    m->sizes.resize(2 * (size_t)nwin);
    for (uint32_t i = 0; i < nwin; ++i) {
        const pc_window &w = windows[i];
        const pc_filters *f = families[w.family];
        SegDev g{};
        g.A = f->A;
        g.B = f->B;
        g.lo = u128{w.lo0, w.lo1};
        g.hi = u128{w.hi0, w.hi1};
        g.v_first = w.first;
        g.width = w.width;
        g.v_end = w.end;
        g.u_off = (uint32_t)m->wb.base[i];
        g.nu = (uint32_t)m->wb.total[i];
        g.v_off = (uint32_t)(m->wb.base[nwin + i] - vstart);
        g.nv = (uint32_t)m->wb.total[nwin + i];
        g.tile_base = tile_base[i];
        g.ntiles = tile_base[i + 1] - tile_base[i];
        g.fam = fam_map[w.family];
        E.segs.push_back(g);
        for (uint32_t t = tile_base[i]; t < tile_base[i + 1]; ++t) E.tile_seg[t] = i;
        m->sizes[2 * i] = g.nu;
        m->sizes[2 * i + 1] = g.nv;
    }
    rc = engine_prepare(E, tuning, m->hold);
    if (!rc) rc = pc_cuda_status(ctx, cudaStreamSynchronize(ctx->stream), "window batch set-up");
    if (rc) {
        delete m;
        return rc;
    }
    *out = m;
    return PC_OK;
}

namespace {

int multi_eager(pc_ctx *ctx, pc_multi *m, pc_stats *stats) {
    Engine &E = m->E;
    int launches = 0;
    PC_CHECK(ctx, cudaEventRecord(ctx->ev[4], ctx->stream));
    // pc_multi_create ran the count pass and its scan to size the lists; the unit counts, offsets
    // and kept words it left depend only on the windows, so the eager run goes straight to the emit
    // pass (a graph replay still runs both passes)
    int rc = winbatch_emit(ctx, m->wb, m->d_lists);
    if (rc) return rc;
    launches += 1;
    PC_CHECK(ctx, cudaEventRecord(ctx->ev[5], ctx->stream));
    rc = engine_eager(E, &launches);
    if (rc) return rc;
    m->counts.assign(E.ntiles * E.stride, 0);
    m->geometry.assign(2 * E.ntiles, 0);
    m->out.assign(2 * std::max<uint64_t>(1, E.out_cap), 0);
    rc = engine_collect(E, m->counts.data(), m->geometry.data(), m->out.data(), &m->n_out);
    m->launches = launches;
    if (!rc || rc == PC_OVERFLOW || rc == PC_ARITHMETIC) {
        engine_stats(E, stats, launches, m->n_out);
        if (stats) stats->window_ms = elapsed_ms(ctx->ev[4], ctx->ev[5]);
    }
    return rc;
}

// Records the whole run (windows, stages 2 and 3, and the copies of the counters) into a graph.
// The deep tier's grid and slice capacity come from the eager run that precedes the capture.
int multi_capture(pc_ctx *ctx, pc_multi *m) {
    Engine &E = m->E;
    cudaStream_t st = ctx->stream;
    const uint64_t nc = std::max<uint64_t>(1, E.ntiles * E.stride), ng = std::max<uint64_t>(1, 2 * E.ntiles);
    if (!m->h_counts) {
        PC_CHECK(ctx, cudaMallocHost((void **)&m->h_counts, nc * 8));
        PC_CHECK(ctx, cudaMallocHost((void **)&m->h_geo, ng * 8));
        PC_CHECK(ctx, cudaMallocHost((void **)&m->h_nout, 16));
        PC_CHECK(ctx, cudaMallocHost((void **)&m->h_deep, (uint64_t)E.grid * 4));
    }
    int rc = engine_match(E, 2);
    if (rc) return rc;
    PC_CHECK(ctx, cudaStreamBeginCapture(st, cudaStreamCaptureModeThreadLocal));
    int launches = 0;
    rc = winbatch_count(ctx, m->wb);
    if (!rc) rc = winbatch_emit(ctx, m->wb, m->d_lists);
    if (!rc) rc = engine_front(E, false, true, &launches);
    if (!rc) rc = engine_back(E, false, &launches);
    if (!rc) rc = pc_cuda_status(ctx, pc_copy(ctx, m->h_nout, E.d_nout, 16, cudaMemcpyDeviceToHost), "capture copy");
    if (!rc && E.ntiles) {
        rc = pc_cuda_status(ctx, pc_copy(ctx, m->h_counts, E.d_counts, E.ntiles * E.stride * 8, cudaMemcpyDeviceToHost),
                            "capture copy");
        if (!rc)
            rc = pc_cuda_status(ctx, pc_copy(ctx, m->h_geo, E.d_geo, 2 * E.ntiles * 8, cudaMemcpyDeviceToHost),
                                "capture copy");
    }
    if (!rc)
        rc = pc_cuda_status(ctx, pc_copy(ctx, m->h_deep, E.d_deep_count, (uint64_t)E.grid * 4, cudaMemcpyDeviceToHost),
                            "capture copy");
    cudaGraph_t g = nullptr;
    const cudaError_t e = cudaStreamEndCapture(st, &g);       // always leave capture mode
    if (!rc && e != cudaSuccess) rc = pc_cuda_fail(ctx, e, "end capture");
    if (rc) {
        if (g) cudaGraphDestroy(g);
        cudaGetLastError();
        return rc;
    }
    m->graph = g;
    PC_CHECK(ctx, cudaGraphInstantiate(&m->exec, g, 0));
    m->launches = launches + 5;
    // the copies recorded into the graph run at every replay, not at capture
    m->graph_d2h = 16 + (E.ntiles ? E.ntiles * E.stride * 8 + 2 * E.ntiles * 8 : 0) + (uint64_t)E.grid * 4;
    ctx->d2h -= m->graph_d2h;
    return PC_OK;
}

int multi_replay(pc_ctx *ctx, pc_multi *m, pc_stats *stats) {
    Engine &E = m->E;
    cudaStream_t st = ctx->stream;
    int rc = engine_match(E, 2);                          // another object may have lowered the limit
    if (rc) return rc;
    PC_CHECK(ctx, cudaEventRecord(ctx->ev[0], st));
    PC_CHECK(ctx, cudaGraphLaunch(m->exec, st));
    ctx->d2h += m->graph_d2h;
    PC_CHECK(ctx, cudaEventRecord(ctx->ev[1], st));
    PC_CHECK(ctx, cudaStreamSynchronize(st));
    for (int b = 0; b < E.grid; ++b)
        if (m->h_deep[b] > E.deep_cap) return pc_fail(ctx, PC_ARITHMETIC, "deep survivor count changed between runs");
    m->counts.assign(m->h_counts, m->h_counts + E.ntiles * E.stride);
    m->geometry.assign(m->h_geo, m->h_geo + 2 * E.ntiles);
    const unsigned long long nout[2] = {m->h_nout[0], m->h_nout[1]};
    m->n_out = nout[0];
    rc = engine_check(E, nout, m->counts.data());
    if (!rc && nout[0]) {
        PC_CHECK(ctx, pc_copy(ctx, m->out.data(), E.d_out, 2 * nout[0] * 8, cudaMemcpyDeviceToHost));
        PC_CHECK(ctx, cudaStreamSynchronize(st));
    }
    if (stats) {
        stats->kernel_ms = elapsed_ms(ctx->ev[0], ctx->ev[1]);
        stats->outputs = m->n_out;
        stats->launches = m->launches;
        stats->work_items = E.deep_max;
        stats->reserved[0] = E.tn.nb;
        stats->reserved[1] = E.tn.K;
        stats->reserved[2] = E.tn.threads;
        stats->reserved[3] = E.tn.nch;
        stats->reserved[4] = 1;
    }
    return rc;
}

}  // namespace

extern "C" int pc_multi_run(pc_ctx *ctx, pc_multi *m, uint32_t flags, pc_stats *stats) {
    if (!m) return pc_fail(ctx, PC_INVALID, "no window batch");
    if (stats) memset(stats, 0, sizeof(*stats));
    auto t0 = std::chrono::steady_clock::now();
    const uint64_t h2d0 = ctx->h2d, d2h0 = ctx->d2h;
    int rc = PC_OK;
    if (!(flags & PC_RUN_GRAPH) || !m->ran) {
        rc = multi_eager(ctx, m, stats);
        if (!rc) m->ran = true;
    }
    if (!rc && (flags & PC_RUN_GRAPH)) {
        if (!m->exec) rc = multi_capture(ctx, m);
        if (!rc) rc = multi_replay(ctx, m, stats);
    }
    if (stats) {
        stats->total_ms = std::chrono::duration<double, std::milli>(std::chrono::steady_clock::now() - t0).count();
        stats->h2d_bytes = ctx->h2d - h2d0;
        stats->d2h_bytes = ctx->d2h - d2h0;
    }
    return rc;
}

extern "C" int pc_multi_layout(const pc_multi *m, uint32_t *tile_base, uint64_t *sizes, uint64_t *info) {
    if (!m) return PC_INVALID;
    const Engine &E = m->E;
    if (tile_base) std::copy(m->tile_base.begin(), m->tile_base.end(), tile_base);
    if (sizes) std::copy(m->sizes.begin(), m->sizes.end(), sizes);
    if (info) {
        info[0] = E.ntiles;
        info[1] = E.stride;
        info[2] = E.nu;
        info[3] = E.nv;
        info[4] = E.deep_cap;
        info[5] = E.tn.nb;
        info[6] = E.tn.K;
        info[7] = E.tn.threads;
    }
    return PC_OK;
}

extern "C" int pc_multi_results(pc_ctx *ctx, const pc_multi *m, uint64_t *counts, uint64_t *geometry, uint64_t *out,
                                uint64_t out_cap, uint64_t *n_out) {
    if (!m || !m->ran) return pc_fail(ctx, PC_INVALID, "window batch has not run");
    if (counts) std::copy(m->counts.begin(), m->counts.end(), counts);
    if (geometry) std::copy(m->geometry.begin(), m->geometry.end(), geometry);
    *n_out = m->n_out;
    if (out) std::copy(m->out.begin(), m->out.begin() + 2 * std::min(m->n_out, out_cap), out);
    return PC_OK;
}

extern "C" int pc_multi_free(pc_ctx *ctx, pc_multi *m) {
    if (!m) return PC_OK;
    cudaStreamSynchronize(ctx->stream);
    delete m;
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

// The body of pc_run_plain_static once its device is current.
static int plain_static_on(int device, const uint64_t *us, uint64_t nu, const uint64_t *vs, uint64_t nv, uint64_t A,
                    uint64_t B, uint64_t lo0, uint64_t lo1, uint64_t hi0, uint64_t hi1, const uint32_t *primes,
                    uint32_t nres, const uint8_t *allowed, uint32_t ng, uint64_t o_counts, uint64_t o_fc,
                    uint64_t o_bits, uint64_t o_us, uint64_t o_vs, uint64_t o_out, uint64_t *counts, uint64_t *out,
                    uint64_t out_cap, char *err, int err_len);

extern "C" int pc_run_plain_static(int device, const uint64_t *us, uint64_t nu, const uint64_t *vs, uint64_t nv,
                                   uint64_t A, uint64_t B, uint64_t lo0, uint64_t lo1, uint64_t hi0, uint64_t hi1,
                                   const uint32_t *primes, uint32_t nres, const uint8_t *allowed, uint64_t *counts,
                                   uint64_t *out, uint64_t out_cap, char *err, int err_len) {
    if (device < 0 || device >= STATIC_MAX_DEVICES) return static_fail(err, err_len, PC_INVALID, "device index out of range");
    if (nres == 0 || nres > PC_MAX_RES || A == 0 || B == 0 || !counts || !primes || !allowed || (nu && !us) ||
        (nv && !vs) || (out_cap && !out))
        return static_fail(err, err_len, PC_INVALID, "invalid plain tile arguments");
    // every size is bounded by the scratch before any offset is formed, so no product below wraps
    constexpr uint64_t too_big = STATIC_SCRATCH_BYTES;
    if (nu > too_big / 8 || nv > too_big / 8 || out_cap > too_big / 16)
        return static_fail(err, err_len, PC_INVALID, "tile exceeds the 16 MiB static scratch of pc_run_plain_static");
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

    // the caller's current device is put back on every return
    int previous = -1;
    cudaError_t e = cudaGetDevice(&previous);
    if (e != cudaSuccess) return static_cuda(err, err_len, e, "cudaGetDevice");
    if (previous != device) {
        e = cudaSetDevice(device);
        if (e != cudaSuccess) return static_cuda(err, err_len, e, "cudaSetDevice");
    }
    const int rc = plain_static_on(device, us, nu, vs, nv, A, B, lo0, lo1, hi0, hi1, primes, nres, allowed, ng,
                                   o_counts, o_fc, o_bits, o_us, o_vs, o_out, counts, out, out_cap, err, err_len);
    if (previous != device) {
        e = cudaSetDevice(previous);
        if (e != cudaSuccess && rc == PC_OK) return static_cuda(err, err_len, e, "cudaSetDevice (restore)");
    }
    return rc;
}

static int plain_static_on(int device, const uint64_t *us, uint64_t nu, const uint64_t *vs, uint64_t nv, uint64_t A,
                    uint64_t B, uint64_t lo0, uint64_t lo1, uint64_t hi0, uint64_t hi1, const uint32_t *primes,
                    uint32_t nres, const uint8_t *allowed, uint32_t ng, uint64_t o_counts, uint64_t o_fc,
                    uint64_t o_bits, uint64_t o_us, uint64_t o_vs, uint64_t o_out, uint64_t *counts, uint64_t *out,
                    uint64_t out_cap, char *err, int err_len) {
    cudaError_t e = cudaSuccess;
    // Set-up, once per device, with that device current.  The cached address belongs to the
    // device's primary context; a process that resets the device (cudaDeviceReset) must not call
    // this entry point on it again.
    if (!g_static_ptr[device]) {
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
