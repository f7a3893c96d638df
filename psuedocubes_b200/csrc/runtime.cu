// Context, memory accounting, device buffers, device-wide scan and the limb self-test.
#include "common.cuh"
#include <algorithm>
#include <cstring>

int pc_fail(pc_ctx *ctx, int code, const std::string &msg) {
    if (ctx) ctx->err = msg;
    return code;
}

int pc_cuda_fail(pc_ctx *ctx, cudaError_t e, const char *what) {
    if (ctx) ctx->err = std::string(what) + ": " + cudaGetErrorString(e);
    return PC_CUDA;
}

int pc_alloc(pc_ctx *ctx, void **ptr, uint64_t bytes) {
    bytes = (bytes + 255) & ~UINT64_C(255);
    if (ctx->in_use + bytes > ctx->cap)
        return pc_fail(ctx, PC_NOMEM, "device memory cap exceeded");
    cudaError_t e = cudaMallocAsync(ptr, bytes, ctx->stream);
    if (e != cudaSuccess) {
        cudaGetLastError();
        return pc_fail(ctx, PC_NOMEM, std::string("device allocation failed: ") + cudaGetErrorString(e));
    }
    ctx->in_use += bytes;
    ctx->peak = std::max(ctx->peak, ctx->in_use);
    return PC_OK;
}

void pc_release(pc_ctx *ctx, void *ptr, uint64_t bytes) {
    if (!ptr) return;
    bytes = (bytes + 255) & ~UINT64_C(255);
    cudaFreeAsync(ptr, ctx->stream);
    ctx->in_use -= std::min(ctx->in_use, bytes);
}

extern "C" int pc_version(void) { return 1; }

extern "C" int pc_device_count(int *count) {
    cudaError_t e = cudaGetDeviceCount(count);
    if (e != cudaSuccess) {
        cudaGetLastError();
        *count = 0;
    }
    return PC_OK;
}

extern "C" const char *pc_last_error(const pc_ctx *ctx) { return ctx ? ctx->err.c_str() : "no context"; }

extern "C" int pc_init(int device, uint64_t mem_cap, double fraction, pc_ctx **out) {
    *out = nullptr;
    if (fraction <= 0.0 || fraction > 1.0) return PC_INVALID;
    pc_ctx *ctx = new pc_ctx();
    ctx->device = device;
    cudaError_t e = cudaSetDevice(device);
    if (e != cudaSuccess) {
        cudaGetLastError();
        delete ctx;
        return PC_CUDA;
    }
    size_t free_b = 0, total_b = 0;
    if (cudaMemGetInfo(&free_b, &total_b) != cudaSuccess || cudaStreamCreateWithFlags(&ctx->stream, cudaStreamNonBlocking) != cudaSuccess) {
        cudaGetLastError();
        delete ctx;
        return PC_CUDA;
    }
    for (auto &ev : ctx->ev) cudaEventCreate(&ev);
    for (auto &ev : ctx->marks) cudaEventCreate(&ev);
    int64_t by_free = (int64_t)free_b - (int64_t)256 * 1024 * 1024;
    int64_t cap = std::min<int64_t>((int64_t)mem_cap, std::min<int64_t>((int64_t)(total_b * fraction), by_free));
    if (cap <= 0) {
        pc_free(ctx);
        return PC_NOMEM;
    }
    ctx->cap = (uint64_t)cap;
    cudaDeviceProp prop;
    cudaGetDeviceProperties(&prop, device);
    ctx->sm_count = prop.multiProcessorCount;
    ctx->cc_major = prop.major;
    ctx->cc_minor = prop.minor;
    strncpy(ctx->name, prop.name, sizeof(ctx->name) - 1);
    // Keep freed stream-ordered allocations cached in the pool between calls.
    cudaMemPool_t pool;
    if (cudaDeviceGetDefaultMemPool(&pool, device) == cudaSuccess) {
        uint64_t threshold = UINT64_MAX;
        cudaMemPoolSetAttribute(pool, cudaMemPoolAttrReleaseThreshold, &threshold);
    }
    cudaGetLastError();
    *out = ctx;
    return PC_OK;
}

extern "C" int pc_host_alloc(uint64_t bytes, void **out) {
    if (!out) return PC_INVALID;
    *out = nullptr;
    if (cudaHostAlloc(out, std::max<uint64_t>(bytes, 16), cudaHostAllocDefault) != cudaSuccess) {
        cudaGetLastError();
        *out = nullptr;
        return PC_NOMEM;
    }
    return PC_OK;
}

extern "C" int pc_host_free(void *p) {
    if (p && cudaFreeHost(p) != cudaSuccess) {
        cudaGetLastError();
        return PC_CUDA;
    }
    return PC_OK;
}

extern "C" int pc_free(pc_ctx *ctx) {
    if (!ctx) return PC_OK;
    if (ctx->stream) cudaStreamSynchronize(ctx->stream);
    for (auto &ev : ctx->ev)
        if (ev) cudaEventDestroy(ev);
    for (auto &ev : ctx->marks)
        if (ev) cudaEventDestroy(ev);
    if (ctx->stream) cudaStreamDestroy(ctx->stream);
    delete ctx;
    return PC_OK;
}

extern "C" int pc_mem_info(const pc_ctx *ctx, uint64_t *in_use, uint64_t *peak, uint64_t *cap) {
    *in_use = ctx->in_use;
    *peak = ctx->peak;
    *cap = ctx->cap;
    return PC_OK;
}

extern "C" int pc_copy_info(const pc_ctx *ctx, uint64_t *h2d, uint64_t *d2h) {
    if (!ctx || !h2d || !d2h) return PC_INVALID;
    *h2d = ctx->h2d;
    *d2h = ctx->d2h;
    return PC_OK;
}

extern "C" int pc_device_info(const pc_ctx *ctx, int *sm_count, int *cc_major, int *cc_minor, char *name, int name_len) {
    *sm_count = ctx->sm_count;
    *cc_major = ctx->cc_major;
    *cc_minor = ctx->cc_minor;
    if (name && name_len > 0) {
        strncpy(name, ctx->name, name_len - 1);
        name[name_len - 1] = 0;
    }
    return PC_OK;
}

extern "C" int pc_sync(pc_ctx *ctx) {
    PC_CHECK(ctx, cudaStreamSynchronize(ctx->stream));
    return PC_OK;
}

extern "C" int pc_mark(pc_ctx *ctx, int slot) {
    if (slot < 0 || slot >= 8) return pc_fail(ctx, PC_INVALID, "timer slot out of range");
    PC_CHECK(ctx, cudaEventRecord(ctx->marks[slot], ctx->stream));
    return PC_OK;
}

extern "C" int pc_elapsed(pc_ctx *ctx, int a, int b, double *ms) {
    if (a < 0 || a >= 8 || b < 0 || b >= 8) return pc_fail(ctx, PC_INVALID, "timer slot out of range");
    PC_CHECK(ctx, cudaEventSynchronize(ctx->marks[b]));
    float f = 0;
    PC_CHECK(ctx, cudaEventElapsedTime(&f, ctx->marks[a], ctx->marks[b]));
    *ms = f;
    return PC_OK;
}

// ------------------------------------------------------------------------------------------
// buffers

extern "C" int pc_buf_upload(pc_ctx *ctx, const uint64_t *host, uint64_t n, pc_buf **out) {
    *out = nullptr;
    pc_buf *b = new pc_buf();
    b->n = n;
    b->bytes = std::max<uint64_t>(n * 8, 16);
    int rc = pc_alloc(ctx, (void **)&b->d, b->bytes);
    if (rc) {
        delete b;
        return rc;
    }
    if (n) {
        cudaError_t e = pc_copy(ctx, b->d, host, n * 8, cudaMemcpyHostToDevice);
        if (e == cudaSuccess) e = cudaStreamSynchronize(ctx->stream);
        if (e != cudaSuccess) {
            pc_release(ctx, b->d, b->bytes);
            delete b;
            return pc_cuda_fail(ctx, e, "upload");
        }
    }
    *out = b;
    return PC_OK;
}

extern "C" int pc_buf_download(pc_ctx *ctx, const pc_buf *buf, uint64_t offset, uint64_t n, uint64_t *host) {
    if (offset > buf->n || n > buf->n - offset) return pc_fail(ctx, PC_INVALID, "download out of range");
    if (!n) return PC_OK;
    PC_CHECK(ctx, pc_copy(ctx, host, buf->d + offset, n * 8, cudaMemcpyDeviceToHost));
    PC_CHECK(ctx, cudaStreamSynchronize(ctx->stream));
    return PC_OK;
}

extern "C" int pc_buf_size(const pc_buf *buf, uint64_t *n) {
    *n = buf ? buf->n : 0;
    return PC_OK;
}

extern "C" int pc_buf_free(pc_ctx *ctx, pc_buf *buf) {
    if (!buf) return PC_OK;
    pc_release(ctx, buf->d, buf->bytes);
    delete buf;
    return PC_OK;
}

__global__ void k_searchsorted(const uint64_t *__restrict__ a, uint64_t n, const uint64_t *__restrict__ q,
                               uint64_t nq, uint64_t *__restrict__ out) {
    uint64_t i = blockIdx.x * (uint64_t)blockDim.x + threadIdx.x;
    if (i >= nq) return;
    uint64_t key = q[i], lo = 0, hi = n;
    while (lo < hi) {
        uint64_t mid = lo + (hi - lo) / 2;
        if (a[mid] < key) lo = mid + 1;
        else hi = mid;
    }
    out[i] = lo;
}

extern "C" int pc_buf_searchsorted(pc_ctx *ctx, const pc_buf *buf, const uint64_t *queries, uint64_t n, uint64_t *positions) {
    if (!n) return PC_OK;
    Scratch s(ctx);
    uint64_t *dq, *dp;
    int rc = s.get(&dq, n);
    if (!rc) rc = s.get(&dp, n);
    if (rc) return rc;
    PC_CHECK(ctx, pc_copy(ctx, dq, queries, n * 8, cudaMemcpyHostToDevice));
    k_searchsorted<<<(unsigned)((n + 255) / 256), 256, 0, ctx->stream>>>(buf->d, buf->n, dq, n, dp);
    PC_LAUNCHED(ctx, "searchsorted");
    PC_CHECK(ctx, pc_copy(ctx, positions, dp, n * 8, cudaMemcpyDeviceToHost));
    PC_CHECK(ctx, cudaStreamSynchronize(ctx->stream));
    return PC_OK;
}

// ------------------------------------------------------------------------------------------
// Exclusive scan of uint64 (three phases: per-block sums, scan of the block sums, add back).

static constexpr int SCAN_T = 512, SCAN_ITEMS = 4, SCAN_TILE = SCAN_T * SCAN_ITEMS;

__device__ __forceinline__ uint64_t block_exclusive_scan(uint64_t v, uint64_t *warp_sums, uint64_t *total) {
    const uint32_t lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
    uint64_t x = v;
#pragma unroll
    for (int d = 1; d < 32; d <<= 1) {
        uint64_t y = __shfl_up_sync(0xffffffffu, x, d);
        if (lane >= (uint32_t)d) x += y;
    }
    if (lane == 31) warp_sums[warp] = x;
    __syncthreads();
    if (warp == 0) {
        uint64_t w = lane < blockDim.x / 32 ? warp_sums[lane] : 0;
#pragma unroll
        for (int d = 1; d < 32; d <<= 1) {
            uint64_t y = __shfl_up_sync(0xffffffffu, w, d);
            if (lane >= (uint32_t)d) w += y;
        }
        warp_sums[lane] = w;
    }
    __syncthreads();
    uint64_t before = warp ? warp_sums[warp - 1] : 0;
    if (total) *total = warp_sums[blockDim.x / 32 - 1];
    return before + x - v;
}

__global__ void k_scan_tiles(const uint64_t *__restrict__ in, uint64_t *__restrict__ out, uint64_t n,
                             uint64_t *__restrict__ tile_sums) {
    __shared__ uint64_t warp_sums[32];
    uint64_t base = blockIdx.x * (uint64_t)SCAN_TILE + threadIdx.x * (uint64_t)SCAN_ITEMS;
    uint64_t v[SCAN_ITEMS], sum = 0;
#pragma unroll
    for (int k = 0; k < SCAN_ITEMS; ++k) {
        v[k] = base + k < n ? in[base + k] : 0;
        sum += v[k];
    }
    uint64_t total;
    uint64_t run = block_exclusive_scan(sum, warp_sums, &total);
#pragma unroll
    for (int k = 0; k < SCAN_ITEMS; ++k) {
        if (base + k < n) out[base + k] = run;
        run += v[k];
    }
    if (threadIdx.x == 0) tile_sums[blockIdx.x] = total;
}

__global__ void k_scan_add(uint64_t *__restrict__ out, uint64_t n, const uint64_t *__restrict__ offsets) {
    uint64_t i = blockIdx.x * (uint64_t)SCAN_TILE + threadIdx.x;
    uint64_t add = offsets[blockIdx.x];
    for (int k = 0; k < SCAN_ITEMS; ++k, i += SCAN_T)
        if (i < n) out[i] += add;
}

// Words of scratch the scan of n values needs (two arrays of tile sums per level).
uint64_t pc_scan_workspace(uint64_t n) {
    uint64_t words = 0;
    for (;;) {
        const uint64_t tiles = (n + SCAN_TILE - 1) / SCAN_TILE;
        words += 2 * (tiles + 1);
        if (tiles <= 1) return words;
        n = tiles;
    }
}

// out[i] = sum in[0..i); *total_dev = sum of all (device pointer, may be null).  in may alias out.
// ws holds pc_scan_workspace(n) words; nothing is allocated and nothing waits for the device, so
// the scan can be recorded into a CUDA graph.
int pc_exclusive_scan_ws(pc_ctx *ctx, const uint64_t *in, uint64_t *out, uint64_t n, uint64_t *total_dev,
                         uint64_t *ws) {
    if (n == 0) {
        if (total_dev) PC_CHECK(ctx, cudaMemsetAsync(total_dev, 0, 8, ctx->stream));
        return PC_OK;
    }
    const uint64_t tiles = (n + SCAN_TILE - 1) / SCAN_TILE;
    uint64_t *sums = ws, *sums_scan = ws + tiles + 1;
    k_scan_tiles<<<(unsigned)tiles, SCAN_T, 0, ctx->stream>>>(in, out, n, sums);
    PC_LAUNCHED(ctx, "scan tiles");
    if (tiles > 1) {
        int rc = pc_exclusive_scan_ws(ctx, sums, sums_scan, tiles, total_dev, ws + 2 * (tiles + 1));
        if (rc) return rc;
        k_scan_add<<<(unsigned)tiles, SCAN_T, 0, ctx->stream>>>(out, n, sums_scan);
        PC_LAUNCHED(ctx, "scan add");
    } else if (total_dev) {
        PC_CHECK(ctx, cudaMemcpyAsync(total_dev, sums, 8, cudaMemcpyDeviceToDevice, ctx->stream));
    }
    return PC_OK;
}

int pc_exclusive_scan_u64(pc_ctx *ctx, const uint64_t *in, uint64_t *out, uint64_t n, uint64_t *total_dev) {
    Scratch s(ctx);
    uint64_t *ws;
    int rc = s.get(&ws, pc_scan_workspace(n));
    if (rc) return rc;
    return pc_exclusive_scan_ws(ctx, in, out, n, total_dev, ws);
}

// ------------------------------------------------------------------------------------------
// limb self-test (kernels/pseudocube.cuh:7-11 semantics)

__global__ void k_wide(const uint64_t *__restrict__ in4, uint64_t *__restrict__ out3, uint64_t n) {
    uint64_t i = blockIdx.x * (uint64_t)blockDim.x + threadIdx.x;
    if (i >= n) return;
    u128 l = mul_wide(in4[4 * i], in4[4 * i + 1]), r = mul_wide(in4[4 * i + 2], in4[4 * i + 3]);
    u128 d = sub128(l, r);
    out3[3 * i] = d.lo;
    out3[3 * i + 1] = d.hi;
    out3[3 * i + 2] = less128(l, r);
}

extern "C" int pc_selftest_wide(pc_ctx *ctx, const uint64_t *in4, uint64_t *out3, uint64_t n) {
    if (!n) return PC_OK;
    Scratch s(ctx);
    uint64_t *din, *dout;
    int rc = s.get(&din, 4 * n);
    if (!rc) rc = s.get(&dout, 3 * n);
    if (rc) return rc;
    PC_CHECK(ctx, pc_copy(ctx, din, in4, 32 * n, cudaMemcpyHostToDevice));
    k_wide<<<(unsigned)((n + 255) / 256), 256, 0, ctx->stream>>>(din, dout, n);
    PC_LAUNCHED(ctx, "wide self-test");
    PC_CHECK(ctx, pc_copy(ctx, out3, dout, 24 * n, cudaMemcpyDeviceToHost));
    PC_CHECK(ctx, cudaStreamSynchronize(ctx->stream));
    return PC_OK;
}
