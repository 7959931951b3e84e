/*
 * xb_sort.cuh
 *
 * Device scans and the stable radix sort used when kds_final is written:
 * prefix sums of the per-slot tuple sizes and ready flags, the running
 * maxima and counts of the window-rank step, and the stable ordering of
 * the groups by their sort-key words (GPU-Sort of the final groups, the
 * work of cuda_gpusort.cu:15-996).
 *
 * Scans are three passes over tiles of XB_SCAN_TILE elements: every CTA
 * reduces its tile, the tile totals are scanned (by the same passes when
 * there are more than one tile's worth of them), and every CTA scans its
 * tile from its total's prefix.  The radix sort orders (key, value) pairs
 * by 8-bit digits, least significant first; each pass counts the digits
 * of every tile per warp, scans the digit-major counts of all tiles, and
 * scatters: warp w takes the 512 consecutive elements of its part of the
 * tile in order, and lanes with equal digits in one step are ranked by
 * lane (__match_any_sync), so the order of equal digits is kept and every
 * pass is stable.
 */
#ifndef XB_SORT_CUH
#define XB_SORT_CUH

#include <cuda_runtime.h>
#include <stdint.h>

#define XB_SCAN_BLOCK   256
#define XB_SCAN_ITEMS   16
#define XB_SCAN_TILE    (XB_SCAN_BLOCK * XB_SCAN_ITEMS)     /* 4096 elements per CTA */

struct XbOpSum {
    template <typename T> __device__ __forceinline__ T operator()(T a, T b) const { return a + b; }
    template <typename T> __device__ __forceinline__ static T identity() { return (T)0; }
};
struct XbOpMax {
    template <typename T> __device__ __forceinline__ T operator()(T a, T b) const { return a > b ? a : b; }
    template <typename T> __device__ __forceinline__ static T identity() { return (T)0; }
};

/* inclusive scan of one value per thread over the CTA (256 threads);
 * *total receives the CTA's total */
template <typename T, typename Op>
__device__ __forceinline__ T xb_block_scan_incl(T v, T *total)
{
    __shared__ T warp_tot[XB_SCAN_BLOCK / 32];
    const Op op;
    const uint32_t lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
#pragma unroll
    for (uint32_t o = 1; o < 32; o <<= 1) {
        const T u = __shfl_up_sync(0xffffffffu, v, o);
        if (lane >= o) v = op(v, u);
    }
    if (lane == 31)
        warp_tot[warp] = v;
    __syncthreads();
    if (warp == 0) {
        T w = lane < XB_SCAN_BLOCK / 32 ? warp_tot[lane] : Op::template identity<T>();
#pragma unroll
        for (uint32_t o = 1; o < 32; o <<= 1) {
            const T u = __shfl_up_sync(0xffffffffu, w, o);
            if (lane >= o) w = op(w, u);
        }
        if (lane < XB_SCAN_BLOCK / 32)
            warp_tot[lane] = w;
    }
    __syncthreads();
    if (warp > 0)
        v = op(warp_tot[warp - 1], v);
    *total = warp_tot[XB_SCAN_BLOCK / 32 - 1];
    __syncthreads();
    return v;
}

/* pass 1: the total of every tile */
template <typename T, typename Op>
__global__ void __launch_bounds__(XB_SCAN_BLOCK)
xb_scan_reduce(const T *in, uint64_t n, T *tile_tot)
{
    const Op op;
    const uint64_t base = (uint64_t)blockIdx.x * XB_SCAN_TILE;
    T v = Op::template identity<T>();
    for (uint32_t i = threadIdx.x; i < XB_SCAN_TILE; i += XB_SCAN_BLOCK) {
        const uint64_t k = base + i;
        if (k < n)
            v = op(v, in[k]);
    }
    T tot;
    xb_block_scan_incl<T, Op>(v, &tot);
    if (threadIdx.x == 0)
        tile_tot[blockIdx.x] = tot;
}

/* pass 3: every tile scanned from the prefix of the tiles before it
 * (tile_pre: exclusive prefixes of the tile totals; nullptr for a single
 * tile); thread t takes XB_SCAN_ITEMS consecutive elements */
template <typename T, typename Op, bool EXCLUSIVE>
__global__ void __launch_bounds__(XB_SCAN_BLOCK)
xb_scan_apply(const T *in, T *out, uint64_t n, const T *tile_pre)
{
    __shared__ T thread_incl[XB_SCAN_BLOCK];
    const Op op;
    const uint64_t base = (uint64_t)blockIdx.x * XB_SCAN_TILE + (uint64_t)threadIdx.x * XB_SCAN_ITEMS;
    T v[XB_SCAN_ITEMS];
    T sum = Op::template identity<T>();
#pragma unroll
    for (uint32_t j = 0; j < XB_SCAN_ITEMS; j++) {
        v[j] = base + j < n ? in[base + j] : Op::template identity<T>();
        sum = op(sum, v[j]);
    }
    T tot;
    thread_incl[threadIdx.x] = xb_block_scan_incl<T, Op>(sum, &tot);
    __syncthreads();
    /* the prefix before this thread's elements */
    T pre = tile_pre ? tile_pre[blockIdx.x] : Op::template identity<T>();
    if (threadIdx.x > 0)
        pre = op(pre, thread_incl[threadIdx.x - 1]);
#pragma unroll
    for (uint32_t j = 0; j < XB_SCAN_ITEMS; j++) {
        const T nxt = op(pre, v[j]);
        if (base + j < n)
            out[base + j] = EXCLUSIVE ? pre : nxt;
        pre = nxt;
    }
}

/* bytes of temporary storage a scan of n elements needs */
template <typename T>
static inline size_t xb_scan_temp_bytes(uint64_t n)
{
    size_t bytes = 0;
    while (n > 1) {
        const uint64_t tiles = (n + XB_SCAN_TILE - 1) / XB_SCAN_TILE;
        bytes += 2 * ((tiles * sizeof(T) + 255) & ~(size_t)255);
        if (tiles <= 1)
            break;
        n = tiles;
    }
    return bytes + 256;
}

/* scan of n elements of in into out (may be the same array) with op Op;
 * temp: xb_scan_temp_bytes<T>(n) bytes of device memory */
template <typename T, typename Op, bool EXCLUSIVE>
static cudaError_t xb_scan(const T *in, T *out, uint64_t n, void *temp, cudaStream_t st)
{
    if (n == 0)
        return cudaSuccess;
    const uint64_t tiles = (n + XB_SCAN_TILE - 1) / XB_SCAN_TILE;
    if (tiles == 1) {
        xb_scan_apply<T, Op, EXCLUSIVE><<<1, XB_SCAN_BLOCK, 0, st>>>(in, out, n, nullptr);
        return cudaGetLastError();
    }
    T *tot = (T *)temp;
    T *pre = (T *)((char *)temp + ((tiles * sizeof(T) + 255) & ~(size_t)255));
    void *rest = (char *)pre + ((tiles * sizeof(T) + 255) & ~(size_t)255);
    xb_scan_reduce<T, Op><<<(unsigned)tiles, XB_SCAN_BLOCK, 0, st>>>(in, n, tot);
    cudaError_t rc = xb_scan<T, Op, true>(tot, pre, tiles, rest, st);
    if (rc != cudaSuccess)
        return rc;
    xb_scan_apply<T, Op, EXCLUSIVE><<<(unsigned)tiles, XB_SCAN_BLOCK, 0, st>>>(in, out, n, pre);
    return cudaGetLastError();
}

/* ---------------------------------------------------------------------
 * stable radix sort of (key, value) pairs by 8-bit digits
 * --------------------------------------------------------------------- */
#define XB_RADIX_BINS   256
#define XB_RADIX_WARPS  (XB_SCAN_BLOCK / 32)
#define XB_RADIX_ROUNDS (XB_SCAN_TILE / XB_SCAN_BLOCK)       /* 16 steps of 32 per warp */

template <typename K>
__device__ __forceinline__ uint32_t xb_digit(K key, uint32_t shift)
{
    return (uint32_t)(key >> shift) & (XB_RADIX_BINS - 1);
}

/* the digits of warp w's part of a tile, counted per warp into cnt[w][d] */
template <typename K>
__device__ __forceinline__ void
xb_radix_count_warp(const K *keys, uint64_t n, uint64_t tile_base, uint32_t shift, uint32_t *cnt_w)
{
    const uint32_t lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
    const uint64_t base = tile_base + (uint64_t)warp * (XB_RADIX_ROUNDS * 32);
    for (uint32_t r = 0; r < XB_RADIX_ROUNDS; r++) {
        const uint64_t k = base + r * 32 + lane;
        const bool in = k < n;
        const uint32_t d = in ? xb_digit(keys[k], shift) : XB_RADIX_BINS;
        const uint32_t peers = __match_any_sync(0xffffffffu, d);
        if (in && (uint32_t)(__ffs(peers) - 1) == lane)
            cnt_w[d] += __popc(peers);
        __syncwarp();
    }
}

/* pass A: per tile, the count of every digit, digit-major (hist[d * tiles + tile]) */
template <typename K>
__global__ void __launch_bounds__(XB_SCAN_BLOCK)
xb_radix_hist(const K *keys, uint64_t n, uint32_t shift, uint32_t *hist, uint32_t tiles)
{
    __shared__ uint32_t cnt[XB_RADIX_WARPS][XB_RADIX_BINS];
    for (uint32_t i = threadIdx.x; i < XB_RADIX_WARPS * XB_RADIX_BINS; i += XB_SCAN_BLOCK)
        (&cnt[0][0])[i] = 0;
    __syncthreads();
    xb_radix_count_warp<K>(keys, n, (uint64_t)blockIdx.x * XB_SCAN_TILE, shift, cnt[threadIdx.x >> 5]);
    __syncthreads();
    for (uint32_t d = threadIdx.x; d < XB_RADIX_BINS; d += XB_SCAN_BLOCK) {
        uint32_t s = 0;
        for (uint32_t w = 0; w < XB_RADIX_WARPS; w++)
            s += cnt[w][d];
        hist[(uint64_t)d * tiles + blockIdx.x] = s;
    }
}

/* pass B: every element to its place: the tile's offset for its digit
 * (scanned hist), the counts of the warps before it, and its rank among
 * the equal digits before it in its warp's part */
template <typename K>
__global__ void __launch_bounds__(XB_SCAN_BLOCK)
xb_radix_scatter(const K *keys_in, const uint32_t *vals_in, K *keys_out, uint32_t *vals_out, uint64_t n,
                 uint32_t shift, const uint32_t *offs, uint32_t tiles)
{
    __shared__ uint32_t cnt[XB_RADIX_WARPS][XB_RADIX_BINS];
    for (uint32_t i = threadIdx.x; i < XB_RADIX_WARPS * XB_RADIX_BINS; i += XB_SCAN_BLOCK)
        (&cnt[0][0])[i] = 0;
    __syncthreads();
    const uint64_t tile_base = (uint64_t)blockIdx.x * XB_SCAN_TILE;
    xb_radix_count_warp<K>(keys_in, n, tile_base, shift, cnt[threadIdx.x >> 5]);
    __syncthreads();
    /* cnt[w][d] becomes the position of warp w's first element of digit d */
    for (uint32_t d = threadIdx.x; d < XB_RADIX_BINS; d += XB_SCAN_BLOCK) {
        uint32_t pos = offs[(uint64_t)d * tiles + blockIdx.x];
        for (uint32_t w = 0; w < XB_RADIX_WARPS; w++) {
            const uint32_t c = cnt[w][d];
            cnt[w][d] = pos;
            pos += c;
        }
    }
    __syncthreads();
    const uint32_t lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
    const uint64_t base = tile_base + (uint64_t)warp * (XB_RADIX_ROUNDS * 32);
    uint32_t *pos_w = cnt[warp];
    for (uint32_t r = 0; r < XB_RADIX_ROUNDS; r++) {
        const uint64_t k = base + r * 32 + lane;
        const bool in = k < n;
        K key = 0;
        uint32_t val = 0;
        if (in) {
            key = keys_in[k];
            val = vals_in[k];
        }
        const uint32_t d = in ? xb_digit(key, shift) : XB_RADIX_BINS;
        const uint32_t peers = __match_any_sync(0xffffffffu, d);
        const uint32_t rank = __popc(peers & ((1u << lane) - 1u));
        if (in) {
            const uint32_t p = pos_w[d] + rank;
            keys_out[p] = key;
            vals_out[p] = val;
        }
        __syncwarp();
        if (in && (uint32_t)(__ffs(peers) - 1) == lane)
            pos_w[d] += __popc(peers);
        __syncwarp();
    }
}

/* bytes of temporary storage xb_radix_sort of n pairs needs */
static inline size_t xb_radix_temp_bytes(uint64_t n)
{
    const uint64_t tiles = (n + XB_SCAN_TILE - 1) / XB_SCAN_TILE;
    const uint64_t h = tiles * XB_RADIX_BINS;
    return 2 * ((h * 4 + 255) & ~(size_t)255) + xb_scan_temp_bytes<uint32_t>(h);
}

/* stable sort of n (key, value) pairs by the key bits [0, bits), 8 at a
 * time; keys/vals in *_a on entry and on return (*_b is the other buffer
 * of each pair); n < 2^32 */
template <typename K>
static cudaError_t xb_radix_sort(K *keys_a, K *keys_b, uint32_t *vals_a, uint32_t *vals_b, uint64_t n,
                                 uint32_t bits, void *temp, cudaStream_t st)
{
    if (n <= 1)
        return cudaSuccess;
    const uint32_t tiles = (uint32_t)((n + XB_SCAN_TILE - 1) / XB_SCAN_TILE);
    const uint64_t h = (uint64_t)tiles * XB_RADIX_BINS;
    uint32_t *hist = (uint32_t *)temp;
    uint32_t *offs = (uint32_t *)((char *)temp + ((h * 4 + 255) & ~(size_t)255));
    void *scan_tmp = (char *)offs + ((h * 4 + 255) & ~(size_t)255);
    K *ki = keys_a, *ko = keys_b;
    uint32_t *vi = vals_a, *vo = vals_b;
    uint32_t passes = 0;
    for (uint32_t shift = 0; shift < bits; shift += 8, passes++) {
        xb_radix_hist<K><<<tiles, XB_SCAN_BLOCK, 0, st>>>(ki, n, shift, hist, tiles);
        cudaError_t rc = xb_scan<uint32_t, XbOpSum, true>(hist, offs, h, scan_tmp, st);
        if (rc != cudaSuccess)
            return rc;
        xb_radix_scatter<K><<<tiles, XB_SCAN_BLOCK, 0, st>>>(ki, vi, ko, vo, n, shift, offs, tiles);
        K *tk = ki; ki = ko; ko = tk;
        uint32_t *tv = vi; vi = vo; vo = tv;
    }
    if (passes & 1) {
        cudaMemcpyAsync(keys_a, ki, n * sizeof(K), cudaMemcpyDeviceToDevice, st);
        cudaMemcpyAsync(vals_a, vi, n * 4, cudaMemcpyDeviceToDevice, st);
    }
    return cudaGetLastError();
}

#endif  /* XB_SORT_CUH */
