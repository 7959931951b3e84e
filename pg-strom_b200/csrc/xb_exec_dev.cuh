/*
 * xb_exec_dev.cuh
 *
 * Device code shared by the interpreting executor kernel (xb_exec.cu) and
 * the session-specialised kernels generated at run time (xb_jit.cpp):
 * launch arguments, the work queue over chunk units, heap / Arrow column
 * access, partial-aggregate state arithmetic and the group tables.
 */
#ifndef XB_EXEC_DEV_CUH
#define XB_EXEC_DEV_CUH
#include "xb_plan.h"
#include "xb_device.cuh"

#define XB_BLOCK        256
#define XB_WARPS        (XB_BLOCK / 32)
#define XB_CLAIM        8           /* heap pages claimed per warp with one atomic; only the
                                     * page after the current one is prefetched into L2, so
                                     * resident warps keep ~16 KB each in flight */
#define XB_ROWS_UNIT    1024        /* rows per unit for ARROW / ROW chunks */
#define XB_MIN_BLOCKS   2           /* resident CTAs per SM the kernel is built for */
#define XB_PROBE_LIMIT  4096        /* max probes in the global group table */

/*
 * Hide a pointer's address space from the compiler.  Group-state atomics
 * (64-bit adds, int128 carries, compensated double adds) on the shared
 * group table measured far faster (0.45 vs 0.68 ms on the 20M-row join
 * workload) when issued through a pointer that may be shared or global
 * than through one the compiler has proven to be shared memory.
 */
__device__ __forceinline__ char *xb_generic_ptr(char *p)
{
    asm volatile("mov.b64 %0, %0;" : "+l"(p));
    return p;
}

/* 32-bit add to a counter in shared memory given by a generic address:
 * the native shared-memory atomic (64-bit shared atomics are not native) */
__device__ __forceinline__ void xb_red_shared_add_u32(void *p, uint32_t v)
{
    asm volatile("red.shared.add.u32 [%0], %1;" :: "r"((uint32_t)__cvta_generic_to_shared(p)), "r"(v) : "memory");
}

/* reductions on global memory given by a generic address that is known to
 * be global: fire-and-forget (red), so the issuing warp does not wait for
 * the L2 round trip as it does for an atomic whose old value it may use
 * (a generic-address atomic is issued as one) */
__device__ __forceinline__ void xb_red_g_add_u64(void *p, unsigned long long v)
{
    asm volatile("red.global.add.u64 [%0], %1;" :: "l"(__cvta_generic_to_global(p)), "l"(v) : "memory");
}

__device__ __forceinline__ void xb_red_g_or_u32(void *p, uint32_t v)
{
    asm volatile("red.global.or.b32 [%0], %1;" :: "l"(__cvta_generic_to_global(p)), "r"(v) : "memory");
}

__device__ __forceinline__ void xb_red_g_min_s64(void *p, long long v)
{
    asm volatile("red.global.min.s64 [%0], %1;" :: "l"(__cvta_generic_to_global(p)), "l"(v) : "memory");
}

__device__ __forceinline__ void xb_red_g_max_s64(void *p, long long v)
{
    asm volatile("red.global.max.s64 [%0], %1;" :: "l"(__cvta_generic_to_global(p)), "l"(v) : "memory");
}

__device__ __forceinline__ void xb_red_g_add_f64(void *p, double v)
{
    asm volatile("red.global.add.f64 [%0], %1;" :: "l"(__cvta_generic_to_global(p)), "d"(v) : "memory");
}

/* add to a little-endian multi-word integer in shared memory (generic
 * address) with native 32-bit shared atomics: each word is added with the
 * carry of the word below, and a carry out of a word is added to the next;
 * words that receive nothing are not touched, so a small positive value
 * costs one atomic.  The carry out of the top word is dropped (the sum is
 * modulo 2^(32 * nwords), as a two's complement accumulator is). */
__device__ __forceinline__ void xb_shared_add_words(void *p, const uint32_t *w, int nwords)
{
    const uint32_t base = (uint32_t)__cvta_generic_to_shared(p);
    uint32_t c = 0;
    for (int k = 0; k < nwords; k++) {
        const uint64_t add = (uint64_t)w[k] + c;
        if (add == 0) { c = 0; continue; }
        if (add == 0x100000000ULL) { c = 1; continue; }
        const uint32_t a = (uint32_t)add;
        uint32_t old;
        asm volatile("atom.shared.add.u32 %0, [%1], %2;" : "=r"(old) : "r"(base + 4 * k), "r"(a) : "memory");
        c = (old + a < old) ? 1u : 0u;
    }
}

__device__ __forceinline__ void xb_shared_add_u64w(void *p, uint64_t v)
{
    const uint32_t w[2] = {(uint32_t)v, (uint32_t)(v >> 32)};
    xb_shared_add_words(p, w, 2);
}

__device__ __forceinline__ void xb_shared_add_i128w(void *p, xb_i128 v)
{
    const unsigned __int128 u = (unsigned __int128)v;
    const uint32_t w[4] = {(uint32_t)u, (uint32_t)(u >> 32), (uint32_t)(u >> 64), (uint32_t)(u >> 96)};
    xb_shared_add_words(p, w, 4);
}

/* ================================================================
 * memory-order helpers (generic addresses: shared or global)
 * ================================================================ */
__device__ __forceinline__ uint32_t xb_ld_acquire(const uint32_t *p)
{
    uint32_t v;
    asm volatile("ld.acquire.gpu.u32 %0, [%1];" : "=r"(v) : "l"(p) : "memory");
    return v;
}
__device__ __forceinline__ void xb_st_release(uint32_t *p, uint32_t v)
{
    asm volatile("st.release.gpu.u32 [%0], %1;" :: "l"(p), "r"(v) : "memory");
}

__device__ __forceinline__ uint32_t xb_ld_relaxed(const uint32_t *p)
{
    uint32_t v;
    asm volatile("ld.relaxed.gpu.u32 %0, [%1];" : "=r"(v) : "l"(p));
    return v;
}

/* ================================================================
 * group-table growth (the device half; the host rehashes the table)
 * ================================================================ */
__device__ __forceinline__ void xb_gt_want_grow(xb_gtable *gt)
{
    if (*(volatile uint32_t *)&gt->grow == 0)
        atomicExch(&gt->grow, 1u);
}

/* count a new entry of the global table; once soft_cap entries are in
 * use the table asks to grow */
__device__ __forceinline__ void xb_gt_count_new(xb_gtable *gt)
{
    const unsigned long long n = atomicAdd((unsigned long long *)&gt->nused, 1ULL) + 1ULL;
    if (n >= gt->soft_cap)
        xb_gt_want_grow(gt);
}

/* a fresh (EMPTY) entry of the dump region for a group the table had no
 * room for; nullptr when the session has none left */
__device__ __forceinline__ char *xb_dump_slot(xb_gtable *gt, uint32_t gent_size)
{
    if (!gt->dump)
        return nullptr;
    xb_gt_want_grow(gt);
    const unsigned long long i = atomicAdd((unsigned long long *)&gt->dump_used, 1ULL);
    return i < gt->dump_cap ? gt->dump + i * (uint64_t)gent_size : nullptr;
}

/* L2 prefetch of a contiguous range by the TMA engine (sm_90+) */
__device__ __forceinline__ void xb_prefetch_l2(const void *p, uint32_t bytes)
{
    asm volatile("cp.async.bulk.prefetch.L2.global [%0], %1;" :: "l"(p), "r"(bytes) : "memory");
}

/* ================================================================
 * partial-aggregate state arithmetic
 * ================================================================ */
__device__ __forceinline__ void xb_atomic_add_i128(uint64_t *p, xb_i128 v)
{
    uint64_t lo = (uint64_t)v;
    uint64_t hi = (uint64_t)((unsigned __int128)v >> 64);
    uint64_t old = atomicAdd((unsigned long long *)&p[0], (unsigned long long)lo);
    if (old + lo < old)
        hi += 1;
    if (hi)
        atomicAdd((unsigned long long *)&p[1], (unsigned long long)hi);
}

/* compensated atomic sum: hi accumulates the rounded sum, lo the exact
 * rounding error of each addition (TwoSum on the value atomicAdd saw) */
__device__ __forceinline__ void xb_atomic_add_f64c(double *hi, double *lo, double x)
{
    double old = atomicAdd(hi, x);
    double s = __dadd_rn(old, x);
    double bp = __dsub_rn(s, old);
    double e = __dadd_rn(__dsub_rn(old, __dsub_rn(s, bp)), __dsub_rn(x, bp));
    if (e != 0.0)
        atomicAdd(lo, e);
}

/* the same two for state in global memory: only the additions whose old
 * value is needed wait for it */
__device__ __forceinline__ void xb_atomic_add_i128_g(uint64_t *p, xb_i128 v)
{
    uint64_t lo = (uint64_t)v;
    uint64_t hi = (uint64_t)((unsigned __int128)v >> 64);
    uint64_t old = atomicAdd((unsigned long long *)&p[0], (unsigned long long)lo);
    if (old + lo < old)
        hi += 1;
    if (hi)
        xb_red_g_add_u64(&p[1], hi);
}

__device__ __forceinline__ void xb_atomic_add_f64c_g(double *hi, double *lo, double x)
{
    double old = atomicAdd(hi, x);
    double s = __dadd_rn(old, x);
    double bp = __dsub_rn(s, old);
    double e = __dadd_rn(__dsub_rn(old, __dsub_rn(s, bp)), __dsub_rn(x, bp));
    if (e != 0.0)
        xb_red_g_add_f64(lo, e);
}

__device__ __forceinline__ double xb_reg_f64(uint64_t v, int rk)
{
    return rk == XB_RK_FLT ? __longlong_as_double(v) : (double)(int64_t)v;
}

/* 10^k for k = 0..18 */
__device__ __forceinline__ int64_t xb_pow10_i64(int k)
{
    int64_t p = 1;
    for (int i = 0; i < k; i++)
        p *= 10;
    return p;
}

/*
 * The value of a numeric varlena rescaled to weight_d, for sums: the same
 * number as xb_numeric_rescale(weight_d, w, v) of xb_numeric_decode, which
 * normalises trailing zeros away first; rescaling the digits as stored
 * gives the same result (the removed digits are zeros).  Short numerics of
 * up to four base-10000 digits are read with aligned 8-byte loads (every
 * aligned word that overlaps the datum lies in its page or buffer) and
 * rescaled in 64-bit arithmetic; others take the general decode.
 * Returns 0, or 1 on a corrupt datum.
 */
__device__ __forceinline__ int
xb_numeric_sum_value(const uint8_t *vl, int weight_d, uint8_t *p_kind, xb_i128 *p_out)
{
    const uintptr_t a = (uintptr_t)vl;
    const uint64_t *wp = (const uint64_t *)(a & ~(uintptr_t)7);
    const uint32_t o = (uint32_t)(a & 7);
    const uint64_t w0 = wp[0];
    const uint32_t h = (uint32_t)(w0 >> (8 * o)) & 0xff;
    const uint32_t len = (h >> 1) & 0x7f;
    /* short varlena, short-format numeric, 0..4 digits, within 3 words */
    if ((h & 1) && h != 1 && len >= 3 && len <= 11 && o + len <= 24) {
        const uint64_t w1 = (o + len > 8) ? wp[1] : 0;
        const uint64_t w2 = (o + len > 16) ? wp[2] : 0;
        auto byte = [&](uint32_t i) -> uint32_t {
            const uint32_t k = o + i;
            const uint64_t w = k < 8 ? w0 : (k < 16 ? w1 : w2);
            return (uint32_t)(w >> (8 * (k & 7))) & 0xff;
        };
        const uint32_t n_head = byte(1) | (byte(2) << 8);
        if ((n_head & 0xC000) == 0x8000 && ((len - 3) & 1) == 0) {
            const uint32_t ndigits = (len - 3) / 2;
            int pgweight = n_head & 0x003F;
            if (n_head & 0x0040)
                pgweight |= ~0x003F;
            int64_t v = 0;
            for (uint32_t i = 0; i < ndigits; i++)
                v = v * 10000 + (int16_t)(byte(3 + 2 * i) | (byte(4 + 2 * i) << 8));
            if (n_head & 0x2000)
                v = -v;
            const int weight_s = 4 * ((int)ndigits - (pgweight + 1));
            const int shift = weight_d - weight_s;
            if (shift == 0 || v == 0) {
                *p_kind = XB_NUM_VALID;
                *p_out = v;
                return 0;
            }
            if (shift < 0 && shift >= -18) {
                *p_kind = XB_NUM_VALID;
                *p_out = v / xb_pow10_i64(-shift);       /* truncates toward zero */
                return 0;
            }
            if (shift > 0 && shift <= 18) {
                const int64_t p = xb_pow10_i64(shift);
                const uint64_t m = v < 0 ? (uint64_t)(-(v + 1)) + 1 : (uint64_t)v;
                if (m <= (uint64_t)INT64_MAX / (uint64_t)p) {
                    *p_kind = XB_NUM_VALID;
                    *p_out = v * p;
                    return 0;
                }
            }
        }
    }
    int16_t w;
    xb_i128 v;
    if (xb_numeric_decode(vl, p_kind, &w, &v))
        return 1;
    *p_out = (*p_kind == XB_NUM_VALID) ? xb_numeric_rescale(weight_d, w, v) : 0;
    return 0;
}

/* per-value updates of the actions that are not combined across lanes */
__device__ __forceinline__ void
xb_agg_numeric_add(char *s, const uint8_t *vl, int16_t weight, xb_status *st)
{
    uint8_t kind; xb_i128 v;
    if (xb_numeric_sum_value(vl, weight, &kind, &v)) {
        XB_RAISE(st, ERRCODE_DEVICE_ERROR, XB_MSG_NUMERIC_CORRUPT);
    } else if (kind == XB_NUM_VALID) {
        atomicAdd((unsigned long long *)s, 1ULL);
        xb_atomic_add_i128((uint64_t *)(s + 8), v);
    } else {
        const uint32_t special = kind == XB_NUM_PINF ? PAGG_NUMERIC_ATTRS__PINF
                               : kind == XB_NUM_NINF ? PAGG_NUMERIC_ATTRS__NINF
                               : PAGG_NUMERIC_ATTRS__NAN;
        atomicOr((unsigned int *)(s + 24), special);
    }
}

/* xb_agg_numeric_add for an entry of a shared-memory group table (shared
 * form): 32-bit counter, 128-bit sum by word atomics; with nc the counter
 * holds the rows NOT counted (a special value, the caller adds NULLs) */
__device__ __forceinline__ void
xb_agg_numeric_add_sm(char *s, const uint8_t *vl, int16_t weight, xb_status *st, bool nc)
{
    uint8_t kind; xb_i128 v;
    if (xb_numeric_sum_value(vl, weight, &kind, &v)) {
        XB_RAISE(st, ERRCODE_DEVICE_ERROR, XB_MSG_NUMERIC_CORRUPT);
    } else if (kind == XB_NUM_VALID) {
        if (!nc)
            xb_red_shared_add_u32(s, 1u);
        xb_shared_add_i128w(s + 8, v);
    } else {
        if (nc)
            xb_red_shared_add_u32(s, 1u);
        const uint32_t special = kind == XB_NUM_PINF ? PAGG_NUMERIC_ATTRS__PINF
                               : kind == XB_NUM_NINF ? PAGG_NUMERIC_ATTRS__NINF
                               : PAGG_NUMERIC_ATTRS__NAN;
        atomicOr((unsigned int *)(s + 24), special);
    }
}

__device__ __forceinline__ void xb_agg_stddev_add(char *s, double x)
{
    atomicAdd((unsigned long long *)s, 1ULL);
    xb_atomic_add_f64c((double *)(s + 8), (double *)(s + 16), x);
    xb_atomic_add_f64c((double *)(s + 24), (double *)(s + 32), x * x);
}

__device__ __forceinline__ void xb_agg_covar_add(char *s, double x, double y)
{
    atomicAdd((unsigned long long *)s, 1ULL);
    xb_atomic_add_f64c((double *)(s + 8), (double *)(s + 16), x);
    xb_atomic_add_f64c((double *)(s + 24), (double *)(s + 32), x * x);
    xb_atomic_add_f64c((double *)(s + 40), (double *)(s + 48), y);
    xb_atomic_add_f64c((double *)(s + 56), (double *)(s + 64), y * y);
    xb_atomic_add_f64c((double *)(s + 72), (double *)(s + 80), x * y);
}

static __device__ __noinline__ void xb_init_states(const xb_plan *plan, char *e)
{
    for (uint32_t i = 0; i < plan->naggs; i++) {
        const xb_agg &a = plan->aggs[i];
        if (a.state_sz == 0)
            continue;
        uint64_t *s = (uint64_t *)(e + a.state_off);
        for (uint32_t k = 0; k < a.state_sz / 8; k++)
            s[k] = 0;
        switch (a.action) {
        case KAGG_ACTION__PMIN_INT32:
        case KAGG_ACTION__PMIN_INT64:
        case KAGG_ACTION__PMIN_FP64:
            s[0] = (uint64_t)INT64_MAX;
            break;
        case KAGG_ACTION__PMAX_INT32:
        case KAGG_ACTION__PMAX_INT64:
        case KAGG_ACTION__PMAX_FP64:
            s[0] = (uint64_t)INT64_MIN;
            break;
        default:
            break;
        }
    }
}

/* merge a shared-memory group entry's states into a global entry */
static __device__ __noinline__ void xb_merge_states(const xb_plan *plan, char *dst, const char *src)
{
    for (uint32_t i = 0; i < plan->naggs; i++) {
        const xb_agg &a = plan->aggs[i];
        if (a.state_sz == 0)
            continue;
        char *d = dst + a.state_off;
        const char *s = src + a.state_off;
        const uint64_t *su = (const uint64_t *)s;
        switch (a.action) {
        case KAGG_ACTION__NROWS_ANY:
        case KAGG_ACTION__NROWS_COND:
            if (su[0]) atomicAdd((unsigned long long *)d, su[0]);
            break;
        case KAGG_ACTION__PMIN_INT32:
        case KAGG_ACTION__PMIN_INT64:
        case KAGG_ACTION__PMIN_FP64:
            if (*(const uint32_t *)(s + 8)) {
                atomicOr((unsigned int *)(d + 8), 1u);
                atomicMin((long long *)d, (long long)su[0]);
            }
            break;
        case KAGG_ACTION__PMAX_INT32:
        case KAGG_ACTION__PMAX_INT64:
        case KAGG_ACTION__PMAX_FP64:
            if (*(const uint32_t *)(s + 8)) {
                atomicOr((unsigned int *)(d + 8), 1u);
                atomicMax((long long *)d, (long long)su[0]);
            }
            break;
        case KAGG_ACTION__PSUM_INT:
        case KAGG_ACTION__PAVG_INT:
            if (su[0]) {
                atomicAdd((unsigned long long *)d, su[0]);
                atomicAdd((unsigned long long *)(d + 8), su[1]);
            }
            break;
        case KAGG_ACTION__PSUM_INT64:
        case KAGG_ACTION__PAVG_INT64:
        case KAGG_ACTION__PSUM_NUMERIC:
        case KAGG_ACTION__PAVG_NUMERIC:
            if (su[0]) {
                atomicAdd((unsigned long long *)d, su[0]);
                xb_atomic_add_i128((uint64_t *)(d + 8),
                                   (xb_i128)(((unsigned __int128)su[2] << 64) | su[1]));
            }
            if (a.state_sz >= 32 && *(const uint32_t *)(s + 24))
                atomicOr((unsigned int *)(d + 24), *(const uint32_t *)(s + 24));
            break;
        case KAGG_ACTION__PSUM_FP:
        case KAGG_ACTION__PAVG_FP:
        case KAGG_ACTION__STDDEV:
        case KAGG_ACTION__COVAR:
            if (su[0]) {
                atomicAdd((unsigned long long *)d, su[0]);
                for (uint32_t k = 8; k + 16 <= a.state_sz; k += 16) {
                    xb_atomic_add_f64c((double *)(d + k), (double *)(d + k + 8),
                                       *(const double *)(s + k));
                    double lo = *(const double *)(s + k + 8);
                    if (lo != 0.0)
                        atomicAdd((double *)(d + k + 8), lo);
                }
            }
            break;
        default:
            break;
        }
    }
}

/* ================================================================
 * group keys
 * ================================================================ */
__device__ __forceinline__ uint32_t xb_numeric_varsize(const uint8_t *vl)
{
    if (vl[0] & 0x01)
        return (vl[0] >> 1) & 0x7f;
    return ((uint32_t)xb_fetch_le(vl, 4) >> 2) & 0x3fffffff;
}

/* key value of register 'reg' for this lane, as a key image */
__device__ __forceinline__ void
xb_key_from_regs(const xb_key &k, const XbRegs &R, uint32_t lane, xb_keyimg *img)
{
    img->isnull = RISNULL(R, k.reg);
    img->val = RVAL(R, k.reg);
    img->len = RAUX(R, k.reg);
}

__device__ __forceinline__ bool
xb_key_equal(const xb_key &k, const xb_keyimg &x, const xb_keyimg &y)
{
    if (x.isnull || y.isnull)
        return x.isnull && y.isnull;        /* NULLs group together */
    if (k.rk == XB_RK_TEXT)
        return x.len == y.len &&
               xb_bytes_eq((const uint8_t *)x.val, (const uint8_t *)y.val, x.len);
    if (k.rk == XB_RK_NUM) {
        int err = 0;
        return xb_numeric_cmp((const uint8_t *)x.val, (const uint8_t *)y.val, &err) == 0 && !err;
    }
    return x.val == y.val;
}

/* copy a key image into an entry; into the arena when 'gt' is given */
__device__ __forceinline__ bool
xb_key_store(const xb_key &k, const xb_keyimg &src, xb_keyimg *dst,
             xb_gtable *gt, xb_status *st)
{
    *dst = src;
    if (src.isnull || !gt)
        return true;
    if (k.rk == XB_RK_TEXT || k.rk == XB_RK_NUM) {
        uint32_t nbytes = (k.rk == XB_RK_TEXT) ? src.len
                                               : xb_numeric_varsize((const uint8_t *)src.val);
        unsigned long long off = atomicAdd((unsigned long long *)&gt->arena_used,
                                           (unsigned long long)((nbytes + 7) & ~7u));
        if (off + nbytes > gt->arena_sz / 2)
            xb_gt_want_grow(gt);
        if (off + nbytes > gt->arena_sz) {
            XB_RAISE(st, ERRCODE_SUSPEND_NO_SPACE, XB_MSG_ARENA_FULL);
            return false;
        }
        char *p = gt->arena + off;
        const char *s = (const char *)src.val;
        for (uint32_t i = 0; i < nbytes; i++)
            p[i] = s[i];
        dst->val = (uint64_t)p;
    }
    return true;
}

/*
 * Find the group whose keys equal 'keys', or create it.  Works on the
 * shared-memory table (gt == nullptr) and on the global table.  An entry
 * is claimed EMPTY->BUSY by CAS, initialised, then published READY with a
 * release store; readers wait (bounded) on BUSY entries.
 * Returns nullptr when the table is full (*full) or on error.
 */
static __device__ __noinline__ char *
xb_group_find(const xb_plan *plan, char *entries, uint64_t cap_mask, uint32_t hash,
              const xb_keyimg *keys, xb_gtable *gt, xb_status *st, bool *full)
{
    const uint32_t gsz = plan->gent_size;
    uint64_t pos = hash & cap_mask;
    uint64_t limit = gt ? (cap_mask < XB_PROBE_LIMIT ? cap_mask : XB_PROBE_LIMIT) : cap_mask;
    for (uint64_t probe = 0; probe <= limit; probe++) {
        char *e = entries + pos * gsz;
        xb_gent_head *h = (xb_gent_head *)e;
        uint32_t s = xb_ld_acquire(&h->state);
        if (s == XB_GSTATE_EMPTY) {
            if (atomicCAS(&h->state, XB_GSTATE_EMPTY, XB_GSTATE_BUSY) == XB_GSTATE_EMPTY) {
                h->hash = hash;
                xb_keyimg *img = (xb_keyimg *)(e + plan->gent_keys_off);
                bool ok = true;
                for (uint32_t k = 0; k < plan->nkeys; k++)
                    ok &= xb_key_store(plan->keys[k], keys[k], &img[k], gt, st);
                xb_init_states(plan, e);
                if (gt)
                    xb_gt_count_new(gt);
                xb_st_release(&h->state, XB_GSTATE_READY);
                return ok ? e : nullptr;
            }
            s = xb_ld_acquire(&h->state);
        }
        uint32_t spins = 0;
        while (s == XB_GSTATE_BUSY) {
            if (++spins > plan->wait_limit) {
                XB_RAISE(st, ERRCODE_DEVICE_ERROR, XB_MSG_WAIT_TIMEOUT);
                return nullptr;
            }
            __nanosleep(20);
            s = xb_ld_acquire(&h->state);
        }
        if (h->hash == hash) {
            const xb_keyimg *img = (const xb_keyimg *)(e + plan->gent_keys_off);
            bool eq = true;
            for (uint32_t k = 0; k < plan->nkeys && eq; k++)
                eq = xb_key_equal(plan->keys[k], img[k], keys[k]);
            if (eq)
                return e;
        }
        pos = (pos + 1) & cap_mask;
    }
    *full = true;
    return nullptr;
}

/* xb_group_find on the global table; a group that finds it without room
 * gets an entry of the dump region (merged into the grown table by the
 * host), and only when that is used up is SUSPEND_NO_SPACE raised */
static __device__ __noinline__ char *
xb_group_find_or_dump(const xb_plan *plan, xb_gtable *gt, uint32_t hash, const xb_keyimg *keys,
                      xb_status *st)
{
    bool full = false;
    char *g = xb_group_find(plan, gt->entries, gt->cap_mask, hash, keys, gt, st, &full);
    if (!g && full) {
        char *slot = xb_dump_slot(gt, plan->gent_size);
        if (slot) {
            full = false;
            g = xb_group_find(plan, slot, 0, hash, keys, gt, st, &full);
        }
        if (!g && full) {
            XB_RAISE(st, ERRCODE_SUSPEND_NO_SPACE, XB_MSG_GTABLE_FULL);
            atomicOr(&gt->overflow, 1u);
        }
    }
    return g;
}

/* ================================================================
 * launch arguments and the source layout
 * ================================================================ */
/* work a launch left when it stopped for its group table to grow: units
 * [unit, unit_end), the first of them from item 'item' on */
struct XbLeft {
    uint64_t unit;
    uint64_t unit_end;
    uint32_t item;
    uint32_t __pad;
};

struct XbExecArgs {
    const xb_plan  *plan;           /* device copy (copied into shared memory) */
    uint32_t        plan_bytes;     /* bytes of the plan copy: header + used code */
    const xb_task  *tasks;          /* work queue: chunks of this launch */
    uint32_t        ntasks;
    uint64_t        nunits;         /* total units over all tasks */
    uint32_t        format;         /* common KDS format of the tasks */
    uint32_t        sm_cap;         /* shared-memory group table entries (0: none) */
    uint32_t        warp_bytes;     /* shared memory of one warp: counters, cursors, registers */
    char           *dst;            /* projection: device kds_dst buffer, or nullptr */
    uint64_t        dst_len;
    xb_gtable      *gt;
    xb_status      *st;
    uint32_t        dyn_only;       /* claim every unit dynamically (CTAs join
                                     * the launch at any time: mixed launches) */
    uint32_t        part_cap;       /* partitioned aggregation: records per bucket */
    char           *part_buf;       /* bucket-major records, or nullptr (update in place) */
    uint32_t       *part_cnt;       /* records claimed per bucket */
    uint32_t        part_shift;     /* bucket = (hash & table mask) >> part_shift */
    uint32_t        resume;         /* a resume launch: left_in first, then claims that
                                     * continue those of the stopped launch */
    XbLeft         *left_out;       /* group-table growth on: where warps that stop
                                     * record their leftover work (nullptr: growth off) */
    uint32_t        left_cap;
    uint32_t        left_in_n;
    const XbLeft   *left_in;        /* resume: the stopped launch's leftover ranges */
    uint64_t        static_base0;   /* resume: units below were handed out statically */
    uint64_t        cursor0;        /* resume: dynamic claims the stopped launch made */
};

/* bucket counters of partitioned aggregation sit one per 128-byte line:
 * every aggregated row claims its slot with an atomic on its bucket's
 * counter, and counters sharing a line would serialise in one L2 slice */
#define XB_PART_CNT_STRIDE  32
#define XB_PART_MAX         (1u << 18)  /* buckets of one partitioned launch */

/* the replay launch of partitioned aggregation (xbj_replay) */
struct XbReplayArgs {
    const xb_plan  *plan;
    xb_gtable      *gt;
    xb_status      *st;
    char           *part_buf;       /* records (a full table marks the ones it left) */
    const uint32_t *part_cnt;
    uint32_t       *cursor;         /* next bucket to claim (zero at launch) */
    uint32_t        part_cap;
    uint32_t        nparts;
    uint32_t        retry;          /* replay only the records marked left */
    uint32_t        part_shift;     /* a bucket holds 1 << part_shift table slots */
};

/* largest existence bitmap of a direct depth (keys), 16 KB */
#define XB_DBITS_MAX_KEYS   (1u << 17)

/* a mixed launch: work item i sends a CTA to command items[i] */
struct XbMixArgs {
    const XbExecArgs *cmds;
    const uint32_t   *items;
    uint32_t          nitems;
    uint32_t         *cursor;       /* next item (zero at launch) */
};

/* per-warp counters, in shared memory */
struct XbWarpState {
    unsigned long long raw, in, out;
    unsigned long long depth[XB_MAX_DEPTH + 1];
};

/* fixed-offset loader of one depth-0 load */
struct XbFix {
    int32_t  off;                   /* attcacheoff of the column */
    uint8_t  ld;
    uint8_t  reg;
    uint16_t __pad;
};

/* column layout shared by every chunk of a launch, and the fixed-offset
 * loaders used while a tuple has no NULL bitmap */
struct XbSrcMeta {
    XbCol    cols[XB_MAX_COLS];
    XbFix    fix[XB_MAX_LOADS];
    int32_t  ncols;
    uint32_t fixed;                 /* 1: every depth-0 load is fixed-width at a cached offset */
    uint32_t fixed_end;             /* payload bytes those loads span */
    uint32_t __pad;
};

#define XB_WARP_HEAD    ((sizeof(XbWarpState) + 15) & ~(size_t)15)

__device__ __forceinline__ uint32_t xb_ld_acquire_cta(const uint32_t *p)
{
    uint32_t v;
    asm volatile("ld.acquire.cta.u32 %0, [%1];" : "=r"(v) : "l"(p) : "memory");
    return v;
}

__device__ __forceinline__ void xb_st_release_cta(uint32_t *p, uint32_t v)
{
    asm volatile("st.release.cta.u32 [%0], %1;" :: "l"(p), "r"(v) : "memory");
}

/* byte width of a fixed-width loader, 0 for varlena */
__device__ __forceinline__ int xb_ld_width(int ld)
{
    switch (ld) {
    case XB_LD_BOOL: return 1;
    case XB_LD_INT2: return 2;
    case XB_LD_INT4: case XB_LD_DATE: case XB_LD_FLT4: return 4;
    case XB_LD_INT8: case XB_LD_FLT8: return 8;
    }
    return 0;
}

/* ---------------------------------------------------------------
 * source units and 32-row batches
 * --------------------------------------------------------------- */
struct alignas(16) XbSrc {
    uint64_t unit;                  /* current unit (global index) */
    uint64_t claim_end;             /* BLOCK: end of the current claim */
    unsigned long long nx_l0;       /* BLOCK, lane 0: first unit of the claim taken ahead */
    unsigned long long sz_l0;       /* BLOCK, lane 0: its size */
    unsigned long long last_dyn;    /* BLOCK, lane 0: start of the last dynamic claim */
    unsigned long long it_l0;       /* BLOCK, lane 0: first item of the claim taken ahead */
    uint64_t static_base;           /* BLOCK: units below are handed out statically */
    uint64_t task_base;             /* units [task_base, task_end) belong to kds */
    uint64_t task_end;
    const kern_data_store *kds;
    const uint8_t *blocks;          /* BLOCK: first heap page of kds */
    const uint8_t *page;            /* BLOCK: current heap page */
    uint32_t row0;                  /* ARROW / ROW: first row of the unit */
    uint32_t item;                  /* next item of the unit */
    uint32_t nitems;                /* items of the unit */
    uint32_t __pad;
    uint32_t grow_buf[4];           /* specialised kernels, lane 0: bytes 48..63 of the
                                     * group table (its 'grow' word), fetched asynchronously */
};

/* chunk owning global unit 'unit' (tasks are sorted by unit_base) */
__device__ __forceinline__ uint32_t
xb_find_task(const xb_task *tasks, uint32_t ntasks, uint64_t unit)
{
    uint32_t lo = 0, hi = ntasks;
    while (hi - lo > 1) {
        uint32_t mid = (lo + hi) >> 1;
        if (tasks[mid].unit_base <= unit) lo = mid; else hi = mid;
    }
    return lo;
}

/* make the chunk owning 'unit' the source's current chunk */
__device__ __forceinline__ void
xb_src_task(const XbExecArgs &args, XbSrc &s, uint64_t unit)
{
    const xb_task &t = args.tasks[xb_find_task(args.tasks, args.ntasks, unit)];
    s.kds = t.kds;
    s.task_base = t.unit_base;
    s.task_end = t.unit_base + t.nunits;
    s.blocks = (args.format == KDS_FORMAT_BLOCK) ? (const uint8_t *)t.kds + t.kds->block_offset : nullptr;
}

/* pull heap page 'unit' into L2 (TMA bulk prefetch); lane 0 issues it */
__device__ __forceinline__ void
xb_prefetch_page(const XbExecArgs &args, const XbSrc &s, uint64_t unit, uint32_t lane)
{
    if (lane != 0 || unit >= args.nunits)
        return;
    const char *p;
    if (unit >= s.task_base && unit < s.task_end) {
        p = (const char *)s.blocks + (unit - s.task_base) * (size_t)PGSTROM_BLCKSZ;
    } else {
        const xb_task &t = args.tasks[xb_find_task(args.tasks, args.ntasks, unit)];
        p = (const char *)t.kds + t.kds->block_offset + (unit - t.unit_base) * (size_t)PGSTROM_BLCKSZ;
    }
    if ((((uintptr_t)p) & 15) == 0)
        xb_prefetch_l2(p, PGSTROM_BLCKSZ);
}

/*
 * Lane 0: the heap-page claim a warp takes after its current one.  A
 * resume launch hands out the stopped launch's leftover ranges first; then
 * pages are claimed from the dynamic cursor with guided sizes (large
 * claims while plenty is left, single pages near the end so that no warp
 * is left with a long tail; one page for a warp's first claim).
 */
__device__ __forceinline__ void
xb_claim_ahead(const XbExecArgs &args, XbSrc &s, bool first)
{
    if (args.resume && args.left_in) {
        const uint32_t i = atomicAdd(&args.st->left_next, 1u);
        if (i < args.left_in_n) {
            const XbLeft L = args.left_in[i];
            s.nx_l0 = L.unit;
            s.sz_l0 = L.unit_end > L.unit ? L.unit_end - L.unit : 0;
            s.it_l0 = L.item;
            return;
        }
    }
    unsigned long long sz = 1;
    if (!first) {
        const unsigned long long warps = (unsigned long long)gridDim.x * (blockDim.x / 32);
        const unsigned long long left = s.last_dyn < args.nunits ? args.nunits - s.last_dyn : 0;
        sz = left / (4 * warps);
        sz = sz < 1 ? 1 : (sz > XB_CLAIM ? XB_CLAIM : sz);
    }
    s.sz_l0 = sz;
    s.it_l0 = 0;
    s.nx_l0 = s.static_base + args.cursor0 + atomicAdd((unsigned long long *)&args.st->unit_cursor, sz);
    s.last_dyn = s.nx_l0;
}

/*
 * Set up a warp's first claim.  Heap pages: each warp first takes a static
 * share of 3/5 of the launch's pages (contiguous, no atomic), then claims
 * the rest dynamically; Arrow / row units are all claimed dynamically.
 */
__device__ __forceinline__ void
xb_src_start(const XbExecArgs &args, XbSrc &s, uint32_t lane)
{
    s.unit = 0;
    s.claim_end = 0;
    s.static_base = 0;
    s.task_base = 0;
    s.task_end = 0;
    s.kds = nullptr;
    s.blocks = nullptr;
    s.page = nullptr;
    s.row0 = 0;
    s.item = 0;
    s.nitems = 0;
    if (args.format != KDS_FORMAT_BLOCK) {
        if (lane == 0) {
            s.nx_l0 = 0;
            s.sz_l0 = 1;
            s.last_dyn = 0;
            s.it_l0 = 0;
        }
        __syncwarp();
        return;
    }
    const uint64_t warps = (uint64_t)gridDim.x * (blockDim.x / 32);
    const uint64_t wid = (uint64_t)blockIdx.x * (blockDim.x / 32) + threadIdx.x / 32;
    const uint64_t share = (args.dyn_only || args.resume) ? 0 : (args.nunits * 3 / 5) / warps;
    s.static_base = args.resume ? args.static_base0 : share * warps;
    /* the lane-0 fields are written by lane 0 only (the state may live in
     * shared memory, read back by every lane) */
    if (lane == 0) {
        s.last_dyn = s.static_base + args.cursor0;
        s.it_l0 = 0;
        if (share > 0) {
            s.nx_l0 = wid * share;
            s.sz_l0 = share;
        } else {
            xb_claim_ahead(args, s, true);
        }
    }
    __syncwarp();
    xb_prefetch_page(args, s, __shfl_sync(XB_FULL, s.nx_l0, 0), lane);
}

/* an Arrow column of the depth-0 loads, resolved once per 1024-row unit
 * for the specialised kernel's fixed-width loads: the unit's first value,
 * the chunk's NULL bitmap (nullptr: none) and how many of the unit's rows
 * have a value inside the buffers (the rest read as NULL, as in
 * xb_arrow_load); ok = 0 sends the column through xb_arrow_load (virtual
 * columns, variable-width and mismatched types) */
struct XbArrowCol {
    const uint8_t *values;
    const uint8_t *nullmap;
    uint32_t nvalid;
    uint32_t ok;
    uint32_t width;                 /* bytes per value (ok columns) */
    uint32_t __pad;
};

/* byte width of the values of an Arrow column read by loader ld when the
 * column's type is the plain fixed-width one the loader expects, else 0 */
__device__ __forceinline__ uint32_t
xb_arrow_fixed_width(const kern_colmeta *cm, int ld)
{
    const int tag = cm->attopts.tag;
    switch (ld) {
    case XB_LD_INT2: case XB_LD_INT4: case XB_LD_INT8: {
        const uint32_t w = ld == XB_LD_INT2 ? 2 : ld == XB_LD_INT4 ? 4 : 8;
        return (tag == ArrowType__Int && cm->attopts.u.integer.bitWidth == w * 8) ? w : 0;
    }
    case XB_LD_FLT8:
        return (tag == ArrowType__FloatingPoint &&
                cm->attopts.u.floating_point.precision == ArrowPrecision__Double) ? 8 : 0;
    case XB_LD_DATE:
        return (tag == ArrowType__Date && cm->attopts.u.date.unit == ArrowDateUnit__Day) ? 4 : 0;
    default:
        return 0;
    }
}

/* lane i resolves depth-0 load i for the unit of rows [row0, row0+nitems) */
__device__ __forceinline__ void
xb_arrow_resolve(const xb_plan *gp, const kern_data_store *kds, uint32_t row0, uint32_t nitems,
                 XbArrowCol *acol, uint32_t lane)
{
    for (uint32_t i = lane; i < gp->nload0; i += 32) {
        const xb_load &l = gp->load0[i];
        XbArrowCol c;
        c.values = nullptr;
        c.nullmap = nullptr;
        c.nvalid = 0;
        c.ok = 0;
        c.width = 0;
        c.__pad = 0;
        if (l.resno < 1 || l.resno > (int)kds->ncols) {
            c.ok = 1;                   /* no such column: every row NULL */
        } else {
            const kern_colmeta *cm = &kds->colmeta[l.resno - 1];
            const uint32_t w = xb_arrow_fixed_width(cm, l.ld);
            if (cm->virtual_offset == 0 && w > 0) {
                uint64_t nv = cm->values_length / w;
                nv = nv > row0 ? nv - row0 : 0;
                if (cm->nullmap_offset) {
                    uint64_t nb = (uint64_t)cm->nullmap_length * 8;
                    nb = nb > row0 ? nb - row0 : 0;
                    nv = nv < nb ? nv : nb;
                    c.nullmap = (const uint8_t *)kds + cm->nullmap_offset;
                }
                c.nvalid = (uint32_t)(nv < nitems ? nv : nitems);
                c.values = (const uint8_t *)kds + cm->values_offset + (uint64_t)row0 * w;
                c.ok = 1;
                c.width = w;
            }
        }
        acol[i] = c;
    }
}

/* lane i: the first XB_ARROW_PF_ROWS rows of an Arrow unit in the column
 * of depth-0 load i, pulled into L2 by the TMA engine (bulk prefetch)
 * when the warp claims the unit (the interpreting kernel; the specialised
 * kernel prefetches a window ahead of every batch instead).  A whole unit
 * per warp would be too much: a launch's warps together would ask for
 * about all of L2, and lines were evicted before their rows were read.
 * Only whole 16-byte pieces inside each column's buffer are prefetched. */
#define XB_ARROW_PF_ROWS    256
__device__ __forceinline__ void
xb_prefetch_arrow_unit(const XbExecArgs &args, const XbSrc &s, uint32_t lane)
{
    const xb_plan *gp = args.plan;
    for (uint32_t i = lane; i < gp->nload0; i += 32) {
        const xb_load &l = gp->load0[i];
        const int w = xb_ld_width(l.ld);
        if (w == 0 || l.ld == XB_LD_BOOL || l.resno < 1 || l.resno > (int)s.kds->ncols)
            continue;
        const kern_colmeta *cm = &s.kds->colmeta[l.resno - 1];
        if (cm->virtual_offset != 0 || cm->values_offset == 0)
            continue;
        const uint32_t nr = s.nitems < XB_ARROW_PF_ROWS ? s.nitems : XB_ARROW_PF_ROWS;
        const uint64_t lo = (uint64_t)s.row0 * w, hi = lo + (uint64_t)nr * w;
        const uint64_t end = hi < cm->values_length ? hi : cm->values_length;
        const uintptr_t a = ((uintptr_t)s.kds + cm->values_offset + lo + 15) & ~(uintptr_t)15;
        const uintptr_t b = ((uintptr_t)s.kds + cm->values_offset + end) & ~(uintptr_t)15;
        if (b > a)
            xb_prefetch_l2((const void *)a, (uint32_t)(b - a));
    }
}

/* the unit this warp takes after its current one (heap pages), or
 * args.nunits when its claims are exhausted */
__device__ __forceinline__ uint64_t xb_following_unit(const XbSrc &s)
{
    return s.unit + 1 < s.claim_end ? s.unit + 1 : __shfl_sync(XB_FULL, s.nx_l0, 0);
}

/* move to the next unit; returns 0 = no more work, 1 = ok, 2 = corrupt page.
 * With pf_next the page after it is prefetched into L2 right away (callers
 * that process a page slowly prefetch it later themselves, closer to use) */
__device__ __forceinline__ int
xb_next_unit(const XbExecArgs &args, XbSrc &s, uint32_t lane, bool pf_next = true)
{
    if (args.format == KDS_FORMAT_BLOCK) {
        s.unit++;
        uint32_t first_item = 0;
        if ((s.unit & 7) == 0 && *(volatile uint32_t *)&args.st->errcode != 0)
            return 0;                   /* another warp failed: stop early */
        if (s.unit >= s.claim_end) {
            /* the claim taken ahead (its atomic has long returned to lane 0) */
            s.unit = __shfl_sync(XB_FULL, s.nx_l0, 0);
            const uint64_t size = __shfl_sync(XB_FULL, s.sz_l0, 0);
            first_item = (uint32_t)__shfl_sync(XB_FULL, s.it_l0, 0);
            if (s.unit >= args.nunits || *(volatile uint32_t *)&args.st->errcode != 0)
                return 0;
            s.claim_end = min(s.unit + size, args.nunits);
            /* lane 0 keeps the next claim until this one is used up */
            if (lane == 0)
                xb_claim_ahead(args, s, false);
        }
        if (s.unit < s.task_base || s.unit >= s.task_end)
            xb_src_task(args, s, s.unit);
        s.page = s.blocks + (s.unit - s.task_base) * (size_t)PGSTROM_BLCKSZ;
        /* the page after this one streams into L2 while this one is decoded */
        if (pf_next)
            xb_prefetch_page(args, s, xb_following_unit(s), lane);
        const uint32_t pd_lower = (uint32_t)xb_fetch_le(s.page + 12, 2);
        s.item = first_item;
        s.nitems = 0;
        if (pd_lower > SizeOfPageHeaderData && pd_lower <= PGSTROM_BLCKSZ)
            s.nitems = (pd_lower - SizeOfPageHeaderData) / sizeof(ItemIdData);
        else if (pd_lower > PGSTROM_BLCKSZ)
            return 2;
        return 1;
    }
    if (*(volatile uint32_t *)&args.st->errcode != 0)
        return 0;
    unsigned long long u = 0;
    uint32_t it = 0;
    if (lane == 0) {
        bool got = false;
        if (args.resume && args.left_in) {
            const uint32_t i = atomicAdd(&args.st->left_next, 1u);
            if (i < args.left_in_n) {
                u = args.left_in[i].unit;
                it = args.left_in[i].item;
                got = true;
            }
        }
        if (!got)
            u = args.cursor0 + atomicAdd((unsigned long long *)&args.st->unit_cursor, 1ULL);
    }
    u = __shfl_sync(XB_FULL, u, 0);
    it = __shfl_sync(XB_FULL, it, 0);
    if (u >= args.nunits)
        return 0;
    if (u < s.task_base || u >= s.task_end)
        xb_src_task(args, s, u);
    s.unit = u;
    s.row0 = (uint32_t)(u - s.task_base) * XB_ROWS_UNIT;
    const uint32_t left = s.kds->nitems > s.row0 ? s.kds->nitems - s.row0 : 0;
    s.nitems = left < XB_ROWS_UNIT ? left : XB_ROWS_UNIT;
    s.item = it;
    if (pf_next && args.format == KDS_FORMAT_ARROW)
        xb_prefetch_arrow_unit(args, s, lane);
    return 1;
}

/*
 * The warp stops claiming work because the group table must grow: lane 0
 * records what the warp still holds, for the resume launch after the host
 * grew the table: the rest of the current unit from next_item on and the
 * rest of the current claim (heap pages: one range), and the claim taken
 * ahead.  Nothing is lost or done twice: every unit is either behind the
 * warp, in these ranges, or not yet claimed from the cursor.
 */
static __device__ __noinline__ void
xb_src_leave(const XbExecArgs &args, const XbSrc &s, uint32_t lane, uint32_t next_item, uint32_t nitems)
{
    if (lane == 0) {
        XbLeft L[2];
        uint32_t n = 0;
        if (args.format == KDS_FORMAT_BLOCK) {
            if (s.unit < s.claim_end) {
                if (next_item < nitems) {
                    L[n].unit = s.unit; L[n].unit_end = s.claim_end; L[n].item = next_item; n++;
                } else if (s.unit + 1 < s.claim_end) {
                    L[n].unit = s.unit + 1; L[n].unit_end = s.claim_end; L[n].item = 0; n++;
                }
            }
            if (s.nx_l0 < args.nunits && s.sz_l0 > 0) {
                L[n].unit = s.nx_l0;
                L[n].unit_end = s.nx_l0 + s.sz_l0 < args.nunits ? s.nx_l0 + s.sz_l0 : args.nunits;
                L[n].item = (uint32_t)s.it_l0;
                n++;
            }
        } else if (s.kds && next_item < nitems) {
            L[n].unit = s.unit; L[n].unit_end = s.unit + 1; L[n].item = next_item; n++;
        }
        atomicExch(&args.st->stopped, 1u);
        if (n) {
            const uint32_t at = atomicAdd(&args.st->left_n, n);
            if (at + n > args.left_cap) {
                XB_RAISE(args.st, ERRCODE_DEVICE_ERROR, XB_MSG_LEFT_FULL);
            } else {
                for (uint32_t i = 0; i < n; i++) {
                    L[i].__pad = 0;
                    args.left_out[at + i] = L[i];
                }
            }
        }
    }
    __syncwarp();
}

/* the warp's view of the group table's growth request (lane 0 loads it) */
__device__ __forceinline__ uint32_t xb_grow_flag(const XbExecArgs &args, uint32_t lane)
{
    return (args.left_out && lane == 0) ? xb_ld_relaxed(&args.gt->grow) : 0u;
}

/* Arrow column -> register (xpu_*_datum_arrow_read) */
__device__ __forceinline__ bool
xb_arrow_load(const kern_data_store *kds, const kern_colmeta *cm, uint32_t row, int ld,
              uint64_t *val, uint32_t *aux, bool *isnull)
{
    if (cm->virtual_offset != 0) {
        if (cm->virtual_offset < 0) { *isnull = true; return true; }
        *isnull = false;
        return xb_load_datum(ld, (const uint8_t *)kds + cm->virtual_offset, val, aux);
    }
    if (cm->nullmap_offset) {
        const uint8_t *nm = (const uint8_t *)kds + cm->nullmap_offset;
        uint32_t b = row >> 3;
        if (b >= cm->nullmap_length || !((nm[b] >> (row & 7)) & 1)) { *isnull = true; return true; }
    }
    const uint8_t *values = (const uint8_t *)kds + cm->values_offset;
    const int tag = cm->attopts.tag;
    *isnull = false;
    *aux = 0;
    switch (ld) {
    case XB_LD_INT2: case XB_LD_INT4: case XB_LD_INT8: {
        uint32_t w = ld == XB_LD_INT2 ? 2 : ld == XB_LD_INT4 ? 4 : 8;
        if (tag != ArrowType__Int || cm->attopts.u.integer.bitWidth != w * 8) return false;
        if ((uint64_t)w * (row + 1) > cm->values_length) { *isnull = true; return true; }
        int64_t v = w == 2 ? (int64_t)((const int16_t *)values)[row]
                  : w == 4 ? (int64_t)((const int32_t *)values)[row]
                           : ((const int64_t *)values)[row];
        *val = (uint64_t)v;
        return true;
    }
    case XB_LD_FLT8:
        if (tag != ArrowType__FloatingPoint || cm->attopts.u.floating_point.precision != ArrowPrecision__Double)
            return false;
        if (8ULL * (row + 1) > cm->values_length) { *isnull = true; return true; }
        *val = ((const uint64_t *)values)[row];
        return true;
    case XB_LD_DATE:
        if (tag != ArrowType__Date) return false;
        if (cm->attopts.u.date.unit == ArrowDateUnit__Day) {
            if (4ULL * (row + 1) > cm->values_length) { *isnull = true; return true; }
            *val = (uint64_t)(int64_t)(int32_t)(((const uint32_t *)values)[row] - 10957u);
        } else {
            if (8ULL * (row + 1) > cm->values_length) { *isnull = true; return true; }
            *val = (uint64_t)(int64_t)(int32_t)(((const uint64_t *)values)[row] / 86400000ULL - 10957ULL);
        }
        return true;
    case XB_LD_BOOL:
        if (tag != ArrowType__Bool) return false;
        if ((row >> 3) >= cm->values_length) { *isnull = true; return true; }
        *val = (values[row >> 3] >> (row & 7)) & 1;
        return true;
    case XB_LD_TEXT: {
        if (tag != ArrowType__Utf8 && tag != ArrowType__Binary && tag != ArrowType__LargeUtf8) return false;
        const uint8_t *extra = (const uint8_t *)kds + cm->extra_offset;
        uint64_t s, e;
        if (tag == ArrowType__LargeUtf8) {
            if (8ULL * (row + 2) > cm->values_length + 8) { *isnull = true; return true; }
            s = ((const uint64_t *)values)[row]; e = ((const uint64_t *)values)[row + 1];
        } else {
            if (4ULL * (row + 2) > cm->values_length + 4) { *isnull = true; return true; }
            s = ((const uint32_t *)values)[row]; e = ((const uint32_t *)values)[row + 1];
        }
        if (s > e || e > cm->extra_length) { *isnull = true; return true; }
        *val = (uint64_t)(extra + s);
        *aux = (uint32_t)(e - s);
        return true;
    }
    default:
        return false;
    }
}


/* ================================================================
 * device projection: rows into a KDS_FORMAT_ROW kds_dst
 * ================================================================ */

/* byte-wise store: tuple attributes follow attalign only, and the trailing
 * row id sits right after a variable-length attribute, so no store into a
 * tuple may assume natural alignment */
__device__ __forceinline__ void xb_store(char *dst, const void *src, uint32_t n)
{
    const char *s = (const char *)src;
    for (uint32_t i = 0; i < n; i++)
        dst[i] = s[i];
}

/*
 * Projected rows are kern_tupitems in the layout of __kern_form_minimal_tuple
 * (xpu_common.cu:1096-1184): a MAXALIGNed header with a NULL bitmap when any
 * attribute is NULL, each non-NULL attribute at its kds_dst column's
 * attalign, text with a 4-byte varlena header, numeric copied as its
 * varlena, and the row id after the last attribute.  The helpers below are
 * called once per attribute with constant ld / attalign by the specialised
 * kernel and from a loop over plan->proj[] by the interpreter.
 */

/* header length (t_hoff, excluding MINIMAL_TUPLE_OFFSET) */
__device__ __forceinline__ uint32_t xb_proj_hoff(uint32_t nattrs, bool hasnull)
{
    return (uint32_t)PGSTROM_MAXALIGN(offsetof(kern_tupitem, t_bits) + (hasnull ? (nattrs + 7) / 8 : 0));
}

/* place attribute (ld, attalign) of value v / aux at offset t of the tuple
 * at base (measure only when base is nullptr); returns the offset after it */
__device__ __forceinline__ uint32_t
xb_proj_attr(char *base, uint32_t t, int attalign, int ld, uint64_t v, uint32_t aux, uint16_t &infomask)
{
    const uint32_t t_next = (uint32_t)PGSTROM_TYPEALIGN(attalign, t);
    char *buf = nullptr;
    if (base) {
        for (uint32_t i = t; i < t_next; i++)
            base[i] = 0;
        buf = base + t_next;
    }
    uint32_t nbytes = 0;
    switch (ld) {
    case XB_LD_BOOL: { const uint8_t x = v ? 1 : 0; nbytes = 1; if (buf) xb_store(buf, &x, 1); break; }
    case XB_LD_INT2: { const int16_t x = (int16_t)v; nbytes = 2; if (buf) xb_store(buf, &x, 2); break; }
    case XB_LD_INT4:
    case XB_LD_DATE: { const int32_t x = (int32_t)v; nbytes = 4; if (buf) xb_store(buf, &x, 4); break; }
    case XB_LD_INT8:
    case XB_LD_FLT8: { nbytes = 8; if (buf) xb_store(buf, &v, 8); break; }
    case XB_LD_TEXT: {
        nbytes = 4 + aux;
        if (buf) {
            const uint32_t hdr = nbytes << 2;               /* SET_VARSIZE */
            xb_store(buf, &hdr, 4);
            xb_store(buf + 4, (const void *)v, aux);
        }
        infomask |= HEAP_HASVARWIDTH;
        break;
    }
    case XB_LD_NUMERIC: {
        const uint8_t *vl = (const uint8_t *)v;
        nbytes = xb_numeric_varsize(vl);
        if (buf) xb_store(buf, vl, nbytes);
        infomask |= HEAP_HASVARWIDTH;
        break;
    }
    default:
        break;
    }
    return t_next + nbytes;
}

/* zero the header and set t_infomask2 / t_hoff / the NULL bitmap */
__device__ __forceinline__ void
xb_proj_head(char *base, uint32_t nattrs, uint32_t hoff, uint32_t nulls)
{
    for (uint32_t i = 0; i < hoff; i++)
        base[i] = 0;
    const uint16_t im2 = (uint16_t)(nattrs & HEAP_NATTS_MASK);
    const uint8_t th = (uint8_t)(hoff + MINIMAL_TUPLE_OFFSET);
    xb_store(base + offsetof(kern_tupitem, t_infomask2), &im2, 2);
    xb_store(base + offsetof(kern_tupitem, t_hoff), &th, 1);
    if (nulls) {
        for (uint32_t j = 0; j < nattrs; j++)
            if (!((nulls >> j) & 1u))
                base[offsetof(kern_tupitem, t_bits) + (j >> 3)] |= (char)(1 << (j & 7));
    }
}

/* t_len, t_infomask and the trailing row id */
__device__ __forceinline__ void
xb_proj_tail(char *base, uint32_t t_len, uint16_t infomask, uint32_t rowid)
{
    xb_store(base + offsetof(kern_tupitem, t_infomask), &infomask, 2);
    xb_store(base, &t_len, 4);
    xb_store(base + t_len - ROWID_SIZE, &rowid, 4);
}

/* kds_dst bytes one row of tuple length t_len takes (the reference's
 * MAXALIGN(MAXALIGN(t_len) + gpusort_htup_margin), cuda_gpujoin.cu:795) */
__device__ __forceinline__ uint32_t xb_proj_rowsz(uint32_t t_len, uint32_t margin)
{
    return (uint32_t)PGSTROM_MAXALIGN(PGSTROM_MAXALIGN(t_len) + margin);
}

/*
 * Claim sz bytes of kds_dst for one row.  Called by the lanes that emit a
 * row, in any divergence: the lanes that arrive together share one claim
 * (the reference instead locks kds_dst->nitems per block,
 * cuda_gpujoin.cu:836-870).  Rows grow from the end of kds_dst, the row
 * index (8-byte offsets from the end) follows the header.
 *
 * The claim first adds its row index and tuple bytes to proj_need; it fits
 * when the sum stays within kds_dst.  proj_need only grows, so the claims
 * that fit are exactly those added before the first one that did not, and
 * together they need at most the buffer: only they then take row slots
 * (proj_nitems) and tuple bytes (proj_usage), so no two of them overlap.
 * Returns the tuple's address and sets *rowid, or returns nullptr (and sets
 * proj_overflow) when the claim does not fit.
 */
__device__ __forceinline__ char *
xb_proj_claim(char *dst, uint64_t dst_len, uint64_t head, uint32_t sz, xb_status *st, uint32_t *rowid)
{
    const uint32_t am = __activemask();
    const uint32_t lane = xb_lane();
    uint32_t incl = sz, total;
    if (am == XB_FULL) {
#pragma unroll
        for (uint32_t o = 1; o < 32; o <<= 1) {
            const uint32_t t = __shfl_up_sync(XB_FULL, incl, o);
            if (lane >= o)
                incl += t;
        }
        total = __shfl_sync(XB_FULL, incl, 31);
    } else {
        incl = 0;
        total = 0;
        for (uint32_t m = am; m; m &= m - 1) {
            const int l = __ffs(m) - 1;
            const uint32_t v = __shfl_sync(am, sz, l);
            total += v;
            if ((uint32_t)l <= lane)
                incl += v;
        }
    }
    const int leader = __ffs(am) - 1;
    const uint32_t count = __popc(am);
    unsigned long long bu = 0;
    uint32_t bn = 0;
    int fits = 0;
    if (lane == (uint32_t)leader) {
        const unsigned long long add = 8ULL * count + total;
        const unsigned long long need = atomicAdd((unsigned long long *)&st->proj_need, add) + add;
        fits = head + need <= dst_len;
        if (fits) {
            bu = atomicAdd((unsigned long long *)&st->proj_usage, (unsigned long long)total);
            bn = atomicAdd(&st->proj_nitems, count);
        } else {
            atomicOr(&st->proj_overflow, 1u);
        }
    }
    fits = __shfl_sync(am, fits, leader);
    if (!fits)
        return nullptr;
    bu = __shfl_sync(am, bu, leader);
    bn = __shfl_sync(am, bn, leader);
    *rowid = bn + __popc(am & ((1u << lane) - 1));
    return dst + dst_len - (bu + incl);
}

/* publish row rowid of the tuple at tp (after the tuple is written) */
__device__ __forceinline__ void
xb_proj_index(char *dst, uint64_t dst_len, uint64_t head, uint32_t rowid, const char *tp)
{
    *(uint64_t *)(dst + head + 8 * (uint64_t)rowid) = (uint64_t)(dst + dst_len - tp);
}

/* interpreter: form and write one row whose attribute j is vals[j] /
 * auxs[j], NULL when bit j of nulls is set.  Into a hashed kds_dst (a
 * pinned inner buffer) the row is a kern_hashitem: its tuple carries the
 * row's hash value and the item is chained into the hash slot
 * (execGpuJoinProjection, cuda_gpujoin.cu:897-915) */
__device__ __forceinline__ void
xb_proj_emit(const xb_plan *plan, char *dst, uint64_t dst_len,
             const uint64_t *vals, const uint32_t *auxs, uint32_t nulls, uint32_t hash, xb_status *st)
{
    const uint32_t n = plan->proj_nattrs;
    const uint32_t hoff = xb_proj_hoff(n, nulls != 0);
    uint16_t im = nulls ? HEAP_HASNULL : 0;
    uint32_t t = hoff;
    for (uint32_t j = 0; j < n; j++)
        if (!((nulls >> j) & 1u))
            t = xb_proj_attr(nullptr, t, plan->proj[j].attalign, plan->proj[j].ld, vals[j], auxs[j], im);
    const uint32_t t_len = t + ROWID_SIZE;
    const uint64_t head = plan->proj_head_len;
    const uint32_t item = plan->proj_hashed ? (uint32_t)offsetof(kern_hashitem, t) : 0;
    uint32_t rowid;
    char *ip = xb_proj_claim(dst, dst_len, head, item + xb_proj_rowsz(t_len, plan->proj_margin), st, &rowid);
    if (!ip)
        return;
    char *tp = ip + item;
    xb_proj_head(tp, n, hoff, nulls);
    if (item)
        xb_store(tp + offsetof(kern_tupitem, hash), &hash, 4);
    t = hoff;
    for (uint32_t j = 0; j < n; j++)
        if (!((nulls >> j) & 1u))
            t = xb_proj_attr(tp, t, plan->proj[j].attalign, plan->proj[j].ld, vals[j], auxs[j], im);
    xb_proj_tail(tp, t_len, im, rowid);
    if (item) {
        uint64_t *slots = (uint64_t *)(dst + head) - plan->proj_nslots;
        const unsigned long long next =
            atomicExch((unsigned long long *)&slots[hash % plan->proj_nslots],
                       (unsigned long long)(dst + dst_len - ip));
        *(uint64_t *)ip = next;
    }
    xb_proj_index(dst, dst_len, head, rowid, tp);
}

/* stage the column layout shared by a launch's chunks and the fixed-offset
 * loaders of the depth-0 loads; all threads of the CTA call this, followed
 * by __syncthreads() */
__device__ __forceinline__ void
xb_setup_meta(const XbExecArgs &args, XbSrcMeta *meta)
{
    const kern_data_store *kds0 = args.tasks[0].kds;
    const int ncols = kds0->ncols < XB_MAX_COLS ? (int)kds0->ncols : XB_MAX_COLS;
    for (int i = threadIdx.x; i < ncols; i += blockDim.x) {
        meta->cols[i].attlen = kds0->colmeta[i].attlen;
        meta->cols[i].attalign = kds0->colmeta[i].attalign > 0 ? kds0->colmeta[i].attalign : 1;
        meta->cols[i].attcacheoff = kds0->colmeta[i].attcacheoff;
    }
    if (threadIdx.x == 0) {
        const xb_plan *gp = args.plan;
        uint32_t fixed = (args.format != KDS_FORMAT_ARROW) ? 1u : 0u, end = 0;
        for (uint32_t i = 0; i < gp->nload0; i++) {
            const xb_load &l = gp->load0[i];
            XbFix f;
            f.off = 0; f.ld = l.ld; f.reg = l.reg; f.__pad = 0;
            if (l.resno < 1 || l.resno > ncols) {
                fixed = 0;
            } else {
                const kern_colmeta &cm = kds0->colmeta[l.resno - 1];
                const int w = xb_ld_width(l.ld);
                /* fixed: a known offset of a naturally aligned datum */
                if (w == 0 || cm.attlen != w || cm.attcacheoff < 0 || (cm.attcacheoff % w) != 0) {
                    fixed = 0;
                } else {
                    f.off = cm.attcacheoff;
                    if ((uint32_t)(cm.attcacheoff + w) > end)
                        end = cm.attcacheoff + w;
                }
            }
            meta->fix[i] = f;
        }
        meta->ncols = ncols;
        meta->fixed = fixed;
        meta->fixed_end = end;
    }
}

#endif  /* XB_EXEC_DEV_CUH */
