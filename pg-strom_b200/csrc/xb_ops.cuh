/*
 * xb_ops.cuh
 *
 * Per-row semantics of the executor's operations, shared by the
 * interpreter (xb_device.cuh: xb_vm_exec, one op for 32 lanes) and by the
 * session-specialised kernels generated at run time (xb_jit.cpp, every op
 * inlined with constant operands).  Each function computes one lane's
 * result from plain values; NULL handling stays with the caller.
 *
 * Semantics follow the reference's device functions:
 *   comparisons      xpu_basetype.cu / xpu_textlib.cu / xpu_numeric.cu
 *                    (__pg_simple_*, float NaN ordering as float8_cmp_internal)
 *   int arithmetic   xpu_basetype.cu:525-720 (overflow -> error)
 *   float arithmetic xpu_basetype.cu:722-880 (overflow / underflow -> error)
 *   casts            xpu_basetype.cu:60-240
 *   AND / OR         xpu_common.cu:1290-1390 (three-valued logic)
 */
#ifndef XB_OPS_CUH
#define XB_OPS_CUH
#include "xb_plan.h"
#include "xb_hash.h"

/* ---------------------------------------------------------------
 * error reporting (first error wins, as STROM_WRITEBACK_ERROR_STATUS)
 * --------------------------------------------------------------- */
__device__ __forceinline__ void xb_raise(xb_status *st, uint32_t code, uint32_t msg, int line)
{
    if (atomicCAS(&st->errcode, 0u, code) == 0u) {
        st->msg_id = msg;
        st->lineno = line;
    }
}
#define XB_RAISE(st, code, msg) xb_raise((st), (code), (msg), __LINE__)

/* ---------------------------------------------------------------
 * text and numeric helpers
 * --------------------------------------------------------------- */

/* byte-string equality; within a 16-byte block the loads are independent
 * (no early exit), so they are issued back to back instead of as a chain */
__device__ __forceinline__ bool xb_bytes_eq(const uint8_t *a, const uint8_t *b, uint32_t n)
{
    if (a == b)
        return true;
    uint32_t i = 0;
    for (; i + 16 <= n; i += 16) {
        uint32_t diff = 0;
#pragma unroll
        for (uint32_t k = 0; k < 16; k++)
            diff |= (uint32_t)(a[i + k] ^ b[i + k]);
        if (diff)
            return false;
    }
    uint32_t diff = 0;
#pragma unroll
    for (uint32_t k = 0; k < 15; k++)
        if (i + k < n)
            diff |= (uint32_t)(a[i + k] ^ b[i + k]);
    return diff == 0;
}

static __device__ __noinline__ bool xb_bytes_eq_ool(const uint8_t *a, const uint8_t *b, uint32_t n)
{
    return xb_bytes_eq(a, b, n);
}

/* numeric comparison (numeric_cmp); *err on a corrupt varlena */
static __device__ __noinline__ int xb_numeric_cmp(const uint8_t *a, const uint8_t *b, int *err)
{
    uint8_t ka, kb; int16_t wa, wb; xb_i128 va, vb;
    if (xb_numeric_decode(a, &ka, &wa, &va) || xb_numeric_decode(b, &kb, &wb, &vb)) {
        *err = 1;
        return 0;
    }
    /* NaN sorts above +Inf, which sorts above every finite value */
    auto rank = [](uint8_t k) { return k == XB_NUM_NAN ? 3 : k == XB_NUM_PINF ? 2 : k == XB_NUM_NINF ? 0 : 1; };
    int ra = rank(ka), rb = rank(kb);
    if (ra != rb) return ra < rb ? -1 : 1;
    if (ra != 1) return 0;
    int w = wa > wb ? wa : wb;
    va = xb_numeric_rescale(w, wa, va);
    vb = xb_numeric_rescale(w, wb, vb);
    return va < vb ? -1 : (va > vb ? 1 : 0);
}

static __device__ __noinline__ uint32_t xb_hash_text_ool(const uint8_t *p, uint32_t len)
{
    return xb_hash_bytes(p, len);
}

/* returns the hash, or sets *bad on a corrupt numeric */
static __device__ __noinline__ uint32_t xb_hash_numeric_ool(const uint8_t *vl, bool *bad)
{
    uint8_t k; int16_t w; xb_i128 v;
    if (xb_numeric_decode(vl, &k, &w, &v)) {
        *bad = true;
        return 0;
    }
    return xb_hash_numeric(k, w, v);
}

/* hash of a value of the given hash kind (xpu_*_datum_hash) */
__device__ __forceinline__ uint32_t
xb_hash_reg(uint32_t hk, uint64_t x, uint32_t aux, bool act, bool *bad)
{
    switch (hk) {
    case XB_HK_W1: return xb_hash_u32((uint32_t)x, 1);
    case XB_HK_W2: return xb_hash_u32((uint32_t)x, 2);
    case XB_HK_W4: return xb_hash_u32((uint32_t)x, 4);
    case XB_HK_W8: return xb_hash_u64(x);
    case XB_HK_TEXT:
        return act ? xb_hash_text_ool((const uint8_t *)x, aux) : 0;
    case XB_HK_NUM:
        return act ? xb_hash_numeric_ool((const uint8_t *)x, bad) : 0;
    }
    return 0;
}

/* ---------------------------------------------------------------
 * comparisons
 * --------------------------------------------------------------- */
__device__ __forceinline__ int xb_cmp3_int(int64_t a, int64_t b)
{
    return a < b ? -1 : (a > b ? 1 : 0);
}

/* float8_cmp_internal: NaN is equal to NaN and above every other value */
__device__ __forceinline__ int xb_cmp3_flt(double a, double b)
{
    const bool na = (a != a), nb = (b != b);
    return na ? (nb ? 0 : 1) : (nb ? -1 : (a < b ? -1 : (a > b ? 1 : 0)));
}

__device__ __forceinline__ bool xb_cmp_sub(int sub, int c)
{
    switch (sub) {
    case XB_CMP_EQ: return c == 0;
    case XB_CMP_NE: return c != 0;
    case XB_CMP_LT: return c < 0;
    case XB_CMP_LE: return c <= 0;
    case XB_CMP_GT: return c > 0;
    default:        return c >= 0;
    }
}

/* three-way compare of two non-NULL values of register kind 'kind'.  Text
 * values only support equality (text_eq / text_ne: 0 or 1). */
__device__ __forceinline__ int
xb_cmp3(int kind, uint64_t x, uint32_t xa, uint64_t y, uint32_t ya, bool act,
        xb_status *st, bool *failed)
{
    if (kind == XB_RK_INT)
        return xb_cmp3_int((int64_t)x, (int64_t)y);
    if (kind == XB_RK_FLT)
        return xb_cmp3_flt(__longlong_as_double(x), __longlong_as_double(y));
    if (kind == XB_RK_TEXT) {
        if (!act)
            return 0;
        return (xa == ya && xb_bytes_eq_ool((const uint8_t *)x, (const uint8_t *)y, xa)) ? 0 : 1;
    }
    if (kind == XB_RK_NUM) {
        if (!act)
            return 0;
        int err = 0;
        const int c = xb_numeric_cmp((const uint8_t *)x, (const uint8_t *)y, &err);
        if (err) {
            XB_RAISE(st, ERRCODE_DEVICE_ERROR, XB_MSG_NUMERIC_CORRUPT);
            *failed = true;
        }
        return c;
    }
    return 0;
}

/* ---------------------------------------------------------------
 * arithmetic and casts
 * --------------------------------------------------------------- */

/* integer operands are int2/int4/int8 values sign-extended to 64 bits; the
 * result must fit the result width (sub's high nibble) */
__device__ __forceinline__ uint64_t
xb_arith_int(int sub, uint64_t x, uint64_t y, bool act, xb_status *st, bool *failed)
{
    const int opr = sub & 0x0f, w = sub & 0xf0;
    const int64_t a = (int64_t)x, b = (int64_t)y;
    int64_t r = 0;
    bool bad = false;
    if (opr == XB_AR_ADD) {
        r = (int64_t)((uint64_t)a + (uint64_t)b);
        bad = ((a ^ r) & (b ^ r)) < 0;
    } else if (opr == XB_AR_SUB) {
        r = (int64_t)((uint64_t)a - (uint64_t)b);
        bad = ((a ^ b) & (a ^ r)) < 0;
    } else if (opr == XB_AR_MUL) {
        r = (int64_t)((uint64_t)a * (uint64_t)b);
        const int64_t hi = __mul64hi(a, b);
        bad = hi != (r >> 63);
    } else if (b == 0) {
        if (act) {
            XB_RAISE(st, ERRCODE_DEVICE_ERROR, XB_MSG_DIV_ZERO);
            *failed = true;
        }
    } else if (b == -1) {
        bad = (a == INT64_MIN);
        r = (int64_t)(0 - (uint64_t)a);
    } else {
        r = a / b;
    }
    if (w == XB_AR_W2) bad |= (r < -32768 || r > 32767);
    else if (w == XB_AR_W4) bad |= (r < INT32_MIN || r > INT32_MAX);
    if (bad && act) {
        XB_RAISE(st, ERRCODE_DEVICE_ERROR, XB_MSG_INT_RANGE);
        *failed = true;
    }
    return (uint64_t)r;
}

__device__ __forceinline__ uint64_t
xb_arith_flt(int sub, uint64_t x, uint64_t y, bool act, xb_status *st, bool *failed)
{
    const int opr = sub & 0x0f;
    const double a = __longlong_as_double(x), b = __longlong_as_double(y);
    double r;
    if (opr == XB_AR_ADD) r = a + b;
    else if (opr == XB_AR_SUB) r = a - b;
    else if (opr == XB_AR_MUL) r = a * b;
    else {
        if (b == 0.0) {
            if (act) {
                XB_RAISE(st, ERRCODE_DEVICE_ERROR, XB_MSG_DIV_ZERO);
                *failed = true;
            }
            r = 0.0;
        } else {
            r = a / b;
            if (r == 0.0 && a != 0.0 && act) {
                XB_RAISE(st, ERRCODE_DEVICE_ERROR, XB_MSG_FLT_RANGE);
                *failed = true;
            }
        }
    }
    if (isinf(r) && !isinf(a) && !isinf(b) && act) {
        XB_RAISE(st, ERRCODE_DEVICE_ERROR, XB_MSG_FLT_RANGE);
        *failed = true;
    }
    return (uint64_t)__double_as_longlong(r);
}

__device__ __forceinline__ uint64_t
xb_cast_op(int sub, uint64_t x, bool act, xb_status *st, bool *failed)
{
    const int64_t v = (int64_t)x;
    int64_t lo = INT64_MIN, hi = INT64_MAX;
    const bool from_flt = (sub == XB_CAST_F82I2 || sub == XB_CAST_F82I4 || sub == XB_CAST_F82I8);
    if (sub == XB_CAST_I2I2 || sub == XB_CAST_F82I2) { lo = -32768; hi = 32767; }
    if (sub == XB_CAST_I2I4 || sub == XB_CAST_F82I4) { lo = INT32_MIN; hi = INT32_MAX; }
    if (sub == XB_CAST_I2F8)
        return (uint64_t)__double_as_longlong((double)v);
    if (sub == XB_CAST_I2BOOL)
        return (v != 0) ? 1 : 0;
    if (from_flt) {
        const double d = rint(__longlong_as_double(x));
        const bool ok = (d == d) && d >= (double)lo && d < -(double)lo;
        if (!ok && act) {
            XB_RAISE(st, ERRCODE_DEVICE_ERROR, XB_MSG_INT_RANGE);
            *failed = true;
        }
        return ok ? (uint64_t)(int64_t)d : 0;
    }
    if ((v < lo || v > hi) && act) {
        XB_RAISE(st, ERRCODE_DEVICE_ERROR, XB_MSG_INT_RANGE);
        *failed = true;
    }
    return (uint64_t)v;
}

/* ---------------------------------------------------------------
 * boolean logic
 * --------------------------------------------------------------- */

/* IS [NOT] TRUE / FALSE / UNKNOWN */
__device__ __forceinline__ bool xb_booltest(int sub, bool isnull, bool v)
{
    switch (sub) {
    case 0: return !isnull && v;        /* IS TRUE */
    case 1: return isnull || !v;        /* IS NOT TRUE */
    case 2: return !isnull && !v;       /* IS FALSE */
    case 3: return isnull || v;         /* IS NOT FALSE */
    case 4: return isnull;              /* IS UNKNOWN */
    default: return !isnull;            /* IS NOT UNKNOWN */
    }
}

/* d AND a: false dominates, else NULL if any NULL */
__device__ __forceinline__ void xb_and3(bool dn, bool dv, bool an, bool av, bool *rn, bool *rv)
{
    const bool dfalse = !dn && !dv, afalse = !an && !av;
    if (dfalse || afalse) { *rv = false; *rn = false; }
    else { *rv = true; *rn = dn || an; }
}

/* d OR a: true dominates, else NULL if any NULL */
__device__ __forceinline__ void xb_or3(bool dn, bool dv, bool an, bool av, bool *rn, bool *rv)
{
    const bool dtrue = !dn && dv, atrue = !an && av;
    if (dtrue || atrue) { *rv = true; *rn = false; }
    else { *rv = false; *rn = dn || an; }
}

/* a IS DISTINCT FROM b */
__device__ __forceinline__ bool
xb_distinct(int kind, bool an, uint64_t x, uint32_t xa, bool bn, uint64_t y, uint32_t ya, bool act)
{
    if (an || bn)
        return an != bn;
    if (kind == XB_RK_TEXT)
        return !(act && xa == ya && xb_bytes_eq((const uint8_t *)x, (const uint8_t *)y, xa));
    if (kind == XB_RK_FLT) {
        const double a = __longlong_as_double(x), b = __longlong_as_double(y);
        return !((a != a && b != b) || a == b);
    }
    return x != y;
}

#endif  /* XB_OPS_CUH */
