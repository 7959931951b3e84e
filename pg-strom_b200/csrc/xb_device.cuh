/*
 * xb_device.cuh
 *
 * Device-side building blocks of the B200 executor:
 *   - the per-warp register file (shared memory, [reg][lane] cells);
 *   - the warp-uniform register VM that runs xb_plan programs;
 *   - PostgreSQL heap tuple and Apache Arrow column decoders;
 *   - group-table insert / lookup / partial-aggregate updates.
 */
#ifndef XB_DEVICE_CUH
#define XB_DEVICE_CUH
#include <stdint.h>
#include "xb_plan.h"
#include "xb_hash.h"

#define XB_FULL         0xffffffffU
#define XB_WAIT_LIMIT   (1u << 22)      /* bounded spin on a BUSY group entry */

/* ---------------------------------------------------------------
 * per-warp register file in shared memory
 * --------------------------------------------------------------- */
struct XbRegs {
    uint64_t   *val;        /* [nregs][32] */
    uint32_t   *aux;        /* [nregs][32] */
    uint32_t   *hc;         /* [nregs][32] hash copied from an inner build */
    uint32_t   *nullm;      /* [nregs]  bit set = NULL */
};

__device__ __forceinline__ uint32_t xb_lane(void)
{
    uint32_t r;
    asm volatile("mov.u32 %0, %%laneid;" : "=r"(r));
    return r;
}

/* bytes of a register file of nregs registers (host and device) */
#define XB_REGS_BYTES(nregs)    (((size_t)(nregs) * (32 * 8 + 32 * 4 + 32 * 4 + 4) + 15) & ~(size_t)15)

__device__ __forceinline__ XbRegs xb_regs_setup(char *base, uint32_t nregs)
{
    XbRegs R;
    R.val = (uint64_t *)base;
    R.aux = (uint32_t *)(base + (size_t)nregs * 256);
    R.hc = (uint32_t *)(base + (size_t)nregs * 384);
    R.nullm = (uint32_t *)(base + (size_t)nregs * 512);
    return R;
}

#define RVAL(R, r)      ((R).val[(r) * 32 + lane])
#define RAUX(R, r)      ((R).aux[(r) * 32 + lane])
#define RHC(R, r)       ((R).hc[(r) * 32 + lane])
#define RISNULL(R, r)   ((((R).nullm[r]) >> lane) & 1u)

/* all lanes call this convergently; writes the NULL ballot of register r.
 * Every lane stores the same (warp-uniform) word, so each lane observes the
 * new value on its next read without a warp barrier; the ballot itself
 * orders this store after every lane's reads of the old value. */
__device__ __forceinline__ void xb_set_null(const XbRegs &R, int r, bool isnull)
{
    const uint32_t m = __ballot_sync(XB_FULL, isnull);
    R.nullm[r] = m;
}

/* rare, register-hungry datum operations kept out of line so that the
 * interpreter loop stays small */
__device__ __noinline__ uint32_t xb_hash_text_ool(const uint8_t *p, uint32_t len)
{
    return xb_hash_bytes(p, len);
}

/* returns the hash, or sets *bad on a corrupt numeric */
__device__ __noinline__ uint32_t xb_hash_numeric_ool(const uint8_t *vl, bool *bad)
{
    uint8_t k; int16_t w; xb_i128 v;
    if (xb_numeric_decode(vl, &k, &w, &v)) {
        *bad = true;
        return 0;
    }
    return xb_hash_numeric(k, w, v);
}

/* hash of a register value of the given hash kind (xpu_*_datum_hash) */
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
 * text helpers
 * --------------------------------------------------------------- */
__device__ __noinline__ bool xb_bytes_eq_ool(const uint8_t *a, const uint8_t *b, uint32_t n);

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

__device__ __noinline__ bool xb_bytes_eq_ool(const uint8_t *a, const uint8_t *b, uint32_t n)
{
    return xb_bytes_eq(a, b, n);
}

__device__ __noinline__ int xb_numeric_cmp(const uint8_t *a, const uint8_t *b, int *err)
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

/* ---------------------------------------------------------------
 * the register VM
 *
 * All 32 lanes execute every instruction (the stream is warp-uniform);
 * 'active' lanes carry a row.  Memory is dereferenced and errors are
 * raised only for active lanes with non-NULL inputs.
 * --------------------------------------------------------------- */
__device__ __forceinline__ bool
xb_vm_exec(const xb_insn *__restrict__ code, uint32_t count, const XbRegs &R,
           uint32_t active_in, xb_status *st)
{
    const uint32_t lane = xb_lane();
    uint32_t active = active_in;
    uint32_t ms0 = 0, ms1 = 0, ms2 = 0, ms3 = 0;   /* lane-mask stack (warp-uniform) */
    int msp = 0;
    bool failed = false;

    xb_insn next = count > 0 ? code[0] : xb_insn();
    for (uint32_t pc = 0; pc < count; pc++) {
        const xb_insn in = next;
        if (pc + 1 < count)
            next = code[pc + 1];            /* overlap the fetch with this op */
        const bool act = ((active >> lane) & 1u) != 0;
        switch (in.op) {
        case XB_OP_END:
            pc = count;
            break;
        case XB_OP_CONST:
            RVAL(R, in.dst) = (uint64_t)in.imm;
            RAUX(R, in.dst) = in.aux;
            xb_set_null(R, in.dst, in.kind != XB_RK_TEXT && in.aux == 1);
            break;
        case XB_OP_MOVE:
            RVAL(R, in.dst) = RVAL(R, in.a);
            RAUX(R, in.dst) = RAUX(R, in.a);
            xb_set_null(R, in.dst, RISNULL(R, in.a));
            break;
        case XB_OP_CMPI: {
            const bool isnull = RISNULL(R, in.a);
            bool res = false;
            if (!isnull) {
                const uint64_t x = RVAL(R, in.a);
                int c;
                if (in.kind == XB_RK_INT) {
                    const int64_t a = (int64_t)x, b = in.imm;
                    c = a < b ? -1 : (a > b ? 1 : 0);
                } else {
                    const double a = __longlong_as_double(x), b = __longlong_as_double(in.imm);
                    const bool na = (a != a), nb = (b != b);
                    c = na ? (nb ? 0 : 1) : (nb ? -1 : (a < b ? -1 : (a > b ? 1 : 0)));
                }
                switch (in.sub) {
                case XB_CMP_EQ: res = (c == 0); break;
                case XB_CMP_NE: res = (c != 0); break;
                case XB_CMP_LT: res = (c < 0); break;
                case XB_CMP_LE: res = (c <= 0); break;
                case XB_CMP_GT: res = (c > 0); break;
                default:        res = (c >= 0); break;
                }
            }
            RVAL(R, in.dst) = res ? 1 : 0;
            xb_set_null(R, in.dst, isnull);
            break;
        }
        case XB_OP_HASH1: {
            uint32_t h = 0xffffffffU;
            if (!RISNULL(R, in.a)) {
                bool bad = false;
                const uint32_t hv = in.sub == XB_HK_CACHED ? RHC(R, in.a)
                                  : xb_hash_reg(in.sub, RVAL(R, in.a), RAUX(R, in.a), act, &bad);
                if (bad) { XB_RAISE(st, ERRCODE_DEVICE_ERROR, XB_MSG_NUMERIC_CORRUPT); failed = true; }
                h = xb_hash_merge(h, hv);
            }
            RVAL(R, in.dst) = h ^ 0xffffffffU;
            xb_set_null(R, in.dst, false);
            break;
        }
        case XB_OP_CMP: {
            bool isnull = RISNULL(R, in.a) || RISNULL(R, in.b);
            bool res = false;
            if (!isnull) {
                uint64_t x = RVAL(R, in.a), y = RVAL(R, in.b);
                int c = 0;
                if (in.kind == XB_RK_INT) {
                    int64_t a = (int64_t)x, b = (int64_t)y;
                    c = a < b ? -1 : (a > b ? 1 : 0);
                } else if (in.kind == XB_RK_FLT) {
                    double a = __longlong_as_double(x), b = __longlong_as_double(y);
                    bool na = (a != a), nb = (b != b);
                    c = na ? (nb ? 0 : 1) : (nb ? -1 : (a < b ? -1 : (a > b ? 1 : 0)));
                } else if (in.kind == XB_RK_TEXT) {
                    uint32_t la = RAUX(R, in.a), lb = RAUX(R, in.b);
                    if (act)
                        c = (la == lb && xb_bytes_eq_ool((const uint8_t *)x, (const uint8_t *)y, la)) ? 0 : 1;
                } else if (in.kind == XB_RK_NUM) {
                    if (act) {
                        int err = 0;
                        c = xb_numeric_cmp((const uint8_t *)x, (const uint8_t *)y, &err);
                        if (err) { XB_RAISE(st, ERRCODE_DEVICE_ERROR, XB_MSG_NUMERIC_CORRUPT); failed = true; }
                    }
                }
                switch (in.sub) {
                case XB_CMP_EQ: res = (c == 0); break;
                case XB_CMP_NE: res = (c != 0); break;
                case XB_CMP_LT: res = (c < 0); break;
                case XB_CMP_LE: res = (c <= 0); break;
                case XB_CMP_GT: res = (c > 0); break;
                default:        res = (c >= 0); break;
                }
            }
            RVAL(R, in.dst) = res ? 1 : 0;
            xb_set_null(R, in.dst, isnull);
            break;
        }
        case XB_OP_ARITH: {
            bool isnull = RISNULL(R, in.a) || RISNULL(R, in.b);
            uint64_t out = 0;
            if (!isnull) {
                uint64_t x = RVAL(R, in.a), y = RVAL(R, in.b);
                int opr = in.sub & 0x0f;
                if (in.kind == XB_RK_INT) {
                    /* operands are int2/int4/int8 values sign-extended to 64 bits;
                     * the result must fit the result type (xpu_basetype.cu:525-720) */
                    const int w = in.sub & 0xf0;
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
                        if (act) { XB_RAISE(st, ERRCODE_DEVICE_ERROR, XB_MSG_DIV_ZERO); failed = true; }
                    } else if (b == -1) {
                        bad = (a == INT64_MIN);
                        r = (int64_t)(0 - (uint64_t)a);
                    } else {
                        r = a / b;
                    }
                    if (w == XB_AR_W2) bad |= (r < -32768 || r > 32767);
                    else if (w == XB_AR_W4) bad |= (r < INT32_MIN || r > INT32_MAX);
                    if (bad && act) { XB_RAISE(st, ERRCODE_DEVICE_ERROR, XB_MSG_INT_RANGE); failed = true; }
                    out = (uint64_t)r;
                } else {
                    double a = __longlong_as_double(x), b = __longlong_as_double(y), r;
                    if (opr == XB_AR_ADD) r = a + b;
                    else if (opr == XB_AR_SUB) r = a - b;
                    else if (opr == XB_AR_MUL) r = a * b;
                    else {
                        if (b == 0.0) {
                            if (act) { XB_RAISE(st, ERRCODE_DEVICE_ERROR, XB_MSG_DIV_ZERO); failed = true; }
                            r = 0.0;
                        } else {
                            r = a / b;
                            if (r == 0.0 && a != 0.0 && act) {
                                XB_RAISE(st, ERRCODE_DEVICE_ERROR, XB_MSG_FLT_RANGE); failed = true;
                            }
                        }
                    }
                    if (isinf(r) && !isinf(a) && !isinf(b) && act) {
                        XB_RAISE(st, ERRCODE_DEVICE_ERROR, XB_MSG_FLT_RANGE); failed = true;
                    }
                    out = (uint64_t)__double_as_longlong(r);
                }
            }
            RVAL(R, in.dst) = out;
            xb_set_null(R, in.dst, isnull);
            break;
        }
        case XB_OP_CAST: {
            bool isnull = RISNULL(R, in.a);
            uint64_t x = RVAL(R, in.a), out = 0;
            if (!isnull) {
                int64_t v = (int64_t)x;
                int64_t lo = INT64_MIN, hi = INT64_MAX;
                bool from_flt = (in.sub == XB_CAST_F82I2 || in.sub == XB_CAST_F82I4 || in.sub == XB_CAST_F82I8);
                if (in.sub == XB_CAST_I2I2 || in.sub == XB_CAST_F82I2) { lo = -32768; hi = 32767; }
                if (in.sub == XB_CAST_I2I4 || in.sub == XB_CAST_F82I4) { lo = INT32_MIN; hi = INT32_MAX; }
                if (in.sub == XB_CAST_I2F8) {
                    out = (uint64_t)__double_as_longlong((double)v);
                } else if (in.sub == XB_CAST_I2BOOL) {
                    out = (v != 0) ? 1 : 0;
                } else if (from_flt) {
                    double d = rint(__longlong_as_double(x));
                    bool ok = (d == d) && d >= (double)lo && d < -(double)lo;
                    if (!ok && act) { XB_RAISE(st, ERRCODE_DEVICE_ERROR, XB_MSG_INT_RANGE); failed = true; }
                    out = ok ? (uint64_t)(int64_t)d : 0;
                } else {
                    if ((v < lo || v > hi) && act) { XB_RAISE(st, ERRCODE_DEVICE_ERROR, XB_MSG_INT_RANGE); failed = true; }
                    out = (uint64_t)v;
                }
            }
            RVAL(R, in.dst) = out;
            xb_set_null(R, in.dst, isnull);
            break;
        }
        case XB_OP_NOT: {
            bool isnull = RISNULL(R, in.a);
            RVAL(R, in.dst) = RVAL(R, in.a) ? 0 : 1;
            xb_set_null(R, in.dst, isnull);
            break;
        }
        case XB_OP_NULLTEST: {
            bool isnull = RISNULL(R, in.a);
            RVAL(R, in.dst) = (in.sub == 0) ? (isnull ? 1 : 0) : (isnull ? 0 : 1);
            xb_set_null(R, in.dst, false);
            break;
        }
        case XB_OP_BOOLTEST: {
            bool isnull = RISNULL(R, in.a);
            bool v = RVAL(R, in.a) != 0;
            bool res;
            switch (in.sub) {
            case 0: res = !isnull && v; break;          /* IS TRUE */
            case 1: res = isnull || !v; break;          /* IS NOT TRUE */
            case 2: res = !isnull && !v; break;         /* IS FALSE */
            case 3: res = isnull || v; break;           /* IS NOT FALSE */
            case 4: res = isnull; break;                /* IS UNKNOWN */
            default: res = !isnull; break;              /* IS NOT UNKNOWN */
            }
            RVAL(R, in.dst) = res ? 1 : 0;
            xb_set_null(R, in.dst, false);
            break;
        }
        case XB_OP_BOOL_INIT:
            RVAL(R, in.dst) = (in.sub == 0) ? 1 : 0;
            xb_set_null(R, in.dst, false);
            break;
        case XB_OP_AND_ACC: {
            /* dst AND a: false dominates, else NULL if any NULL */
            bool dn = RISNULL(R, in.dst), an = RISNULL(R, in.a);
            bool dv = RVAL(R, in.dst) != 0, av = RVAL(R, in.a) != 0;
            bool dfalse = !dn && !dv, afalse = !an && !av;
            bool rv, rn;
            if (dfalse || afalse) { rv = false; rn = false; }
            else { rv = true; rn = dn || an; }
            RVAL(R, in.dst) = rv ? 1 : 0;
            xb_set_null(R, in.dst, rn);
            break;
        }
        case XB_OP_OR_ACC: {
            bool dn = RISNULL(R, in.dst), an = RISNULL(R, in.a);
            bool dv = RVAL(R, in.dst) != 0, av = RVAL(R, in.a) != 0;
            bool dtrue = !dn && dv, atrue = !an && av;
            bool rv, rn;
            if (dtrue || atrue) { rv = true; rn = false; }
            else { rv = false; rn = dn || an; }
            RVAL(R, in.dst) = rv ? 1 : 0;
            xb_set_null(R, in.dst, rn);
            break;
        }
        case XB_OP_MASK_PUSH:
            switch (msp) {
            case 0: ms0 = active; break;
            case 1: ms1 = active; break;
            case 2: ms2 = active; break;
            case 3: ms3 = active; break;
            default: break;                     /* deeper: restored to active_in */
            }
            msp++;
            break;
        case XB_OP_MASK_NARROW: {
            bool an = RISNULL(R, in.a);
            bool av = RVAL(R, in.a) != 0;
            bool drop = (in.sub == 0) ? (!an && !av) : (!an && av);
            active &= ~__ballot_sync(XB_FULL, drop);
            break;
        }
        case XB_OP_MASK_POP:
            msp--;
            switch (msp) {
            case 0: active = ms0; break;
            case 1: active = ms1; break;
            case 2: active = ms2; break;
            case 3: active = ms3; break;
            default: active = active_in; break;
            }
            break;
        case XB_OP_HASH_INIT:
            RVAL(R, in.dst) = 0xffffffffULL;
            xb_set_null(R, in.dst, false);
            break;
        case XB_OP_HASH_ADD: {
            uint32_t h = (uint32_t)RVAL(R, in.dst);
            if (!RISNULL(R, in.a)) {
                bool bad = false;
                const uint32_t hv = in.sub == XB_HK_CACHED ? RHC(R, in.a)
                                  : xb_hash_reg(in.sub, RVAL(R, in.a), RAUX(R, in.a), act, &bad);
                if (bad) { XB_RAISE(st, ERRCODE_DEVICE_ERROR, XB_MSG_NUMERIC_CORRUPT); failed = true; }
                h = xb_hash_merge(h, hv);
            }
            RVAL(R, in.dst) = h;
            break;
        }
        case XB_OP_HASH_FINI:
            RVAL(R, in.dst) = (uint32_t)RVAL(R, in.dst) ^ 0xffffffffU;
            break;
        case XB_OP_DISTINCT: {
            bool an = RISNULL(R, in.a), bn = RISNULL(R, in.b);
            bool res;
            if (an || bn) {
                res = (an != bn);
            } else {
                uint64_t x = RVAL(R, in.a), y = RVAL(R, in.b);
                if (in.kind == XB_RK_TEXT) {
                    uint32_t la = RAUX(R, in.a), lb = RAUX(R, in.b);
                    res = !(act && la == lb && xb_bytes_eq((const uint8_t *)x, (const uint8_t *)y, la));
                } else if (in.kind == XB_RK_FLT) {
                    double a = __longlong_as_double(x), b = __longlong_as_double(y);
                    res = !((a != a && b != b) || a == b);
                } else {
                    res = (x != y);
                }
            }
            RVAL(R, in.dst) = res ? 1 : 0;
            xb_set_null(R, in.dst, false);
            break;
        }
        default:
            if (lane == 0) XB_RAISE(st, ERRCODE_DEVICE_FATAL, XB_MSG_NONE);
            failed = true;
            pc = count;
            break;
        }
    }
    __syncwarp();
    return !__any_sync(XB_FULL, failed);
}

/* out-of-line entry for callers other than the executor's main loop */
__device__ __noinline__ bool
xb_vm_run(const xb_insn *__restrict__ code, uint32_t count, XbRegs R,
          uint32_t active_in, xb_status *st)
{
    return xb_vm_exec(code, count, R, active_in, st);
}

/* ---------------------------------------------------------------
 * attribute loaders (heap datum image -> register), per
 * xpu_*_datum_heap_read: fixed-width values are fetched byte-safely,
 * text keeps (VARDATA_ANY, VARSIZE_ANY_EXHDR), numeric keeps the varlena.
 * --------------------------------------------------------------- */
__device__ __forceinline__ uint64_t xb_fetch_le(const uint8_t *p, int n)
{
    uint64_t v = 0;
    if ((((uintptr_t)p) & (n - 1)) == 0) {
        if (n == 8) return *(const uint64_t *)p;
        if (n == 4) return *(const uint32_t *)p;
        if (n == 2) return *(const uint16_t *)p;
        return *p;
    }
    for (int i = 0; i < n; i++)
        v |= ((uint64_t)p[i]) << (8 * i);
    return v;
}

/* returns false on an unsupported (external/compressed) varlena */
__device__ __forceinline__ bool
xb_load_datum(int ld, const uint8_t *addr, uint64_t *val, uint32_t *aux)
{
    switch (ld) {
    case XB_LD_BOOL: *val = addr[0] ? 1 : 0; *aux = 0; return true;
    case XB_LD_INT2: *val = (uint64_t)(int64_t)(int16_t)xb_fetch_le(addr, 2); *aux = 0; return true;
    case XB_LD_INT4:
    case XB_LD_DATE: *val = (uint64_t)(int64_t)(int32_t)xb_fetch_le(addr, 4); *aux = 0; return true;
    case XB_LD_INT8:
    case XB_LD_FLT8: *val = xb_fetch_le(addr, 8); *aux = 0; return true;
    case XB_LD_FLT4: {
        uint32_t b = (uint32_t)xb_fetch_le(addr, 4);
        *val = (uint64_t)__double_as_longlong((double)__int_as_float((int)b));
        *aux = 0;
        return true;
    }
    case XB_LD_TEXT: {
        uint8_t h = addr[0];
        if (h == 0x01 || (h & 0x03) == 0x02)
            return false;               /* external or compressed */
        if (h & 0x01) {
            if (((h >> 1) & 0x7f) < 1)
                return false;
            *val = (uint64_t)(addr + 1);
            *aux = ((h >> 1) & 0x7f) - 1;
        } else {
            uint32_t len = ((uint32_t)xb_fetch_le(addr, 4) >> 2) & 0x3fffffff;
            if (len < 4)
                return false;
            *val = (uint64_t)(addr + 4);
            *aux = len - 4;
        }
        return true;
    }
    case XB_LD_NUMERIC: {
        uint8_t h = addr[0];
        if (h == 0x01 || (h & 0x03) == 0x02)
            return false;
        *val = (uint64_t)addr;
        *aux = 0;
        return true;
    }
    }
    return false;
}

/* length of an attribute image at addr (attlen > 0: fixed; -1: varlena),
 * or 0 if the header itself does not fit in 'avail' bytes */
__device__ __forceinline__ uint32_t xb_att_size(int attlen, const uint8_t *addr, uint32_t avail)
{
    if (attlen > 0)
        return (uint32_t)attlen;
    if (avail < 1)
        return 0;
    uint8_t h = addr[0];
    if (h == 0x01) {
        if (avail < 2) return 0;
        return 2 + ((addr[1] == 18) ? 16 : (addr[1] == 1 ? 8 : 0));  /* VARSIZE_EXTERNAL */
    }
    if (h & 0x01)
        return (h >> 1) & 0x7f;
    if (avail < 4)
        return 0;
    return ((uint32_t)xb_fetch_le(addr, 4) >> 2) & 0x3fffffff;
}

/* column attributes needed to walk a tuple */
struct XbCol {
    int16_t attlen;
    int8_t  attalign;
    int8_t  __pad;
    int32_t attcacheoff;
};

/*
 * Decode one heap/minimal tuple payload into registers, following
 * __kern_extract_common_tuple (xpu_common.cu:60-130): attcacheoff fast
 * path while the tuple has no NULL bitmap, then the sequential walk with
 * per-attribute alignment (TYPEALIGN unless a non-pad varlena byte) and
 * NULL-bitmap tests.  Attributes beyond the tuple's natts are NULL.
 * Values are written to vals/auxs[dst * stride] where dst is the load's
 * register (by_load_index false: a warp register file) or the load's
 * position (true: SoA columns); bit i of *nullbits is set when load i is
 * NULL.
 * Every access is checked against payload_len; returns false on a corrupt
 * or unsupported (external / compressed) datum.
 */
__device__ __forceinline__ bool
xb_decode_tuple(const XbCol *cols, int ncols, const uint8_t *nullmap,
                const uint8_t *payload, uint32_t payload_len,
                const xb_load *loads, int nloads,
                uint64_t *vals, uint32_t *auxs, uint32_t stride,
                bool by_load_index, uint32_t *nullbits)
{
    int li = 0;
    uint32_t offset = 0;
    int resno = 1;
    uint32_t nb = 0;
    if (!nullmap) {
        while (li < nloads && loads[li].resno <= ncols) {
            const XbCol c = cols[loads[li].resno - 1];
            if (c.attcacheoff < 0)
                break;
            offset = (uint32_t)c.attcacheoff;
            if (offset >= payload_len)
                return false;
            const uint8_t *addr = payload + offset;
            uint32_t sz = xb_att_size(c.attlen, addr, payload_len - offset);
            if (sz == 0 || sz > payload_len - offset)
                return false;
            const uint32_t dst = (by_load_index ? (uint32_t)li : loads[li].reg) * stride;
            if (!xb_load_datum(loads[li].ld, addr, &vals[dst], &auxs[dst]))
                return false;
            resno = loads[li].resno + 1;
            offset += sz;
            li++;
        }
    }
    for (; resno <= ncols && li < nloads; resno++) {
        const XbCol c = cols[resno - 1];
        const uint8_t *addr = nullptr;
        if (!(nullmap && !((nullmap[(resno - 1) >> 3] >> ((resno - 1) & 7)) & 1))) {
            if (c.attlen > 0) {
                offset = (offset + c.attalign - 1) & ~(uint32_t)(c.attalign - 1);
            } else {
                if (offset >= payload_len)
                    return false;
                if (payload[offset] == 0)
                    offset = (offset + c.attalign - 1) & ~(uint32_t)(c.attalign - 1);
            }
            if (offset >= payload_len)
                return false;
            addr = payload + offset;
            uint32_t sz = xb_att_size(c.attlen, addr, payload_len - offset);
            if (sz == 0 || sz > payload_len - offset)
                return false;
            offset += sz;
        }
        if (loads[li].resno == resno) {
            if (!addr) {
                nb |= (1u << li);
            } else {
                const uint32_t dst = (by_load_index ? (uint32_t)li : loads[li].reg) * stride;
                if (!xb_load_datum(loads[li].ld, addr, &vals[dst], &auxs[dst]))
                    return false;
            }
            li++;
        }
    }
    for (; li < nloads; li++)
        nb |= (1u << li);
    *nullbits = nb;
    return true;
}

#endif  /* XB_DEVICE_CUH */
