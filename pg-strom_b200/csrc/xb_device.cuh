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
#include "xb_ops.cuh"

#define XB_FULL         0xffffffffU

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

#ifndef XB_JIT      /* the session-specialised kernels have no interpreter */
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
                const int c = in.kind == XB_RK_INT
                    ? xb_cmp3_int((int64_t)x, in.imm)
                    : xb_cmp3_flt(__longlong_as_double(x), __longlong_as_double(in.imm));
                res = xb_cmp_sub(in.sub, c);
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
            const bool isnull = RISNULL(R, in.a) || RISNULL(R, in.b);
            bool res = false;
            if (!isnull) {
                const int c = xb_cmp3(in.kind, RVAL(R, in.a), RAUX(R, in.a), RVAL(R, in.b), RAUX(R, in.b),
                                      act, st, &failed);
                res = xb_cmp_sub(in.sub, c);
            }
            RVAL(R, in.dst) = res ? 1 : 0;
            xb_set_null(R, in.dst, isnull);
            break;
        }
        case XB_OP_ARITH: {
            const bool isnull = RISNULL(R, in.a) || RISNULL(R, in.b);
            uint64_t out = 0;
            if (!isnull)
                out = in.kind == XB_RK_INT
                    ? xb_arith_int(in.sub, RVAL(R, in.a), RVAL(R, in.b), act, st, &failed)
                    : xb_arith_flt(in.sub, RVAL(R, in.a), RVAL(R, in.b), act, st, &failed);
            RVAL(R, in.dst) = out;
            xb_set_null(R, in.dst, isnull);
            break;
        }
        case XB_OP_CAST: {
            const bool isnull = RISNULL(R, in.a);
            uint64_t out = 0;
            if (!isnull)
                out = xb_cast_op(in.sub, RVAL(R, in.a), act, st, &failed);
            RVAL(R, in.dst) = out;
            xb_set_null(R, in.dst, isnull);
            break;
        }
        case XB_OP_NOT: {
            const bool isnull = RISNULL(R, in.a);
            RVAL(R, in.dst) = RVAL(R, in.a) ? 0 : 1;
            xb_set_null(R, in.dst, isnull);
            break;
        }
        case XB_OP_NULLTEST: {
            const bool isnull = RISNULL(R, in.a);
            RVAL(R, in.dst) = (in.sub == 0) ? (isnull ? 1 : 0) : (isnull ? 0 : 1);
            xb_set_null(R, in.dst, false);
            break;
        }
        case XB_OP_BOOLTEST:
            RVAL(R, in.dst) = xb_booltest(in.sub, RISNULL(R, in.a), RVAL(R, in.a) != 0) ? 1 : 0;
            xb_set_null(R, in.dst, false);
            break;
        case XB_OP_BOOL_INIT:
            RVAL(R, in.dst) = (in.sub == 0) ? 1 : 0;
            xb_set_null(R, in.dst, false);
            break;
        case XB_OP_AND_ACC: {
            bool rn, rv;
            xb_and3(RISNULL(R, in.dst), RVAL(R, in.dst) != 0, RISNULL(R, in.a), RVAL(R, in.a) != 0, &rn, &rv);
            RVAL(R, in.dst) = rv ? 1 : 0;
            xb_set_null(R, in.dst, rn);
            break;
        }
        case XB_OP_OR_ACC: {
            bool rn, rv;
            xb_or3(RISNULL(R, in.dst), RVAL(R, in.dst) != 0, RISNULL(R, in.a), RVAL(R, in.a) != 0, &rn, &rv);
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
        case XB_OP_DISTINCT:
            RVAL(R, in.dst) = xb_distinct(in.kind, RISNULL(R, in.a), RVAL(R, in.a), RAUX(R, in.a),
                                          RISNULL(R, in.b), RVAL(R, in.b), RAUX(R, in.b), act) ? 1 : 0;
            xb_set_null(R, in.dst, false);
            break;
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
static __device__ __noinline__ bool
xb_vm_run(const xb_insn *__restrict__ code, uint32_t count, XbRegs R,
          uint32_t active_in, xb_status *st)
{
    return xb_vm_exec(code, count, R, active_in, st);
}

#endif  /* XB_JIT */

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
