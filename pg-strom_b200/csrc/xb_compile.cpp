/*
 * xb_compile.cpp
 *
 * OpenSession-time translation of PG-Strom's kern_session_info bytecode
 * into the xb_plan register program executed by the B200 kernels.
 *
 * The reference resolves fn_dptr for every node and walks the expression
 * tree per row through indirect calls (gpu_service.c:3115-3317,
 * xpu_common.h:2694 EXEC_KERN_EXPRESSION).  Here every tree is validated
 * once, the way __resolveDevicePointersWalker does (gpu_service.c:3156-3251:
 * length, trailing magic, argument bounds), and lowered into a flat,
 * warp-uniform instruction list.  Per-node semantics follow:
 *   ConstExpr / ParamExpr / VarExpr          xpu_common.cu:390-470
 *   BoolExpr And/Or/Not                      xpu_common.cu:472-551
 *   NullTest / BoolTest / DistinctFrom       xpu_common.cu:553-700
 *   HashValue (seed 0xffffffff, rot-3 merge) xpu_common.cu:1363-1398
 *   SaveExpr                                 xpu_common.cu:1400-1427
 *   JoinQuals (pushed-down quals)            xpu_common.cu:1442-1481
 *   integer / float operators                xpu_basetype.cu:525-760
 *   comparison templates                     xpu_basetype.h:67-138
 * Layout of the emitted bytecode follows codegen.c (:1643-1900,
 * :3149-3700, :3961-4357).
 */
#include <cstdio>
#include <cstring>
#include <cstdarg>
#include <string>
#include <vector>
#include "xb_plan.h"
#include "xb_compile.h"

namespace {

struct Sig { int op; uint8_t vmop; uint8_t sub; uint8_t kind; uint8_t nargs; };

struct Compiler {
    const kern_session_info *session;
    size_t      session_sz;
    uint64_t    dev_session;        /* device address of the session copy */
    xb_plan    *plan;
    int         ntemps;             /* next temporary register */
    int         slot_type[XB_MAX_REGS];
    int         slot_ld[XB_MAX_REGS];
    std::string err;

    bool fail(const char *fmt, ...)
    {
        if (err.empty()) {
            char buf[256];
            va_list ap;
            va_start(ap, fmt);
            vsnprintf(buf, sizeof(buf), fmt, ap);
            va_end(ap);
            err = buf;
        }
        return false;
    }

    /* ---- bytecode access with bounds checks ---- */
    const kern_expression *kexp_at(uint32_t offset)
    {
        if (offset == 0)
            return nullptr;
        if ((uint64_t)offset + KEXP_HEADSZ > session_sz || (offset & 7) != 0) {
            fail("kern_expression offset %u out of the session (%zu bytes)",
                 offset, session_sz);
            return nullptr;
        }
        const kern_expression *kexp =
            (const kern_expression *)((const char *)session + offset);
        if (!check_kexp(kexp, (const char *)session + session_sz))
            return nullptr;
        return kexp;
    }

    bool check_kexp(const kern_expression *kexp, const char *limit)
    {
        const char *base = (const char *)kexp;
        if (base + KEXP_HEADSZ > limit)
            return fail("kern_expression header overruns its container");
        if (kexp->len < KEXP_HEADSZ + sizeof(uint32_t) || base + kexp->len > limit)
            return fail("kern_expression length %u is broken", kexp->len);
        uint32_t magic;
        memcpy(&magic, base + kexp->len - sizeof(uint32_t), sizeof(uint32_t));
        if (magic != KEXP_MAGIC_OF(kexp->exptype, kexp->opcode))
            return fail("kern_expression magic mismatch (opcode=%d)", kexp->opcode);
        if (kexp->nr_args > 0) {
            if (kexp->args_offset < KEXP_HEADSZ || kexp->args_offset > kexp->len)
                return fail("kern_expression args_offset %u is broken", kexp->args_offset);
        }
        return true;
    }

    /* iterate arguments: returns nullptr at the end or on error */
    const kern_expression *first_arg(const kern_expression *kexp)
    {
        if (kexp->nr_args == 0)
            return nullptr;
        const kern_expression *karg =
            (const kern_expression *)((const char *)kexp + kexp->args_offset);
        if (!check_kexp(karg, (const char *)kexp + kexp->len))
            return nullptr;
        return karg;
    }
    const kern_expression *next_arg(const kern_expression *kexp,
                                    const kern_expression *karg)
    {
        const kern_expression *knext = (const kern_expression *)
            ((const char *)karg + PGSTROM_MAXALIGN(karg->len));
        if (!check_kexp(knext, (const char *)kexp + kexp->len))
            return nullptr;
        return knext;
    }

    /* packed sub-expression (xpu_common.h:2953-2968) */
    const kern_expression *packed_at(const kern_expression *kpack, int index)
    {
        if (!kpack)
            return nullptr;
        if (kpack->opcode != FuncOpCode__Packed) {
            fail("expected a Packed expression, got opcode %d", kpack->opcode);
            return nullptr;
        }
        if (index < 0 || (uint32_t)index >= kpack->u.pack.npacked)
            return nullptr;
        size_t off_pos = offsetof(kern_expression, u.pack.offset) + sizeof(uint32_t) * index;
        if (off_pos + sizeof(uint32_t) > kpack->len) {
            fail("Packed offset table overruns the expression");
            return nullptr;
        }
        uint32_t off = kpack->u.pack.offset[index];
        if (off == 0)
            return nullptr;
        if (off < KEXP_HEADSZ || (off & 7) != 0 || off >= kpack->len) {
            fail("Packed sub-expression offset %u is broken", off);
            return nullptr;
        }
        const kern_expression *karg = (const kern_expression *)((const char *)kpack + off);
        if (!check_kexp(karg, (const char *)kpack + kpack->len))
            return nullptr;
        return karg;
    }

    /* ---- code emission ---- */
    int emit(uint8_t op, int dst, int a = 0, int b = 0, int sub = 0,
             int kind = 0, int aux = 0, int64_t imm = 0)
    {
        if (plan->ninsns >= XB_MAX_INSNS) {
            fail("expression program exceeds %d instructions", XB_MAX_INSNS);
            return -1;
        }
        xb_insn *in = &plan->insns[plan->ninsns++];
        in->op = op; in->dst = (uint8_t)dst; in->a = (uint8_t)a; in->b = (uint8_t)b;
        in->sub = (uint8_t)sub; in->kind = (uint8_t)kind; in->aux = (uint16_t)aux;
        in->imm = imm;
        return 0;
    }

    int new_temp(int rk)
    {
        if (ntemps >= XB_MAX_REGS) {
            fail("expression needs more than %d registers", XB_MAX_REGS);
            return -1;
        }
        plan->rk[ntemps] = (uint8_t)rk;
        return ntemps++;
    }

    static bool type_info(int type_code, int *rk, int *ld, int *hk)
    {
        switch (type_code) {
        case TypeOpCode__bool:   *rk = XB_RK_INT;  *ld = XB_LD_BOOL;    *hk = XB_HK_W1; return true;
        case TypeOpCode__int2:   *rk = XB_RK_INT;  *ld = XB_LD_INT2;    *hk = XB_HK_W2; return true;
        case TypeOpCode__int4:   *rk = XB_RK_INT;  *ld = XB_LD_INT4;    *hk = XB_HK_W4; return true;
        case TypeOpCode__int8:   *rk = XB_RK_INT;  *ld = XB_LD_INT8;    *hk = XB_HK_W8; return true;
        case TypeOpCode__float8: *rk = XB_RK_FLT;  *ld = XB_LD_FLT8;    *hk = XB_HK_W8; return true;
        case TypeOpCode__numeric:*rk = XB_RK_NUM;  *ld = XB_LD_NUMERIC; *hk = XB_HK_NUM; return true;
        case TypeOpCode__text:
        case TypeOpCode__bytea:  *rk = XB_RK_TEXT; *ld = XB_LD_TEXT;    *hk = XB_HK_TEXT; return true;
        case TypeOpCode__date:   *rk = XB_RK_INT;  *ld = XB_LD_DATE;    *hk = XB_HK_W4; return true;
        case TypeOpCode__time:
        case TypeOpCode__timestamp:
        case TypeOpCode__timestamptz:
                                 *rk = XB_RK_INT;  *ld = XB_LD_INT8;    *hk = XB_HK_W8; return true;
        default:
            return false;
        }
    }

    /* load a constant datum image (byval bytes or varlena) into a register */
    int emit_const(int type_code, const char *addr, size_t avail, bool isnull)
    {
        int rk, ld, hk;
        if (!type_info(type_code, &rk, &ld, &hk)) {
            fail("constant of type code %d is not supported", type_code);
            return -1;
        }
        int r = new_temp(rk);
        if (r < 0)
            return -1;
        if (isnull) {
            emit(XB_OP_CONST, r, 0, 0, 0, rk, 1, 0);
            return r;
        }
        int64_t imm = 0;
        int aux = 0;
        auto need = [&](size_t n) {
            if (n > avail) { fail("constant datum overruns the session"); return false; }
            return true;
        };
        switch (ld) {
        case XB_LD_BOOL:  if (!need(1)) return -1; imm = (*(const uint8_t *)addr) ? 1 : 0; break;
        case XB_LD_INT2:  { int16_t v; if (!need(2)) return -1; memcpy(&v, addr, 2); imm = v; break; }
        case XB_LD_INT4:
        case XB_LD_DATE:  { int32_t v; if (!need(4)) return -1; memcpy(&v, addr, 4); imm = v; break; }
        case XB_LD_INT8:
        case XB_LD_FLT8:  { if (!need(8)) return -1; memcpy(&imm, addr, 8); break; }
        case XB_LD_TEXT: {
            const uint8_t *p = (const uint8_t *)addr;
            if (!need(1)) return -1;
            uint64_t hdr, len;
            if (VARATT_IS_1B_E(p) || VARATT_IS_4B_C(p)) {
                fail("external or compressed varlena constant");
                return -1;
            }
            if (VARATT_IS_1B(p)) { hdr = 1; len = VARSIZE_1B(p); }
            else { uint32_t h; if (!need(4)) return -1; memcpy(&h, p, 4); hdr = 4; len = (h >> 2) & 0x3fffffff; }
            if (len < hdr || !need(len)) { fail("broken varlena constant"); return -1; }
            if (len - hdr > 0xffff) { fail("text constant longer than 65535 bytes"); return -1; }
            imm = (int64_t)(dev_session + (uint64_t)(addr - (const char *)session) + hdr);
            aux = (int)(len - hdr);
            break;
        }
        case XB_LD_NUMERIC: {
            if (!need(1)) return -1;
            imm = (int64_t)(dev_session + (uint64_t)(addr - (const char *)session));
            break;
        }
        default:
            fail("constant loader %d is not supported", ld);
            return -1;
        }
        emit(XB_OP_CONST, r, 0, 0, 0, rk, aux, imm);
        return r;
    }

    /* true if evaluating kexp can neither raise an error nor dereference
     * memory, so it may run on lanes whose earlier AND/OR argument already
     * decided the result (no lane-mask narrowing needed) */
    bool is_safe(const kern_expression *kexp, int depth = 0)
    {
        if (depth > 16)
            return false;
        switch (kexp->opcode) {
        case FuncOpCode__ConstExpr:
        case FuncOpCode__ParamExpr:
        case FuncOpCode__VarExpr:
            return true;
        case FuncOpCode__NullTestExpr_IsNull:
        case FuncOpCode__NullTestExpr_IsNotNull:
        case FuncOpCode__BoolExpr_Not:
        case FuncOpCode__BoolExpr_And:
        case FuncOpCode__BoolExpr_Or:
            break;
        default: {
            Sig s = {0, 0, 0, 0, 0};
            if (!lookup(kexp->opcode, &s) || s.vmop != XB_OP_CMP ||
                s.kind == XB_RK_TEXT || s.kind == XB_RK_NUM)
                return false;
            break;
        }
        }
        const kern_expression *karg = first_arg(kexp);
        for (uint32_t i = 0; i < kexp->nr_args; i++) {
            if (!karg || !is_safe(karg, depth + 1))
                return false;
            if (i + 1 < kexp->nr_args)
                karg = next_arg(kexp, karg);
        }
        return true;
    }

    /* fixed-width constant operand usable as an immediate */
    bool const_imm(const kern_expression *kexp, int64_t *imm)
    {
        if (kexp->opcode != FuncOpCode__ConstExpr || kexp->u.c.const_isnull)
            return false;
        const char *addr = kexp->u.c.const_value;
        const char *end = (const char *)kexp + kexp->len - sizeof(uint32_t);
        switch (kexp->exptype) {
        case TypeOpCode__int2: { int16_t v; if (end - addr < 2) return false; memcpy(&v, addr, 2); *imm = v; return true; }
        case TypeOpCode__int4:
        case TypeOpCode__date: { int32_t v; if (end - addr < 4) return false; memcpy(&v, addr, 4); *imm = v; return true; }
        case TypeOpCode__int8:
        case TypeOpCode__float8: { if (end - addr < 8) return false; memcpy(imm, addr, 8); return true; }
        default: return false;
        }
    }

    /* ---- expression translation: returns the result register ---- */
    int expr(const kern_expression *kexp)
    {
        if (!kexp)
            return fail("missing expression"), -1;
        switch (kexp->opcode) {
        case FuncOpCode__ConstExpr: {
            const char *addr = kexp->u.c.const_value;
            const char *end = (const char *)kexp + kexp->len - sizeof(uint32_t);
            return emit_const(kexp->exptype, addr, (size_t)(end - addr), kexp->u.c.const_isnull);
        }
        case FuncOpCode__ParamExpr: {
            uint32_t pid = kexp->u.p.param_id;
            if (pid >= session->nparams ||
                offsetof(kern_session_info, poffset) + sizeof(uint32_t) * (pid + 1) > session_sz)
                return emit_const(kexp->exptype, nullptr, 0, true);
            uint32_t off = session->poffset[pid];
            if (off == 0 || off >= session_sz)
                return emit_const(kexp->exptype, nullptr, 0, true);
            return emit_const(kexp->exptype, (const char *)session + off, session_sz - off, false);
        }
        case FuncOpCode__VarExpr: {
            int slot = kexp->u.v.var_slot_id;
            if (slot < 0 || slot >= (int)plan->nslots)
                return fail("VarExpr slot %d out of range", slot), -1;
            if (slot_type[slot] != kexp->exptype)
                return fail("VarExpr type %d mismatches slot %d type %d",
                            kexp->exptype, slot, slot_type[slot]), -1;
            return slot;
        }
        case FuncOpCode__BoolExpr_And:
        case FuncOpCode__BoolExpr_Or: {
            bool is_and = (kexp->opcode == FuncOpCode__BoolExpr_And);
            if (kexp->exptype != TypeOpCode__bool || kexp->nr_args < 1)
                return fail("malformed BoolExpr"), -1;
            int t = new_temp(XB_RK_INT);
            if (t < 0) return -1;
            const bool masked = !is_safe(kexp);
            emit(XB_OP_BOOL_INIT, t, 0, 0, is_and ? 0 : 1);
            if (masked)
                emit(XB_OP_MASK_PUSH, 0);
            const kern_expression *karg = first_arg(kexp);
            for (uint32_t i = 0; i < kexp->nr_args; i++) {
                if (!karg) return fail("BoolExpr argument %u is broken", i), -1;
                if (karg->exptype != TypeOpCode__bool)
                    return fail("BoolExpr argument is not bool"), -1;
                int r = expr(karg);
                if (r < 0) return -1;
                emit(is_and ? XB_OP_AND_ACC : XB_OP_OR_ACC, t, r);
                if (i + 1 < kexp->nr_args) {
                    if (masked)
                        emit(XB_OP_MASK_NARROW, 0, r, 0, is_and ? 0 : 1);
                    karg = next_arg(kexp, karg);
                }
            }
            if (masked)
                emit(XB_OP_MASK_POP, 0);
            return t;
        }
        case FuncOpCode__BoolExpr_Not: {
            if (kexp->nr_args != 1) return fail("malformed BoolExpr_Not"), -1;
            int r = expr(first_arg(kexp));
            if (r < 0) return -1;
            int t = new_temp(XB_RK_INT);
            if (t < 0) return -1;
            emit(XB_OP_NOT, t, r);
            return t;
        }
        case FuncOpCode__NullTestExpr_IsNull:
        case FuncOpCode__NullTestExpr_IsNotNull: {
            if (kexp->nr_args != 1) return fail("malformed NullTestExpr"), -1;
            int r = expr(first_arg(kexp));
            if (r < 0) return -1;
            int t = new_temp(XB_RK_INT);
            if (t < 0) return -1;
            emit(XB_OP_NULLTEST, t, r, 0,
                 kexp->opcode == FuncOpCode__NullTestExpr_IsNull ? 0 : 1);
            return t;
        }
        case FuncOpCode__BoolTestExpr_IsTrue:
        case FuncOpCode__BoolTestExpr_IsNotTrue:
        case FuncOpCode__BoolTestExpr_IsFalse:
        case FuncOpCode__BoolTestExpr_IsNotFalse:
        case FuncOpCode__BoolTestExpr_IsUnknown:
        case FuncOpCode__BoolTestExpr_IsNotUnknown: {
            if (kexp->nr_args != 1) return fail("malformed BoolTestExpr"), -1;
            int r = expr(first_arg(kexp));
            if (r < 0) return -1;
            int t = new_temp(XB_RK_INT);
            if (t < 0) return -1;
            emit(XB_OP_BOOLTEST, t, r, 0, kexp->opcode - FuncOpCode__BoolTestExpr_IsTrue);
            return t;
        }
        case FuncOpCode__SaveExpr: {
            if (kexp->nr_args != 1) return fail("malformed SaveExpr"), -1;
            int slot = kexp->u.save.sv_slot_id;
            if (slot < 0 || slot >= (int)plan->nslots)
                return fail("SaveExpr slot %d out of range", slot), -1;
            const kern_expression *karg = first_arg(kexp);
            if (!karg) return fail("SaveExpr argument is broken"), -1;
            if (karg->exptype != kexp->exptype || slot_type[slot] != kexp->exptype)
                return fail("SaveExpr type mismatch"), -1;
            int r = expr(karg);
            if (r < 0) return -1;
            if (r != slot)
                emit(XB_OP_MOVE, slot, r);
            return slot;
        }
        case FuncOpCode__HashValue: {
            if (kexp->nr_args == 1) {
                const kern_expression *karg = first_arg(kexp);
                int rk, ld, hk;
                if (!karg) return fail("HashValue argument is broken"), -1;
                if (!type_info(karg->exptype, &rk, &ld, &hk))
                    return fail("HashValue on unsupported type %d", karg->exptype), -1;
                int r = expr(karg);
                if (r < 0) return -1;
                int t1 = new_temp(XB_RK_INT);
                if (t1 < 0) return -1;
                emit(XB_OP_HASH1, t1, r, 0, hk, rk);
                return t1;
            }
            int t = new_temp(XB_RK_INT);
            if (t < 0) return -1;
            emit(XB_OP_HASH_INIT, t);
            const kern_expression *karg = first_arg(kexp);
            for (uint32_t i = 0; i < kexp->nr_args; i++) {
                if (!karg) return fail("HashValue argument %u is broken", i), -1;
                int rk, ld, hk;
                if (!type_info(karg->exptype, &rk, &ld, &hk))
                    return fail("HashValue on unsupported type %d", karg->exptype), -1;
                int r = expr(karg);
                if (r < 0) return -1;
                emit(XB_OP_HASH_ADD, t, r, 0, hk, rk);
                if (i + 1 < kexp->nr_args)
                    karg = next_arg(kexp, karg);
            }
            emit(XB_OP_HASH_FINI, t);
            return t;
        }
        case FuncOpCode__DistinctFrom: {
            if (kexp->nr_args != 2) return fail("malformed DistinctFrom"), -1;
            const kern_expression *k1 = first_arg(kexp);
            const kern_expression *k2 = k1 ? next_arg(kexp, k1) : nullptr;
            if (!k1 || !k2) return fail("DistinctFrom arguments are broken"), -1;
            int rk1, rk2, ld, hk;
            if (!type_info(k1->exptype, &rk1, &ld, &hk) || !type_info(k2->exptype, &rk2, &ld, &hk) ||
                rk1 != rk2 || rk1 == XB_RK_NUM)
                return fail("DistinctFrom on unsupported types"), -1;
            int a = expr(k1); if (a < 0) return -1;
            int b = expr(k2); if (b < 0) return -1;
            int t = new_temp(XB_RK_INT);
            if (t < 0) return -1;
            emit(XB_OP_DISTINCT, t, a, b, 0, rk1);
            return t;
        }
        default:
            return func(kexp);
        }
    }

    /* built-in operator / function opcodes */
    int func(const kern_expression *kexp)
    {
        int op = kexp->opcode;
        Sig s = {0, 0, 0, 0, 0};
        if (!lookup(op, &s))
            return fail("device function opcode %d is not supported", op), -1;
        if ((int)kexp->nr_args != s.nargs)
            return fail("opcode %d expects %d arguments", op, s.nargs), -1;
        int regs[2] = {0, 0};
        const kern_expression *karg = first_arg(kexp);
        if (s.vmop == XB_OP_CMP && (s.kind == XB_RK_INT || s.kind == XB_RK_FLT) && s.nargs == 2 && karg) {
            const kern_expression *k2 = next_arg(kexp, karg);
            int64_t imm;
            if (k2 && const_imm(k2, &imm)) {
                int a = expr(karg);
                if (a < 0) return -1;
                int t = new_temp(XB_RK_INT);
                if (t < 0) return -1;
                emit(XB_OP_CMPI, t, a, 0, s.sub, s.kind, 0, imm);
                return t;
            }
        }
        for (int i = 0; i < s.nargs; i++) {
            if (!karg) return fail("argument %d of opcode %d is broken", i, op), -1;
            regs[i] = expr(karg);
            if (regs[i] < 0) return -1;
            if (i + 1 < s.nargs)
                karg = next_arg(kexp, karg);
        }
        int rk, ld, hk;
        if (!type_info(kexp->exptype, &rk, &ld, &hk))
            return fail("result type %d of opcode %d is not supported", kexp->exptype, op), -1;
        int t = new_temp(rk);
        if (t < 0) return -1;
        emit(s.vmop, t, regs[0], regs[1], s.sub, s.kind);
        return t;
    }

    template <typename S>
    static bool lookup(int op, S *s)
    {
        /* integer binary operators: int{2,4,8}x{2,4,8} {pl,mi,mul,div,eq,...} */
        static const struct { int code; int res_w; } *none = nullptr; (void)none;
#define ARITH(CODE, W, SUB) case FuncOpCode__##CODE: s->op = op; s->vmop = XB_OP_ARITH; \
        s->sub = (uint8_t)((SUB) | (W)); s->kind = XB_RK_INT; s->nargs = 2; return true;
#define ICMP(CODE, SUB) case FuncOpCode__##CODE: s->op = op; s->vmop = XB_OP_CMP; \
        s->sub = SUB; s->kind = XB_RK_INT; s->nargs = 2; return true;
#define FCMP(CODE, SUB) case FuncOpCode__##CODE: s->op = op; s->vmop = XB_OP_CMP; \
        s->sub = SUB; s->kind = XB_RK_FLT; s->nargs = 2; return true;
#define NCMP(CODE, SUB) case FuncOpCode__##CODE: s->op = op; s->vmop = XB_OP_CMP; \
        s->sub = SUB; s->kind = XB_RK_NUM; s->nargs = 2; return true;
#define TCMP(CODE, SUB) case FuncOpCode__##CODE: s->op = op; s->vmop = XB_OP_CMP; \
        s->sub = SUB; s->kind = XB_RK_TEXT; s->nargs = 2; return true;
#define FARITH(CODE, SUB) case FuncOpCode__##CODE: s->op = op; s->vmop = XB_OP_ARITH; \
        s->sub = SUB; s->kind = XB_RK_FLT; s->nargs = 2; return true;
#define CAST(CODE, SUB) case FuncOpCode__##CODE: s->op = op; s->vmop = XB_OP_CAST; \
        s->sub = SUB; s->kind = 0; s->nargs = 1; return true;
#define INT_FAMILY(PFX, W) \
        ARITH(PFX##pl, W, XB_AR_ADD) ARITH(PFX##mi, W, XB_AR_SUB) \
        ARITH(PFX##mul, W, XB_AR_MUL) ARITH(PFX##div, W, XB_AR_DIV) \
        ICMP(PFX##eq, XB_CMP_EQ) ICMP(PFX##ne, XB_CMP_NE) ICMP(PFX##lt, XB_CMP_LT) \
        ICMP(PFX##le, XB_CMP_LE) ICMP(PFX##gt, XB_CMP_GT) ICMP(PFX##ge, XB_CMP_GE)
        switch (op) {
        INT_FAMILY(int2, XB_AR_W2)
        INT_FAMILY(int24, XB_AR_W4)
        INT_FAMILY(int28, XB_AR_W8)
        INT_FAMILY(int42, XB_AR_W4)
        INT_FAMILY(int4, XB_AR_W4)
        INT_FAMILY(int48, XB_AR_W8)
        INT_FAMILY(int82, XB_AR_W8)
        INT_FAMILY(int84, XB_AR_W8)
        INT_FAMILY(int8, XB_AR_W8)
        FARITH(float8pl, XB_AR_ADD) FARITH(float8mi, XB_AR_SUB)
        FARITH(float8mul, XB_AR_MUL) FARITH(float8div, XB_AR_DIV)
        FCMP(float8eq, XB_CMP_EQ) FCMP(float8ne, XB_CMP_NE) FCMP(float8lt, XB_CMP_LT)
        FCMP(float8le, XB_CMP_LE) FCMP(float8gt, XB_CMP_GT) FCMP(float8ge, XB_CMP_GE)
        ICMP(date_eq, XB_CMP_EQ) ICMP(date_ne, XB_CMP_NE) ICMP(date_lt, XB_CMP_LT)
        ICMP(date_le, XB_CMP_LE) ICMP(date_gt, XB_CMP_GT) ICMP(date_ge, XB_CMP_GE)
        NCMP(numeric_eq, XB_CMP_EQ) NCMP(numeric_ne, XB_CMP_NE) NCMP(numeric_lt, XB_CMP_LT)
        NCMP(numeric_le, XB_CMP_LE) NCMP(numeric_gt, XB_CMP_GT) NCMP(numeric_ge, XB_CMP_GE)
        TCMP(text_eq, XB_CMP_EQ) TCMP(text_ne, XB_CMP_NE)
        CAST(int2_to_int4, XB_CAST_I2I4) CAST(int2_to_int8, XB_CAST_I2I8)
        CAST(int4_to_int2, XB_CAST_I2I2) CAST(int4_to_int8, XB_CAST_I2I8)
        CAST(int8_to_int2, XB_CAST_I2I2) CAST(int8_to_int4, XB_CAST_I2I4)
        CAST(int2_to_float8, XB_CAST_I2F8) CAST(int4_to_float8, XB_CAST_I2F8)
        CAST(int8_to_float8, XB_CAST_I2F8)
        CAST(float8_to_int2, XB_CAST_F82I2) CAST(float8_to_int4, XB_CAST_F82I4)
        CAST(float8_to_int8, XB_CAST_F82I8)
        CAST(int4_to_bool, XB_CAST_I2BOOL)
        default:
            return false;
        }
#undef ARITH
#undef ICMP
#undef FCMP
#undef NCMP
#undef TCMP
#undef FARITH
#undef CAST
#undef INT_FAMILY
    }

    /* compile one top-level expression into a program */
    bool program(const kern_expression *kexp, xb_prog *prog, bool want_bool)
    {
        prog->start = (uint16_t)plan->ninsns;
        prog->count = 0;
        prog->result = -1;
        if (!kexp)
            return true;
        if (want_bool && kexp->exptype != TypeOpCode__bool)
            return fail("qualifier is not a bool expression");
        ntemps = plan->nslots;
        int r = expr(kexp);
        if (r < 0)
            return false;
        prog->count = (uint16_t)(plan->ninsns - prog->start);
        prog->result = (int16_t)r;
        if ((uint32_t)ntemps > plan->nregs)
            plan->nregs = ntemps;
        return err.empty();
    }

    /* JoinQuals: every argument must hold for an inner join.  Argument
     * 'skip' (if >= 0) is evaluated by the fused probe instead. */
    bool join_program(const kern_expression *kexp, xb_prog *prog, int skip = -1)
    {
        prog->start = (uint16_t)plan->ninsns;
        prog->count = 0;
        prog->result = -1;
        if (!kexp)
            return true;
        if (kexp->opcode != FuncOpCode__JoinQuals || kexp->exptype != TypeOpCode__bool)
            return fail("malformed JoinQuals");
        ntemps = plan->nslots;
        /* the arguments that remain for the VM */
        std::vector<const kern_expression *> args;
        {
            const kern_expression *k = first_arg(kexp);
            for (uint32_t i = 0; i < kexp->nr_args; i++) {
                if (!k) return fail("JoinQuals argument %u is broken", i);
                if (k->exptype != TypeOpCode__bool)
                    return fail("JoinQuals argument is not bool");
                if ((int)i != skip)
                    args.push_back(k);
                if (i + 1 < kexp->nr_args)
                    k = next_arg(kexp, k);
            }
        }
        if (args.empty())
            return err.empty();         /* everything done by the fused probe */
        if (args.size() == 1) {
            const kern_expression *k1 = args[0];
            int r = expr(k1);
            if (r < 0) return false;
            prog->count = (uint16_t)(plan->ninsns - prog->start);
            prog->result = (int16_t)r;
            if ((uint32_t)ntemps > plan->nregs)
                plan->nregs = ntemps;
            return err.empty();
        }
        bool masked = false;
        for (const kern_expression *k : args)
            if (!is_safe(k)) masked = true;
        int t = new_temp(XB_RK_INT);
        if (t < 0) return false;
        emit(XB_OP_BOOL_INIT, t, 0, 0, 0);
        if (masked)
            emit(XB_OP_MASK_PUSH, 0);
        for (size_t i = 0; i < args.size(); i++) {
            int r = expr(args[i]);
            if (r < 0) return false;
            emit(XB_OP_AND_ACC, t, r);
            if (i + 1 < args.size() && masked)
                emit(XB_OP_MASK_NARROW, 0, r, 0, 0);
        }
        if (masked)
            emit(XB_OP_MASK_POP, 0);
        prog->count = (uint16_t)(plan->ninsns - prog->start);
        prog->result = (int16_t)t;
        if ((uint32_t)ntemps > plan->nregs)
            plan->nregs = ntemps;
        return err.empty();
    }

    /* sequence of SaveExpr (AggFuncs arguments) */
    bool save_program(const kern_expression *kexp, xb_prog *prog)
    {
        prog->start = (uint16_t)plan->ninsns;
        prog->count = 0;
        prog->result = -1;
        ntemps = plan->nslots;
        const kern_expression *karg = first_arg(kexp);
        for (uint32_t i = 0; i < kexp->nr_args; i++) {
            if (!karg) return fail("AggFuncs argument %u is broken", i);
            if (karg->opcode != FuncOpCode__SaveExpr)
                return fail("AggFuncs argument is not a SaveExpr");
            if (expr(karg) < 0)
                return false;
            if (i + 1 < kexp->nr_args)
                karg = next_arg(kexp, karg);
        }
        prog->count = (uint16_t)(plan->ninsns - prog->start);
        if ((uint32_t)ntemps > plan->nregs)
            plan->nregs = ntemps;
        return err.empty();
    }

    /*
     * Device projection (codegen_build_projection, codegen.c:3880-3950):
     * the Projection expression's arguments are VarExpr (the slot already
     * holds the value) or SaveExpr (compute into a slot); u.proj.slot_id[]
     * names the slot of every output attribute, and the session's
     * projection_kds_dst is the KDS_FORMAT_ROW header rows are written to.
     */
    bool projection()
    {
        plan->has_proj = 0;
        if (!session->xpucode_projection)
            return true;
        const kern_expression *kp = kexp_at(session->xpucode_projection);
        if (!err.empty()) return false;
        if (!kp || kp->opcode != FuncOpCode__Projection)
            return fail("malformed Projection expression");
        const int nattrs = kp->u.proj.nattrs;
        if (nattrs < 1 || nattrs > XB_MAX_PROJ ||
            offsetof(kern_expression, u.proj.slot_id) + sizeof(uint16_t) * nattrs > kp->len)
            return fail("Projection has %d attributes (max %d)", nattrs, XB_MAX_PROJ);
        /* argument programs: SaveExpr into slots; VarExpr needs nothing */
        plan->proj_args.start = (uint16_t)plan->ninsns;
        plan->proj_args.count = 0;
        plan->proj_args.result = -1;
        ntemps = plan->nslots;
        const kern_expression *karg = first_arg(kp);
        for (uint32_t i = 0; i < kp->nr_args; i++) {
            if (!karg) return fail("Projection argument %u is broken", i);
            if (karg->opcode == FuncOpCode__SaveExpr) {
                if (expr(karg) < 0)
                    return false;
            } else if (karg->opcode != FuncOpCode__VarExpr) {
                return fail("Projection argument %u is neither VarExpr nor SaveExpr", i);
            }
            if (i + 1 < kp->nr_args)
                karg = next_arg(kp, karg);
        }
        plan->proj_args.count = (uint16_t)(plan->ninsns - plan->proj_args.start);
        /* the hash value of a row bound for a pinned inner buffer
         * (execGpuJoinProjection, cuda_gpujoin.cu:797-823) */
        plan->proj_hashed = 0;
        if (kp->u.proj.hash != 0) {
            const kern_expression *kh = (const kern_expression *)((const char *)kp + kp->u.proj.hash);
            if (kp->u.proj.hash + offsetof(kern_expression, u) > kp->len || kh->len < offsetof(kern_expression, u) ||
                kp->u.proj.hash + kh->len > kp->len || kh->opcode != FuncOpCode__HashValue)
                return fail("malformed Projection hash value");
            if (!program(kh, &plan->proj_hash, false))
                return false;
            plan->proj_hashed = 1;
        }
        plan->proj_all.start = plan->proj_args.start;
        plan->proj_all.count = (uint16_t)(plan->ninsns - plan->proj_args.start);
        plan->proj_all.result = -1;
        if ((uint32_t)ntemps > plan->nregs)
            plan->nregs = ntemps;
        /* the destination header */
        const uint64_t off = session->projection_kds_dst;
        if (off == 0 || off + sizeof(kern_data_store) > session_sz)
            return fail("projection without a kds_dst header");
        const kern_data_store *kd = (const kern_data_store *)((const char *)session + off);
        if (kd->format != (plan->proj_hashed ? KDS_FORMAT_HASH : KDS_FORMAT_ROW))
            return fail("projection into KDS format '%c' is not supported%s", kd->format,
                        plan->proj_hashed ? " (a hashed projection writes KDS_FORMAT_HASH)" : "");
        const uint64_t hl = KDS_HEAD_LENGTH(kd);
        if (off + hl > session_sz || (plan->proj_hashed ? kd->hash_nslots == 0 : kd->hash_nslots != 0))
            return fail("projection kds_dst header is broken");
        plan->proj_nslots = kd->hash_nslots;
        /* attributes past kds_dst's columns are not written (as in
         * __kern_form_minimal_tuple, xpu_common.cu:1113-1114) */
        const int nout = (int)kd->ncols < nattrs ? (int)kd->ncols : nattrs;
        if (nout < 1)
            return fail("projection kds_dst has no columns");
        for (int j = 0; j < nout; j++) {
            const int slot = kp->u.proj.slot_id[j];
            if (slot < 0 || slot >= (int)plan->nslots)
                return fail("projected slot %d out of range", slot);
            const kern_colmeta &cm = kd->colmeta[j];
            xb_projcol &pc = plan->proj[j];
            pc.reg = (uint8_t)slot;
            pc.ld = (uint8_t)slot_ld[slot];
            pc.attlen = cm.attlen;
            pc.attalign = cm.attalign > 0 ? cm.attalign : 1;
            int w = 0;
            switch (pc.ld) {
            case XB_LD_BOOL: w = 1; break;
            case XB_LD_INT2: w = 2; break;
            case XB_LD_INT4: case XB_LD_DATE: case XB_LD_FLT4: w = 4; break;
            case XB_LD_INT8: case XB_LD_FLT8: w = 8; break;
            default: w = -1; break;
            }
            if (pc.attlen != w)
                return fail("projected attribute %d: column length %d does not fit its value", j, pc.attlen);
        }
        plan->proj_nattrs = (uint32_t)nout;
        plan->proj_margin = session->gpusort_htup_margin;
        /* a hashed kds_dst keeps its hash slots between the header and the
         * row index */
        plan->proj_head_len = (uint32_t)(hl + (plan->proj_hashed ? 8ULL * kd->hash_nslots : 0));
        plan->has_proj = 1;
        return true;
    }

    /* GPU-Sort of the final groups (kern_gpusort_prep_buffer and the
     * comparators of cuda_gpusort.cu:15-400): each key becomes one or two
     * order-preserving 64-bit words computed from the group entry */
    bool gpusort()
    {
        plan->nsort = 0;
        plan->sort_window = 0;
        plan->sort_limit = 0;
        if (!session->xpucode_gpusort_keydesc)
            return true;
        if (!plan->has_groupby)
            return fail("GPU-Sort without GROUP BY is not supported");
        const kern_expression *ks = kexp_at(session->xpucode_gpusort_keydesc);
        if (!err.empty()) return false;
        if (!ks || ks->opcode != FuncOpCode__SortKeys)
            return fail("malformed SortKeys expression");
        const int nkeys = ks->u.sort.nkeys;
        if (nkeys < 1 || nkeys > XB_MAX_SORTKEYS ||
            offsetof(kern_expression, u.sort.desc) + sizeof(kern_sortkey_desc) * (size_t)nkeys > ks->len)
            return fail("SortKeys has %d keys (1..%d)", nkeys, XB_MAX_SORTKEYS);
        for (int i = 0; i < nkeys; i++) {
            const kern_sortkey_desc &d = ks->u.sort.desc[i];
            if (d.src_anum < 1 || d.src_anum > plan->naggs)
                return fail("sort key %d: attribute %u out of range", i, d.src_anum);
            const xb_agg &a = plan->aggs[d.src_anum - 1];
            xb_sortkey &k = plan->sort[i];
            k.kind = d.kind;
            k.agg = (uint16_t)(d.src_anum - 1);
            k.asc = d.order_asc ? 1 : 0;
            k.nulls_first = d.nulls_first ? 1 : 0;
            k.words = 1;
            bool ok = false;
            switch (d.kind) {
            case KSORT_KEY_KIND__VREF:
                if (a.action == KAGG_ACTION__NROWS_ANY || a.action == KAGG_ACTION__NROWS_COND)
                    ok = true;
                else if (a.action == KAGG_ACTION__VREF && a.key_index >= 0) {
                    const uint8_t ld = plan->keys[a.key_index].ld;
                    ok = ld == XB_LD_BOOL || ld == XB_LD_INT2 || ld == XB_LD_INT4 || ld == XB_LD_INT8 ||
                         ld == XB_LD_DATE || ld == XB_LD_FLT8 || ld == XB_LD_FLT4;
                }
                break;
            case KSORT_KEY_KIND__PMINMAX_INT64:
                ok = a.action == KAGG_ACTION__PMIN_INT32 || a.action == KAGG_ACTION__PMIN_INT64 ||
                     a.action == KAGG_ACTION__PMAX_INT32 || a.action == KAGG_ACTION__PMAX_INT64;
                break;
            case KSORT_KEY_KIND__PMINMAX_FP64:
                ok = a.action == KAGG_ACTION__PMIN_FP64 || a.action == KAGG_ACTION__PMAX_FP64;
                break;
            case KSORT_KEY_KIND__PSUM_INT64:
            case KSORT_KEY_KIND__PSUM_NUMERIC:
                ok = a.action == KAGG_ACTION__PSUM_INT || a.action == KAGG_ACTION__PSUM_INT64 ||
                     a.action == KAGG_ACTION__PSUM_NUMERIC;
                if (a.action != KAGG_ACTION__PSUM_INT)
                    k.words = 2;                /* 128-bit sums */
                break;
            case KSORT_KEY_KIND__PSUM_FP64:
                ok = a.action == KAGG_ACTION__PSUM_FP;
                break;
            case KSORT_KEY_KIND__PAVG_INT64:
            case KSORT_KEY_KIND__PAVG_FP64:
            case KSORT_KEY_KIND__PAVG_NUMERIC:
                ok = a.action == KAGG_ACTION__PAVG_INT || a.action == KAGG_ACTION__PAVG_INT64 ||
                     a.action == KAGG_ACTION__PAVG_FP || a.action == KAGG_ACTION__PAVG_NUMERIC;
                break;
            case KSORT_KEY_KIND__PVARIANCE_SAMP:
            case KSORT_KEY_KIND__PVARIANCE_POP:
                ok = a.action == KAGG_ACTION__STDDEV;
                break;
            case KSORT_KEY_KIND__PCOVAR_CORR: case KSORT_KEY_KIND__PCOVAR_SAMP:
            case KSORT_KEY_KIND__PCOVAR_POP: case KSORT_KEY_KIND__PCOVAR_AVGX:
            case KSORT_KEY_KIND__PCOVAR_AVGY: case KSORT_KEY_KIND__PCOVAR_COUNT:
                ok = a.action == KAGG_ACTION__COVAR;
                break;
            case KSORT_KEY_KIND__NITEMS:
                ok = a.state_sz >= 8 && a.action != KAGG_ACTION__VREF &&
                     a.action != KAGG_ACTION__NROWS_ANY && a.action != KAGG_ACTION__NROWS_COND &&
                     !(a.action >= KAGG_ACTION__PMIN_INT32 && a.action <= KAGG_ACTION__PMAX_FP64);
                break;
            default:
                break;
            }
            if (!ok)
                return fail("sort key %d: kind %u over attribute %u (action %u) is not supported",
                            i, d.kind, d.src_anum, a.action);
        }
        plan->nsort = (uint32_t)nkeys;
        const char wf = ks->u.sort.window_rank_func;
        if (wf) {
            if (wf != KSORT_WINDOW_FUNC__ROW_NUMBER && wf != KSORT_WINDOW_FUNC__RANK &&
                wf != KSORT_WINDOW_FUNC__DENSE_RANK)
                return fail("unknown window function '%c'", wf);
            if ((int)ks->u.sort.window_partby_nkeys + (int)ks->u.sort.window_orderby_nkeys > nkeys)
                return fail("window keys exceed the sort keys");
            plan->sort_window = wf;
            plan->sort_partby = (uint8_t)ks->u.sort.window_partby_nkeys;
            plan->sort_orderby = (uint8_t)ks->u.sort.window_orderby_nkeys;
            plan->sort_rank_limit = ks->u.sort.window_rank_limit;
        } else if (session->gpusort_limit_count > 0) {
            plan->sort_limit = session->gpusort_limit_count;
        }
        return true;
    }

    bool loadvars(const kern_expression *kexp, int depth, xb_load *out, uint32_t *nout)
    {
        *nout = 0;
        if (!kexp)
            return true;
        if (kexp->opcode != FuncOpCode__LoadVars || kexp->exptype != TypeOpCode__int4)
            return fail("malformed LoadVars at depth %d", depth);
        if (kexp->u.load.depth != depth)
            return fail("LoadVars depth %d mismatch (expected %d)", kexp->u.load.depth, depth);
        int n = kexp->u.load.nitems;
        if (n < 0 || n > XB_MAX_LOADS ||
            offsetof(kern_expression, u.load.desc) + sizeof(kern_varload_desc) * n > kexp->len)
            return fail("LoadVars at depth %d has %d items", depth, n);
        int prev = -32768;
        for (int i = 0; i < n; i++) {
            const kern_varload_desc *vl = &kexp->u.load.desc[i];
            int slot = vl->vl_slot_id;
            if (slot < 0 || slot >= (int)plan->nslots)
                return fail("LoadVars slot %d out of range", slot);
            if (vl->vl_resno < prev)
                return fail("LoadVars descriptors are not sorted by resno");
            prev = vl->vl_resno;
            if (vl->vl_resno <= 0)
                return fail("system column reference (resno %d) is not supported", vl->vl_resno);
            if (vl->vl_resno > XB_MAX_COLS)
                return fail("attribute number %d exceeds %d", vl->vl_resno, XB_MAX_COLS);
            out[i].resno = vl->vl_resno;
            out[i].reg = (uint8_t)slot;
            out[i].ld = (uint8_t)slot_ld[slot];
        }
        *nout = (uint32_t)n;
        return true;
    }

    static int state_size(int action)
    {
        switch (action) {
        case KAGG_ACTION__VREF:          return 0;
        case KAGG_ACTION__NROWS_ANY:
        case KAGG_ACTION__NROWS_COND:    return 8;
        case KAGG_ACTION__PMIN_INT32:
        case KAGG_ACTION__PMIN_INT64:
        case KAGG_ACTION__PMAX_INT32:
        case KAGG_ACTION__PMAX_INT64:
        case KAGG_ACTION__PMIN_FP64:
        case KAGG_ACTION__PMAX_FP64:     return 16;
        case KAGG_ACTION__PSUM_INT:
        case KAGG_ACTION__PAVG_INT:      return 16;
        case KAGG_ACTION__PSUM_INT64:
        case KAGG_ACTION__PAVG_INT64:    return 24;
        case KAGG_ACTION__PSUM_FP:
        case KAGG_ACTION__PAVG_FP:       return 24;
        case KAGG_ACTION__PSUM_NUMERIC:
        case KAGG_ACTION__PAVG_NUMERIC:  return 32;
        case KAGG_ACTION__STDDEV:        return 40;
        case KAGG_ACTION__COVAR:         return 88;
        default:                         return -1;
        }
    }

    static int typmod_weight(int32_t typmod)
    {
        /* __numeric_typmod_weight (xpu_numeric.h:417-429); __DBL_DIG__ = 15 */
        int w = 15;
        if (typmod >= 0) {
            w = (((typmod - VARHDRSZ) & 0x7ff) ^ 1024) - 1024;
            if (w < 0) w = 0;
            if (w > 15) w = 15;
        }
        return w;
    }

    bool groupby()
    {
        const kern_expression *kact = kexp_at(session->xpucode_groupby_actions);
        if (!err.empty()) return false;
        if (!kact) {
            plan->has_groupby = 0;
            return true;
        }
        if (kact->opcode != FuncOpCode__AggFuncs)
            return fail("malformed AggFuncs (opcode %d)", kact->opcode);
        const kern_expression *khash = kexp_at(session->xpucode_groupby_keyhash);
        const kern_expression *kload = kexp_at(session->xpucode_groupby_keyload);
        const kern_expression *kcomp = kexp_at(session->xpucode_groupby_keycomp);
        if (!err.empty()) return false;
        if (khash && khash->opcode != FuncOpCode__HashValue)
            return fail("malformed GROUP BY key hash");
        if (kload && kload->opcode != FuncOpCode__LoadVars)
            return fail("malformed GROUP BY key load");
        (void)kcomp;
        plan->has_groupby = (khash && kload) ? 1 : 2;

        int nattrs = kact->u.pagg.nattrs;
        if (nattrs <= 0 || nattrs > XB_MAX_AGGS ||
            offsetof(kern_expression, u.pagg.desc) + sizeof(kern_aggregate_desc) * nattrs > kact->len)
            return fail("AggFuncs has %d attributes", nattrs);
        const kern_data_store *kds_final = nullptr;
        if (session->groupby_kds_final) {
            if ((uint64_t)session->groupby_kds_final + offsetof(kern_data_store, colmeta) > session_sz)
                return fail("groupby_kds_final is out of the session");
            kds_final = (const kern_data_store *)((const char *)session + session->groupby_kds_final);
            if ((uint64_t)session->groupby_kds_final + KDS_HEAD_LENGTH(kds_final) > session_sz)
                return fail("groupby_kds_final header is out of the session");
            if (kds_final->ncols < (uint32_t)nattrs)
                return fail("kds_final has %u columns but AggFuncs has %d", kds_final->ncols, nattrs);
            /* grouped results are KDS_FORMAT_HASH; the single tuple of an
             * aggregate without GROUP BY is KDS_FORMAT_ROW
             * (executor.c:655-697, cuda_gpupreagg.cu:1015-1016) */
            if (kds_final->format != KDS_FORMAT_HASH &&
                !(plan->has_groupby == 2 && kds_final->format == KDS_FORMAT_ROW))
                return fail("kds_final format '%c' does not fit the GROUP BY", kds_final->format);
        } else {
            return fail("GROUP BY session without groupby_kds_final");
        }

        uint32_t off = sizeof(xb_gent_head);
        plan->gent_keys_off = off;
        plan->nkeys = 0;
        plan->nkeys_text = 0;
        /* keys first (16B images) */
        for (int j = 0; j < nattrs; j++) {
            const kern_aggregate_desc *d = &kact->u.pagg.desc[j];
            if (d->action != KAGG_ACTION__VREF)
                continue;
            if (plan->has_groupby != 1)
                return fail("grouping key without GROUP BY key hash");
            if (plan->nkeys >= XB_MAX_KEYS)
                return fail("more than %d grouping keys", XB_MAX_KEYS);
            int slot = d->arg0_slot_id;
            if (slot < 0 || slot >= (int)plan->nslots)
                return fail("grouping key slot %d out of range", slot);
            int rk, ld, hk;
            if (!type_info(slot_type[slot], &rk, &ld, &hk))
                return fail("grouping key type %d not supported", slot_type[slot]);
            xb_key *k = &plan->keys[plan->nkeys];
            k->reg = (uint8_t)slot; k->rk = (uint8_t)rk; k->ld = (uint8_t)ld; k->hk = (uint8_t)hk;
            k->off = (uint16_t)(off + 16 * plan->nkeys);
            if (rk == XB_RK_TEXT || rk == XB_RK_NUM)
                plan->nkeys_text++;
            plan->nkeys++;
        }
        off += 16 * plan->nkeys;
        for (int j = 0; j < nattrs; j++) {
            const kern_aggregate_desc *d = &kact->u.pagg.desc[j];
            const kern_colmeta *cm = &kds_final->colmeta[j];
            xb_agg *a = &plan->aggs[j];
            int sz = state_size(d->action);
            if (sz < 0)
                return fail("partial aggregate action %d is not supported", d->action);
            a->action = d->action;
            a->arg0 = d->arg0_slot_id;
            a->arg1 = d->arg1_slot_id;
            a->filter = d->filter_slot_id;
            a->typmod = d->typmod;
            a->weight = (int16_t)typmod_weight(d->typmod);
            a->key_index = -1;
            a->attlen = cm->attlen;
            a->attalign = cm->attalign;
            if (a->attalign != 1 && a->attalign != 2 && a->attalign != 4 && a->attalign != 8)
                return fail("kds_final column %d has alignment %d", j, a->attalign);
            for (int16_t s : {a->arg0, a->arg1, a->filter})
                if (s >= (int)plan->nslots)
                    return fail("aggregate argument slot %d out of range", s);
            if (d->action == KAGG_ACTION__VREF) {
                for (uint32_t k = 0; k < plan->nkeys; k++)
                    if (plan->keys[k].reg == d->arg0_slot_id) { a->key_index = (int16_t)k; break; }
                a->state_off = 0;
                a->state_sz = 0;
                continue;
            }
            if (d->action != KAGG_ACTION__NROWS_ANY && a->arg0 < 0)
                return fail("aggregate action %d without argument", d->action);
            if ((d->action == KAGG_ACTION__PSUM_NUMERIC || d->action == KAGG_ACTION__PAVG_NUMERIC) &&
                slot_type[a->arg0] != TypeOpCode__numeric)
                return fail("numeric aggregate over a non-numeric argument");
            if (d->action == KAGG_ACTION__COVAR && a->arg1 < 0)
                return fail("covariance aggregate without 2nd argument");
            a->state_off = (uint16_t)off;
            a->state_sz = (uint16_t)sz;
            off += sz;
        }
        plan->naggs = nattrs;
        plan->gent_size = (uint32_t)PGSTROM_TYPEALIGN(16, off);

        /* programs: AggFuncs' SaveExpr arguments, then key hash, emitted
         * back to back (the kernel runs them as one stream) */
        if (!save_program(kact, &plan->gb_args))
            return false;
        if (khash && !program(khash, &plan->gb_keyhash, false))
            return false;
        if (khash && plan->gb_keyhash.start != plan->gb_args.start + plan->gb_args.count)
            return fail("group-by programs are not contiguous");
        return true;
    }

    static bool is_int_eq(int op)
    {
        switch (op) {
        case FuncOpCode__int2eq: case FuncOpCode__int24eq: case FuncOpCode__int28eq:
        case FuncOpCode__int42eq: case FuncOpCode__int4eq: case FuncOpCode__int48eq:
        case FuncOpCode__int82eq: case FuncOpCode__int84eq: case FuncOpCode__int8eq:
        case FuncOpCode__date_eq:
            return true;
        }
        return false;
    }

    /*
     * Fused probe: HashValue(Var x) at this depth and a join qual
     * "x = y" with y loaded from the inner relation at this depth.  The
     * kernel then hashes x inline and compares y's pre-decoded column
     * directly while walking the index; returns the index of the join qual
     * it absorbs, or -1.
     */
    int detect_fused_probe(const kern_expression *kh, const kern_expression *kj, xb_inner *in)
    {
        in->fast_key = -1;
        if (!kh || !kj || kh->nr_args != 1 || kj->opcode != FuncOpCode__JoinQuals)
            return -1;
        const kern_expression *hv = first_arg(kh);
        if (!hv || hv->opcode != FuncOpCode__VarExpr)
            return -1;
        int rk, ld, hk;
        if (!type_info(hv->exptype, &rk, &ld, &hk) || rk != XB_RK_INT)
            return -1;
        const int sx = hv->u.v.var_slot_id;
        const kern_expression *q = first_arg(kj);
        for (uint32_t i = 0; i < kj->nr_args && q; i++) {
            if (is_int_eq(q->opcode) && q->nr_args == 2 && !(q->expflags & KEXP_FLAG__IS_PUSHED_DOWN)) {
                const kern_expression *a = first_arg(q);
                const kern_expression *b = a ? next_arg(q, a) : nullptr;
                if (a && b && a->opcode == FuncOpCode__VarExpr && b->opcode == FuncOpCode__VarExpr) {
                    int sa = a->u.v.var_slot_id, sb = b->u.v.var_slot_id;
                    int sy = (sa == sx) ? sb : (sb == sx) ? sa : -1;
                    for (uint32_t k = 0; sy >= 0 && k < in->nloads; k++) {
                        if (in->load[k].reg == sy && plan->rk[sy] == XB_RK_INT) {
                            const int kld = in->load[k].ld;
                            in->fast_key = (int16_t)k;
                            in->fast_outer = (uint8_t)sx;
                            in->fast_hk = (uint8_t)hk;
                            in->key32 = (kld == XB_LD_INT2 || kld == XB_LD_INT4 || kld == XB_LD_DATE) ? 1 : 0;
                            return (int)i;
                        }
                    }
                }
            }
            if (i + 1 < kj->nr_args)
                q = next_arg(kj, q);
        }
        return -1;
    }

    /* registers read by instructions [start, start + count) */
    void reads_of(const xb_prog &p, uint64_t *mask)
    {
        for (uint32_t i = p.start; i < (uint32_t)p.start + p.count; i++) {
            const xb_insn &in = plan->insns[i];
            switch (in.op) {
            case XB_OP_CONST: case XB_OP_BOOL_INIT: case XB_OP_HASH_INIT:
            case XB_OP_MASK_PUSH: case XB_OP_MASK_POP: case XB_OP_END:
                break;
            case XB_OP_CMP: case XB_OP_ARITH: case XB_OP_DISTINCT:
                *mask |= (1ULL << in.a) | (1ULL << in.b);
                break;
            case XB_OP_AND_ACC: case XB_OP_OR_ACC: case XB_OP_HASH_ADD: case XB_OP_HASH_FINI:
                *mask |= (1ULL << in.a) | (1ULL << in.dst);
                break;
            default:
                *mask |= (1ULL << in.a);
                break;
            }
        }
    }

    /* an inner load is live if its register is read after its join */
    void compute_liveness()
    {
        uint64_t later = 0;     /* registers read by group-by and aggregates */
        reads_of(plan->gb_args, &later);
        reads_of(plan->gb_keyhash, &later);
        reads_of(plan->proj_args, &later);
        reads_of(plan->proj_hash, &later);
        for (uint32_t j = 0; plan->has_proj && j < plan->proj_nattrs; j++)
            later |= 1ULL << plan->proj[j].reg;
        for (uint32_t j = 0; j < plan->naggs; j++)
            for (int16_t r : {plan->aggs[j].arg0, plan->aggs[j].arg1, plan->aggs[j].filter})
                if (r >= 0) later |= 1ULL << r;
        for (uint32_t k = 0; k < plan->nkeys; k++)
            later |= 1ULL << plan->keys[k].reg;
        for (int d = (int)plan->nrels; d >= 1; d--) {
            xb_inner *in = &plan->inner[d];
            uint64_t here = later;
            reads_of(plan->join_quals[d], &here);
            in->live = 0;
            for (uint32_t k = 0; k < in->nloads; k++)
                if (here & (1ULL << in->load[k].reg))
                    in->live |= 1u << k;
            /* registers read at this depth are needed from shallower depths */
            reads_of(plan->join_quals[d], &later);
            reads_of(plan->hash_value[d], &later);
            if (in->fast_key >= 0)
                later |= 1ULL << in->fast_outer;
        }
    }

    /*
     * Join quals that read only the inner row of their own depth (and
     * constants), e.g. "d.flag < 3", give the same answer for every outer
     * row that meets that inner row.  When they cannot raise an error they
     * run once per inner row in the build instead, and rows that fail are
     * left out of the hash index: every probe is spared the qual and the
     * load of its inputs.  Outer rows that matched only such inner rows
     * find no match either way, and the depth's row counts are unchanged.
     */
    void hoist_inner_quals(uint32_t d)
    {
        xb_prog &q = plan->join_quals[d];
        const xb_inner *in = &plan->inner[d];
        if (!q.count)
            return;
        uint64_t avail = 0;
        for (uint32_t k = 0; k < in->nloads; k++)
            avail |= 1ULL << in->load[k].reg;
        for (uint32_t i = q.start; i < (uint32_t)q.start + q.count; i++) {
            const xb_insn &x = plan->insns[i];
            uint64_t reads = 0;
            bool safe = true;
            switch (x.op) {
            case XB_OP_END: case XB_OP_MASK_PUSH: case XB_OP_MASK_POP:
            case XB_OP_CONST: case XB_OP_BOOL_INIT:
                break;
            case XB_OP_MOVE: case XB_OP_NOT: case XB_OP_NULLTEST: case XB_OP_BOOLTEST:
            case XB_OP_MASK_NARROW:
                reads = 1ULL << x.a;
                break;
            case XB_OP_CMPI:
                reads = 1ULL << x.a;
                safe = x.kind == XB_RK_INT || x.kind == XB_RK_FLT;
                break;
            case XB_OP_CMP: case XB_OP_DISTINCT:
                reads = (1ULL << x.a) | (1ULL << x.b);
                safe = x.kind == XB_RK_INT || x.kind == XB_RK_FLT || x.kind == XB_RK_TEXT;
                break;
            case XB_OP_AND_ACC: case XB_OP_OR_ACC:
                reads = (1ULL << x.a) | (1ULL << x.dst);
                break;
            default:
                safe = false;       /* arithmetic, casts, hashes: may raise */
                break;
            }
            if (!safe || (reads & ~avail))
                return;
            switch (x.op) {
            case XB_OP_END: case XB_OP_MASK_PUSH: case XB_OP_MASK_POP: case XB_OP_MASK_NARROW:
                break;
            default:
                avail |= 1ULL << x.dst;     /* later instructions may read it */
                break;
            }
        }
        plan->inner[d].build_qual = q;
        q.count = 0;
        q.result = -1;
    }

    /*
     * GROUP BY keys that are all columns loaded at one inner depth (a
     * grouping by dimension attributes): the build numbers the distinct key
     * tuples among that relation's rows, and the specialised kernel finds
     * a row's group entry by that number.  Keys must compare by their bits:
     * integers, floats, and text whose hash is cached (those columns get
     * canonical pointers, one address per distinct string).
     */
    void choose_gid_depth()
    {
        plan->gid_depth = 0;
        if (plan->has_groupby != 1 || plan->nkeys == 0)
            return;
        uint64_t written = 0;
        for (uint32_t i = 0; i < plan->ninsns; i++) {
            const xb_insn &x = plan->insns[i];
            if (x.op != XB_OP_END && x.op != XB_OP_MASK_PUSH && x.op != XB_OP_MASK_NARROW &&
                x.op != XB_OP_MASK_POP)
                written |= 1ULL << x.dst;
        }
        int dd = -1;
        for (uint32_t k = 0; k < plan->nkeys; k++) {
            const xb_key &key = plan->keys[k];
            if (key.rk == XB_RK_NUM || (written & (1ULL << key.reg)))
                return;
            int found = -1;
            for (uint32_t d = 1; d <= plan->nrels && found < 0; d++)
                for (uint32_t j = 0; j < plan->inner[d].nloads; j++)
                    if (plan->inner[d].load[j].reg == key.reg) {
                        found = (int)d;
                        if (key.rk == XB_RK_TEXT && !((plan->inner[d].hashed >> j) & 1u))
                            return;
                        break;
                    }
            if (found < 0 || (dd >= 0 && found != dd))
                return;
            dd = found;
        }
        plan->gid_depth = (uint32_t)dd;
    }

    /*
     * Hashes of text / numeric values that come straight from an inner
     * relation's column (a group key taken from a dimension table, a join
     * key carried to a deeper depth) depend only on the inner row: the
     * build computes them once per inner row and HASH ops read that copy.
     * Applies when the register is loaded at exactly one inner depth and
     * never written by an instruction.
     */
    void mark_cached_hashes()
    {
        uint64_t written = 0;
        for (uint32_t i = 0; i < plan->ninsns; i++) {
            const xb_insn &x = plan->insns[i];
            switch (x.op) {
            case XB_OP_END: case XB_OP_MASK_PUSH: case XB_OP_MASK_NARROW: case XB_OP_MASK_POP:
                break;
            default:
                written |= 1ULL << x.dst;
                break;
            }
        }
        uint64_t outer = 0;
        for (uint32_t i = 0; i < plan->nload0; i++)
            outer |= 1ULL << plan->load0[i].reg;
        for (uint32_t i = 0; i < plan->ninsns; i++) {
            xb_insn &x = plan->insns[i];
            if ((x.op != XB_OP_HASH1 && x.op != XB_OP_HASH_ADD) ||
                (x.sub != XB_HK_TEXT && x.sub != XB_HK_NUM))
                continue;
            const uint64_t bit = 1ULL << x.a;
            if ((written & bit) || (outer & bit))
                continue;
            int found_d = -1, found_k = -1, nfound = 0;
            for (uint32_t d = 1; d <= plan->nrels; d++)
                for (uint32_t k = 0; k < plan->inner[d].nloads; k++)
                    if (plan->inner[d].load[k].reg == x.a) {
                        found_d = (int)d; found_k = (int)k; nfound++;
                    }
            if (nfound != 1)
                continue;
            plan->inner[found_d].hashed |= 1u << found_k;
            x.sub = XB_HK_CACHED;
        }
    }

    bool run(const kern_multirels *kmrels)
    {
        memset(plan, 0, sizeof(xb_plan));
        plan->magic = XB_PLAN_MAGIC;
        plan->wait_limit = XB_WAIT_LIMIT;
        plan->plan_sz = sizeof(xb_plan);
        if (session_sz < sizeof(kern_session_info))
            return fail("session is shorter than kern_session_info");
        plan->task_kind = session->xpu_task_flags & (DEVTASK__SCAN | DEVTASK__JOIN | DEVTASK__PREAGG);
        /* kvars slots (xpu_common.h:2839-2848) */
        uint32_t nslots = session->kcxt_kvars_nslots;
        if (nslots > XB_MAX_REGS - 8)
            return fail("session has %u kvars slots (max %d)", nslots, XB_MAX_REGS - 8);
        plan->nslots = nslots;
        plan->nregs = nslots;
        if (nslots > 0) {
            uint64_t defs = session->kcxt_kvars_defs;
            if (defs == 0 || defs + sizeof(kern_varslot_desc) * (uint64_t)nslots > session_sz)
                return fail("kvars slot descriptors are out of the session");
            const kern_varslot_desc *vs = (const kern_varslot_desc *)((const char *)session + defs);
            for (uint32_t i = 0; i < nslots; i++) {
                int rk, ld, hk;
                if (!type_info(vs[i].vs_type_code, &rk, &ld, &hk))
                    return fail("kvars slot %u has unsupported type code %d", i, vs[i].vs_type_code);
                plan->rk[i] = (uint8_t)rk;
                slot_type[i] = vs[i].vs_type_code;
                slot_ld[i] = ld;
            }
        }
        uint32_t nrels = kmrels ? kmrels->num_inner_rels : 0;
        if (nrels > XB_MAX_DEPTH)
            return fail("%u inner relations (max %d)", nrels, XB_MAX_DEPTH);
        plan->nrels = nrels;

        if (session->xpucode_gist_evals_packed)
            return fail("GiST-index joins are not supported by this build");

        const kern_expression *kload = kexp_at(session->xpucode_load_vars_packed);
        if (!err.empty()) return false;
        if (!loadvars(packed_at(kload, 0), 0, plan->load0, &plan->nload0))
            return false;
        plan->max_resno0 = 0;
        for (uint32_t i = 0; i < plan->nload0; i++)
            if (plan->load0[i].resno > plan->max_resno0)
                plan->max_resno0 = plan->load0[i].resno;
        if (!err.empty()) return false;

        const kern_expression *kqual = kexp_at(session->xpucode_scan_quals);
        if (!err.empty()) return false;
        if (!program(kqual, &plan->scan_quals, true))
            return false;

        const kern_expression *khash = kexp_at(session->xpucode_hash_values_packed);
        const kern_expression *kjoin = kexp_at(session->xpucode_join_quals_packed);
        if (!err.empty()) return false;
        for (uint32_t d = 1; d <= nrels; d++) {
            if (kmrels->chunks[d - 1].is_nestloop)
                return fail("nested-loop join at depth %u is not supported", d);
            if (kmrels->chunks[d - 1].left_outer || kmrels->chunks[d - 1].right_outer)
                return fail("outer join at depth %u is not supported", d);
            if (kmrels->chunks[d - 1].gist_offset)
                return fail("GiST join at depth %u is not supported", d);
            xb_inner *in = &plan->inner[d];
            if (!loadvars(packed_at(kload, d), d, in->load, &in->nloads))
                return false;
            const kern_expression *kh = packed_at(khash, d);
            if (!err.empty()) return false;
            if (!kh)
                return fail("hash join at depth %u has no HashValue", d);
            if (kh->opcode != FuncOpCode__HashValue)
                return fail("malformed HashValue at depth %u", d);
            if (!program(kh, &plan->hash_value[d], false))
                return false;
            const kern_expression *kj = packed_at(kjoin, d);
            if (!err.empty()) return false;
            int skip = detect_fused_probe(kh, kj, in);
            if (!err.empty()) return false;
            if (!join_program(kj, &plan->join_quals[d], skip))
                return false;
            hoist_inner_quals(d);
        }
        if (!groupby())
            return false;
        if (!projection())
            return false;
        if (!gpusort())
            return false;
        compute_liveness();
        mark_cached_hashes();
        choose_gid_depth();
        if (plan->has_groupby) {
            const bool kh = plan->has_groupby == 1 && plan->gb_keyhash.count > 0;
            plan->gb_all.start = plan->gb_args.count ? plan->gb_args.start : plan->gb_keyhash.start;
            plan->gb_all.count = (uint16_t)(plan->gb_args.count + (kh ? plan->gb_keyhash.count : 0));
            plan->gb_all.result = kh ? plan->gb_keyhash.result : (int16_t)-1;
        }
        if (plan->has_groupby == 0 && !plan->has_proj && !(plan->task_kind & DEVTASK__PREAGG))
            return fail("scan/join without device projection or GROUP BY is not supported");
        if (plan->has_groupby && plan->has_proj)
            return fail("a session with both GROUP BY and device projection is not supported");
        return err.empty();
    }
};

}   /* namespace */

extern "C" int
xb_compile_session(const kern_session_info *session, size_t session_sz,
                   uint64_t dev_session_base,
                   const kern_multirels *kmrels,
                   xb_plan *plan, char *errmsg, size_t errlen)
{
    Compiler c;
    memset(c.slot_type, 0, sizeof(c.slot_type));
    memset(c.slot_ld, 0, sizeof(c.slot_ld));
    c.session = session;
    c.session_sz = session_sz;
    c.dev_session = dev_session_base;
    c.plan = plan;
    c.ntemps = 0;
    if (!c.run(kmrels)) {
        if (errmsg && errlen > 0)
            snprintf(errmsg, errlen, "%s", c.err.empty() ? "unknown translation error" : c.err.c_str());
        return -1;
    }
    return 0;
}
