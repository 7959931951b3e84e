/*
 * xb_oracle.c -- CPU oracle for the scan / hash-join / pre-aggregation path.
 *
 * TEST INFRASTRUCTURE ONLY.  This is a sequential, single-threaded
 * restatement of the reference algorithm used as the checker in tests/,
 * __graft_entry__.smoke() and bench.py's cpu_baseline leg.  The product
 * (pg-strom_b200/) never links, loads or calls it.
 *
 * It follows the reference's per-row semantics one tuple at a time, in
 * chunk order:
 *   heap page walk, LP_NORMAL items in line-pointer order
 *                       cuda_gpuscan.cu:405-534 (__gpuscan_load_source_block)
 *   tuple decode        xpu_common.cu:60-252 (__kern_extract_common_tuple,
 *                       kern_extract_heap_tuple / _minimal_tuple)
 *   Arrow decode        xpu_common.cu:257-378, xpu_basetype.cu:243-310,
 *                       xpu_timelib.cu:76-120
 *   expression tree     xpu_common.cu:390-1090 (Const/Param/Var/Bool/NullTest),
 *                       xpu_basetype.cu:525-760, xpu_basetype.h:67-138
 *   HashValue           xpu_common.cu:1363-1398 + pg_hash_any :2898-3041
 *   hash join           cuda_gpujoin.cu:304-494: hash % hash_nslots chain walk
 *                       over KDS_FORMAT_HASH, t.hash compare, JoinQuals
 *   GROUP BY            cuda_gpupreagg.cu:1196-1774: SaveExpr arguments,
 *                       key hash, key equality, partial-state updates
 *   kds_final tuples    cuda_gpupreagg.cu:18-223 (__writeOutOneTuplePreAgg)
 *   projected rows      cuda_gpujoin.cu:753-800 + xpu_common.cu:1096-1184
 *                       (execGpuJoinProjection, __kern_form_minimal_tuple)
 * Floating-point sums are accumulated in row order in plain FP64: this is
 * the "FP64 sequentially ordered sum" the GPU results are compared with.
 *
 * Parity pinned: against PG-Strom's own functions host-compiled from its
 * sources (oracle/ref_harness.cpp: tuple and Arrow decode, quals, hash
 * joins and aggregate arguments computed by the reference, groups equal
 * with rtol=0; projected tuples byte for byte against its
 * kern_form_minimal_tuple), against the golden vectors those functions
 * produced (tests/golden/ref_*.json), against the reference's own Arrow
 * test file and its CSV, and against the reference's device kernel built
 * for sm_100a (oracle/ref_gpu.cpp).
 */
#include <stdint.h>
#include <stdlib.h>
#include <string.h>
#include <stdio.h>
#include <math.h>
#include "pgstrom_abi.h"

typedef __int128 i128;

#define XO_MAXSLOTS 64
#define XO_MAXDEPTH 8

/* ---------------- hash_any (lookup3 hashlittle, as PostgreSQL) ---------------- */
#define ROT(x,k) (((x) << (k)) | ((x) >> (32 - (k))))
static uint32_t xo_hash_any(const uint8_t *k, uint32_t len)
{
    uint32_t a, b, c;
    a = b = c = 0x9e3779b9U + len + 3923095U;
    while (len >= 12) {
        a += k[0] | (k[1] << 8) | (k[2] << 16) | ((uint32_t)k[3] << 24);
        b += k[4] | (k[5] << 8) | (k[6] << 16) | ((uint32_t)k[7] << 24);
        c += k[8] | (k[9] << 8) | (k[10] << 16) | ((uint32_t)k[11] << 24);
        a -= c; a ^= ROT(c, 4);  c += b;
        b -= a; b ^= ROT(a, 6);  a += c;
        c -= b; c ^= ROT(b, 8);  b += a;
        a -= c; a ^= ROT(c, 16); c += b;
        b -= a; b ^= ROT(a, 19); a += c;
        c -= b; c ^= ROT(b, 4);  b += a;
        k += 12; len -= 12;
    }
    switch (len) {
    case 11: c += ((uint32_t)k[10] << 24); /* fall through */
    case 10: c += ((uint32_t)k[9] << 16);  /* fall through */
    case 9:  c += ((uint32_t)k[8] << 8);   /* fall through */
    case 8:  b += ((uint32_t)k[7] << 24);  /* fall through */
    case 7:  b += ((uint32_t)k[6] << 16);  /* fall through */
    case 6:  b += ((uint32_t)k[5] << 8);   /* fall through */
    case 5:  b += k[4];                    /* fall through */
    case 4:  a += ((uint32_t)k[3] << 24);  /* fall through */
    case 3:  a += ((uint32_t)k[2] << 16);  /* fall through */
    case 2:  a += ((uint32_t)k[1] << 8);   /* fall through */
    case 1:  a += k[0];
    }
    c ^= b; c -= ROT(b, 14);
    a ^= c; a -= ROT(c, 11);
    b ^= a; b -= ROT(a, 25);
    c ^= b; c -= ROT(b, 16);
    a ^= c; a -= ROT(c, 4);
    b ^= a; b -= ROT(a, 14);
    c ^= b; c -= ROT(b, 24);
    return c;
}

uint32_t xo_hash_bytes(const void *p, uint32_t len) { return xo_hash_any((const uint8_t *)p, len); }

/* ---------------- datum ---------------- */
enum { DK_NULL = 0, DK_INT, DK_FLT, DK_TEXT, DK_NUM };
typedef struct {
    int     kind;           /* DK_* ; DK_NULL means SQL NULL */
    int     type_code;
    int64_t i;
    double  f;
    const uint8_t *p;       /* text payload, or numeric varlena */
    uint32_t len;
} xo_datum;

typedef struct {
    char    msg[256];
    int     failed;
} xo_err;

static int xo_fail(xo_err *e, const char *fmt, const char *s)
{
    if (!e->failed) {
        snprintf(e->msg, sizeof(e->msg), fmt, s);
        e->failed = 1;
    }
    return 0;
}

/* numeric varlena -> (kind, scale, value); xpu_numeric.h:216-277 */
static int xo_numeric(const uint8_t *vl, int *kind, int *weight, i128 *value)
{
    uint32_t len, hdr;
    if (vl[0] & 1) {
        if (vl[0] == 1) return -1;
        len = (vl[0] >> 1) & 0x7f; hdr = 1;
    } else {
        if ((vl[0] & 3) == 2) return -1;
        uint32_t h; memcpy(&h, vl, 4); len = h >> 2; hdr = 4;
    }
    if (len < hdr + 2) return -1;
    const uint8_t *nc = vl + hdr;
    uint32_t nclen = len - hdr;
    uint16_t head; memcpy(&head, nc, 2);
    if ((head & 0xC000) == 0xC000) {
        *kind = head == 0xC000 ? 1 : head == 0xD000 ? 2 : head == 0xF000 ? 3 : -1;
        *weight = 0; *value = 0;
        return *kind < 0 ? -1 : 0;
    }
    int w, ndig, neg;
    const uint8_t *dig;
    if ((head & 0xC000) == 0x8000) {
        w = head & 0x3F; if (head & 0x40) w |= ~0x3F;
        dig = nc + 2; ndig = (nclen - 2) / 2; neg = (head & 0x2000) != 0;
    } else {
        int16_t w16; memcpy(&w16, nc + 2, 2); w = w16;
        dig = nc + 4; ndig = (nclen - 4) / 2; neg = (head & 0xC000) == 0x4000;
    }
    i128 v = 0;
    for (int i = 0; i < ndig; i++) {
        int16_t d; memcpy(&d, dig + 2 * i, 2);
        if ((v >> 114) != 0) return -2;
        v = v * 10000 + d;
    }
    if (neg) v = -v;
    int sc = 4 * (ndig - (w + 1));
    if (v == 0) sc = 0;
    else {
        while (sc > 0) {
            if (sc >= 5 && v % 100000 == 0) { v /= 100000; sc -= 5; }
            else if (sc >= 4 && v % 10000 == 0) { v /= 10000; sc -= 4; }
            else if (sc >= 3 && v % 1000 == 0) { v /= 1000; sc -= 3; }
            else if (sc >= 2 && v % 100 == 0) { v /= 100; sc -= 2; }
            else if (sc >= 1 && v % 10 == 0) { v /= 10; sc -= 1; }
            else break;
        }
    }
    *kind = 0; *weight = sc; *value = v;
    return 0;
}

static i128 xo_rescale(int wd, int ws, i128 v)
{
    while (wd > ws) { v *= 10; ws++; }
    while (wd < ws) { v /= 10; ws--; }
    return v;
}

static int xo_numeric_cmp(const uint8_t *a, const uint8_t *b, xo_err *e)
{
    int ka, kb, wa, wb; i128 va, vb;
    if (xo_numeric(a, &ka, &wa, &va) || xo_numeric(b, &kb, &wb, &vb)) {
        xo_fail(e, "%s", "corrupted numeric");
        return 0;
    }
    int ra = ka == 1 ? 3 : ka == 2 ? 2 : ka == 3 ? 0 : 1;
    int rb = kb == 1 ? 3 : kb == 2 ? 2 : kb == 3 ? 0 : 1;
    if (ra != rb) return ra < rb ? -1 : 1;
    if (ra != 1) return 0;
    int w = wa > wb ? wa : wb;
    va = xo_rescale(w, wa, va); vb = xo_rescale(w, wb, vb);
    return va < vb ? -1 : va > vb ? 1 : 0;
}

/* heap datum image -> datum (xpu_*_datum_heap_read) */
static int xo_read_datum(int type_code, const uint8_t *addr, xo_datum *d, xo_err *e)
{
    d->type_code = type_code;
    switch (type_code) {
    case TypeOpCode__bool:   d->kind = DK_INT; d->i = addr[0] != 0; return 1;
    case TypeOpCode__int2:   { int16_t v; memcpy(&v, addr, 2); d->kind = DK_INT; d->i = v; return 1; }
    case TypeOpCode__int4:
    case TypeOpCode__date:   { int32_t v; memcpy(&v, addr, 4); d->kind = DK_INT; d->i = v; return 1; }
    case TypeOpCode__int8:
    case TypeOpCode__time:
    case TypeOpCode__timestamp:
    case TypeOpCode__timestamptz: { int64_t v; memcpy(&v, addr, 8); d->kind = DK_INT; d->i = v; return 1; }
    case TypeOpCode__float8: { double v; memcpy(&v, addr, 8); d->kind = DK_FLT; d->f = v; return 1; }
    case TypeOpCode__text:
    case TypeOpCode__bytea:
        if (addr[0] == 1 || (addr[0] & 3) == 2)
            return xo_fail(e, "%s", "external or compressed varlena");
        d->kind = DK_TEXT;
        if (addr[0] & 1) { d->p = addr + 1; d->len = ((addr[0] >> 1) & 0x7f) - 1; }
        else { uint32_t h; memcpy(&h, addr, 4); d->p = addr + 4; d->len = (h >> 2) - 4; }
        return 1;
    case TypeOpCode__numeric:
        if (addr[0] == 1 || (addr[0] & 3) == 2)
            return xo_fail(e, "%s", "external or compressed numeric");
        d->kind = DK_NUM; d->p = addr;
        return 1;
    }
    return xo_fail(e, "%s", "unsupported datum type");
}

/* ---------------- session ---------------- */
typedef struct xo_group {
    struct xo_group *next;
    uint32_t    hash;
    xo_datum    keys[8];
    uint8_t    *keybytes;       /* owned copies of text/numeric keys */
    /* states, per aggregate column */
    struct {
        int64_t  nitems;
        int64_t  i64;
        i128     i128v;
        double   f[5];
        uint32_t valid;
        uint32_t special;
    } st[32];
} xo_group;

typedef struct xo_sess {
    const kern_session_info *session;
    size_t      session_sz;
    const kern_multirels *kmrels;
    int         nslots;
    int         slot_type[XO_MAXSLOTS];
    int         nrels;
    const kern_expression *load[XO_MAXDEPTH + 1];
    const kern_expression *scan_quals;
    const kern_expression *hash_value[XO_MAXDEPTH + 1];
    const kern_expression *join_quals[XO_MAXDEPTH + 1];
    const kern_data_store *inner[XO_MAXDEPTH + 1];
    const kern_expression *gb_actions;
    const kern_expression *gb_keyhash;
    int         has_keys;
    int         nattrs;
    const kern_data_store *kds_final_head;
    /* device projection: formed rows, MAXALIGNed one after another */
    const kern_expression *proj;
    const kern_data_store *kds_dst_head;
    uint8_t    *proj_buf;
    uint64_t    proj_len, proj_cap, proj_nrows, proj_usage;
    xo_datum    slot[XO_MAXSLOTS];
    /* groups */
    xo_group  **htab;
    uint64_t    hsize;
    uint64_t    ngroups;
    xo_group  **order;          /* insertion order */
    uint64_t    order_cap;
    /* statistics */
    uint64_t    nitems_raw, nitems_in, nitems_out;
    uint64_t    nitems_depth[XO_MAXDEPTH + 1];
    xo_err      err;
} xo_sess;

static const kern_expression *kexp_at(xo_sess *s, uint32_t off)
{
    if (off == 0 || off >= s->session_sz)
        return NULL;
    return (const kern_expression *)((const char *)s->session + off);
}

static const kern_expression *first_arg(const kern_expression *k)
{
    return k->nr_args > 0 ? (const kern_expression *)((const char *)k + k->args_offset) : NULL;
}

static const kern_expression *next_arg(const kern_expression *k)
{
    return (const kern_expression *)((const char *)k + PGSTROM_MAXALIGN(k->len));
}

static const kern_expression *packed(const kern_expression *k, int idx)
{
    if (!k || idx < 0 || (uint32_t)idx >= k->u.pack.npacked || k->u.pack.offset[idx] == 0)
        return NULL;
    return (const kern_expression *)((const char *)k + k->u.pack.offset[idx]);
}

/* ---------------- expression evaluation ---------------- */
static int eval(xo_sess *s, const kern_expression *k, xo_datum *r);

static int cmp_datum(int sub, const xo_datum *a, const xo_datum *b, xo_err *e)
{
    int c = 0;
    if (a->kind == DK_INT && b->kind == DK_INT) c = a->i < b->i ? -1 : a->i > b->i;
    else if (a->kind == DK_FLT && b->kind == DK_FLT) {
        int na = isnan(a->f), nb = isnan(b->f);
        c = na ? (nb ? 0 : 1) : nb ? -1 : (a->f < b->f ? -1 : a->f > b->f);
    } else if (a->kind == DK_TEXT && b->kind == DK_TEXT)
        c = (a->len == b->len && memcmp(a->p, b->p, a->len) == 0) ? 0 : 1;
    else if (a->kind == DK_NUM && b->kind == DK_NUM)
        c = xo_numeric_cmp(a->p, b->p, e);
    switch (sub) {
    case 0: return c == 0;
    case 1: return c != 0;
    case 2: return c < 0;
    case 3: return c <= 0;
    case 4: return c > 0;
    default: return c >= 0;
    }
}

static int func_kind(int op, int *sub, int *width, int *cls)
{
    /* cls: 1 int arith, 2 flt arith, 3 compare, 4 cast */
    static const struct { const char *pfx; int w; } fam[] = {0};
    (void)fam;
#define IFAM(P, W) \
    if (op == FuncOpCode__##P##pl)  { *cls = 1; *sub = 0; *width = W; return 1; } \
    if (op == FuncOpCode__##P##mi)  { *cls = 1; *sub = 1; *width = W; return 1; } \
    if (op == FuncOpCode__##P##mul) { *cls = 1; *sub = 2; *width = W; return 1; } \
    if (op == FuncOpCode__##P##div) { *cls = 1; *sub = 3; *width = W; return 1; } \
    if (op == FuncOpCode__##P##eq)  { *cls = 3; *sub = 0; return 1; } \
    if (op == FuncOpCode__##P##ne)  { *cls = 3; *sub = 1; return 1; } \
    if (op == FuncOpCode__##P##lt)  { *cls = 3; *sub = 2; return 1; } \
    if (op == FuncOpCode__##P##le)  { *cls = 3; *sub = 3; return 1; } \
    if (op == FuncOpCode__##P##gt)  { *cls = 3; *sub = 4; return 1; } \
    if (op == FuncOpCode__##P##ge)  { *cls = 3; *sub = 5; return 1; }
    IFAM(int2, 2) IFAM(int24, 4) IFAM(int28, 8) IFAM(int42, 4) IFAM(int4, 4)
    IFAM(int48, 8) IFAM(int82, 8) IFAM(int84, 8) IFAM(int8, 8)
#undef IFAM
    if (op == FuncOpCode__float8pl)  { *cls = 2; *sub = 0; return 1; }
    if (op == FuncOpCode__float8mi)  { *cls = 2; *sub = 1; return 1; }
    if (op == FuncOpCode__float8mul) { *cls = 2; *sub = 2; return 1; }
    if (op == FuncOpCode__float8div) { *cls = 2; *sub = 3; return 1; }
#define CMP6(P) \
    if (op == FuncOpCode__##P##eq) { *cls = 3; *sub = 0; return 1; } \
    if (op == FuncOpCode__##P##ne) { *cls = 3; *sub = 1; return 1; } \
    if (op == FuncOpCode__##P##lt) { *cls = 3; *sub = 2; return 1; } \
    if (op == FuncOpCode__##P##le) { *cls = 3; *sub = 3; return 1; } \
    if (op == FuncOpCode__##P##gt) { *cls = 3; *sub = 4; return 1; } \
    if (op == FuncOpCode__##P##ge) { *cls = 3; *sub = 5; return 1; }
    CMP6(float8) CMP6(date_) CMP6(numeric_)
#undef CMP6
    if (op == FuncOpCode__text_eq) { *cls = 3; *sub = 0; return 1; }
    if (op == FuncOpCode__text_ne) { *cls = 3; *sub = 1; return 1; }
    if (op == FuncOpCode__int2_to_int4 || op == FuncOpCode__int2_to_int8 ||
        op == FuncOpCode__int4_to_int8) { *cls = 4; *sub = 0; return 1; }
    if (op == FuncOpCode__int4_to_int2 || op == FuncOpCode__int8_to_int2) { *cls = 4; *sub = 2; return 1; }
    if (op == FuncOpCode__int8_to_int4) { *cls = 4; *sub = 4; return 1; }
    if (op == FuncOpCode__int2_to_float8 || op == FuncOpCode__int4_to_float8 ||
        op == FuncOpCode__int8_to_float8) { *cls = 4; *sub = 10; return 1; }
    if (op == FuncOpCode__float8_to_int2) { *cls = 4; *sub = 12; return 1; }
    if (op == FuncOpCode__float8_to_int4) { *cls = 4; *sub = 14; return 1; }
    if (op == FuncOpCode__float8_to_int8) { *cls = 4; *sub = 18; return 1; }
    if (op == FuncOpCode__int4_to_bool) { *cls = 4; *sub = 20; return 1; }
    return 0;
}

static int eval_hash(xo_sess *s, const kern_expression *k, xo_datum *r)
{
    uint32_t h = 0xffffffffU;
    const kern_expression *a = first_arg(k);
    for (uint32_t i = 0; i < k->nr_args; i++, a = next_arg(a)) {
        xo_datum d;
        if (!eval(s, a, &d)) return 0;
        if (d.kind == DK_NULL) continue;
        uint32_t hv = 0;
        switch (a->exptype) {
        case TypeOpCode__bool: { uint8_t b = (uint8_t)d.i; hv = xo_hash_any(&b, 1); break; }
        case TypeOpCode__int2: { int16_t v = (int16_t)d.i; hv = xo_hash_any((uint8_t *)&v, 2); break; }
        case TypeOpCode__int4:
        case TypeOpCode__date: { int32_t v = (int32_t)d.i; hv = xo_hash_any((uint8_t *)&v, 4); break; }
        case TypeOpCode__int8:
        case TypeOpCode__time:
        case TypeOpCode__timestamp:
        case TypeOpCode__timestamptz: hv = xo_hash_any((uint8_t *)&d.i, 8); break;
        case TypeOpCode__float8: hv = xo_hash_any((uint8_t *)&d.f, 8); break;
        case TypeOpCode__text:
        case TypeOpCode__bytea: hv = xo_hash_any(d.p, d.len); break;
        case TypeOpCode__numeric: {
            int kind, w; i128 v;
            if (xo_numeric(d.p, &kind, &w, &v)) return xo_fail(&s->err, "%s", "corrupted numeric");
            if (kind) { uint8_t kk = (uint8_t)kind; hv = xo_hash_any(&kk, 1); }
            else { int16_t w16 = (int16_t)w; hv = xo_hash_any((uint8_t *)&w16, 2) ^ xo_hash_any((uint8_t *)&v, 16); }
            break;
        }
        default:
            return xo_fail(&s->err, "%s", "hash of unsupported type");
        }
        h = ((h >> 3) | (h << 29)) ^ hv;
    }
    r->kind = DK_INT; r->type_code = TypeOpCode__int4;
    r->i = (uint32_t)(h ^ 0xffffffffU);
    return 1;
}

static int eval(xo_sess *s, const kern_expression *k, xo_datum *r)
{
    memset(r, 0, sizeof(*r));
    r->type_code = k->exptype;
    switch (k->opcode) {
    case FuncOpCode__ConstExpr:
        if (k->u.c.const_isnull) { r->kind = DK_NULL; return 1; }
        return xo_read_datum(k->exptype, (const uint8_t *)k->u.c.const_value, r, &s->err);
    case FuncOpCode__ParamExpr: {
        uint32_t pid = k->u.p.param_id;
        if (pid >= s->session->nparams || s->session->poffset[pid] == 0) { r->kind = DK_NULL; return 1; }
        return xo_read_datum(k->exptype, (const uint8_t *)s->session + s->session->poffset[pid], r, &s->err);
    }
    case FuncOpCode__VarExpr: {
        int slot = k->u.v.var_slot_id;
        if (slot >= s->nslots) return xo_fail(&s->err, "%s", "slot out of range");
        *r = s->slot[slot];
        return 1;
    }
    case FuncOpCode__SaveExpr: {
        int slot = k->u.save.sv_slot_id;
        xo_datum d;
        if (!eval(s, first_arg(k), &d)) return 0;
        s->slot[slot] = d;
        *r = d;
        return 1;
    }
    case FuncOpCode__BoolExpr_And:
    case FuncOpCode__BoolExpr_Or: {
        int is_and = k->opcode == FuncOpCode__BoolExpr_And, anynull = 0;
        const kern_expression *a = first_arg(k);
        for (uint32_t i = 0; i < k->nr_args; i++, a = next_arg(a)) {
            xo_datum d;
            if (!eval(s, a, &d)) return 0;
            if (d.kind == DK_NULL) anynull = 1;
            else if (is_and ? !d.i : d.i) { r->kind = DK_INT; r->i = is_and ? 0 : 1; return 1; }
        }
        if (anynull) r->kind = DK_NULL; else { r->kind = DK_INT; r->i = is_and ? 1 : 0; }
        return 1;
    }
    case FuncOpCode__BoolExpr_Not: {
        xo_datum d;
        if (!eval(s, first_arg(k), &d)) return 0;
        if (d.kind == DK_NULL) r->kind = DK_NULL; else { r->kind = DK_INT; r->i = !d.i; }
        return 1;
    }
    case FuncOpCode__NullTestExpr_IsNull:
    case FuncOpCode__NullTestExpr_IsNotNull: {
        xo_datum d;
        if (!eval(s, first_arg(k), &d)) return 0;
        r->kind = DK_INT;
        r->i = (k->opcode == FuncOpCode__NullTestExpr_IsNull) == (d.kind == DK_NULL);
        return 1;
    }
    case FuncOpCode__HashValue:
        return eval_hash(s, k, r);
    default:
        break;
    }
    int sub = 0, width = 0, cls = 0;
    if (!func_kind(k->opcode, &sub, &width, &cls))
        return xo_fail(&s->err, "%s", "unsupported function opcode");
    xo_datum x, y;
    memset(&y, 0, sizeof(y));
    const kern_expression *a = first_arg(k);
    if (!eval(s, a, &x)) return 0;
    if (cls != 4 && !eval(s, next_arg(a), &y)) return 0;
    if (x.kind == DK_NULL || (cls != 4 && y.kind == DK_NULL)) { r->kind = DK_NULL; return 1; }
    if (cls == 3) {
        r->kind = DK_INT;
        r->i = cmp_datum(sub, &x, &y, &s->err);
        return !s->err.failed;
    }
    if (cls == 1) {
        i128 v;
        if (sub == 0) v = (i128)x.i + y.i;
        else if (sub == 1) v = (i128)x.i - y.i;
        else if (sub == 2) v = (i128)x.i * y.i;
        else {
            if (y.i == 0) return xo_fail(&s->err, "%s", "division by zero");
            v = (y.i == -1) ? -(i128)x.i : (i128)(x.i / y.i);
        }
        i128 lo = width == 2 ? -32768 : width == 4 ? INT32_MIN : INT64_MIN;
        i128 hi = width == 2 ? 32767 : width == 4 ? INT32_MAX : INT64_MAX;
        if (v < lo || v > hi) return xo_fail(&s->err, "%s", "integer out of range");
        r->kind = DK_INT; r->i = (int64_t)v;
        return 1;
    }
    if (cls == 2) {
        double v;
        if (sub == 0) v = x.f + y.f;
        else if (sub == 1) v = x.f - y.f;
        else if (sub == 2) v = x.f * y.f;
        else {
            if (y.f == 0.0) return xo_fail(&s->err, "%s", "division by zero");
            v = x.f / y.f;
            if (v == 0.0 && x.f != 0.0) return xo_fail(&s->err, "%s", "float out of range");
        }
        if (isinf(v) && !isinf(x.f) && !isinf(y.f)) return xo_fail(&s->err, "%s", "float out of range");
        r->kind = DK_FLT; r->f = v;
        return 1;
    }
    /* casts */
    if (sub <= 4) {
        int64_t lo = sub == 2 ? -32768 : sub == 4 ? INT32_MIN : INT64_MIN;
        int64_t hi = sub == 2 ? 32767 : sub == 4 ? INT32_MAX : INT64_MAX;
        if (x.i < lo || x.i > hi) return xo_fail(&s->err, "%s", "integer out of range");
        r->kind = DK_INT; r->i = x.i;
        return 1;
    }
    if (sub == 10) { r->kind = DK_FLT; r->f = (double)x.i; return 1; }
    if (sub == 20) { r->kind = DK_INT; r->i = x.i != 0; return 1; }
    {
        double d = rint(x.f);
        double lo = sub == 12 ? -32768.0 : sub == 14 ? (double)INT32_MIN : (double)INT64_MIN;
        if (isnan(d) || d < lo || d >= -lo) return xo_fail(&s->err, "%s", "integer out of range");
        r->kind = DK_INT; r->i = (int64_t)d;
        return 1;
    }
}

/* ---------------- tuple decode ---------------- */
static int decode_tuple(xo_sess *s, const kern_data_store *kds, int natts,
                        const uint8_t *nullmap, const uint8_t *payload,
                        const kern_expression *kload)
{
    if (!kload) return 1;
    int n = kload->u.load.nitems;
    const kern_varload_desc *vl = kload->u.load.desc;
    int li = 0, resno = 1;
    uint32_t off = 0;
    if (!nullmap) {
        while (li < n && vl[li].vl_resno <= natts) {
            const kern_colmeta *cm = &kds->colmeta[vl[li].vl_resno - 1];
            if (cm->attcacheoff < 0) break;
            off = cm->attcacheoff;
            const uint8_t *addr = payload + off;
            if (!xo_read_datum(s->slot_type[vl[li].vl_slot_id], addr, &s->slot[vl[li].vl_slot_id], &s->err))
                return 0;
            resno = vl[li].vl_resno + 1;
            if (cm->attlen > 0) off += cm->attlen;
            else if (addr[0] & 1) off += (addr[0] >> 1) & 0x7f;
            else { uint32_t h; memcpy(&h, addr, 4); off += h >> 2; }
            li++;
        }
    }
    for (; resno <= natts && li < n; resno++) {
        const kern_colmeta *cm = &kds->colmeta[resno - 1];
        const uint8_t *addr = NULL;
        if (!(nullmap && !((nullmap[(resno - 1) >> 3] >> ((resno - 1) & 7)) & 1))) {
            int al = cm->attalign > 0 ? cm->attalign : 1;
            if (cm->attlen > 0 || payload[off] == 0)
                off = (off + al - 1) & ~(uint32_t)(al - 1);
            addr = payload + off;
            if (cm->attlen > 0) off += cm->attlen;
            else if (addr[0] & 1) off += (addr[0] >> 1) & 0x7f;
            else { uint32_t h; memcpy(&h, addr, 4); off += h >> 2; }
        }
        if (vl[li].vl_resno == resno) {
            xo_datum *d = &s->slot[vl[li].vl_slot_id];
            if (!addr) { memset(d, 0, sizeof(*d)); d->kind = DK_NULL; }
            else if (!xo_read_datum(s->slot_type[vl[li].vl_slot_id], addr, d, &s->err)) return 0;
            li++;
        }
    }
    for (; li < n; li++) {
        memset(&s->slot[vl[li].vl_slot_id], 0, sizeof(xo_datum));
        s->slot[vl[li].vl_slot_id].kind = DK_NULL;
    }
    return 1;
}

/* ---------------- group-by ---------------- */
static int key_equal(const xo_datum *a, const xo_datum *b, xo_err *e)
{
    if (a->kind == DK_NULL || b->kind == DK_NULL) return a->kind == b->kind;
    if (a->kind == DK_TEXT) return a->len == b->len && memcmp(a->p, b->p, a->len) == 0;
    if (a->kind == DK_NUM) return xo_numeric_cmp(a->p, b->p, e) == 0;
    if (a->kind == DK_FLT) { int64_t x, y; memcpy(&x, &a->f, 8); memcpy(&y, &b->f, 8); return x == y; }
    return a->i == b->i;
}

static uint32_t numeric_varsize(const uint8_t *p)
{
    if (p[0] & 1) return (p[0] >> 1) & 0x7f;
    uint32_t h; memcpy(&h, p, 4); return h >> 2;
}

static double as_f64(const xo_datum *d) { return d->kind == DK_FLT ? d->f : (double)d->i; }

static int groupby_row(xo_sess *s)
{
    const kern_expression *kact = s->gb_actions;
    const kern_expression *a = first_arg(kact);
    for (uint32_t i = 0; i < kact->nr_args; i++, a = next_arg(a)) {
        xo_datum d;
        if (!eval(s, a, &d)) return 0;
    }
    uint32_t hash = 0;
    if (s->gb_keyhash) {
        xo_datum h;
        if (!eval(s, s->gb_keyhash, &h)) return 0;
        hash = (uint32_t)h.i;
    }
    /* collect keys (VREF columns) */
    xo_datum keys[8];
    int nkeys = 0;
    for (int j = 0; j < s->nattrs; j++) {
        const kern_aggregate_desc *d = &kact->u.pagg.desc[j];
        if (d->action == KAGG_ACTION__VREF && nkeys < 8)
            keys[nkeys++] = s->slot[d->arg0_slot_id];
    }
    uint64_t b = hash % s->hsize;
    xo_group *g;
    for (g = s->htab[b]; g; g = g->next) {
        if (g->hash != hash) continue;
        int eq = 1;
        for (int k = 0; k < nkeys && eq; k++) eq = key_equal(&g->keys[k], &keys[k], &s->err);
        if (eq) break;
    }
    if (!g) {
        g = (xo_group *)calloc(1, sizeof(xo_group));
        g->hash = hash;
        size_t nb = 0;
        for (int k = 0; k < nkeys; k++) {
            if (keys[k].kind == DK_TEXT) nb += keys[k].len;
            if (keys[k].kind == DK_NUM) nb += numeric_varsize(keys[k].p);
        }
        g->keybytes = nb ? (uint8_t *)malloc(nb) : NULL;
        uint8_t *kp = g->keybytes;
        for (int k = 0; k < nkeys; k++) {
            g->keys[k] = keys[k];
            if (keys[k].kind == DK_TEXT) { memcpy(kp, keys[k].p, keys[k].len); g->keys[k].p = kp; kp += keys[k].len; }
            if (keys[k].kind == DK_NUM) { uint32_t sz = numeric_varsize(keys[k].p); memcpy(kp, keys[k].p, sz); g->keys[k].p = kp; kp += sz; }
        }
        for (int j = 0; j < s->nattrs && j < 32; j++) {
            int act = kact->u.pagg.desc[j].action;
            if (act == KAGG_ACTION__PMIN_INT32 || act == KAGG_ACTION__PMIN_INT64) g->st[j].i64 = INT64_MAX;
            if (act == KAGG_ACTION__PMAX_INT32 || act == KAGG_ACTION__PMAX_INT64) g->st[j].i64 = INT64_MIN;
            if (act == KAGG_ACTION__PMIN_FP64) g->st[j].f[0] = 1.7976931348623157e308;
            if (act == KAGG_ACTION__PMAX_FP64) g->st[j].f[0] = -1.7976931348623157e308;
        }
        g->next = s->htab[b];
        s->htab[b] = g;
        if (s->ngroups == s->order_cap) {
            s->order_cap = s->order_cap ? s->order_cap * 2 : 1024;
            s->order = (xo_group **)realloc(s->order, sizeof(xo_group *) * s->order_cap);
        }
        s->order[s->ngroups++] = g;
    }
    /* update states (__update_groupby__*) */
    for (int j = 0; j < s->nattrs && j < 32; j++) {
        const kern_aggregate_desc *d = &kact->u.pagg.desc[j];
        if (d->filter_slot_id >= 0) {
            const xo_datum *f = &s->slot[d->filter_slot_id];
            if (f->kind == DK_NULL || !f->i) continue;
        }
        const xo_datum *x = d->arg0_slot_id >= 0 ? &s->slot[d->arg0_slot_id] : NULL;
        int xn = !x || x->kind == DK_NULL;
        switch (d->action) {
        case KAGG_ACTION__NROWS_ANY: g->st[j].nitems++; break;
        case KAGG_ACTION__NROWS_COND: if (!xn) g->st[j].nitems++; break;
        case KAGG_ACTION__PMIN_INT32: case KAGG_ACTION__PMIN_INT64:
            if (!xn) { g->st[j].valid = 1; if (x->i < g->st[j].i64) g->st[j].i64 = x->i; } break;
        case KAGG_ACTION__PMAX_INT32: case KAGG_ACTION__PMAX_INT64:
            if (!xn) { g->st[j].valid = 1; if (x->i > g->st[j].i64) g->st[j].i64 = x->i; } break;
        case KAGG_ACTION__PMIN_FP64:
            if (!xn) {
                double v = as_f64(x), c = g->st[j].f[0];
                /* float8 ordering: NaN is larger than every other value */
                int lt = isnan(v) ? 0 : (isnan(c) ? 1 : v < c);
                if (!g->st[j].valid || lt) g->st[j].f[0] = v;
                g->st[j].valid = 1;
            }
            break;
        case KAGG_ACTION__PMAX_FP64:
            if (!xn) {
                double v = as_f64(x), c = g->st[j].f[0];
                int gt = isnan(c) ? 0 : (isnan(v) ? 1 : v > c);
                if (!g->st[j].valid || gt) g->st[j].f[0] = v;
                g->st[j].valid = 1;
            }
            break;
        case KAGG_ACTION__PSUM_INT: case KAGG_ACTION__PAVG_INT:
            if (!xn) { g->st[j].nitems++; g->st[j].i64 = (int64_t)((uint64_t)g->st[j].i64 + (uint64_t)x->i); } break;
        case KAGG_ACTION__PSUM_INT64: case KAGG_ACTION__PAVG_INT64:
            if (!xn) { g->st[j].nitems++; g->st[j].i128v += x->i; } break;
        case KAGG_ACTION__PSUM_FP: case KAGG_ACTION__PAVG_FP:
            if (!xn) { g->st[j].nitems++; g->st[j].f[0] += as_f64(x); } break;
        case KAGG_ACTION__PSUM_NUMERIC: case KAGG_ACTION__PAVG_NUMERIC:
            if (!xn) {
                int kind, w; i128 v;
                if (xo_numeric(x->p, &kind, &w, &v)) return xo_fail(&s->err, "%s", "corrupted numeric");
                if (kind == 0) {
                    int wt = 15;
                    if (d->typmod >= 0) { wt = (((d->typmod - 4) & 0x7ff) ^ 1024) - 1024; if (wt < 0) wt = 0; if (wt > 15) wt = 15; }
                    g->st[j].nitems++;
                    g->st[j].i128v += xo_rescale(wt, w, v);
                } else {
                    g->st[j].special |= kind == 2 ? PAGG_NUMERIC_ATTRS__PINF
                                      : kind == 3 ? PAGG_NUMERIC_ATTRS__NINF : PAGG_NUMERIC_ATTRS__NAN;
                }
            }
            break;
        case KAGG_ACTION__STDDEV:
            if (!xn) { double v = as_f64(x); g->st[j].nitems++; g->st[j].f[0] += v; g->st[j].f[1] += v * v; }
            break;
        case KAGG_ACTION__COVAR: {
            const xo_datum *y = &s->slot[d->arg1_slot_id];
            if (!xn && y->kind != DK_NULL) {
                double vx = as_f64(x), vy = as_f64(y);
                g->st[j].nitems++;
                g->st[j].f[0] += vx; g->st[j].f[1] += vx * vx;
                g->st[j].f[2] += vy; g->st[j].f[3] += vy * vy; g->st[j].f[4] += vx * vy;
            }
            break;
        }
        default: break;
        }
    }
    return 1;
}

/* ---------------- joins ---------------- */
static int join_quals_ok(xo_sess *s, const kern_expression *kj, int *ok)
{
    *ok = 1;
    if (!kj) return 1;
    const kern_expression *a = first_arg(kj);
    for (uint32_t i = 0; i < kj->nr_args; i++, a = next_arg(a)) {
        xo_datum d;
        if (!eval(s, a, &d)) return 0;
        if (d.kind == DK_NULL || !d.i) { *ok = 0; return 1; }
    }
    return 1;
}

/* one projected datum at t of base (measure only when base is NULL);
 * returns its length (the xpu_*_datum_write of the slot's type) */
static uint32_t proj_datum(const xo_datum *d, uint8_t *base)
{
    switch (d->type_code) {
    case TypeOpCode__bool:   if (base) base[0] = d->i ? 1 : 0; return 1;
    case TypeOpCode__int2:   { int16_t v = (int16_t)d->i; if (base) memcpy(base, &v, 2); return 2; }
    case TypeOpCode__int4:
    case TypeOpCode__date:   { int32_t v = (int32_t)d->i; if (base) memcpy(base, &v, 4); return 4; }
    case TypeOpCode__int8:
    case TypeOpCode__time:
    case TypeOpCode__timestamp:
    case TypeOpCode__timestamptz: { if (base) memcpy(base, &d->i, 8); return 8; }
    case TypeOpCode__float8: { if (base) memcpy(base, &d->f, 8); return 8; }
    case TypeOpCode__text:
    case TypeOpCode__bytea: {
        uint32_t n = 4 + d->len;
        if (base) { uint32_t h = n << 2; memcpy(base, &h, 4); memcpy(base + 4, d->p, d->len); }
        return n;
    }
    case TypeOpCode__numeric: {
        uint32_t n = numeric_varsize(d->p);
        if (base) memcpy(base, d->p, n);
        return n;
    }
    }
    return 0;
}

/* form one row (__kern_form_minimal_tuple, xpu_common.cu:1096-1184) into
 * base, or measure it when base is NULL; returns t_len */
static uint32_t proj_form(xo_sess *s, int nattrs, uint8_t *base, uint32_t rowid)
{
    const uint16_t *slot_id = s->proj->u.proj.slot_id;
    const kern_data_store *kd = s->kds_dst_head;
    int hasnull = 0;
    for (int j = 0; j < nattrs; j++)
        if (slot_id[j] >= s->nslots || s->slot[slot_id[j]].kind == DK_NULL) { hasnull = 1; break; }
    uint32_t t = (uint32_t)PGSTROM_MAXALIGN(offsetof(kern_tupitem, t_bits) + (hasnull ? (nattrs + 7) / 8 : 0));
    uint16_t infomask = hasnull ? HEAP_HASNULL : 0;
    kern_tupitem *ti = (kern_tupitem *)base;
    if (base) {
        memset(base, 0, t);
        ti->t_infomask2 = (uint16_t)(nattrs & HEAP_NATTS_MASK);
        ti->t_hoff = (uint8_t)(t + MINIMAL_TUPLE_OFFSET);
    }
    for (int j = 0; j < nattrs; j++) {
        if (slot_id[j] >= s->nslots) continue;
        const xo_datum *d = &s->slot[slot_id[j]];
        if (d->kind == DK_NULL) continue;
        int al = kd->colmeta[j].attalign > 0 ? kd->colmeta[j].attalign : 1;
        uint32_t tn = (uint32_t)PGSTROM_TYPEALIGN(al, t);
        if (base && tn > t) memset(base + t, 0, tn - t);
        uint32_t n = proj_datum(d, base ? base + tn : NULL);
        if (kd->colmeta[j].attlen == -1) infomask |= HEAP_HASVARWIDTH;
        if (base && hasnull) ti->t_bits[j >> 3] |= (uint8_t)(1u << (j & 7));
        t = tn + n;
    }
    t += ROWID_SIZE;
    if (base) {
        ti->t_len = t;
        ti->t_infomask = infomask;
        memcpy(base + t - ROWID_SIZE, &rowid, 4);
    }
    return t;
}

/* projection of one output row: the Projection arguments fill their
 * slots, then the row is formed (execGpuJoinProjection,
 * cuda_gpujoin.cu:753-800, kern_estimate_minimal_tuple xpu_common.cu:1245-1292) */
static int proj_row(xo_sess *s)
{
    const kern_expression *kp = s->proj;
    const kern_expression *a = first_arg(kp);
    for (uint32_t i = 0; i < kp->nr_args; i++, a = next_arg(a)) {
        xo_datum d;
        if (!eval(s, a, &d)) return 0;
    }
    /* rows bound for a pinned inner buffer carry their hash value
     * (execGpuJoinProjection, cuda_gpujoin.cu:797-823) */
    uint32_t hash = 0;
    if (kp->u.proj.hash != 0) {
        xo_datum h;
        if (!eval(s, (const kern_expression *)((const char *)kp + kp->u.proj.hash), &h)) return 0;
        hash = (uint32_t)h.i;
    }
    int nattrs = kp->u.proj.nattrs;
    if (nattrs > (int)s->kds_dst_head->ncols) nattrs = s->kds_dst_head->ncols;
    uint32_t tl = proj_form(s, nattrs, NULL, 0);
    uint64_t need = PGSTROM_MAXALIGN(tl);
    if (s->proj_len + need > s->proj_cap) {
        uint64_t cap = s->proj_cap ? s->proj_cap * 2 : 1 << 16;
        while (cap < s->proj_len + need) cap *= 2;
        s->proj_buf = (uint8_t *)realloc(s->proj_buf, cap);
        s->proj_cap = cap;
    }
    memset(s->proj_buf + s->proj_len, 0, need);
    proj_form(s, nattrs, s->proj_buf + s->proj_len, (uint32_t)s->proj_nrows);
    ((kern_tupitem *)(s->proj_buf + s->proj_len))->hash = hash;
    s->proj_len += need;
    s->proj_nrows++;
    s->proj_usage += PGSTROM_MAXALIGN(PGSTROM_MAXALIGN(tl) + s->session->gpusort_htup_margin);
    return 1;
}

static int process_depth(xo_sess *s, int depth)
{
    if (depth > s->nrels) {
        s->nitems_out++;
        return s->gb_actions ? groupby_row(s) : s->proj ? proj_row(s) : 1;
    }
    xo_datum h;
    if (!eval(s, s->hash_value[depth], &h)) return 0;
    uint32_t hash = (uint32_t)h.i;
    const kern_data_store *kds = s->inner[depth];
    const uint64_t *hslot = (const uint64_t *)((const char *)kds + KDS_HEAD_LENGTH(kds));
    uint64_t off = hslot[hash % kds->hash_nslots];
    uint32_t guard = 0;
    while (off != 0 && off != UINT64_MAX) {
        if (++guard > kds->nitems + 1) return xo_fail(&s->err, "%s", "hash chain loop");
        const kern_hashitem *hi = (const kern_hashitem *)((const char *)kds + kds->length - off);
        if (hi->t.hash == hash) {
            const kern_tupitem *ti = &hi->t;
            int natts = ti->t_infomask2 & HEAP_NATTS_MASK;
            if (natts > (int)kds->ncols) natts = kds->ncols;
            const uint8_t *payload = (const uint8_t *)ti + ti->t_hoff - MINIMAL_TUPLE_OFFSET;
            if (!decode_tuple(s, kds, natts, (ti->t_infomask & HEAP_HASNULL) ? ti->t_bits : NULL,
                              payload, s->load[depth]))
                return 0;
            int ok;
            if (!join_quals_ok(s, s->join_quals[depth], &ok)) return 0;
            if (ok) {
                s->nitems_depth[depth]++;
                if (!process_depth(s, depth + 1)) return 0;
            }
        }
        off = hi->next;
    }
    return 1;
}

static int process_row(xo_sess *s)
{
    if (s->scan_quals) {
        xo_datum q;
        if (!eval(s, s->scan_quals, &q)) return 0;
        if (q.kind == DK_NULL || !q.i) return 1;
    }
    s->nitems_in++;
    return process_depth(s, 1);
}

/* ---------------- public API ---------------- */
int xo_open(const void *session, uint64_t session_sz, const void *kmrels, uint64_t kmrels_sz,
            xo_sess **p_sess, char *errmsg, int errlen)
{
    (void)kmrels_sz;
    xo_sess *s = (xo_sess *)calloc(1, sizeof(xo_sess));
    s->session = (const kern_session_info *)session;
    s->session_sz = session_sz;
    s->kmrels = (const kern_multirels *)kmrels;
    s->nslots = s->session->kcxt_kvars_nslots;
    if (s->nslots > XO_MAXSLOTS) { snprintf(errmsg, errlen, "too many slots"); free(s); return -1; }
    const kern_varslot_desc *vs = (const kern_varslot_desc *)((const char *)session + s->session->kcxt_kvars_defs);
    for (int i = 0; i < s->nslots; i++) s->slot_type[i] = vs[i].vs_type_code;
    s->nrels = kmrels ? (int)s->kmrels->num_inner_rels : 0;
    const kern_expression *kl = kexp_at(s, s->session->xpucode_load_vars_packed);
    const kern_expression *kh = kexp_at(s, s->session->xpucode_hash_values_packed);
    const kern_expression *kj = kexp_at(s, s->session->xpucode_join_quals_packed);
    for (int d = 0; d <= s->nrels; d++) {
        s->load[d] = packed(kl, d);
        if (d > 0) {
            s->hash_value[d] = packed(kh, d);
            s->join_quals[d] = packed(kj, d);
            s->inner[d] = (const kern_data_store *)((const char *)kmrels + s->kmrels->chunks[d - 1].kds_offset);
        }
    }
    s->scan_quals = kexp_at(s, s->session->xpucode_scan_quals);
    s->gb_actions = kexp_at(s, s->session->xpucode_groupby_actions);
    s->gb_keyhash = kexp_at(s, s->session->xpucode_groupby_keyhash);
    if (s->gb_actions) {
        s->nattrs = s->gb_actions->u.pagg.nattrs;
        s->kds_final_head = (const kern_data_store *)((const char *)session + s->session->groupby_kds_final);
    }
    if (!s->gb_actions && s->session->xpucode_projection) {
        s->proj = kexp_at(s, s->session->xpucode_projection);
        s->kds_dst_head = (const kern_data_store *)((const char *)session + s->session->projection_kds_dst);
    }
    s->hsize = 1 << 20;
    s->htab = (xo_group **)calloc(s->hsize, sizeof(xo_group *));
    *p_sess = s;
    return 0;
}

int xo_exec(xo_sess *s, const kern_data_store *kds, char *errmsg, int errlen)
{
    if (kds->format == KDS_FORMAT_BLOCK) {
        for (uint32_t b = 0; b < kds->nitems; b++) {
            const uint8_t *page = (const uint8_t *)kds + kds->block_offset + (uint64_t)b * PGSTROM_BLCKSZ;
            uint16_t lower; memcpy(&lower, page + 12, 2);
            uint32_t nlp = lower > 24 ? (lower - 24) / 4 : 0;
            for (uint32_t i = 0; i < nlp; i++) {
                uint32_t lp; memcpy(&lp, page + 24 + 4 * i, 4);
                if (ITEMID_FLAGS(lp) != LP_NORMAL) continue;
                const uint8_t *htup = page + ITEMID_OFF(lp);
                uint16_t im2, im; memcpy(&im2, htup + 18, 2); memcpy(&im, htup + 20, 2);
                int natts = im2 & HEAP_NATTS_MASK;
                if (natts > (int)kds->ncols) natts = kds->ncols;
                s->nitems_raw++;
                if (!decode_tuple(s, kds, natts, (im & HEAP_HASNULL) ? htup + 23 : NULL,
                                  htup + htup[22], s->load[0]) || !process_row(s)) {
                    snprintf(errmsg, errlen, "%s", s->err.msg);
                    return -1;
                }
            }
        }
    } else if (kds->format == KDS_FORMAT_ARROW) {
        const kern_expression *kl = s->load[0];
        for (uint32_t row = 0; row < kds->nitems; row++) {
            s->nitems_raw++;
            for (int li = 0; kl && li < kl->u.load.nitems; li++) {
                const kern_varload_desc *vl = &kl->u.load.desc[li];
                xo_datum *d = &s->slot[vl->vl_slot_id];
                memset(d, 0, sizeof(*d));
                d->kind = DK_NULL;
                if (vl->vl_resno > (int)kds->ncols) continue;
                const kern_colmeta *cm = &kds->colmeta[vl->vl_resno - 1];
                if (cm->nullmap_offset) {
                    const uint8_t *nm = (const uint8_t *)kds + cm->nullmap_offset;
                    if ((row >> 3) >= cm->nullmap_length || !((nm[row >> 3] >> (row & 7)) & 1)) continue;
                }
                const uint8_t *vals = (const uint8_t *)kds + cm->values_offset;
                int tc = s->slot_type[vl->vl_slot_id];
                /* a row past the values buffer reads as NULL, as the
                 * reference's readers have it (KDS_ARROW_REF_SIMPLE_DATUM,
                 * KDS_ARROW_REF_VARLENA32_DATUM, xpu_common.h:1557-1605) */
                if (tc == TypeOpCode__bool) {
                    /* bit-packed values (xpu_bool_datum_arrow_read,
                     * xpu_basetype.cu:37-57).  That reader does not bound
                     * the bitmap; a row past it reads as NULL here, as the
                     * reference's other fixed-width readers have it and as
                     * the device's reader does */
                    if (((uint64_t)row >> 3) >= cm->values_length)
                        continue;
                } else {
                    const uint64_t unitsz = tc == TypeOpCode__int2 ? 2 :
                                            (tc == TypeOpCode__int4 || tc == TypeOpCode__date ||
                                             tc == TypeOpCode__text) ? 4 : 8;
                    if (unitsz * ((uint64_t)row + 1) > cm->values_length)
                        continue;
                }
                if (tc == TypeOpCode__text) {
                    const uint32_t *o = (const uint32_t *)vals;
                    if (o[row] > o[row + 1] || o[row + 1] > cm->extra_length || o[row + 1] - o[row] > 0x4ffffff8U)
                        continue;
                }
                d->type_code = tc;
                switch (tc) {
                case TypeOpCode__bool: d->kind = DK_INT; d->i = (vals[row >> 3] >> (row & 7)) & 1; break;
                case TypeOpCode__int2: d->kind = DK_INT; d->i = ((const int16_t *)vals)[row]; break;
                case TypeOpCode__int4: d->kind = DK_INT; d->i = ((const int32_t *)vals)[row]; break;
                case TypeOpCode__int8: d->kind = DK_INT; d->i = ((const int64_t *)vals)[row]; break;
                case TypeOpCode__float8: d->kind = DK_FLT; d->f = ((const double *)vals)[row]; break;
                case TypeOpCode__date:
                    d->kind = DK_INT;
                    d->i = (int32_t)(((const uint32_t *)vals)[row] - 10957u);
                    break;
                case TypeOpCode__text: {
                    const uint32_t *o = (const uint32_t *)vals;
                    d->kind = DK_TEXT; d->p = (const uint8_t *)kds + cm->extra_offset + o[row];
                    d->len = o[row + 1] - o[row];
                    break;
                }
                default:
                    snprintf(errmsg, errlen, "unsupported Arrow column type");
                    return -1;
                }
            }
            if (!process_row(s)) { snprintf(errmsg, errlen, "%s", s->err.msg); return -1; }
        }
    } else if (kds->format == KDS_FORMAT_ROW) {
        /* rows by index (__gpuscan_load_source_row, cuda_gpuscan.cu:646-700):
         * the row index after the hash slots holds each kern_tupitem's
         * offset back from the chunk's end (KDS_GET_TUPITEM,
         * xpu_common.h:1337-1345); the tuple's header and data follow the
         * heap tuple's from t_infomask2 on, MINIMAL_TUPLE_OFFSET bytes
         * later (kern_extract_minimal_tuple, xpu_common.cu:132-191).  Rows
         * carry no transaction attributes here (they would be checked for
         * visibility); an empty slot is no row */
        const uint64_t *rowindex = (const uint64_t *)((const char *)kds + KDS_HEAD_LENGTH(kds)) + kds->hash_nslots;
        for (uint32_t row = 0; row < kds->nitems; row++) {
            const uint64_t off = rowindex[row];
            if (off == 0) continue;
            if (off > kds->length || off < 16 || ((kds->length - off) & 7) != 0) {
                snprintf(errmsg, errlen, "KDS_FORMAT_ROW row %u is out of the chunk", row);
                return -1;
            }
            const uint8_t *ti = (const uint8_t *)kds + kds->length - off;
            uint32_t t_len; memcpy(&t_len, ti, 4);
            uint16_t im2, im; memcpy(&im2, ti + 10, 2); memcpy(&im, ti + 12, 2);
            const uint32_t t_hoff = ti[14];
            if (ti[8] != 0 || t_hoff < MINIMAL_TUPLE_OFFSET + 15 || t_hoff - MINIMAL_TUPLE_OFFSET > t_len ||
                t_len > off) {
                snprintf(errmsg, errlen, "KDS_FORMAT_ROW row %u is broken", row);
                return -1;
            }
            int natts = im2 & HEAP_NATTS_MASK;
            if (natts > (int)kds->ncols) natts = kds->ncols;
            s->nitems_raw++;
            if (!decode_tuple(s, kds, natts, (im & HEAP_HASNULL) ? ti + 15 : NULL,
                              ti + t_hoff - MINIMAL_TUPLE_OFFSET, s->load[0]) || !process_row(s)) {
                snprintf(errmsg, errlen, "%s", s->err.msg);
                return -1;
            }
        }
    } else {
        snprintf(errmsg, errlen, "unsupported KDS format");
        return -1;
    }
    return 0;
}

void xo_stats(xo_sess *s, uint64_t *out)
{
    out[0] = s->nitems_raw;
    out[1] = s->nitems_in;
    out[2] = s->nitems_out;
    for (int d = 1; d <= XO_MAXDEPTH; d++) out[2 + d] = s->nitems_depth[d];
}

/* write kds_final (the same layout as __writeOutOneTuplePreAgg); returns
 * required length, writing only if buf_sz is large enough.  Grouped
 * results are KDS_FORMAT_HASH (kern_hashitems chained into hash slots);
 * an aggregate without GROUP BY keys writes its one tuple into a
 * KDS_FORMAT_ROW buffer (no hash slots, a bare kern_tupitem), as
 * __insertOneTupleNoGroups does (cuda_gpupreagg.cu:1005-1036) into the
 * ROW header executor.c:690-695 sets up */
uint64_t xo_final(xo_sess *s, void *buf, uint64_t buf_sz)
{
    if (!s->gb_actions) return 0;
    const kern_data_store *fh = s->kds_final_head;
    uint64_t head_len = KDS_HEAD_LENGTH(fh);
    uint64_t ng = s->ngroups;
    const int row_fmt = fh->format == KDS_FORMAT_ROW;
    const uint64_t link = row_fmt ? 0 : 8;     /* kern_hashitem.next */
    uint64_t nslots = row_fmt ? 0 : KDS_GET_HASHSLOT_WIDTH(ng);
    int nattrs = s->nattrs;
    uint32_t hoff0 = (uint32_t)PGSTROM_MAXALIGN(15 + (nattrs + 7) / 8);
    /* pass 1: sizes */
    uint64_t *sizes = (uint64_t *)malloc(sizeof(uint64_t) * (ng ? ng : 1));
    uint64_t items = 0;
    for (uint64_t gi = 0; gi < ng; gi++) {
        xo_group *g = s->order[gi];
        uint32_t t = hoff0;
        int kk = 0;
        for (int j = 0; j < nattrs; j++) {
            const kern_aggregate_desc *d = &s->gb_actions->u.pagg.desc[j];
            const kern_colmeta *cm = &fh->colmeta[j];
            t = (uint32_t)PGSTROM_TYPEALIGN(cm->attalign, t);
            switch (d->action) {
            case KAGG_ACTION__VREF: {
                xo_datum *k = &g->keys[kk++];
                if (k->kind == DK_NULL) break;
                int tc = s->slot_type[d->arg0_slot_id];
                if (k->kind == DK_TEXT) t += 4 + k->len;
                else if (k->kind == DK_NUM) t += numeric_varsize(k->p);
                else if (tc == TypeOpCode__bool) t += 1;
                else if (tc == TypeOpCode__int2) t += 2;
                else if (tc == TypeOpCode__int4 || tc == TypeOpCode__date) t += 4;
                else t += 8;
                break;
            }
            case KAGG_ACTION__NROWS_ANY: case KAGG_ACTION__NROWS_COND: t += 8; break;
            case KAGG_ACTION__PMIN_INT32: case KAGG_ACTION__PMIN_INT64: case KAGG_ACTION__PMAX_INT32:
            case KAGG_ACTION__PMAX_INT64: case KAGG_ACTION__PMIN_FP64: case KAGG_ACTION__PMAX_FP64: t += 16; break;
            case KAGG_ACTION__PSUM_INT: case KAGG_ACTION__PAVG_INT: t += 24; break;
            case KAGG_ACTION__PSUM_FP: case KAGG_ACTION__PAVG_FP: t += 24; break;
            case KAGG_ACTION__PSUM_INT64: case KAGG_ACTION__PAVG_INT64:
            case KAGG_ACTION__PSUM_NUMERIC: case KAGG_ACTION__PAVG_NUMERIC: t += 32; break;
            case KAGG_ACTION__STDDEV: t += 32; break;
            case KAGG_ACTION__COVAR: t += 56; break;
            }
        }
        t += 4;
        sizes[gi] = PGSTROM_MAXALIGN(link + t);
        items += sizes[gi];
    }
    uint64_t length = head_len + 8 * nslots + 8 * ng + items;
    if (!buf || buf_sz < length) { free(sizes); return length; }
    char *out = (char *)buf;
    memset(out, 0, length);
    memcpy(out, fh, head_len);
    kern_data_store *kh = (kern_data_store *)out;
    kh->length = length; kh->usage = items; kh->nitems = (uint32_t)ng;
    kh->format = row_fmt ? KDS_FORMAT_ROW : KDS_FORMAT_HASH; kh->hash_nslots = (uint32_t)nslots;
    uint64_t *hslot = (uint64_t *)(out + head_len);
    uint64_t *rowidx = hslot + nslots;
    uint64_t pos = head_len + 8 * nslots + 8 * ng;
    for (uint64_t gi = 0; gi < ng; gi++) {
        xo_group *g = s->order[gi];
        kern_hashitem *hi = (kern_hashitem *)(out + pos);
        kern_tupitem *ti = (kern_tupitem *)(out + pos + link);
        char *base = (char *)ti;
        uint16_t infomask = HEAP_HASNULL;
        uint32_t t = hoff0;
        int kk = 0;
        ti->hash = g->hash;
        ti->t_infomask2 = (uint16_t)nattrs;
        ti->t_hoff = (uint8_t)(hoff0 + MINIMAL_TUPLE_OFFSET);
        for (int j = 0; j < nattrs; j++) {
            const kern_aggregate_desc *d = &s->gb_actions->u.pagg.desc[j];
            const kern_colmeta *cm = &fh->colmeta[j];
            t = (uint32_t)PGSTROM_TYPEALIGN(cm->attalign, t);
            char *p = base + t;
            uint32_t nb = 0;
            switch (d->action) {
            case KAGG_ACTION__VREF: {
                xo_datum *k = &g->keys[kk++];
                if (k->kind == DK_NULL) break;
                int tc = s->slot_type[d->arg0_slot_id];
                if (k->kind == DK_TEXT) { nb = 4 + k->len; uint32_t h = nb << 2; memcpy(p, &h, 4); memcpy(p + 4, k->p, k->len); infomask |= HEAP_HASVARWIDTH; }
                else if (k->kind == DK_NUM) { nb = numeric_varsize(k->p); memcpy(p, k->p, nb); infomask |= HEAP_HASVARWIDTH; }
                else if (tc == TypeOpCode__bool) { nb = 1; p[0] = (char)k->i; }
                else if (tc == TypeOpCode__int2) { nb = 2; int16_t v = (int16_t)k->i; memcpy(p, &v, 2); }
                else if (tc == TypeOpCode__int4 || tc == TypeOpCode__date) { nb = 4; int32_t v = (int32_t)k->i; memcpy(p, &v, 4); }
                else if (k->kind == DK_FLT) { nb = 8; memcpy(p, &k->f, 8); }
                else { nb = 8; memcpy(p, &k->i, 8); }
                break;
            }
            case KAGG_ACTION__NROWS_ANY: case KAGG_ACTION__NROWS_COND:
                nb = 8; memcpy(p, &g->st[j].nitems, 8); break;
            case KAGG_ACTION__PMIN_INT32: case KAGG_ACTION__PMIN_INT64:
            case KAGG_ACTION__PMAX_INT32: case KAGG_ACTION__PMAX_INT64: {
                kagg_state__pminmax_int64_packed r = { 16 << 2, g->st[j].valid ? 1u : 0u, g->st[j].i64 };
                nb = 16; memcpy(p, &r, 16); infomask |= HEAP_HASVARWIDTH; break;
            }
            case KAGG_ACTION__PMIN_FP64: case KAGG_ACTION__PMAX_FP64: {
                kagg_state__pminmax_fp64_packed r = { 16 << 2, g->st[j].valid ? 1u : 0u, g->st[j].f[0] };
                nb = 16; memcpy(p, &r, 16); infomask |= HEAP_HASVARWIDTH; break;
            }
            case KAGG_ACTION__PSUM_INT: case KAGG_ACTION__PAVG_INT: {
                kagg_state__psum_int_packed r = { 24 << 2, 0, g->st[j].nitems, g->st[j].i64 };
                nb = 24; memcpy(p, &r, 24); infomask |= HEAP_HASVARWIDTH; break;
            }
            case KAGG_ACTION__PSUM_FP: case KAGG_ACTION__PAVG_FP: {
                kagg_state__psum_fp_packed r = { 24 << 2, 0, g->st[j].nitems, g->st[j].f[0] };
                nb = 24; memcpy(p, &r, 24); infomask |= HEAP_HASVARWIDTH; break;
            }
            case KAGG_ACTION__PSUM_INT64: case KAGG_ACTION__PAVG_INT64:
            case KAGG_ACTION__PSUM_NUMERIC: case KAGG_ACTION__PAVG_NUMERIC: {
                kagg_state__psum_numeric_packed r;
                int is_num = d->action == KAGG_ACTION__PSUM_NUMERIC || d->action == KAGG_ACTION__PAVG_NUMERIC;
                int wt = 15;
                if (d->typmod >= 0) { wt = (((d->typmod - 4) & 0x7ff) ^ 1024) - 1024; if (wt < 0) wt = 0; if (wt > 15) wt = 15; }
                r.vl_len_ = 32 << 2;
                r.attrs = is_num ? ((uint32_t)wt | g->st[j].special) : 0;
                r.nitems = (uint64_t)g->st[j].nitems;
                r.sum.u64_lo = (uint64_t)g->st[j].i128v;
                r.sum.u64_hi = (uint64_t)((unsigned __int128)g->st[j].i128v >> 64);
                nb = 32; memcpy(p, &r, 32); infomask |= HEAP_HASVARWIDTH; break;
            }
            case KAGG_ACTION__STDDEV: {
                kagg_state__stddev_packed r = { 32 << 2, 0, g->st[j].nitems, g->st[j].f[0], g->st[j].f[1] };
                nb = 32; memcpy(p, &r, 32); infomask |= HEAP_HASVARWIDTH; break;
            }
            case KAGG_ACTION__COVAR: {
                kagg_state__covar_packed r = { 56 << 2, 0, g->st[j].nitems, g->st[j].f[0], g->st[j].f[1],
                                               g->st[j].f[2], g->st[j].f[3], g->st[j].f[4] };
                nb = 56; memcpy(p, &r, 56); infomask |= HEAP_HASVARWIDTH; break;
            }
            }
            if (nb) ti->t_bits[j >> 3] |= (uint8_t)(1u << (j & 7));
            t += nb;
        }
        t += 4;
        ti->t_len = t;
        ti->t_infomask = infomask;
        uint32_t rowid = (uint32_t)gi;
        memcpy(base + t - 4, &rowid, 4);
        rowidx[gi] = length - (pos + link);
        if (!row_fmt) {
            uint64_t slot = g->hash % nslots;
            hi->next = hslot[slot];
            hslot[slot] = length - pos;
        }
        pos += sizes[gi];
    }
    free(sizes);
    return length;
}

/* projected rows so far: copies them (MAXALIGNed kern_tupitems, row id =
 * their order) into buf when it is large enough; returns their bytes and
 * sets the row count and the kds_dst usage the reference would take */
uint64_t xo_proj_rows(xo_sess *s, void *buf, uint64_t buf_sz, uint64_t *p_nrows, uint64_t *p_usage)
{
    if (p_nrows) *p_nrows = s->proj_nrows;
    if (p_usage) *p_usage = s->proj_usage;
    if (buf && buf_sz >= s->proj_len && s->proj_len)
        memcpy(buf, s->proj_buf, s->proj_len);
    return s->proj_len;
}

/* forget the projected rows (next chunk's kds_dst) */
void xo_proj_reset(xo_sess *s)
{
    s->proj_len = s->proj_nrows = s->proj_usage = 0;
}

void xo_close(xo_sess *s)
{
    if (!s) return;
    free(s->proj_buf);
    for (uint64_t i = 0; i < s->ngroups; i++) {
        free(s->order[i]->keybytes);
        free(s->order[i]);
    }
    free(s->order);
    free(s->htab);
    free(s);
}
