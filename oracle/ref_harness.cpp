/*
 * ref_harness.cpp -- TEST INFRASTRUCTURE ONLY.
 *
 * Drives PG-Strom's own expression / type library, host-compiled from the
 * reference sources (src/xpu_common.cu, xpu_basetype.cu, xpu_numeric.cu,
 * xpu_textlib.cu, xpu_timelib.cu, ... by oracle/Makefile "ref"), over the
 * same session bytecode and chunks the CUDA path consumes.  It resolves
 * fn_dptr / expr_ops / vs_ops against the reference's catalogs the way
 * __resolveDevicePointers does (gpu_service.c:3115-3317), then runs a
 * sequential scan -> hash join -> group-by loop in which every tuple
 * decode, qualifier, hash value and aggregate argument is computed by the
 * reference's functions (ExecLoadVarsOuterHeap, ExecLoadVarsOuterArrow,
 * ExecLoadVarsMinimalTuple,
 * ExecMoveKernelVariables, EXEC_KERN_EXPRESSION, ExecGpuJoinQuals,
 * pg_hash_any, xpu_*_datum_write, and for projection sessions
 * kern_estimate_minimal_tuple / kern_form_minimal_tuple, whose tuples are
 * returned as they are).  Only the group accumulation itself is
 * restated (its reference form is device-only code), with exact int128
 * and row-ordered FP64 sums.  Results are returned as JSON text.
 *
 * Compiled against the reference headers; never part of the product.
 */
#include <array>
#include <string>
#include <vector>
#include <map>
#include <cmath>
#include <cstdio>
#include "xpu_common.h"

/* run-time properties the device kernels keep in shared memory */
uint32_t stromTaskProp__cuda_dindex = 0;
uint32_t stromTaskProp__cuda_stack_limit = 0;
int32_t  stromTaskProp__partition_divisor = 0;
int32_t  stromTaskProp__partition_reminder = 0;

static const xpu_datum_operators *lookup_type(TypeOpCode code)
{
    for (int i = 0; builtin_xpu_types_catalog[i].type_opcode != TypeOpCode__Invalid; i++)
        if (builtin_xpu_types_catalog[i].type_opcode == code)
            return builtin_xpu_types_catalog[i].type_ops;
    return NULL;
}

static xpu_function_t lookup_func(FuncOpCode code)
{
    for (int i = 0; builtin_xpu_functions_catalog[i].func_opcode != FuncOpCode__Invalid; i++)
        if (builtin_xpu_functions_catalog[i].func_opcode == code)
            return builtin_xpu_functions_catalog[i].func_dptr;
    return NULL;
}

static bool resolve(kern_expression *kexp, std::string &err)
{
    kexp->fn_dptr = lookup_func(kexp->opcode);
    kexp->expr_ops = lookup_type(kexp->exptype);
    if (!kexp->fn_dptr || !kexp->expr_ops) {
        err = "unresolved opcode " + std::to_string(kexp->opcode) + "/" + std::to_string(kexp->exptype);
        return false;
    }
    kern_expression *karg = KEXP_FIRST_ARG(kexp);
    for (uint32_t i = 0; i < kexp->nr_args; i++, karg = KEXP_NEXT_ARG(karg)) {
        if (!__KEXP_IS_VALID(kexp, karg)) {
            err = "bytecode corruption at opcode " + std::to_string(kexp->opcode);
            return false;
        }
        if (!resolve(karg, err))
            return false;
    }
    return true;
}

struct Group {
    std::vector<std::string> keys;      /* hex of xpu_datum_write output, "" = NULL */
    std::vector<int64_t> n;
    std::vector<__int128> isum;
    std::vector<double> fsum, fsum2, fext;
    std::vector<int> valid;
    std::vector<std::array<double, 5>> fm;  /* stddev: sx, sxx; covar: sx, sxx, sy, syy, sxy */
};

struct RefSess {
    std::vector<char> sess;
    kern_session_info *session;
    kern_multirels *kmrels;
    int nrels;
    std::map<std::pair<uint32_t, std::string>, Group> groups;
    std::vector<std::pair<uint32_t, std::string>> order;
    uint64_t nraw = 0, nin = 0, nout = 0;
    std::string err;
    std::vector<std::string> proj;      /* projected tuples (hex), row id cut off */
};

static std::string hexof(const char *p, int n)
{
    static const char *d = "0123456789abcdef";
    std::string s;
    for (int i = 0; i < n; i++) {
        s += d[((uint8_t)p[i]) >> 4];
        s += d[((uint8_t)p[i]) & 15];
    }
    return s;
}

extern "C" uint32_t ref_hash_any(const void *p, int len) { return pg_hash_any(p, len); }

/* numeric varlena -> kind, weight, value (lo, hi) via the reference */
extern "C" int ref_numeric_decode(const void *vl, int *kind, int *weight, uint64_t *lo, uint64_t *hi)
{
    uint8_t k; int16_t w; int128_t v;
    const char *emsg = __decimal_from_varlena(&k, &w, &v, (const varlena *)vl);
    if (emsg) return -1;
    *kind = k; *weight = w; *lo = (uint64_t)v; *hi = (uint64_t)(v >> 64);
    return 0;
}

extern "C" void *ref_open(const void *session, uint64_t sz, void *kmrels, char *errbuf, int errlen)
{
    RefSess *s = new RefSess();
    s->sess.assign((const char *)session, (const char *)session + sz + 64);
    s->session = (kern_session_info *)s->sess.data();
    s->kmrels = (kern_multirels *)kmrels;
    s->nrels = kmrels ? s->kmrels->num_inner_rels : 0;
    /* resolve every expression (gpu_service.c:3255-3317) */
    uint32_t offs[] = { s->session->xpucode_load_vars_packed, s->session->xpucode_move_vars_packed,
                        s->session->xpucode_scan_quals, s->session->xpucode_join_quals_packed,
                        s->session->xpucode_hash_values_packed, s->session->xpucode_groupby_keyhash,
                        s->session->xpucode_groupby_keyload, s->session->xpucode_groupby_keycomp,
                        s->session->xpucode_groupby_actions, s->session->xpucode_projection };
    for (uint32_t off : offs) {
        if (off && !resolve((kern_expression *)((char *)s->session + off), s->err)) {
            snprintf(errbuf, errlen, "%s", s->err.c_str());
            delete s;
            return NULL;
        }
    }
    kern_varslot_desc *vs = SESSION_KVARS_SLOT_DESC(s->session);
    for (uint32_t i = 0; i < s->session->kcxt_kvars_nslots; i++) {
        vs[i].vs_ops = lookup_type(vs[i].vs_type_code);
        if (!vs[i].vs_ops) {
            snprintf(errbuf, errlen, "unresolved slot type %d", vs[i].vs_type_code);
            delete s;
            return NULL;
        }
    }
    /* inner KDS pointers (host side of KERN_MULTIRELS_INNER_KDS) */
    for (int d = 0; d < s->nrels; d++)
        s->kmrels->chunks[d].kds_in = (kern_data_store *)((char *)s->kmrels + s->kmrels->chunks[d].kds_offset);
    return s;
}

static void group_row(RefSess *s, kern_context *kcxt)
{
    kern_session_info *session = s->session;
    kern_expression *kact = SESSION_KEXP_GROUPBY_ACTIONS(session);
    kern_expression *khash = SESSION_KEXP_GROUPBY_KEYHASH(session);
    kern_expression *karg = KEXP_FIRST_ARG(kact);
    for (uint32_t i = 0; i < kact->nr_args; i++, karg = KEXP_NEXT_ARG(karg)) {
        if (!EXEC_KERN_EXPRESSION(kcxt, karg, NULL)) {
            s->err = "SaveExpr failed";
            return;
        }
    }
    uint32_t hash = 0;
    if (khash) {
        xpu_int4_t h;
        if (!EXEC_KERN_EXPRESSION(kcxt, khash, &h)) { s->err = "key hash failed"; return; }
        hash = (uint32_t)h.value;
    }
    std::string keyid;
    std::vector<std::string> keys;
    int nattrs = kact->u.pagg.nattrs;
    for (int j = 0; j < nattrs; j++) {
        const kern_aggregate_desc *d = &kact->u.pagg.desc[j];
        if (d->action != KAGG_ACTION__VREF) continue;
        xpu_datum_t *x = kcxt->kvars_slot[d->arg0_slot_id];
        if (XPU_DATUM_ISNULL(x)) { keys.push_back(""); keyid += "|N"; continue; }
        char buf[1024];
        int n = x->expr_ops->xpu_datum_write(kcxt, buf, NULL, x);
        keys.push_back(hexof(buf, n));
        keyid += "|" + keys.back();
    }
    auto gk = std::make_pair(hash, keyid);
    auto it = s->groups.find(gk);
    if (it == s->groups.end()) {
        Group g;
        g.keys = keys;
        g.n.assign(nattrs, 0); g.isum.assign(nattrs, 0);
        g.fsum.assign(nattrs, 0.0); g.fsum2.assign(nattrs, 0.0); g.fext.assign(nattrs, 0.0);
        g.valid.assign(nattrs, 0);
        g.fm.assign(nattrs, std::array<double, 5>{0.0, 0.0, 0.0, 0.0, 0.0});
        it = s->groups.emplace(gk, g).first;
        s->order.push_back(gk);
    }
    Group &g = it->second;
    for (int j = 0; j < nattrs; j++) {
        const kern_aggregate_desc *d = &kact->u.pagg.desc[j];
        xpu_datum_t *x = d->arg0_slot_id >= 0 ? kcxt->kvars_slot[d->arg0_slot_id] : NULL;
        bool xn = !x || XPU_DATUM_ISNULL(x);
        switch (d->action) {
        case KAGG_ACTION__NROWS_ANY: g.n[j]++; break;
        case KAGG_ACTION__NROWS_COND: if (!xn) g.n[j]++; break;
        case KAGG_ACTION__PSUM_INT: case KAGG_ACTION__PAVG_INT:
        case KAGG_ACTION__PSUM_INT64: case KAGG_ACTION__PAVG_INT64:
            if (!xn) {
                int64_t v = (x->expr_ops == &xpu_int8_ops) ? ((xpu_int8_t *)x)->value
                          : (x->expr_ops == &xpu_int4_ops) ? ((xpu_int4_t *)x)->value
                          : ((xpu_int2_t *)x)->value;
                g.n[j]++; g.isum[j] += v;
            }
            break;
        case KAGG_ACTION__PSUM_FP: case KAGG_ACTION__PAVG_FP:
            if (!xn) { g.n[j]++; g.fsum[j] += ((xpu_float8_t *)x)->value; }
            break;
        case KAGG_ACTION__PSUM_NUMERIC: case KAGG_ACTION__PAVG_NUMERIC:
            if (!xn) {
                xpu_numeric_t *num = (xpu_numeric_t *)x;
                if (!xpu_numeric_validate(kcxt, num)) { s->err = "numeric"; return; }
                if (num->kind == XPU_NUMERIC_KIND__VALID) {
                    g.n[j]++;
                    g.isum[j] += __normalize_numeric_int128(__numeric_typmod_weight(d->typmod),
                                                            num->weight, num->u.value);
                }
            }
            break;
        case KAGG_ACTION__PMIN_FP64: case KAGG_ACTION__PMAX_FP64:
            if (!xn) {
                double v = ((xpu_float8_t *)x)->value;
                bool take = !g.valid[j] || (d->action == KAGG_ACTION__PMIN_FP64 ? v < g.fext[j] : v > g.fext[j]);
                if (take) g.fext[j] = v;
                g.valid[j] = 1;
            }
            break;
        case KAGG_ACTION__STDDEV:
            /* __update_groupby__pstddev (cuda_gpupreagg.cu:1448-1466):
             * count, sum of x, sum of x*x in FP64; the argument fetched by
             * the reference's __preagg_fetch_xdatum_as_float64 */
            if (x) {
                float8_t v;
                if (__preagg_fetch_xdatum_as_float64(&v, x)) {
                    g.n[j]++; g.fm[j][0] += v; g.fm[j][1] += v * v;
                }
            }
            break;
        case KAGG_ACTION__COVAR: {
            /* __update_groupby__pcovar (cuda_gpupreagg.cu:1470-1492): both
             * arguments fetched, then the five sums */
            xpu_datum_t *y = d->arg1_slot_id >= 0 ? kcxt->kvars_slot[d->arg1_slot_id] : NULL;
            float8_t xv, yv;
            if (x && y && __preagg_fetch_xdatum_as_float64(&xv, x) &&
                __preagg_fetch_xdatum_as_float64(&yv, y)) {
                g.n[j]++;
                g.fm[j][0] += xv; g.fm[j][1] += xv * xv;
                g.fm[j][2] += yv; g.fm[j][3] += yv * yv;
                g.fm[j][4] += xv * yv;
            }
            break;
        }
        case KAGG_ACTION__PMIN_INT32: case KAGG_ACTION__PMIN_INT64:
        case KAGG_ACTION__PMAX_INT32: case KAGG_ACTION__PMAX_INT64:
            /* state printed as [valid, value]: n holds the valid flag */
            if (!xn) {
                int64_t v = (x->expr_ops == &xpu_int8_ops) ? ((xpu_int8_t *)x)->value
                          : (x->expr_ops == &xpu_int4_ops) ? ((xpu_int4_t *)x)->value
                          : ((xpu_int2_t *)x)->value;
                bool is_min = (d->action == KAGG_ACTION__PMIN_INT32 || d->action == KAGG_ACTION__PMIN_INT64);
                bool take = !g.n[j] || (is_min ? v < g.isum[j] : v > g.isum[j]);
                if (take) g.isum[j] = v;
                g.n[j] = 1;
            }
            break;
        default:
            break;
        }
    }
}

/* a projection session's row: its tuple as the reference's own
 * kern_estimate_minimal_tuple / kern_form_minimal_tuple write it into a
 * KDS_FORMAT_ROW kds_dst (execGpuJoinProjection, cuda_gpujoin.cu:754-936) */
static void project_row(RefSess *s, kern_context *kcxt)
{
    kern_session_info *session = s->session;
    const kern_expression *kproj = SESSION_KEXP_PROJECTION(session);
    const kern_data_store *kds_dst = SESSION_KDS_DST_HEAD(session);
    if (!kds_dst) { s->err = "projection without a kds_dst head"; return; }
    int sz = kern_estimate_minimal_tuple(kcxt, kproj, kds_dst);
    if (sz < 0) { s->err = "kern_estimate_minimal_tuple failed"; return; }
    std::vector<uint64_t> buf((sz + 64) / 8 + 1, 0);
    kern_tupitem *titem = (kern_tupitem *)buf.data();
    int len = kern_form_minimal_tuple(kcxt, kproj, kds_dst, titem, (uint32_t)s->proj.size());
    if (len < ROWID_SIZE || len > sz + 8) { s->err = "kern_form_minimal_tuple failed"; return; }
    s->proj.push_back(hexof((const char *)titem, len - ROWID_SIZE));
}

static void process_depth(RefSess *s, kern_context *kcxt, int depth,
                          std::vector<std::vector<char>> &kvecs)
{
    kern_session_info *session = s->session;
    if (depth > s->nrels) {
        s->nout++;
        if (depth > 0) {
            kcxt->kvecs_curr_buffer = kvecs[depth - 1].data();
            kcxt->kvecs_curr_id = 0;
        }
        if (session->xpucode_projection)
            project_row(s, kcxt);
        if (session->xpucode_groupby_actions)
            group_row(s, kcxt);
        return;
    }
    /* expressions of this depth read outer values from the previous depth's kvec */
    kcxt->kvecs_curr_buffer = kvecs[depth - 1].data();
    kcxt->kvecs_curr_id = 0;
    xpu_int4_t hash;
    kern_expression *kh = SESSION_KEXP_HASH_VALUE(session, depth);
    if (!EXEC_KERN_EXPRESSION(kcxt, kh, &hash)) { s->err = "hash value failed"; return; }
    kern_data_store *kds_hash = s->kmrels->chunks[depth - 1].kds_in;
    for (kern_hashitem *hi = KDS_HASH_FIRST_ITEM(kds_hash, hash.value); hi != NULL;
         hi = KDS_HASH_NEXT_ITEM(kds_hash, hi->next)) {
        if (hi->t.hash != (uint32_t)hash.value) continue;
        kcxt->kvecs_curr_buffer = kvecs[depth - 1].data();
        kcxt->kvecs_curr_id = 0;
        if (!ExecLoadVarsMinimalTuple(kcxt, SESSION_KEXP_LOAD_VARS(session, depth), depth, kds_hash, &hi->t)) {
            s->err = "inner load failed"; return;
        }
        int status;
        if (!ExecGpuJoinQuals(kcxt, SESSION_KEXP_JOIN_QUALS(session, depth), &status)) {
            s->err = "join quals failed"; return;
        }
        if (status > 0) {
            /* move this depth's values to its kvec (ExecMoveKernelVariables) */
            if (!ExecMoveKernelVariables(kcxt, SESSION_KEXP_MOVE_VARS(session, depth), kvecs[depth].data(), 0)) {
                s->err = "move vars failed"; return;
            }
            process_depth(s, kcxt, depth + 1, kvecs);
            if (!s->err.empty()) return;
        }
    }
}

extern "C" int ref_exec(void *handle, const kern_data_store *kds, char *errbuf, int errlen)
{
    RefSess *s = (RefSess *)handle;
    kern_session_info *session = s->session;
    kern_context *kcxt;
    INIT_KERNEL_CONTEXT(kcxt, session, NULL);
    std::vector<std::vector<char>> kvecs(s->nrels + 2, std::vector<char>(session->kcxt_kvecs_bufsz + 64));
    if (kds->format == KDS_FORMAT_ARROW) {
        /* Arrow columns: rows by index through the reference's Arrow
         * readers (ExecLoadVarsOuterArrow -> kern_extract_arrow_tuple,
         * xpu_common.cu:1636-1673, :257-378) */
        for (uint32_t i = 0; i < kds->nitems; i++) {
            s->nraw++;
            kcxt_reset(kcxt);
            kcxt->kvecs_curr_buffer = NULL;
            kcxt->kvecs_curr_id = 0;
            if (!ExecLoadVarsOuterArrow(kcxt, SESSION_KEXP_LOAD_VARS(session, 0),
                                        SESSION_KEXP_SCAN_QUALS(session), kds, i)) {
                if (kcxt->errcode) { snprintf(errbuf, errlen, "%s", kcxt->error_message); return -1; }
                continue;
            }
            s->nin++;
            if (!ExecMoveKernelVariables(kcxt, SESSION_KEXP_MOVE_VARS(session, 0), kvecs[0].data(), 0)) {
                snprintf(errbuf, errlen, "move vars at depth 0 failed");
                return -1;
            }
            process_depth(s, kcxt, 1, kvecs);
            if (!s->err.empty() || kcxt->errcode) {
                snprintf(errbuf, errlen, "%s %s", s->err.c_str(),
                         kcxt->error_message ? kcxt->error_message : "");
                return -1;
            }
        }
        return 0;
    }
    if (kds->format == KDS_FORMAT_ROW) {
        /* rows by index as __gpuscan_load_source_row reads them
         * (cuda_gpuscan.cu:646-700): KDS_GET_TUPITEM, the depth-0 load by
         * ExecLoadVarsMinimalTuple, then the scan quals; the rows carry no
         * transaction attributes (the visibility check is device code) */
        kern_expression *kquals = SESSION_KEXP_SCAN_QUALS(session);
        for (uint32_t i = 0; i < kds->nitems; i++) {
            kern_tupitem *titem = KDS_GET_TUPITEM(kds, i);
            if (!titem) continue;
            if (titem->has_xact_attrs) {
                snprintf(errbuf, errlen, "ref harness: row %u carries transaction attributes", i);
                return -1;
            }
            s->nraw++;
            kcxt_reset(kcxt);
            kcxt->kvecs_curr_buffer = NULL;
            kcxt->kvecs_curr_id = 0;
            if (!ExecLoadVarsMinimalTuple(kcxt, SESSION_KEXP_LOAD_VARS(session, 0), 0, kds, titem)) {
                snprintf(errbuf, errlen, "%s", kcxt->errcode ? kcxt->error_message : "row load failed");
                return -1;
            }
            if (kquals) {
                xpu_bool_t ok;
                if (!EXEC_KERN_EXPRESSION(kcxt, kquals, &ok)) {
                    snprintf(errbuf, errlen, "%s", kcxt->error_message ? kcxt->error_message : "quals failed");
                    return -1;
                }
                if (XPU_DATUM_ISNULL(&ok) || !ok.value)
                    continue;
            }
            s->nin++;
            if (!ExecMoveKernelVariables(kcxt, SESSION_KEXP_MOVE_VARS(session, 0), kvecs[0].data(), 0)) {
                snprintf(errbuf, errlen, "move vars at depth 0 failed");
                return -1;
            }
            process_depth(s, kcxt, 1, kvecs);
            if (!s->err.empty() || kcxt->errcode) {
                snprintf(errbuf, errlen, "%s %s", s->err.c_str(),
                         kcxt->error_message ? kcxt->error_message : "");
                return -1;
            }
        }
        return 0;
    }
    if (kds->format != KDS_FORMAT_BLOCK) {
        snprintf(errbuf, errlen, "ref harness handles KDS_FORMAT_BLOCK, KDS_FORMAT_ARROW and KDS_FORMAT_ROW");
        return -1;
    }
    for (uint32_t b = 0; b < kds->nitems; b++) {
        PageHeaderData *page = KDS_BLOCK_PGPAGE(kds, b);
        uint32_t nlp = PageGetMaxOffsetNumber((Page)page);
        for (uint32_t i = 0; i < nlp; i++) {
            ItemIdData *lpp = &page->pd_linp[i];
            if (!ItemIdIsNormal(lpp)) continue;
            HeapTupleHeaderData *htup = (HeapTupleHeaderData *)PageGetItem((Page)page, lpp);
            s->nraw++;
            kcxt_reset(kcxt);
            kcxt->kvecs_curr_buffer = NULL;
            kcxt->kvecs_curr_id = 0;
            if (!ExecLoadVarsOuterHeap(kcxt, SESSION_KEXP_LOAD_VARS(session, 0),
                                       SESSION_KEXP_SCAN_QUALS(session), kds, htup)) {
                if (kcxt->errcode) { snprintf(errbuf, errlen, "%s", kcxt->error_message); return -1; }
                continue;
            }
            s->nin++;
            if (!ExecMoveKernelVariables(kcxt, SESSION_KEXP_MOVE_VARS(session, 0), kvecs[0].data(), 0)) {
                snprintf(errbuf, errlen, "move vars at depth 0 failed");
                return -1;
            }
            process_depth(s, kcxt, 1, kvecs);
            if (!s->err.empty() || kcxt->errcode) {
                snprintf(errbuf, errlen, "%s %s", s->err.c_str(),
                         kcxt->error_message ? kcxt->error_message : "");
                return -1;
            }
        }
    }
    return 0;
}

static std::string i128str(__int128 v)
{
    if (v == 0) return "0";
    bool neg = v < 0;
    unsigned __int128 u = neg ? -(unsigned __int128)v : (unsigned __int128)v;
    std::string s;
    while (u) { s += char('0' + (int)(u % 10)); u /= 10; }
    if (neg) s += '-';
    return std::string(s.rbegin(), s.rend());
}

/* JSON: {"nitems_raw":..,"nitems_in":..,"nitems_out":..,"groups":[{"hash":h,"keys":[hex|null],
 *        "states":[[...],...]}]} ; returns the required length */
extern "C" uint64_t ref_result(void *handle, char *buf, uint64_t bufsz)
{
    RefSess *s = (RefSess *)handle;
    kern_expression *kact = SESSION_KEXP_GROUPBY_ACTIONS(s->session);
    std::string out = "{\"nitems_raw\":" + std::to_string(s->nraw) + ",\"nitems_in\":" +
                      std::to_string(s->nin) + ",\"nitems_out\":" + std::to_string(s->nout) + ",\"rows\":[";
    for (size_t i = 0; i < s->proj.size(); i++)
        out += (i ? ",\"" : "\"") + s->proj[i] + "\"";
    out += "],\"groups\":[";
    bool first = true;
    for (auto &gk : s->order) {
        Group &g = s->groups[gk];
        if (!first) out += ",";
        first = false;
        out += "{\"hash\":" + std::to_string(gk.first) + ",\"keys\":[";
        for (size_t k = 0; k < g.keys.size(); k++) {
            if (k) out += ",";
            out += g.keys[k].empty() ? "null" : "\"" + g.keys[k] + "\"";
        }
        out += "],\"states\":[";
        bool f2 = true;
        for (int j = 0; j < kact->u.pagg.nattrs; j++) {
            const kern_aggregate_desc *d = &kact->u.pagg.desc[j];
            if (d->action == KAGG_ACTION__VREF) continue;
            if (!f2) out += ",";
            f2 = false;
            char tmp[128];
            switch (d->action) {
            case KAGG_ACTION__NROWS_ANY: case KAGG_ACTION__NROWS_COND:
                out += std::to_string(g.n[j]); break;
            case KAGG_ACTION__PSUM_FP: case KAGG_ACTION__PAVG_FP:
                snprintf(tmp, sizeof(tmp), "[%lld,%.17g]", (long long)g.n[j], g.fsum[j]);
                out += tmp; break;
            case KAGG_ACTION__PMIN_FP64: case KAGG_ACTION__PMAX_FP64:
                snprintf(tmp, sizeof(tmp), "[%d,%.17g]", g.valid[j], g.fext[j]);
                out += tmp; break;
            case KAGG_ACTION__STDDEV:
                snprintf(tmp, sizeof(tmp), "[%lld,%.17g,%.17g]", (long long)g.n[j], g.fm[j][0], g.fm[j][1]);
                out += tmp; break;
            case KAGG_ACTION__COVAR: {
                char big[256];
                snprintf(big, sizeof(big), "[%lld,%.17g,%.17g,%.17g,%.17g,%.17g]", (long long)g.n[j],
                         g.fm[j][0], g.fm[j][1], g.fm[j][2], g.fm[j][3], g.fm[j][4]);
                out += big; break;
            }
            default:
                out += "[" + std::to_string(g.n[j]) + ",\"" + i128str(g.isum[j]) + "\"]"; break;
            }
        }
        out += "]}";
    }
    out += "]}";
    if (buf && bufsz > out.size()) memcpy(buf, out.c_str(), out.size() + 1);
    return out.size() + 1;
}

/* the row counters alone (nitems_raw, nitems_in, nitems_out), without
 * writing the groups out: for timing the reference over chunks whose
 * groups are millions */
extern "C" void ref_counts(void *handle, uint64_t *out)
{
    RefSess *s = (RefSess *)handle;
    out[0] = s->nraw;
    out[1] = s->nin;
    out[2] = s->nout;
}

extern "C" void ref_close(void *handle) { delete (RefSess *)handle; }
