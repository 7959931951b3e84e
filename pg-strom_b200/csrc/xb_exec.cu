/*
 * xb_exec.cu
 *
 * B200 (sm_100a) kernels of the scan / hash-join / pre-aggregation path and
 * the C ABI declared in include/xpu_b200.h.
 *
 * Kernels:
 *   xb_build_inner   decodes the inner relation (KDS_FORMAT_HASH, built on
 *                    the host by gpu_join.c:2129-2164) into SoA register
 *                    images and an open-addressing (hash,row) index;
 *   xb_exec_kernel   persistent executor: warps claim heap pages (or Arrow /
 *                    row groups), decode tuples, run scan quals, probe the
 *                    joins depth-first and update the GROUP BY tables.  Heap
 *                    pages of the next claim are prefetched into L2 by the
 *                    TMA engine (cp.async.bulk.prefetch.L2) while the current
 *                    ones are decoded;
 *   xb_final_*       materialise kds_final in the reference layout.
 *
 * Reference counterparts: kern_gpujoin_main (cuda_gpujoin.cu:1050-1279),
 * __gpuscan_load_source_block/_arrow/_row (cuda_gpuscan.cu:405-727),
 * execGpuJoinHashJoin (cuda_gpujoin.cu:304-494), execGpuPreAggGroupBy and
 * friends (cuda_gpupreagg.cu:1112-2326), __writeOutOneTuplePreAgg
 * (cuda_gpupreagg.cu:18-223).
 */
#include <cuda_runtime.h>
#include <algorithm>
#include <deque>
#include <map>
#include <mutex>
#include <thread>
#include <chrono>
#include <tuple>
#include <unordered_map>
#include <vector>
#include <string>
#include <cstring>
#include <cstdio>
#include <cstdlib>
#include <cstdarg>
#include "xb_plan.h"
#include "xb_device.cuh"
#include "xb_exec_dev.cuh"
#include "xb_compile.h"
#include "xb_jit.h"
#include "xb_sort.cuh"
#include "xpu_b200.h"
#include "xb_host.h"
#include "xb_final.h"

/* ================================================================
 * executor kernel
 * ================================================================ */
/* probe cursor of one join depth for the 32 lanes of a warp (shared memory) */
struct XbCursor {
    unsigned long long okey[32];    /* outer key (fused probe comparing a key column) */
    uint32_t pos[32];               /* next index slot to visit */
    uint32_t tag[32];               /* hash value, or the 32-bit key */
    uint32_t live;                  /* lanes whose probe chain may hold more rows */
    uint32_t __pad[3];
};

/* ---------------------------------------------------------------
 * group table access from the register file
 * --------------------------------------------------------------- */

/* do the lane's group keys (registers) equal the entry's key images? */
__device__ __forceinline__ bool
xb_key_match(const xb_plan *plan, const char *e, const XbRegs &R, uint32_t lane)
{
    const xb_keyimg *img = (const xb_keyimg *)(e + plan->gent_keys_off);
    for (uint32_t k = 0; k < plan->nkeys; k++) {
        const xb_key &key = plan->keys[k];
        const xb_keyimg x = img[k];
        const bool rn = RISNULL(R, key.reg) != 0;
        if (x.isnull || rn) {
            if (!(x.isnull && rn))
                return false;
            continue;
        }
        const uint64_t v = RVAL(R, key.reg);
        if (x.val == v && (key.rk != XB_RK_TEXT || x.len == RAUX(R, key.reg)))
            continue;               /* same bits, or the same key bytes */
        if (key.rk == XB_RK_TEXT) {
            if (x.len != RAUX(R, key.reg) ||
                !xb_bytes_eq_ool((const uint8_t *)x.val, (const uint8_t *)v, x.len))
                return false;
        } else if (key.rk == XB_RK_NUM) {
            int err = 0;
            if (xb_numeric_cmp((const uint8_t *)x.val, (const uint8_t *)v, &err) != 0 || err)
                return false;
        } else {
            return false;
        }
    }
    return true;
}

/*
 * Claim an EMPTY entry for the lane's group: 0 = another lane claimed it
 * first, 1 = claimed and published READY, 2 = claimed but the key bytes
 * did not fit the arena (error raised).  Rare, so out of line.
 */
__device__ __noinline__ int
xb_group_claim(const xb_plan *plan, char *e, XbRegs R, uint32_t hash,
               xb_gtable *gt, xb_status *st)
{
    const uint32_t lane = xb_lane();
    xb_gent_head *h = (xb_gent_head *)e;
    if (atomicCAS(&h->state, XB_GSTATE_EMPTY, XB_GSTATE_BUSY) != XB_GSTATE_EMPTY)
        return 0;
    h->hash = hash;
    xb_keyimg *img = (xb_keyimg *)(e + plan->gent_keys_off);
    bool ok = true;
    for (uint32_t k = 0; k < plan->nkeys; k++) {
        const xb_key &key = plan->keys[k];
        xb_keyimg src;
        src.isnull = RISNULL(R, key.reg);
        src.val = RVAL(R, key.reg);
        src.len = RAUX(R, key.reg);
        ok &= xb_key_store(key, src, &img[k], gt, st);
    }
    xb_init_states(plan, e);
    if (gt) {
        xb_gt_count_new(gt);
        xb_st_release(&h->state, XB_GSTATE_READY);
    } else {
        xb_st_release_cta(&h->state, XB_GSTATE_READY);
    }
    return ok ? 1 : 2;
}

/*
 * Find or create the lane's group entry: the shared-memory table (SMEM,
 * gt == nullptr; entries visible to this CTA only) or the global table.
 * Returns nullptr when the table is full (*full) or on an error.
 */
template <bool SMEM>
__device__ __forceinline__ char *
xb_group_get(const xb_plan *plan, const XbRegs &R, uint32_t lane, char *entries,
             uint64_t cap_mask, uint32_t hash, xb_gtable *gt, xb_status *st, bool *full)
{
    const uint32_t gsz = plan->gent_size;
    uint64_t pos = hash & cap_mask;
    const uint64_t limit = SMEM ? cap_mask : (cap_mask < XB_PROBE_LIMIT ? cap_mask : XB_PROBE_LIMIT);
    for (uint64_t probe = 0; probe <= limit; probe++) {
        char *e = entries + pos * gsz;
        xb_gent_head *h = (xb_gent_head *)e;
        uint32_t s = SMEM ? xb_ld_acquire_cta(&h->state) : xb_ld_acquire(&h->state);
        if (s == XB_GSTATE_EMPTY) {
            const int rc = xb_group_claim(plan, e, R, hash, gt, st);
            if (rc == 1)
                return e;
            if (rc == 2)
                return nullptr;
            s = SMEM ? xb_ld_acquire_cta(&h->state) : xb_ld_acquire(&h->state);
        }
        uint32_t spins = 0;
        while (s == XB_GSTATE_BUSY) {
            if (++spins > plan->wait_limit) {
                XB_RAISE(st, ERRCODE_DEVICE_ERROR, XB_MSG_WAIT_TIMEOUT);
                return nullptr;
            }
            __nanosleep(20);
            s = SMEM ? xb_ld_acquire_cta(&h->state) : xb_ld_acquire(&h->state);
        }
        if (h->hash == hash && xb_key_match(plan, e, R, lane))
            return e;
        pos = (pos + 1) & cap_mask;
    }
    *full = true;
    return nullptr;
}

/* per-lane update of the actions that are not combined across a warp */
__device__ __forceinline__ void
xb_update_one(const xb_agg &a, char *s, const XbRegs &R, uint32_t lane, const uint8_t *rk,
              xb_status *st)
{
    if (RISNULL(R, a.arg0))
        return;
    const uint64_t v0 = RVAL(R, a.arg0);
    switch (a.action) {
    case KAGG_ACTION__PSUM_NUMERIC:
    case KAGG_ACTION__PAVG_NUMERIC:
        xb_agg_numeric_add(s, (const uint8_t *)v0, a.weight, st);
        break;
    case KAGG_ACTION__STDDEV:
        xb_agg_stddev_add(s, xb_reg_f64(v0, rk[a.arg0]));
        break;
    case KAGG_ACTION__COVAR:
        if (!RISNULL(R, a.arg1))
            xb_agg_covar_add(s, xb_reg_f64(v0, rk[a.arg0]), xb_reg_f64(RVAL(R, a.arg1), rk[a.arg1]));
        break;
    default:
        break;
    }
}

/*
 * __updateOneTupleGroupBy + __update_groupby__* (cuda_gpupreagg.cu:1196-1605)
 * for a warp: lanes whose rows fall into the same group entry are combined
 * first (the lowest such lane sums, counts, mins or maxes its peers' values
 * from the register file) and one atomic per state field is issued per
 * distinct group.  Numeric sums and the variance families stay per lane.
 * All lanes call this; e == nullptr for lanes without a row.
 */
__device__ __forceinline__ void
xb_update_states_warp(const xb_plan *plan, char *e, const XbRegs &R, uint32_t lane, xb_status *st)
{
    const uint32_t peers = __match_any_sync(XB_FULL, (unsigned long long)e);
    const bool leader = e != nullptr && (uint32_t)(__ffs(peers) - 1) == lane;
    for (uint32_t i = 0; i < plan->naggs; i++) {
        const xb_agg &a = plan->aggs[i];
        if (a.state_sz == 0 || !e)
            continue;
        char *s = e + a.state_off;
        const uint32_t act = a.action;
        const bool combined = !(act == KAGG_ACTION__PSUM_NUMERIC || act == KAGG_ACTION__PAVG_NUMERIC ||
                                act == KAGG_ACTION__STDDEV || act == KAGG_ACTION__COVAR);
        if (!combined) {
            if (a.filter >= 0 && (RISNULL(R, a.filter) || RVAL(R, a.filter) == 0))
                continue;
            xb_update_one(a, s, R, lane, plan->rk, st);
            continue;
        }
        if (!leader)
            continue;
        const bool flt = a.arg0 >= 0 && plan->rk[a.arg0] == XB_RK_FLT;
        const uint32_t nm0 = a.arg0 >= 0 ? R.nullm[a.arg0] : XB_FULL;
        const uint32_t nmf = a.filter >= 0 ? R.nullm[a.filter] : 0;
        unsigned long long cnt = 0;
        xb_i128 isum = 0;
        double fs = 0.0, fc = 0.0;
        long long mn = INT64_MAX, mx = INT64_MIN;
        for (uint32_t m = peers; m; m &= m - 1) {
            const uint32_t p = __ffs(m) - 1;
            if (a.filter >= 0 && (((nmf >> p) & 1u) || R.val[a.filter * 32 + p] == 0))
                continue;
            if (act == KAGG_ACTION__NROWS_ANY) {
                cnt++;
                continue;
            }
            if ((nm0 >> p) & 1u)
                continue;
            const uint64_t v = R.val[a.arg0 * 32 + p];
            cnt++;
            switch (act) {
            case KAGG_ACTION__PMIN_INT32: case KAGG_ACTION__PMIN_INT64:
                mn = min(mn, (long long)v);
                break;
            case KAGG_ACTION__PMAX_INT32: case KAGG_ACTION__PMAX_INT64:
                mx = max(mx, (long long)v);
                break;
            case KAGG_ACTION__PMIN_FP64:
                mn = min(mn, (long long)xb_f64_ordered(xb_reg_f64(v, plan->rk[a.arg0])));
                break;
            case KAGG_ACTION__PMAX_FP64:
                mx = max(mx, (long long)xb_f64_ordered(xb_reg_f64(v, plan->rk[a.arg0])));
                break;
            case KAGG_ACTION__PSUM_INT: case KAGG_ACTION__PAVG_INT:
            case KAGG_ACTION__PSUM_INT64: case KAGG_ACTION__PAVG_INT64:
                isum += (xb_i128)(int64_t)v;
                break;
            case KAGG_ACTION__PSUM_FP: case KAGG_ACTION__PAVG_FP: {
                /* TwoSum: fs + fc carries the peers' sum exactly up to fc's rounding */
                const double x = flt ? __longlong_as_double(v) : (double)(int64_t)v;
                const double t = __dadd_rn(fs, x);
                const double bp = __dsub_rn(t, fs);
                fc += __dadd_rn(__dsub_rn(fs, __dsub_rn(t, bp)), __dsub_rn(x, bp));
                fs = t;
                break;
            }
            default:
                break;
            }
        }
        if (cnt == 0)
            continue;
        switch (act) {
        case KAGG_ACTION__NROWS_ANY:
        case KAGG_ACTION__NROWS_COND:
            atomicAdd((unsigned long long *)s, cnt);
            break;
        case KAGG_ACTION__PMIN_INT32: case KAGG_ACTION__PMIN_INT64: case KAGG_ACTION__PMIN_FP64:
            atomicOr((unsigned int *)(s + 8), 1u);
            atomicMin((long long *)s, mn);
            break;
        case KAGG_ACTION__PMAX_INT32: case KAGG_ACTION__PMAX_INT64: case KAGG_ACTION__PMAX_FP64:
            atomicOr((unsigned int *)(s + 8), 1u);
            atomicMax((long long *)s, mx);
            break;
        case KAGG_ACTION__PSUM_INT: case KAGG_ACTION__PAVG_INT:
            atomicAdd((unsigned long long *)s, cnt);
            atomicAdd((unsigned long long *)(s + 8), (unsigned long long)(uint64_t)isum);
            break;
        case KAGG_ACTION__PSUM_INT64: case KAGG_ACTION__PAVG_INT64:
            atomicAdd((unsigned long long *)s, cnt);
            xb_atomic_add_i128((uint64_t *)(s + 8), isum);
            break;
        case KAGG_ACTION__PSUM_FP: case KAGG_ACTION__PAVG_FP:
            atomicAdd((unsigned long long *)s, cnt);
            xb_atomic_add_f64c((double *)(s + 8), (double *)(s + 16), fs);
            if (fc != 0.0)
                atomicAdd((double *)(s + 16), fc);
            break;
        default:
            break;
        }
    }
}

/* ---------------------------------------------------------------
 * hash-join probe cursors
 * --------------------------------------------------------------- */

/* start depth-d probes for the lanes with 'live' set */
__device__ __forceinline__ void
xb_cursor_start(const xb_inner *in, XbCursor *cu, uint32_t lane, bool live,
                uint32_t hash, uint32_t tag, uint64_t okey)
{
    cu->pos[lane] = hash & in->cap_mask;
    cu->tag[lane] = tag;
    cu->okey[lane] = okey;
    cu->live = __ballot_sync(XB_FULL, live && in->nitems > 0);
}

/* fused probe: hash the outer key register inline (HashValue of one
 * int-family Var, xpu_basetype.cu datum_hash + pg_hash_merge) */
__device__ __forceinline__ void
xb_cursor_start_fused(const xb_inner *in, XbCursor *cu, const XbRegs &R, uint32_t lane, uint32_t mask)
{
    const uint32_t ox = in->fast_outer;
    const uint64_t okey = RVAL(R, ox);
    bool live = ((mask >> lane) & 1u) && !RISNULL(R, ox);   /* NULL = anything is never true */
    uint32_t hv;
    switch (in->fast_hk) {
    case XB_HK_W1: hv = xb_hash_u32((uint32_t)okey, 1); break;
    case XB_HK_W2: hv = xb_hash_u32((uint32_t)okey, 2); break;
    case XB_HK_W4: hv = xb_hash_u32((uint32_t)okey, 4); break;
    default:       hv = xb_hash_u64(okey); break;
    }
    const uint32_t hash = xb_hash_merge(0xffffffffU, hv) ^ 0xffffffffU;
    uint32_t tag = hash;
    if (in->key32) {
        tag = (uint32_t)okey;
        if ((int64_t)okey != (int64_t)(int32_t)okey)
            live = false;               /* outside any 32-bit inner key */
    }
    xb_cursor_start(in, cu, lane, live, hash, tag, okey);
}

/* next candidate inner row of every live lane; returns the lanes that got one */
__device__ __forceinline__ uint32_t
xb_cursor_next(const xb_inner *in, XbCursor *cu, uint32_t lane, uint32_t *p_row)
{
    bool live = (cu->live >> lane) & 1u;
    bool got = false;
    uint32_t row = 0;
    if (live) {
        const int fast = in->fast_key;
        const uint64_t *kcol = (fast >= 0 && !in->key32) ? in->vals + (size_t)fast * in->nitems : nullptr;
        const uint32_t *kn = (kcol && ((in->hasnull >> fast) & 1u))
                             ? in->nulls + (size_t)fast * ((in->nitems + 31) / 32) : nullptr;
        const uint32_t cap_mask = in->cap_mask;
        const uint32_t tag = cu->tag[lane];
        const uint64_t okey = cu->okey[lane];
        uint32_t pos = cu->pos[lane];
        for (uint32_t probe = 0; probe <= cap_mask; probe++) {
            const uint64_t ent = __ldg((const unsigned long long *)&in->index[pos]);
            pos = (pos + 1) & cap_mask;
            if (ent == 0) { live = false; break; }
            if ((uint32_t)(ent >> 32) != tag)
                continue;
            const uint32_t r = (uint32_t)ent - 1;
            if (in->unique_hash)
                live = false;           /* no other inner row has this tag */
            if (kcol) {
                const bool knull = kn && ((__ldg(&kn[r / 32]) >> (r % 32)) & 1u);
                if (knull || __ldg((const unsigned long long *)&kcol[r]) != okey) {
                    if (!live) break;
                    continue;
                }
            }
            row = r;
            got = true;
            break;
        }
        cu->pos[lane] = pos;
    }
    cu->live = __ballot_sync(XB_FULL, live);
    *p_row = row;
    return __ballot_sync(XB_FULL, got);
}

/* copy the live pre-decoded inner columns of row 'row' into the registers
 * of the lanes in 'cand' (other lanes read NULL) */
__device__ __forceinline__ void
xb_load_inner(const xb_inner *in, const XbRegs &R, const uint8_t *rk, uint32_t lane,
              uint32_t cand, uint32_t row)
{
    const bool mine = (cand >> lane) & 1u;
    const uint32_t n = in->nitems;
    const uint32_t words = (n + 31) / 32;
    const uint32_t live = in->live, hasnull = in->hasnull, hashed = in->hashed;
    for (uint32_t k = 0; k < in->nloads; k++) {
        if (!((live >> k) & 1u))
            continue;
        const uint32_t reg = in->load[k].reg;
        bool isnull = !mine;
        if (mine) {
            RVAL(R, reg) = __ldg((const unsigned long long *)&in->vals[(size_t)k * n + row]);
            if (rk[reg] == XB_RK_TEXT)
                RAUX(R, reg) = __ldg(&in->auxs[(size_t)k * n + row]);
            if ((hashed >> k) & 1u)
                RHC(R, reg) = __ldg(&in->hashes[(size_t)k * n + row]);
            if ((hasnull >> k) & 1u)
                isnull = (__ldg(&in->nulls[(size_t)k * words + row / 32]) >> (row % 32)) & 1u;
        }
        xb_set_null(R, reg, isnull);
    }
}

/* lanes of 'mask' where program p's result is TRUE (all of mask if p is empty) */
__device__ __forceinline__ uint32_t
xb_prog_pass(const xb_prog &p, const XbRegs &R, uint32_t lane, uint32_t mask)
{
    if (!p.count)
        return mask;
    const bool ok = ((mask >> lane) & 1u) && !RISNULL(R, p.result) && RVAL(R, p.result) != 0;
    return __ballot_sync(XB_FULL, ok);
}

/* decode one heap tuple (HeapTupleHeaderData at htup, lp_len len) */
__device__ __forceinline__ bool
xb_decode_heap(const xb_plan *plan, const XbSrcMeta *meta, const XbRegs &R, uint32_t lane,
               const uint8_t *htup, uint32_t len, uint32_t *nullbits)
{
    const uint16_t infomask2 = (uint16_t)xb_fetch_le(htup + 18, 2);
    const uint16_t infomask = (uint16_t)xb_fetch_le(htup + 20, 2);
    const uint32_t t_hoff = htup[22];
    const int natts_raw = infomask2 & HEAP_NATTS_MASK;
    if (t_hoff < SizeofHeapTupleHeader || t_hoff > len)
        return false;
    if (meta->fixed && !(infomask & HEAP_HASNULL) && natts_raw >= plan->max_resno0 &&
        len - t_hoff >= meta->fixed_end) {
        /* attcacheoff fast path: every loaded column sits at a known offset */
        const uint8_t *payload = htup + t_hoff;
        for (uint32_t i = 0; i < plan->nload0; i++) {
            const XbFix f = meta->fix[i];
            xb_load_datum(f.ld, payload + f.off, &RVAL(R, f.reg), &RAUX(R, f.reg));
        }
        *nullbits = 0;
        return true;
    }
    int natts = natts_raw < meta->ncols ? natts_raw : meta->ncols;
    const uint8_t *nullmap = (infomask & HEAP_HASNULL) ? htup + SizeofHeapTupleHeader : nullptr;
    if (nullmap && SizeofHeapTupleHeader + (natts + 7) / 8 > t_hoff)
        return false;
    return xb_decode_tuple(meta->cols, natts, nullmap, htup + t_hoff, len - t_hoff,
                           plan->load0, plan->nload0, R.val + lane, R.aux + lane, 32, false, nullbits);
}

/*
 * Decode the next batch of up to 32 source rows into the register file.
 * Returns the lanes holding a row; *done when the warp has no more work,
 * *failed on corrupt input (error raised).
 */
__device__ __forceinline__ uint32_t
xb_fetch_batch(const XbExecArgs &args, const xb_plan *plan, const XbSrcMeta *meta,
               const XbRegs &R, XbSrc &s, uint32_t lane, XbWarpState *ws, bool *done, bool *failed)
{
    while (s.item >= s.nitems) {
        const int rc = xb_next_unit(args, s, lane);
        if (rc == 0) { *done = true; return 0; }
        if (rc == 2) {
            if (lane == 0) XB_RAISE(args.st, ERRCODE_DEVICE_ERROR, XB_MSG_BAD_PAGE);
            *failed = true;
            return 0;
        }
    }
    const uint32_t idx = s.item + lane;
    s.item += 32;
    bool exists = false, ok = false;
    uint32_t nullbits = 0;
    if (idx < s.nitems) {
        if (args.format == KDS_FORMAT_BLOCK) {
            const uint32_t lp = (uint32_t)xb_fetch_le(s.page + SizeOfPageHeaderData + 4 * idx, 4);
            if (ITEMID_FLAGS(lp) == LP_NORMAL) {
                const uint32_t off = ITEMID_OFF(lp), len = ITEMID_LEN(lp);
                exists = true;
                if (off >= SizeOfPageHeaderData && len >= SizeofHeapTupleHeader &&
                    off + len <= PGSTROM_BLCKSZ)
                    ok = xb_decode_heap(plan, meta, R, lane, s.page + off, len, &nullbits);
            }
        } else if (args.format == KDS_FORMAT_ARROW) {
            const uint32_t row = s.row0 + idx;
            exists = true;
            ok = true;
            for (uint32_t i = 0; i < plan->nload0; i++) {
                const xb_load &ldd = plan->load0[i];
                bool isnull = true;
                if (ldd.resno <= (int)s.kds->ncols) {
                    const kern_colmeta *cm = &s.kds->colmeta[ldd.resno - 1];
                    if (!xb_arrow_load(s.kds, cm, row, ldd.ld, &RVAL(R, ldd.reg), &RAUX(R, ldd.reg), &isnull)) {
                        ok = false;
                        XB_RAISE(args.st, ERRCODE_DEVICE_ERROR, XB_MSG_ARROW_TYPE);
                        break;
                    }
                }
                if (isnull) nullbits |= 1u << i;
            }
        } else {
            const kern_data_store *kds = s.kds;
            const uint64_t *rowindex = (const uint64_t *)((const char *)kds + KDS_HEAD_LENGTH(kds)) + kds->hash_nslots;
            const uint64_t off = rowindex[s.row0 + idx];
            if (off != 0) {
                exists = true;
                if (off <= kds->length && ((kds->length - off) & 7) == 0) {
                    const uint8_t *t = (const uint8_t *)kds + kds->length - off;
                    const kern_tupitem *ti = (const kern_tupitem *)t;
                    const uint32_t pay = (uint32_t)ti->t_hoff - MINIMAL_TUPLE_OFFSET;
                    int natts = ti->t_infomask2 & HEAP_NATTS_MASK;
                    if (natts > meta->ncols) natts = meta->ncols;
                    const bool hasnull = (ti->t_infomask & HEAP_HASNULL) != 0;
                    if (!ti->has_xact_attrs && ti->t_hoff >= MINIMAL_TUPLE_OFFSET + 15 &&
                        pay <= ti->t_len && off >= ti->t_len &&
                        (!hasnull || 15u + (natts + 7) / 8 <= pay))
                        ok = xb_decode_tuple(meta->cols, natts, hasnull ? ti->t_bits : nullptr,
                                             t + pay, ti->t_len - pay, plan->load0, plan->nload0,
                                             R.val + lane, R.aux + lane, 32, false, &nullbits);
                }
            }
        }
        if (exists && !ok && args.format != KDS_FORMAT_ARROW)
            XB_RAISE(args.st, ERRCODE_DEVICE_ERROR, XB_MSG_BAD_TUPLE);
    }
    const uint32_t ex = __ballot_sync(XB_FULL, exists);
    if (lane == 0)
        ws->raw += __popc(ex);
    if (__any_sync(XB_FULL, exists && !ok)) {
        *failed = true;
        return 0;
    }
    for (uint32_t i = 0; i < plan->nload0; i++)
        xb_set_null(R, plan->load0[i].reg, !ok || ((nullbits >> i) & 1u));
    return __ballot_sync(XB_FULL, ok);
}

/*
 * The executor: one persistent launch per batch of chunks.  Each warp runs
 * the GpuScan / GpuJoin / GpuPreAgg pipeline of kern_gpujoin_main
 * (cuda_gpujoin.cu:1050) as a depth state machine over 32-row batches:
 *
 *   FETCH   decode the next batch (heap page items, Arrow rows, ROW tuples),
 *           run the scan quals                               depth 0
 *   ENTER   start the hash probes of depth d for the passing lanes
 *           (fused inline hash, or the HashValue program)    depth 1..n
 *   PROBE   next candidate inner row per lane, load its pre-decoded
 *           columns, run the join quals, descend on success; when no lane
 *           has a candidate left, return to depth d-1
 *   d > n   group-by: arguments + key hash program, group-table find or
 *           create, warp-combined state updates
 *
 * Every program runs through the single interpreter call site of the loop.
 *
 * Shared memory of a CTA:
 *   [plan copy: header + used code][XbSrcMeta][group table]
 *   [per warp: XbWarpState, XbCursor[nrels], register file]
 */
#define XB_ST_FETCH     0
#define XB_ST_ENTER     1
#define XB_ST_PROBE     2

/* one launch's (or one mixed-launch command's) work for this CTA; ends
 * with the CTA's counters and shared group table flushed, without a final
 * barrier */
__device__ __forceinline__ void
xb_exec_body(const XbExecArgs &args, char *smem)
{
    const uint32_t lane = threadIdx.x & 31;
    const uint32_t warp = threadIdx.x >> 5;

    xb_plan *plan = (xb_plan *)smem;
    XbSrcMeta *meta = (XbSrcMeta *)(smem + args.plan_bytes);
    char *sm_entries = (char *)meta + ((sizeof(XbSrcMeta) + 15) & ~(size_t)15);
    const size_t sm_bytes = (size_t)args.sm_cap * args.plan->gent_size;
    char *wbase = sm_entries + sm_bytes + (size_t)warp * args.warp_bytes;
    XbWarpState *ws = (XbWarpState *)wbase;
    const uint32_t nrels_arg = args.plan->nrels;
    XbCursor *cursors = (XbCursor *)(wbase + XB_WARP_HEAD);   /* cursors[d - 1] */

    /* stage the plan (and only the VM code it uses) in shared memory */
    {
        const uint4 *src = (const uint4 *)args.plan;
        uint4 *dst = (uint4 *)plan;
        for (uint32_t i = threadIdx.x; i < args.plan_bytes / 16; i += blockDim.x)
            dst[i] = src[i];
    }
    /* all chunks of a launch share one column layout (checked by the host) */
    xb_setup_meta(args, meta);
    for (size_t i = threadIdx.x; i < sm_bytes / 4; i += blockDim.x)
        ((uint32_t *)sm_entries)[i] = 0;
    for (size_t i = lane; i < XB_WARP_HEAD / 4; i += 32)
        ((uint32_t *)ws)[i] = 0;
    __syncthreads();

    const XbRegs R = xb_regs_setup(wbase + XB_WARP_HEAD + sizeof(XbCursor) * nrels_arg, plan->nregs);
    for (uint32_t r = lane; r < plan->nregs; r += 32)
        R.nullm[r] = XB_FULL;
    if (lane == 0)
        for (uint32_t d = 0; d < nrels_arg; d++)
            cursors[d].live = 0;
    __syncwarp();

    char *const sm_tab = args.sm_cap ? sm_entries : nullptr;
    const uint32_t sm_mask = args.sm_cap ? args.sm_cap - 1 : 0;
    xb_gtable *const gt = args.gt;
    xb_status *const st = args.st;
    const uint32_t nrels = plan->nrels;

    XbSrc src;
    xb_src_start(args, src, lane);

    uint32_t stage = XB_ST_FETCH, d = 0, mask = 0;
    for (;;) {
        const xb_prog *prog;
        if (stage == XB_ST_FETCH) {
            if (args.left_out && __shfl_sync(XB_FULL, xb_grow_flag(args, lane), 0)) {
                /* the table is to grow: leave the rest for the resume launch */
                xb_src_leave(args, src, lane, src.item, src.nitems);
                break;
            }
            bool done = false, failed = false;
            mask = xb_fetch_batch(args, plan, meta, R, src, lane, ws, &done, &failed);
            if (done || failed)
                break;
            if (!mask)
                continue;
            prog = &plan->scan_quals;
        } else if (stage == XB_ST_ENTER) {
            if (d > nrels) {
                if (lane == 0)
                    ws->out += __popc(mask);
                if (!plan->has_groupby && !plan->has_proj) {
                    d = nrels;
                    stage = nrels ? XB_ST_PROBE : XB_ST_FETCH;
                    continue;
                }
                prog = plan->has_proj ? &plan->proj_all : &plan->gb_all;
            } else {
                const xb_inner *in = &plan->inner[d];
                if (in->fast_key >= 0) {
                    xb_cursor_start_fused(in, &cursors[d - 1], R, lane, mask);
                    stage = XB_ST_PROBE;
                    continue;
                }
                prog = &plan->hash_value[d];
            }
        } else {
            uint32_t row;
            const xb_inner *in = &plan->inner[d];
            const uint32_t cand = xb_cursor_next(in, &cursors[d - 1], lane, &row);
            if (!cand) {
                d--;
                stage = d ? XB_ST_PROBE : XB_ST_FETCH;
                continue;
            }
            xb_load_inner(in, R, plan->rk, lane, cand, row);
            mask = cand;
            prog = &plan->join_quals[d];
        }

        /* the interpreter call site */
        if (prog->count && !xb_vm_exec(plan->insns + prog->start, prog->count, R, mask, st))
            break;

        if (stage == XB_ST_FETCH) {
            const uint32_t pass = xb_prog_pass(*prog, R, lane, mask);
            if (lane == 0)
                ws->in += __popc(pass);
            if (pass) {
                d = 1;
                mask = pass;
                stage = XB_ST_ENTER;
            }
        } else if (stage == XB_ST_ENTER) {
            if (d > nrels && plan->has_proj) {
                /* projection: each passing lane writes one row into kds_dst */
                uint64_t pv[XB_MAX_PROJ];
                uint32_t pa[XB_MAX_PROJ];
                uint32_t pn = 0;
                for (uint32_t j = 0; j < plan->proj_nattrs; j++) {
                    const uint32_t r = plan->proj[j].reg;
                    pv[j] = RVAL(R, r);
                    pa[j] = RAUX(R, r);
                    if (RISNULL(R, r))
                        pn |= 1u << j;
                }
                const uint32_t ph = plan->proj_hashed ? (uint32_t)RVAL(R, plan->proj_hash.result) : 0;
                if ((mask >> lane) & 1u)
                    xb_proj_emit(plan, args.dst, args.dst_len, pv, pa, pn, ph, st);
                __syncwarp();
                d = nrels;
                stage = nrels ? XB_ST_PROBE : XB_ST_FETCH;
            } else if (d > nrels) {
                /* group-by: find or create each lane's group, then update */
                const uint32_t hash = plan->has_groupby == 1 ? (uint32_t)RVAL(R, plan->gb_keyhash.result) : 0;
                char *e = nullptr;
                bool bad = false;
                if ((mask >> lane) & 1u) {
                    bool full = false;
                    if (sm_tab)
                        e = xb_group_get<true>(plan, R, lane, sm_tab, sm_mask, hash, nullptr, st, &full);
                    if (!e) {
                        full = false;
                        e = xb_group_get<false>(plan, R, lane, gt->entries, gt->cap_mask, hash, gt, st, &full);
                        if (!e && full) {
                            /* no room: an entry of the dump region */
                            char *slot = xb_dump_slot(gt, plan->gent_size);
                            if (slot) {
                                full = false;
                                e = xb_group_get<false>(plan, R, lane, slot, 0, hash, gt, st, &full);
                            }
                        }
                        if (!e && full) {
                            XB_RAISE(st, ERRCODE_SUSPEND_NO_SPACE, XB_MSG_GTABLE_FULL);
                            atomicOr(&gt->overflow, 1u);
                        }
                    }
                    bad = (e == nullptr);
                }
                if (__any_sync(XB_FULL, bad))
                    break;
                xb_update_states_warp(plan, e, R, lane, st);
                d = nrels;
                stage = nrels ? XB_ST_PROBE : XB_ST_FETCH;
            } else {
                const xb_inner *in = &plan->inner[d];
                const uint32_t hash = (uint32_t)RVAL(R, prog->result);
                xb_cursor_start(in, &cursors[d - 1], lane, (mask >> lane) & 1u, hash, hash, 0);
                stage = XB_ST_PROBE;
            }
        } else {
            const uint32_t ok = xb_prog_pass(*prog, R, lane, mask);
            if (lane == 0)
                ws->depth[d] += __popc(ok);
            if (ok) {
                d++;
                mask = ok;
                stage = XB_ST_ENTER;
            }
        }
    }

    /* per-warp statistics */
    if (lane == 0) {
        atomicAdd((unsigned long long *)&st->nitems_raw, ws->raw);
        atomicAdd((unsigned long long *)&st->nitems_in, ws->in);
        atomicAdd((unsigned long long *)&st->nitems_out, ws->out);
        for (uint32_t dd = 1; dd <= nrels && dd <= XB_MAX_DEPTH; dd++)
            atomicAdd((unsigned long long *)&st->nitems_depth[dd], ws->depth[dd]);
    }
    __syncthreads();

    /* merge the shared-memory group table into the global table */
    if (args.sm_cap) {
        for (uint32_t i = threadIdx.x; i < args.sm_cap; i += blockDim.x) {
            char *e = sm_entries + (size_t)i * plan->gent_size;
            const xb_gent_head *h = (const xb_gent_head *)e;
            if (h->state != XB_GSTATE_READY)
                continue;
            const xb_keyimg *img = (const xb_keyimg *)(e + plan->gent_keys_off);
            char *g = xb_group_find_or_dump(plan, gt, h->hash, img, st);
            if (g)
                xb_merge_states(plan, g, e);
        }
    }
}

__global__ void __launch_bounds__(XB_BLOCK, XB_MIN_BLOCKS)
xb_exec_kernel(const __grid_constant__ XbExecArgs args)
{
    extern __shared__ __align__(16) char smem[];
    xb_exec_body(args, smem);
}

/*
 * Mixed launch: commands of many sessions (each one chunk, its own plan,
 * group table and status) in one persistent kernel fed from a device work
 * queue.  Work item i sends a CTA to command items[i]: it stages that
 * command's plan and column layout, claims the command's units
 * dynamically with the other CTAs that joined it until none is left,
 * merges its shared group table into the command's table and takes the
 * next item.  A large command is listed several times so that several CTAs
 * join it; items are ordered largest command first.
 */
__global__ void __launch_bounds__(XB_BLOCK, XB_MIN_BLOCKS)
xb_mixed_kernel(const __grid_constant__ XbMixArgs m)
{
    extern __shared__ __align__(16) char smem[];
    __shared__ XbExecArgs cmd;
    __shared__ uint32_t item;
    for (;;) {
        if (threadIdx.x == 0) {
            item = atomicAdd(m.cursor, 1u);
            if (item < m.nitems)
                cmd = m.cmds[m.items[item]];
        }
        __syncthreads();
        if (item >= m.nitems)
            break;
        xb_exec_body(cmd, smem);
        __syncthreads();
    }
}

/* ================================================================
 * inner relation build
 * ================================================================ */
struct XbBuildArgs {
    const kern_data_store *kds;     /* KDS_FORMAT_HASH inner buffer (device) */
    xb_inner       *in;             /* device copy of the plan's inner descriptor */
    const xb_plan  *plan;           /* device plan: code of the build-time quals */
    xb_status      *st;
};

/*
 * Decode an inner relation into SoA register images and insert its rows
 * into the hash index.  Warps take 32 rows at a time; when the depth has
 * join quals over the inner row alone (xb_inner.build_qual), they run here
 * through the interpreter on a per-warp register file in dynamic shared
 * memory and only passing rows are indexed.
 */
__global__ void __launch_bounds__(XB_BLOCK)
xb_build_inner(XbBuildArgs args)
{
    __shared__ XbCol cols[XB_MAX_COLS];
    extern __shared__ __align__(16) char bregs[];
    const kern_data_store *kds = args.kds;
    xb_inner *in = args.in;
    const uint32_t lane = threadIdx.x & 31;
    const uint32_t warp = threadIdx.x >> 5;
    const int ncols = kds->ncols < XB_MAX_COLS ? (int)kds->ncols : XB_MAX_COLS;
    for (int i = threadIdx.x; i < ncols; i += blockDim.x) {
        cols[i].attlen = kds->colmeta[i].attlen;
        cols[i].attalign = kds->colmeta[i].attalign > 0 ? kds->colmeta[i].attalign : 1;
        cols[i].attcacheoff = kds->colmeta[i].attcacheoff;
    }
    const xb_prog q = in->build_qual;
    const bool filter = q.count > 0;
    const uint32_t nregs = args.plan->nregs;
    XbRegs R = xb_regs_setup(bregs + (size_t)warp * XB_REGS_BYTES(nregs), nregs);
    if (filter)
        for (uint32_t r = lane; r < nregs; r += 32)
            R.nullm[r] = XB_FULL;
    __syncthreads();
    const uint64_t *rowindex = (const uint64_t *)((const char *)kds + KDS_HEAD_LENGTH(kds)) + kds->hash_nslots;
    const uint32_t n = in->nitems;
    const uint32_t words = (n + 31) / 32;
    const uint32_t stride = gridDim.x * XB_WARPS * 32;
    for (uint32_t base = (blockIdx.x * XB_WARPS + warp) * 32; base < n; base += stride) {
        const uint32_t row = base + lane;
        uint32_t nullbits = 0, hash = 0;
        bool ok = false;
        if (row < n) {
            const uint64_t off = rowindex[row];
            if (off != 0 && off <= kds->length && ((kds->length - off) & 7) == 0) {
                const kern_tupitem *ti = (const kern_tupitem *)((const char *)kds + kds->length - off);
                const uint32_t pay = (uint32_t)ti->t_hoff - MINIMAL_TUPLE_OFFSET;
                int natts = ti->t_infomask2 & HEAP_NATTS_MASK;
                if (natts > ncols) natts = ncols;
                const bool hasnull = (ti->t_infomask & HEAP_HASNULL) != 0;
                if (ti->t_hoff >= MINIMAL_TUPLE_OFFSET + 15 && pay <= ti->t_len && off >= ti->t_len &&
                    (!hasnull || 15u + (natts + 7) / 8 <= pay))
                    ok = xb_decode_tuple(cols, natts, hasnull ? ti->t_bits : nullptr,
                                         (const uint8_t *)ti + pay, ti->t_len - pay, in->load, in->nloads,
                                         in->vals + row, in->auxs + row, n, true, &nullbits);
                hash = ti->hash;
            }
            if (!ok)
                XB_RAISE(args.st, ERRCODE_DEVICE_ERROR, XB_MSG_BAD_TUPLE);
        }
        if (ok && nullbits) {
            for (uint32_t k = 0; k < in->nloads; k++) {
                if ((nullbits >> k) & 1u)
                    atomicOr(&in->nulls[(size_t)k * words + row / 32], 1u << (row % 32));
            }
            atomicOr(&in->hasnull, nullbits);
        }
        /* datum hashes of the columns whose hash later stages read */
        for (uint32_t k = 0; ok && in->hashed && k < in->nloads; k++) {
            if (!((in->hashed >> k) & 1u) || ((nullbits >> k) & 1u))
                continue;
            bool bad = false;
            const uint32_t hk = in->load[k].ld == XB_LD_NUMERIC ? XB_HK_NUM : XB_HK_TEXT;
            in->hashes[(size_t)k * n + row] = xb_hash_reg(hk, in->vals[(size_t)k * n + row],
                                                          in->auxs[(size_t)k * n + row], true, &bad);
            if (bad)
                XB_RAISE(args.st, ERRCODE_DEVICE_ERROR, XB_MSG_NUMERIC_CORRUPT);
        }
        bool pass = ok;
        if (filter) {
            /* the row's loaded columns into the register file, then the quals */
            for (uint32_t k = 0; k < in->nloads; k++) {
                const uint32_t reg = in->load[k].reg;
                if (ok) {
                    RVAL(R, reg) = in->vals[(size_t)k * n + row];
                    RAUX(R, reg) = in->auxs[(size_t)k * n + row];
                }
                xb_set_null(R, reg, !ok || ((nullbits >> k) & 1u));
            }
            const uint32_t m = __ballot_sync(XB_FULL, ok);
            if (m) {
                if (!xb_vm_run(args.plan->insns + q.start, q.count, R, m, args.st))
                    pass = false;
                else
                    pass = ok && !RISNULL(R, q.result) && RVAL(R, q.result) != 0;
            }
        }
        if (!pass)
            continue;
        /* index insert at hash & mask (linear probing).  Entries hold
         * (hash << 32 | row + 1), or (key << 32 | row + 1) for a 32-bit
         * fused join key; a NULL fused key can never satisfy the join. */
        uint32_t tag = hash;
        if (in->key32) {
            const int k = in->fast_key;
            if ((nullbits >> k) & 1u)
                continue;
            tag = (uint32_t)in->vals[(size_t)k * n + row];
        }
        const unsigned long long ent = ((unsigned long long)tag << 32) | (row + 1);
        uint64_t pos = hash & in->cap_mask;
        for (uint32_t probe = 0; probe <= in->cap_mask; probe++) {
            unsigned long long old = atomicCAS((unsigned long long *)&in->index[pos], 0ULL, ent);
            if (old == 0)
                break;
            if ((uint32_t)(old >> 32) == tag)
                atomicExch(&in->unique_hash, 0u);   /* a second row with this tag */
            pos = (pos + 1) & in->cap_mask;
        }
        if (in->key32) {
            atomicMin(&in->dkey_min, (int32_t)tag);
            atomicMax(&in->dkey_max, (int32_t)tag);
            atomicAdd(&in->nindexed, 1u);
        }
    }
}

/* existence bitmap of a direct table: one thread per 32 keys */
__global__ void __launch_bounds__(XB_BLOCK)
xb_build_dbits(xb_inner *in)
{
    const uint32_t words = in->dbits_words;
    for (uint32_t w = blockIdx.x * blockDim.x + threadIdx.x; w < words; w += gridDim.x * blockDim.x) {
        uint32_t bits = 0;
        for (uint32_t b = 0; b < 32; b++) {
            const uint32_t k = w * 32 + b;
            if (k < in->drange && in->dtab[k] != 0)
                bits |= 1u << b;
        }
        in->dbits[w] = bits;
    }
}

/* pack the live columns of every indexed row into its direct record */
__global__ void __launch_bounds__(XB_BLOCK)
xb_build_drec(xb_inner *in, const xb_plan *plan)
{
    const uint64_t cap = (uint64_t)in->cap_mask + 1;
    const uint32_t n = in->nitems;
    const uint32_t words = (n + 31) / 32;
    for (uint64_t i = blockIdx.x * (uint64_t)blockDim.x + threadIdx.x; i < cap;
         i += (uint64_t)gridDim.x * blockDim.x) {
        const uint64_t ent = in->index[i];
        if (ent == 0)
            continue;
        const int32_t key = (int32_t)(uint32_t)(ent >> 32);
        const uint32_t row = (uint32_t)ent - 1;
        char *rec = in->dpay + (size_t)(uint32_t)((int64_t)key - in->dkey_min) * in->drec_size;
        uint32_t head = 0x80000000U;
        if (in->gid_on)
            *(uint32_t *)(rec + 4) = in->gids[row];
        for (uint32_t k = 0; k < in->nloads; k++) {
            if (!((in->live >> k) & 1u))
                continue;
            int ov, oa, oh;
            xb_drec_layout(in, plan->rk, (int)k, &ov, &oa, &oh);
            if ((in->nulls[(size_t)k * words + row / 32] >> (row % 32)) & 1u)
                head |= 1u << k;
            *(uint64_t *)(rec + ov) = in->vals[(size_t)k * n + row];
            if (oa >= 0) *(uint32_t *)(rec + oa) = in->auxs[(size_t)k * n + row];
            if (oh >= 0) *(uint32_t *)(rec + oh) = in->hashes[(size_t)k * n + row];
        }
        *(uint32_t *)rec = head;
    }
}

/* ---------------------------------------------------------------
 * dense group ids of an inner relation's GROUP BY key tuples
 * --------------------------------------------------------------- */

/* load index (at this depth) of group key k, or -1 */
__device__ __forceinline__ int xb_gid_load(const xb_plan *plan, const xb_inner *in, uint32_t k)
{
    for (uint32_t j = 0; j < in->nloads; j++)
        if (in->load[j].reg == plan->keys[k].reg)
            return (int)j;
    return -1;
}

/* do inner rows a and b hold the same key tuple (NULLs equal, values by bits) */
__device__ __forceinline__ bool
xb_gid_same(const xb_plan *plan, const xb_inner *in, uint32_t a, uint32_t b)
{
    const uint32_t n = in->nitems, words = (n + 31) / 32;
    for (uint32_t k = 0; k < plan->nkeys; k++) {
        const int j = xb_gid_load(plan, in, k);
        const bool na = (in->nulls[(size_t)j * words + a / 32] >> (a % 32)) & 1u;
        const bool nb = (in->nulls[(size_t)j * words + b / 32] >> (b % 32)) & 1u;
        if (na != nb)
            return false;
        if (na)
            continue;
        if (in->vals[(size_t)j * n + a] != in->vals[(size_t)j * n + b])
            return false;
        if (plan->keys[k].rk == XB_RK_TEXT && in->auxs[(size_t)j * n + a] != in->auxs[(size_t)j * n + b])
            return false;
    }
    return true;
}

/* rep[row] = first-inserted row with the same key tuple */
__global__ void __launch_bounds__(XB_BLOCK)
xb_gid_rep(const xb_plan *plan, const xb_inner *in, uint32_t *table, uint32_t tmask, uint32_t *rep)
{
    const uint32_t n = in->nitems, words = (n + 31) / 32;
    for (uint32_t row = blockIdx.x * blockDim.x + threadIdx.x; row < n;
         row += gridDim.x * blockDim.x) {
        uint64_t h = 0x9e3779b97f4a7c15ULL;
        for (uint32_t k = 0; k < plan->nkeys; k++) {
            const int j = xb_gid_load(plan, in, k);
            const bool isnull = (in->nulls[(size_t)j * words + row / 32] >> (row % 32)) & 1u;
            const uint64_t v = isnull ? 0x5a5a5a5aULL : in->vals[(size_t)j * n + row];
            h = (h ^ v) * 0x100000001b3ULL;
            h ^= h >> 29;
        }
        uint32_t pos = (uint32_t)h & tmask;
        rep[row] = row;
        for (uint32_t probe = 0; probe <= tmask; probe++) {
            const uint32_t old = atomicCAS(&table[pos], 0u, row + 1);
            if (old == 0)
                break;
            if (xb_gid_same(plan, in, old - 1, row)) {
                rep[row] = old - 1;
                break;
            }
            pos = (pos + 1) & tmask;
        }
    }
}

/* number the representatives, then give every row its representative's id */
__global__ void __launch_bounds__(XB_BLOCK)
xb_gid_number(xb_inner *in, const uint32_t *rep, uint32_t *counter)
{
    for (uint32_t row = blockIdx.x * blockDim.x + threadIdx.x; row < in->nitems;
         row += gridDim.x * blockDim.x)
        if (rep[row] == row)
            in->gids[row] = atomicAdd(counter, 1u);
}

__global__ void __launch_bounds__(XB_BLOCK)
xb_gid_fill(xb_inner *in, const uint32_t *rep)
{
    for (uint32_t row = blockIdx.x * blockDim.x + threadIdx.x; row < in->nitems;
         row += gridDim.x * blockDim.x)
        if (rep[row] != row)
            in->gids[row] = in->gids[rep[row]];
}

/* fill the direct-address table of a unique 32-bit key from the index */
__global__ void __launch_bounds__(XB_BLOCK)
xb_build_direct(xb_inner *in)
{
    const uint64_t cap = (uint64_t)in->cap_mask + 1;
    for (uint64_t i = blockIdx.x * (uint64_t)blockDim.x + threadIdx.x; i < cap;
         i += (uint64_t)gridDim.x * blockDim.x) {
        const uint64_t ent = in->index[i];
        if (ent == 0)
            continue;
        const int32_t key = (int32_t)(uint32_t)(ent >> 32);
        in->dtab[(uint32_t)((int64_t)key - in->dkey_min)] = (uint32_t)ent;     /* row + 1 */
    }
}

/*
 * Point every non-NULL value of text column k at the first-inserted row
 * holding the same bytes (a per-column dedupe through a temporary
 * open-addressing table of row + 1 entries).
 */
__global__ void __launch_bounds__(XB_BLOCK)
xb_canon_text(xb_inner *in, uint32_t k, uint32_t *table, uint32_t tmask, xb_status *st)
{
    const uint32_t n = in->nitems;
    const uint32_t words = (n + 31) / 32;
    uint64_t *vals = in->vals + (size_t)k * n;
    const uint32_t *auxs = in->auxs + (size_t)k * n;
    const uint32_t *hashes = in->hashes + (size_t)k * n;
    const uint32_t *nulls = in->nulls + (size_t)k * words;
    for (uint32_t row = blockIdx.x * blockDim.x + threadIdx.x; row < n;
         row += gridDim.x * blockDim.x) {
        if ((nulls[row / 32] >> (row % 32)) & 1u)
            continue;
        const uint32_t h = hashes[row], len = auxs[row];
        const uint8_t *v = (const uint8_t *)vals[row];
        uint32_t pos = h & tmask;
        for (uint32_t probe = 0; probe <= tmask; probe++) {
            const uint32_t old = atomicCAS(&table[pos], 0u, row + 1);
            if (old == 0)
                break;                          /* this row represents its bytes */
            const uint32_t r = old - 1;         /* a representative: never rewritten */
            if (hashes[r] == h && auxs[r] == len &&
                xb_bytes_eq((const uint8_t *)vals[r], v, len)) {
                vals[row] = vals[r];
                break;
            }
            pos = (pos + 1) & tmask;
        }
    }
    (void)st;
}

/* ================================================================
 * Final: kds_final materialisation
 * ================================================================ */

/* byte-wise store: kds_final columns follow the header's attalign, and the
 * trailing row-id sits right after a variable-length key, so no store in a
 * group tuple may assume natural alignment */

/* one partial-aggregate tuple (__writeOutOneTuplePreAgg layout,
 * cuda_gpupreagg.cu:18-223); returns t_len.  ti == nullptr only measures. */
__device__ uint32_t
xb_write_group_tuple(const xb_plan *plan, const char *e, kern_tupitem *ti, uint32_t rowid)
{
    const uint32_t nattrs = plan->naggs;
    uint32_t t_hoff = (uint32_t)PGSTROM_MAXALIGN(15 + (nattrs + 7) / 8);
    uint16_t infomask = HEAP_HASNULL;
    char *base = (char *)ti;
    if (ti) {
        for (uint32_t i = 0; i < t_hoff; i++) base[i] = 0;
        const uint16_t im2 = (uint16_t)(nattrs & HEAP_NATTS_MASK);
        const uint8_t hoff = (uint8_t)(t_hoff + MINIMAL_TUPLE_OFFSET);
        const uint32_t hash = ((const xb_gent_head *)e)->hash;
        xb_store(base + offsetof(kern_tupitem, hash), &hash, 4);
        xb_store(base + offsetof(kern_tupitem, t_infomask2), &im2, 2);
        xb_store(base + offsetof(kern_tupitem, t_hoff), &hoff, 1);
    }
    const xb_keyimg *keys = (const xb_keyimg *)(e + plan->gent_keys_off);
    for (uint32_t j = 0; j < nattrs; j++) {
        const xb_agg &a = plan->aggs[j];
        uint32_t t_next = (uint32_t)PGSTROM_TYPEALIGN(a.attalign, t_hoff);
        if (ti)
            for (uint32_t i = t_hoff; i < t_next; i++) base[i] = 0;
        char *buf = ti ? base + t_next : nullptr;
        uint32_t nbytes = 0;
        const uint64_t *su = (const uint64_t *)(e + a.state_off);
        switch (a.action) {
        case KAGG_ACTION__VREF: {
            if (a.key_index < 0) break;
            const xb_key &k = plan->keys[a.key_index];
            const xb_keyimg &img = keys[a.key_index];
            if (img.isnull) break;
            switch (k.ld) {
            case XB_LD_BOOL: { uint8_t v = (uint8_t)img.val; nbytes = 1; if (buf) xb_store(buf, &v, 1); break; }
            case XB_LD_INT2: { int16_t v = (int16_t)img.val; nbytes = 2; if (buf) xb_store(buf, &v, 2); break; }
            case XB_LD_INT4:
            case XB_LD_DATE: { int32_t v = (int32_t)img.val; nbytes = 4; if (buf) xb_store(buf, &v, 4); break; }
            case XB_LD_INT8:
            case XB_LD_FLT8: { nbytes = 8; if (buf) xb_store(buf, &img.val, 8); break; }
            case XB_LD_FLT4: {
                float v = (float)__longlong_as_double(img.val);
                nbytes = 4;
                if (buf) xb_store(buf, &v, 4);
                break;
            }
            case XB_LD_TEXT: {
                nbytes = 4 + img.len;
                if (buf) {
                    const uint32_t hdr = nbytes << 2;           /* SET_VARSIZE */
                    xb_store(buf, &hdr, 4);
                    xb_store(buf + 4, (const void *)img.val, img.len);
                }
                infomask |= HEAP_HASVARWIDTH;
                break;
            }
            case XB_LD_NUMERIC: {
                const uint8_t *vl = (const uint8_t *)img.val;
                nbytes = xb_numeric_varsize(vl);
                if (buf) xb_store(buf, vl, nbytes);
                infomask |= HEAP_HASVARWIDTH;
                break;
            }
            }
            break;
        }
        case KAGG_ACTION__NROWS_ANY:
        case KAGG_ACTION__NROWS_COND:
            nbytes = 8;
            if (buf) xb_store(buf, &su[0], 8);
            break;
        case KAGG_ACTION__PMIN_INT32:
        case KAGG_ACTION__PMIN_INT64:
        case KAGG_ACTION__PMAX_INT32:
        case KAGG_ACTION__PMAX_INT64: {
            kagg_state__pminmax_int64_packed r;
            nbytes = sizeof(r);
            r.vl_len_ = (int32_t)(nbytes << 2);
            r.attrs = *(const uint32_t *)(su + 1) ? PAGG_MINMAX_ATTRS__VALID : 0;
            r.value = (int64_t)su[0];
            if (buf) xb_store(buf, &r, nbytes);
            infomask |= HEAP_HASVARWIDTH;
            break;
        }
        case KAGG_ACTION__PMIN_FP64:
        case KAGG_ACTION__PMAX_FP64: {
            kagg_state__pminmax_fp64_packed r;
            const bool valid = *(const uint32_t *)(su + 1) != 0;
            nbytes = sizeof(r);
            r.vl_len_ = (int32_t)(nbytes << 2);
            r.attrs = valid ? PAGG_MINMAX_ATTRS__VALID : 0;
            r.value = valid ? xb_f64_from_ordered((int64_t)su[0])
                            : (a.action == KAGG_ACTION__PMIN_FP64 ? 1.7976931348623157e308
                                                                   : -1.7976931348623157e308);
            if (buf) xb_store(buf, &r, nbytes);
            infomask |= HEAP_HASVARWIDTH;
            break;
        }
        case KAGG_ACTION__PSUM_INT:
        case KAGG_ACTION__PAVG_INT: {
            kagg_state__psum_int_packed r;
            nbytes = sizeof(r);
            r.vl_len_ = (int32_t)(nbytes << 2);
            r.attrs = 0;
            r.nitems = (int64_t)su[0];
            r.sum = (int64_t)su[1];
            if (buf) xb_store(buf, &r, nbytes);
            infomask |= HEAP_HASVARWIDTH;
            break;
        }
        case KAGG_ACTION__PSUM_INT64:
        case KAGG_ACTION__PAVG_INT64:
        case KAGG_ACTION__PSUM_NUMERIC:
        case KAGG_ACTION__PAVG_NUMERIC: {
            kagg_state__psum_numeric_packed r;
            const bool is_num = (a.action == KAGG_ACTION__PSUM_NUMERIC || a.action == KAGG_ACTION__PAVG_NUMERIC);
            nbytes = sizeof(r);
            r.vl_len_ = (int32_t)(nbytes << 2);
            r.attrs = is_num ? (((uint32_t)a.weight & PAGG_NUMERIC_ATTRS__WEIGHT) |
                                *(const uint32_t *)(su + 3)) : 0;
            r.nitems = su[0];
            r.sum.u64_lo = su[1];
            r.sum.u64_hi = su[2];
            if (buf) xb_store(buf, &r, nbytes);
            infomask |= HEAP_HASVARWIDTH;
            break;
        }
        case KAGG_ACTION__PSUM_FP:
        case KAGG_ACTION__PAVG_FP: {
            kagg_state__psum_fp_packed r;
            const double *d = (const double *)su;
            nbytes = sizeof(r);
            r.vl_len_ = (int32_t)(nbytes << 2);
            r.attrs = 0;
            r.nitems = (int64_t)su[0];
            r.sum = __dadd_rn(d[1], d[2]);
            if (buf) xb_store(buf, &r, nbytes);
            infomask |= HEAP_HASVARWIDTH;
            break;
        }
        case KAGG_ACTION__STDDEV: {
            kagg_state__stddev_packed r;
            const double *d = (const double *)su;
            nbytes = sizeof(r);
            r.vl_len_ = (int32_t)(nbytes << 2);
            r.attrs = 0;
            r.nitems = (int64_t)su[0];
            r.sum_x = __dadd_rn(d[1], d[2]);
            r.sum_x2 = __dadd_rn(d[3], d[4]);
            if (buf) xb_store(buf, &r, nbytes);
            infomask |= HEAP_HASVARWIDTH;
            break;
        }
        case KAGG_ACTION__COVAR: {
            kagg_state__covar_packed r;
            const double *d = (const double *)su;
            nbytes = sizeof(r);
            r.vl_len_ = (int32_t)(nbytes << 2);
            r.attrs = 0;
            r.nitems = (int64_t)su[0];
            r.sum_x = __dadd_rn(d[1], d[2]);
            r.sum_xx = __dadd_rn(d[3], d[4]);
            r.sum_y = __dadd_rn(d[5], d[6]);
            r.sum_yy = __dadd_rn(d[7], d[8]);
            r.sum_xy = __dadd_rn(d[9], d[10]);
            if (buf) xb_store(buf, &r, nbytes);
            infomask |= HEAP_HASVARWIDTH;
            break;
        }
        default:
            break;
        }
        if (ti && nbytes > 0)
            base[offsetof(kern_tupitem, t_bits) + (j >> 3)] |= (char)(1u << (j & 7));
        t_hoff = t_next + nbytes;
    }
    t_hoff += ROWID_SIZE;
    if (ti) {
        xb_store(base + offsetof(kern_tupitem, t_len), &t_hoff, 4);
        xb_store(base + offsetof(kern_tupitem, t_infomask), &infomask, 2);
        xb_store(base + t_hoff - ROWID_SIZE, &rowid, 4);        /* KERN_TUPITEM_SET_ROWID */
    }
    return t_hoff;
}

__global__ void xb_final_sizes(XbFinalArgs args)
{
    const xb_plan *plan = args.plan;
    for (uint64_t i = blockIdx.x * (uint64_t)blockDim.x + threadIdx.x; i < args.cap;
         i += (uint64_t)gridDim.x * blockDim.x) {
        const char *e = args.gt->entries + i * plan->gent_size;
        const xb_gent_head *h = (const xb_gent_head *)e;
        if (h->state == XB_GSTATE_READY && (!args.keep || args.keep[i] >= 0) &&
            (args.part_div < 2 || h->hash % args.part_div == args.part_rem)) {
            uint32_t t_len = xb_write_group_tuple(plan, e, nullptr, 0);
            args.sizes[i] = PGSTROM_MAXALIGN((args.row_format ? 0 : offsetof(kern_hashitem, t)) + t_len);
            args.flags[i] = 1;
        } else {
            args.sizes[i] = 0;
            args.flags[i] = 0;
        }
    }
}

__global__ void xb_final_write(XbFinalArgs args)
{
    const xb_plan *plan = args.plan;
    kern_data_store *kds = (kern_data_store *)args.kds_final;
    uint64_t *hslots = (uint64_t *)(args.kds_final + KDS_HEAD_LENGTH(kds));
    uint64_t *rowindex = hslots + args.nslots;
    for (uint64_t i = blockIdx.x * (uint64_t)blockDim.x + threadIdx.x; i < args.cap;
         i += (uint64_t)gridDim.x * blockDim.x) {
        if (!args.flags[i])
            continue;
        const char *e = args.gt->entries + i * plan->gent_size;
        const uint32_t rank = args.keep ? (uint32_t)args.keep[i] : args.flag_scan[i];
        const uint64_t item_off = args.items_base + args.size_scan[i];
        if (args.row_format) {
            /* KDS_FORMAT_ROW: the tuple itself, found through the row index */
            kern_tupitem *ti = (kern_tupitem *)(args.kds_final + item_off);
            xb_write_group_tuple(plan, e, ti, rank);
            rowindex[rank] = args.length - item_off;
            continue;
        }
        kern_hashitem *hitem = (kern_hashitem *)(args.kds_final + item_off);
        xb_write_group_tuple(plan, e, &hitem->t, rank);
        rowindex[rank] = args.length - (item_off + offsetof(kern_hashitem, t));
        const uint32_t hash = ((const xb_gent_head *)e)->hash;
        unsigned long long mine = args.length - item_off;
        unsigned long long prev = atomicExch((unsigned long long *)&hslots[hash % args.nslots], mine);
        hitem->next = prev;
    }
}

/* ----------------------------------------------------------------
 * GPU-Sort of the final groups (kern_gpusort_prep_buffer,
 * kern_gpusort_exec_bitonic and the window-rank kernels of
 * cuda_gpusort.cu:15-996): every sort key of a group becomes one or two
 * 64-bit words whose unsigned order is the key's SQL order (descending
 * keys complemented) and a NULL flag; the groups are then ordered by
 * stable radix passes from the last key's lowest word to the first key's
 * NULL flag, and LIMIT or the window rank picks the groups kept.
 * ---------------------------------------------------------------- */

__device__ __forceinline__ uint64_t xb_sort_i64(int64_t v)
{
    return (uint64_t)v ^ (1ULL << 63);
}

__device__ __forceinline__ uint64_t xb_sort_f64(double d)
{
    if (d != d)
        return ~0ULL;                               /* NaN sorts above every value */
    if (d == 0.0)
        d = 0.0;                                    /* -0 equals +0 */
    const uint64_t b = (uint64_t)__double_as_longlong(d);
    return (b >> 63) ? ~b : (b | (1ULL << 63));
}

__global__ void xb_sort_gather(XbSortArgs a)
{
    for (uint64_t i = blockIdx.x * (uint64_t)blockDim.x + threadIdx.x; i < a.cap;
         i += (uint64_t)gridDim.x * blockDim.x)
        if (a.flags[i])
            a.ents[a.flag_scan[i]] = (uint32_t)i;
}

__global__ void xb_sort_keys(XbSortArgs a)
{
    const xb_plan *plan = a.plan;
    for (uint32_t r = blockIdx.x * blockDim.x + threadIdx.x; r < a.n; r += gridDim.x * blockDim.x) {
        const char *e = a.gt->entries + (uint64_t)a.ents[r] * plan->gent_size;
        const xb_keyimg *img = (const xb_keyimg *)(e + plan->gent_keys_off);
        for (uint32_t k = 0; k < plan->nsort; k++) {
            const xb_sortkey &sk = plan->sort[k];
            const xb_agg &ag = plan->aggs[sk.agg];
            const uint64_t *su = (const uint64_t *)(e + ag.state_off);
            const double *sd = (const double *)su;
            bool isnull = false;
            uint64_t hi = 0, lo = 0;
            const int64_t n = (int64_t)su[0];
            switch (sk.kind) {
            case KSORT_KEY_KIND__VREF:
                if (ag.action == KAGG_ACTION__VREF) {
                    const xb_keyimg &ki = img[ag.key_index];
                    const uint8_t ld = plan->keys[ag.key_index].ld;
                    isnull = ki.isnull != 0;
                    hi = (ld == XB_LD_FLT8 || ld == XB_LD_FLT4) ? xb_sort_f64(__longlong_as_double(ki.val))
                                                               : xb_sort_i64((int64_t)ki.val);
                } else {
                    hi = xb_sort_i64((int64_t)su[0]);       /* count */
                }
                break;
            case KSORT_KEY_KIND__PMINMAX_INT64:
            case KSORT_KEY_KIND__PMINMAX_FP64:
                /* the state is an order-preserving int64 (xb_f64_ordered for
                 * float8) with its valid flag */
                isnull = *(const uint32_t *)(su + 1) == 0;
                hi = xb_sort_i64((int64_t)su[0]);
                break;
            case KSORT_KEY_KIND__PSUM_INT64:
            case KSORT_KEY_KIND__PSUM_NUMERIC:
                isnull = n == 0;
                if (sk.words == 1) {
                    hi = xb_sort_i64((int64_t)su[1]);
                } else {
                    hi = xb_sort_i64((int64_t)su[2]);
                    lo = su[1];
                    const uint32_t sp = ag.state_sz >= 32 ? (*(const uint32_t *)(su + 3) & ~PAGG_NUMERIC_ATTRS__WEIGHT) : 0;
                    if (sp & PAGG_NUMERIC_ATTRS__NAN) { hi = ~0ULL; lo = ~0ULL; }
                    else if (sp & PAGG_NUMERIC_ATTRS__PINF) { hi = ~0ULL; lo = ~1ULL; }
                    else if (sp & PAGG_NUMERIC_ATTRS__NINF) { hi = 0; lo = 0; }
                }
                break;
            case KSORT_KEY_KIND__PSUM_FP64:
                isnull = n == 0;
                hi = xb_sort_f64(sd[1] + sd[2]);
                break;
            case KSORT_KEY_KIND__PAVG_INT64:
            case KSORT_KEY_KIND__PAVG_FP64:
            case KSORT_KEY_KIND__PAVG_NUMERIC: {
                isnull = n == 0;
                double sum;
                if (ag.action == KAGG_ACTION__PAVG_INT)
                    sum = (double)(int64_t)su[1];
                else if (ag.action == KAGG_ACTION__PAVG_FP)
                    sum = sd[1] + sd[2];
                else    /* 128-bit sum; the scale is one per column, so it keeps the order */
                    sum = (double)(xb_i128)(((unsigned __int128)su[2] << 64) | su[1]);
                hi = xb_sort_f64(isnull ? 0.0 : sum / (double)n);
                break;
            }
            case KSORT_KEY_KIND__PVARIANCE_SAMP:
            case KSORT_KEY_KIND__PVARIANCE_POP: {
                const bool samp = sk.kind == KSORT_KEY_KIND__PVARIANCE_SAMP;
                isnull = samp ? n < 2 : n < 1;
                const double dn = (double)n, sx = sd[1] + sd[2], sxx = sd[3] + sd[4];
                const double num = dn * sxx - sx * sx;
                hi = xb_sort_f64(isnull ? 0.0 : (num < 0.0 ? 0.0 : num) / (dn * (samp ? dn - 1.0 : dn)));
                break;
            }
            case KSORT_KEY_KIND__PCOVAR_CORR: case KSORT_KEY_KIND__PCOVAR_SAMP:
            case KSORT_KEY_KIND__PCOVAR_POP: case KSORT_KEY_KIND__PCOVAR_AVGX:
            case KSORT_KEY_KIND__PCOVAR_AVGY: case KSORT_KEY_KIND__PCOVAR_COUNT: {
                const double dn = (double)n;
                const double sx = sd[1] + sd[2], sxx = sd[3] + sd[4], sy = sd[5] + sd[6];
                const double syy = sd[7] + sd[8], sxy = sd[9] + sd[10];
                double v = 0.0;
                switch (sk.kind) {
                case KSORT_KEY_KIND__PCOVAR_COUNT: v = dn; break;
                case KSORT_KEY_KIND__PCOVAR_AVGX: isnull = n < 1; v = sx / dn; break;
                case KSORT_KEY_KIND__PCOVAR_AVGY: isnull = n < 1; v = sy / dn; break;
                case KSORT_KEY_KIND__PCOVAR_POP: isnull = n < 1; v = (sxy - sx * sy / dn) / dn; break;
                case KSORT_KEY_KIND__PCOVAR_SAMP: isnull = n < 2; v = (sxy - sx * sy / dn) / (dn - 1.0); break;
                default: {
                    const double vx = dn * sxx - sx * sx, vy = dn * syy - sy * sy;
                    isnull = n < 1 || vx <= 0.0 || vy <= 0.0;
                    v = (dn * sxy - sx * sy) / sqrt(vx * vy);
                    break;
                }
                }
                hi = xb_sort_f64(isnull ? 0.0 : v);
                break;
            }
            case KSORT_KEY_KIND__NITEMS:
                hi = xb_sort_i64(n);
                break;
            default:
                break;
            }
            if (isnull) {
                hi = 0;
                lo = 0;
            } else if (!sk.asc) {
                hi = ~hi;
                lo = ~lo;
            }
            a.keyw[(2ULL * k) * a.n + r] = hi;
            a.keyw[(2ULL * k + 1) * a.n + r] = lo;
            /* the flag sorts as the key's most significant part */
            a.nul[(uint64_t)k * a.n + r] = (uint8_t)(isnull ? (sk.nulls_first ? 0 : 1) : (sk.nulls_first ? 1 : 0));
        }
    }
}

/* the key of one radix pass, in the current order */
__global__ void xb_sort_pass_key64(const uint64_t *col, const uint32_t *idx, uint64_t *out, uint32_t n)
{
    for (uint32_t p = blockIdx.x * blockDim.x + threadIdx.x; p < n; p += gridDim.x * blockDim.x)
        out[p] = col[idx[p]];
}

__global__ void xb_sort_pass_key8(const uint8_t *col, const uint32_t *idx, uint8_t *out, uint32_t n)
{
    for (uint32_t p = blockIdx.x * blockDim.x + threadIdx.x; p < n; p += gridDim.x * blockDim.x)
        out[p] = col[idx[p]];
}

/* groups kept, in order: LIMIT, or the window rank of each group within
 * its partition (row_number / rank / dense_rank) against its limit */

__device__ __forceinline__ bool
xb_sort_keys_equal(const XbRankArgs &a, uint32_t k0, uint32_t k1, uint32_t r, uint32_t q)
{
    for (uint32_t k = k0; k < k1; k++) {
        if (a.nul[(uint64_t)k * a.n + r] != a.nul[(uint64_t)k * a.n + q] ||
            a.keyw[(2ULL * k) * a.n + r] != a.keyw[(2ULL * k) * a.n + q] ||
            a.keyw[(2ULL * k + 1) * a.n + r] != a.keyw[(2ULL * k + 1) * a.n + q])
            return false;
    }
    return true;
}

__global__ void xb_sort_bounds(XbRankArgs a)
{
    const uint32_t pb = a.plan->sort_partby, ob = a.plan->sort_orderby;
    for (uint32_t p = blockIdx.x * blockDim.x + threadIdx.x; p < a.n; p += gridDim.x * blockDim.x) {
        bool part = p == 0, peer = p == 0;
        if (p > 0) {
            const uint32_t r = a.idx[p], q = a.idx[p - 1];
            part = !xb_sort_keys_equal(a, 0, pb, r, q);
            peer = part || !xb_sort_keys_equal(a, pb, pb + ob, r, q);
        }
        a.part_start[p] = part ? p : 0;
        a.peer_start[p] = peer ? p : 0;
        a.peer_flag[p] = peer ? 1 : 0;
    }
}


__global__ void xb_sort_keepflag(XbKeepArgs a)
{
    const xb_plan *plan = a.plan;
    for (uint32_t p = blockIdx.x * blockDim.x + threadIdx.x; p < a.n; p += gridDim.x * blockDim.x) {
        bool keep = true;
        if (plan->sort_window) {
            const uint32_t ps = a.part_start[p];
            uint64_t rank;
            if (plan->sort_window == KSORT_WINDOW_FUNC__ROW_NUMBER)
                rank = p - ps + 1;
            else if (plan->sort_window == KSORT_WINDOW_FUNC__RANK)
                rank = a.peer_start[p] - ps + 1;
            else
                rank = a.peer_cnt[p] - a.peer_cnt[ps] + 1;
            keep = plan->sort_rank_limit == 0 || rank <= plan->sort_rank_limit;
        } else if (plan->sort_limit > 0) {
            keep = (int64_t)p < plan->sort_limit;
        }
        a.keep_flag[p] = keep ? 1 : 0;
    }
}

__global__ void xb_sort_keep(XbKeepArgs a, const uint32_t *keep_scan, int64_t *keep)
{
    for (uint32_t p = blockIdx.x * blockDim.x + threadIdx.x; p < a.n; p += gridDim.x * blockDim.x)
        keep[a.ents[a.idx[p]]] = a.keep_flag[p] ? (int64_t)keep_scan[p] : -1;
}

__global__ void xb_iota_u32(uint32_t *out, uint32_t n)
{
    for (uint32_t p = blockIdx.x * blockDim.x + threadIdx.x; p < n; p += gridDim.x * blockDim.x)
        out[p] = p;
}

/* ----------------------------------------------------------------
 * merge of another kds_final (kern_gpupreagg_final_merge,
 * cuda_gpupreagg.cu:2331-2432, reading the keys back as
 * ExecLoadKeysFromGroupByFinal does, xpu_common.cu:1675-1727)
 * ---------------------------------------------------------------- */


/* one packed partial state back into the group-entry form (the inverse of
 * xb_write_group_tuple); returns its bytes in the tuple */
__device__ uint32_t
xb_read_state(const xb_agg &a, const char *p, bool present, uint64_t *su)
{
    for (uint32_t k = 0; k < a.state_sz / 8; k++)
        su[k] = 0;
    switch (a.action) {
    case KAGG_ACTION__NROWS_ANY:
    case KAGG_ACTION__NROWS_COND:
        if (present) xb_store((char *)su, p, 8);
        return 8;
    case KAGG_ACTION__PMIN_INT32: case KAGG_ACTION__PMIN_INT64:
    case KAGG_ACTION__PMAX_INT32: case KAGG_ACTION__PMAX_INT64: {
        kagg_state__pminmax_int64_packed r;
        if (!present) return sizeof(r);
        xb_store((char *)&r, p, sizeof(r));
        su[0] = (uint64_t)r.value;
        *(uint32_t *)(su + 1) = (r.attrs & PAGG_MINMAX_ATTRS__VALID) ? 1u : 0u;
        return sizeof(r);
    }
    case KAGG_ACTION__PMIN_FP64: case KAGG_ACTION__PMAX_FP64: {
        kagg_state__pminmax_fp64_packed r;
        if (!present) return sizeof(r);
        xb_store((char *)&r, p, sizeof(r));
        const bool valid = (r.attrs & PAGG_MINMAX_ATTRS__VALID) != 0;
        su[0] = valid ? (uint64_t)xb_f64_ordered(r.value) : 0;
        *(uint32_t *)(su + 1) = valid ? 1u : 0u;
        return sizeof(r);
    }
    case KAGG_ACTION__PSUM_INT: case KAGG_ACTION__PAVG_INT: {
        kagg_state__psum_int_packed r;
        if (!present) return sizeof(r);
        xb_store((char *)&r, p, sizeof(r));
        su[0] = (uint64_t)r.nitems;
        su[1] = (uint64_t)r.sum;
        return sizeof(r);
    }
    case KAGG_ACTION__PSUM_INT64: case KAGG_ACTION__PAVG_INT64:
    case KAGG_ACTION__PSUM_NUMERIC: case KAGG_ACTION__PAVG_NUMERIC: {
        kagg_state__psum_numeric_packed r;
        if (!present) return sizeof(r);
        xb_store((char *)&r, p, sizeof(r));
        su[0] = r.nitems;
        su[1] = r.sum.u64_lo;
        su[2] = r.sum.u64_hi;
        if (a.state_sz >= 32)
            *(uint32_t *)(su + 3) = r.attrs & ~PAGG_NUMERIC_ATTRS__WEIGHT;
        return sizeof(r);
    }
    case KAGG_ACTION__PSUM_FP: case KAGG_ACTION__PAVG_FP: {
        kagg_state__psum_fp_packed r;
        if (!present) return sizeof(r);
        xb_store((char *)&r, p, sizeof(r));
        su[0] = (uint64_t)r.nitems;
        ((double *)su)[1] = r.sum;
        return sizeof(r);
    }
    case KAGG_ACTION__STDDEV: {
        kagg_state__stddev_packed r;
        if (!present) return sizeof(r);
        xb_store((char *)&r, p, sizeof(r));
        su[0] = (uint64_t)r.nitems;
        ((double *)su)[1] = r.sum_x;
        ((double *)su)[3] = r.sum_x2;
        return sizeof(r);
    }
    case KAGG_ACTION__COVAR: {
        kagg_state__covar_packed r;
        if (!present) return sizeof(r);
        xb_store((char *)&r, p, sizeof(r));
        su[0] = (uint64_t)r.nitems;
        ((double *)su)[1] = r.sum_x;
        ((double *)su)[3] = r.sum_xx;
        ((double *)su)[5] = r.sum_y;
        ((double *)su)[7] = r.sum_yy;
        ((double *)su)[9] = r.sum_xy;
        return sizeof(r);
    }
    default:
        return 0;
    }
}

/* every group tuple of the other kds_final: its keys are looked up (or
 * created) in this session's global table and its partial states merged */
__global__ void __launch_bounds__(XB_BLOCK)
xb_merge_final(XbMergeArgs args)
{
    const xb_plan *plan = args.plan;
    const kern_data_store *kds = args.kds;
    const uint64_t *rowindex = (const uint64_t *)((const char *)kds + KDS_HEAD_LENGTH(kds)) + kds->hash_nslots;
    for (uint32_t i = blockIdx.x * blockDim.x + threadIdx.x; i < kds->nitems; i += gridDim.x * blockDim.x) {
        const uint64_t off = rowindex[i];
        if (off == 0 || off > kds->length || ((kds->length - off) & 7) != 0) {
            XB_RAISE(args.st, ERRCODE_DEVICE_ERROR, XB_MSG_BAD_TUPLE);
            continue;
        }
        const kern_tupitem *ti = (const kern_tupitem *)((const char *)kds + kds->length - off);
        const char *base = (const char *)ti;
        const uint32_t t_len = ti->t_len;
        uint32_t t = (uint32_t)ti->t_hoff - MINIMAL_TUPLE_OFFSET;
        const bool hasnull = (ti->t_infomask & HEAP_HASNULL) != 0;
        if (off < t_len || t > t_len) {
            XB_RAISE(args.st, ERRCODE_DEVICE_ERROR, XB_MSG_BAD_TUPLE);
            continue;
        }
        /* the source entry in the group-entry form */
        alignas(16) char src[XB_GENT_MAX];
        for (uint32_t k = 0; k < plan->gent_size && k < XB_GENT_MAX; k++)
            src[k] = 0;
        xb_keyimg *img = (xb_keyimg *)(src + plan->gent_keys_off);
        bool bad = false;
        for (uint32_t j = 0; j < plan->naggs && !bad; j++) {
            const xb_agg &a = plan->aggs[j];
            const bool present = !hasnull || ((ti->t_bits[j >> 3] >> (j & 7)) & 1u);
            t = (uint32_t)PGSTROM_TYPEALIGN(a.attalign > 0 ? a.attalign : 1, t);
            const char *p = base + t;
            uint32_t nbytes = 0;
            if (a.action == KAGG_ACTION__VREF) {
                if (a.key_index < 0)
                    continue;
                const xb_key &k = plan->keys[a.key_index];
                xb_keyimg &ki = img[a.key_index];
                ki.isnull = !present;
                if (!present)
                    continue;
                switch (k.ld) {
                case XB_LD_BOOL: ki.val = *(const uint8_t *)p; nbytes = 1; break;
                case XB_LD_INT2: { int16_t v; xb_store((char *)&v, p, 2); ki.val = (uint64_t)(int64_t)v; nbytes = 2; break; }
                case XB_LD_INT4:
                case XB_LD_DATE: { int32_t v; xb_store((char *)&v, p, 4); ki.val = (uint64_t)(int64_t)v; nbytes = 4; break; }
                case XB_LD_INT8:
                case XB_LD_FLT8: xb_store((char *)&ki.val, p, 8); nbytes = 8; break;
                case XB_LD_FLT4: {
                    float v; xb_store((char *)&v, p, 4);
                    ki.val = (uint64_t)__double_as_longlong((double)v);
                    nbytes = 4;
                    break;
                }
                case XB_LD_TEXT: {
                    uint32_t h; xb_store((char *)&h, p, 4);
                    nbytes = h >> 2;
                    ki.val = (uint64_t)(p + 4);
                    ki.len = nbytes - 4;
                    break;
                }
                case XB_LD_NUMERIC:
                    nbytes = xb_numeric_varsize((const uint8_t *)p);
                    ki.val = (uint64_t)p;
                    ki.len = 0;
                    break;
                default:
                    bad = true;
                    break;
                }
            } else {
                nbytes = xb_read_state(a, p, present, (uint64_t *)(src + a.state_off));
            }
            if (present)
                t += nbytes;
            if (t > t_len)
                bad = true;
        }
        if (bad) {
            XB_RAISE(args.st, ERRCODE_DEVICE_ERROR, XB_MSG_BAD_TUPLE);
            continue;
        }
        char *g = xb_group_find_or_dump(plan, args.gt, ti->hash, img, args.st);
        if (g)
            xb_merge_states(plan, g, src);
    }
}

/* ----------------------------------------------------------------
 * group-table growth: the live entries of the old table rehashed into a
 * larger one, then the dump entries (groups created while the table had
 * no room) merged in.  Key bytes live in the key arena; when the arena is
 * replaced by a larger copy, key pointers are moved with it.
 * ---------------------------------------------------------------- */
struct XbGrowArgs {
    const xb_plan  *plan;
    const char     *old_entries;
    uint64_t        old_cap;
    char           *dump;
    uint64_t        ndump;
    xb_gtable      *gt;             /* the new table (device) */
    xb_status      *st;
    const char     *arena_old;      /* key pointers in [arena_old, +arena_old_sz) move */
    uint64_t        arena_old_sz;
    char           *arena_new;
};

__device__ __forceinline__ void
xb_gt_relocate_keys(const xb_plan *plan, char *e, const XbGrowArgs &a)
{
    if (a.arena_new == a.arena_old)
        return;
    xb_keyimg *img = (xb_keyimg *)(e + plan->gent_keys_off);
    for (uint32_t k = 0; k < plan->nkeys; k++) {
        if (img[k].isnull || (plan->keys[k].rk != XB_RK_TEXT && plan->keys[k].rk != XB_RK_NUM))
            continue;
        const uint64_t v = img[k].val, lo = (uint64_t)a.arena_old;
        if (v >= lo && v < lo + a.arena_old_sz)
            img[k].val = (uint64_t)a.arena_new + (v - lo);
    }
}

__global__ void __launch_bounds__(XB_BLOCK)
xb_gt_rehash(XbGrowArgs a)
{
    const xb_plan *plan = a.plan;
    const uint32_t gsz = plan->gent_size;
    xb_gtable *gt = a.gt;
    for (uint64_t i = blockIdx.x * (uint64_t)blockDim.x + threadIdx.x; i < a.old_cap;
         i += (uint64_t)gridDim.x * blockDim.x) {
        const char *e = a.old_entries + i * gsz;
        const xb_gent_head *h = (const xb_gent_head *)e;
        if (h->state != XB_GSTATE_READY)
            continue;
        /* keys are distinct: the first EMPTY slot of the probe sequence */
        uint64_t pos = h->hash & gt->cap_mask;
        bool placed = false;
        for (uint64_t probe = 0; probe <= gt->cap_mask; probe++) {
            char *d = gt->entries + pos * gsz;
            xb_gent_head *dh = (xb_gent_head *)d;
            if (atomicCAS(&dh->state, XB_GSTATE_EMPTY, XB_GSTATE_BUSY) == XB_GSTATE_EMPTY) {
                for (uint32_t w = 1; w < gsz / 8; w++)
                    ((uint64_t *)d)[w] = ((const uint64_t *)e)[w];
                dh->hash = h->hash;
                xb_gt_relocate_keys(plan, d, a);
                atomicAdd((unsigned long long *)&gt->nused, 1ULL);
                xb_st_release(&dh->state, XB_GSTATE_READY);
                placed = true;
                break;
            }
            pos = (pos + 1) & gt->cap_mask;
        }
        if (!placed) {
            XB_RAISE(a.st, ERRCODE_SUSPEND_NO_SPACE, XB_MSG_GTABLE_FULL);
            atomicOr(&gt->overflow, 1u);
        }
    }
}

__global__ void __launch_bounds__(XB_BLOCK)
xb_gt_merge_dump(XbGrowArgs a)
{
    const xb_plan *plan = a.plan;
    const uint32_t gsz = plan->gent_size;
    for (uint64_t i = blockIdx.x * (uint64_t)blockDim.x + threadIdx.x; i < a.ndump;
         i += (uint64_t)gridDim.x * blockDim.x) {
        char *e = a.dump + i * gsz;
        const xb_gent_head *h = (const xb_gent_head *)e;
        if (h->state != XB_GSTATE_READY)
            continue;
        xb_gt_relocate_keys(plan, e, a);
        const xb_keyimg *img = (const xb_keyimg *)(e + plan->gent_keys_off);
        bool full = false;
        char *g = xb_group_find(plan, a.gt->entries, a.gt->cap_mask, h->hash, img, a.gt, a.st, &full);
        if (g)
            xb_merge_states(plan, g, e);
        else if (full) {
            XB_RAISE(a.st, ERRCODE_SUSPEND_NO_SPACE, XB_MSG_GTABLE_FULL);
            atomicOr(&a.gt->overflow, 1u);
        }
    }
}

/* ----------------------------------------------------------------
 * inner-buffer rebuild: rows of a hashed projection (or any HASH / ROW
 * chunk whose tuples carry their hash) appended into a KDS_FORMAT_HASH
 * buffer and chained into its hash slots (kern_buffer_reconstruction,
 * cuda_gpujoin.cu:18-71); with a divisor, only the rows whose hash falls
 * into one partition (kern_buffer_partitioning, cuda_gpujoin.cu:76-138)
 * ---------------------------------------------------------------- */

__global__ void __launch_bounds__(XB_BLOCK)
xb_inner_rebuild(XbRebuildArgs args)
{
    kern_data_store *dst = args.dst;
    const kern_data_store *src = args.src;
    const uint64_t *rowidx = (const uint64_t *)((const char *)src + args.src_rowidx);
    const uint32_t nslots = dst->hash_nslots;
    uint64_t *slots = (uint64_t *)((char *)dst + args.dst_head);
    const uint32_t lane = threadIdx.x & 31;
    const uint32_t n = src->nitems;
    for (uint32_t base = blockIdx.x * blockDim.x; base < n; base += gridDim.x * blockDim.x) {
        const uint32_t i = base + threadIdx.x;
        const kern_tupitem *t = nullptr;
        uint32_t sz = 0;
        if (i < n) {
            const uint64_t off = rowidx[i];
            if (off < sizeof(kern_tupitem) || off > src->length - args.src_rowidx || (off & 7) != 0) {
                atomicOr(args.overflow, 2u);            /* a broken row index */
            } else {
                t = (const kern_tupitem *)((const char *)src + src->length - off);
                const uint32_t t_len = t->t_len;
                if (t_len < offsetof(kern_tupitem, t_bits) || t_len > off)
                    atomicOr(args.overflow, 2u);
                else if (args.divisor < 2 || t->hash % args.divisor == args.remainder)
                    sz = (uint32_t)PGSTROM_MAXALIGN(offsetof(kern_hashitem, t) + t_len);
            }
        }
        /* one claim of row ids and bytes per warp */
        const uint32_t want = __ballot_sync(XB_FULL, sz > 0);
        uint32_t incl = sz;
#pragma unroll
        for (uint32_t o = 1; o < 32; o <<= 1) {
            const uint32_t v = __shfl_up_sync(XB_FULL, incl, o);
            if (lane >= o) incl += v;
        }
        const uint32_t total = __shfl_sync(XB_FULL, incl, 31);
        unsigned long long bu = 0;
        uint32_t bn = 0;
        if (lane == 0 && want) {
            bn = atomicAdd(&dst->nitems, (uint32_t)__popc(want));
            bu = atomicAdd((unsigned long long *)&dst->usage, (unsigned long long)total);
        }
        bn = __shfl_sync(XB_FULL, bn, 0);
        bu = __shfl_sync(XB_FULL, bu, 0);
        if (!sz)
            continue;
        const uint32_t row_id = bn + __popc(want & ((1u << lane) - 1));
        const uint64_t offset = bu + incl;              /* from the end to the item */
        const uint64_t need = args.dst_head + 8ULL * nslots + 8ULL * ((uint64_t)row_id + 1);
        if (offset > dst->length || dst->length - offset < need) {
            atomicOr(args.overflow, 1u);
            continue;
        }
        char *item = (char *)dst + dst->length - offset;
        /* the tuple in 8-byte words: both items are MAXALIGN'd and sized */
        const uint32_t t_len = t->t_len;
        const uint64_t *sw = (const uint64_t *)t;
        uint64_t *dw = (uint64_t *)(item + offsetof(kern_hashitem, t));
        for (uint32_t k = 0; k < (t_len + 7) / 8; k++)
            dw[k] = sw[k];
        xb_store(item + offsetof(kern_hashitem, t) + t_len - ROWID_SIZE, &row_id, 4);
        const uint32_t hash = t->hash;
        *(uint64_t *)item = atomicExch((unsigned long long *)&slots[hash % nslots], (unsigned long long)offset);
        uint64_t *dri = (uint64_t *)((char *)dst + args.dst_head) + nslots;
        dri[row_id] = offset - offsetof(kern_hashitem, t);
    }
}

/* ================================================================
 * host side
 * ================================================================ */
static void xb_inner_entry_free(xpuB200Device *dev, xb_inner_entry *e)
{
    for (void *p : e->allocs)
        cudaFreeAsync(p, dev->stream);
    cudaStreamSynchronize(dev->stream);
    delete e;
}

/* drop unreferenced entries, least recently used first, while the cache
 * holds more than its budget; inner_lock held */
void xb_inner_evict_locked(xpuB200Device *dev)
{
    while (dev->inner_bytes > dev->inner_budget) {
        int victim = -1;
        for (size_t i = 0; i < dev->inner_cache.size(); i++) {
            xb_inner_entry *e = dev->inner_cache[i];
            if (e->refs == 0 && (victim < 0 || e->last_use < dev->inner_cache[victim]->last_use))
                victim = (int)i;
        }
        if (victim < 0)
            return;
        xb_inner_entry *e = dev->inner_cache[victim];
        dev->inner_cache.erase(dev->inner_cache.begin() + victim);
        dev->inner_bytes -= e->bytes;
        xb_inner_entry_free(dev, e);
    }
}

/* the identity of an inner build: the caller's handle for the inner
 * relations' contents, and everything of the translated session the build
 * reads (descriptors before the build, the programs of the join quals it
 * evaluates with their constants, the group-id inputs) */
static uint64_t xb_inner_key(const xpuB200Device *dev, uint64_t handle, const xb_plan *plan, uint64_t kmrels_sz)
{
    uint64_t h = 1469598103934665603ULL;
    auto mix = [&](const void *p, size_t n) {
        const unsigned char *c = (const unsigned char *)p;
        for (size_t i = 0; i < n; i++) { h ^= c[i]; h *= 1099511628211ULL; }
    };
    mix(&dev->dindex, sizeof(dev->dindex));
    mix(&handle, sizeof(handle));
    mix(&kmrels_sz, sizeof(kmrels_sz));
    mix(&plan->nrels, sizeof(plan->nrels));
    mix(&plan->gid_depth, sizeof(plan->gid_depth));
    mix(&plan->gent_size, sizeof(plan->gent_size));
    mix(&plan->nkeys, sizeof(plan->nkeys));
    mix(plan->keys, sizeof(xb_key) * plan->nkeys);
    mix(&plan->nregs, sizeof(plan->nregs));
    for (uint32_t d = 1; d <= plan->nrels; d++) {
        mix(&plan->inner[d], sizeof(xb_inner));
        const xb_prog &q = plan->inner[d].build_qual;
        if (q.count && q.start + q.count <= plan->ninsns)
            mix(plan->insns + q.start, sizeof(xb_insn) * q.count);
    }
    return h;
}

static xb_inner_entry *xb_inner_cache_get(xpuB200Device *dev, uint64_t key)
{
    std::lock_guard<std::mutex> g(dev->inner_lock);
    for (xb_inner_entry *e : dev->inner_cache)
        if (e->key == key) {
            e->refs++;
            e->last_use = ++dev->inner_clock;
            return e;
        }
    return nullptr;
}

static void xb_inner_cache_put(xpuB200Device *dev, xb_inner_entry *e)
{
    std::lock_guard<std::mutex> g(dev->inner_lock);
    if (e->refs > 0)
        e->refs--;
    e->last_use = ++dev->inner_clock;
    xb_inner_evict_locked(dev);
}

cudaStream_t xb_get_stream(xpuB200Device *dev)
{
    {
        std::lock_guard<std::mutex> g(dev->pool_lock);
        if (!dev->free_streams.empty()) {
            cudaStream_t st = dev->free_streams.back();
            dev->free_streams.pop_back();
            return st;
        }
    }
    cudaStream_t st = nullptr;
    if (cudaStreamCreateWithFlags(&st, cudaStreamNonBlocking) != cudaSuccess)
        return nullptr;
    return st;
}

void xb_put_stream(xpuB200Device *dev, cudaStream_t st)
{
    if (!st) return;
    std::lock_guard<std::mutex> g(dev->pool_lock);
    dev->free_streams.push_back(st);
}

static xb_status *xb_get_status(xpuB200Device *dev)
{
    std::lock_guard<std::mutex> g(dev->pool_lock);
    if (dev->free_status.empty()) {
        const int n = 64;
        xb_status *blk = nullptr;
        if (cudaMallocHost((void **)&blk, sizeof(xb_status) * n) != cudaSuccess)
            return nullptr;
        dev->status_blocks.push_back(blk);
        for (int i = 0; i < n; i++)
            dev->free_status.push_back(blk + i);
    }
    xb_status *p = dev->free_status.back();
    dev->free_status.pop_back();
    return p;
}

static void xb_put_status(xpuB200Device *dev, xb_status *p)
{
    if (!p) return;
    std::lock_guard<std::mutex> g(dev->pool_lock);
    dev->free_status.push_back(p);
}



/* shared group-table capacity 'cap' and the launch geometry that follows
 * from it (shared memory of both kernels, the interpreter's grid); the
 * specialised kernels are prepared again at their next launch */
int xb_set_sm_cap(xpuB200Session *s, uint32_t cap)
{
    const xb_plan *plan = s->h_plan;
    size_t smem = s->plan_bytes + PGSTROM_TYPEALIGN(16, sizeof(XbSrcMeta)) +
                  (size_t)cap * plan->gent_size + (size_t)XB_WARPS * s->warp_bytes;
    s->smem_bytes = smem;
    if (smem > s->dev->smem_optin)
        return -1;
    int per_sm = 0;
    cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, xb_exec_kernel, XB_BLOCK, smem);
    if (per_sm < 1)
        return -1;
    s->sm_cap = cap;
    s->grid = per_sm * s->dev->nsm;
    s->jit_smem = PGSTROM_TYPEALIGN(16, sizeof(XbSrcMeta)) + sizeof(XbSrc) * XB_WARPS +
                  (size_t)cap * xb_jit_sm_stride(plan->gent_size ? plan->gent_size : 16);
    /* existence bitmaps staged after the group table (16-byte aligned) */
    size_t bits = 0;
    for (uint32_t d = 1; d <= plan->nrels; d++)
        bits += (size_t)plan->inner[d].dbits_words * 4;
    if (bits)
        s->jit_smem = PGSTROM_TYPEALIGN(16, s->jit_smem) + PGSTROM_TYPEALIGN(16, bits);
    for (int f = 0; f < 256; f++)
        s->jit_tried[f] = false;
    return 0;
}

const char *xb_msg_text(uint32_t id)
{
    switch (id) {
    case XB_MSG_INT_RANGE:        return "integer value out of range";
    case XB_MSG_DIV_ZERO:         return "division by zero";
    case XB_MSG_FLT_RANGE:        return "float value out of range";
    case XB_MSG_NUMERIC_RANGE:    return "numeric value is out of range";
    case XB_MSG_NUMERIC_CORRUPT:  return "corrupted numeric datum";
    case XB_MSG_VARLENA_EXTERNAL: return "external or compressed varlena is not supported";
    case XB_MSG_BAD_TUPLE:        return "corrupted tuple or unsupported datum in the chunk";
    case XB_MSG_GTABLE_FULL:      return "GpuPreAgg(GroupBy) - no space to write";
    case XB_MSG_WAIT_TIMEOUT:     return "group entry wait timed out";
    case XB_MSG_ARENA_FULL:       return "GpuPreAgg(GroupBy) - no space for variable-length keys";
    case XB_MSG_BAD_PAGE:         return "corrupted heap page";
    case XB_MSG_ARROW_TYPE:       return "Arrow column type does not match the device type";
    case XB_MSG_NUMERIC_TYPE:     return "numeric key or argument of an unsupported form";
    case XB_MSG_LEFT_FULL:        return "no room to record the work left for after the group table grows";
    default:                      return "device error";
    }
}

static_assert(XBJ_WARPS_PER_CTA == XB_WARPS, "specialised kernels assume the executor's CTA size");
/* the specialised kernels fetch bytes 48..63 of the group table (16-byte
 * aligned) for its 'grow' word, the second word there */
static_assert(offsetof(xb_gtable, grow) == 52 && offsetof(xb_gtable, overflow) == 48,
              "the group table's grow word moved");
static_assert(offsetof(XbSrc, grow_buf) % 16 == 0, "XbSrc.grow_buf must be 16-byte aligned");

int xb_set_error(kern_errorbuf *err, uint32_t code, const char *func, int line,
                        const char *fmt, ...)
{
    if (err) {
        memset(err, 0, sizeof(*err));
        err->errcode = code;
        err->lineno = line;
        snprintf(err->filename, sizeof(err->filename), "%s", "xb_exec.cu");
        snprintf(err->funcname, sizeof(err->funcname), "%s", func);
        va_list ap;
        va_start(ap, fmt);
        vsnprintf(err->message, sizeof(err->message), fmt, ap);
        va_end(ap);
    }
    return (int)code;
}
int xb_cuda_rc(cudaError_t rc, kern_errorbuf *err, const char *func, int line)
{
    if (rc == cudaSuccess)
        return 0;
    return xb_set_error(err, ERRCODE_DEVICE_FATAL, func, line, "%s", cudaGetErrorString(rc));
}


extern "C" int
xpuB200Init(int cuda_dindex, uint64_t hbm_budget, xpuB200Device **p_dev, kern_errorbuf *err)
{
    xb_clear_error(err);
    int ndev = 0;
    XB_CUDA(cudaGetDeviceCount(&ndev), err);
    if (cuda_dindex < 0 || cuda_dindex >= ndev)
        return XB_ERR(err, ERRCODE_DEVICE_FATAL, "GPU%d is not available (%d devices)", cuda_dindex, ndev);
    XB_CUDA(cudaSetDevice(cuda_dindex), err);
    cudaDeviceProp prop;
    XB_CUDA(cudaGetDeviceProperties(&prop, cuda_dindex), err);
    if (prop.major < 10)
        return XB_ERR(err, ERRCODE_DEVICE_FATAL, "GPU%d is sm_%d%d; this build needs sm_100a",
                      cuda_dindex, prop.major, prop.minor);
    xpuB200Device *dev = new xpuB200Device();
    dev->dindex = cuda_dindex;
    dev->nsm = prop.multiProcessorCount;
    if (hbm_budget == 0) {
        size_t fr = 0, tot = 0;
        cudaMemGetInfo(&fr, &tot);
        hbm_budget = (uint64_t)(fr * 0.9);
    }
    dev->hbm_budget = hbm_budget;
    /* sessions allocate from the device's stream-ordered pool; keep freed
     * memory in the pool instead of returning it at every synchronisation */
    {
        cudaMemPool_t pool;
        if (cudaDeviceGetDefaultMemPool(&pool, cuda_dindex) == cudaSuccess) {
            uint64_t keep = UINT64_MAX;
            cudaMemPoolSetAttribute(pool, cudaMemPoolAttrReleaseThreshold, &keep);
        }
    }
    /* the kernels shared by all sessions opt in to the whole of shared
     * memory once, so that no session lowers another's limit */
    dev->smem_optin = prop.sharedMemPerBlockOptin;
    if (cudaFuncSetAttribute(xb_exec_kernel, cudaFuncAttributeMaxDynamicSharedMemorySize,
                             (int)dev->smem_optin) != cudaSuccess ||
        cudaFuncSetAttribute(xb_mixed_kernel, cudaFuncAttributeMaxDynamicSharedMemorySize,
                             (int)(dev->smem_optin - sizeof(XbExecArgs) - 16)) != cudaSuccess ||
        cudaFuncSetAttribute(xb_build_inner, cudaFuncAttributeMaxDynamicSharedMemorySize,
                             (int)(dev->smem_optin - sizeof(XbCol) * XB_MAX_COLS)) != cudaSuccess) {
        delete dev;
        return XB_ERR(err, ERRCODE_DEVICE_FATAL, "cannot opt in to %zu bytes of shared memory",
                      (size_t)prop.sharedMemPerBlockOptin);
    }
    cudaError_t rc = cudaStreamCreateWithFlags(&dev->stream, cudaStreamNonBlocking);
    if (rc != cudaSuccess) {
        delete dev;
        return XB_ERR(err, ERRCODE_DEVICE_FATAL, "cudaStreamCreate: %s", cudaGetErrorString(rc));
    }
    *p_dev = dev;
    return 0;
}

extern "C" void
xpuB200Shutdown(xpuB200Device *dev)
{
    if (!dev) return;
    cudaSetDevice(dev->dindex);
    xb_sched_destroy(dev);
    for (xb_inner_entry *e : dev->inner_cache)
        xb_inner_entry_free(dev, e);
    dev->inner_cache.clear();
    for (auto &kv : dev->chunk_cache)
        cudaFreeAsync(kv.second.base, dev->stream);
    dev->chunk_cache.clear();
    cudaStreamSynchronize(dev->stream);
    cudaStreamDestroy(dev->stream);
    for (cudaStream_t st : dev->free_streams)
        cudaStreamDestroy(st);
    for (xb_status *b : dev->status_blocks)
        cudaFreeHost(b);
    delete dev;
}

static void xb_session_free(xpuB200Session *s)
{
    cudaSetDevice(s->dev->dindex);
    /* a background build goes on into the process-wide cache */
    for (int f = 0; f < 256; f++)
        if (s->jit_job[f])
            xb_jit_job_release(s->jit_job[f]);
    /* session memory comes from the device's stream-ordered pool, on the
     * session's stream: freeing it waits for no other stream (a plain
     * cudaFree would wait for the whole device, i.e. every other session's
     * work) */
    cudaStream_t st = s->stream;
    for (void *p : s->d_allocs)
        cudaFreeAsync(p, st);
    if (s->d_src) cudaFreeAsync(s->d_src, st);
    if (s->d_tasks) cudaFreeAsync(s->d_tasks, st);
    if (s->d_dst) cudaFreeAsync(s->d_dst, st);
    if (s->part_buf) cudaFreeAsync(s->part_buf, st);
    if (s->part_cnt) cudaFreeAsync(s->part_cnt, st);
    for (int i = 0; i < 2; i++)
        if (s->d_left[i]) cudaFreeAsync(s->d_left[i], st);
    if (s->h_plan && s->h_plan->has_groupby && s->h_gt.dump)
        cudaFreeAsync(s->h_gt.dump, st);
    cudaStreamSynchronize(st);
    if (s->inner_entry)
        xb_inner_cache_put(s->dev, s->inner_entry);
    xb_put_status(s->dev, s->h_status);
    if (s->h_plan) free(s->h_plan);
    for (cudaEvent_t e : s->ev_part)
        if (e) cudaEventDestroy(e);
    cudaEventDestroy(s->ev0);
    cudaEventDestroy(s->ev1);
    xb_put_stream(s->dev, s->stream);
    delete s;
}

static int xb_dalloc(xpuB200Session *s, size_t sz, void **p, kern_errorbuf *err)
{
    cudaError_t rc = cudaMallocAsync(p, sz < 256 ? 256 : sz, s->stream);
    if (rc != cudaSuccess) {
        *p = nullptr;
        cudaGetLastError();
        return XB_ERR(err, ERRCODE_DEVICE_FATAL, "cudaMalloc(%zu): %s", sz, cudaGetErrorString(rc));
    }
    s->d_allocs.push_back(*p);
    s->d_alloc_sz.push_back(sz);
    return 0;
}

static uint64_t xb_next_pow2(uint64_t x)
{
    uint64_t p = 1;
    while (p < x) p <<= 1;
    return p;
}

extern "C" int
xpuB200OpenSession(xpuB200Device *dev, const kern_session_info *session, uint64_t session_sz,
                   const kern_multirels *kmrels, uint64_t kmrels_sz,
                   xpuB200Session **p_sess, kern_errorbuf *err)
{
    xb_clear_error(err);
    *p_sess = nullptr;
    if (!dev || !session || session_sz < sizeof(kern_session_info))
        return XB_ERR(err, ERRCODE_DEVICE_ERROR, "invalid OpenSession arguments");
    XB_CUDA(cudaSetDevice(dev->dindex), err);
    xpuB200Session *s = new xpuB200Session();
    s->dev = dev;
    /* every session has its own stream, so that one session's launches,
     * copies and waits never wait for another's */
    s->stream = xb_get_stream(dev);
    if (!s->stream) {
        delete s;
        return XB_ERR(err, ERRCODE_DEVICE_FATAL, "cudaStreamCreate failed");
    }
    cudaEventCreate(&s->ev0);
    cudaEventCreate(&s->ev1);
    for (cudaEvent_t &e : s->ev_part)
        cudaEventCreate(&e);
    int rc;
    char msg[256];
#define FAIL(...) do { rc = XB_ERR(err, __VA_ARGS__); xb_session_free(s); return rc; } while (0)
#define DALLOC(sz, ptr) do { if ((rc = xb_dalloc(s, (sz), (void **)(ptr), err)) != 0) { xb_session_free(s); return rc; } } while (0)

    s->h_session.assign((const char *)session, (const char *)session + session_sz);
    DALLOC(session_sz, &s->d_session);
    if (kmrels) {
        if (kmrels_sz < offsetof(kern_multirels, chunks) ||
            kmrels->num_inner_rels > XB_MAX_DEPTH ||
            offsetof(kern_multirels, chunks) + sizeof(kmrels->chunks[0]) * kmrels->num_inner_rels > kmrels_sz)
            FAIL(ERRCODE_DEVICE_ERROR, "kern_multirels is broken");
    }
    s->h_plan = (xb_plan *)calloc(1, sizeof(xb_plan));
    if (xb_compile_session(session, session_sz, (uint64_t)s->d_session, kmrels,
                           s->h_plan, msg, sizeof(msg)) != 0)
        FAIL(ERRCODE_DEVICE_ERROR, "bytecode translation: %s", msg);
    xb_plan *plan = s->h_plan;
    cudaStream_t st = s->stream;
    if (cudaMemcpyAsync(s->d_session, session, session_sz, cudaMemcpyHostToDevice, st) != cudaSuccess)
        FAIL(ERRCODE_DEVICE_FATAL, "session upload failed");
    DALLOC(sizeof(xb_status), &s->d_status);
    s->h_status = xb_get_status(dev);
    if (!s->h_status)
        FAIL(ERRCODE_DEVICE_FATAL, "cudaMallocHost failed");
    cudaMemsetAsync(s->d_status, 0, sizeof(xb_status), st);

    /* inner relations built before for the same join_inner_handle and
     * build inputs are used as they are */
    xb_inner_entry *hit = nullptr;
    uint64_t ikey = 0;
    const uint64_t ihandle = ((const kern_session_info *)session)->join_inner_handle;
    if (kmrels && plan->nrels > 0 && ihandle != 0) {
        ikey = xb_inner_key(dev, ihandle, plan, kmrels_sz);
        hit = xb_inner_cache_get(dev, ikey);
        if (hit) {
            for (uint32_t d = 1; d <= plan->nrels; d++)
                plan->inner[d] = hit->inner[d];
            s->inner_entry = hit;
            s->inner_hit = true;
        }
    }
    const size_t ia0 = s->d_allocs.size();
    /* inner relations: upload and build indexes */
    if (kmrels && plan->nrels > 0 && !hit) {
        DALLOC(kmrels_sz, &s->d_kmrels);
        if (cudaMemcpyAsync(s->d_kmrels, kmrels, kmrels_sz, cudaMemcpyHostToDevice, st) != cudaSuccess)
            FAIL(ERRCODE_DEVICE_FATAL, "inner buffer upload failed");
        for (uint32_t d = 1; d <= plan->nrels; d++) {
            uint64_t koff = kmrels->chunks[d - 1].kds_offset;
            if (koff == 0 || koff + sizeof(kern_data_store) > kmrels_sz)
                FAIL(ERRCODE_DEVICE_ERROR, "inner KDS at depth %u is out of the buffer", d);
            const kern_data_store *hk = (const kern_data_store *)((const char *)kmrels + koff);
            if (hk->format != KDS_FORMAT_HASH || koff + hk->length > kmrels_sz ||
                KDS_HEAD_LENGTH(hk) + sizeof(uint64_t) * ((uint64_t)hk->hash_nslots + hk->nitems) > hk->length)
                FAIL(ERRCODE_DEVICE_ERROR, "inner KDS at depth %u is not a valid KDS_FORMAT_HASH", d);
            xb_inner *in = &plan->inner[d];
            in->nitems = hk->nitems;
            uint64_t cap = xb_next_pow2((uint64_t)hk->nitems * 2 + 64);
            in->cap_mask = (uint32_t)(cap - 1);
            in->unique_hash = 1;
            uint32_t n = hk->nitems > 0 ? hk->nitems : 1;
            uint32_t words = (n + 31) / 32;
            uint32_t nl = in->nloads > 0 ? in->nloads : 1;
            DALLOC(cap * 8, &in->index);
            DALLOC((size_t)nl * n * 8, &in->vals);
            DALLOC((size_t)nl * n * 4, &in->auxs);
            DALLOC((size_t)nl * words * 4, &in->nulls);
            in->hashes = nullptr;
            in->dkey_min = INT32_MAX;
            in->dkey_max = INT32_MIN;
            in->nindexed = 0;
            in->direct = 0;
            in->drange = 0;
            in->dtab = nullptr;
            in->drec_size = 0;
            in->dpay = nullptr;
            in->gid_on = 0;
            in->ngids = 0;
            in->gids = nullptr;
            in->dbits_words = 0;
            in->dbits = nullptr;
            if (in->hashed)
                DALLOC((size_t)nl * n * 4, &in->hashes);
            cudaMemsetAsync(in->index, 0, cap * 8, st);
            cudaMemsetAsync(in->nulls, 0, (size_t)nl * words * 4, st);
        }
    }
    const size_t ia1 = s->d_allocs.size();
    /* group-by tables */
    if (plan->has_groupby) {
        double est = ((const kern_session_info *)s->h_session.data())->groupby_ngroups_estimation;
        if (!(est >= 1.0)) est = 1.0;
        if (plan->has_groupby == 2) est = 1.0;
        /* open addressing at a load of at most 1/4 (small tables) or 1/2
         * (above a million groups, where the table's bytes matter) */
        uint64_t cap = xb_next_pow2((uint64_t)(est * (est > 1e6 ? 2 : 4)) + 1024);
        uint64_t max_cap = (dev->hbm_budget / 4) / plan->gent_size;
        if (cap > max_cap) cap = xb_next_pow2(max_cap / 2 + 1);
        uint64_t arena = plan->nkeys_text ? (64ULL << 20) + cap * 32 : 256;
        s->h_gt.cap_mask = cap - 1;
        s->h_gt.nused = 0;
        s->h_gt.arena_sz = arena;
        s->h_gt.arena_used = 0;
        s->h_gt.overflow = 0;
        s->h_gt.grow = 0;
        s->h_gt.soft_cap = cap / 2;
        s->h_gt.dump = nullptr;
        s->h_gt.dump_cap = 0;
        s->h_gt.dump_used = 0;
        DALLOC(cap * plan->gent_size, &s->h_gt.entries);
        DALLOC(arena, &s->h_gt.arena);
        cudaMemsetAsync(s->h_gt.entries, 0, cap * plan->gent_size, st);
        DALLOC(sizeof(xb_gtable), &s->d_gt);
        cudaMemcpyAsync(s->d_gt, &s->h_gt, sizeof(xb_gtable), cudaMemcpyHostToDevice, st);
        /* shared-memory table for small group counts */
        if (est <= 2048 && plan->gent_size <= 256) {
            uint32_t smc = (uint32_t)xb_next_pow2((uint64_t)(est * 4) + 16);
            if (smc < 32) smc = 32;
            while ((size_t)smc * plan->gent_size > 48 * 1024 && smc > 32) smc >>= 1;
            if ((size_t)smc * plan->gent_size <= 48 * 1024)
                s->sm_cap = smc;
        }
    }
    /* test hooks, inert unless set: XPU_B200_WAIT_LIMIT shortens the
     * bounded wait on a BUSY group entry; XPU_B200_TEST_BUSY_GROUPS=1 marks
     * every global entry BUSY, as if its creator never published it, so
     * that every lookup runs its wait out and the launch reports
     * XB_MSG_WAIT_TIMEOUT */
    if (const char *wl = getenv("XPU_B200_WAIT_LIMIT")) {
        const unsigned long v = strtoul(wl, nullptr, 10);
        if (v > 0 && v < XB_WAIT_LIMIT)
            plan->wait_limit = (uint32_t)v;
    }
    if (plan->has_groupby) {
        const char *busy = getenv("XPU_B200_TEST_BUSY_GROUPS");
        if (busy && busy[0] == '1') {
            const uint64_t n = s->h_gt.cap_mask + 1, gsz = plan->gent_size;
            std::vector<char> img(n * gsz, 0);
            for (uint64_t i = 0; i < n; i++)
                ((xb_gent_head *)(img.data() + i * gsz))->state = XB_GSTATE_BUSY;
            cudaMemcpyAsync(s->h_gt.entries, img.data(), img.size(), cudaMemcpyHostToDevice, st);
            cudaStreamSynchronize(st);
        }
    }
    DALLOC(sizeof(xb_plan), &s->d_plan);
    cudaMemcpyAsync(s->d_plan, plan, sizeof(xb_plan), cudaMemcpyHostToDevice, st);

    /* build inner indexes on the device */
    for (uint32_t d = 1; !hit && d <= plan->nrels; d++) {
        XbBuildArgs ba;
        ba.kds = (const kern_data_store *)(s->d_kmrels + kmrels->chunks[d - 1].kds_offset);
        ba.in = &s->d_plan->inner[d];
        ba.plan = s->d_plan;
        ba.st = s->d_status;
        uint32_t n = plan->inner[d].nitems;
        int grid = (int)((n + XB_BLOCK - 1) / XB_BLOCK);
        if (grid < 1) grid = 1;
        if (grid > dev->nsm * 8) grid = dev->nsm * 8;
        const size_t bsmem = plan->inner[d].build_qual.count ? (size_t)XB_WARPS * XB_REGS_BYTES(plan->nregs) : 0;
        if (bsmem + sizeof(XbCol) * XB_MAX_COLS > dev->smem_optin)
            FAIL(ERRCODE_DEVICE_FATAL, "inner build needs %zu bytes of shared memory", bsmem);
        xb_build_inner<<<grid, XB_BLOCK, bsmem, st>>>(ba);
    }
    /* canonical text pointers for hashed text columns: equal strings of one
     * inner column share one address, so group keys taken from them compare
     * by pointer */
    for (uint32_t d = 1; !hit && d <= plan->nrels; d++) {
        const xb_inner *in = &plan->inner[d];
        for (uint32_t k = 0; k < in->nloads; k++) {
            if (!((in->hashed >> k) & 1u) || in->load[k].ld != XB_LD_TEXT || in->nitems == 0)
                continue;
            const uint64_t tcap = xb_next_pow2((uint64_t)in->nitems * 2 + 64);
            uint32_t *table = nullptr;
            if (cudaMallocAsync((void **)&table, tcap * 4, st) != cudaSuccess)
                FAIL(ERRCODE_DEVICE_FATAL, "OpenSession: no device memory for text canonicalisation");
            cudaMemsetAsync(table, 0, tcap * 4, st);
            int grid = (int)((in->nitems + XB_BLOCK - 1) / XB_BLOCK);
            if (grid > dev->nsm * 8) grid = dev->nsm * 8;
            xb_canon_text<<<grid, XB_BLOCK, 0, st>>>(&s->d_plan->inner[d], k, table,
                                                      (uint32_t)(tcap - 1), s->d_status);
            cudaFreeAsync(table, st);
        }
    }
    if (cudaStreamSynchronize(st) != cudaSuccess)
        FAIL(ERRCODE_DEVICE_FATAL, "OpenSession: %s", cudaGetErrorString(cudaGetLastError()));
    cudaMemcpy(s->h_status, s->d_status, sizeof(xb_status), cudaMemcpyDeviceToHost);
    if (s->h_status->errcode)
        FAIL(s->h_status->errcode, "inner relation build: %s", xb_msg_text(s->h_status->msg_id));
    /* refresh the host copy of the inner descriptors (unique_hash) */
    cudaMemcpy(s->h_plan, s->d_plan, sizeof(xb_plan), cudaMemcpyDeviceToHost);
    /* dense group ids when every GROUP BY key is a column of one inner
     * relation; the specialised kernels then index the shared-memory group
     * table by id.  Needs the shared table to hold every id. */
    const size_t ia2 = s->d_allocs.size();
    if (hit && hit->gid_cap && s->sm_cap < hit->gid_cap)
        s->sm_cap = hit->gid_cap;
    if (!hit && s->h_plan->gid_depth >= 1 && s->h_plan->gid_depth <= plan->nrels && plan->gent_size > 0) {
        const uint32_t d = s->h_plan->gid_depth;
        xb_inner *in = &s->h_plan->inner[d];
        const uint32_t n = in->nitems;
        const uint32_t limit = (48 * 1024) / plan->gent_size;
        if (n > 0) {
            DALLOC((size_t)n * 4, &in->gids);
            cudaMemcpyAsync(&s->d_plan->inner[d], in, sizeof(xb_inner), cudaMemcpyHostToDevice, st);
            const uint64_t tcap = xb_next_pow2((uint64_t)n * 2 + 64);
            uint32_t *table = nullptr, *rep = nullptr, *counter = nullptr;
            if (cudaMallocAsync((void **)&table, tcap * 4, st) != cudaSuccess ||
                cudaMallocAsync((void **)&rep, (size_t)n * 4, st) != cudaSuccess ||
                cudaMallocAsync((void **)&counter, 4, st) != cudaSuccess)
                FAIL(ERRCODE_DEVICE_FATAL, "OpenSession: no device memory for group ids");
            cudaMemsetAsync(table, 0, tcap * 4, st);
            cudaMemsetAsync(counter, 0, 4, st);
            int grid = (int)((n + XB_BLOCK - 1) / XB_BLOCK);
            if (grid > dev->nsm * 8) grid = dev->nsm * 8;
            xb_gid_rep<<<grid, XB_BLOCK, 0, st>>>(s->d_plan, &s->d_plan->inner[d], table, (uint32_t)(tcap - 1), rep);
            xb_gid_number<<<grid, XB_BLOCK, 0, st>>>(&s->d_plan->inner[d], rep, counter);
            xb_gid_fill<<<grid, XB_BLOCK, 0, st>>>(&s->d_plan->inner[d], rep);
            uint32_t ngids = 0;
            cudaMemcpyAsync(&ngids, counter, 4, cudaMemcpyDeviceToHost, st);
            cudaFreeAsync(table, st);
            cudaFreeAsync(rep, st);
            cudaFreeAsync(counter, st);
            if (cudaStreamSynchronize(st) != cudaSuccess)
                FAIL(ERRCODE_DEVICE_FATAL, "OpenSession: %s", cudaGetErrorString(cudaGetLastError()));
            const uint32_t cap = (uint32_t)xb_next_pow2(ngids > 32 ? ngids : 32);
            if (ngids >= 1 && ngids <= limit && (size_t)cap * plan->gent_size <= 48 * 1024) {
                in->gid_on = 1;
                in->ngids = ngids;
                if (s->sm_cap < cap)
                    s->sm_cap = cap;
                cudaMemcpyAsync(&s->d_plan->inner[d], in, sizeof(xb_inner), cudaMemcpyHostToDevice, st);
            }
        }
    }
    /* direct-address tables for unique, dense 32-bit join keys (used by the
     * session-specialised kernels; the interpreter keeps probing the index) */
    for (uint32_t d = 1; !hit && d <= plan->nrels; d++) {
        xb_inner *in = &s->h_plan->inner[d];
        if (!in->key32 || !in->unique_hash || in->nindexed == 0 || in->dkey_max < in->dkey_min)
            continue;
        const uint64_t range = (uint64_t)((int64_t)in->dkey_max - in->dkey_min) + 1;
        const uint64_t limit = (uint64_t)in->nitems * 4 > 4096 ? (uint64_t)in->nitems * 4 : 4096;
        if (range > limit || range > (1ULL << 28))
            continue;
        DALLOC(range * 4, &in->dtab);
        cudaMemsetAsync(in->dtab, 0, range * 4, st);
        in->drange = (uint32_t)range;
        in->direct = 1;
        /* live columns packed per key when the records stay small */
        const uint32_t rs = xb_drec_layout(in, s->h_plan->rk, -1, nullptr, nullptr, nullptr);
        if (in->live && rs <= 64) {
            DALLOC(range * rs, &in->dpay);
            cudaMemsetAsync(in->dpay, 0, range * rs, st);
            in->drec_size = rs;
        }
        /* a depth that only filters (no columns of its rows are used):
         * an existence bitmap, staged in shared memory by the specialised
         * kernels when it is small */
        if (!in->live && range <= XB_DBITS_MAX_KEYS) {
            in->dbits_words = (uint32_t)((range + 31) / 32);
            DALLOC((size_t)in->dbits_words * 4, &in->dbits);
        }
        cudaMemcpyAsync(&s->d_plan->inner[d], in, sizeof(xb_inner), cudaMemcpyHostToDevice, st);
        int grid = (int)((in->cap_mask + 1ULL + XB_BLOCK - 1) / XB_BLOCK);
        if (grid > dev->nsm * 8) grid = dev->nsm * 8;
        xb_build_direct<<<grid, XB_BLOCK, 0, st>>>(&s->d_plan->inner[d]);
        if (in->dpay)
            xb_build_drec<<<grid, XB_BLOCK, 0, st>>>(&s->d_plan->inner[d], s->d_plan);
        if (in->dbits) {
            int g2 = (int)((in->dbits_words + XB_BLOCK - 1) / XB_BLOCK);
            xb_build_dbits<<<g2 > 0 ? g2 : 1, XB_BLOCK, 0, st>>>(&s->d_plan->inner[d]);
        }
    }
    if (cudaStreamSynchronize(st) != cudaSuccess)
        FAIL(ERRCODE_DEVICE_FATAL, "OpenSession: %s", cudaGetErrorString(cudaGetLastError()));
    const size_t ia3 = s->d_allocs.size();
    /* a new build with a handle goes into the cache: its device memory
     * leaves the session's and stays while any session uses it */
    if (!hit && ikey != 0) {
        xb_inner_entry *e = new xb_inner_entry();
        e->key = ikey;
        e->nrels = plan->nrels;
        for (uint32_t d = 0; d <= XB_MAX_DEPTH; d++)
            e->inner[d] = s->h_plan->inner[d];
        const uint32_t gd = s->h_plan->gid_depth;
        e->gid_cap = (gd >= 1 && gd <= plan->nrels && s->h_plan->inner[gd].gid_on)
            ? (uint32_t)xb_next_pow2(s->h_plan->inner[gd].ngids > 32 ? s->h_plan->inner[gd].ngids : 32) : 0;
        std::vector<void *> keep_p;
        std::vector<uint64_t> keep_sz;
        for (size_t i = 0; i < s->d_allocs.size(); i++) {
            if ((i >= ia0 && i < ia1) || (i >= ia2 && i < ia3)) {
                e->allocs.push_back(s->d_allocs[i]);
                e->bytes += s->d_alloc_sz[i];
            } else {
                keep_p.push_back(s->d_allocs[i]);
                keep_sz.push_back(s->d_alloc_sz[i]);
            }
        }
        s->d_allocs.swap(keep_p);
        s->d_alloc_sz.swap(keep_sz);
        s->d_kmrels = nullptr;
        e->refs = 1;
        std::lock_guard<std::mutex> g(dev->inner_lock);
        e->last_use = ++dev->inner_clock;
        dev->inner_cache.push_back(e);
        dev->inner_bytes += e->bytes;
        s->inner_entry = e;
    }

    /* launch geometry */
    s->warp_bytes = (uint32_t)(XB_WARP_HEAD + sizeof(XbCursor) * plan->nrels + XB_REGS_BYTES(plan->nregs));
    s->plan_bytes = (uint32_t)PGSTROM_TYPEALIGN(16, offsetof(xb_plan, insns) +
                                                 sizeof(xb_insn) * (size_t)plan->ninsns);
    s->sm_cap_default = s->sm_cap;
    if (xb_set_sm_cap(s, s->sm_cap) != 0)
        FAIL(ERRCODE_DEVICE_FATAL, "executor kernel does not fit on an SM (%zu bytes smem)", s->smem_bytes);
    {
        const char *env = getenv("XPU_B200_JIT");
        s->jit_enabled = !(env && env[0] == '0');
        s->jit_msg = s->jit_enabled ? "not built yet" : "disabled";
    }
#undef FAIL
#undef DALLOC
    *p_sess = s;
    return 0;
}

extern "C" void
xpuB200CloseSession(xpuB200Session *sess)
{
    if (sess) {
        xb_sched_drain_session(sess);
        xb_session_free(sess);
    }
}

/* remember the heap layout of the first heap chunk a session sees, before
 * its specialised kernel is built: the kernel reads the depth-0 columns at
 * these offsets (and checks each launch's layout against them); session
 * lock held */
static void xb_note_walk(xb_plan *p, const kern_data_store *h);
static void xb_note_layout_plan(xb_plan *p, const kern_data_store *h);

void xb_note_layout(xpuB200Session *s, const kern_data_store *h)
{
    if (s->jit_tried[KDS_FORMAT_BLOCK])
        return;
    xb_note_layout_plan(s->h_plan, h);
}

/* the same on a translated plan, for the generator's tests */
extern "C" void xb_plan_note_layout(xb_plan *p, const kern_data_store *h)
{
    xb_note_layout_plan(p, h);
}

static void xb_note_layout_plan(xb_plan *p, const kern_data_store *h)
{
    if (h->format != KDS_FORMAT_BLOCK || p->lay_valid || p->walk_ncols)
        return;
    xb_note_walk(p, h);
    uint32_t end = 0;
    for (uint32_t i = 0; i < p->nload0; i++) {
        const xb_load &l = p->load0[i];
        int w = 0;
        switch (l.ld) {
        case XB_LD_BOOL: w = 1; break;
        case XB_LD_INT2: w = 2; break;
        case XB_LD_INT4: case XB_LD_DATE: case XB_LD_FLT4: w = 4; break;
        case XB_LD_INT8: case XB_LD_FLT8: w = 8; break;
        default: return;
        }
        if (l.resno < 1 || l.resno > (int)h->ncols || l.resno > (int)h->nr_colmeta)
            return;
        const kern_colmeta &cm = h->colmeta[l.resno - 1];
        if (cm.attlen != w || cm.attcacheoff < 0 || (cm.attcacheoff % w) != 0)
            return;
        p->lay_off[i] = cm.attcacheoff;
        if ((uint32_t)(cm.attcacheoff + w) > end)
            end = cm.attcacheoff + w;
    }
    p->lay_end = end;
    p->lay_valid = p->nload0 > 0 ? 1 : 0;
}

/* the column descriptors up to the last depth-0 column, when every one of
 * them is fixed-width (1..8 bytes) or a varlena and every fixed-width
 * load is naturally aligned by its column's attalign: the specialised
 * kernel then walks tuples with NULLs, or with varlena columns before a
 * loaded column, in straight-line code (checked against each launch's
 * columns) */
static void xb_note_walk(xb_plan *p, const kern_data_store *h)
{
    p->walk_ncols = 0;
    const int n = p->max_resno0;
    if (p->nload0 == 0 || n < 1 || n > XB_MAX_COLS || n > (int)h->ncols || n > (int)h->nr_colmeta)
        return;
    for (int j = 0; j < n; j++) {
        const kern_colmeta &cm = h->colmeta[j];
        const int al = cm.attalign;
        if (!(cm.attlen == -1 || (cm.attlen >= 1 && cm.attlen <= 8)) || !(al == 1 || al == 2 || al == 4 || al == 8))
            return;
        p->walk_len[j] = cm.attlen;
        p->walk_align[j] = (int8_t)al;
    }
    for (uint32_t i = 0; i < p->nload0; i++) {
        const xb_load &l = p->load0[i];
        if (l.resno < 1 || l.resno > n)
            return;
        const int len = p->walk_len[l.resno - 1], al = p->walk_align[l.resno - 1];
        int w = 0;
        switch (l.ld) {
        case XB_LD_BOOL: w = 1; break;
        case XB_LD_INT2: w = 2; break;
        case XB_LD_INT4: case XB_LD_DATE: case XB_LD_FLT4: w = 4; break;
        case XB_LD_INT8: case XB_LD_FLT8: w = 8; break;
        case XB_LD_TEXT: case XB_LD_NUMERIC: w = -1; break;
        default: return;
        }
        if (len != w || (w > 0 && al < w))
            return;
    }
    p->walk_ncols = (uint32_t)n;
}

/* units of one chunk (pages, or 1024-row groups) */
uint32_t xb_chunk_units(const kern_data_store *head)
{
    if (head->format == KDS_FORMAT_BLOCK)
        return head->nitems;
    return (head->nitems + XB_ROWS_UNIT - 1) / XB_ROWS_UNIT;
}

/* launch the executor over a device-resident task table, on a stream
 * with a status of the caller's */
int xb_launch_on(xpuB200Session *s, const xb_task *d_tasks, uint32_t ntasks,
                        uint64_t nunits, uint32_t format, cudaStream_t stream, xb_status *d_status,
                        kern_errorbuf *err);

/* ----------------------------------------------------------------
 * launch-shape tuning: resident CTAs per SM of the specialised kernels and
 * the shared group table's capacity, measured on a batch of chunks and
 * remembered per GPU for every session of the same plan shape and default
 * table capacity (the caller's group-count estimate)
 * ---------------------------------------------------------------- */
std::mutex g_tune_lock;
std::map<std::tuple<int, uint64_t, uint32_t>, xb_tune_choice> g_tune;
std::map<std::pair<int, uint64_t>, int> g_tune_minb;

std::tuple<int, uint64_t, uint32_t> xb_tune_key(xpuB200Session *s, uint32_t format)
{
    return std::make_tuple(s->dev->dindex, xb_jit_shape_key(s->h_plan, format), s->sm_cap_default);
}

static bool xb_tune_lookup(xpuB200Session *s, uint32_t format, xb_tune_choice *c)
{
    {
        std::lock_guard<std::mutex> g(g_tune_lock);
        if (g_tune.empty())
            return false;
    }
    const auto key = xb_tune_key(s, format);
    std::lock_guard<std::mutex> g(g_tune_lock);
    auto it = g_tune.find(key);
    if (it != g_tune.end()) {
        *c = it->second;
        return true;
    }
    auto im = g_tune_minb.find(std::make_pair(std::get<0>(key), std::get<1>(key)));
    if (im == g_tune_minb.end())
        return false;
    c->minb = im->second;
    c->sm_cap = s->sm_cap;
    return true;
}

/* the session-specialised kernel of this format (nullptr: use the
 * interpreter), built on first use; session lock held */
/*
 * The session's specialised kernel for a source format, built at its first
 * use.  wait == false (served launches): a kernel the process has not
 * built yet is built on a background thread while this launch, and the
 * next ones until it is there, run on the interpreting kernel, so that a
 * request of a new plan shape does not wait seconds for NVRTC.
 */
static void xb_session_adopt_jit(xpuB200Session *s, uint32_t format, int rc, double ms, const char *msg);

void *xb_session_jit(xpuB200Session *s, uint32_t format, bool wait)
{
    if (!s->jit_enabled || format >= 256)
        return nullptr;
    if (!s->tune_looked_up) {
        /* a launch shape tuned for this plan shape by another session */
        s->tune_looked_up = true;
        xb_tune_choice c;
        if (xb_tune_lookup(s, format, &c)) {
            s->jit_minb = c.minb;
            if (c.sm_cap != s->sm_cap && xb_set_sm_cap(s, c.sm_cap) != 0)
                xb_set_sm_cap(s, s->sm_cap_default);
        }
    }
    if (s->jit_tried[format])
        return s->jit_fn[format];
    char msg[1024] = {0};
    double ms = 0.0;
    if (!s->jit_job[format] && !wait) {
        const int lrc = xb_jit_lookup_minb(s->h_plan, format, s->dev->dindex, s->jit_minb, &s->jit_fn[format],
                                           &s->jit_mixfn[format], &s->jit_replay[format]);
        if (lrc == 1) {
            s->jit_job[format] = xb_jit_build_async(s->h_plan, format, s->dev->dindex, s->jit_minb);
            if (s->jit_job[format]) {
                s->jit_msg = "building in the background";
                return nullptr;
            }
        } else {
            xb_session_adopt_jit(s, format, lrc, 0.0, "not buildable");
            return s->jit_fn[format];
        }
    }
    if (s->jit_job[format]) {
        int prc;
        while ((prc = xb_jit_job_poll(s->jit_job[format], &s->jit_fn[format], &s->jit_mixfn[format],
                                      &s->jit_replay[format], &ms, msg, sizeof(msg))) == 1) {
            if (!wait)
                return nullptr;
            std::this_thread::sleep_for(std::chrono::milliseconds(2));
        }
        xb_jit_job_release(s->jit_job[format]);
        s->jit_job[format] = nullptr;
        xb_session_adopt_jit(s, format, prc, ms, msg);
        return s->jit_fn[format];
    }
    const int crc = xb_jit_compile_minb(s->h_plan, format, s->dev->dindex, s->jit_minb, &s->jit_fn[format],
                                        &s->jit_mixfn[format], &s->jit_replay[format], &ms, msg, sizeof(msg));
    xb_session_adopt_jit(s, format, crc, ms, msg);
    return s->jit_fn[format];
}

/* the kernels just found or built (rc 0), or the reason there are none */
static void xb_session_adopt_jit(xpuB200Session *s, uint32_t format, int rc, double ms, const char *msg)
{
    s->jit_tried[format] = true;
    {
        int per_sm = 0, mix_sm = 0;
        if (rc != 0) {
            s->jit_fn[format] = nullptr;
            s->jit_mixfn[format] = nullptr;
            s->jit_replay[format] = nullptr;
            s->jit_msg = msg;
        } else if ((s->jit_smem_fmt[format] = s->jit_smem + xb_jit_stage_bytes(format)) == 0 ||
                   xb_jit_prepare(s->jit_fn[format], XB_BLOCK, s->jit_smem_fmt[format], &per_sm) != 0) {
            s->jit_fn[format] = nullptr;
            s->jit_mixfn[format] = nullptr;
            s->jit_msg = "specialised kernel does not fit on an SM";
        } else {
            /* the mixed kernel is shared by sessions of one plan shape with
             * their own table sizes: it opts in to all shared memory that
             * its static shared memory leaves */
            if (s->jit_mixfn[format] &&
                xb_jit_prepare(s->jit_mixfn[format], XB_BLOCK,
                               s->dev->smem_optin - xb_jit_static_smem(s->jit_mixfn[format]) - 16, &mix_sm) != 0)
                s->jit_mixfn[format] = nullptr;
            s->jit_grid[format] = per_sm * s->dev->nsm;
            int rp = 0;
            if (s->jit_replay[format] && xb_jit_prepare(s->jit_replay[format], XB_BLOCK, 0, &rp) != 0)
                s->jit_replay[format] = nullptr;
            s->jit_replay_grid[format] = rp * s->dev->nsm;
            s->jit_compile_ms += ms;
            s->jit_msg = "ok";
        }
    }
}

static int xb_launch_tasks(xpuB200Session *s, const xb_task *d_tasks, uint32_t ntasks,
                           uint64_t nunits, uint32_t format, kern_errorbuf *err)
{
    return xb_launch_on(s, d_tasks, ntasks, nunits, format, s->stream, s->d_status, err);
}

/* partitioned aggregation for this launch: a keyed GROUP BY whose groups
 * live in a global table larger than L2 defers each row's update into the
 * bucket of its table slot; a bucket covers a slice of the table small
 * enough for the slices the replay's CTAs work on together to stay in L2.
 * Rows past a full bucket are updated in place, so any bucket size is
 * correct.  Used by
 * prepared batches whose table is several times L2 (the records of a batch
 * take device memory in proportion to its rows, which the serving path's
 * admission does not budget); XPU_B200_PARTITION=1 uses it for every
 * launch on the session's stream over a table above 64 MB, =0 never;
 * XPU_B200_PART_CAP=n (a test hook) clips the buckets to n records, so
 * that rows past full buckets are updated in place while others of the
 * same groups are deferred.  Session lock held.  Returns whether it is
 * used. */
/* table slots of one bucket of partitioned aggregation: about 128 KB of
 * global table (1024 of the Arrow group-by's 112-byte entries; measured
 * against 512, 2048 and 4096 slots); XPU_B200_PART_SLOTS=n (a power of two,
 * 64..65536) sets it */
static uint32_t xb_replay_slots(const xb_plan *plan)
{
    static const uint32_t forced = [] {
        const char *e = getenv("XPU_B200_PART_SLOTS");
        const unsigned long v = e ? strtoul(e, nullptr, 10) : 0;
        return (v >= 64 && v <= 65536 && (v & (v - 1)) == 0) ? (uint32_t)v : 0u;
    }();
    if (forced)
        return forced;
    const uint64_t gsz = plan->gent_size ? plan->gent_size : 16;
    uint32_t c = 8192;
    while (c > 64 && c * gsz > (128u << 10))
        c >>= 1;
    return c;
}

static bool xb_part_prepare(xpuB200Session *s, uint64_t nunits, uint32_t format, cudaStream_t stream)
{
    const char *env = getenv("XPU_B200_PARTITION");
    const bool force = env && env[0] == '1';
    if ((env && env[0] == '0') || (!force && !s->in_batch))
        return false;
    /* the bucket buffers are the session's: only launches on the session's
     * own stream use them (served launches on pooled slot streams may run
     * concurrently with each other and would share them) */
    if (stream != s->stream)
        return false;
    const xb_plan *plan = s->h_plan;
    if (plan->has_groupby != 1 || s->sm_cap != 0)
        return false;
    const uint32_t rec = xb_jit_part_rec_size(plan, format);
    const uint64_t cap = s->h_gt.cap_mask + 1;
    const uint64_t table = cap * plan->gent_size;
    if (rec == 0 || table <= (force ? (64ULL << 20) : (512ULL << 20)))
        return false;
    /* one bucket per slice of the table that a replay CTA's shared table
     * covers: at the table's load its groups fit in shared memory */
    uint64_t np = cap / xb_replay_slots(plan);
    while (np > XB_PART_MAX)
        np >>= 1;
    if (np < 8 || np * 2 > cap)
        return false;
    uint32_t lg_cap = 0, lg_np = 0;
    while ((1ULL << lg_cap) < cap) lg_cap++;
    while ((1ULL << lg_np) < np) lg_np++;
    const uint64_t rows = format == KDS_FORMAT_BLOCK ? nunits * 291ULL : nunits * (uint64_t)XB_ROWS_UNIT;
    uint64_t per = (rows + rows / 4) / np + 256;
    /* at most a quarter of the device budget for the records */
    const uint64_t limit = s->dev->hbm_budget / 4;
    if (per * np * rec > limit)
        per = limit / (np * rec);
    if (per < 256 || per > 0xffffffffULL)
        return false;
    const char *cap_env = getenv("XPU_B200_PART_CAP");
    const uint64_t cap_force = cap_env ? strtoull(cap_env, nullptr, 10) : 0;
    const uint64_t bytes = per * np * rec;
    if (!s->part_buf || s->part_bytes < bytes || s->nparts != np) {
        if (s->part_buf) cudaFreeAsync(s->part_buf, stream);
        if (s->part_cnt) cudaFreeAsync(s->part_cnt, stream);
        s->part_buf = nullptr;
        s->part_cnt = nullptr;
        s->part_bytes = 0;
        if (cudaMallocAsync((void **)&s->part_buf, bytes, stream) != cudaSuccess ||
            /* the bucket counters, then the replay's bucket cursor */
            cudaMallocAsync((void **)&s->part_cnt, sizeof(uint32_t) * XB_PART_CNT_STRIDE * (np + 1), stream) !=
                cudaSuccess) {
            cudaGetLastError();
            if (s->part_buf) cudaFreeAsync(s->part_buf, stream);
            s->part_buf = nullptr;
            s->part_cnt = nullptr;
            return false;
        }
        s->part_bytes = bytes;
    }
    s->part_cap = (uint32_t)(s->part_bytes / (np * rec));
    if (cap_force > 0 && cap_force < s->part_cap)
        s->part_cap = (uint32_t)cap_force;
    s->nparts = (uint32_t)np;
    s->part_shift = lg_cap - lg_np;
    s->part_rec = rec;
    return true;
}

/* ----------------------------------------------------------------
 * group-table growth (host side)
 *
 * The reference's service answers SUSPEND_NO_SPACE on kds_final by
 * expanding the buffer and relaunching the suspended kernel
 * (gpu_service.c:2418-2470, :3872-3879; resume at cuda_gpujoin.cu:
 * 1098-1103).  Here the table asks to grow before it is full: once half of
 * its slots are in use (or half of the key arena), every warp of a launch
 * on the session's stream stops after its current 32-row batch and records
 * the work it held (XbLeft ranges).  Groups that meanwhile find the table
 * without room take an entry of the dump region.  The host then rehashes
 * the live entries into a table at least twice as large, merges the dump
 * entries in, and a resume launch processes the recorded ranges and the
 * units nobody had claimed.  No row is applied twice or lost.
 * ---------------------------------------------------------------- */


/* the dump region, sized for a launch of 'grid' CTAs: every CTA's shared
 * table merged at exit, plus the rows in flight after the table asked to
 * grow (two 32-row batches per warp: the one a warp is in when the request
 * comes, and one more if its look at the flag came just before) when the
 * table's free half is smaller than twice those */
static int xb_dump_ensure(xpuB200Session *s, int grid, uint32_t sm_cap, cudaStream_t st, kern_errorbuf *err)
{
    const uint64_t cap = s->h_gt.cap_mask + 1;
    const uint64_t inflight = (uint64_t)grid * XB_WARPS * 64;
    uint64_t need = (uint64_t)grid * sm_cap;
    if (cap / 2 < 2 * inflight)
        need += inflight;
    if (need < 1024)
        need = 1024;
    if (s->h_gt.dump && s->h_gt.dump_cap >= need)
        return 0;
    if (s->h_gt.dump) {
        /* entries a served or mixed launch left in the old region join the
         * table before the region is replaced */
        int rc = xb_gt_settle(s, err);
        if (rc) return rc;
    }
    const uint64_t gsz = s->h_plan->gent_size;
    char *d = nullptr;
    if (cudaMallocAsync((void **)&d, need * gsz, st) != cudaSuccess) {
        cudaGetLastError();
        return XB_ERR(err, ERRCODE_DEVICE_FATAL, "out of device memory for the group dump (%llu entries)",
                      (unsigned long long)need);
    }
    cudaMemsetAsync(d, 0, need * gsz, st);
    if (s->h_gt.dump)
        cudaFreeAsync(s->h_gt.dump, st);
    s->h_gt.dump = d;
    s->h_gt.dump_cap = need;
    static_assert(offsetof(xb_gtable, dump_cap) == offsetof(xb_gtable, dump) + 8, "dump fields");
    XB_CUDA(cudaMemcpyAsync(&s->d_gt->dump, &s->h_gt.dump, 16, cudaMemcpyHostToDevice, st), err);
    return 0;
}

/* the device's copy of the group table header (synchronises the stream) */
int xb_gt_read(xpuB200Session *s, xb_gtable *g, kern_errorbuf *err)
{
    XB_CUDA(cudaMemcpyAsync(g, s->d_gt, sizeof(xb_gtable), cudaMemcpyDeviceToHost, s->stream), err);
    XB_CUDA(cudaStreamSynchronize(s->stream), err);
    return 0;
}

/* replace a tracked session allocation by another one */
static void xb_swap_alloc(xpuB200Session *s, void *old_p, void *new_p, uint64_t new_sz)
{
    for (size_t i = 0; i < s->d_allocs.size(); i++) {
        if (s->d_allocs[i] == old_p) {
            s->d_allocs[i] = new_p;
            s->d_alloc_sz[i] = new_sz;
            return;
        }
    }
    s->d_allocs.push_back(new_p);
    s->d_alloc_sz.push_back(new_sz);
}

/* grow the group table: at least twice the slots, and room for
 * min_entries groups at a load of 1/4 (1/2 above a million); the key
 * arena doubles when more than half of it is used.  Session lock held;
 * the stream is idle on entry and on return. */
int xb_gt_grow(xpuB200Session *s, uint64_t min_entries, kern_errorbuf *err)
{
    cudaStream_t st = s->stream;
    const xb_plan *plan = s->h_plan;
    xb_gtable g;
    int rc = xb_gt_read(s, &g, err);
    if (rc) return rc;
    const uint64_t gsz = plan->gent_size;
    const uint64_t cap = g.cap_mask + 1;
    const uint64_t ndump = g.dump_used < g.dump_cap ? g.dump_used : g.dump_cap;
    uint64_t want = g.nused > min_entries ? g.nused : min_entries;
    uint64_t new_cap = xb_next_pow2(want * (want > 1000000 ? 2 : 4) + 1024);
    if (new_cap < cap * 2)
        new_cap = cap * 2;
    const uint64_t max_cap = (s->dev->hbm_budget / 4) / gsz;
    if (new_cap > max_cap) {
        uint64_t c = xb_next_pow2(max_cap / 2 + 1);
        if (c <= cap)
            return XB_ERR(err, ERRCODE_SUSPEND_NO_SPACE,
                          "GpuPreAgg(GroupBy) - the group table of %llu slots cannot grow within the "
                          "device memory budget", (unsigned long long)cap);
        new_cap = c;
    }
    /* the key arena: a larger copy when more than half of it is used */
    char *arena_new = g.arena;
    uint64_t arena_new_sz = g.arena_sz;
    const uint64_t arena_used = g.arena_used < g.arena_sz ? g.arena_used : g.arena_sz;
    if (plan->nkeys_text && g.arena_used > g.arena_sz / 2) {
        arena_new_sz = g.arena_sz * 2 > g.arena_used * 4 ? g.arena_sz * 2 : g.arena_used * 4;
        if (cudaMallocAsync((void **)&arena_new, arena_new_sz, st) != cudaSuccess) {
            cudaGetLastError();
            return XB_ERR(err, ERRCODE_DEVICE_FATAL, "out of device memory growing the key arena");
        }
        cudaMemcpyAsync(arena_new, g.arena, arena_used, cudaMemcpyDeviceToDevice, st);
    }
    char *entries_new = nullptr;
    if (cudaMallocAsync((void **)&entries_new, new_cap * gsz, st) != cudaSuccess) {
        cudaGetLastError();
        if (arena_new != g.arena) cudaFreeAsync(arena_new, st);
        return XB_ERR(err, ERRCODE_DEVICE_FATAL, "out of device memory growing the group table to %llu slots",
                      (unsigned long long)new_cap);
    }
    cudaMemsetAsync(entries_new, 0, new_cap * gsz, st);
    xb_gtable ng = g;
    ng.cap_mask = new_cap - 1;
    ng.nused = 0;
    ng.entries = entries_new;
    ng.arena = arena_new;
    ng.arena_sz = arena_new_sz;
    ng.arena_used = arena_used;
    ng.overflow = 0;
    ng.grow = 0;
    ng.soft_cap = new_cap / 2;
    ng.dump_used = 0;
    XB_CUDA(cudaMemcpyAsync(s->d_gt, &ng, sizeof(xb_gtable), cudaMemcpyHostToDevice, st), err);
    XB_CUDA(cudaMemsetAsync(s->d_status, 0, sizeof(xb_status), st), err);
    XbGrowArgs ga;
    ga.plan = s->d_plan;
    ga.old_entries = g.entries;
    ga.old_cap = cap;
    ga.dump = g.dump;
    ga.ndump = ndump;
    ga.gt = s->d_gt;
    ga.st = s->d_status;
    ga.arena_old = g.arena;
    ga.arena_old_sz = g.arena_sz;
    ga.arena_new = arena_new;
    const int grid = s->dev->nsm * 8;
    xb_gt_rehash<<<grid, XB_BLOCK, 0, st>>>(ga);
    if (ndump) {
        xb_gt_merge_dump<<<grid, XB_BLOCK, 0, st>>>(ga);
        cudaMemsetAsync(g.dump, 0, ndump * gsz, st);
    }
    cudaError_t lrc = cudaGetLastError();
    if (lrc != cudaSuccess)
        return XB_ERR(err, ERRCODE_DEVICE_FATAL, "group table growth: %s", cudaGetErrorString(lrc));
    rc = xb_wait_status(s, err);
    cudaFreeAsync(g.entries, st);
    xb_swap_alloc(s, g.entries, entries_new, new_cap * gsz);
    if (arena_new != g.arena) {
        cudaFreeAsync(g.arena, st);
        xb_swap_alloc(s, g.arena, arena_new, arena_new_sz);
    }
    s->h_gt = ng;
    s->grow_count++;
    return rc;
}

/* pending dump entries (left by launches that do not stop for growth:
 * served and mixed launches) merged into a grown table; session lock held */
int xb_gt_settle(xpuB200Session *s, kern_errorbuf *err)
{
    if (!s->h_plan->has_groupby || !s->h_gt.dump)
        return 0;
    xb_gtable g;
    int rc = xb_gt_read(s, &g, err);
    if (rc) return rc;
    if (g.dump_used == 0)
        return 0;
    return xb_gt_grow(s, 0, err);
}

/* sum of two launches' statistics */
static void xb_status_add(xb_status *t, const xb_status *h)
{
    t->nitems_raw += h->nitems_raw;
    t->nitems_in += h->nitems_in;
    t->nitems_out += h->nitems_out;
    for (uint32_t d = 0; d <= XB_MAX_DEPTH; d++)
        t->nitems_depth[d] += h->nitems_depth[d];
}

int xb_launch_on(xpuB200Session *s, const xb_task *d_tasks, uint32_t ntasks,
                        uint64_t nunits, uint32_t format, cudaStream_t stream, xb_status *d_status,
                        kern_errorbuf *err)
{
    XbExecArgs a;
    memset(&a, 0, sizeof(a));
    a.plan = s->d_plan;
    a.plan_bytes = s->plan_bytes;
    a.tasks = d_tasks;
    a.ntasks = ntasks;
    a.nunits = nunits;
    a.format = format;
    a.sm_cap = s->sm_cap;
    a.warp_bytes = s->warp_bytes;
    a.dst = s->launch_dst;
    a.dst_len = s->launch_dst_len;
    a.dyn_only = 0;
    a.gt = s->d_gt;
    a.st = d_status;
    /* served launches (pooled slot streams) do not wait for a kernel build */
    void *fn = xb_session_jit(s, format, stream == s->stream);
    int grid = fn ? s->jit_grid[format] : s->grid;
    uint64_t warps_needed = (format == KDS_FORMAT_BLOCK) ? (nunits + XB_CLAIM - 1) / XB_CLAIM : nunits;
    if ((uint64_t)grid * XB_WARPS > warps_needed)
        grid = (int)((warps_needed + XB_WARPS - 1) / XB_WARPS);
    if (grid < 1) grid = 1;
    if (stream == s->stream && s->run_growth) {
        /* group-table growth (xb_run): warps that see the table ask to
         * grow record their leftover work here and stop */
        a.left_out = s->d_left[s->run_left_sel];
        a.left_cap = s->left_cap;
        if (s->run_resume) {
            a.resume = 1;
            a.left_in = s->d_left[s->run_left_sel ^ 1];
            a.left_in_n = s->run_left_in_n;
            a.static_base0 = s->run_static_base0;
            a.cursor0 = s->run_cursor0;
        } else {
            /* the static share each warp takes first (xb_src_start) */
            const uint64_t warps = (uint64_t)grid * XB_WARPS;
            s->run_static_base0 = format == KDS_FORMAT_BLOCK ? ((nunits * 3 / 5) / warps) * warps : 0;
        }
        if (xb_dump_ensure(s, grid, s->sm_cap, stream, err) != 0)
            return err ? err->errcode : ERRCODE_DEVICE_FATAL;
    }
    if (format < 256)
        s->ran_kind[format] = fn ? 'j' : 'v';
    const bool part = fn && s->jit_replay[format] && xb_part_prepare(s, nunits, format, stream);
    if (part) {
        a.part_buf = s->part_buf;
        a.part_cnt = s->part_cnt;
        a.part_cap = s->part_cap;
        a.part_shift = s->part_shift;
        cudaMemsetAsync(s->part_cnt, 0, sizeof(uint32_t) * XB_PART_CNT_STRIDE * (s->nparts + 1), stream);
        s->part_used = true;
    }
    if (fn) {
        if (part)
            cudaEventRecord(s->ev_part[0], stream);
        if (xb_jit_launch(fn, grid, XB_BLOCK, s->jit_smem_fmt[format], (void *)stream, &a) != 0)
            return XB_ERR(err, ERRCODE_DEVICE_FATAL, "specialised kernel launch failed");
        if (part) {
            cudaEventRecord(s->ev_part[1], stream);
            XbReplayArgs ra;
            memset(&ra, 0, sizeof(ra));
            ra.plan = s->d_plan;
            ra.gt = s->d_gt;
            ra.st = d_status;
            ra.part_buf = s->part_buf;
            ra.part_cnt = s->part_cnt;
            ra.part_cap = s->part_cap;
            ra.nparts = s->nparts;
            ra.cursor = s->part_cnt + (size_t)s->nparts * XB_PART_CNT_STRIDE;
            ra.part_shift = s->part_shift;
            if (xb_jit_launch(s->jit_replay[format], s->jit_replay_grid[format], XB_BLOCK, 0, (void *)stream,
                              &ra) != 0)
                return XB_ERR(err, ERRCODE_DEVICE_FATAL, "replay kernel launch failed");
            cudaEventRecord(s->ev_part[2], stream);
        }
    } else {
        xb_exec_kernel<<<grid, XB_BLOCK, s->smem_bytes, stream>>>(a);
    }
    cudaError_t rc = cudaGetLastError();
    if (rc != cudaSuccess)
        return XB_ERR(err, ERRCODE_DEVICE_FATAL, "kernel launch: %s", cudaGetErrorString(rc));
    return 0;
}

/* a single chunk as the session's one-task work queue */
static int xb_exec_task_of(xpuB200Session *s, const kern_data_store *d_kds,
                           const kern_data_store *h_kds_head, xb_task *t, kern_errorbuf *err)
{
    if (h_kds_head->format != KDS_FORMAT_BLOCK && h_kds_head->format != KDS_FORMAT_ARROW &&
        h_kds_head->format != KDS_FORMAT_ROW)
        return XB_ERR(err, ERRCODE_DEVICE_ERROR, "unsupported KDS format '%c'", h_kds_head->format);
    if (!s->d_tasks) {
        XB_CUDA(cudaMallocAsync((void **)&s->d_tasks, sizeof(xb_task) * 16, s->stream), err);
        s->d_tasks_cap = 16;
    }
    t->kds = d_kds;
    t->unit_base = 0;
    t->nunits = xb_chunk_units(h_kds_head);
    t->format = (uint32_t)h_kds_head->format;
    XB_CUDA(cudaMemcpyAsync(s->d_tasks, t, sizeof(*t), cudaMemcpyHostToDevice, s->stream), err);
    return 0;
}

/* single-chunk launch through the session's task buffer */
static int xb_launch_exec(xpuB200Session *s, const kern_data_store *d_kds,
                          const kern_data_store *h_kds_head, kern_errorbuf *err)
{
    xb_task t;
    int rc = xb_exec_task_of(s, d_kds, h_kds_head, &t, err);
    if (rc) return rc;
    return xb_launch_tasks(s, s->d_tasks, 1, t.nunits, t.format, err);
}

/* [off, off + len) lies inside [0, total), without a wrapping sum */
static inline bool xb_within(uint64_t off, uint64_t len, uint64_t total)
{
    return off <= total && len <= total - off;
}

int xb_check_kds(const kern_data_store *kds, kern_errorbuf *err)
{
    if (kds->format == KDS_FORMAT_BLOCK) {
        if ((uint64_t)kds->block_offset + (uint64_t)PGSTROM_BLCKSZ * kds->nitems > kds->length ||
            kds->block_offset < KDS_HEAD_LENGTH(kds))
            return XB_ERR(err, ERRCODE_DEVICE_ERROR, "KDS_FORMAT_BLOCK chunk is broken");
    } else if (kds->format == KDS_FORMAT_ARROW) {
        if (KDS_HEAD_LENGTH(kds) > kds->length)
            return XB_ERR(err, ERRCODE_DEVICE_ERROR, "chunk header is broken");
    } else if (kds->format == KDS_FORMAT_ROW) {
        /* the kernels read the row index (after the hash slots) up to nitems */
        if (!xb_within(KDS_HEAD_LENGTH(kds), 8ULL * ((uint64_t)kds->hash_nslots + kds->nitems), kds->length))
            return XB_ERR(err, ERRCODE_DEVICE_ERROR, "KDS_FORMAT_ROW chunk is broken");
    } else {
        return XB_ERR(err, ERRCODE_DEVICE_ERROR, "unsupported KDS format '%c'", kds->format);
    }
    if (kds->format == KDS_FORMAT_ARROW) {
        /* the kernels read colmeta[] up to ncols */
        if (kds->ncols > kds->nr_colmeta)
            return XB_ERR(err, ERRCODE_DEVICE_ERROR, "Arrow chunk has %u columns but %u column descriptors",
                          (unsigned)kds->ncols, (unsigned)kds->nr_colmeta);
        for (uint32_t j = 0; j < kds->ncols; j++) {
            const kern_colmeta *cm = &kds->colmeta[j];
            if (cm->virtual_offset != 0)
                continue;
            if (!xb_within(cm->nullmap_offset, cm->nullmap_length, kds->length) ||
                !xb_within(cm->values_offset, cm->values_length, kds->length) ||
                !xb_within(cm->extra_offset, cm->extra_length, kds->length))
                return XB_ERR(err, ERRCODE_DEVICE_ERROR, "Arrow column %u is out of the chunk", j);
            /* value arrays are read with their natural width */
            if ((cm->values_offset & 7) != 0)
                return XB_ERR(err, ERRCODE_DEVICE_ERROR, "Arrow column %u values are not 8-byte aligned", j);
        }
    }
    return 0;
}

/* the chunk checks ExecTask applies before a launch, for the host-side
 * tests (no device needed) */
extern "C" int xb_kds_check(const kern_data_store *kds, kern_errorbuf *err)
{
    xb_clear_error(err);
    return xb_check_kds(kds, err);
}

/* wait for the launch and read its status (errors reported by the kernel) */
int xb_wait_status(xpuB200Session *s, kern_errorbuf *err)
{
    cudaStream_t st = s->stream;
    cudaMemcpyAsync(s->h_status, s->d_status, sizeof(xb_status), cudaMemcpyDeviceToHost, st);
    cudaError_t rc = cudaStreamSynchronize(st);
    if (rc != cudaSuccess)
        return XB_ERR(err, ERRCODE_DEVICE_FATAL, "ExecTask: %s", cudaGetErrorString(rc));
    const xb_status *hs = s->h_status;
    if (hs->errcode)
        return xb_set_error(err, hs->errcode, "xb_exec_kernel", hs->lineno, "%s", xb_msg_text(hs->msg_id));
    return 0;
}

/* a finished launch's statistics (status hs) into *results */
void xb_fill_results(const xb_status *hs, uint32_t nrels, kern_exec_results *results)
{
    if (!results)
        return;
    uint32_t cap = results->num_rels;
    results->nitems_raw = (uint32_t)hs->nitems_raw;
    results->nitems_in = (uint32_t)hs->nitems_in;
    results->nitems_out = (uint32_t)hs->nitems_out;
    results->num_rels = nrels;
    for (uint32_t d = 1; d <= nrels && d <= cap; d++) {
        results->stats[d - 1].nitems_roj = 0;
        results->stats[d - 1].nitems_gist = 0;
        results->stats[d - 1].nitems_out = (uint32_t)hs->nitems_depth[d];
    }
}

/* add a finished launch's statistics (status hs) to the session and to
 * *results */
void xb_account_status(xpuB200Session *s, const xb_status *hs, kern_exec_results *results)
{
    s->total_raw += hs->nitems_raw;
    s->total_in += hs->nitems_in;
    s->total_out += hs->nitems_out;
    for (uint32_t d = 1; d <= s->h_plan->nrels; d++)
        s->total_depth[d] += hs->nitems_depth[d];
    xb_fill_results(hs, s->h_plan->nrels, results);
}

static void xb_account(xpuB200Session *s, kern_exec_results *results)
{
    xb_account_status(s, s->h_status, results);
}


/* the replay of partitioned aggregation again, for the records a full
 * table left (after the table grew) */
static int xb_replay_retry(xpuB200Session *s, uint32_t format, kern_errorbuf *err)
{
    XB_CUDA(cudaMemsetAsync(s->d_status, 0, sizeof(xb_status), s->stream), err);
    uint32_t *cursor = s->part_cnt + (size_t)s->nparts * XB_PART_CNT_STRIDE;
    XB_CUDA(cudaMemsetAsync(cursor, 0, sizeof(uint32_t), s->stream), err);
    XbReplayArgs ra;
    memset(&ra, 0, sizeof(ra));
    ra.plan = s->d_plan;
    ra.gt = s->d_gt;
    ra.st = s->d_status;
    ra.part_buf = s->part_buf;
    ra.part_cnt = s->part_cnt;
    ra.cursor = cursor;
    ra.part_cap = s->part_cap;
    ra.nparts = s->nparts;
    ra.part_shift = s->part_shift;
    ra.retry = 1;
    if (!s->jit_replay[format] ||
        xb_jit_launch(s->jit_replay[format], s->jit_replay_grid[format], XB_BLOCK, 0, (void *)s->stream, &ra) != 0)
        return XB_ERR(err, ERRCODE_DEVICE_FATAL, "replay kernel launch failed");
    return xb_wait_status(s, err);
}

/*
 * Run a work queue on the session's stream to the end, growing the group
 * table as often as it asks to: after each launch the host grows the
 * table when asked (or when dump entries wait), replays the records a
 * full table left, and issues a resume launch for the work the stopped
 * warps recorded plus the units nobody claimed.  The statistics of all
 * launches are added to the session and written to *results.  timed:
 * ev0 / ev1 bracket every launch of the run.
 */
/* can the session's groups outnumber what its table holds below the
 * growth threshold?  Not without GROUP BY keys (one group), nor when the
 * keys come numbered from an inner relation (at most that many groups) */
static bool xb_groups_may_grow(const xpuB200Session *s)
{
    const xb_plan *plan = s->h_plan;
    if (plan->has_groupby != 1 || !s->h_gt.entries)
        return false;
    const uint32_t gd = plan->gid_depth;
    if (gd >= 1 && gd <= plan->nrels && plan->inner[gd].gid_on &&
        (uint64_t)plan->inner[gd].ngids < s->h_gt.soft_cap)
        return false;
    return true;
}

int xb_run(xpuB200Session *s, const xb_task *d_tasks, uint32_t ntasks, uint64_t nunits,
                  uint32_t format, kern_exec_results *results, kern_errorbuf *err, bool timed)
{
    cudaStream_t st = s->stream;
    /* warps look for a growth request only where one can come */
    const bool growth = xb_groups_may_grow(s);
    if (growth && !s->d_left[0]) {
        /* two leftover records per warp of the largest grid (8 CTAs per SM) */
        const uint32_t cap = 2u * (uint32_t)s->dev->nsm * 8u * XB_WARPS;
        for (int i = 0; i < 2; i++)
            if (cudaMallocAsync((void **)&s->d_left[i], sizeof(XbLeft) * cap, st) != cudaSuccess) {
                cudaGetLastError();
                return XB_ERR(err, ERRCODE_DEVICE_FATAL, "out of device memory for leftover ranges");
            }
        s->left_cap = cap;
    }
    xb_status total;
    memset(&total, 0, sizeof(total));
    s->run_growth = growth;
    s->run_resume = false;
    s->run_left_sel = 0;
    s->run_cursor0 = 0;
    int rc = 0;
    for (uint32_t round = 0;; round++) {
        if (round > 64) {
            rc = XB_ERR(err, ERRCODE_DEVICE_ERROR, "the group table kept asking to grow (%u launches)", round);
            break;
        }
        if ((rc = xb_set_cuda(cudaMemsetAsync(s->d_status, 0, sizeof(xb_status), st), err)) != 0)
            break;
        if (timed && round == 0)
            cudaEventRecord(s->ev0, st);
        rc = xb_launch_tasks(s, d_tasks, ntasks, nunits, format, err);
        if (rc) break;
        if (timed)
            cudaEventRecord(s->ev1, st);
        rc = xb_wait_status(s, err);
        if (rc) break;
        const xb_status hs = *s->h_status;
        xb_status_add(&total, &hs);
        if (!growth)
            break;
        xb_gtable g;
        if ((rc = xb_gt_read(s, &g, err)) != 0)
            break;
        if (g.grow || g.dump_used) {
            if ((rc = xb_gt_grow(s, 0, err)) != 0)
                break;
        }
        /* the replay's records that found the table full, after it grew */
        bool left = hs.replay_left != 0;
        for (uint32_t r = 0; left && r < 64; r++) {
            if ((rc = xb_replay_retry(s, format, err)) != 0)
                break;
            left = s->h_status->replay_left != 0;
            if ((rc = xb_gt_read(s, &g, err)) != 0)
                break;
            if (g.grow || g.dump_used)
                if ((rc = xb_gt_grow(s, 0, err)) != 0)
                    break;
        }
        if (rc) break;
        if (left) {
            rc = XB_ERR(err, ERRCODE_DEVICE_ERROR, "deferred group updates kept finding the table full");
            break;
        }
        if (!hs.stopped)
            break;
        /* resume: the ranges the stopped warps recorded, then the units
         * the stopped launch's cursor had not handed out */
        s->run_resume = true;
        s->run_left_in_n = hs.left_n;
        s->run_cursor0 += hs.unit_cursor;
        s->run_left_sel ^= 1;
    }
    s->run_growth = false;
    s->run_resume = false;
    if (rc == 0)
        xb_account_status(s, &total, results);
    return rc;
}

static int xb_place_src(xpuB200Session *s, const kern_data_store *kds_src, int kds_src_on_device,
                        kern_data_store *p_head, std::vector<char> *p_hbuf,
                        const kern_data_store **p_dkds, kern_errorbuf *err);

extern "C" int
xpuB200ExecTask(xpuB200Session *s, const kern_data_store *kds_src, int kds_src_on_device,
                kern_exec_results *results, kern_errorbuf *err)
{
    xb_clear_error(err);
    if (!s || !kds_src)
        return XB_ERR(err, ERRCODE_DEVICE_ERROR, "invalid ExecTask arguments");
    std::lock_guard<std::mutex> g(s->lock);
    if (s->h_plan->has_proj)
        return XB_ERR(err, ERRCODE_DEVICE_ERROR,
                      "the session projects rows into kds_dst: use xpuB200ExecTaskDst");
    XB_CUDA(cudaSetDevice(s->dev->dindex), err);
    kern_data_store head;
    const kern_data_store *d_kds;
    std::vector<char> hbuf;
    int rc = xb_place_src(s, kds_src, kds_src_on_device, &head, &hbuf, &d_kds, err);
    if (rc) return rc;
    xb_task t;
    rc = xb_exec_task_of(s, d_kds, kds_src_on_device ? (const kern_data_store *)hbuf.data() : &head, &t, err);
    if (rc) return rc;
    return xb_run(s, s->d_tasks, 1, t.nunits, t.format, results, err);
}

/* validate a chunk and make it device-resident: host chunks are copied to
 * the session's staging buffer so that heap pages start 16-byte aligned */
static int xb_place_src(xpuB200Session *s, const kern_data_store *kds_src, int kds_src_on_device,
                        kern_data_store *p_head, std::vector<char> *p_hbuf,
                        const kern_data_store **p_dkds, kern_errorbuf *err)
{
    cudaStream_t st = s->stream;
    kern_data_store &head = *p_head;
    std::vector<char> &hbuf = *p_hbuf;
    const kern_data_store *d_kds;
    if (kds_src_on_device) {
        if (((uintptr_t)kds_src & 7) != 0)
            return XB_ERR(err, ERRCODE_DEVICE_ERROR, "device chunk is not 8-byte aligned");
        XB_CUDA(cudaMemcpy(&head, kds_src, offsetof(kern_data_store, colmeta), cudaMemcpyDeviceToHost), err);
        uint64_t hl = KDS_HEAD_LENGTH(&head);
        hbuf.resize(hl);
        XB_CUDA(cudaMemcpy(hbuf.data(), kds_src, hl, cudaMemcpyDeviceToHost), err);
        int rc = xb_check_kds((const kern_data_store *)hbuf.data(), err);
        if (rc) return rc;
        d_kds = kds_src;
    } else {
        int rc = xb_check_kds(kds_src, err);
        if (rc) return rc;
        head = *kds_src;
        /* place the chunk so that heap pages start on a 16-byte boundary */
        uint64_t shift = (kds_src->format == KDS_FORMAT_BLOCK) ? ((16 - (kds_src->block_offset & 15)) & 15) : 0;
        uint64_t need = kds_src->length + shift + 64;
        if (need > s->d_src_cap) {
            if (s->d_src) cudaFreeAsync(s->d_src, st);
            s->d_src = nullptr;
            s->d_src_cap = 0;
            XB_CUDA(cudaMallocAsync((void **)&s->d_src, need + (need >> 3), st), err);
            s->d_src_cap = need + (need >> 3);
        }
        XB_CUDA(cudaMemcpyAsync(s->d_src + shift, kds_src, kds_src->length, cudaMemcpyHostToDevice, st), err);
        d_kds = (const kern_data_store *)(s->d_src + shift);
    }
    xb_note_layout(s, kds_src_on_device ? (const kern_data_store *)hbuf.data() : kds_src);
    *p_dkds = d_kds;
    return 0;
}

extern "C" int
xpuB200ExecTaskDst(xpuB200Session *s, const kern_data_store *kds_src, int kds_src_on_device,
                   void *kds_dst, uint64_t dst_sz, int kds_dst_on_device, uint64_t *p_required,
                   kern_exec_results *results, kern_errorbuf *err)
{
    xb_clear_error(err);
    if (!s || !kds_src || !kds_dst)
        return XB_ERR(err, ERRCODE_DEVICE_ERROR, "invalid ExecTaskDst arguments");
    std::lock_guard<std::mutex> g(s->lock);
    const xb_plan *plan = s->h_plan;
    if (!plan->has_proj)
        return XB_ERR(err, ERRCODE_DEVICE_ERROR, "the session has no device projection");
    const kern_session_info *session = (const kern_session_info *)s->h_session.data();
    const kern_data_store *tmpl = (const kern_data_store *)(s->h_session.data() + session->projection_kds_dst);
    const uint64_t head_len = plan->proj_head_len;
    const uint64_t len = dst_sz & ~7ULL;
    if (len < head_len + 8)
        return XB_ERR(err, ERRCODE_DEVICE_ERROR, "kds_dst of %llu bytes cannot hold a row",
                      (unsigned long long)dst_sz);
    XB_CUDA(cudaSetDevice(s->dev->dindex), err);
    cudaStream_t st = s->stream;
    kern_data_store head;
    const kern_data_store *d_kds;
    std::vector<char> hbuf;
    int rc = xb_place_src(s, kds_src, kds_src_on_device, &head, &hbuf, &d_kds, err);
    if (rc) return rc;
    char *d_dst;
    if (kds_dst_on_device) {
        if (((uintptr_t)kds_dst & 7) != 0)
            return XB_ERR(err, ERRCODE_DEVICE_ERROR, "device kds_dst is not 8-byte aligned");
        d_dst = (char *)kds_dst;
    } else {
        if (len > s->d_dst_cap) {
            if (s->d_dst) cudaFreeAsync(s->d_dst, st);
            s->d_dst = nullptr;
            s->d_dst_cap = 0;
            XB_CUDA(cudaMallocAsync((void **)&s->d_dst, len, st), err);
            s->d_dst_cap = len;
        }
        d_dst = s->d_dst;
    }
    XB_CUDA(cudaMemsetAsync(s->d_status, 0, sizeof(xb_status), st), err);
    const uint64_t hl0 = KDS_HEAD_LENGTH(tmpl);     /* hash slots follow, when hashed */
    if (plan->proj_hashed)
        XB_CUDA(cudaMemsetAsync(d_dst + hl0, 0, head_len - hl0, st), err);
    s->launch_dst = d_dst;
    s->launch_dst_len = len;
    rc = xb_launch_exec(s, d_kds, kds_src_on_device ? (const kern_data_store *)hbuf.data() : &head, err);
    s->launch_dst = nullptr;
    s->launch_dst_len = 0;
    if (rc) return rc;
    rc = xb_wait_status(s, err);
    if (rc) return rc;
    const xb_status *hs = s->h_status;
    const uint64_t nitems = hs->proj_nitems, usage = hs->proj_usage;
    const uint64_t required = head_len + hs->proj_need;
    if (p_required)
        *p_required = required;
    if (hs->proj_overflow)
        return XB_ERR(err, ERRCODE_SUSPEND_NO_SPACE, "kds_dst needs %llu bytes (buffer %llu)",
                      (unsigned long long)required, (unsigned long long)len);
    /* the header: the session's kds_dst definition with this chunk's rows
     * (a hashed kds_dst keeps the hash slots the kernel chained) */
    std::vector<char> hd((const char *)tmpl, (const char *)tmpl + hl0);
    kern_data_store *kh = (kern_data_store *)hd.data();
    kh->length = len;
    kh->nitems = (uint32_t)nitems;
    kh->usage = usage;
    kh->format = plan->proj_hashed ? KDS_FORMAT_HASH : KDS_FORMAT_ROW;
    kh->hash_nslots = plan->proj_hashed ? plan->proj_nslots : 0;
    if (kds_dst_on_device) {
        XB_CUDA(cudaMemcpyAsync(d_dst, hd.data(), hl0, cudaMemcpyHostToDevice, st), err);
    } else {
        char *h = (char *)kds_dst;
        memcpy(h, hd.data(), hl0);
        if (head_len > hl0)
            XB_CUDA(cudaMemcpyAsync(h + hl0, d_dst + hl0, head_len - hl0, cudaMemcpyDeviceToHost, st), err);
        if (nitems)
            XB_CUDA(cudaMemcpyAsync(h + head_len, d_dst + head_len, 8 * nitems, cudaMemcpyDeviceToHost, st), err);
        if (usage)
            XB_CUDA(cudaMemcpyAsync(h + len - usage, d_dst + len - usage, usage, cudaMemcpyDeviceToHost, st), err);
    }
    XB_CUDA(cudaStreamSynchronize(st), err);
    xb_account(s, results);
    return 0;
}

extern "C" int
xpuB200TimeExecTask(xpuB200Session *s, const kern_data_store *kds_src_dev, int niters,
                    double *p_msec, kern_errorbuf *err)
{
    xb_clear_error(err);
    std::lock_guard<std::mutex> g(s->lock);
    XB_CUDA(cudaSetDevice(s->dev->dindex), err);
    kern_data_store head;
    if (((uintptr_t)kds_src_dev & 7) != 0)
        return XB_ERR(err, ERRCODE_DEVICE_ERROR, "device chunk is not 8-byte aligned");
    XB_CUDA(cudaMemcpy(&head, kds_src_dev, offsetof(kern_data_store, colmeta), cudaMemcpyDeviceToHost), err);
    std::vector<char> hbuf(KDS_HEAD_LENGTH(&head));
    XB_CUDA(cudaMemcpy(hbuf.data(), kds_src_dev, hbuf.size(), cudaMemcpyDeviceToHost), err);
    int rc = xb_check_kds((const kern_data_store *)hbuf.data(), err);
    if (rc) return rc;
    float total = 0.0f;
    xb_task t;
    rc = xb_exec_task_of(s, kds_src_dev, (const kern_data_store *)hbuf.data(), &t, err);
    if (rc) return rc;
    for (int i = 0; i < niters; i++) {
        rc = xb_run(s, s->d_tasks, 1, t.nunits, t.format, nullptr, err, true);
        if (rc) return rc;
        float ms = 0.0f;
        cudaEventElapsedTime(&ms, s->ev0, s->ev1);
        total += ms;
    }
    *p_msec = niters > 0 ? total / niters : 0.0;
    return 0;
}

/* ----------------------------------------------------------------
 * Final without device allocations
 *
 * xpuB200Final allocates its work arrays (per-slot tuple sizes, their
 * prefix sums, scan storage) and a device copy of kds_final from the
 * device's memory pool on every call.  Some callers cannot do that: a
 * service that has reserved the GPU's memory up front and hands out pieces
 * of its own pool (as PG-Strom's GPU service does with its device memory),
 * or one that must not allocate device memory while other sessions'
 * kernels run (a plain cudaFree waits for the whole device).  This variant writes
 * kds_final into memory the caller already owns and keeps its work arrays
 * in the fixed array below, which lives in the library's module on every
 * GPU that loads it until the process exits.
 * ---------------------------------------------------------------- */
#define XB_FINAL_SCRATCH_BYTES  (8ULL << 20)        /* 8 MiB per GPU */
#define XB_FINAL_SCRATCH_DEVS   64

static __device__ __align__(256) char xb_final_scratch[XB_FINAL_SCRATCH_BYTES];

/* device address of xb_final_scratch on each GPU, looked up once per device
 * (the host-side symbol is not a device address) */
static void *xb_final_scratch_dptr[XB_FINAL_SCRATCH_DEVS];
/* every session on one GPU shares that GPU's array: one call at a time
 * per GPU (calls for different GPUs use different arrays and run freely) */
static std::mutex xb_final_scratch_lock[XB_FINAL_SCRATCH_DEVS];


extern "C" int
xpuB200FinalNoAlloc(xpuB200Session *s, void *kds_final_dev, uint64_t buf_sz, uint64_t *p_required,
                    kern_exec_results *results, kern_errorbuf *err)
{
    xb_clear_error(err);
    if (!s)
        return XB_ERR(err, ERRCODE_DEVICE_ERROR, "invalid FinalNoAlloc arguments");
    xb_sched_drain_session(s);
    std::lock_guard<std::mutex> g(s->lock);
    const int dindex = s->dev->dindex;
    if (dindex < 0 || dindex >= XB_FINAL_SCRATCH_DEVS)
        return XB_ERR(err, ERRCODE_DEVICE_ERROR, "FinalNoAlloc supports GPUs 0..%d", XB_FINAL_SCRATCH_DEVS - 1);
    std::lock_guard<std::mutex> gs(xb_final_scratch_lock[dindex]);
    XB_CUDA(cudaSetDevice(dindex), err);
    if (!xb_final_scratch_dptr[dindex]) {
        void *ptr = nullptr;
        cudaError_t rc = cudaGetSymbolAddress(&ptr, xb_final_scratch);
        if (rc != cudaSuccess || !ptr) {
            cudaGetLastError();
            return XB_ERR(err, ERRCODE_DEVICE_FATAL, "FinalNoAlloc: scratch address on GPU %d: %s",
                          dindex, cudaGetErrorString(rc));
        }
        xb_final_scratch_dptr[dindex] = ptr;
    }
    char *scratch = (char *)xb_final_scratch_dptr[dindex];
    cudaStream_t st = s->stream;
    const xb_plan *plan = s->h_plan;
    if (results) {
        uint32_t cap = results->num_rels;
        results->nitems_raw = (uint32_t)s->total_raw;
        results->nitems_in = (uint32_t)s->total_in;
        results->nitems_out = (uint32_t)s->total_out;
        results->num_rels = plan->nrels;
        for (uint32_t d = 1; d <= plan->nrels && d <= cap; d++)
            results->stats[d - 1].nitems_out = (uint32_t)s->total_depth[d];
        results->final_plan_task = true;
    }
    if (plan->nsort)
        return XB_ERR(err, ERRCODE_DEVICE_ERROR, "a session with GPU-Sort keys needs xpuB200Final");
    if (!plan->has_groupby) {
        if (p_required) *p_required = 0;
        return 0;
    }
    if (s->h_gt.dump) {
        /* groups in the dump region join the table only when it grows,
         * which allocates: that is xpuB200Final's work */
        xb_gtable gh;
        int grc = xb_gt_read(s, &gh, err);
        if (grc) return grc;
        if (gh.dump_used)
            return XB_ERR(err, ERRCODE_DEVICE_ERROR,
                          "FinalNoAlloc: %llu groups wait for the group table to grow; use xpuB200Final",
                          (unsigned long long)gh.dump_used);
    }
    const kern_session_info *session = (const kern_session_info *)s->h_session.data();
    const kern_data_store *fh = (const kern_data_store *)(s->h_session.data() + session->groupby_kds_final);
    const uint64_t head_len = KDS_HEAD_LENGTH(fh);
    const uint64_t cap = s->h_gt.cap_mask + 1;
    const bool row_fmt = fh->format == KDS_FORMAT_ROW;

    /* scratch layout: sizes | size prefix sums | flags | flag prefix sums | scan storage */
    const uint64_t off_sscan = xb_align256(cap * 8);
    const uint64_t off_flags = off_sscan + xb_align256(cap * 8);
    const uint64_t off_fscan = off_flags + xb_align256(cap * 4);
    const uint64_t off_temp = off_fscan + xb_align256(cap * 4);
    uint64_t *d_sizes = (uint64_t *)scratch;
    uint64_t *d_size_scan = (uint64_t *)(scratch + off_sscan);
    uint32_t *d_flags = (uint32_t *)(scratch + off_flags);
    uint32_t *d_flag_scan = (uint32_t *)(scratch + off_fscan);
    void *d_temp = scratch + off_temp;
    const uint64_t tsz_max = xb_scan_temp_bytes<uint64_t>(cap);
    if (off_temp + tsz_max > XB_FINAL_SCRATCH_BYTES)
        return XB_ERR(err, ERRCODE_DEVICE_ERROR,
                      "FinalNoAlloc: the session's group table has %llu slots and needs %llu bytes of work "
                      "space, above this entry point's fixed %llu bytes; use xpuB200Final",
                      (unsigned long long)cap, (unsigned long long)(off_temp + tsz_max),
                      (unsigned long long)XB_FINAL_SCRATCH_BYTES);
    if (kds_final_dev) {
        cudaPointerAttributes pa;
        if (cudaPointerGetAttributes(&pa, kds_final_dev) != cudaSuccess) {
            cudaGetLastError();
            return XB_ERR(err, ERRCODE_DEVICE_ERROR, "FinalNoAlloc: kds_final_dev is not CUDA memory");
        }
        const bool ok = (pa.type == cudaMemoryTypeDevice && pa.device == dindex) ||
                        pa.type == cudaMemoryTypeManaged ||
                        (pa.type == cudaMemoryTypeHost && pa.devicePointer == kds_final_dev);
        if (!ok)
            return XB_ERR(err, ERRCODE_DEVICE_ERROR,
                          "FinalNoAlloc: kds_final_dev must be memory of GPU %d (or mapped host memory)", dindex);
    }
    /* the previous call's values are still in the array: xb_final_sizes
     * writes every size and flag below cap, and the scans overwrite their
     * outputs, so no part of it needs clearing first */
    XbFinalArgs fa;
    memset(&fa, 0, sizeof(fa));
    fa.plan = s->d_plan;
    fa.gt = s->d_gt;
    fa.cap = cap;
    fa.sizes = d_sizes;
    fa.flags = d_flags;
    fa.size_scan = d_size_scan;
    fa.flag_scan = d_flag_scan;
    fa.row_format = row_fmt ? 1 : 0;
    const int grid = s->dev->nsm * 8;
    xb_final_sizes<<<grid, XB_BLOCK, 0, st>>>(fa);
    xb_scan<uint64_t, XbOpSum, true>(d_sizes, d_size_scan, cap, d_temp, st);
    xb_scan<uint32_t, XbOpSum, true>(d_flags, d_flag_scan, cap, d_temp, st);
    uint64_t last_size = 0, last_scan = 0;
    uint32_t last_flag = 0, last_fscan = 0;
    cudaMemcpyAsync(&last_size, d_sizes + cap - 1, 8, cudaMemcpyDeviceToHost, st);
    cudaMemcpyAsync(&last_scan, d_size_scan + cap - 1, 8, cudaMemcpyDeviceToHost, st);
    cudaMemcpyAsync(&last_flag, d_flags + cap - 1, 4, cudaMemcpyDeviceToHost, st);
    cudaMemcpyAsync(&last_fscan, d_flag_scan + cap - 1, 4, cudaMemcpyDeviceToHost, st);
    if (cudaStreamSynchronize(st) != cudaSuccess)
        return XB_ERR(err, ERRCODE_DEVICE_FATAL, "FinalNoAlloc: %s", cudaGetErrorString(cudaGetLastError()));
    const uint64_t items = last_scan + last_size;
    const uint64_t ngroups = (uint64_t)last_fscan + last_flag;
    const uint64_t nslots = row_fmt ? 0 : KDS_GET_HASHSLOT_WIDTH(ngroups);
    const uint64_t items_base = head_len + 8 * nslots + 8 * ngroups;
    const uint64_t length = items_base + items;
    if (p_required) *p_required = length;
    if (results) {
        results->final_nitems = (uint32_t)ngroups;
        results->final_usage = items;
        results->final_total = length;
    }
    if (!kds_final_dev || buf_sz < length) {
        if (!kds_final_dev && buf_sz == 0)
            return 0;           /* size query only */
        return XB_ERR(err, ERRCODE_SUSPEND_NO_SPACE, "kds_final needs %llu bytes (buffer %llu)",
                      (unsigned long long)length, (unsigned long long)buf_sz);
    }
    char *d_out = (char *)kds_final_dev;
    std::vector<char> head((const char *)fh, (const char *)fh + head_len);
    kern_data_store *kh = (kern_data_store *)head.data();
    kh->length = length;
    kh->usage = items;
    kh->nitems = (uint32_t)ngroups;
    kh->format = row_fmt ? KDS_FORMAT_ROW : KDS_FORMAT_HASH;
    kh->hash_nslots = (uint32_t)nslots;
    cudaMemcpyAsync(d_out, head.data(), head_len, cudaMemcpyHostToDevice, st);
    /* slots, row index and items: the padding between and after the
     * tuples' attributes is zero, so equal results are equal bytes */
    cudaMemsetAsync(d_out + head_len, 0, length - head_len, st);
    fa.kds_final = d_out;
    fa.items_base = items_base;
    fa.length = length;
    fa.nslots = (uint32_t)nslots;
    xb_final_write<<<grid, XB_BLOCK, 0, st>>>(fa);
    if (cudaStreamSynchronize(st) != cudaSuccess)
        return XB_ERR(err, ERRCODE_DEVICE_FATAL, "FinalNoAlloc: %s", cudaGetErrorString(cudaGetLastError()));
    return 0;
}

extern "C" int
xpuB200CopyToDevice(xpuB200Device *dev, void *dptr, const void *src, uint64_t sz)
{
    cudaSetDevice(dev->dindex);
    return cudaMemcpy(dptr, src, sz, cudaMemcpyHostToDevice) == cudaSuccess ? 0 : ERRCODE_DEVICE_FATAL;
}

extern "C" int
xpuB200CopyToHost(xpuB200Device *dev, void *dst, const void *dptr, uint64_t sz)
{
    cudaSetDevice(dev->dindex);
    return cudaMemcpy(dst, dptr, sz, cudaMemcpyDeviceToHost) == cudaSuccess ? 0 : ERRCODE_DEVICE_FATAL;
}

extern "C" int
xpuB200SessionInfo(xpuB200Session *s, char *buf, uint64_t buf_sz)
{
    if (!s || !buf) return ERRCODE_DEVICE_ERROR;
    const xb_plan *p = s->h_plan;
    /* which kernel runs each format: "jit" (session-specialised) or "vm" */
    std::string kinds, msg;
    for (int f : {KDS_FORMAT_ROW, KDS_FORMAT_BLOCK, KDS_FORMAT_ARROW}) {
        if (!s->ran_kind[f])
            continue;
        if (!kinds.empty()) kinds += ", ";
        kinds += std::string("\"") + (char)f + "\": \"" + (s->ran_kind[f] == 'j' ? "jit" : "vm") + "\"";
    }
    for (char c : s->jit_msg)
        msg += (c == '"' || c == '\\' || (unsigned char)c < 32) ? ' ' : c;
    float scan_ms = 0.0f, replay_ms = 0.0f;
    if (s->part_used && cudaEventQuery(s->ev_part[2]) == cudaSuccess) {
        cudaEventElapsedTime(&scan_ms, s->ev_part[0], s->ev_part[1]);
        cudaEventElapsedTime(&replay_ms, s->ev_part[1], s->ev_part[2]);
    }
    cudaGetLastError();
    snprintf(buf, buf_sz,
             "{\"nregs\": %u, \"nslots\": %u, \"nrels\": %u, \"ninsns\": %u, \"has_groupby\": %u, "
             "\"nkeys\": %u, \"naggs\": %u, \"gent_size\": %u, \"gtable_cap\": %llu, "
             "\"sm_cap\": %u, \"smem_bytes\": %zu, \"grid\": %d, \"unique_hash\": [%u, %u, %u], "
             "\"jit_enabled\": %s, \"kernels\": {%s}, \"jit_compile_ms\": %.1f, \"jit_msg\": \"%s\", "
             "\"jit_ctas_per_sm\": %d, \"sm_cap_default\": %u, \"inner_cache\": %s, "
             "\"partitions\": %u, \"partition_used\": %s, \"gtable_grew\": %u, \"gtable_dump_cap\": %llu, "
             "\"last_part_scan_ms\": %.3f, \"last_part_replay_ms\": %.3f}",
             p->nregs, p->nslots, p->nrels, p->ninsns, p->has_groupby, p->nkeys, p->naggs,
             p->gent_size, (unsigned long long)(s->h_gt.cap_mask + 1), s->sm_cap, s->smem_bytes,
             s->grid, p->inner[1].unique_hash, p->inner[2].unique_hash, p->inner[3].unique_hash,
             s->jit_enabled ? "true" : "false", kinds.c_str(), s->jit_compile_ms, msg.c_str(),
             s->jit_minb, s->sm_cap_default,
             s->inner_hit ? "\"hit\"" : s->inner_entry ? "\"built\"" : "\"none\"",
             s->nparts, s->part_used ? "true" : "false", s->grow_count,
             (unsigned long long)(p->has_groupby ? s->h_gt.dump_cap : 0), scan_ms, replay_ms);
    return 0;
}

extern "C" uint32_t
xpuB200HashBytes(const void *data, uint32_t len)
{
    return xb_hash_bytes((const uint8_t *)data, len);
}
