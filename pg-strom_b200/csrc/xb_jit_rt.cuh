/*
 * xb_jit_rt.cuh
 *
 * Skeleton of the session-specialised executor kernel.  xb_jit.cpp emits,
 * for one translated session (xb_plan) and one source format, a CUDA
 * translation unit of the form
 *
 *     #include "xb_exec_dev.cuh"
 *     #define XBJ_NREGS ... (plan constants)
 *     struct XbjRegs { ... };          registers as plain locals
 *     #include "xb_jit_rt.cuh"         this file: prototypes + kernel
 *     ... generated definitions of xbj_decode / xbj_pipeline ...
 *
 * compiled by NVRTC for sm_100a.  Each lane carries one source row through
 * decode, scan quals, every join depth (per-lane probe loops over the
 * inner hash indexes) and the group-by update, with the plan's bytecode
 * turned into straight-line code over registers.  Units (heap pages,
 * 1024-row groups) are claimed per warp from the launch's work queue
 * exactly as in the interpreting kernel (xb_exec.cu), and the statistics,
 * shared-memory group table and error reporting are the same.
 */
#ifndef XBJ_RT_TAIL
#ifndef XB_JIT_RT_CUH
#define XB_JIT_RT_CUH

#ifndef XBJ_ARROW_AHEAD
#define XBJ_ARROW_AHEAD 4       /* 32-row batches an Arrow column's lines are prefetched ahead */
#endif

#ifndef XBJ_PF_LEAD
#define XBJ_PF_LEAD     32      /* rows of a page left when the next page is prefetched (0: none) */
#endif

struct XbjEnv {
    const xb_plan  *plan;           /* device plan (global memory) */
    xb_status      *st;
    xb_gtable      *gt;
    char           *gt_entries;     /* global group table */
    uint64_t        gt_mask;
    char           *sm_tab;         /* shared-memory group table, or nullptr */
    uint32_t        sm_mask;
    uint32_t        lane;
    char           *dst;            /* projection: kds_dst and its length */
    uint64_t        dst_len;
    const uint32_t *sbits;          /* existence bitmaps in shared memory */
    char           *part_buf;       /* partitioned aggregation (XbExecArgs) */
    uint32_t       *part_cnt;
    uint32_t        part_cap;
    uint32_t        part_shift;
    uint32_t        replay;         /* in the replay: a full table leaves the record for later */
};

/* per-thread counters, 32-bit to spare registers; flushed into the launch
 * totals whenever one passes 2^31 (checked once per batch) */
struct XbjCnt {
    uint32_t raw, in, out;
    uint32_t depth[XB_MAX_DEPTH + 1];
    uint64_t gready;                /* group-id entries this lane has seen ready */
};

__device__ __forceinline__ void xbj_flush_cnt(XbjCnt &C, xb_status *st)
{
    atomicAdd((unsigned long long *)&st->nitems_raw, (unsigned long long)C.raw);
    atomicAdd((unsigned long long *)&st->nitems_in, (unsigned long long)C.in);
    atomicAdd((unsigned long long *)&st->nitems_out, (unsigned long long)C.out);
    C.raw = C.in = C.out = 0;
#pragma unroll
    for (int d = 1; d <= XBJ_NRELS; d++) {
        atomicAdd((unsigned long long *)&st->nitems_depth[d], (unsigned long long)C.depth[d]);
        C.depth[d] = 0;
    }
}

/* generated per session: decode item idx of the current unit (page: heap
 * page of a BLOCK chunk; kds / row0: chunk and first row of an ARROW or ROW
 * unit; lp: the heap item's line pointer; acol: an ARROW unit's resolved
 * columns) */
__device__ __forceinline__ bool
xbj_decode(XbjRegs &R, const XbExecArgs &args, const uint8_t *page, const kern_data_store *kds,
           uint32_t row0, const XbSrcMeta *meta, uint32_t idx, uint32_t lp, bool lay_ok, bool &exists,
           xb_status *st, const XbArrowCol *acol);

#ifdef XBJ_BITS
/* generated: copy the filter depths' existence bitmaps into shared memory
 * (all threads of the CTA); returns their bytes */
__device__ __forceinline__ uint32_t xbj_stage_bits(uint32_t *sb, const xb_plan *plan);
#endif

#ifdef XBJ_LAYOUT
/* generated: the launch's heap layout is the one the kernel is built for */
__device__ __forceinline__ bool xbj_layout_ok(const XbSrcMeta *meta);
#endif

/* line pointer i of a heap page of nitems items (0 = LP_UNUSED past the end) */
__device__ __forceinline__ uint32_t xbj_itemid(const uint8_t *page, uint32_t nitems, uint32_t i)
{
    return i < nitems ? (uint32_t)xb_fetch_le(page + SizeOfPageHeaderData + 4 * i, 4) : 0u;
}

__device__ __forceinline__ void xbj_prefetch_l1(const void *p)
{
    asm volatile("prefetch.global.L1 [%0];" :: "l"(p));
}

/* pull the tuple of line pointer lp into L1 (both ends: it may straddle a line) */
__device__ __forceinline__ void xbj_prefetch_tuple(const uint8_t *page, uint32_t lp)
{
    if (ITEMID_FLAGS(lp) == LP_NORMAL) {
        const uint32_t off = ITEMID_OFF(lp), len = ITEMID_LEN(lp);
        if (len > 0 && off + len <= PGSTROM_BLCKSZ) {
            xbj_prefetch_l1(page + off);
            xbj_prefetch_l1(page + off + len - 1);
        }
    }
}

__device__ __forceinline__ void
xbj_pipeline(XbjRegs &R, const XbjEnv &E, XbjCnt &C, bool &failed);

#ifdef XBJ_PART
/* the record's NULL-mask word carries this bit while the record waits for
 * the group table to grow (a replay that found the table without room) */
#define XBJ_REC_LEFT    0x80000000u
/* generated: a deferred row's record, and the group update of one row
 * (returns true when, replaying, the table had no room for the group) */
__device__ __forceinline__ void xbj_rec_load(const char *rec, XbjRegs &R, uint32_t &ghash);
__device__ __forceinline__ bool xbj_group_row(XbjRegs &R, const XbjEnv &E, const uint32_t ghash, bool &failed);
#endif

#ifdef XBJ_MERGE_SM
/* generated: merge of a shared-table entry (shared form) into the global
 * table's entry g */
__device__ __noinline__ void xbj_merge_sm(char *g, const char *e);
#endif

#ifdef XBJ_STAGE
/* ---- heap pages staged in shared memory ------------------------------
 * Every warp owns one 8 KB page buffer and an mbarrier.  A page whose
 * address is 16-byte aligned is copied into the buffer by one bulk copy
 * (cp.async.bulk, the TMA engine: one instruction for the whole page, no
 * per-lane global loads) and the warp decodes it from shared memory; a
 * page that is not aligned is read in place.  Waits are bounded. */
#define XBJ_STAGE_WAIT_LIMIT    (1u << 22)

__device__ __forceinline__ uint32_t xbj_smem_addr(const void *p)
{
    return (uint32_t)__cvta_generic_to_shared(p);
}

__device__ __forceinline__ void xbj_mbar_init(uint64_t *mbar)
{
    asm volatile("mbarrier.init.shared::cta.b64 [%0], 1;" :: "r"(xbj_smem_addr(mbar)) : "memory");
    asm volatile("fence.proxy.async.shared::cta;" ::: "memory");
}

/* lane 0: copy 8 KB from global gsrc into the shared buffer, completing
 * on mbar (generic reads of the buffer before this are ordered first) */
__device__ __forceinline__ void xbj_stage_issue(void *buf, const void *gsrc, uint64_t *mbar)
{
    asm volatile("fence.proxy.async.shared::cta;" ::: "memory");
    asm volatile("mbarrier.arrive.expect_tx.shared::cta.b64 _, [%0], %1;"
                 :: "r"(xbj_smem_addr(mbar)), "r"((uint32_t)PGSTROM_BLCKSZ) : "memory");
    asm volatile("cp.async.bulk.shared::cluster.global.mbarrier::complete_tx::bytes [%0], [%1], %2, [%3];"
                 :: "r"(xbj_smem_addr(buf)), "l"(gsrc), "r"((uint32_t)PGSTROM_BLCKSZ), "r"(xbj_smem_addr(mbar))
                 : "memory");
}

/* wait for phase 'parity' of mbar; false when the wait gave up */
__device__ __forceinline__ bool xbj_stage_wait(uint64_t *mbar, uint32_t parity)
{
    const uint32_t a = xbj_smem_addr(mbar);
    for (uint32_t i = 0; i < XBJ_STAGE_WAIT_LIMIT; i++) {
        uint32_t done;
        asm volatile("{\n\t.reg .pred p;\n\t"
                     "mbarrier.try_wait.parity.shared::cta.b64 p, [%1], %2;\n\t"
                     "selp.u32 %0, 1, 0, p;\n\t}"
                     : "=r"(done) : "r"(a), "r"(parity) : "memory");
        if (done)
            return true;
    }
    return false;
}
#endif

/* 16 bytes of the group table holding its 'grow' word, copied into shared
 * memory through L2 (cp.async.cg: no L1 copy that could be stale) */
__device__ __forceinline__ void xbj_grow_fetch(uint32_t *buf, const xb_gtable *gt)
{
    asm volatile("cp.async.cg.shared.global [%0], [%1], 16;\n\t"
                 "cp.async.commit_group;"
                 :: "r"((uint32_t)__cvta_generic_to_shared(buf)), "l"((const char *)gt + 48) : "memory");
}

/* lane 0: the fetched 'grow' word, once its copy has landed */
__device__ __forceinline__ uint32_t xbj_grow_seen(const uint32_t *buf, uint32_t lane)
{
    if (lane != 0)
        return 0;
    asm volatile("cp.async.wait_all;" ::: "memory");
    return *(volatile const uint32_t *)&buf[1];
}

__device__ __forceinline__ unsigned long long xbj_warp_sum(unsigned long long v)
{
#pragma unroll
    for (int o = 16; o > 0; o >>= 1)
        v += __shfl_down_sync(XB_FULL, v, o);
    return v;
}

/* one launch's (or one mixed-launch command's) work for this CTA; ends
 * with the counters and the shared group table flushed, without a final
 * barrier */
__device__ __forceinline__ void
xbj_body(const XbExecArgs &args, char *smem)
{
    const uint32_t lane = threadIdx.x & 31;
    XbSrcMeta *meta = (XbSrcMeta *)smem;
    /* warp-uniform work-distribution state lives in shared memory, not in
     * registers (read once per unit) */
    XbSrc *wsrc = (XbSrc *)(smem + ((sizeof(XbSrcMeta) + 15) & ~(size_t)15));
    char *sm_entries = (char *)(wsrc + XB_WARPS);
    const size_t sm_bytes = (size_t)args.sm_cap * XBJ_SM_STRIDE;

    xb_setup_meta(args, meta);
    for (size_t i = threadIdx.x; i < sm_bytes / 4; i += blockDim.x)
        ((uint32_t *)sm_entries)[i] = 0;
    /* after the group table: the existence bitmaps of filter depths */
    uint32_t *sbits = (uint32_t *)(((uintptr_t)(sm_entries + sm_bytes) + 15) & ~(uintptr_t)15);
#ifdef XBJ_BITS
    const uint32_t sbits_bytes = xbj_stage_bits(sbits, args.plan);
#else
    const uint32_t sbits_bytes = 0;
#endif
    __syncthreads();

#ifdef XBJ_LAYOUT
    const bool lay_ok = xbj_layout_ok(meta);
#else
    const bool lay_ok = false;
#endif
    XbjEnv E;
    E.plan = args.plan;
    E.st = args.st;
    E.gt = args.gt;
    E.gt_entries = args.gt ? args.gt->entries : nullptr;
    E.gt_mask = args.gt ? args.gt->cap_mask : 0;
    E.sm_tab = args.sm_cap ? sm_entries : nullptr;
    E.sm_mask = args.sm_cap ? args.sm_cap - 1 : 0;
    E.lane = lane;
    E.dst = args.dst;
    E.dst_len = args.dst_len;
    E.sbits = sbits;
    E.part_buf = args.part_buf;
    E.part_cnt = args.part_cnt;
    E.part_cap = args.part_cap;
    E.part_shift = args.part_shift;
    E.replay = 0;
    XbjCnt C;
    C.raw = C.in = C.out = 0;
    C.gready = 0;
#pragma unroll
    for (int d = 0; d <= XB_MAX_DEPTH; d++)
        C.depth[d] = 0;

    XbSrc &src = wsrc[threadIdx.x >> 5];
#ifdef XBJ_ACOLS
    /* the warp's Arrow columns, resolved for its current unit */
    __shared__ XbArrowCol acol_all[XB_WARPS][XBJ_ACOLS];
    XbArrowCol *acol = acol_all[threadIdx.x >> 5];
#else
    XbArrowCol *acol = nullptr;
#endif
#ifdef XBJ_STAGE
    /* this warp's page buffer and its mbarrier, after the group table */
    char *stage_base = (char *)(((uintptr_t)((char *)sbits + sbits_bytes) + 127) & ~(uintptr_t)127);
    char *sbuf = stage_base + (size_t)(threadIdx.x >> 5) * PGSTROM_BLCKSZ;
    uint64_t *mbar = (uint64_t *)(stage_base + (size_t)XB_WARPS * PGSTROM_BLCKSZ) + (threadIdx.x >> 5);
    uint32_t sphase = 0;
    bool staged = false;            /* the current page is in sbuf */
    if (lane == 0)
        xbj_mbar_init(mbar);
    __syncwarp();
#endif
    xb_src_start(args, src, lane);
    const uint8_t *page = nullptr;
    const kern_data_store *kds = nullptr;
    uint32_t row0 = 0, item = 0, nitems = 0;
    /* heap pages are software-pipelined over the batches of a page: the
     * line pointers of the next batch are in registers and its tuples are
     * being pulled into L1 while this batch runs; the line pointers of the
     * batch after that are in flight */
    uint32_t lp_next = 0, lp_after = 0;

    for (;;) {
        bool done = false;
        while (item >= nitems) {
            const int rc = xb_next_unit(args, src, lane, args.format == KDS_FORMAT_ROW);
            if (rc == 0) { done = true; break; }
            if (rc == 2) {
                if (lane == 0) XB_RAISE(args.st, ERRCODE_DEVICE_ERROR, XB_MSG_BAD_PAGE);
                done = true;
                break;
            }
            page = src.page;
            kds = src.kds;
            row0 = src.row0;
            item = src.item;            /* 0, or where a resumed range starts */
            nitems = src.nitems;
#ifdef XBJ_STAGE
            staged = false;
            if ((((uintptr_t)page) & 15) == 0) {
                __syncwarp();           /* every lane is done with the buffer */
                if (lane == 0)
                    xbj_stage_issue(sbuf, page, mbar);
                __syncwarp();
                const bool ok_ = xbj_stage_wait(mbar, sphase);
                sphase ^= 1u;
                if (!__all_sync(XB_FULL, ok_)) {
                    if (lane == 0) XB_RAISE(args.st, ERRCODE_DEVICE_ERROR, XB_MSG_WAIT_TIMEOUT);
                    /* the copy is still owed to this barrier: wait once more */
                    xbj_stage_wait(mbar, sphase ^ 1u);
                    done = true;
                    break;
                }
                page = (const uint8_t *)sbuf;
                staged = true;
            }
#endif
            if (args.format == KDS_FORMAT_BLOCK) {
                lp_next = xbj_itemid(page, nitems, item + lane);
                lp_after = xbj_itemid(page, nitems, item + lane + 32);
            }
#ifdef XBJ_ACOLS
            __syncwarp();           /* every lane is done with the last unit's columns */
            xb_arrow_resolve(args.plan, kds, row0, nitems, acol, lane);
            __syncwarp();
#endif
        }
        if (done)
            break;
        /* the group table's growth request: lane 0 fetches it into shared
         * memory by an asynchronous copy now and looks at it after the
         * batch, so no register is held and no latency is waited for */
        if (args.left_out && lane == 0)
            xbj_grow_fetch(src.grow_buf, args.gt);
        const uint32_t idx = item + lane;
        uint32_t lp = 0;
#ifdef XBJ_ACOLS
        /* the columns' lines XBJ_ARROW_AHEAD batches ahead into L2: lane t
         * takes line t % 2 of column t / 2 (32 values of at most 8 bytes) */
        if (lane < 2 * XBJ_ACOLS) {
            const XbArrowCol &c_ = acol[lane >> 1];
            const uint32_t r_ = item + 32 * XBJ_ARROW_AHEAD;
            /* the first row of the line: a row of the batch, inside the buffer */
            const uint32_t rr_ = c_.width ? r_ + (lane & 1) * (128 / c_.width) : 0;
            if (c_.ok && c_.width && rr_ < r_ + 32 && rr_ < c_.nvalid)
                asm volatile("prefetch.global.L2 [%0];" :: "l"(c_.values + (size_t)rr_ * c_.width));
        }
#endif
        /* the warp's next heap page streams into L2 while the last
         * XBJ_PF_LEAD rows of this one are processed: early enough to
         * arrive, late enough not to be evicted by the pages streaming
         * through L2 meanwhile */
        if (XBJ_PF_LEAD > 0 && args.format == KDS_FORMAT_BLOCK && item + XBJ_PF_LEAD >= nitems &&
            (item < 32 || item + XBJ_PF_LEAD < nitems + 32))
            xb_prefetch_page(args, src, xb_following_unit(src), lane);
        if (args.format == KDS_FORMAT_BLOCK) {
            lp = lp_next;
            lp_next = lp_after;
            /* (the fast decode of a known layout reads the tuple with two
             * wide loads; there the L1 prefetch only costs issue slots) */
            if (!(lay_ok && XBJ_LAY_FIXED)
#ifdef XBJ_STAGE
                && !staged
#endif
                )
                xbj_prefetch_tuple(page, lp_next);
            lp_after = xbj_itemid(page, nitems, idx + 64);
        }
        item += 32;
        bool failed = false;
        if (idx < nitems) {
            XbjRegs R;
            bool exists = false;
            const bool ok = xbj_decode(R, args, page, kds, row0, meta, idx, lp, lay_ok, exists, args.st, acol);
            if (exists)
                C.raw++;
            if (exists && !ok)
                failed = true;
            else if (ok)
                xbj_pipeline(R, E, C, failed);
        }
        uint32_t big = C.out | C.in | C.raw;
#pragma unroll
        for (int d = 1; d <= XBJ_NRELS; d++)
            big |= C.depth[d];
        if (big & 0x80000000u)
            xbj_flush_cnt(C, args.st);
        if (__any_sync(XB_FULL, failed))
            break;
        if (args.left_out && __shfl_sync(XB_FULL, xbj_grow_seen(src.grow_buf, lane), 0)) {
            /* the table is to grow: leave the rest for the resume launch */
            xb_src_leave(args, src, lane, item, nitems);
            break;
        }
    }

#ifdef XBJ_STAGE
    /* the barrier's memory becomes group-table or buffer space again */
    __syncwarp();
    if (lane == 0)
        asm volatile("mbarrier.inval.shared::cta.b64 [%0];" :: "r"(xbj_smem_addr(mbar)) : "memory");
#endif
    /* statistics */
    {
        const unsigned long long raw = xbj_warp_sum(C.raw);
        const unsigned long long in = xbj_warp_sum(C.in);
        const unsigned long long out = xbj_warp_sum(C.out);
        /* (64-bit sums: 32 lanes' 32-bit counts may exceed 2^32) */
        if (lane == 0) {
            atomicAdd((unsigned long long *)&args.st->nitems_raw, raw);
            atomicAdd((unsigned long long *)&args.st->nitems_in, in);
            atomicAdd((unsigned long long *)&args.st->nitems_out, out);
        }
#pragma unroll
        for (int d = 1; d <= XBJ_NRELS; d++) {
            const unsigned long long v = xbj_warp_sum(C.depth[d]);
            if (lane == 0)
                atomicAdd((unsigned long long *)&args.st->nitems_depth[d], v);
        }
    }
    __syncthreads();

    /* merge the shared-memory group table into the global table */
    if (args.sm_cap) {
        const xb_plan *plan = args.plan;
        for (uint32_t i = threadIdx.x; i < args.sm_cap; i += blockDim.x) {
            char *e = sm_entries + (size_t)i * XBJ_SM_STRIDE;
            const xb_gent_head *h = (const xb_gent_head *)e;
            if (h->state != XB_GSTATE_READY)
                continue;
            const xb_keyimg *img = (const xb_keyimg *)(e + XBJ_KEYS_OFF);
            char *g = xb_group_find_or_dump(plan, args.gt, h->hash, img, args.st);
            if (g)
#ifdef XBJ_MERGE_SM
                xbj_merge_sm(g, e);
#else
                xb_merge_states(plan, g, e);
#endif
        }
    }
}

extern "C" __global__ void __launch_bounds__(XB_BLOCK, XBJ_MIN_BLOCKS)
xbj_kernel(const __grid_constant__ XbExecArgs args)
{
    extern __shared__ __align__(16) char smem[];
    xbj_body(args, smem);
}

/* mixed launch of commands of sessions that share this kernel (same plan
 * shape; their constants, tables and statuses come with each command):
 * work item i sends a CTA to command items[i], as in xb_mixed_kernel */
extern "C" __global__ void __launch_bounds__(XB_BLOCK, XBJ_MIN_BLOCKS)
xbj_mixed_kernel(const __grid_constant__ XbMixArgs m)
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
        xbj_body(cmd, smem);
        __syncthreads();
    }
}

#endif  /* XB_JIT_RT_CUH */
#else   /* XBJ_RT_TAIL */
#ifndef XB_JIT_RT_TAIL_DONE
#define XB_JIT_RT_TAIL_DONE
/* ---- the tail: included again at the end of the generated source (after
 * XBJ_RT_TAIL is defined), where every generated definition is known ---- */

#ifdef XBJ_PART
/* replay of the deferred rows.  A bucket holds the rows whose groups have
 * their home slot in one slice of the global table (1 << part_shift
 * slots).  Each CTA claims buckets in order, so the CTAs work on
 * neighbouring slices together and the slices stay in L2; the bucket's
 * records and its slice are pulled into L2 by the TMA engine when it is
 * claimed.  Every row updates its group in the global table (the same
 * update as in place).  A row whose group the table and its dump have no
 * room for (the table asked to grow meanwhile) is marked and replayed
 * after the growth (retry). */
extern "C" __global__ void __launch_bounds__(XB_BLOCK, XBJ_MIN_BLOCKS)
xbj_replay(const __grid_constant__ XbReplayArgs args)
{
    __shared__ uint32_t cur;            /* the CTA's bucket */
    XbjEnv E;
    E.plan = args.plan;
    E.st = args.st;
    E.gt = args.gt;
    E.gt_entries = args.gt->entries;
    E.gt_mask = args.gt->cap_mask;
    E.sm_tab = nullptr;
    E.sm_mask = 0;
    E.lane = threadIdx.x & 31;
    E.dst = nullptr;
    E.dst_len = 0;
    E.sbits = nullptr;
    E.part_buf = nullptr;
    E.part_cnt = nullptr;
    E.part_cap = 0;
    E.part_shift = 0;
    E.replay = 1;
    for (;;) {
        if (threadIdx.x == 0)
            cur = atomicAdd(args.cursor, 1u);
        __syncthreads();
        const uint32_t b = cur;
        if (b >= args.nparts)
            break;
        const uint32_t cnt = args.part_cnt[(size_t)b * XB_PART_CNT_STRIDE];
        const uint32_t n = cnt < args.part_cap ? cnt : args.part_cap;
        char *base = args.part_buf + (uint64_t)b * args.part_cap * XBJ_REC_SIZE;
        if (threadIdx.x == 0 && !args.retry && n) {
            const uint64_t rb = (uint64_t)n * XBJ_REC_SIZE;
            /* (a bulk prefetch starts on a 16-byte boundary: a bucket of
             * records of a size that is no multiple of 16 may not) */
            if ((((uintptr_t)base) & 15) == 0 && rb >= 16)
                xb_prefetch_l2(base, (uint32_t)(rb < (1u << 20) ? rb : (1u << 20)) & ~15u);
            if (args.part_shift && ((uint64_t)b << args.part_shift) <= E.gt_mask) {
                const uint64_t sb = ((uint64_t)XBJ_GENT_SIZE << args.part_shift);
                const char *sl = E.gt_entries + ((uint64_t)b << args.part_shift) * XBJ_GENT_SIZE;
                if ((((uintptr_t)sl) & 15) == 0 && sb <= (1u << 20))
                    xb_prefetch_l2(sl, (uint32_t)sb & ~15u);
            }
        }
        for (uint32_t i = threadIdx.x; i < n; i += blockDim.x) {
            char *rec = base + (uint64_t)i * XBJ_REC_SIZE;
            /* a retry replays only the records a full table left behind */
            if (args.retry && !(((const uint32_t *)rec)[1] & XBJ_REC_LEFT))
                continue;
            XbjRegs R;
            uint32_t ghash;
            xbj_rec_load(rec, R, ghash);
            bool failed = false;
            const bool table_full = xbj_group_row(R, E, ghash, failed);
            if (table_full) {
                ((uint32_t *)rec)[1] |= XBJ_REC_LEFT;
                if (!args.st->replay_left)
                    atomicExch(&args.st->replay_left, 1u);
            } else if (args.retry) {
                ((uint32_t *)rec)[1] &= ~XBJ_REC_LEFT;
            }
        }
        /* every thread has read cur */
        __syncthreads();
    }
}
#endif

#endif  /* XB_JIT_RT_TAIL_DONE */
#endif  /* XBJ_RT_TAIL */
