/*
 * xb_final.h
 *
 * The final-stage kernels of the device translation unit (xb_exec.cu) and
 * their arguments: kds_final materialisation, GPU-Sort of the groups, the
 * merge of another kds_final into a session's group table and the
 * inner-buffer rebuild.  The host services that launch them live in
 * xb_final.cu (xpuB200Final, xpuB200MergeFinal, xpuB200FinalParts,
 * xpuB200InnerRebuild) and in xb_exec.cu (xpuB200FinalNoAlloc).  Internal;
 * the public interface is include/xpu_b200.h.
 */
#ifndef XB_FINAL_H
#define XB_FINAL_H

#include <cuda_runtime.h>
#include <cstdint>
#include "xb_plan.h"
#include "xb_exec_dev.cuh"

#define XB_GENT_MAX     2048    /* largest group entry a merge stages per thread */

/* kds_final materialisation: per-entry tuple sizes, then the tuples */
struct XbFinalArgs {
    const xb_plan  *plan;
    xb_gtable      *gt;
    uint64_t        cap;
    uint64_t       *sizes;          /* per entry: item bytes (0 if empty) */
    uint32_t       *flags;          /* per entry: 1 if ready */
    uint64_t       *size_scan;
    uint32_t       *flag_scan;
    char           *kds_final;      /* device buffer (header already in place) */
    uint64_t        items_base;     /* offset of the first item */
    uint64_t        length;
    uint32_t        nslots;
    uint32_t        row_format;     /* KDS_FORMAT_ROW (no GROUP BY keys): kern_tupitems
                                     * without hash links, nslots 0 */
    uint32_t        part_div;       /* >= 2: only the groups with hash % part_div == part_rem */
    uint32_t        part_rem;
    const int64_t  *keep;           /* GPU-Sort: output position per entry, -1 dropped
                                     * (nullptr: every group, in table order) */
};

/* GPU-Sort: the sort keys of the ready groups, as radix words */
struct XbSortArgs {
    const xb_plan  *plan;
    const xb_gtable *gt;
    uint64_t        cap;
    const uint32_t *flags;          /* per entry: 1 if ready */
    const uint32_t *flag_scan;
    uint32_t       *ents;           /* per rank: entry index */
    uint64_t       *keyw;           /* word w of key k at keyw[(2k + w) * n + r] */
    uint8_t        *nul;            /* NULL flag of key k at nul[k * n + r] */
    uint32_t        n;
};

/* groups kept, in order: LIMIT, or the window rank of each group within
 * its partition (row_number / rank / dense_rank) against its limit */
struct XbRankArgs {
    const xb_plan  *plan;
    const uint32_t *idx;            /* rank of the group at each sorted position */
    const uint64_t *keyw;
    const uint8_t  *nul;
    uint32_t        n;
    uint32_t       *part_start;     /* position that starts a new partition, else 0 */
    uint32_t       *peer_start;     /* position that starts a new peer group, else 0 */
    uint32_t       *peer_flag;      /* 1 where a peer group starts */
};

struct XbKeepArgs {
    const xb_plan  *plan;
    const uint32_t *idx;
    const uint32_t *ents;
    uint32_t        n;
    const uint32_t *part_start;     /* after the max-scan: the partition's first position */
    const uint32_t *peer_start;     /* after the max-scan */
    const uint32_t *peer_cnt;       /* inclusive sum of peer_flag */
    uint32_t       *keep_flag;
};

/* merge of another kds_final into the session's group table */
struct XbMergeArgs {
    const xb_plan          *plan;
    const kern_data_store  *kds;        /* the other kds_final (device copy) */
    xb_gtable              *gt;
    xb_status              *st;
};

/* inner-buffer rebuild into a KDS_FORMAT_HASH buffer */
struct XbRebuildArgs {
    kern_data_store        *dst;
    const kern_data_store  *src;
    uint64_t                dst_head;   /* KDS_HEAD_LENGTH(dst) */
    uint64_t                src_rowidx; /* offset of src's row index */
    uint32_t                divisor;    /* 0: every row */
    uint32_t                remainder;
    uint32_t               *overflow;
};

/* the kernels (xb_exec.cu) */
__global__ void xb_final_sizes(XbFinalArgs args);
__global__ void xb_final_write(XbFinalArgs args);
__global__ void xb_sort_gather(XbSortArgs a);
__global__ void xb_sort_keys(XbSortArgs a);
__global__ void xb_sort_pass_key64(const uint64_t *col, const uint32_t *idx, uint64_t *out, uint32_t n);
__global__ void xb_sort_pass_key8(const uint8_t *col, const uint32_t *idx, uint8_t *out, uint32_t n);
__global__ void xb_sort_bounds(XbRankArgs a);
__global__ void xb_sort_keepflag(XbKeepArgs a);
__global__ void xb_sort_keep(XbKeepArgs a, const uint32_t *keep_scan, int64_t *keep);
__global__ void xb_iota_u32(uint32_t *out, uint32_t n);
__global__ void __launch_bounds__(XB_BLOCK) xb_merge_final(XbMergeArgs args);
__global__ void __launch_bounds__(XB_BLOCK) xb_inner_rebuild(XbRebuildArgs args);

/* 256-byte alignment of the work arrays carved from one buffer */
static inline uint64_t xb_align256(uint64_t x)
{
    return (x + 255) & ~255ULL;
}

#endif  /* XB_FINAL_H */
