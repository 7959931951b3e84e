/*
 * xb_plan.h
 *
 * The compiled form of one PG-Strom session, as executed by the B200
 * kernels.  OpenSession translates the kern_session_info bytecode
 * (LoadVars / ScanQuals / HashValue / JoinQuals / GroupBy*) into this
 * structure once; every ExecTask then runs it without re-reading the
 * kern_expression trees.
 *
 * Execution model (device):
 *   - one warp processes 32 source rows at a time (one row per lane);
 *   - every kvars slot of the session is a VM register; registers live in
 *     shared memory as [reg][lane] 64-bit cells plus a 32-bit aux word and
 *     a per-register NULL ballot, so the interpreter's instruction stream
 *     is warp-uniform (no divergence on dispatch);
 *   - expression trees become straight-line register programs (xb_insn);
 *     AND/OR keep SQL 3-valued semantics and short-circuit by narrowing the
 *     lane mask instead of branching;
 *   - hash joins probe a rebuilt open-addressing index over the inner
 *     KDS_FORMAT_HASH rows, whose referenced columns are pre-decoded into
 *     SoA register images at OpenSession;
 *   - GROUP BY updates a per-CTA shared-memory table, spilling to a global
 *     open-addressing table in HBM; Final materialises kds_final in the
 *     reference's KDS_FORMAT_HASH / kagg_state__* layout.
 */
#ifndef XB_PLAN_H
#define XB_PLAN_H
#include <stdint.h>
#include "pgstrom_abi.h"

#define XB_MAX_REGS         48      /* kvars slots + temporaries */
#define XB_MAX_DEPTH        6       /* inner relations per session */
#define XB_MAX_LOADS        32      /* LoadVars descriptors per depth */
#define XB_MAX_KEYS         8       /* GROUP BY keys */
#define XB_MAX_AGGS         32      /* partial aggregate columns */
#define XB_MAX_INSNS        384     /* VM instructions per session */
#define XB_MAX_COLS         64      /* source columns decoded per tuple */
#define XB_MAX_PROJ         32      /* attributes of a projected row */
#define XB_MASK_STACK       8

/* register kinds */
#define XB_RK_INT       1   /* bool/int2/int4/int8/date/time/timestamp as int64 */
#define XB_RK_FLT       2   /* float8 as IEEE754 double */
#define XB_RK_TEXT      3   /* payload pointer + length (aux) */
#define XB_RK_NUM       4   /* pointer to a numeric varlena */

/* how a register is loaded from a tuple attribute */
#define XB_LD_BOOL      1
#define XB_LD_INT2      2
#define XB_LD_INT4      3
#define XB_LD_INT8      4
#define XB_LD_FLT8      5
#define XB_LD_FLT4      6
#define XB_LD_DATE      7
#define XB_LD_TEXT      8   /* text / varchar / bpchar / bytea */
#define XB_LD_NUMERIC   9

/* VM opcodes */
#define XB_OP_END           0
#define XB_OP_CONST         1   /* dst <- imm (kind); aux=1 -> NULL; text: aux=len */
#define XB_OP_MOVE          2   /* dst <- a */
#define XB_OP_CMP           3   /* dst <- a <sub> b, kind = operand kind */
#define XB_OP_ARITH         4   /* dst <- a <sub> b, checked */
#define XB_OP_CAST          5   /* dst <- cast(a), sub = cast kind */
#define XB_OP_NOT           6
#define XB_OP_NULLTEST      7   /* sub: 0=IS NULL, 1=IS NOT NULL */
#define XB_OP_BOOLTEST      8   /* sub: 0..5 = IsTrue..IsNotUnknown */
#define XB_OP_BOOL_INIT     9   /* dst <- TRUE (sub=0, AND) / FALSE (sub=1, OR) */
#define XB_OP_AND_ACC       10  /* dst <- dst AND a (3-valued) */
#define XB_OP_OR_ACC        11  /* dst <- dst OR a (3-valued) */
#define XB_OP_MASK_PUSH     12
#define XB_OP_MASK_NARROW   13  /* sub 0: drop lanes where a IS FALSE; 1: where a IS TRUE */
#define XB_OP_MASK_POP      14
#define XB_OP_HASH_INIT     15  /* dst <- 0xffffffff */
#define XB_OP_HASH_ADD      16  /* dst <- merge(dst, hash(a)); skips NULL; sub = hash kind */
#define XB_OP_HASH_FINI     17  /* dst <- dst ^ 0xffffffff */
#define XB_OP_DISTINCT      18  /* dst <- a IS DISTINCT FROM b (kind) */
#define XB_OP_CMPI          19  /* dst <- a <sub> imm (kind INT or FLT), NULL if a NULL */
#define XB_OP_HASH1         20  /* dst <- HashValue(a): init, add (sub = hash kind), final */

/* XB_OP_CMP sub-ops */
#define XB_CMP_EQ   0
#define XB_CMP_NE   1
#define XB_CMP_LT   2
#define XB_CMP_LE   3
#define XB_CMP_GT   4
#define XB_CMP_GE   5

/* XB_OP_ARITH sub-ops: low nibble = operator, high nibble = result width */
#define XB_AR_ADD   0
#define XB_AR_SUB   1
#define XB_AR_MUL   2
#define XB_AR_DIV   3
#define XB_AR_W2    (1 << 4)
#define XB_AR_W4    (2 << 4)
#define XB_AR_W8    (3 << 4)

/* XB_OP_CAST sub-ops */
#define XB_CAST_I2I2    1   /* to int2 with range check */
#define XB_CAST_I2I4    2
#define XB_CAST_I2I8    3
#define XB_CAST_I2F8    4
#define XB_CAST_F82I2   5
#define XB_CAST_F82I4   6
#define XB_CAST_F82I8   7
#define XB_CAST_I2BOOL  8

/* XB_OP_HASH_ADD kinds: byte width of the hashed value, or special */
#define XB_HK_W1    1
#define XB_HK_W2    2
#define XB_HK_W4    4
#define XB_HK_W8    8
#define XB_HK_TEXT  20
#define XB_HK_NUM   21
#define XB_HK_CACHED 22     /* hash precomputed by the inner build (text/numeric
                             * column of a join's inner relation) */

typedef struct xb_insn {
    uint8_t     op;
    uint8_t     dst;
    uint8_t     a;
    uint8_t     b;
    uint8_t     sub;
    uint8_t     kind;
    uint16_t    aux;
    int64_t     imm;
} xb_insn;

typedef struct xb_prog {
    uint16_t    start;      /* first instruction in xb_plan.insns */
    uint16_t    count;      /* 0 = no program */
    int16_t     result;     /* register holding the result, or -1 */
    uint16_t    __pad;
} xb_prog;

typedef struct xb_load {
    int16_t     resno;      /* attribute number (1-based; <0 system column) */
    uint8_t     reg;
    uint8_t     ld;         /* XB_LD_* */
} xb_load;

/* a pre-decoded inner relation (one join depth) */
typedef struct xb_inner {
    uint32_t    nitems;
    uint32_t    cap_mask;       /* index capacity - 1 (power of two) */
    uint32_t    unique_hash;    /* 1 if all inner hash values differ */
    uint32_t    nloads;
    uint64_t   *index;          /* (hash << 32) | (row + 1); 0 = empty */
    uint64_t   *vals;           /* [nloads][nitems] register images */
    uint32_t   *auxs;           /* [nloads][nitems] */
    uint32_t   *nulls;          /* [nloads][(nitems+31)/32] bit = NULL */
    uint32_t    hasnull;        /* bit k: inner column k has NULLs (set by the build) */
    uint32_t    live;           /* bit k: register of load k is read after the join */
    /* fused probe: HashValue(outer) + JoinQuals(outer = inner key) */
    int16_t     fast_key;       /* load index of the inner key, -1: no fused probe */
    uint8_t     fast_outer;     /* outer key register */
    uint8_t     fast_hk;        /* hash kind of the outer key */
    uint32_t    key32;          /* index entries hold (key32 << 32 | row + 1):
                                 * the fused key is int2 / int4 / date */
    xb_prog     build_qual;     /* join quals over this inner row alone, run once per
                                 * inner row by the build; failing rows stay out of index */
    /* direct addressing: a unique, dense 32-bit fused key maps straight to
     * its row through dtab[key - dkey_min] (row + 1, 0 = none) */
    int32_t     dkey_min;       /* smallest / largest indexed key (build) */
    int32_t     dkey_max;
    uint32_t    nindexed;       /* rows inserted into the index (build) */
    uint32_t    direct;         /* 1: dtab is valid */
    uint32_t    drange;         /* dkey_max - dkey_min + 1 */
    uint32_t   *dtab;
    /* dense group ids: when every GROUP BY key is a column of this depth,
     * gids[row] numbers the distinct key tuples of the inner rows (0..ngids-1) */
    uint32_t    gid_on;         /* 1: gids valid (and carried in direct records) */
    uint32_t    ngids;
    uint32_t   *gids;
    /* direct records: the live columns of the row of key k packed at
     * dpay + (k - dkey_min) * drec_size (layout: xb_drec_layout) */
    uint32_t    drec_size;
    /* existence bitmap of a direct depth whose rows carry no columns (a
     * pure filter): bit k - dkey_min is set when key k has a row; small
     * enough to be staged in shared memory by the specialised kernels */
    uint32_t    dbits_words;    /* 0: none */
    char       *dpay;
    uint32_t   *dbits;
    uint32_t    hashed;         /* bit k: hash of load k precomputed into hashes[] */
    uint32_t   *hashes;         /* [nloads][nitems] datum hashes (hashed loads) */
    xb_load     load[XB_MAX_LOADS];
} xb_inner;

/* one GPU-Sort key over the group entries (kern_sortkey_desc) */
#define XB_MAX_SORTKEYS 8
typedef struct xb_sortkey {
    uint16_t    kind;           /* KSORT_KEY_KIND__* */
    uint16_t    agg;            /* index into aggs[] (src_anum - 1) */
    uint8_t     asc;
    uint8_t     nulls_first;
    uint8_t     words;          /* 64-bit words of the encoded key (1 or 2) */
    uint8_t     __pad;
} xb_sortkey;

/* one partial-aggregate (or grouping key) column of the kds_final tuple */
typedef struct xb_agg {
    uint16_t    action;         /* KAGG_ACTION__* */
    int16_t     arg0;           /* register, or -1 */
    int16_t     arg1;
    int16_t     filter;         /* register of FILTER clause, or -1 */
    int32_t     typmod;
    uint16_t    state_off;      /* byte offset of the state in a group entry */
    uint16_t    state_sz;
    int16_t     weight;         /* numeric: __numeric_typmod_weight(typmod) */
    int16_t     key_index;      /* VREF: index into keys[], else -1 */
    /* kds_final column attributes */
    int16_t     attlen;
    int8_t      attalign;
    int8_t      __pad;
} xb_agg;

typedef struct xb_key {
    uint8_t     reg;
    uint8_t     rk;             /* XB_RK_* */
    uint8_t     ld;             /* XB_LD_* of the key type (for write-out) */
    uint8_t     hk;             /* XB_HK_* */
    uint16_t    off;            /* offset of the key image in a group entry */
    uint16_t    __pad;
} xb_key;

/* one attribute of a projected row (kds_dst column) */
typedef struct xb_projcol {
    int16_t     attlen;         /* kds_dst column */
    int8_t      attalign;
    uint8_t     ld;             /* XB_LD_* of the source slot: how to write it */
    uint8_t     reg;            /* source register (kvars slot) */
    uint8_t     __pad[3];
} xb_projcol;

typedef struct xb_plan {
    uint32_t    magic;
    uint32_t    plan_sz;
    uint32_t    nregs;
    uint32_t    nslots;
    uint32_t    nrels;
    uint32_t    task_kind;      /* DEVTASK__* bits */
    uint8_t     rk[XB_MAX_REGS];

    /* depth 0: source tuples */
    uint32_t    nload0;
    int32_t     max_resno0;
    /* heap layout the specialised kernel is built for (host side, from the
     * first heap chunk a session sees): the cached offset of every depth-0
     * load, all fixed-width and naturally aligned, and their end */
    uint32_t    lay_valid;
    uint32_t    lay_end;
    int32_t     lay_off[XB_MAX_LOADS];
    /* the column descriptors of columns 1..walk_ncols (attlen 1..8 or -1,
     * attalign), for a generated walk over tuples with NULLs or varlena
     * columns before a loaded one; walk_ncols 0: none */
    uint32_t    walk_ncols;
    int16_t     walk_len[XB_MAX_COLS];
    int8_t      walk_align[XB_MAX_COLS];
    xb_load     load0[XB_MAX_LOADS];
    xb_prog     scan_quals;

    /* depth 1..nrels: hash joins */
    xb_prog     hash_value[XB_MAX_DEPTH + 1];
    xb_prog     join_quals[XB_MAX_DEPTH + 1];
    xb_inner    inner[XB_MAX_DEPTH + 1];

    /* group-by */
    uint32_t    has_groupby;    /* 1: GROUP BY keys, 2: no-group aggregation */
    xb_prog     gb_args;        /* SaveExpr argument evaluation */
    xb_prog     gb_keyhash;
    xb_prog     gb_all;         /* gb_args followed by gb_keyhash, as one program */
    uint32_t    nkeys;
    xb_key      keys[XB_MAX_KEYS];
    uint32_t    naggs;
    xb_agg      aggs[XB_MAX_AGGS];
    uint32_t    gent_size;      /* bytes of one group entry (multiple of 16) */
    uint32_t    gid_depth;      /* inner depth holding every group key (0: none) */
    uint32_t    gent_keys_off;
    uint32_t    nkeys_text;     /* number of text/numeric keys (arena use) */

    /* device projection into kds_dst (execGpuJoinProjection) */
    uint32_t    has_proj;
    uint32_t    proj_nattrs;
    uint32_t    proj_margin;    /* gpusort_htup_margin added to every row */
    uint32_t    proj_head_len;  /* KDS_HEAD_LENGTH of the kds_dst template */
    xb_prog     proj_args;      /* SaveExpr programs filling the projected slots */
    xb_projcol  proj[XB_MAX_PROJ];
    /* rows go into a KDS_FORMAT_HASH kds_dst (a pinned inner buffer): the
     * hash of every row (u.proj.hash) and the destination's hash slots */
    uint32_t    proj_hashed;
    uint32_t    proj_nslots;
    xb_prog     proj_hash;
    xb_prog     proj_all;       /* proj_args, then proj_hash: one program */

    /* GPU-Sort of the groups at Final (SortKeys, gpusort_limit_count) */
    uint32_t    nsort;
    xb_sortkey  sort[XB_MAX_SORTKEYS];
    char        sort_window;    /* KSORT_WINDOW_FUNC__*, or 0 */
    uint8_t     sort_partby;    /* leading keys that partition the window */
    uint8_t     sort_orderby;   /* keys after them that order it */
    uint8_t     __pad4;
    uint32_t    sort_rank_limit;
    int64_t     sort_limit;     /* LIMIT without a window function; 0: none */

    /* spins a lane waits on a BUSY group entry before it gives up with
     * XB_MSG_WAIT_TIMEOUT (XB_WAIT_LIMIT unless a test shortens it) */
    uint32_t    wait_limit;

    /* VM code */
    uint32_t    ninsns;
    xb_insn     insns[XB_MAX_INSNS];
} xb_plan;

#define XB_PLAN_MAGIC   0x78623230U     /* 'xb20' */
#define XB_WAIT_LIMIT   (1u << 22)      /* default bounded spin on a BUSY group entry */

#ifdef __CUDACC__
#define XB_PLAN_HD __host__ __device__ inline
#else
#define XB_PLAN_HD static inline
#endif

/*
 * Layout of a direct record: a u32 header (bit 31: a row holds this key,
 * bit k: load k is NULL), the u32 group id when gid_on, then one u32 per
 * live text length and per live
 * precomputed hash, then the u64 value of every live load (8-aligned);
 * the size is a multiple of 16.  Offsets of load k are -1 where absent.
 * Returns the record size.
 */
XB_PLAN_HD uint32_t
xb_drec_layout(const xb_inner *in, const uint8_t *rk, int k, int *off_val, int *off_aux, int *off_hash)
{
    uint32_t off = in->gid_on ? 8 : 4;      /* header, then the group id */
    if (off_val) *off_val = -1;
    if (off_aux) *off_aux = -1;
    if (off_hash) *off_hash = -1;
    for (uint32_t j = 0; j < in->nloads; j++) {
        if (!((in->live >> j) & 1u))
            continue;
        if (rk[in->load[j].reg] == XB_RK_TEXT) {
            if ((int)j == k && off_aux) *off_aux = (int)off;
            off += 4;
        }
        if ((in->hashed >> j) & 1u) {
            if ((int)j == k && off_hash) *off_hash = (int)off;
            off += 4;
        }
    }
    off = (off + 7) & ~7u;
    for (uint32_t j = 0; j < in->nloads; j++) {
        if (!((in->live >> j) & 1u))
            continue;
        if ((int)j == k && off_val) *off_val = (int)off;
        off += 8;
    }
    return (off + 15) & ~15u;
}

/* group entry header (global and shared-memory tables) */
#define XB_GSTATE_EMPTY 0u
#define XB_GSTATE_BUSY  1u
#define XB_GSTATE_READY 2u
typedef struct xb_gent_head {
    uint32_t    hash;
    uint32_t    state;
} xb_gent_head;

/* key image inside a group entry: 16 bytes per key */
typedef struct xb_keyimg {
    uint64_t    val;        /* int/float bits, or pointer to the key bytes */
    uint32_t    len;        /* text length */
    uint32_t    isnull;
} xb_keyimg;

/* one chunk of a launch's work queue (device): units are heap pages for
 * KDS_FORMAT_BLOCK and 1024-row groups for ARROW / ROW chunks */
typedef struct xb_task {
    const kern_data_store *kds;
    uint64_t    unit_base;      /* first global unit of this chunk */
    uint32_t    nunits;
    uint32_t    format;
} xb_task;

/* global group table.  It grows between launches (the host rehashes it
 * into a larger one, as the reference's service expands kds_final on
 * SUSPEND_NO_SPACE, gpu_service.c:2418-2470): a launch that sees 'grow'
 * stops claiming work and records what it left (XbLeft ranges); groups
 * that find the table without room meanwhile take an entry of the dump
 * region, merged into the grown table before the work resumes */
typedef struct xb_gtable {
    uint64_t    cap_mask;
    uint64_t    nused;          /* number of claimed entries (dump entries included) */
    char       *entries;        /* cap * gent_size bytes */
    char       *arena;          /* text/numeric key bytes */
    uint64_t    arena_sz;
    uint64_t    arena_used;
    uint32_t    overflow;       /* set when the table, the dump or the arena ran out */
    uint32_t    grow;           /* set when the table wants to grow: nused reached
                                 * soft_cap, a dump entry was taken or the arena
                                 * passed half of its bytes */
    uint64_t    soft_cap;       /* entries at which growth is requested */
    char       *dump;           /* entries (global form) of groups created while the
                                 * table had no room, or nullptr */
    uint64_t    dump_cap;
    uint64_t    dump_used;
} xb_gtable;

/* execution statistics and error state, one per launch (device) */
typedef struct xb_status {
    uint32_t    errcode;
    int32_t     lineno;
    uint32_t    msg_id;
    uint32_t    __pad;
    uint64_t    nitems_raw;
    uint64_t    nitems_in;
    uint64_t    nitems_out;
    uint64_t    nitems_depth[XB_MAX_DEPTH + 1];
    uint32_t    stopped;        /* warps stopped claiming work for the group table to grow */
    uint32_t    left_n;         /* leftover ranges they recorded */
    uint32_t    left_next;      /* resume launch: next leftover range to take */
    uint32_t    replay_left;    /* replay: records left for after the table grows */
    uint64_t    __pad1[2];
    /* work distribution counter, alone in its 128-byte line: every warp's
     * claim lands here, away from the error word every warp polls */
    uint64_t    unit_cursor;
    uint64_t    __pad2[15];
    /* projection output: proj_need counts the row index and tuple bytes
     * of every claim, including those past the end of kds_dst (so that
     * the host learns the size needed); proj_usage / proj_nitems place
     * only the claims that fit */
    uint64_t    proj_need;
    uint64_t    proj_usage;
    uint32_t    proj_nitems;
    uint32_t    proj_overflow;
    uint64_t    __pad3[13];
} xb_status;

/* error message ids reported by device code */
#define XB_MSG_NONE             0
#define XB_MSG_INT_RANGE        1
#define XB_MSG_DIV_ZERO         2
#define XB_MSG_FLT_RANGE        3
#define XB_MSG_NUMERIC_RANGE    4
#define XB_MSG_NUMERIC_CORRUPT  5
#define XB_MSG_VARLENA_EXTERNAL 6
#define XB_MSG_BAD_TUPLE        7
#define XB_MSG_GTABLE_FULL      8
#define XB_MSG_WAIT_TIMEOUT     9
#define XB_MSG_ARENA_FULL       10
#define XB_MSG_BAD_PAGE         11
#define XB_MSG_ARROW_TYPE       12
#define XB_MSG_NUMERIC_TYPE     13
#define XB_MSG_LEFT_FULL        14

#endif  /* XB_PLAN_H */
