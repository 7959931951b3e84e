/*
 * pgstrom_abi.h
 *
 * Wire/device ABI shared with PG-Strom's host side: the kern_data_store
 * (KDS) chunk formats, PostgreSQL heap page / tuple / varlena layout, the
 * kern_expression bytecode, kern_session_info, kern_multirels, the
 * XpuCommand request frame and the partial-aggregation state records.
 *
 * Every struct below must be byte-for-byte identical to the corresponding
 * definition in the reference (PG-Strom 6.2, src/xpu_common.h and
 * src/cuda_common.h), because these buffers are produced by PG-Strom's
 * planner/executor (codegen.c, executor.c, relscan.c, gpu_join.c) and read
 * back by PostgreSQL (aggfuncs.c).  The layouts are restated here in plain
 * C; tests/test_abi.py checks sizeof/offsetof of each struct against a
 * table generated from the reference headers.
 *
 * Pointer-typed fields that the reference fills in on the GPU-service side
 * (kern_expression.expr_ops / fn_dptr, kern_varslot_desc.vs_ops,
 * kern_multirels.chunks[].kds_in / kbuf_parts) are declared as opaque
 * 64-bit slots: this implementation never dereferences them.
 */
#ifndef PGSTROM_ABI_H
#define PGSTROM_ABI_H
#include <stddef.h>
#include <stdint.h>
#include <stdbool.h>

#ifdef __cplusplus
extern "C" {
#endif

/* ---------------------------------------------------------------
 * fundamental constants (xpu_common.h:170-205)
 * --------------------------------------------------------------- */
#define PGSTROM_BLCKSZ          8192
#define PGSTROM_NAMEDATALEN     64
#define PGSTROM_MAXALIGN(x)     (((uint64_t)(x) + 7) & ~((uint64_t)7))
#define PGSTROM_TYPEALIGN(a,x)  (((uint64_t)(x) + ((a) - 1)) & ~((uint64_t)((a) - 1)))
#define PGSTROM_CHUNK_SIZE      (65534UL << 10)   /* pg_strom.h:701 */

typedef uint32_t Oid_t;

#if defined(__CUDACC__)
#define PGSTROM_INLINE  static inline __host__ __device__
#else
#define PGSTROM_INLINE  static inline
#endif

/* ---------------------------------------------------------------
 * error reporting (xpu_common.h:441-457)
 * --------------------------------------------------------------- */
#define ERRCODE_STROM_SUCCESS       0
#define ERRCODE_SUSPEND_FALLBACK    'f'
#define ERRCODE_SUSPEND_NO_SPACE    'd'
#define ERRCODE_DEVICE_ERROR        'E'
#define ERRCODE_DEVICE_FATAL        'F'
#define ERRCODE_IS_SUSPEND(x)       ((x) >= 'a' && (x) <= 'z')

#define KERN_ERRORBUF_FILENAME_LEN  32
#define KERN_ERRORBUF_FUNCNAME_LEN  64
#define KERN_ERRORBUF_MESSAGE_LEN   200
typedef struct {
    uint32_t    errcode;
    int32_t     lineno;
    char        filename[KERN_ERRORBUF_FILENAME_LEN + 1];
    char        funcname[KERN_ERRORBUF_FUNCNAME_LEN + 1];
    char        message[KERN_ERRORBUF_MESSAGE_LEN + 1];
} kern_errorbuf;

/* ---------------------------------------------------------------
 * Arrow type options (arrow_defs.h:445-479)
 * --------------------------------------------------------------- */
#define ArrowType__Null             1
#define ArrowType__Int              2
#define ArrowType__FloatingPoint    3
#define ArrowType__Binary           4
#define ArrowType__Utf8             5
#define ArrowType__Bool             6
#define ArrowType__Decimal          7
#define ArrowType__Date             8
#define ArrowType__Time             9
#define ArrowType__Timestamp        10
#define ArrowType__LargeUtf8        20
#define ArrowPrecision__Half        0
#define ArrowPrecision__Single      1
#define ArrowPrecision__Double      2
#define ArrowDateUnit__Day          0
#define ArrowDateUnit__MilliSecond  1

typedef struct {
    int32_t     tag;            /* ArrowTypeTag */
    int16_t     unitsz;
    uint16_t    align;
    union {
        struct { uint16_t bitWidth; uint8_t is_signed; } integer;
        struct { int32_t precision; } floating_point;
        struct { uint16_t precision; uint16_t scale; uint16_t bitWidth; } decimal;
        struct { int32_t unit; } date;
        struct { int32_t unit; } time;
        struct { int32_t unit; } timestamp;
        struct { int32_t unit; } interval;
        struct { uint32_t byteWidth; } fixed_size_binary;
    } u;
} ArrowTypeOptions;

/* ---------------------------------------------------------------
 * kern_colmeta / kern_data_store (xpu_common.h:661-851)
 * --------------------------------------------------------------- */
#define TYPE_KIND__NULL         'n'
#define TYPE_KIND__BASE         'b'

typedef struct kern_colmeta {
    bool        attbyval;
    int8_t      attalign;
    int16_t     attlen;
    int16_t     attnum;
    int16_t     attcacheoff;
    Oid_t       atttypid;
    int32_t     atttypmod;
    int8_t      atttypkind;
    char        kds_format;
    int16_t     dtype_sizeof;
    uint32_t    kds_offset;
    uint16_t    idx_subattrs;
    uint16_t    num_subattrs;
    char        attname[PGSTROM_NAMEDATALEN];
    ArrowTypeOptions attopts;
    int32_t     field_index;
    int64_t     virtual_offset;
    uint64_t    nullmap_offset;
    uint64_t    nullmap_length;
    uint64_t    values_offset;
    uint64_t    values_length;
    uint64_t    extra_offset;
    uint64_t    extra_length;
} kern_colmeta;

#define KDS_FORMAT_ROW          'r'
#define KDS_FORMAT_HASH         'h'
#define KDS_FORMAT_BLOCK        'b'
#define KDS_FORMAT_COLUMN       'c'
#define KDS_FORMAT_ARROW        'a'
#define KDS_FORMAT_FALLBACK     'f'

typedef struct kern_data_store {
    uint64_t    length;
    uint64_t    usage;
    uint32_t    nitems;
    uint32_t    ncols;
    char        format;
    bool        has_varlena;
    bool        tdhasoid;
    Oid_t       tdtypeid;
    int32_t     tdtypmod;
    Oid_t       table_oid;
    uint32_t    hash_nslots;
    uint32_t    block_offset;
    uint32_t    block_nloaded;
    uint32_t    column_nrooms;
    uint32_t    arrow_virtual_usage;
    uint32_t    parquet_row_group;
    bool        parquet_parallel_load;
    bool        parquet_cache_enabled;
    uint32_t    nr_colmeta;
    kern_colmeta colmeta[1];
} kern_data_store;

PGSTROM_INLINE uint64_t KDS_HEAD_LENGTH(const kern_data_store *kds)
{
    return PGSTROM_MAXALIGN(offsetof(kern_data_store, colmeta) +
                            sizeof(kern_colmeta) * kds->nr_colmeta);
}

/* hash-slot width of KDS_FORMAT_HASH (xpu_common.h:1388-1396) */
PGSTROM_INLINE uint64_t KDS_GET_HASHSLOT_WIDTH(uint64_t nitems)
{
    if (nitems <= 5000)
        return 20000UL;
    if (nitems <= 4000000)
        return 20000UL + 2 * nitems;
    return 8020000UL + nitems;
}

/* ---------------------------------------------------------------
 * PostgreSQL heap page / tuple layout (xpu_common.h:925-1128)
 * --------------------------------------------------------------- */
typedef struct {
    struct { uint16_t bi_hi; uint16_t bi_lo; } ip_blkid;
    uint16_t    ip_posid;
} ItemPointerData;

typedef struct HeapTupleHeaderData {
    union {
        struct { uint32_t t_xmin; uint32_t t_xmax; uint32_t t_field3; } t_heap;
        struct { int32_t datum_len_; int32_t datum_typmod; Oid_t datum_typeid; } t_datum;
    } t_choice;
    ItemPointerData t_ctid;
    uint16_t    t_infomask2;
    uint16_t    t_infomask;
    uint8_t     t_hoff;
    uint8_t     t_bits[1];
} HeapTupleHeaderData;

#define HEAP_HASNULL            0x0001
#define HEAP_HASVARWIDTH        0x0002
#define HEAP_HASEXTERNAL        0x0004
#define HEAP_XMIN_COMMITTED     0x0100
#define HEAP_XMIN_INVALID       0x0200
#define HEAP_XMAX_INVALID       0x0800
#define HEAP_NATTS_MASK         0x07FF
#define SizeofHeapTupleHeader   23

typedef uint32_t ItemIdData;        /* lp_off:15, lp_flags:2, lp_len:15 */
#define ITEMID_OFF(x)           ((x) & 0x7fffU)
#define ITEMID_FLAGS(x)         (((x) >> 15) & 0x3U)
#define ITEMID_LEN(x)           (((x) >> 17) & 0x7fffU)
#define ITEMID_MAKE(off,flags,len) \
    ((uint32_t)(off) | ((uint32_t)(flags) << 15) | ((uint32_t)(len) << 17))
#define LP_UNUSED   0
#define LP_NORMAL   1
#define LP_REDIRECT 2
#define LP_DEAD     3

typedef struct PageHeaderData {
    uint32_t    pd_parent_blkno;    /* pd_lsn in PostgreSQL proper */
    uint32_t    pd_parent_item;
    uint16_t    pd_checksum;
    uint16_t    pd_flags;
    uint16_t    pd_lower;
    uint16_t    pd_upper;
    uint16_t    pd_special;
    uint16_t    pd_pagesize_version;
    uint32_t    pd_prune_xid;
    ItemIdData  pd_linp[1];
} PageHeaderData;
#define SizeOfPageHeaderData    24
#define PD_ALL_VISIBLE          0x0004

/* ---------------------------------------------------------------
 * KDS items (xpu_common.h:1175-1258)
 * --------------------------------------------------------------- */
typedef struct kern_tupitem {
    uint32_t    t_len;
    uint32_t    hash;
    uint8_t     has_xact_attrs;
    uint8_t     __padding__;
    uint16_t    t_infomask2;
    uint16_t    t_infomask;
    uint8_t     t_hoff;
    uint8_t     t_bits[1];
} kern_tupitem;
/* distance between a HeapTupleHeader's t_infomask2 and kern_tupitem's */
#define MINIMAL_TUPLE_OFFSET    (18 - 10)
#define ROWID_SIZE              4

typedef struct kern_hashitem {
    uint64_t    next;
    kern_tupitem t __attribute__((aligned(8)));
} kern_hashitem;

/* ---------------------------------------------------------------
 * varlena (xpu_common.h:1641-1826)
 * --------------------------------------------------------------- */
#define VARHDRSZ                4
#define VARATT_IS_1B(p)         ((((const uint8_t *)(p))[0] & 0x01) == 0x01)
#define VARATT_IS_1B_E(p)       ((((const uint8_t *)(p))[0]) == 0x01)
#define VARATT_IS_4B_U(p)       ((((const uint8_t *)(p))[0] & 0x03) == 0x00)
#define VARATT_IS_4B_C(p)       ((((const uint8_t *)(p))[0] & 0x03) == 0x02)
#define VARATT_NOT_PAD_BYTE(p)  (*((const uint8_t *)(p)) != 0)
#define VARSIZE_1B(p)           ((((const uint8_t *)(p))[0] >> 1) & 0x7F)

/* ---------------------------------------------------------------
 * partial aggregation (xpu_common.h:2328-2471)
 * --------------------------------------------------------------- */
#define KAGG_ACTION__VREF           101
#define KAGG_ACTION__VREF_NOKEY     102
#define KAGG_ACTION__NROWS_ANY      201
#define KAGG_ACTION__NROWS_COND     202
#define KAGG_ACTION__PMIN_INT32     302
#define KAGG_ACTION__PMIN_INT64     303
#define KAGG_ACTION__PMIN_FP64      304
#define KAGG_ACTION__PMAX_INT32     402
#define KAGG_ACTION__PMAX_INT64     403
#define KAGG_ACTION__PMAX_FP64      404
#define KAGG_ACTION__PSUM_INT       501
#define KAGG_ACTION__PSUM_INT64     502
#define KAGG_ACTION__PSUM_FP        503
#define KAGG_ACTION__PSUM_NUMERIC   504
#define KAGG_ACTION__PAVG_INT       601
#define KAGG_ACTION__PAVG_INT64     602
#define KAGG_ACTION__PAVG_FP        603
#define KAGG_ACTION__PAVG_NUMERIC   604
#define KAGG_ACTION__STDDEV         701
#define KAGG_ACTION__COVAR          801

#define PAGG_MINMAX_ATTRS__VALID    0x0001
#define PAGG_NUMERIC_ATTRS__WEIGHT  0x00ffffU
#define PAGG_NUMERIC_ATTRS__NAN     0x010000U
#define PAGG_NUMERIC_ATTRS__PINF    0x020000U
#define PAGG_NUMERIC_ATTRS__NINF    0x040000U

typedef struct { uint64_t u64_lo; uint64_t u64_hi; } int128_packed_t;

typedef struct { int32_t vl_len_; uint32_t attrs; int64_t value; } kagg_state__pminmax_int64_packed;
typedef struct { int32_t vl_len_; uint32_t attrs; double value; }  kagg_state__pminmax_fp64_packed;
typedef struct { int32_t vl_len_; uint32_t attrs; int64_t nitems; int64_t sum; } kagg_state__psum_int_packed;
typedef struct { int32_t vl_len_; uint32_t attrs; int64_t nitems; double sum; }  kagg_state__psum_fp_packed;
typedef struct { int32_t vl_len_; uint32_t attrs; uint64_t nitems; int128_packed_t sum; } kagg_state__psum_numeric_packed;
typedef struct { int32_t vl_len_; uint32_t attrs; int64_t nitems; double sum_x; double sum_x2; } kagg_state__stddev_packed;
typedef struct { int32_t vl_len_; uint32_t attrs; int64_t nitems;
                 double sum_x; double sum_xx; double sum_y; double sum_yy; double sum_xy; } kagg_state__covar_packed;

typedef struct {
    uint16_t    action;
    int16_t     arg0_slot_id;
    int16_t     arg1_slot_id;
    int16_t     filter_slot_id;
    int32_t     typmod;
} kern_aggregate_desc;

/* GPU-Sort key descriptors (xpu_common.h:2474-2520) */
#define KSORT_KEY_KIND__VREF                0
#define KSORT_KEY_KIND__PMINMAX_INT64       1
#define KSORT_KEY_KIND__PMINMAX_FP64        2
#define KSORT_KEY_KIND__PSUM_INT64          3
#define KSORT_KEY_KIND__PSUM_FP64           4
#define KSORT_KEY_KIND__PSUM_NUMERIC        5
#define KSORT_KEY_KIND__PAVG_INT64          6
#define KSORT_KEY_KIND__PAVG_FP64           7
#define KSORT_KEY_KIND__PAVG_NUMERIC        8
#define KSORT_KEY_KIND__PVARIANCE_SAMP      9
#define KSORT_KEY_KIND__PVARIANCE_POP       10
#define KSORT_KEY_KIND__PCOVAR_CORR         11
#define KSORT_KEY_KIND__PCOVAR_SAMP         12
#define KSORT_KEY_KIND__PCOVAR_POP          13
#define KSORT_KEY_KIND__PCOVAR_AVGX         14
#define KSORT_KEY_KIND__PCOVAR_AVGY         15
#define KSORT_KEY_KIND__PCOVAR_COUNT        16
#define KSORT_KEY_KIND__NITEMS              23
#define KSORT_WINDOW_FUNC__ROW_NUMBER       'n'
#define KSORT_WINDOW_FUNC__RANK             'r'
#define KSORT_WINDOW_FUNC__DENSE_RANK       'd'

typedef struct {
    uint16_t    kind;               /* KSORT_KEY_KIND__* */
    int8_t      nulls_first;
    int8_t      order_asc;
    uint16_t    src_anum;           /* attribute of the kds_final tuple */
    uint16_t    buf_offset;
    int32_t     key_type_code;      /* TypeOpCode */
    uint64_t    key_ops;            /* device pointer slot, unused here */
} kern_sortkey_desc;

/* ---------------------------------------------------------------
 * kern_expression bytecode (xpu_common.h:2507-2723)
 * --------------------------------------------------------------- */
typedef struct { int16_t vl_resno; int16_t vl_slot_id; } kern_varload_desc;
typedef struct { int32_t vm_offset; int16_t vm_slot_id; bool vm_from_xdatum; } kern_varmove_desc;

typedef struct kern_varslot_desc {
    int32_t     vs_type_code;       /* TypeOpCode */
    bool        vs_typbyval;
    int8_t      vs_typalign;
    int16_t     vs_typlen;
    int32_t     vs_typmod;
    int32_t     vs_offset;
    uint16_t    idx_subfield;
    uint16_t    num_subfield;
    uint64_t    vs_ops;             /* device pointer slot, unused here */
} kern_varslot_desc;

#define KERN_EXPRESSION_MAGIC       0x4b657870U
#define KEXP_FLAG__IS_PUSHED_DOWN   0x0001U
#define SPECIAL_DEPTH__PREAGG_FINAL (-2)

typedef struct kern_expression {
    uint32_t    len;
    int32_t     exptype;            /* TypeOpCode */
    uint64_t    expr_ops;           /* device pointer slot, unused here */
    uint32_t    expflags;
    int32_t     opcode;             /* FuncOpCode */
    uint64_t    fn_dptr;            /* device pointer slot, unused here */
    uint32_t    nr_args;
    uint32_t    args_offset;
    union {
        char    data[1] __attribute__((aligned(8)));
        struct {
            Oid_t   const_type;
            bool    const_isnull;
            char    const_value[1] __attribute__((aligned(8)));
        } c;
        struct { uint32_t param_id; char __data[1]; } p;
        struct { int32_t var_offset; uint16_t var_slot_id; char __data[1]; } v;
        struct { uint16_t sv_slot_id; char data[1] __attribute__((aligned(8))); } save;
        struct { int32_t depth; int32_t nitems; kern_varload_desc desc[1]; } load;
        struct { int32_t depth; int32_t nitems; kern_varmove_desc desc[1]; } move;
        struct { int32_t nattrs; kern_aggregate_desc desc[1]; } pagg;
        struct { uint32_t hash; int32_t nattrs; uint16_t slot_id[1]; } proj;
        struct { uint32_t npacked; uint32_t offset[1]; } pack;
        struct { uint32_t case_comp; uint32_t case_else; char data[1] __attribute__((aligned(8))); } casewhen;
        struct { uint16_t elem_slot_id; char data[1] __attribute__((aligned(8))); } saop;
        struct {
            uint64_t    elem_ops;
            int32_t     elem_type;
            uint32_t    nslots;
            uint32_t    default_offset;
            char        __padding[4];
            uint32_t    hslots[1] __attribute__((aligned(8)));
        } haop;
        struct {
            uint32_t    gist_oid;
            int16_t     gist_depth;
            uint16_t    htup_slot_id;
            int32_t     htup_offset;
            kern_varload_desc ivar_desc;
            char        data[1] __attribute__((aligned(8)));
        } gist;
        struct {
            int32_t     nkeys;
            bool        needs_finalization;
            char        window_rank_func;
            uint32_t    window_rank_limit;
            uint16_t    window_partby_nkeys;
            uint16_t    window_orderby_nkeys;
            kern_sortkey_desc desc[1];
        } sort;
    } u;
} kern_expression;

#define KEXP_HEADSZ             offsetof(kern_expression, u)
#define KEXP_MAGIC_OF(exptype, opcode) \
    (KERN_EXPRESSION_MAGIC ^ ((uint32_t)(exptype) << 6) ^ ((uint32_t)(opcode) << 14))

/* ---------------------------------------------------------------
 * session / commands (xpu_common.h:2762-2919)
 * --------------------------------------------------------------- */
#define DEVKIND__NVIDIA_GPU         0x00000001U
#define DEVTASK__MERGE_FINAL_BUFFER 0x00020000U
#define DEVTASK__SCAN               0x10000000U
#define DEVTASK__JOIN               0x20000000U
#define DEVTASK__PREAGG             0x40000000U

#define XpuCommandTag__Success          0
#define XpuCommandTag__Error            1
#define XpuCommandTag__SuccessHalfWay   2
#define XpuCommandTag__OpenSession      100
#define XpuCommandTag__XpuTaskExec      110
#define XpuCommandTag__XpuTaskFinal     119
#define XpuCommandMagicNumber           0xdeadbeafU

typedef struct kern_session_info {
    uint64_t    query_plan_id;
    uint32_t    kcxt_kvars_nrooms;
    uint32_t    kcxt_kvars_nslots;
    uint32_t    kcxt_kvars_defs;
    uint32_t    kcxt_kvecs_bufsz;
    uint32_t    kcxt_kvecs_ndims;
    uint32_t    kcxt_extra_bufsz;
    uint32_t    cuda_stack_size;
    uint32_t    xpu_task_flags;
    int64_t     optimal_gpus;
    uint32_t    xpucode_load_vars_packed;
    uint32_t    xpucode_move_vars_packed;
    uint32_t    xpucode_scan_quals;
    uint32_t    xpucode_join_quals_packed;
    uint32_t    xpucode_hash_values_packed;
    uint32_t    xpucode_gist_evals_packed;
    uint32_t    xpucode_projection;
    uint32_t    xpucode_groupby_keyhash;
    uint32_t    xpucode_groupby_keyload;
    uint32_t    xpucode_groupby_keycomp;
    uint32_t    xpucode_groupby_actions;
    uint32_t    xpucode_gpusort_keydesc;
    int64_t     hostEpochTimestamp;
    uint32_t    session_xact_state;
    uint32_t    session_timezone;
    uint32_t    session_encode;
    int32_t     session_currency_frac_digits;
    uint64_t    pinned_inner_buffer_partition_size;
    uint32_t    projection_kds_dst;
    uint32_t    select_into_pathname;
    uint32_t    select_into_kds_head;
    uint32_t    select_into_projdesc;
    uint32_t    pgsql_port_number;
    uint32_t    pgsql_plan_node_id;
    uint32_t    join_inner_handle;
    uint32_t    groupby_kds_final;
    uint32_t    groupby_prepfn_bufsz;
    float       groupby_ngroups_estimation;
    uint32_t    gpusort_htup_margin;
    int32_t     gpusort_limit_count;
    uint32_t    fallback_kds_head;
    uint32_t    fallback_desc_defs;
    uint32_t    fallback_desc_nitems;
    uint32_t    nparams;
    uint32_t    poffset[1];
} kern_session_info;

typedef struct {
    int32_t     scan_relidx;
    uint32_t    kds_src_pathname;
    uint32_t    kds_src_iovec;
    uint32_t    kds_src_offset;
    char        data[1] __attribute__((aligned(8)));
} kern_exec_task;

typedef struct {
    int32_t     scan_relidx;
    uint32_t    chunks_offset;
    uint32_t    chunks_nitems;
    uint32_t    ojmap_offset;
    uint32_t    ojmap_length;
    bool        right_outer_join;
    bool        final_plan_task;
    uint32_t    final_nitems;
    uint64_t    final_usage;
    uint64_t    final_total;
    uint32_t    final_sorting_msec;
    uint32_t    final_reconstruction_msec;
    uint32_t    join_reconstruction_msec;
    uint32_t    select_into_nblocks;
    uint32_t    npages_direct_read;
    uint32_t    npages_vfs_read;
    uint32_t    nchunks_parquet_read;
    uint32_t    ncaches_parquet_load;
    uint32_t    nitems_raw;
    uint32_t    nitems_in;
    uint32_t    nitems_out;
    uint32_t    num_rels;
    struct {
        uint32_t nitems_roj;
        uint32_t nitems_gist;
        uint32_t nitems_out;
    } stats[1];
} kern_exec_results;

typedef struct { void *prev; void *next; } pgstrom_dlist_node;

typedef struct {
    uint32_t    magic;
    uint32_t    tag;
    uint64_t    length;
    void       *priv;
    pgstrom_dlist_node chain;
    union {
        kern_errorbuf       error;
        kern_session_info   session;
        kern_exec_task      task;
        kern_exec_results   results;
        struct {
            kern_errorbuf   error;
            uint32_t        npages_direct_read;
            uint32_t        npages_vfs_read;
            kern_data_store kds_src;
        } fallback;
    } u;
} XpuCommand;

/* ---------------------------------------------------------------
 * inner relations for GpuJoin (xpu_common.h:3494-3516)
 * --------------------------------------------------------------- */
typedef struct kern_multirels {
    uint64_t    length;
    uint64_t    ojmap_sz;
    uint64_t    kbuf_part_offset;
    uint32_t    num_inner_rels;
    struct {
        uint64_t    kds_in;         /* device pointer slot, unused here */
        uint64_t    kbuf_parts;     /* device pointer slot, unused here */
        uint64_t    kds_offset;
        uint64_t    ojmap_offset;
        uint64_t    gist_offset;
        int16_t     gist_ctid_resno;
        bool        is_nestloop;
        bool        left_outer;
        bool        right_outer;
        bool        pinned_buffer;
        uint64_t    buffer_id;
    } chunks[1];
} kern_multirels;

#ifdef __cplusplus
}
#endif
#include "pgstrom_opcodes.h"
#endif  /* PGSTROM_ABI_H */
