/*
 * Prints sizeof/offsetof of every ABI struct field this implementation
 * relies on.  Compiled twice: with -DUSE_REFERENCE against PG-Strom's
 * src/xpu_common.h + src/cuda_common.h (by oracle/gen_abi_golden.sh, which
 * writes tests/golden/abi_layout.txt), and without it against
 * include/pgstrom_abi.h (by tests/test_abi.py).  Both outputs must match.
 */
#include <stdio.h>
#include <stddef.h>
#ifdef USE_REFERENCE
#define CUDA_MAXTHREADS_PER_BLOCK 512
#include "xpu_common.h"
typedef ItemIdData ItemIdData_t;
#else
#include "pgstrom_abi.h"
#endif

#define S(T)    printf("sizeof %s %zu\n", #T, sizeof(T))
#define O(T,F)  printf("offsetof %s.%s %zu\n", #T, #F, offsetof(T,F))

int main(void)
{
    S(kern_errorbuf); O(kern_errorbuf, lineno); O(kern_errorbuf, filename);
    O(kern_errorbuf, funcname); O(kern_errorbuf, message);
    S(ArrowTypeOptions);
    S(kern_colmeta);
    O(kern_colmeta, attbyval); O(kern_colmeta, attalign); O(kern_colmeta, attlen);
    O(kern_colmeta, attnum); O(kern_colmeta, attcacheoff); O(kern_colmeta, atttypid);
    O(kern_colmeta, atttypmod); O(kern_colmeta, atttypkind); O(kern_colmeta, kds_format);
    O(kern_colmeta, dtype_sizeof); O(kern_colmeta, kds_offset); O(kern_colmeta, idx_subattrs);
    O(kern_colmeta, num_subattrs); O(kern_colmeta, attname); O(kern_colmeta, attopts);
    O(kern_colmeta, field_index); O(kern_colmeta, virtual_offset); O(kern_colmeta, nullmap_offset);
    O(kern_colmeta, nullmap_length); O(kern_colmeta, values_offset); O(kern_colmeta, values_length);
    O(kern_colmeta, extra_offset); O(kern_colmeta, extra_length);
    S(kern_data_store);
    O(kern_data_store, length); O(kern_data_store, usage); O(kern_data_store, nitems);
    O(kern_data_store, ncols); O(kern_data_store, format); O(kern_data_store, has_varlena);
    O(kern_data_store, tdhasoid); O(kern_data_store, tdtypeid); O(kern_data_store, tdtypmod);
    O(kern_data_store, table_oid); O(kern_data_store, hash_nslots); O(kern_data_store, block_offset);
    O(kern_data_store, block_nloaded); O(kern_data_store, column_nrooms);
    O(kern_data_store, arrow_virtual_usage); O(kern_data_store, parquet_row_group);
    O(kern_data_store, nr_colmeta); O(kern_data_store, colmeta);
    S(HeapTupleHeaderData); O(HeapTupleHeaderData, t_ctid); O(HeapTupleHeaderData, t_infomask2);
    O(HeapTupleHeaderData, t_infomask); O(HeapTupleHeaderData, t_hoff); O(HeapTupleHeaderData, t_bits);
    S(PageHeaderData); O(PageHeaderData, pd_flags); O(PageHeaderData, pd_lower);
    O(PageHeaderData, pd_upper); O(PageHeaderData, pd_special); O(PageHeaderData, pd_linp);
    S(kern_tupitem); O(kern_tupitem, hash); O(kern_tupitem, has_xact_attrs);
    O(kern_tupitem, t_infomask2); O(kern_tupitem, t_infomask); O(kern_tupitem, t_hoff);
    O(kern_tupitem, t_bits);
    S(kern_hashitem); O(kern_hashitem, t);
    S(kagg_state__pminmax_int64_packed); S(kagg_state__pminmax_fp64_packed);
    S(kagg_state__psum_int_packed); S(kagg_state__psum_fp_packed);
    S(kagg_state__psum_numeric_packed); O(kagg_state__psum_numeric_packed, sum);
    S(kagg_state__stddev_packed); S(kagg_state__covar_packed);
    S(kern_aggregate_desc); O(kern_aggregate_desc, typmod);
    S(kern_varload_desc); S(kern_varmove_desc); O(kern_varmove_desc, vm_from_xdatum);
    S(kern_varslot_desc); O(kern_varslot_desc, vs_offset); O(kern_varslot_desc, vs_ops);
    S(kern_expression);
    O(kern_expression, exptype); O(kern_expression, expr_ops); O(kern_expression, expflags);
    O(kern_expression, opcode); O(kern_expression, fn_dptr); O(kern_expression, nr_args);
    O(kern_expression, args_offset); O(kern_expression, u);
    O(kern_expression, u.c.const_isnull); O(kern_expression, u.c.const_value);
    O(kern_expression, u.v.var_slot_id); O(kern_expression, u.save.data);
    O(kern_expression, u.load.nitems); O(kern_expression, u.load.desc);
    O(kern_expression, u.move.desc); O(kern_expression, u.pagg.desc);
    O(kern_expression, u.pack.offset);
    S(kern_session_info);
    O(kern_session_info, kcxt_kvars_nrooms); O(kern_session_info, kcxt_kvars_defs);
    O(kern_session_info, kcxt_kvecs_bufsz); O(kern_session_info, xpu_task_flags);
    O(kern_session_info, optimal_gpus); O(kern_session_info, xpucode_load_vars_packed);
    O(kern_session_info, xpucode_scan_quals); O(kern_session_info, xpucode_join_quals_packed);
    O(kern_session_info, xpucode_hash_values_packed); O(kern_session_info, xpucode_projection);
    O(kern_session_info, xpucode_groupby_keyhash); O(kern_session_info, xpucode_groupby_keyload);
    O(kern_session_info, xpucode_groupby_keycomp); O(kern_session_info, xpucode_groupby_actions);
    O(kern_session_info, hostEpochTimestamp); O(kern_session_info, session_encode);
    O(kern_session_info, pinned_inner_buffer_partition_size);
    O(kern_session_info, projection_kds_dst); O(kern_session_info, join_inner_handle);
    O(kern_session_info, groupby_kds_final); O(kern_session_info, groupby_prepfn_bufsz);
    O(kern_session_info, groupby_ngroups_estimation); O(kern_session_info, gpusort_htup_margin);
    O(kern_session_info, fallback_kds_head); O(kern_session_info, nparams);
    O(kern_session_info, poffset);
    S(kern_exec_task); O(kern_exec_task, kds_src_offset); O(kern_exec_task, data);
    S(kern_exec_results); O(kern_exec_results, final_nitems); O(kern_exec_results, final_usage);
    O(kern_exec_results, nitems_raw); O(kern_exec_results, num_rels); O(kern_exec_results, stats);
    S(XpuCommand); O(XpuCommand, tag); O(XpuCommand, length); O(XpuCommand, u);
    S(kern_multirels); O(kern_multirels, num_inner_rels); O(kern_multirels, chunks);
    O(kern_multirels, chunks[0].kds_offset); O(kern_multirels, chunks[0].gist_ctid_resno);
    O(kern_multirels, chunks[0].is_nestloop); O(kern_multirels, chunks[0].buffer_id);
    O(kern_multirels, chunks[1]);
    return 0;
}
