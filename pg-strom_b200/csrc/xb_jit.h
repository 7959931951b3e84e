/*
 * xb_jit.h
 *
 * Session-specialised executor kernels: source generation from a translated
 * session (xb_plan), NVRTC compilation for sm_100a and launch through the
 * driver API.  See xb_jit.cpp.
 */
#ifndef XB_JIT_H
#define XB_JIT_H
#include <stddef.h>
#include <stdint.h>
#include "xb_plan.h"

#define XBJ_WARPS_PER_CTA       8   /* 256-thread CTAs (XB_BLOCK) */
#define XBJ_MIN_BLOCKS_DEFAULT  4   /* resident CTAs of 256 threads per SM (measured best for the join and Arrow workloads) */

#ifdef __cplusplus
extern "C" {
#endif

/* bytes between the entries of a specialised kernel's shared group table */
uint32_t xb_jit_sm_stride(uint32_t gent_size);

/* shared memory the specialised kernel of 'format' adds for staging
 * heap pages (0: pages are read in place; XPU_B200_JIT_STAGE=1 enables) */
size_t xb_jit_stage_bytes(uint32_t format);

/* the generated CUDA source (for inspection); *p_len = its length */
int xb_jit_source(const xb_plan *plan, uint32_t format, char *buf, size_t bufsz, size_t *p_len);

/* build (or find in the process-wide cache) the kernels of plan + format
 * on device dindex: *p_func the per-launch kernel (xbj_kernel), *p_mixfn
 * (if not NULL) the mixed-launch kernel (xbj_mixed_kernel, parameter block
 * XbMixArgs); both CUfunctions */
int xb_jit_compile(const xb_plan *plan, uint32_t format, int dindex,
                   void **p_func, void **p_mixfn, double *p_compile_ms, char *errbuf, size_t errlen);

/* xb_jit_compile for kernels bounded to min_blocks resident CTAs of 256
 * threads per SM (1..8; 0: the default) */
int xb_jit_compile_minb(const xb_plan *plan, uint32_t format, int dindex, int min_blocks,
                        void **p_func, void **p_mixfn, void **p_replay, double *p_compile_ms,
                        char *errbuf, size_t errlen);

/* the kernels of plan + format if the process-wide cache has them
 * already: 0 found, 1 not built yet, -1 not buildable */
int xb_jit_lookup_minb(const xb_plan *plan, uint32_t format, int dindex, int min_blocks,
                       void **p_func, void **p_mixfn, void **p_replay);

/* build the kernels of plan + format on a background thread (the plan is
 * copied); returns a job handle or NULL.  xb_jit_job_poll: 1 while
 * building, 0 built (outputs filled), -1 failed (errbuf says why).  A job
 * released before it finished still completes into the cache. */
void *xb_jit_build_async(const xb_plan *plan, uint32_t format, int dindex, int min_blocks);
int   xb_jit_job_poll(void *job, void **p_func, void **p_mixfn, void **p_replay, double *p_compile_ms,
                      char *errbuf, size_t errlen);
void  xb_jit_job_release(void *job);

/* bytes of one deferred-row record of partitioned aggregation for plan
 * and source format (0: its kernel does not defer group updates); the replay kernel is
 * xbj_replay (parameter block XbReplayArgs), returned by
 * xb_jit_compile_minb's p_replay */
uint32_t xb_jit_part_rec_size(const xb_plan *plan, uint32_t format);

/* a key naming the plan shape of plan + format: sessions whose specialised
 * kernels differ only in their launch bounds share it */
uint64_t xb_jit_shape_key(const xb_plan *plan, uint32_t format);

/* compile only (no device needed): cubin size and NVRTC milliseconds */
int xb_jit_check(const xb_plan *plan, uint32_t format, uint64_t *p_cubin_bytes, double *p_compile_ms,
                 char *errbuf, size_t errlen);

/* allow 'smem' bytes of dynamic shared memory; resident CTAs per SM */
int xb_jit_prepare(void *func, int block, size_t smem, int *p_per_sm);

/* bytes of static shared memory of a kernel (0 when unknown) */
size_t xb_jit_static_smem(void *func);

/* resident CTAs per SM with 'smem' bytes (the limit already allowed) */
int xb_jit_occupancy(void *func, int block, size_t smem, int *p_per_sm);

/* launch with one kernel parameter block ('args' points to XbExecArgs,
 * or to XbMixArgs for the mixed-launch kernel) */
int xb_jit_launch(void *func, int grid, int block, size_t smem, void *stream, void *args);

#ifdef __cplusplus
}
#endif
#endif  /* XB_JIT_H */
