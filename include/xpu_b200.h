/*
 * xpu_b200.h
 *
 * C ABI of the B200-native GpuScan / GpuJoin / GpuPreAgg executor.
 *
 * PG-Strom's GPU service (src/gpu_service.c) receives three XpuCommands from
 * PostgreSQL backends and, for each XpuTaskExec, launches kern_gpujoin_main
 * (src/cuda_gpujoin.cu:1050).  This library is the drop-in replacement for
 * everything below that socket: the service keeps its protocol handling and
 * calls these entry points instead of cuLaunchKernel.  All structs crossing
 * the boundary are the reference's own wire formats (pgstrom_abi.h); no
 * C++ or torch type appears here.
 *
 * Conventions (kept from the reference):
 *   - a non-zero return value is one of ERRCODE_* ('E', 'F', 'd', 'f') and
 *     *err is filled like kern_errorbuf in gpuClientELog;
 *   - the session blob and inner buffer are copied by the callee
 *     (gpu_service.c:3363-3371); kds_src belongs to the caller;
 *   - one session may be used from several threads; calls on the same
 *     session are serialised internally.
 */
#ifndef XPU_B200_H
#define XPU_B200_H
#include <stddef.h>
#include <stdint.h>
#include "pgstrom_abi.h"

#ifdef __cplusplus
extern "C" {
#endif

typedef struct xpuB200Device  xpuB200Device;
typedef struct xpuB200Session xpuB200Session;

/*
 * Attach GPU 'cuda_dindex' and reserve bookkeeping for up to hbm_budget
 * bytes of device memory (0 = 90% of free memory).
 * Replaces gpuservSetupGpuContext / gpuservSetupGpuModule
 * (gpu_service.c:6463, :6231-6319).  No runtime compilation: the kernels
 * are built into this library for sm_100a.
 */
int  xpuB200Init(int cuda_dindex, uint64_t hbm_budget,
                 xpuB200Device **p_dev, kern_errorbuf *err);
void xpuB200Shutdown(xpuB200Device *dev);

/*
 * Open a query session: validate and translate the session bytecode,
 * upload the inner relations of a GpuJoin (kmrels may be NULL) and build
 * their device hash indexes, and allocate the GROUP BY final buffer.
 * Replaces gpuservHandleOpenSession (gpu_service.c:3320-3410) together
 * with __setupGpuQueryJoinInnerBuffer (:2198-2354) and the kds_final
 * allocation of getGpuQueryBuffer (:2357-2412).
 */
int  xpuB200OpenSession(xpuB200Device *dev,
                        const kern_session_info *session, uint64_t session_sz,
                        const kern_multirels *kmrels, uint64_t kmrels_sz,
                        xpuB200Session **p_sess, kern_errorbuf *err);

/*
 * Execute one chunk (KDS_FORMAT_BLOCK heap pages, KDS_FORMAT_ARROW, or
 * KDS_FORMAT_ROW).  kds_src is a host pointer unless kds_src_on_device is
 * non-zero, in which case it is a device pointer on this GPU.  Statistics
 * (nitems_raw / nitems_in / nitems_out / stats[]) are written to *results
 * when results is not NULL; results->num_rels must give the capacity of
 * results->stats[].  Pre-aggregated groups stay on the device until
 * xpuB200Final.
 * Replaces gpuservHandleGpuTaskExec / __gpuservLaunchGpuTaskExecKernel
 * (gpu_service.c:4006-4290, :3760-4003).
 */
int  xpuB200ExecTask(xpuB200Session *sess,
                     const kern_data_store *kds_src, int kds_src_on_device,
                     kern_exec_results *results, kern_errorbuf *err);

/*
 * Execute one chunk of a session whose bytecode projects rows
 * (kern_session_info.xpucode_projection without GROUP BY): every row that
 * passes the scan quals and the joins is formed as a kern_tupitem and
 * written into kds_dst, a KDS_FORMAT_ROW buffer of dst_sz bytes laid out
 * like the session's projection_kds_dst header (row index after the
 * header, tuples packed from the end).  kds_dst is a host pointer unless
 * kds_dst_on_device is non-zero (then a device pointer on this GPU, 8-byte
 * aligned).  *p_required receives the bytes the chunk's rows need.  If they
 * do not fit, ERRCODE_SUSPEND_NO_SPACE is returned, kds_dst's header is not
 * written (a host kds_dst is not touched at all) and the caller runs the
 * chunk again with a buffer of *p_required bytes; the statistics of that
 * failed run are not accumulated.
 * Replaces the kds_dst allocation of gpuservHandleGpuTaskExec
 * (gpu_service.c:4158-4176) together with the projection step of the
 * kernels (execGpuJoinProjection, cuda_gpujoin.cu:753-900) and the
 * NO_SPACE write-back of
 * __gpuservLaunchGpuTaskExecKernel (gpu_service.c:3894-3908).
 */
int  xpuB200ExecTaskDst(xpuB200Session *sess,
                        const kern_data_store *kds_src, int kds_src_on_device,
                        void *kds_dst, uint64_t dst_sz, int kds_dst_on_device,
                        uint64_t *p_required,
                        kern_exec_results *results, kern_errorbuf *err);

/*
 * Materialise the final buffer in the reference's KDS_FORMAT_HASH layout
 * (kern_hashitem tuples with kagg_state__* partial states), as read by
 * pgstromScanNextTuple (executor.c:861-883) and finalised by aggfuncs.c.
 * If buf_sz is smaller than the result, nothing is copied, *p_required is
 * set and ERRCODE_SUSPEND_NO_SPACE is returned.
 * Replaces gpuservHandleGpuTaskFinal (gpu_service.c:5685-5882).
 */
int  xpuB200Final(xpuB200Session *sess, void *kds_final_buf, uint64_t buf_sz,
                  uint64_t *p_required, kern_exec_results *results,
                  kern_errorbuf *err);

/*
 * xpuB200Final for callers that cannot allocate GPU memory: a service that
 * reserved the device's memory at start-up and sub-allocates its own pool,
 * or one that must not call cudaMalloc / cudaFree while other sessions run
 * (cudaFree waits for the whole device).  No counterpart in the reference:
 * its GPU service allocates kds_final itself.
 *
 * kds_final is written in the same layout as xpuB200Final's, but into
 * kds_final_dev, memory the caller owns on the session's GPU (device
 * memory, managed memory or mapped pinned host memory), of buf_sz bytes.
 * With kds_final_dev NULL and buf_sz 0 only *p_required is set.  Nothing is
 * allocated: the work arrays live in one fixed 8 MiB array per GPU,
 * enough for a session whose group table has up to 262,144 slots (tables
 * are powers of two; about 65,000 groups at the default sizing).  Larger
 * tables are rejected with ERRCODE_DEVICE_ERROR and a message saying so
 * (use xpuB200Final for them).
 *
 * The first call on each GPU looks up the array's device address; make
 * that first call before capturing any stream.  All calls in a process
 * for one GPU share that GPU's array: they are serialised by a lock per
 * GPU and each returns after its GPU work has finished.  Work that
 * overlapped on the GPU would race on the shared array.
 */
int  xpuB200FinalNoAlloc(xpuB200Session *sess, void *kds_final_dev, uint64_t buf_sz,
                         uint64_t *p_required, kern_exec_results *results, kern_errorbuf *err);

/*
 * Merge another GPU's (or session's) partial-aggregation result into this
 * session's group table, so that a following xpuB200Final returns the
 * groups of both.  kds_final is a KDS_FORMAT_HASH buffer that xpuB200Final
 * (or xpuB200FinalNoAlloc) of a session with the same GROUP BY program
 * wrote: every group tuple is decoded, its keys looked up (or inserted) by
 * the tuple's hash and its partial states added into the matching entry
 * with the same reduction operations the chunk launches use.
 * kds_final_on_device != 0: kds_final is device memory readable by this
 * session's GPU (its own memory, or a peer's with peer access enabled);
 * otherwise it is host memory that is copied in first.
 * Replaces the secondary-buffer merge of __gpuservHandleGpuPreAggFinal
 * (gpu_service.c:5442-5518) that launches kern_gpupreagg_final_merge
 * (cuda_gpupreagg.cu:2329-2432).
 */
int  xpuB200MergeFinal(xpuB200Session *sess, const kern_data_store *kds_final,
                       int kds_final_on_device, kern_errorbuf *err);

/*
 * The session's groups as nparts hash partitions, for the exchange step of
 * a multi-GPU pre-aggregation whose groups are too many to gather on one
 * GPU: part p holds the groups whose hash % nparts == p, each a
 * KDS_FORMAT_HASH kds_final of its own in xpuB200Final's layout.  The parts
 * are written back to back into parts_dev, device memory of the session's
 * GPU that the caller owns (cudaMalloc'd, so that it can be shared with
 * the other GPUs by CUDA IPC, or sent by NCCL), of buf_sz bytes; part p
 * starts at part_offsets[p] (256-byte aligned; nparts + 1 entries, the last
 * one the total).  With parts_dev NULL and buf_sz 0 only the offsets and
 * *p_required are set.  GPU r then merges part r of every GPU into a fresh
 * session with xpuB200MergeFinal(kds_final_on_device = 1), reading it in
 * place from the peer's memory over NVLink, so that every group ends on
 * exactly one GPU.  No counterpart in the reference, which merges every
 * GPU's kds_final into the first GPU's (__gpuservHandleGpuPreAggFinal,
 * gpu_service.c:5442-5518).
 */
int  xpuB200FinalParts(xpuB200Session *sess, uint32_t nparts, void *parts_dev, uint64_t buf_sz,
                       uint64_t *part_offsets, uint64_t *p_required, kern_errorbuf *err);

void xpuB200CloseSession(xpuB200Session *sess);

/*
 * Serving form: asynchronous chunk commands with continuous batching.
 * xpuB200Submit queues one chunk command of a session (kds_src a host
 * pointer, or a device pointer when kds_src_on_device; a host chunk must
 * stay valid until its ticket is polled done) and returns a ticket.  The
 * device keeps up to 4 launches in flight on their own streams: whenever
 * one is free (checked on every Submit and Poll) the queued commands are
 * admitted in arrival order while their staging bytes fit the admission
 * budget; a command of at least alone_units units (heap pages or 1024-row
 * groups; default 256) runs alone on its session's specialised kernel, the
 * smaller ones run together in one mixed launch.  xpuB200Poll reports
 * whether a ticket is done (waiting for it when wait is non-zero) and then
 * returns its statistics in *results, or its error; a ticket is reported
 * done once.  Groups accumulate in the session as with xpuB200ExecTask;
 * xpuB200Final and xpuB200CloseSession first wait for the session's
 * submitted commands.  xpuB200ServeConfig sets the admission budget in
 * bytes and alone_units (0 keeps a value).  The default budget,
 * XPU_B200_ADMIT_FREE_HBM, admits by the device's free memory: a launch is
 * admitted while the staging bytes of its commands fit the GPU's free HBM
 * (cudaMemGetInfo, plus the slot's own reusable staging buffer) less a
 * reserve of 1 GiB or 5% of the device, whichever is larger; any other
 * value is a fixed budget for the staging bytes in flight.  A command is
 * always admitted when nothing else is in flight.  xpuB200MemInfo reports
 * the free and total device memory and the reserve, for a service loop
 * that admits whole queries (OpenSession) by free HBM.  Replaces the
 * per-command worker threads of gpuservGpuWorkerMain
 * (gpu_service.c:5951-5964) with one scheduler per GPU, and the device
 * memory accounting of the GPU service's memory pool
 * (gpu_service.c:6757-6817).
 */
#define XPU_B200_ADMIT_FREE_HBM     UINT64_MAX
int  xpuB200Submit(xpuB200Session *sess, const kern_data_store *kds_src, int kds_src_on_device,
                   uint64_t *p_ticket, kern_errorbuf *err);
int  xpuB200Poll(xpuB200Device *dev, uint64_t ticket, int wait, int *p_done,
                 kern_exec_results *results, kern_errorbuf *err);
int  xpuB200ServeConfig(xpuB200Device *dev, uint64_t admit_bytes, uint32_t alone_units,
                        kern_errorbuf *err);
int  xpuB200MemInfo(xpuB200Device *dev, uint64_t *p_free, uint64_t *p_total, uint64_t *p_reserve);

/*
 * Mixed batches (the batched form of many sessions' XpuTaskExec): chunk
 * commands of different sessions, each a device-resident chunk of its own
 * session, run together in one persistent kernel fed from a device work
 * queue.  CTAs are sent to commands largest first, several to a large one;
 * each claims the command's units dynamically, runs the command's own
 * bytecode against its own group table, and moves on.  Sessions of one
 * plan shape (bytecode equal up to constants) share one specialised
 * kernel; the batch runs one persistent launch per kernel (the
 * interpreter's for the rest), concurrently.  A run is captured once as a
 * CUDA graph (status reset, the launches, status read-back) and replayed by
 * every xpuB200MixExec / xpuB200MixTime.  xpuB200MixInfo reports the
 * launches of a run and how many commands run specialised code.
 * xpuB200MixExec fills results[i] and errs[i] per command (either array
 * may be NULL) and returns 0, or the first command error.  Each command's
 * groups accumulate in its session, as with xpuB200ExecTask.  No
 * counterpart in the reference, whose service launches one kernel per
 * command (__gpuservLaunchGpuTaskExecKernel, gpu_service.c:3760-4003).
 */
typedef struct xpuB200Mix xpuB200Mix;
int  xpuB200MixCreate(xpuB200Device *dev, uint32_t ncmds, xpuB200Session *const *sess,
                      const kern_data_store *const *kds_dev, xpuB200Mix **p_mix,
                      kern_errorbuf *err);
int  xpuB200MixExec(xpuB200Mix *mix, kern_exec_results *const *results, kern_errorbuf *errs);
int  xpuB200MixTime(xpuB200Mix *mix, int niters, double *p_msec, kern_errorbuf *err);
int  xpuB200MixInfo(const xpuB200Mix *mix, uint64_t *p_bytes, uint64_t *p_units,
                    uint32_t *p_items, uint32_t *p_launches, uint32_t *p_specialised);
void xpuB200MixDestroy(xpuB200Mix *mix);

/*
 * Whole-command entry point for a service loop: handles the three command
 * tags gpuservGpuWorkerMain dispatches (gpu_service.c:5951-5964):
 *   XpuCommandTag__OpenSession  -> *p_sess is created (kmrels may be NULL)
 *   XpuCommandTag__XpuTaskExec  -> kds_src at xcmd->u.task.kds_src_offset
 *   XpuCommandTag__XpuTaskFinal -> resp carries results + kds_final
 * The response (XpuCommandTag__Success / __Error) is written into resp
 * (capacity resp_sz bytes); returns 0 or an ERRCODE_*.
 */
int  xpuB200HandleCommand(xpuB200Device *dev, xpuB200Session **p_sess,
                          const XpuCommand *xcmd,
                          const kern_multirels *kmrels, uint64_t kmrels_sz,
                          XpuCommand *resp, uint64_t resp_sz);

/*
 * Prepared batches (the batched form of XpuTaskExec): many device-resident
 * chunks of one session, validated once, executed by ONE persistent kernel
 * launch whose warps claim work units (heap pages / 1024-row groups) from a
 * device queue spanning all chunks.  The reference issues one
 * kern_gpujoin_main launch plus a stream synchronisation per 64 MB chunk
 * (gpu_service.c:3934-3948); a batch replaces those with a single launch.
 * All chunks must share the session's column layout and KDS format.
 */
typedef struct xpuB200Batch xpuB200Batch;
int  xpuB200BatchCreate(xpuB200Session *sess, const kern_data_store *const *kds_dev,
                        uint32_t nchunks, xpuB200Batch **p_batch, kern_errorbuf *err);
int  xpuB200BatchExec(xpuB200Batch *batch, kern_exec_results *results, kern_errorbuf *err);
/* runs the batch niters times; average kernel milliseconds (CUDA events on
 * the session stream) in *p_msec */
int  xpuB200BatchTime(xpuB200Batch *batch, int niters, double *p_msec, kern_errorbuf *err);
/*
 * Autotuning of the session's launch shape on the batch's chunks: the
 * resident CTAs per SM the session-specialised kernel is built for (2, 3, 4,
 * 6, 8; each a separately compiled kernel) and then the capacity of the
 * per-CTA shared-memory group table (the default, twice it, none), each
 * measured with CUDA events on a fresh group table.  The fastest shape is
 * kept by the session and remembered for this GPU: later sessions of the
 * same plan shape and default table capacity (every chunk command of one
 * query template) adopt it at their first launch; sessions of the same plan
 * shape with another default capacity (other group-count estimates, as in
 * a mixed batch) adopt its CTA bound.  Call it before the session executes chunks (otherwise
 * ERRCODE_DEVICE_ERROR); the group table is empty again on return.  flags
 * must be 0.  report (if not NULL) receives a JSON text with every measured
 * shape.  Join partition fan-out is not a parameter: inner relations are
 * kept whole (direct-address tables or one hash index) in HBM/L2.
 * No counterpart in the reference (its launch shape comes from
 * gpuOptimalBlockSize, gpu_service.c:3797-3810, over the
 * occupancy calculation of gpu_device.c:1121).
 */
int  xpuB200BatchTune(xpuB200Batch *batch, uint32_t flags, char *report, size_t report_len,
                      kern_errorbuf *err);
void xpuB200BatchDestroy(xpuB200Batch *batch);

/*
 * Pinned inner buffers: rows that a scan projected into a KDS_FORMAT_HASH
 * kds_dst (a session whose Projection carries a hash value, u.proj.hash)
 * are appended into one KDS_FORMAT_HASH buffer on the device and chained
 * into its hash slots, ready to be the inner relation of a join.  Both
 * buffers are device memory of this GPU.  kds_dst: a KDS_FORMAT_HASH
 * header with its length, hash_nslots, nitems and usage (0 and 0 when
 * empty; every call appends), the hash slots zeroed before the first call.
 * kds_src: KDS_FORMAT_HASH or KDS_FORMAT_ROW whose tuples carry their
 * hash, with the same columns.  hash_divisor >= 2 appends only the rows
 * with hash % hash_divisor == hash_remainder (one partition of the inner
 * relation, for a join whose inner side is split across GPUs); 0 appends
 * every row.  *p_required (if not NULL) receives the bytes kds_dst's rows
 * take; when they do not fit, ERRCODE_SUSPEND_NO_SPACE is returned and
 * kds_dst must be rebuilt larger.  Row order is not deterministic (rows
 * are claimed concurrently), as in the reference.
 * Replaces kern_buffer_reconstruction (cuda_gpujoin.cu:18-71) and
 * kern_buffer_partitioning (cuda_gpujoin.cu:76-138), launched by the GPU
 * service's pinned inner-buffer setup (gpu_service.c:1748-2197).
 */
/*
 * Inner relations resident across sessions.  A session whose
 * kern_session_info.join_inner_handle is not 0 keeps the inner relations
 * it uploaded and indexed (kern_multirels) on the device under that handle:
 * a later session with the same handle and the same build inputs (the
 * translated inner descriptors and the join quals evaluated at the build,
 * constants included) uses them as they are, with no upload and no build.
 * The caller guarantees that one handle always names the same
 * kern_multirels contents, as the reference's join_inner_handle names one
 * inner buffer shared by the sessions of a query (gpu_service.c:2357-2412).
 * Built relations stay after their last session closes while the cache
 * holds at most max_bytes (default 16 GiB; least recently used first out).
 * max_bytes == UINT64_MAX only reads *p_cached_bytes (the bytes held now).
 */
int  xpuB200InnerCacheConfig(xpuB200Device *dev, uint64_t max_bytes, uint64_t *p_cached_bytes,
                             kern_errorbuf *err);

/*
 * Outer-table chunks resident in HBM across sessions: the device-side
 * copy of a table that GPU-Cache keeps (src/gpu_cache.c), and the chunks
 * relscan.c / Arrow_Fdw would otherwise read and send for every query.
 * xpuB200ChunkCachePut places chunk chunk_no of table table_handle on the
 * device (from host memory, or device memory with kds_on_device; heap
 * pages 16-byte aligned), or finds it there, and returns its device
 * address in *p_kds_dev for ExecTask / Submit / batches with
 * kds_src_on_device; xpuB200ChunkCacheGet only finds (1: not resident).
 * Both pin the chunk until xpuB200ChunkCacheRelease; unpinned chunks stay
 * while the cache holds at most max_bytes (xpuB200ChunkCacheConfig,
 * default 64 GiB; least recently used first out; UINT64_MAX only reads
 * *p_cached_bytes).  The caller guarantees that one (table_handle,
 * chunk_no) always names the same contents.
 */
int  xpuB200ChunkCachePut(xpuB200Device *dev, uint64_t table_handle, uint32_t chunk_no,
                          const kern_data_store *kds, int kds_on_device,
                          const kern_data_store **p_kds_dev, kern_errorbuf *err);
int  xpuB200ChunkCacheGet(xpuB200Device *dev, uint64_t table_handle, uint32_t chunk_no,
                          const kern_data_store **p_kds_dev);
int  xpuB200ChunkCacheRelease(xpuB200Device *dev, const kern_data_store *kds_dev);
int  xpuB200ChunkCacheConfig(xpuB200Device *dev, uint64_t max_bytes, uint64_t *p_cached_bytes,
                             kern_errorbuf *err);

/*
 * Storage → HBM chunk ingest (GPUDirect Storage).  Replaces the file read
 * of the GPU service before a KDS_FORMAT_BLOCK / KDS_FORMAT_ARROW chunk is
 * run (__gpuservLoadKdsCommon, src/gpu_service.c:3415-3466, calling
 * gpuDirectFileReadIOV, src/extra.c:569-630, with the I/O vector of
 * strom_io_chunk entries, src/heterodb_extra.h:37-43).  The first
 * base_offset bytes of kds_head (the KDS header and block numbers) are
 * copied to kds_dev; then, for each I/O chunk, nr_pages pages of
 * XPU_B200_IO_PAGE bytes starting at file page fchunk_id are read from
 * 'pathname' into kds_dev + base_offset + m_offset (the reference places
 * kds_dev so that kds_dev + base_offset is page aligned, the alignment
 * direct DMA wants; any 16-byte alignment is accepted here).  With
 * try_direct, and with XPU_B200_CUFILE=1 in the environment (on hosts
 * without the nvidia-fs driver a cuFile read was seen never to return, so
 * the library does not enter libcufile unless the host says it may), pages
 * are read by cuFileRead (libcufile, bound at run time); the pages cuFile does not
 * read, and all pages without try_direct or without a working cuFile
 * driver, go through a pinned bounce buffer.  *p_npages_direct and
 * *p_npages_vfs count the two (the reference's npages_direct_read /
 * npages_vfs_read).  Synchronous; kds_dev is device memory of 'dev'.
 */
#define XPU_B200_IO_PAGE            4096
typedef struct {
    uint64_t    m_offset;       /* destination offset from kds_dev + base_offset */
    uint32_t    fchunk_id;      /* first file page (of XPU_B200_IO_PAGE bytes) */
    uint32_t    nr_pages;       /* pages to read */
} xpuB200IoChunk;

int  xpuB200ChunkReadDirect(xpuB200Device *dev, const char *pathname,
                            const kern_data_store *kds_head, uint64_t base_offset,
                            const xpuB200IoChunk *ioc, uint32_t nr_chunks,
                            void *kds_dev, uint64_t kds_dev_sz, int try_direct,
                            uint32_t *p_npages_direct, uint32_t *p_npages_vfs, kern_errorbuf *err);

int  xpuB200InnerRebuild(xpuB200Device *dev, kern_data_store *kds_dst, const kern_data_store *kds_src,
                         uint32_t hash_divisor, uint32_t hash_remainder, uint64_t *p_required,
                         kern_errorbuf *err);

/* Device memory helpers for callers that keep chunks resident in HBM. */
int  xpuB200DeviceAlloc(xpuB200Device *dev, uint64_t sz, void **p_dptr);
int  xpuB200DeviceFree(xpuB200Device *dev, void *dptr);
int  xpuB200CopyToDevice(xpuB200Device *dev, void *dptr, const void *src, uint64_t sz);
int  xpuB200CopyToHost(xpuB200Device *dev, void *dst, const void *dptr, uint64_t sz);

/*
 * Time one ExecTask over a device-resident chunk 'niters' times with CUDA
 * events on the session's stream (no host synchronisation inside the timed
 * region other than at its end); returns the average kernel milliseconds
 * in *p_msec.  Used by the benchmark to report the kernel roofline.
 */
int  xpuB200TimeExecTask(xpuB200Session *sess, const kern_data_store *kds_src_dev,
                         int niters, double *p_msec, kern_errorbuf *err);

/* Diagnostics: translated plan summary and host-side hash self test. */
int  xpuB200SessionInfo(xpuB200Session *sess, char *buf, uint64_t buf_sz);
uint32_t xpuB200HashBytes(const void *data, uint32_t len);

#ifdef __cplusplus
}
#endif
#endif  /* XPU_B200_H */
