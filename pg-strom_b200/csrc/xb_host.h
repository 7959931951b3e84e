/*
 * xb_host.h
 *
 * Host-side state of the C ABI, shared by the library's translation units:
 * the device and session objects, the tuner's cache, the error helpers, and
 * the functions of the core (xb_exec.cu: kernels, sessions, ExecTask,
 * Final, growth) that the services call -- xb_batch.cu (prepared and mixed
 * batches, launch-shape tuning) and xb_serve.cu (serving scheduler, device
 * memory helpers, resident chunk cache).  Internal; the public interface is
 * include/xpu_b200.h.
 */
#ifndef XB_HOST_H
#define XB_HOST_H

#include <cuda_runtime.h>
#include <map>
#include <mutex>
#include <string>
#include <tuple>
#include <vector>
#include <cstring>
#include "xb_plan.h"
#include "xb_exec_dev.cuh"
#include "xb_compile.h"
#include "xb_jit.h"
#include "xpu_b200.h"

struct xpuB200Device {
    int             dindex;
    int             nsm;
    uint64_t        hbm_budget;
    size_t          smem_optin;     /* dynamic shared memory a CTA may opt in to */
    cudaStream_t    stream;
    struct xb_sched *sched = nullptr; /* asynchronous commands (created by the first submit) */
    /* recycled per-session resources: creating a stream or pinning host
     * memory costs far more than a query's own host work */
    std::mutex      pool_lock;
    std::vector<cudaStream_t> free_streams;
    std::vector<xb_status *> free_status;
    std::vector<xb_status *> status_blocks;
    /* inner relations built for sessions with a join_inner_handle, kept
     * while sessions use them and, within inner_budget bytes, after */
    std::mutex      inner_lock;
    std::vector<struct xb_inner_entry *> inner_cache;
    uint64_t        inner_budget = 16ULL << 30;
    uint64_t        inner_bytes = 0;
    uint64_t        inner_clock = 0;
    /* outer-table chunks resident across sessions (xpuB200ChunkCache*) */
    std::mutex      chunk_lock;
    std::map<std::pair<uint64_t, uint32_t>, struct xb_chunk_entry> chunk_cache;
    uint64_t        chunk_budget = 64ULL << 30;
    uint64_t        chunk_bytes = 0;
    uint64_t        chunk_clock = 0;
};

/* one resident chunk: the device copy of a caller's chunk, placed so that
 * heap pages start 16-byte aligned; refs counts the callers using it */
struct xb_chunk_entry {
    char           *base = nullptr;
    const kern_data_store *kds = nullptr;
    uint64_t        bytes = 0;
    uint32_t        refs = 0;
    uint64_t        last_use = 0;
};

/* one cached set of inner relations: the built descriptors (with their
 * device memory) of every depth */
struct xb_inner_entry {
    uint64_t        key;
    uint32_t        nrels;
    xb_inner        inner[XB_MAX_DEPTH + 1];
    uint32_t        gid_cap;        /* shared table slots the group ids need (0: none) */
    std::vector<void *> allocs;
    uint64_t        bytes = 0;
    uint32_t        refs = 0;
    uint64_t        last_use = 0;
};

struct xb_sched;

struct xpuB200Session {
    xpuB200Device  *dev;
    cudaStream_t    stream = nullptr;
    std::mutex      lock;
    std::vector<char> h_session;
    char           *d_session = nullptr;
    char           *d_kmrels = nullptr;
    xb_plan        *h_plan = nullptr;
    xb_plan        *d_plan = nullptr;
    std::vector<void *> d_allocs;
    std::vector<uint64_t> d_alloc_sz;
    xb_inner_entry *inner_entry = nullptr;  /* cached inner relations in use */
    bool            inner_hit = false;      /* found built by an earlier session */
    xb_gtable       h_gt = {};
    xb_gtable      *d_gt = nullptr;
    xb_status      *d_status = nullptr;
    xb_status      *h_status = nullptr;     /* pinned */
    char           *d_src = nullptr;
    uint64_t        d_src_cap = 0;
    xb_task        *d_tasks = nullptr;      /* work queue of single-chunk launches */
    uint32_t        d_tasks_cap = 0;
    uint32_t        sm_cap = 0;
    uint32_t        warp_bytes = 0;
    uint32_t        plan_bytes = 0;
    size_t          smem_bytes = 0;
    int             grid = 0;
    uint64_t        total_raw = 0, total_in = 0, total_out = 0;
    uint64_t        total_depth[XB_MAX_DEPTH + 1] = {0};
    cudaEvent_t     ev0, ev1;
    /* partitioned aggregation: the last such launch's scan and replay,
     * bracketed on the session stream (diagnostics, xpuB200SessionInfo) */
    cudaEvent_t     ev_part[3] = {nullptr, nullptr, nullptr};
    /* session-specialised kernels, per source format (index: KDS format) */
    bool            jit_enabled = true;
    bool            jit_tried[256] = {false};
    void           *jit_fn[256] = {nullptr};
    void           *jit_mixfn[256] = {nullptr};    /* its mixed-launch kernel */
    void           *jit_job[256] = {nullptr};      /* a background build of it, pending */
    char            ran_kind[256] = {0};   /* 'j' / 'v': kernel last launched per format */
    uint32_t        sched_refs = 0;        /* submitted commands not yet finished */
    /* device projection: staging buffer for host kds_dst, and the buffer of
     * the launch in progress */
    char           *d_dst = nullptr;
    uint64_t        d_dst_cap = 0;
    char           *launch_dst = nullptr;
    uint64_t        launch_dst_len = 0;
    int             jit_grid[256] = {0};
    size_t          jit_smem = 0;           /* without page staging */
    size_t          jit_smem_fmt[256] = {0}; /* per format, with its page staging */
    double          jit_compile_ms = 0.0;
    std::string     jit_msg;
    /* launch shape: resident CTAs per SM the specialised kernels are built
     * for (0: default) and the shared group table's default capacity, as
     * tuned by xpuB200BatchTune or adopted from its process-wide cache */
    int             jit_minb = 0;
    uint32_t        sm_cap_default = 0;
    bool            tune_looked_up = false;
    /* partitioned aggregation: deferred rows bucketed by table slot */
    void           *jit_replay[256] = {nullptr};
    int             jit_replay_grid[256] = {0};
    char           *part_buf = nullptr;
    uint32_t       *part_cnt = nullptr;
    uint64_t        part_bytes = 0;
    uint32_t        part_cap = 0;
    uint32_t        part_shift = 0;
    uint32_t        nparts = 0;
    uint32_t        part_rec = 0;
    bool            part_used = false;
    bool            in_batch = false;       /* a prepared batch's launch is being issued */
    /* group-table growth: where stopped warps record their leftover work
     * (two lists: a resume launch reads one and records into the other),
     * and the launch xb_run is issuing */
    XbLeft         *d_left[2] = {nullptr, nullptr};
    uint32_t        left_cap = 0;
    bool            run_growth = false;
    bool            run_resume = false;
    uint32_t        run_left_sel = 0;
    uint32_t        run_left_in_n = 0;
    uint64_t        run_static_base0 = 0;
    uint64_t        run_cursor0 = 0;
    uint32_t        grow_count = 0;         /* times the group table grew */
};

/* launch-shape tuning: the choices measured per plan shape (xpuB200BatchTune),
 * adopted by later sessions of the shape */
struct xb_tune_choice {
    int         minb;
    uint32_t    sm_cap;
};
extern std::mutex g_tune_lock;
/* per (GPU, plan shape, default table capacity) */
extern std::map<std::tuple<int, uint64_t, uint32_t>, xb_tune_choice> g_tune;
/* per plan shape alone: the CTA bound last tuned for it, adopted by
 * sessions whose default table capacity was not tuned (another group-count
 * estimate) */
extern std::map<std::pair<int, uint64_t>, int> g_tune_minb;

/* errors: the reference's ERRCODE_* with a filled kern_errorbuf */
#define XB_ERR(err, code, ...) xb_set_error((err), (code), __func__, __LINE__, __VA_ARGS__)
/* a CUDA call's result as 0 or a filled ERRCODE_DEVICE_FATAL */
#define xb_set_cuda(call_rc, err) xb_cuda_rc((call_rc), (err), __func__, __LINE__)
#define XB_CUDA(call, err) do {                                               \
        cudaError_t __rc = (call);                                            \
        if (__rc != cudaSuccess)                                              \
            return XB_ERR((err), ERRCODE_DEVICE_FATAL, "%s: %s", #call,       \
                          cudaGetErrorString(__rc));                          \
    } while (0)

static inline void xb_clear_error(kern_errorbuf *err)
{
    if (err) memset(err, 0, sizeof(*err));
}

/* the core's functions the services call (xb_exec.cu) */
void xb_account_status(xpuB200Session *s, const xb_status *hs, kern_exec_results *results);
int xb_check_kds(const kern_data_store *kds, kern_errorbuf *err);
uint32_t xb_chunk_units(const kern_data_store *head);
void xb_fill_results(const xb_status *hs, uint32_t nrels, kern_exec_results *results);
cudaStream_t xb_get_stream(xpuB200Device *dev);
void xb_inner_evict_locked(xpuB200Device *dev);
int xb_launch_on(xpuB200Session *s, const xb_task *d_tasks, uint32_t ntasks, uint64_t nunits, uint32_t format,
                 cudaStream_t stream, xb_status *d_status, kern_errorbuf *err);
const char *xb_msg_text(uint32_t id);
void xb_note_layout(xpuB200Session *s, const kern_data_store *h);
void xb_put_stream(xpuB200Device *dev, cudaStream_t st);
int xb_run(xpuB200Session *s, const xb_task *d_tasks, uint32_t ntasks, uint64_t nunits,
           uint32_t format, kern_exec_results *results, kern_errorbuf *err, bool timed = false);
void *xb_session_jit(xpuB200Session *s, uint32_t format, bool wait = true);
int xb_set_error(kern_errorbuf *err, uint32_t code, const char *func, int line, const char *fmt, ...);
int xb_cuda_rc(cudaError_t rc, kern_errorbuf *err, const char *func, int line);
int xb_set_sm_cap(xpuB200Session *s, uint32_t cap);
std::tuple<int, uint64_t, uint32_t> xb_tune_key(xpuB200Session *s, uint32_t format);

/* the group table's host side (xb_exec.cu), which the final stage
 * (xb_final.cu) also drives: read its header, grow it, settle the groups
 * waiting in its dump, wait for the session's launch and read its status */
int xb_gt_read(xpuB200Session *s, xb_gtable *g, kern_errorbuf *err);
int xb_gt_grow(xpuB200Session *s, uint64_t min_entries, kern_errorbuf *err);
int xb_gt_settle(xpuB200Session *s, kern_errorbuf *err);
int xb_wait_status(xpuB200Session *s, kern_errorbuf *err);

/* mixed launches (xb_batch.cu), which the serving scheduler also issues:
 * the commands grouped by the kernel they run on, one launch per group */
struct xb_mix_group {
    void           *jfn = nullptr;  /* xbj_mixed_kernel, or nullptr: xb_mixed_kernel */
    std::vector<uint32_t> cmds;     /* command indexes */
    std::vector<uint32_t> items;    /* work queue: command index per item */
    size_t          smem = 0;
    int             grid = 0;
};
void *xb_mix_kernel_of(xpuB200Session *s, uint32_t format, bool wait = true);
int xb_mix_plan(xpuB200Device *dev, const std::vector<xpuB200Session *> &sess,
                const std::vector<uint32_t> &formats, const std::vector<uint64_t> &units,
                std::vector<xb_mix_group> &groups, kern_errorbuf *err, bool wait = true);
int xb_mix_launch(const xb_mix_group &g, const XbMixArgs &ma, cudaStream_t stream, kern_errorbuf *err);

/* the scheduler's, which the core calls (xb_serve.cu) */
void xb_sched_drain_session(xpuB200Session *s);
void xb_sched_destroy(xpuB200Device *dev);

/* the interpreting kernel of mixed launches (xb_exec.cu) */
__global__ void __launch_bounds__(XB_BLOCK, XB_MIN_BLOCKS) xb_mixed_kernel(const __grid_constant__ XbMixArgs m);

#endif  /* XB_HOST_H */
