/*
 * xb_batch.cu
 *
 * Prepared batches (many device-resident chunks of one session in one
 * persistent launch, xpuB200Batch*), launch-shape tuning of the
 * specialised kernels (xpuB200BatchTune) and mixed batches (chunk commands
 * of many sessions in one launch per plan shape, replayed from a CUDA
 * graph, xpuB200Mix*).  The reference issues one launch and one stream
 * synchronisation per 64 MB chunk (__gpuservLaunchGpuTaskExecKernel,
 * gpu_service.c:3760-4003); these calls are this library's batched forms
 * of the same ExecTask.
 */
#include <cuda_runtime.h>
#include <algorithm>
#include <map>
#include <mutex>
#include <string>
#include <tuple>
#include <vector>
#include <cstdio>
#include <cstring>
#include "xb_host.h"

/* ----------------------------------------------------------------
 * prepared batches: many device-resident chunks in one persistent launch
 * ---------------------------------------------------------------- */
struct xpuB200Batch {
    xpuB200Session *sess;
    xb_task        *d_tasks;
    uint32_t        ntasks;
    uint64_t        nunits;
    uint32_t        format;
    uint64_t        bytes;          /* sum of chunk lengths */
    uint64_t        rows;           /* rows (ARROW/ROW) or pages (BLOCK) */
};

extern "C" int
xpuB200BatchCreate(xpuB200Session *s, const kern_data_store *const *kds_dev, uint32_t nchunks,
                   xpuB200Batch **p_batch, kern_errorbuf *err)
{
    xb_clear_error(err);
    *p_batch = nullptr;
    if (!s || !kds_dev || nchunks == 0)
        return XB_ERR(err, ERRCODE_DEVICE_ERROR, "invalid batch arguments");
    std::lock_guard<std::mutex> g(s->lock);
    if (s->h_plan->has_proj)
        return XB_ERR(err, ERRCODE_DEVICE_ERROR,
                      "the session projects rows into kds_dst: use xpuB200ExecTaskDst");
    XB_CUDA(cudaSetDevice(s->dev->dindex), err);
    std::vector<xb_task> tasks(nchunks);
    std::vector<char> first_head;
    uint64_t base = 0, bytes = 0, rows = 0;
    uint32_t format = 0;
    for (uint32_t i = 0; i < nchunks; i++) {
        kern_data_store head;
        if (((uintptr_t)kds_dev[i] & 7) != 0)
            return XB_ERR(err, ERRCODE_DEVICE_ERROR, "chunk %u is not 8-byte aligned", i);
        XB_CUDA(cudaMemcpy(&head, kds_dev[i], offsetof(kern_data_store, colmeta), cudaMemcpyDeviceToHost), err);
        std::vector<char> hb(KDS_HEAD_LENGTH(&head));
        XB_CUDA(cudaMemcpy(hb.data(), kds_dev[i], hb.size(), cudaMemcpyDeviceToHost), err);
        const kern_data_store *h = (const kern_data_store *)hb.data();
        int rc = xb_check_kds(h, err);
        if (rc) return rc;
        if (i == 0) {
            first_head = hb;
            format = (uint32_t)h->format;
            xb_note_layout(s, h);
        } else {
            /* one launch decodes every chunk with the same column layout */
            const kern_data_store *f = (const kern_data_store *)first_head.data();
            if ((uint32_t)h->format != format || h->ncols != f->ncols ||
                (h->format != KDS_FORMAT_ARROW &&
                 memcmp(h->colmeta, f->colmeta, sizeof(kern_colmeta) * h->ncols) != 0))
                return XB_ERR(err, ERRCODE_DEVICE_ERROR, "chunk %u of the batch has another layout", i);
        }
        tasks[i].kds = kds_dev[i];
        tasks[i].unit_base = base;
        tasks[i].nunits = xb_chunk_units(h);
        tasks[i].format = format;
        base += tasks[i].nunits;
        bytes += h->length;
        rows += h->nitems;
    }
    xpuB200Batch *b = new xpuB200Batch();
    b->sess = s;
    b->ntasks = nchunks;
    b->nunits = base;
    b->format = format;
    b->bytes = bytes;
    b->rows = rows;
    if (cudaMalloc((void **)&b->d_tasks, sizeof(xb_task) * nchunks) != cudaSuccess) {
        delete b;
        return XB_ERR(err, ERRCODE_DEVICE_FATAL, "out of device memory for the batch");
    }
    cudaMemcpy(b->d_tasks, tasks.data(), sizeof(xb_task) * nchunks, cudaMemcpyHostToDevice);
    *p_batch = b;
    return 0;
}

extern "C" int
xpuB200BatchExec(xpuB200Batch *b, kern_exec_results *results, kern_errorbuf *err)
{
    xb_clear_error(err);
    if (!b)
        return XB_ERR(err, ERRCODE_DEVICE_ERROR, "invalid batch");
    xpuB200Session *s = b->sess;
    std::lock_guard<std::mutex> g(s->lock);
    XB_CUDA(cudaSetDevice(s->dev->dindex), err);
    s->in_batch = true;
    int rc = xb_run(s, b->d_tasks, b->ntasks, b->nunits, b->format, results, err);
    s->in_batch = false;
    return rc;
}

extern "C" int
xpuB200BatchTime(xpuB200Batch *b, int niters, double *p_msec, kern_errorbuf *err)
{
    xb_clear_error(err);
    xpuB200Session *s = b->sess;
    std::lock_guard<std::mutex> g(s->lock);
    XB_CUDA(cudaSetDevice(s->dev->dindex), err);
    float total = 0.0f;
    for (int i = 0; i < niters; i++) {
        s->in_batch = true;
        int rc = xb_run(s, b->d_tasks, b->ntasks, b->nunits, b->format, nullptr, err, true);
        s->in_batch = false;
        if (rc) return rc;
        float ms = 0.0f;
        cudaEventElapsedTime(&ms, s->ev0, s->ev1);
        total += ms;
    }
    *p_msec = niters > 0 ? total / niters : 0.0;
    return 0;
}

/* the session's group table and statistics back to their state after
 * OpenSession; session lock held */
static void xb_reset_groups(xpuB200Session *s)
{
    cudaStream_t st = s->stream;
    if (s->h_plan->has_groupby) {
        cudaMemsetAsync(s->h_gt.entries, 0, (s->h_gt.cap_mask + 1) * s->h_plan->gent_size, st);
        if (s->h_gt.dump)
            cudaMemsetAsync(s->h_gt.dump, 0, s->h_gt.dump_cap * s->h_plan->gent_size, st);
        s->h_gt.nused = 0;
        s->h_gt.arena_used = 0;
        s->h_gt.overflow = 0;
        s->h_gt.grow = 0;
        s->h_gt.dump_used = 0;
        s->h_gt.soft_cap = (s->h_gt.cap_mask + 1) / 2;
        cudaMemcpyAsync(s->d_gt, &s->h_gt, sizeof(xb_gtable), cudaMemcpyHostToDevice, st);
    }
    cudaMemsetAsync(s->d_status, 0, sizeof(xb_status), st);
    cudaStreamSynchronize(st);
    s->total_raw = s->total_in = s->total_out = 0;
    for (uint32_t d = 0; d <= XB_MAX_DEPTH; d++)
        s->total_depth[d] = 0;
}

extern "C" int
xpuB200BatchTune(xpuB200Batch *b, uint32_t flags, char *report, size_t report_len, kern_errorbuf *err)
{
    xb_clear_error(err);
    if (!b || flags != 0)
        return XB_ERR(err, ERRCODE_DEVICE_ERROR, "invalid BatchTune arguments");
    xpuB200Session *s = b->sess;
    xb_sched_drain_session(s);
    std::lock_guard<std::mutex> g(s->lock);
    if (s->total_raw != 0)
        return XB_ERR(err, ERRCODE_DEVICE_ERROR, "tune a session before it executes chunks");
    XB_CUDA(cudaSetDevice(s->dev->dindex), err);
    s->tune_looked_up = true;               /* measured here, not adopted */
    const xb_plan *plan = s->h_plan;
    const uint32_t fmt = b->format;
    bool gid = false;
    for (uint32_t d = 1; d <= plan->nrels; d++)
        gid |= plan->inner[d].gid_on != 0;
    const uint32_t sm0 = s->sm_cap_default;
    /* group ids index the shared table directly: its size is then fixed */
    std::vector<uint32_t> sms;
    if (!gid && plan->has_groupby && sm0 > 0) {
        if ((size_t)sm0 * 2 * plan->gent_size <= 48 * 1024)
            sms.push_back(sm0 * 2);
        sms.push_back(0);
    }
    std::vector<int> minbs;
    if (s->jit_enabled)
        minbs = {2, 3, 4, 6, 8};
    else
        minbs = {0};
    struct cand { int minb; uint32_t sm; double ms; const char *kernel; };
    std::vector<cand> done;
    int rc = 0;
    auto measure = [&](int minb, uint32_t smc) -> int {
        s->jit_minb = minb;
        if (xb_set_sm_cap(s, smc) != 0)
            return 1;                       /* does not fit: skipped */
        double best = 1e30;
        for (int r = 0; r < 3 && rc == 0; r++) {      /* the first run builds and warms */
            xb_reset_groups(s);
            s->in_batch = true;
            rc = xb_run(s, b->d_tasks, b->ntasks, b->nunits, fmt, nullptr, err, true);
            s->in_batch = false;
            if (rc) break;
            float ms = 0.0f;
            cudaEventElapsedTime(&ms, s->ev0, s->ev1);
            if (r > 0 && ms < best) best = ms;
        }
        if (rc)
            return -1;
        if (minb > 0 && !s->jit_fn[fmt])
            return 1;                       /* the specialised kernel was not built */
        done.push_back({minb, smc, best, s->jit_fn[fmt] ? "jit" : "vm"});
        return 0;
    };
    /* coordinate search: CTAs per SM at the default table, then the table */
    for (int m : minbs)
        if (measure(m, sm0) < 0) break;
    if (rc == 0 && !done.empty()) {
        int bm = done[0].minb;
        double bt = done[0].ms;
        for (const cand &c : done)
            if (c.ms < bt) { bt = c.ms; bm = c.minb; }
        for (uint32_t c : sms)
            if (measure(bm, c) < 0) break;
    }
    cand best = {0, sm0, 0.0, "none"};
    if (rc == 0 && !done.empty()) {
        best = done[0];
        for (const cand &c : done)
            if (c.ms < best.ms) best = c;
    }
    s->jit_minb = best.minb;
    if (xb_set_sm_cap(s, best.sm) != 0)
        xb_set_sm_cap(s, sm0);
    xb_reset_groups(s);
    s->tune_looked_up = true;
    if (rc)
        return rc;
    if (done.empty())
        return XB_ERR(err, ERRCODE_DEVICE_ERROR, "no launch shape could be measured");
    {
        const auto key = xb_tune_key(s, fmt);
        std::lock_guard<std::mutex> tg(g_tune_lock);
        g_tune[key] = xb_tune_choice{best.minb, best.sm};
        g_tune_minb[std::make_pair(std::get<0>(key), std::get<1>(key))] = best.minb;
    }
    if (report && report_len) {
        std::string r = "{\"format\": \"" + std::string(1, (char)fmt) + "\", \"candidates\": [";
        char buf[256];
        for (size_t i = 0; i < done.size(); i++) {
            snprintf(buf, sizeof(buf), "%s{\"ctas_per_sm\": %d, \"sm_groups\": %u, \"kernel\": \"%s\", \"ms\": %.4f}",
                     i ? ", " : "", done[i].minb, done[i].sm, done[i].kernel, done[i].ms);
            r += buf;
        }
        snprintf(buf, sizeof(buf), "], \"best\": {\"ctas_per_sm\": %d, \"sm_groups\": %u, \"ms\": %.4f}, "
                 "\"default_sm_groups\": %u}", best.minb, best.sm, best.ms, sm0);
        r += buf;
        snprintf(report, report_len, "%s", r.c_str());
    }
    return 0;
}

extern "C" void
xpuB200BatchDestroy(xpuB200Batch *b)
{
    if (!b) return;
    cudaSetDevice(b->sess->dev->dindex);
    cudaFree(b->d_tasks);
    delete b;
}

/* ================================================================
 * mixed batches: chunk commands of many sessions in one launch
 * ================================================================ */
/* units one CTA takes of a command before another CTA is sent to join it */
#define XB_MIX_JOIN_UNITS   16

/* one persistent launch of a mixed batch: the commands that share a kernel
 * (a specialised mixed kernel of one plan shape, or the interpreter) */

/* the mixed kernel a command of session s (chunk format) runs on */
void *xb_mix_kernel_of(xpuB200Session *s, uint32_t format, bool wait)
{
    std::lock_guard<std::mutex> g(s->lock);
    return xb_session_jit(s, format, wait) ? s->jit_mixfn[format] : nullptr;
}

/* split commands into launches by kernel and build each work queue:
 * largest command first, listed once per XB_MIX_JOIN_UNITS of its units
 * (at most once per CTA) */
int xb_mix_plan(xpuB200Device *dev, const std::vector<xpuB200Session *> &sess,
                const std::vector<uint32_t> &formats, const std::vector<uint64_t> &units,
                std::vector<xb_mix_group> &groups, kern_errorbuf *err, bool wait)
{
    groups.clear();
    for (uint32_t i = 0; i < sess.size(); i++) {
        void *k = xb_mix_kernel_of(sess[i], formats[i], wait);
        if (formats[i] < 256)
            sess[i]->ran_kind[formats[i]] = k ? 'j' : 'v';
        size_t g = 0;
        while (g < groups.size() && groups[g].jfn != k)
            g++;
        if (g == groups.size()) {
            groups.emplace_back();
            groups.back().jfn = k;
        }
        groups[g].cmds.push_back(i);
        const size_t sm = k ? sess[i]->jit_smem_fmt[formats[i]] : sess[i]->smem_bytes;
        if (sm > groups[g].smem)
            groups[g].smem = sm;
    }
    for (xb_mix_group &g : groups) {
        const size_t st = g.jfn ? xb_jit_static_smem(g.jfn) : sizeof(XbExecArgs);
        if (g.smem + st + 16 > dev->smem_optin)
            return XB_ERR(err, ERRCODE_DEVICE_FATAL, "mixed launch needs %zu bytes of shared memory", g.smem);
        int per_sm = 0;
        if (g.jfn)
            xb_jit_occupancy(g.jfn, XB_BLOCK, g.smem, &per_sm);
        else
            cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, xb_mixed_kernel, XB_BLOCK, g.smem);
        if (per_sm < 1)
            return XB_ERR(err, ERRCODE_DEVICE_FATAL, "mixed kernel does not fit on an SM (%zu bytes)", g.smem);
        g.grid = per_sm * dev->nsm;
        std::vector<uint32_t> order(g.cmds);
        std::stable_sort(order.begin(), order.end(), [&](uint32_t a, uint32_t b) { return units[a] > units[b]; });
        for (uint32_t i : order) {
            uint64_t k = (units[i] + XB_MIX_JOIN_UNITS - 1) / XB_MIX_JOIN_UNITS;
            k = k < 1 ? 1 : (k > (uint64_t)g.grid ? g.grid : k);
            for (uint64_t j = 0; j < k; j++)
                g.items.push_back(i);
        }
    }
    return 0;
}

/* launch one group of a mixed batch on a stream */
int xb_mix_launch(const xb_mix_group &g, const XbMixArgs &ma, cudaStream_t stream, kern_errorbuf *err)
{
    if (g.jfn) {
        XbMixArgs a = ma;
        if (xb_jit_launch(g.jfn, g.grid, XB_BLOCK, g.smem, (void *)stream, &a) != 0)
            return XB_ERR(err, ERRCODE_DEVICE_FATAL, "specialised mixed kernel launch failed");
    } else {
        xb_mixed_kernel<<<g.grid, XB_BLOCK, g.smem, stream>>>(ma);
    }
    cudaError_t rc = cudaGetLastError();
    if (rc != cudaSuccess)
        return XB_ERR(err, ERRCODE_DEVICE_FATAL, "mixed launch: %s", cudaGetErrorString(rc));
    return 0;
}

struct xpuB200Mix {
    xpuB200Device  *dev;
    uint32_t        ncmds = 0;
    std::vector<xpuB200Session *> sess;
    std::vector<xb_mix_group> groups;
    xb_task        *d_tasks = nullptr;
    XbExecArgs     *d_cmds = nullptr;
    uint32_t       *d_items = nullptr;
    uint32_t        nitems = 0;
    uint32_t       *d_cursor = nullptr;     /* one per group, 32 bytes apart */
    xb_status      *d_status = nullptr;
    xb_status      *h_status = nullptr;     /* pinned */
    cudaStream_t    stream = nullptr;
    std::vector<cudaStream_t> aux;          /* a branch per further group */
    std::vector<cudaEvent_t> forks, joins;
    cudaGraph_t     graph = nullptr;
    cudaGraphExec_t gexec = nullptr;
    cudaEvent_t     ev0 = nullptr, ev1 = nullptr;
    uint64_t        bytes = 0, units = 0;
};

static void xb_mix_free(xpuB200Mix *m)
{
    if (!m) return;
    cudaSetDevice(m->dev->dindex);
    if (m->gexec) cudaGraphExecDestroy(m->gexec);
    if (m->graph) cudaGraphDestroy(m->graph);
    if (m->ev0) cudaEventDestroy(m->ev0);
    if (m->ev1) cudaEventDestroy(m->ev1);
    for (cudaEvent_t e : m->forks) cudaEventDestroy(e);
    for (cudaEvent_t e : m->joins) cudaEventDestroy(e);
    for (cudaStream_t a : m->aux) cudaStreamDestroy(a);
    if (m->stream) cudaStreamDestroy(m->stream);
    cudaFree(m->d_tasks);
    cudaFree(m->d_cmds);
    cudaFree(m->d_items);
    cudaFree(m->d_cursor);
    cudaFree(m->d_status);
    if (m->h_status) cudaFreeHost(m->h_status);
    delete m;
}

extern "C" int
xpuB200MixCreate(xpuB200Device *dev, uint32_t ncmds, xpuB200Session *const *sess,
                 const kern_data_store *const *kds_dev, xpuB200Mix **p_mix, kern_errorbuf *err)
{
    xb_clear_error(err);
    *p_mix = nullptr;
    if (!dev || !sess || !kds_dev || ncmds == 0)
        return XB_ERR(err, ERRCODE_DEVICE_ERROR, "invalid mixed batch arguments");
    XB_CUDA(cudaSetDevice(dev->dindex), err);
    std::vector<xb_task> tasks(ncmds);
    std::vector<uint64_t> units(ncmds);
    std::vector<uint32_t> formats(ncmds);
    uint64_t bytes = 0, total_units = 0;
    for (uint32_t i = 0; i < ncmds; i++) {
        xpuB200Session *s = sess[i];
        if (!s || s->dev != dev)
            return XB_ERR(err, ERRCODE_DEVICE_ERROR, "command %u: no session on this GPU", i);
        if (s->h_plan->has_proj)
            return XB_ERR(err, ERRCODE_DEVICE_ERROR, "command %u: projection sessions run through xpuB200ExecTaskDst", i);
        if (((uintptr_t)kds_dev[i] & 7) != 0)
            return XB_ERR(err, ERRCODE_DEVICE_ERROR, "command %u: chunk is not 8-byte aligned", i);
        kern_data_store head;
        XB_CUDA(cudaMemcpy(&head, kds_dev[i], offsetof(kern_data_store, colmeta), cudaMemcpyDeviceToHost), err);
        std::vector<char> hb(KDS_HEAD_LENGTH(&head));
        XB_CUDA(cudaMemcpy(hb.data(), kds_dev[i], hb.size(), cudaMemcpyDeviceToHost), err);
        const kern_data_store *h = (const kern_data_store *)hb.data();
        int rc = xb_check_kds(h, err);
        if (rc) return rc;
        {
            std::lock_guard<std::mutex> g(s->lock);
            xb_note_layout(s, h);
        }
        tasks[i].kds = kds_dev[i];
        tasks[i].unit_base = 0;
        tasks[i].nunits = xb_chunk_units(h);
        tasks[i].format = (uint32_t)h->format;
        units[i] = tasks[i].nunits;
        formats[i] = tasks[i].format;
        total_units += units[i];
        bytes += h->length;
    }
    xpuB200Mix *m = new xpuB200Mix();
    m->dev = dev;
    m->ncmds = ncmds;
    m->sess.assign(sess, sess + ncmds);
    m->bytes = bytes;
    m->units = total_units;
    int rc = xb_mix_plan(dev, m->sess, formats, units, m->groups, err);
    if (rc) {
        xb_mix_free(m);
        return rc;
    }
    const size_t ng = m->groups.size();
    std::vector<uint32_t> items;
    std::vector<size_t> item_off;
    for (const xb_mix_group &g : m->groups) {
        item_off.push_back(items.size());
        items.insert(items.end(), g.items.begin(), g.items.end());
    }
    m->nitems = (uint32_t)items.size();
    auto fail = [&](const char *what) {
        xb_mix_free(m);
        return XB_ERR(err, ERRCODE_DEVICE_FATAL, "mixed batch: %s", what);
    };
    if (cudaMalloc((void **)&m->d_tasks, sizeof(xb_task) * ncmds) != cudaSuccess ||
        cudaMalloc((void **)&m->d_cmds, sizeof(XbExecArgs) * ncmds) != cudaSuccess ||
        cudaMalloc((void **)&m->d_items, sizeof(uint32_t) * items.size()) != cudaSuccess ||
        cudaMalloc((void **)&m->d_cursor, 32 * ng) != cudaSuccess ||
        cudaMalloc((void **)&m->d_status, sizeof(xb_status) * ncmds) != cudaSuccess ||
        cudaMallocHost((void **)&m->h_status, sizeof(xb_status) * ncmds) != cudaSuccess)
        return fail("out of memory");
    std::vector<XbExecArgs> cmds(ncmds);
    for (uint32_t i = 0; i < ncmds; i++) {
        xpuB200Session *s = sess[i];
        XbExecArgs &a = cmds[i];
        memset(&a, 0, sizeof(a));
        a.plan = s->d_plan;
        a.plan_bytes = s->plan_bytes;
        a.tasks = m->d_tasks + i;
        a.ntasks = 1;
        a.nunits = tasks[i].nunits;
        a.format = tasks[i].format;
        a.sm_cap = s->sm_cap;
        a.warp_bytes = s->warp_bytes;
        a.gt = s->d_gt;
        a.st = m->d_status + i;
        a.dyn_only = 1;
    }
    if (cudaMemcpy(m->d_tasks, tasks.data(), sizeof(xb_task) * ncmds, cudaMemcpyHostToDevice) != cudaSuccess ||
        cudaMemcpy(m->d_cmds, cmds.data(), sizeof(XbExecArgs) * ncmds, cudaMemcpyHostToDevice) != cudaSuccess ||
        cudaMemcpy(m->d_items, items.data(), sizeof(uint32_t) * items.size(), cudaMemcpyHostToDevice) != cudaSuccess)
        return fail("upload failed");
    if (cudaStreamCreateWithFlags(&m->stream, cudaStreamNonBlocking) != cudaSuccess ||
        cudaEventCreate(&m->ev0) != cudaSuccess || cudaEventCreate(&m->ev1) != cudaSuccess)
        return fail("stream setup failed");
    for (size_t g = 1; g < ng; g++) {
        cudaStream_t a;
        cudaEvent_t f, j;
        if (cudaStreamCreateWithFlags(&a, cudaStreamNonBlocking) != cudaSuccess)
            return fail("stream setup failed");
        m->aux.push_back(a);
        if (cudaEventCreateWithFlags(&f, cudaEventDisableTiming) != cudaSuccess)
            return fail("event setup failed");
        m->forks.push_back(f);
        if (cudaEventCreateWithFlags(&j, cudaEventDisableTiming) != cudaSuccess)
            return fail("event setup failed");
        m->joins.push_back(j);
    }
    /* one run = clear the statuses and the queue cursors, one persistent
     * launch per kernel group (concurrent branches), the statuses back to
     * the host: captured once, replayed */
    if (cudaStreamBeginCapture(m->stream, cudaStreamCaptureModeThreadLocal) != cudaSuccess)
        return fail("stream capture failed");
    kern_errorbuf lerr;
    int lrc = 0;
    cudaMemsetAsync(m->d_status, 0, sizeof(xb_status) * ncmds, m->stream);
    cudaMemsetAsync(m->d_cursor, 0, 32 * ng, m->stream);
    for (size_t g = 1; g < ng; g++) {
        cudaEventRecord(m->forks[g - 1], m->stream);
        cudaStreamWaitEvent(m->aux[g - 1], m->forks[g - 1], 0);
    }
    for (size_t g = 0; g < ng && !lrc; g++) {
        XbMixArgs ma;
        ma.cmds = m->d_cmds;
        ma.items = m->d_items + item_off[g];
        ma.nitems = (uint32_t)m->groups[g].items.size();
        ma.cursor = m->d_cursor + 8 * g;
        lrc = xb_mix_launch(m->groups[g], ma, g == 0 ? m->stream : m->aux[g - 1], &lerr);
    }
    for (size_t g = 1; g < ng; g++) {
        cudaEventRecord(m->joins[g - 1], m->aux[g - 1]);
        cudaStreamWaitEvent(m->stream, m->joins[g - 1], 0);
    }
    cudaMemcpyAsync(m->h_status, m->d_status, sizeof(xb_status) * ncmds, cudaMemcpyDeviceToHost, m->stream);
    cudaError_t crc = cudaStreamEndCapture(m->stream, &m->graph);
    if (lrc) {
        if (err) *err = lerr;
        xb_mix_free(m);
        return lrc;
    }
    if (crc != cudaSuccess || cudaGraphInstantiate(&m->gexec, m->graph, 0) != cudaSuccess)
        return fail("graph capture failed");
    *p_mix = m;
    return 0;
}

/* lock the distinct sessions of a mixed batch, in address order */
static std::vector<std::unique_lock<std::mutex>> xb_mix_lock(xpuB200Mix *m)
{
    std::vector<xpuB200Session *> u(m->sess);
    std::sort(u.begin(), u.end());
    u.erase(std::unique(u.begin(), u.end()), u.end());
    std::vector<std::unique_lock<std::mutex>> locks;
    for (xpuB200Session *s : u)
        locks.emplace_back(s->lock);
    return locks;
}

extern "C" int
xpuB200MixExec(xpuB200Mix *m, kern_exec_results *const *results, kern_errorbuf *errs)
{
    if (!m)
        return ERRCODE_DEVICE_ERROR;
    for (uint32_t i = 0; errs && i < m->ncmds; i++)
        xb_clear_error(&errs[i]);
    auto locks = xb_mix_lock(m);
    kern_errorbuf *e0 = errs;
    XB_CUDA(cudaSetDevice(m->dev->dindex), e0);
    XB_CUDA(cudaGraphLaunch(m->gexec, m->stream), e0);
    XB_CUDA(cudaStreamSynchronize(m->stream), e0);
    int first = 0;
    for (uint32_t i = 0; i < m->ncmds; i++) {
        const xb_status *hs = &m->h_status[i];
        if (hs->errcode) {
            int rc = xb_set_error(errs ? &errs[i] : nullptr, hs->errcode, "xb_mixed_kernel", hs->lineno,
                                  "%s", xb_msg_text(hs->msg_id));
            if (!first) first = rc;
            continue;
        }
        xb_account_status(m->sess[i], hs, results ? results[i] : nullptr);
    }
    return first;
}

extern "C" int
xpuB200MixTime(xpuB200Mix *m, int niters, double *p_msec, kern_errorbuf *err)
{
    xb_clear_error(err);
    if (!m)
        return XB_ERR(err, ERRCODE_DEVICE_ERROR, "invalid mixed batch");
    auto locks = xb_mix_lock(m);
    XB_CUDA(cudaSetDevice(m->dev->dindex), err);
    float total = 0.0f;
    for (int it = 0; it < niters; it++) {
        XB_CUDA(cudaEventRecord(m->ev0, m->stream), err);
        XB_CUDA(cudaGraphLaunch(m->gexec, m->stream), err);
        XB_CUDA(cudaEventRecord(m->ev1, m->stream), err);
        XB_CUDA(cudaStreamSynchronize(m->stream), err);
        for (uint32_t i = 0; i < m->ncmds; i++)
            if (m->h_status[i].errcode)
                return xb_set_error(err, m->h_status[i].errcode, "xb_mixed_kernel", m->h_status[i].lineno,
                                    "command %u: %s", i, xb_msg_text(m->h_status[i].msg_id));
        float ms = 0.0f;
        cudaEventElapsedTime(&ms, m->ev0, m->ev1);
        total += ms;
    }
    *p_msec = niters > 0 ? total / niters : 0.0;
    return 0;
}

extern "C" int
xpuB200MixInfo(const xpuB200Mix *m, uint64_t *p_bytes, uint64_t *p_units, uint32_t *p_items,
               uint32_t *p_launches, uint32_t *p_specialised)
{
    if (!m) return ERRCODE_DEVICE_ERROR;
    if (p_bytes) *p_bytes = m->bytes;
    if (p_units) *p_units = m->units;
    if (p_items) *p_items = m->nitems;
    if (p_launches) *p_launches = (uint32_t)m->groups.size();
    if (p_specialised) {
        uint32_t n = 0;
        for (const xb_mix_group &g : m->groups)
            if (g.jfn) n += (uint32_t)g.cmds.size();
        *p_specialised = n;
    }
    return 0;
}

extern "C" void
xpuB200MixDestroy(xpuB200Mix *m)
{
    xb_mix_free(m);
}

