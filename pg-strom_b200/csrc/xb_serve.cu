/*
 * xb_serve.cu
 *
 * Serving (xpuB200Submit / Poll / ServeConfig / MemInfo): asynchronous
 * chunk commands with continuous batching and admission by free device
 * memory; xpuB200HandleCommand, the dispatch of the reference's GPU-service
 * worker (gpuservGpuWorkerMain, gpu_service.c:5951-5964); device memory
 * helpers; the inner-relation cache's budget; and outer-table chunks
 * resident in HBM across sessions (xpuB200ChunkCache*).
 */
#include <cuda_runtime.h>
#include <algorithm>
#include <chrono>
#include <deque>
#include <map>
#include <mutex>
#include <thread>
#include <unordered_map>
#include <vector>
#include <cstdio>
#include <cstring>
#include "xb_host.h"

/* ================================================================
 * serving: asynchronous chunk commands with continuous batching
 * ================================================================
 *
 * xpuB200Submit queues a chunk command of any session; the scheduler keeps
 * up to XB_SLOTS launches in flight on their own streams.  Whenever a slot
 * is free (checked on every Submit and Poll), the queued commands are
 * admitted in arrival order while their staging bytes fit the admission
 * budget: a large command of a session with a specialised kernel runs
 * alone on it, the small ones go together into one mixed launch
 * (xb_mixed_kernel).  Commands that arrive while others are on the GPU are
 * admitted as slots and memory free up, so their work overlaps on the
 * device.  A finished command's statistics are added to its session and
 * kept for xpuB200Poll; its groups are in the session's group table.
 */
/* the device's free and total memory, and the reserve admission keeps */
static void xb_mem_info(xpuB200Device *dev, uint64_t *p_free, uint64_t *p_total, uint64_t *p_reserve)
{
    size_t fr = 0, tot = 0;
    cudaSetDevice(dev->dindex);
    if (cudaMemGetInfo(&fr, &tot) != cudaSuccess) {
        cudaGetLastError();
        fr = tot = 0;
    }
    *p_free = fr;
    *p_total = tot;
    const uint64_t r = tot / 20;
    *p_reserve = r > (1ULL << 30) ? r : (1ULL << 30);
}

#define XB_SLOTS            4       /* launches in flight per GPU */
#define XB_SLOT_CMDS        256     /* commands of one mixed launch */
#define XB_ALONE_UNITS      256     /* commands of this many units run alone */

struct xb_cmd {
    uint64_t        ticket;
    xpuB200Session *s;
    const kern_data_store *kds;     /* the caller's chunk */
    int             on_device;
    uint64_t        length;
    uint64_t        shift;          /* staging offset that aligns heap pages */
    uint64_t        units;
    uint32_t        format;
    const kern_data_store *d_kds;   /* the chunk on the device, once launched */
};

struct xb_done {
    int             rc;             /* 0, or the command's error code */
    kern_errorbuf   err;
    xb_status       st;
    uint32_t        nrels;
};

struct xb_slot {
    cudaStream_t    stream = nullptr;
    cudaEvent_t     done = nullptr;
    bool            busy = false;
    bool            alone = false;
    std::vector<xb_cmd> cmds;
    uint64_t        staged = 0;     /* admission bytes held by this launch */
    char           *d_stage = nullptr;
    uint64_t        stage_cap = 0;
    xb_status      *d_status = nullptr;
    xb_status      *h_status = nullptr;     /* pinned */
    xb_task        *d_tasks = nullptr, *h_tasks = nullptr;
    XbExecArgs     *d_cmds = nullptr, *h_cmds = nullptr;
    uint32_t       *d_items = nullptr, *h_items = nullptr;
    uint32_t        items_cap = 0;
    uint32_t       *d_cursor = nullptr;
};

struct xb_sched {
    std::mutex      lock;
    uint64_t        next_ticket = 1;
    std::deque<xb_cmd> pending;
    xb_slot         slot[XB_SLOTS];
    std::unordered_map<uint64_t, xb_done> done;
    uint64_t        admit_bytes = 0;
    uint64_t        inflight_bytes = 0;
    uint32_t        alone_units = XB_ALONE_UNITS;
    int             mix_grid_per_sm[2] = {0, 0};
};

static void xb_slot_free(xb_slot &sl)
{
    if (sl.stream) { cudaStreamSynchronize(sl.stream); cudaStreamDestroy(sl.stream); }
    if (sl.done) cudaEventDestroy(sl.done);
    cudaFree(sl.d_stage);
    cudaFree(sl.d_status);
    cudaFree(sl.d_tasks);
    cudaFree(sl.d_cmds);
    cudaFree(sl.d_items);
    cudaFree(sl.d_cursor);
    if (sl.h_status) cudaFreeHost(sl.h_status);
    if (sl.h_tasks) cudaFreeHost(sl.h_tasks);
    if (sl.h_cmds) cudaFreeHost(sl.h_cmds);
    if (sl.h_items) cudaFreeHost(sl.h_items);
    sl = xb_slot();
}

static int xb_sched_init(xpuB200Device *dev, kern_errorbuf *err)
{
    if (dev->sched)
        return 0;
    xb_sched *q = new xb_sched();
    q->admit_bytes = XPU_B200_ADMIT_FREE_HBM;
    for (int i = 0; i < XB_SLOTS; i++) {
        xb_slot &sl = q->slot[i];
        if (cudaStreamCreateWithFlags(&sl.stream, cudaStreamNonBlocking) != cudaSuccess ||
            cudaEventCreateWithFlags(&sl.done, cudaEventDisableTiming) != cudaSuccess ||
            cudaMalloc((void **)&sl.d_status, sizeof(xb_status) * XB_SLOT_CMDS) != cudaSuccess ||
            cudaMallocHost((void **)&sl.h_status, sizeof(xb_status) * XB_SLOT_CMDS) != cudaSuccess ||
            cudaMalloc((void **)&sl.d_tasks, sizeof(xb_task) * XB_SLOT_CMDS) != cudaSuccess ||
            cudaMallocHost((void **)&sl.h_tasks, sizeof(xb_task) * XB_SLOT_CMDS) != cudaSuccess ||
            cudaMalloc((void **)&sl.d_cmds, sizeof(XbExecArgs) * XB_SLOT_CMDS) != cudaSuccess ||
            cudaMallocHost((void **)&sl.h_cmds, sizeof(XbExecArgs) * XB_SLOT_CMDS) != cudaSuccess ||
            cudaMalloc((void **)&sl.d_cursor, 16) != cudaSuccess) {
            for (int j = 0; j <= i; j++)
                xb_slot_free(q->slot[j]);
            delete q;
            return XB_ERR(err, ERRCODE_DEVICE_FATAL, "cannot set up the command scheduler");
        }
    }
    dev->sched = q;
    return 0;
}

/* finish the launch of slot sl if its work is done; sched lock held */
static void xb_sched_retire(xb_sched *q, xb_slot &sl, bool wait)
{
    if (!sl.busy)
        return;
    cudaError_t rc = wait ? cudaEventSynchronize(sl.done) : cudaEventQuery(sl.done);
    if (rc == cudaErrorNotReady)
        return;
    for (size_t i = 0; i < sl.cmds.size(); i++) {
        const xb_cmd &c = sl.cmds[i];
        xb_done d;
        memset(&d, 0, sizeof(d));
        d.nrels = c.s->h_plan->nrels;
        if (rc != cudaSuccess) {
            d.rc = xb_set_error(&d.err, ERRCODE_DEVICE_FATAL, "xpuB200Poll", __LINE__, "%s",
                                cudaGetErrorString(rc));
        } else {
            d.st = sl.h_status[i];
            if (d.st.errcode) {
                d.rc = xb_set_error(&d.err, d.st.errcode, sl.alone ? "xb_exec_kernel" : "xb_mixed_kernel",
                                    d.st.lineno, "%s", xb_msg_text(d.st.msg_id));
            } else {
                std::lock_guard<std::mutex> g(c.s->lock);
                xb_account_status(c.s, &d.st, nullptr);
            }
        }
        c.s->sched_refs--;
        q->done[c.ticket] = d;
    }
    q->inflight_bytes -= sl.staged;
    sl.staged = 0;
    sl.cmds.clear();
    sl.busy = false;
}

/* copy the host chunks of cmds into the slot's staging buffer; sched lock held */
static int xb_sched_stage(xb_slot &sl, std::vector<xb_cmd> &cmds, kern_errorbuf *err)
{
    uint64_t need = 0;
    for (const xb_cmd &c : cmds)
        if (!c.on_device)
            need += PGSTROM_TYPEALIGN(256, c.length + c.shift);
    if (need > sl.stage_cap) {
        cudaStreamSynchronize(sl.stream);
        cudaFree(sl.d_stage);
        sl.d_stage = nullptr;
        sl.stage_cap = 0;
        uint64_t cap = need < (64ULL << 20) ? (64ULL << 20) : need;
        XB_CUDA(cudaMalloc((void **)&sl.d_stage, cap), err);
        sl.stage_cap = cap;
    }
    uint64_t off = 0;
    for (xb_cmd &c : cmds) {
        if (c.on_device) {
            c.d_kds = c.kds;
            continue;
        }
        XB_CUDA(cudaMemcpyAsync(sl.d_stage + off + c.shift, c.kds, c.length, cudaMemcpyHostToDevice, sl.stream), err);
        c.d_kds = (const kern_data_store *)(sl.d_stage + off + c.shift);
        off += PGSTROM_TYPEALIGN(256, c.length + c.shift);
    }
    return 0;
}

/* launch the next admitted commands on slot sl; sched lock held */
static int xb_sched_launch(xpuB200Device *dev, xb_sched *q, xb_slot &sl, kern_errorbuf *err)
{
    std::vector<xb_cmd> take;
    uint64_t bytes = 0;
    /* admission: by the device's free memory (the slot's staging buffer
     * is reusable), or against a fixed budget for the bytes in flight */
    uint64_t room;
    if (q->admit_bytes == XPU_B200_ADMIT_FREE_HBM) {
        uint64_t fr = 0, tot = 0, reserve = 0;
        xb_mem_info(dev, &fr, &tot, &reserve);
        room = (fr > reserve ? fr - reserve : 0) + sl.stage_cap;
    } else {
        room = q->admit_bytes > q->inflight_bytes ? q->admit_bytes - q->inflight_bytes : 0;
    }
    const xb_cmd &f = q->pending.front();
    const bool alone = f.units >= q->alone_units && f.s->jit_enabled;
    void *kern = alone ? nullptr : xb_mix_kernel_of(f.s, f.format, false);
    while (!q->pending.empty() && take.size() < (alone ? 1u : (size_t)XB_SLOT_CMDS)) {
        const xb_cmd &c = q->pending.front();
        if (!alone && c.units >= q->alone_units && c.s->jit_enabled)
            break;                      /* a large one runs alone, in a later launch */
        if (!alone && xb_mix_kernel_of(c.s, c.format, false) != kern)
            break;                      /* another kernel: a launch of its own */
        const uint64_t b = c.on_device ? 0 : c.length + c.shift + 256;
        if (bytes + b > room && (!take.empty() || q->inflight_bytes > 0))
            break;                      /* admission: wait for memory to free up */
        bytes += b;
        take.push_back(c);
        q->pending.pop_front();
    }
    if (take.empty())
        return 0;
    sl.busy = true;
    sl.alone = alone;
    sl.staged = bytes;
    q->inflight_bytes += bytes;
    sl.cmds = take;
    int rc = xb_sched_stage(sl, sl.cmds, err);
    const uint32_t n = (uint32_t)sl.cmds.size();
    if (!rc) {
        for (uint32_t i = 0; i < n; i++) {
            const xb_cmd &c = sl.cmds[i];
            sl.h_tasks[i].kds = c.d_kds;
            sl.h_tasks[i].unit_base = 0;
            sl.h_tasks[i].nunits = c.units;
            sl.h_tasks[i].format = c.format;
        }
        if (cudaMemcpyAsync(sl.d_tasks, sl.h_tasks, sizeof(xb_task) * n, cudaMemcpyHostToDevice, sl.stream) != cudaSuccess ||
            cudaMemsetAsync(sl.d_status, 0, sizeof(xb_status) * n, sl.stream) != cudaSuccess)
            rc = XB_ERR(err, ERRCODE_DEVICE_FATAL, "scheduler upload failed");
    }
    if (!rc && alone) {
        xpuB200Session *s = sl.cmds[0].s;
        std::lock_guard<std::mutex> g(s->lock);
        rc = xb_launch_on(s, sl.d_tasks, 1, sl.cmds[0].units, sl.cmds[0].format, sl.stream, sl.d_status, err);
    } else if (!rc) {
        /* one mixed launch of commands that share a kernel */
        std::vector<xpuB200Session *> ss(n);
        std::vector<uint32_t> fm(n);
        std::vector<uint64_t> un(n);
        for (uint32_t i = 0; i < n; i++) {
            ss[i] = sl.cmds[i].s;
            fm[i] = sl.cmds[i].format;
            un[i] = sl.cmds[i].units;
        }
        std::vector<xb_mix_group> groups;
        rc = xb_mix_plan(dev, ss, fm, un, groups, err, false);
        const xb_mix_group *g = groups.empty() ? nullptr : &groups[0];
        if (!rc && g && g->items.size() > sl.items_cap) {
            cudaStreamSynchronize(sl.stream);
            cudaFree(sl.d_items);
            if (sl.h_items) cudaFreeHost(sl.h_items);
            sl.d_items = nullptr;
            sl.h_items = nullptr;
            sl.items_cap = 0;
            const uint32_t cap = (uint32_t)g->items.size() * 2;
            if (cudaMalloc((void **)&sl.d_items, sizeof(uint32_t) * cap) != cudaSuccess ||
                cudaMallocHost((void **)&sl.h_items, sizeof(uint32_t) * cap) != cudaSuccess)
                rc = XB_ERR(err, ERRCODE_DEVICE_FATAL, "scheduler: out of memory for the work queue");
            else
                sl.items_cap = cap;
        }
        if (!rc && g) {
            memcpy(sl.h_items, g->items.data(), sizeof(uint32_t) * g->items.size());
            for (uint32_t i = 0; i < n; i++) {
                xpuB200Session *s = sl.cmds[i].s;
                XbExecArgs &a = sl.h_cmds[i];
                memset(&a, 0, sizeof(a));
                a.plan = s->d_plan;
                a.plan_bytes = s->plan_bytes;
                a.tasks = sl.d_tasks + i;
                a.ntasks = 1;
                a.nunits = sl.cmds[i].units;
                a.format = sl.cmds[i].format;
                a.sm_cap = s->sm_cap;
                a.warp_bytes = s->warp_bytes;
                a.gt = s->d_gt;
                a.st = sl.d_status + i;
                a.dyn_only = 1;
            }
            XbMixArgs ma;
            ma.cmds = sl.d_cmds;
            ma.items = sl.d_items;
            ma.nitems = (uint32_t)g->items.size();
            ma.cursor = sl.d_cursor;
            cudaMemcpyAsync(sl.d_cmds, sl.h_cmds, sizeof(XbExecArgs) * n, cudaMemcpyHostToDevice, sl.stream);
            cudaMemcpyAsync(sl.d_items, sl.h_items, sizeof(uint32_t) * g->items.size(), cudaMemcpyHostToDevice, sl.stream);
            cudaMemsetAsync(sl.d_cursor, 0, 16, sl.stream);
            rc = xb_mix_launch(*g, ma, sl.stream, err);
        }
    }
    if (!rc) {
        if (cudaMemcpyAsync(sl.h_status, sl.d_status, sizeof(xb_status) * n, cudaMemcpyDeviceToHost, sl.stream) != cudaSuccess ||
            cudaEventRecord(sl.done, sl.stream) != cudaSuccess)
            rc = XB_ERR(err, ERRCODE_DEVICE_FATAL, "scheduler: status read-back failed");
    }
    if (rc) {
        /* the launch did not happen: its commands finish with the error */
        cudaStreamSynchronize(sl.stream);
        for (const xb_cmd &c : sl.cmds) {
            xb_done d;
            memset(&d, 0, sizeof(d));
            d.rc = rc;
            if (err) d.err = *err;
            d.nrels = c.s->h_plan->nrels;
            c.s->sched_refs--;
            q->done[c.ticket] = d;
        }
        q->inflight_bytes -= sl.staged;
        sl.staged = 0;
        sl.cmds.clear();
        sl.busy = false;
    }
    return rc;
}

/* retire finished launches and launch admitted commands; sched lock held */
static void xb_sched_progress(xpuB200Device *dev, xb_sched *q)
{
    for (int i = 0; i < XB_SLOTS; i++)
        xb_sched_retire(q, q->slot[i], false);
    for (int i = 0; i < XB_SLOTS && !q->pending.empty(); i++) {
        xb_slot &sl = q->slot[i];
        if (sl.busy)
            continue;
        kern_errorbuf e;
        xb_sched_launch(dev, q, sl, &e);    /* errors are recorded per command */
    }
}

/* block until one in-flight launch finishes (one holding 'who' if given);
 * called with the lock held through lk, which is released while waiting */
static void xb_sched_wait_one(xb_sched *q, std::unique_lock<std::mutex> &lk, const xpuB200Session *who)
{
    int pick = -1;
    for (int i = 0; i < XB_SLOTS && pick < 0; i++) {
        if (!q->slot[i].busy)
            continue;
        if (!who)
            pick = i;
        for (const xb_cmd &c : q->slot[i].cmds)
            if (c.s == who)
                pick = i;
    }
    for (int i = 0; i < XB_SLOTS && pick < 0; i++)
        if (q->slot[i].busy)
            pick = i;
    if (pick < 0)
        return;
    cudaEvent_t ev = q->slot[pick].done;
    lk.unlock();
    cudaEventSynchronize(ev);
    lk.lock();
}

void xb_sched_drain_session(xpuB200Session *s)
{
    xpuB200Device *dev = s->dev;
    xb_sched *q = dev->sched;
    if (!q)
        return;
    cudaSetDevice(dev->dindex);
    std::unique_lock<std::mutex> lk(q->lock);
    for (;;) {
        xb_sched_progress(dev, q);
        if (s->sched_refs == 0)
            break;
        xb_sched_wait_one(q, lk, s);
    }
}

void xb_sched_destroy(xpuB200Device *dev)
{
    xb_sched *q = dev->sched;
    if (!q)
        return;
    for (int i = 0; i < XB_SLOTS; i++)
        xb_slot_free(q->slot[i]);
    delete q;
    dev->sched = nullptr;
}

/* the CUDA device index of a device handle, for the storage reader (xb_direct.cpp) */
extern "C" int
xb_device_index(const xpuB200Device *dev)
{
    return dev->dindex;
}

extern "C" int
xpuB200MemInfo(xpuB200Device *dev, uint64_t *p_free, uint64_t *p_total, uint64_t *p_reserve)
{
    if (!dev)
        return ERRCODE_DEVICE_ERROR;
    uint64_t fr, tot, res;
    xb_mem_info(dev, &fr, &tot, &res);
    if (p_free) *p_free = fr;
    if (p_total) *p_total = tot;
    if (p_reserve) *p_reserve = res;
    return 0;
}

extern "C" int
xpuB200ServeConfig(xpuB200Device *dev, uint64_t admit_bytes, uint32_t alone_units, kern_errorbuf *err)
{
    xb_clear_error(err);
    if (!dev)
        return XB_ERR(err, ERRCODE_DEVICE_ERROR, "invalid device");
    XB_CUDA(cudaSetDevice(dev->dindex), err);
    int rc = xb_sched_init(dev, err);
    if (rc) return rc;
    std::lock_guard<std::mutex> g(dev->sched->lock);
    if (admit_bytes)
        dev->sched->admit_bytes = admit_bytes;
    if (alone_units)
        dev->sched->alone_units = alone_units;
    return 0;
}

extern "C" int
xpuB200Submit(xpuB200Session *s, const kern_data_store *kds_src, int kds_src_on_device,
              uint64_t *p_ticket, kern_errorbuf *err)
{
    xb_clear_error(err);
    if (!s || !kds_src || !p_ticket)
        return XB_ERR(err, ERRCODE_DEVICE_ERROR, "invalid Submit arguments");
    if (s->h_plan->has_proj)
        return XB_ERR(err, ERRCODE_DEVICE_ERROR, "projection sessions run through xpuB200ExecTaskDst");
    xpuB200Device *dev = s->dev;
    XB_CUDA(cudaSetDevice(dev->dindex), err);
    int rc = xb_sched_init(dev, err);
    if (rc) return rc;
    /* the chunk header, checked now */
    xb_cmd c;
    memset(&c, 0, sizeof(c));
    std::vector<char> hb;
    kern_data_store head;
    if (kds_src_on_device) {
        if (((uintptr_t)kds_src & 7) != 0)
            return XB_ERR(err, ERRCODE_DEVICE_ERROR, "device chunk is not 8-byte aligned");
        XB_CUDA(cudaMemcpy(&head, kds_src, offsetof(kern_data_store, colmeta), cudaMemcpyDeviceToHost), err);
        hb.resize(KDS_HEAD_LENGTH(&head));
        XB_CUDA(cudaMemcpy(hb.data(), kds_src, hb.size(), cudaMemcpyDeviceToHost), err);
    } else {
        hb.assign((const char *)kds_src, (const char *)kds_src + KDS_HEAD_LENGTH(kds_src));
    }
    const kern_data_store *h = (const kern_data_store *)hb.data();
    rc = xb_check_kds(h, err);
    if (rc) return rc;
    if (kds_src_on_device && h->format == KDS_FORMAT_BLOCK &&
        (((uintptr_t)kds_src + h->block_offset) & 15) != 0)
        return XB_ERR(err, ERRCODE_DEVICE_ERROR, "heap pages of a device chunk must start 16-byte aligned");
    {
        std::lock_guard<std::mutex> g(s->lock);
        xb_note_layout(s, h);
    }
    c.s = s;
    c.kds = kds_src;
    c.on_device = kds_src_on_device;
    c.length = h->length;
    c.shift = (!kds_src_on_device && h->format == KDS_FORMAT_BLOCK) ? ((16 - (h->block_offset & 15)) & 15) : 0;
    c.units = xb_chunk_units(h);
    c.format = (uint32_t)h->format;
    xb_sched *q = dev->sched;
    std::lock_guard<std::mutex> g(q->lock);
    c.ticket = q->next_ticket++;
    s->sched_refs++;
    q->pending.push_back(c);
    xb_sched_progress(dev, q);
    *p_ticket = c.ticket;
    return 0;
}

extern "C" int
xpuB200Poll(xpuB200Device *dev, uint64_t ticket, int wait, int *p_done,
            kern_exec_results *results, kern_errorbuf *err)
{
    xb_clear_error(err);
    if (p_done) *p_done = 0;
    if (!dev || !dev->sched)
        return XB_ERR(err, ERRCODE_DEVICE_ERROR, "no command was submitted on this device");
    XB_CUDA(cudaSetDevice(dev->dindex), err);
    xb_sched *q = dev->sched;
    std::unique_lock<std::mutex> lk(q->lock);
    for (;;) {
        xb_sched_progress(dev, q);
        auto it = q->done.find(ticket);
        if (it != q->done.end()) {
            const xb_done d = it->second;
            q->done.erase(it);
            if (p_done) *p_done = 1;
            if (d.rc) {
                if (err) *err = d.err;
                return d.rc;
            }
            xb_fill_results(&d.st, d.nrels, results);
            return 0;
        }
        bool known = ticket > 0 && ticket < q->next_ticket;
        if (known) {
            known = false;
            for (const xb_cmd &c : q->pending)
                if (c.ticket == ticket) known = true;
            for (int i = 0; i < XB_SLOTS && !known; i++)
                for (const xb_cmd &c : q->slot[i].cmds)
                    if (c.ticket == ticket) known = true;
        }
        if (!known)
            return XB_ERR(err, ERRCODE_DEVICE_ERROR, "unknown ticket %llu", (unsigned long long)ticket);
        if (!wait)
            return 0;
        xb_sched_wait_one(q, lk, nullptr);
    }
}

extern "C" int
xpuB200HandleCommand(xpuB200Device *dev, xpuB200Session **p_sess, const XpuCommand *xcmd,
                     const kern_multirels *kmrels, uint64_t kmrels_sz,
                     XpuCommand *resp, uint64_t resp_sz)
{
    kern_errorbuf ebuf;
    int rc = 0;
    if (!xcmd || xcmd->magic != XpuCommandMagicNumber || !resp ||
        resp_sz < offsetof(XpuCommand, u) + sizeof(kern_errorbuf))
        return ERRCODE_DEVICE_ERROR;
    memset(resp, 0, offsetof(XpuCommand, u));
    resp->magic = XpuCommandMagicNumber;
    const uint64_t head = offsetof(XpuCommand, u);
    switch (xcmd->tag) {
    case XpuCommandTag__OpenSession:
        rc = xpuB200OpenSession(dev, &xcmd->u.session, xcmd->length - head, kmrels, kmrels_sz,
                                p_sess, &ebuf);
        if (!rc) {
            resp->tag = XpuCommandTag__Success;
            resp->length = head;
        }
        break;
    case XpuCommandTag__XpuTaskExec: {
        const kern_data_store *kds = (const kern_data_store *)((const char *)xcmd + xcmd->u.task.kds_src_offset);
        if (!*p_sess || xcmd->u.task.kds_src_offset == 0 ||
            xcmd->u.task.kds_src_offset + sizeof(kern_data_store) > xcmd->length ||
            xcmd->u.task.kds_src_offset + kds->length > xcmd->length) {
            rc = XB_ERR(&ebuf, ERRCODE_DEVICE_ERROR, "malformed XpuTaskExec command");
            break;
        }
        uint32_t nrels = (*p_sess)->h_plan->nrels;
        uint64_t rsz = head + offsetof(kern_exec_results, stats) + sizeof(resp->u.results.stats[0]) * (nrels + 1);
        if (resp_sz < rsz) { rc = XB_ERR(&ebuf, ERRCODE_DEVICE_ERROR, "response buffer too small"); break; }
        memset(&resp->u.results, 0, rsz - head);
        resp->u.results.num_rels = nrels;
        if ((*p_sess)->h_plan->has_proj) {
            /* the projected rows follow the results as one KDS_FORMAT_ROW
             * chunk, cut down to header + row index + tuples like
             * __gpuClientWriteBackOneChunk (gpu_service.c:2818-2846) */
            const uint64_t rhead = PGSTROM_MAXALIGN(rsz);
            if (resp_sz < rhead + 64) { rc = XB_ERR(&ebuf, ERRCODE_DEVICE_ERROR, "response buffer too small"); break; }
            char *dst = (char *)resp + rhead;
            const uint64_t len = (resp_sz - rhead) & ~7ULL;
            uint64_t required = 0;
            rc = xpuB200ExecTaskDst(*p_sess, kds, 0, dst, len, 0, &required, &resp->u.results, &ebuf);
            if (rc == ERRCODE_SUSPEND_NO_SPACE) {
                rc = XB_ERR(&ebuf, ERRCODE_DEVICE_ERROR,
                            "response buffer too small for the projected rows (%llu bytes needed)",
                            (unsigned long long)(rhead + required));
                break;
            }
            if (rc) break;
            kern_data_store *kd = (kern_data_store *)dst;
            /* offsets from the end (row index, hash chains) stay valid */
            const uint64_t hsz = KDS_HEAD_LENGTH(kd) + 8 * (uint64_t)kd->hash_nslots +
                                 PGSTROM_MAXALIGN(8 * (uint64_t)kd->nitems);
            if (kd->usage)
                memmove(dst + hsz, dst + len - kd->usage, kd->usage);
            kd->length = hsz + kd->usage;
            resp->u.results.chunks_offset = (uint32_t)rhead;
            resp->u.results.chunks_nitems = 1;
            resp->tag = XpuCommandTag__Success;
            resp->length = rhead + kd->length;
            break;
        }
        rc = xpuB200ExecTask(*p_sess, kds, 0, &resp->u.results, &ebuf);
        if (!rc) {
            resp->tag = XpuCommandTag__Success;
            resp->length = rsz;
        }
        break;
    }
    case XpuCommandTag__XpuTaskFinal: {
        if (!*p_sess) { rc = XB_ERR(&ebuf, ERRCODE_DEVICE_ERROR, "XpuTaskFinal without a session"); break; }
        uint32_t nrels = (*p_sess)->h_plan->nrels;
        uint64_t rhead = head + PGSTROM_MAXALIGN(offsetof(kern_exec_results, stats) +
                                                 sizeof(resp->u.results.stats[0]) * (nrels + 1));
        if (resp_sz < rhead) { rc = XB_ERR(&ebuf, ERRCODE_DEVICE_ERROR, "response buffer too small"); break; }
        memset(&resp->u.results, 0, rhead - head);
        resp->u.results.num_rels = nrels;
        uint64_t required = 0;
        rc = xpuB200Final(*p_sess, (char *)resp + rhead, resp_sz - rhead, &required,
                          &resp->u.results, &ebuf);
        if (!rc) {
            resp->tag = XpuCommandTag__Success;
            resp->u.results.chunks_offset = (uint32_t)rhead;
            resp->u.results.chunks_nitems = required > 0 ? 1 : 0;
            resp->u.results.final_plan_task = true;
            resp->length = rhead + required;
        }
        break;
    }
    default:
        rc = XB_ERR(&ebuf, ERRCODE_DEVICE_ERROR, "unknown XpuCommand tag %u", xcmd->tag);
        break;
    }
    if (rc) {
        resp->tag = XpuCommandTag__Error;
        resp->length = head + sizeof(kern_errorbuf);
        memcpy(&resp->u.error, &ebuf, sizeof(kern_errorbuf));
    }
    return rc;
}

extern "C" int
xpuB200DeviceAlloc(xpuB200Device *dev, uint64_t sz, void **p_dptr)
{
    cudaSetDevice(dev->dindex);
    if (cudaMalloc(p_dptr, sz) != cudaSuccess) { cudaGetLastError(); return ERRCODE_DEVICE_FATAL; }
    return 0;
}

extern "C" int
xpuB200DeviceFree(xpuB200Device *dev, void *dptr)
{
    cudaSetDevice(dev->dindex);
    return cudaFree(dptr) == cudaSuccess ? 0 : ERRCODE_DEVICE_FATAL;
}

extern "C" int
xpuB200InnerCacheConfig(xpuB200Device *dev, uint64_t max_bytes, uint64_t *p_cached_bytes, kern_errorbuf *err)
{
    xb_clear_error(err);
    if (!dev)
        return XB_ERR(err, ERRCODE_DEVICE_ERROR, "invalid InnerCacheConfig arguments");
    XB_CUDA(cudaSetDevice(dev->dindex), err);
    std::lock_guard<std::mutex> g(dev->inner_lock);
    if (max_bytes != UINT64_MAX)
        dev->inner_budget = max_bytes;
    xb_inner_evict_locked(dev);
    if (p_cached_bytes)
        *p_cached_bytes = dev->inner_bytes;
    return 0;
}

/* ----------------------------------------------------------------
 * outer-table chunks resident in HBM across sessions
 * ---------------------------------------------------------------- */
/* drop unused chunks, least recently used first, while the cache holds
 * more than its budget; chunk_lock held */
static void xb_chunk_evict_locked(xpuB200Device *dev)
{
    while (dev->chunk_bytes > dev->chunk_budget) {
        auto victim = dev->chunk_cache.end();
        for (auto it = dev->chunk_cache.begin(); it != dev->chunk_cache.end(); ++it)
            if (it->second.refs == 0 &&
                (victim == dev->chunk_cache.end() || it->second.last_use < victim->second.last_use))
                victim = it;
        if (victim == dev->chunk_cache.end())
            return;                     /* every chunk is in use */
        cudaFreeAsync(victim->second.base, dev->stream);
        dev->chunk_bytes -= victim->second.bytes;
        dev->chunk_cache.erase(victim);
    }
}

extern "C" int
xpuB200ChunkCachePut(xpuB200Device *dev, uint64_t table_handle, uint32_t chunk_no,
                     const kern_data_store *kds, int kds_on_device,
                     const kern_data_store **p_kds_dev, kern_errorbuf *err)
{
    xb_clear_error(err);
    if (!dev || !kds || !p_kds_dev)
        return XB_ERR(err, ERRCODE_DEVICE_ERROR, "invalid ChunkCachePut arguments");
    XB_CUDA(cudaSetDevice(dev->dindex), err);
    std::lock_guard<std::mutex> g(dev->chunk_lock);
    const auto key = std::make_pair(table_handle, chunk_no);
    auto it = dev->chunk_cache.find(key);
    if (it != dev->chunk_cache.end()) {
        it->second.refs++;
        it->second.last_use = ++dev->chunk_clock;
        *p_kds_dev = it->second.kds;
        return 0;
    }
    /* the header, to place the chunk and check it */
    std::vector<char> hb(offsetof(kern_data_store, colmeta));
    if (kds_on_device) {
        XB_CUDA(cudaMemcpy(hb.data(), kds, hb.size(), cudaMemcpyDeviceToHost), err);
        const kern_data_store *h = (const kern_data_store *)hb.data();
        hb.resize(KDS_HEAD_LENGTH(h));
        XB_CUDA(cudaMemcpy(hb.data(), kds, hb.size(), cudaMemcpyDeviceToHost), err);
    } else {
        hb.assign((const char *)kds, (const char *)kds + KDS_HEAD_LENGTH(kds));
    }
    const kern_data_store *h = (const kern_data_store *)hb.data();
    int rc = xb_check_kds(h, err);
    if (rc) return rc;
    /* heap pages start 16-byte aligned on the device */
    const uint64_t shift = h->format == KDS_FORMAT_BLOCK ? (16 - (h->block_offset & 15)) & 15 : 0;
    const uint64_t bytes = h->length + shift;
    char *base = nullptr;
    if (cudaMallocAsync((void **)&base, bytes, dev->stream) != cudaSuccess) {
        cudaGetLastError();
        return XB_ERR(err, ERRCODE_DEVICE_FATAL, "out of device memory for a resident chunk of %llu bytes",
                      (unsigned long long)h->length);
    }
    XB_CUDA(cudaMemcpyAsync(base + shift, kds, h->length,
                            kds_on_device ? cudaMemcpyDeviceToDevice : cudaMemcpyHostToDevice, dev->stream), err);
    /* the chunk is complete before any other stream reads it */
    XB_CUDA(cudaStreamSynchronize(dev->stream), err);
    xb_chunk_entry e;
    e.base = base;
    e.kds = (const kern_data_store *)(base + shift);
    e.bytes = bytes;
    e.refs = 1;
    e.last_use = ++dev->chunk_clock;
    dev->chunk_cache[key] = e;
    dev->chunk_bytes += bytes;
    xb_chunk_evict_locked(dev);
    *p_kds_dev = e.kds;
    return 0;
}

extern "C" int
xpuB200ChunkCacheGet(xpuB200Device *dev, uint64_t table_handle, uint32_t chunk_no,
                     const kern_data_store **p_kds_dev)
{
    if (!dev || !p_kds_dev)
        return ERRCODE_DEVICE_ERROR;
    std::lock_guard<std::mutex> g(dev->chunk_lock);
    auto it = dev->chunk_cache.find(std::make_pair(table_handle, chunk_no));
    if (it == dev->chunk_cache.end())
        return 1;
    it->second.refs++;
    it->second.last_use = ++dev->chunk_clock;
    *p_kds_dev = it->second.kds;
    return 0;
}

extern "C" int
xpuB200ChunkCacheRelease(xpuB200Device *dev, const kern_data_store *kds_dev)
{
    if (!dev)
        return ERRCODE_DEVICE_ERROR;
    cudaSetDevice(dev->dindex);
    std::lock_guard<std::mutex> g(dev->chunk_lock);
    for (auto &kv : dev->chunk_cache) {
        if (kv.second.kds == kds_dev && kv.second.refs > 0) {
            kv.second.refs--;
            xb_chunk_evict_locked(dev);
            return 0;
        }
    }
    return ERRCODE_DEVICE_ERROR;
}

extern "C" int
xpuB200ChunkCacheConfig(xpuB200Device *dev, uint64_t max_bytes, uint64_t *p_cached_bytes, kern_errorbuf *err)
{
    xb_clear_error(err);
    if (!dev)
        return XB_ERR(err, ERRCODE_DEVICE_ERROR, "invalid device");
    XB_CUDA(cudaSetDevice(dev->dindex), err);
    std::lock_guard<std::mutex> g(dev->chunk_lock);
    if (max_bytes != UINT64_MAX) {
        dev->chunk_budget = max_bytes;
        xb_chunk_evict_locked(dev);
    }
    if (p_cached_bytes)
        *p_cached_bytes = dev->chunk_bytes;
    return 0;
}

