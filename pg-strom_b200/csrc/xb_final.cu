/*
 * xb_final.cu
 *
 * Host services of the final stage, over the kernels of the device
 * translation unit (xb_exec.cu, declared in xb_final.h):
 *
 *   xpuB200Final        kds_final in the reference layout, with GPU-Sort /
 *                       LIMIT / window rank of the groups
 *   xpuB200MergeFinal   another kds_final merged into a session's groups
 *   xpuB200FinalParts   the groups as hash partitions for the exchange step
 *   xpuB200InnerRebuild rows appended into a KDS_FORMAT_HASH inner buffer
 */
#include <cuda_runtime.h>
#include <algorithm>
#include <mutex>
#include <vector>
#include <cstring>
#include <cstdio>
#include "xb_plan.h"
#include "xb_exec_dev.cuh"
#include "xb_sort.cuh"
#include "xpu_b200.h"
#include "xb_host.h"
#include "xb_final.h"

/* GPU-Sort of the session's groups: *p_keep receives, per group-table
 * entry, the group's output position or -1 (dropped by LIMIT or the window
 * rank).  fa carries the table and the flag arrays; alloc places device
 * memory that the caller frees.  Returns 0, or -1 when out of memory. */
template <typename Alloc>
static int xb_final_sort(xpuB200Session *s, XbFinalArgs fa, cudaStream_t st, Alloc alloc, int64_t **p_keep)
{
    const xb_plan *plan = s->h_plan;
    const uint64_t cap = fa.cap;
    const int grid = s->dev->nsm * 8;
    fa.keep = nullptr;
    xb_final_sizes<<<grid, XB_BLOCK, 0, st>>>(fa);              /* flags of every group */
    void *d_t = nullptr;
    if (!alloc(xb_scan_temp_bytes<uint32_t>(cap), &d_t)) return -1;
    if (xb_scan<uint32_t, XbOpSum, true>(fa.flags, fa.flag_scan, cap, d_t, st) != cudaSuccess) return -1;
    uint32_t lf = 0, ls = 0;
    cudaMemcpyAsync(&lf, fa.flags + cap - 1, 4, cudaMemcpyDeviceToHost, st);
    cudaMemcpyAsync(&ls, fa.flag_scan + cap - 1, 4, cudaMemcpyDeviceToHost, st);
    if (cudaStreamSynchronize(st) != cudaSuccess) return -1;
    const uint32_t n = lf + ls;
    int64_t *keep = nullptr;
    if (!alloc(cap * 8, (void **)&keep)) return -1;
    cudaMemsetAsync(keep, 0xff, cap * 8, st);
    *p_keep = keep;
    if (n == 0)
        return 0;
    const uint32_t nk = plan->nsort;
    uint32_t *ents, *idx, *idx2, *part, *peer, *pflag, *pcnt, *kflag, *kscan;
    uint64_t *keyw, *k64a, *k64b;
    uint8_t *nul, *k8a, *k8b;
    if (!alloc((size_t)n * 4, (void **)&ents) || !alloc((size_t)n * 4, (void **)&idx) ||
        !alloc((size_t)n * 4, (void **)&idx2) || !alloc((size_t)n * 16 * nk, (void **)&keyw) ||
        !alloc((size_t)n * nk, (void **)&nul) || !alloc((size_t)n * 8, (void **)&k64a) ||
        !alloc((size_t)n * 8, (void **)&k64b) || !alloc((size_t)n, (void **)&k8a) ||
        !alloc((size_t)n, (void **)&k8b) || !alloc((size_t)n * 4, (void **)&part) ||
        !alloc((size_t)n * 4, (void **)&peer) || !alloc((size_t)n * 4, (void **)&pflag) ||
        !alloc((size_t)n * 4, (void **)&pcnt) || !alloc((size_t)n * 4, (void **)&kflag) ||
        !alloc((size_t)n * 4, (void **)&kscan))
        return -1;
    XbSortArgs sa;
    sa.plan = s->d_plan;
    sa.gt = s->d_gt;
    sa.cap = cap;
    sa.flags = fa.flags;
    sa.flag_scan = fa.flag_scan;
    sa.ents = ents;
    sa.keyw = keyw;
    sa.nul = nul;
    sa.n = n;
    int g2 = (int)((n + XB_BLOCK - 1) / XB_BLOCK);
    if (g2 > grid) g2 = grid;
    xb_sort_gather<<<grid, XB_BLOCK, 0, st>>>(sa);
    xb_sort_keys<<<g2, XB_BLOCK, 0, st>>>(sa);
    xb_iota_u32<<<g2, XB_BLOCK, 0, st>>>(idx, n);
    /* temporary storage for the largest of the sort and scan passes */
    const size_t tt = std::max(xb_radix_temp_bytes(n), xb_scan_temp_bytes<uint32_t>(n));
    void *d_tt = nullptr;
    if (!alloc(tt, &d_tt)) return -1;
    /* stable passes, least significant first: for each key from the last,
     * its low word, its high word, then its NULL flag (each a stable radix
     * sort of the word gathered in the current order, carrying the group
     * indexes along) */
    for (int k = (int)nk - 1; k >= 0; k--) {
        for (int w = 1; w >= 0; w--) {
            if (w == 1 && plan->sort[k].words < 2)
                continue;
            xb_sort_pass_key64<<<g2, XB_BLOCK, 0, st>>>(keyw + (2ULL * k + w) * n, idx, k64a, n);
            if (xb_radix_sort<uint64_t>(k64a, k64b, idx, idx2, n, 64, d_tt, st) != cudaSuccess) return -1;
        }
        xb_sort_pass_key8<<<g2, XB_BLOCK, 0, st>>>(nul + (uint64_t)k * n, idx, k8a, n);
        if (xb_radix_sort<uint8_t>(k8a, k8b, idx, idx2, n, 8, d_tt, st) != cudaSuccess) return -1;
    }
    XbRankArgs ra;
    ra.plan = s->d_plan;
    ra.idx = idx;
    ra.keyw = keyw;
    ra.nul = nul;
    ra.n = n;
    ra.part_start = part;
    ra.peer_start = peer;
    ra.peer_flag = pflag;
    if (plan->sort_window) {
        xb_sort_bounds<<<g2, XB_BLOCK, 0, st>>>(ra);
        if (xb_scan<uint32_t, XbOpMax, false>(part, part, n, d_tt, st) != cudaSuccess ||
            xb_scan<uint32_t, XbOpMax, false>(peer, peer, n, d_tt, st) != cudaSuccess ||
            xb_scan<uint32_t, XbOpSum, false>(pflag, pcnt, n, d_tt, st) != cudaSuccess)
            return -1;
    }
    XbKeepArgs ka;
    ka.plan = s->d_plan;
    ka.idx = idx;
    ka.ents = ents;
    ka.n = n;
    ka.part_start = part;
    ka.peer_start = peer;
    ka.peer_cnt = pcnt;
    ka.keep_flag = kflag;
    xb_sort_keepflag<<<g2, XB_BLOCK, 0, st>>>(ka);
    if (xb_scan<uint32_t, XbOpSum, true>(kflag, kscan, n, d_tt, st) != cudaSuccess) return -1;
    xb_sort_keep<<<g2, XB_BLOCK, 0, st>>>(ka, kscan, keep);
    return cudaGetLastError() == cudaSuccess ? 0 : -1;
}

extern "C" int
xpuB200Final(xpuB200Session *s, void *kds_final_buf, uint64_t buf_sz, uint64_t *p_required,
             kern_exec_results *results, kern_errorbuf *err)
{
    xb_clear_error(err);
    if (!s)
        return XB_ERR(err, ERRCODE_DEVICE_ERROR, "invalid Final arguments");
    xb_sched_drain_session(s);
    std::lock_guard<std::mutex> g(s->lock);
    XB_CUDA(cudaSetDevice(s->dev->dindex), err);
    cudaStream_t st = s->stream;
    const xb_plan *plan = s->h_plan;
    if (results) {
        uint32_t cap = results->num_rels;
        results->nitems_raw = (uint32_t)s->total_raw;
        results->nitems_in = (uint32_t)s->total_in;
        results->nitems_out = (uint32_t)s->total_out;
        results->num_rels = plan->nrels;
        for (uint32_t d = 1; d <= plan->nrels && d <= cap; d++)
            results->stats[d - 1].nitems_out = (uint32_t)s->total_depth[d];
        results->final_plan_task = true;
    }
    if (!plan->has_groupby) {
        if (p_required) *p_required = 0;
        return 0;
    }
    /* groups waiting in the dump region join the table first */
    int src = xb_gt_settle(s, err);
    if (src) return src;
    const kern_session_info *session = (const kern_session_info *)s->h_session.data();
    const kern_data_store *fh = (const kern_data_store *)(s->h_session.data() + session->groupby_kds_final);
    const uint64_t head_len = KDS_HEAD_LENGTH(fh);
    const uint64_t cap = s->h_gt.cap_mask + 1;
    const bool row_fmt = fh->format == KDS_FORMAT_ROW;

    uint64_t *d_sizes = nullptr, *d_size_scan = nullptr;
    uint32_t *d_flags = nullptr, *d_flag_scan = nullptr;
    char *d_out = nullptr;
    void *d_temp = nullptr;
    int rc = 0;
    std::vector<void *> tmp;
    auto alloc = [&](size_t sz, void **p) -> bool {
        if (cudaMallocAsync(p, sz < 256 ? 256 : sz, st) != cudaSuccess) { cudaGetLastError(); return false; }
        tmp.push_back(*p);
        return true;
    };
    auto cleanup = [&]() { for (void *p : tmp) cudaFreeAsync(p, st); };
    if (!alloc(cap * 8, (void **)&d_sizes) || !alloc(cap * 8, (void **)&d_size_scan) ||
        !alloc(cap * 4, (void **)&d_flags) || !alloc(cap * 4, (void **)&d_flag_scan)) {
        cleanup();
        return XB_ERR(err, ERRCODE_DEVICE_FATAL, "out of device memory in Final");
    }
    XbFinalArgs fa;
    memset(&fa, 0, sizeof(fa));
    fa.plan = s->d_plan;
    fa.gt = s->d_gt;
    fa.cap = cap;
    fa.sizes = d_sizes;
    fa.flags = d_flags;
    fa.size_scan = d_size_scan;
    fa.flag_scan = d_flag_scan;
    fa.row_format = row_fmt ? 1 : 0;
    int grid = s->dev->nsm * 8;
    if (plan->nsort) {
        int64_t *d_keep = nullptr;
        if (xb_final_sort(s, fa, st, alloc, &d_keep) != 0) {
            cleanup();
            return XB_ERR(err, ERRCODE_DEVICE_FATAL, "GPU-Sort of the groups failed (%s)",
                          cudaGetErrorString(cudaGetLastError()));
        }
        fa.keep = d_keep;
    }
    /* the global table's entries pointer lives in h_gt */
    xb_final_sizes<<<grid, XB_BLOCK, 0, st>>>(fa);
    if (!alloc(xb_scan_temp_bytes<uint64_t>(cap), &d_temp)) {
        cleanup();
        return XB_ERR(err, ERRCODE_DEVICE_FATAL, "out of device memory in Final");
    }
    xb_scan<uint64_t, XbOpSum, true>(d_sizes, d_size_scan, cap, d_temp, st);
    xb_scan<uint32_t, XbOpSum, true>(d_flags, d_flag_scan, cap, d_temp, st);
    uint64_t last_size = 0, last_scan = 0;
    uint32_t last_flag = 0, last_fscan = 0;
    cudaMemcpyAsync(&last_size, d_sizes + cap - 1, 8, cudaMemcpyDeviceToHost, st);
    cudaMemcpyAsync(&last_scan, d_size_scan + cap - 1, 8, cudaMemcpyDeviceToHost, st);
    cudaMemcpyAsync(&last_flag, d_flags + cap - 1, 4, cudaMemcpyDeviceToHost, st);
    cudaMemcpyAsync(&last_fscan, d_flag_scan + cap - 1, 4, cudaMemcpyDeviceToHost, st);
    if (cudaStreamSynchronize(st) != cudaSuccess) {
        cleanup();
        return XB_ERR(err, ERRCODE_DEVICE_FATAL, "Final: %s", cudaGetErrorString(cudaGetLastError()));
    }
    const uint64_t items = last_scan + last_size;
    const uint64_t ngroups = (uint64_t)last_fscan + last_flag;
    const uint64_t nslots = row_fmt ? 0 : KDS_GET_HASHSLOT_WIDTH(ngroups);
    const uint64_t items_base = head_len + 8 * nslots + 8 * ngroups;
    const uint64_t length = items_base + items;
    if (p_required) *p_required = length;
    if (results) {
        results->final_nitems = (uint32_t)ngroups;
        results->final_usage = items;
        results->final_total = length;
    }
    if (!kds_final_buf || buf_sz < length) {
        cleanup();
        if (!kds_final_buf && buf_sz == 0)
            return 0;           /* size query only */
        return XB_ERR(err, ERRCODE_SUSPEND_NO_SPACE, "kds_final needs %llu bytes (buffer %llu)",
                      (unsigned long long)length, (unsigned long long)buf_sz);
    }
    if (!alloc(length, (void **)&d_out)) {
        cleanup();
        return XB_ERR(err, ERRCODE_DEVICE_FATAL, "out of device memory for kds_final (%llu bytes)",
                      (unsigned long long)length);
    }
    /* header: the session's kds_final definition with the actual sizes */
    std::vector<char> head((const char *)fh, (const char *)fh + head_len);
    kern_data_store *kh = (kern_data_store *)head.data();
    kh->length = length;
    kh->usage = items;
    kh->nitems = (uint32_t)ngroups;
    kh->format = row_fmt ? KDS_FORMAT_ROW : KDS_FORMAT_HASH;
    kh->hash_nslots = (uint32_t)nslots;
    cudaMemcpyAsync(d_out, head.data(), head_len, cudaMemcpyHostToDevice, st);
    /* slots, row index and items: the padding between and after the
     * tuples' attributes is zero, so equal results are equal bytes */
    cudaMemsetAsync(d_out + head_len, 0, length - head_len, st);
    fa.kds_final = d_out;
    fa.items_base = items_base;
    fa.length = length;
    fa.nslots = (uint32_t)nslots;
    xb_final_write<<<grid, XB_BLOCK, 0, st>>>(fa);
    cudaMemcpyAsync(kds_final_buf, d_out, length, cudaMemcpyDeviceToHost, st);
    if (cudaStreamSynchronize(st) != cudaSuccess)
        rc = XB_ERR(err, ERRCODE_DEVICE_FATAL, "Final: %s", cudaGetErrorString(cudaGetLastError()));
    cleanup();
    return rc;
}

extern "C" int
xpuB200MergeFinal(xpuB200Session *s, const kern_data_store *kds_final, int kds_final_on_device,
                  kern_errorbuf *err)
{
    xb_clear_error(err);
    if (!s || !kds_final)
        return XB_ERR(err, ERRCODE_DEVICE_ERROR, "invalid MergeFinal arguments");
    xb_sched_drain_session(s);
    std::lock_guard<std::mutex> g(s->lock);
    const xb_plan *plan = s->h_plan;
    if (!plan->has_groupby)
        return XB_ERR(err, ERRCODE_DEVICE_ERROR, "the session has no GROUP BY");
    XB_CUDA(cudaSetDevice(s->dev->dindex), err);
    cudaStream_t st = s->stream;
    /* the header, checked on the host */
    kern_data_store head;
    std::vector<char> hb;
    if (kds_final_on_device) {
        XB_CUDA(cudaMemcpy(&head, kds_final, offsetof(kern_data_store, colmeta), cudaMemcpyDeviceToHost), err);
        hb.resize(KDS_HEAD_LENGTH(&head));
        XB_CUDA(cudaMemcpy(hb.data(), kds_final, hb.size(), cudaMemcpyDeviceToHost), err);
    } else {
        hb.assign((const char *)kds_final, (const char *)kds_final + KDS_HEAD_LENGTH(kds_final));
    }
    const kern_data_store *h = (const kern_data_store *)hb.data();
    const kern_session_info *session = (const kern_session_info *)s->h_session.data();
    const char fmt = ((const kern_data_store *)(s->h_session.data() + session->groupby_kds_final))->format;
    if (h->format != fmt || h->ncols != plan->naggs || (fmt == KDS_FORMAT_ROW && h->hash_nslots != 0) ||
        KDS_HEAD_LENGTH(h) + 8 * ((uint64_t)h->hash_nslots + h->nitems) > h->length)
        return XB_ERR(err, ERRCODE_DEVICE_ERROR, "kds_final to merge is not this session's KDS_FORMAT_%s",
                      fmt == KDS_FORMAT_ROW ? "ROW" : "HASH");
    if (h->nitems == 0)
        return 0;
    if (plan->gent_size > XB_GENT_MAX)
        return XB_ERR(err, ERRCODE_DEVICE_ERROR, "group entries of %u bytes cannot be merged", plan->gent_size);
    const kern_data_store *d_kds = kds_final;
    char *d_copy = nullptr;
    if (!kds_final_on_device) {
        XB_CUDA(cudaMallocAsync((void **)&d_copy, h->length, st), err);
        XB_CUDA(cudaMemcpyAsync(d_copy, kds_final, h->length, cudaMemcpyHostToDevice, st), err);
        d_kds = (const kern_data_store *)d_copy;
    }
    /* room for every incoming group before the merge (the table grows as
     * for chunk launches when it would pass half of its slots) */
    {
        xb_gtable gh;
        int rc = xb_gt_read(s, &gh, err);
        if (!rc && (gh.dump_used || gh.nused + h->nitems > gh.soft_cap))
            rc = xb_gt_grow(s, gh.nused + h->nitems, err);
        if (rc) {
            if (d_copy) cudaFreeAsync(d_copy, st);
            return rc;
        }
    }
    XB_CUDA(cudaMemsetAsync(s->d_status, 0, sizeof(xb_status), st), err);
    XbMergeArgs ma;
    ma.plan = s->d_plan;
    ma.kds = d_kds;
    ma.gt = s->d_gt;
    ma.st = s->d_status;
    int grid = (int)((h->nitems + XB_BLOCK - 1) / XB_BLOCK);
    if (grid > s->dev->nsm * 8) grid = s->dev->nsm * 8;
    xb_merge_final<<<grid, XB_BLOCK, 0, st>>>(ma);
    if (d_copy)
        cudaFreeAsync(d_copy, st);
    int mrc = xb_wait_status(s, err);
    if (mrc) return mrc;
    return xb_gt_settle(s, err);
}

/* ----------------------------------------------------------------
 * the session's groups as hash partitions, for the exchange step of a
 * multi-GPU pre-aggregation: part p holds the groups whose hash % nparts
 * is p, as a KDS_FORMAT_HASH kds_final of its own (the same layout as
 * xpuB200Final's).  The parts lie back to back in one device buffer the
 * caller owns, each at a 256-byte aligned offset, so that the buffer can
 * be handed to the other GPUs whole (CUDA IPC, or NCCL all-to-all); each
 * GPU then merges the parts destined for it with xpuB200MergeFinal,
 * reading them in place from the peer's memory.
 * ---------------------------------------------------------------- */
extern "C" int
xpuB200FinalParts(xpuB200Session *s, uint32_t nparts, void *parts_dev, uint64_t buf_sz,
                  uint64_t *part_offsets, uint64_t *p_required, kern_errorbuf *err)
{
    xb_clear_error(err);
    if (!s || nparts < 1 || nparts > 4096 || !part_offsets)
        return XB_ERR(err, ERRCODE_DEVICE_ERROR, "invalid FinalParts arguments");
    xb_sched_drain_session(s);
    std::lock_guard<std::mutex> g(s->lock);
    XB_CUDA(cudaSetDevice(s->dev->dindex), err);
    const xb_plan *plan = s->h_plan;
    if (plan->has_groupby != 1)
        return XB_ERR(err, ERRCODE_DEVICE_ERROR, "FinalParts needs a session with GROUP BY keys");
    if (plan->nsort)
        return XB_ERR(err, ERRCODE_DEVICE_ERROR, "GPU-Sort applies to the merged groups, not to their parts");
    int rc = xb_gt_settle(s, err);
    if (rc) return rc;
    cudaStream_t st = s->stream;
    const kern_session_info *session = (const kern_session_info *)s->h_session.data();
    const kern_data_store *fh = (const kern_data_store *)(s->h_session.data() + session->groupby_kds_final);
    const uint64_t head_len = KDS_HEAD_LENGTH(fh);
    const uint64_t cap = s->h_gt.cap_mask + 1;
    std::vector<void *> tmp;
    auto cleanup = [&]() { for (void *p : tmp) cudaFreeAsync(p, st); };
    auto alloc = [&](size_t sz, void **p) -> bool {
        if (cudaMallocAsync(p, sz < 256 ? 256 : sz, st) != cudaSuccess) { cudaGetLastError(); return false; }
        tmp.push_back(*p);
        return true;
    };
    uint64_t *d_sizes, *d_size_scan;
    uint32_t *d_flags, *d_flag_scan;
    void *d_temp = nullptr;
    if (!alloc(cap * 8, (void **)&d_sizes) || !alloc(cap * 8, (void **)&d_size_scan) ||
        !alloc(cap * 4, (void **)&d_flags) || !alloc(cap * 4, (void **)&d_flag_scan)) {
        cleanup();
        return XB_ERR(err, ERRCODE_DEVICE_FATAL, "out of device memory in FinalParts");
    }
    const size_t tsz_max = xb_scan_temp_bytes<uint64_t>(cap);
    if (!alloc(tsz_max, &d_temp)) {
        cleanup();
        return XB_ERR(err, ERRCODE_DEVICE_FATAL, "out of device memory in FinalParts");
    }
    XbFinalArgs fa;
    memset(&fa, 0, sizeof(fa));
    fa.plan = s->d_plan;
    fa.gt = s->d_gt;
    fa.cap = cap;
    fa.sizes = d_sizes;
    fa.flags = d_flags;
    fa.size_scan = d_size_scan;
    fa.flag_scan = d_flag_scan;
    fa.part_div = nparts;
    const int grid = s->dev->nsm * 8;
    /* sizes of part p (its items and groups) into the arrays */
    auto size_part = [&](uint32_t p, uint64_t *p_items, uint64_t *p_groups) -> int {
        fa.part_rem = p;
        xb_final_sizes<<<grid, XB_BLOCK, 0, st>>>(fa);
        xb_scan<uint64_t, XbOpSum, true>(d_sizes, d_size_scan, cap, d_temp, st);
        xb_scan<uint32_t, XbOpSum, true>(d_flags, d_flag_scan, cap, d_temp, st);
        uint64_t last_size = 0, last_scan = 0;
        uint32_t last_flag = 0, last_fscan = 0;
        cudaMemcpyAsync(&last_size, d_sizes + cap - 1, 8, cudaMemcpyDeviceToHost, st);
        cudaMemcpyAsync(&last_scan, d_size_scan + cap - 1, 8, cudaMemcpyDeviceToHost, st);
        cudaMemcpyAsync(&last_flag, d_flags + cap - 1, 4, cudaMemcpyDeviceToHost, st);
        cudaMemcpyAsync(&last_fscan, d_flag_scan + cap - 1, 4, cudaMemcpyDeviceToHost, st);
        if (cudaStreamSynchronize(st) != cudaSuccess)
            return -1;
        *p_items = last_scan + last_size;
        *p_groups = (uint64_t)last_fscan + last_flag;
        return 0;
    };
    std::vector<uint64_t> items(nparts), groups(nparts);
    uint64_t total = 0;
    for (uint32_t p = 0; p < nparts; p++) {
        if (size_part(p, &items[p], &groups[p]) != 0) {
            cleanup();
            return XB_ERR(err, ERRCODE_DEVICE_FATAL, "FinalParts: %s", cudaGetErrorString(cudaGetLastError()));
        }
        const uint64_t nslots = KDS_GET_HASHSLOT_WIDTH(groups[p]);
        part_offsets[p] = total;
        total += xb_align256(head_len + 8 * nslots + 8 * groups[p] + items[p]);
    }
    part_offsets[nparts] = total;
    if (p_required) *p_required = total;
    if (!parts_dev || buf_sz < total) {
        cleanup();
        if (!parts_dev && buf_sz == 0)
            return 0;           /* size query only */
        return XB_ERR(err, ERRCODE_SUSPEND_NO_SPACE, "the parts need %llu bytes (buffer %llu)",
                      (unsigned long long)total, (unsigned long long)buf_sz);
    }
    std::vector<char> head((const char *)fh, (const char *)fh + head_len);
    for (uint32_t p = 0; p < nparts; p++) {
        uint64_t it, ng;
        if (size_part(p, &it, &ng) != 0) {
            cleanup();
            return XB_ERR(err, ERRCODE_DEVICE_FATAL, "FinalParts: %s", cudaGetErrorString(cudaGetLastError()));
        }
        const uint64_t nslots = KDS_GET_HASHSLOT_WIDTH(ng);
        const uint64_t items_base = head_len + 8 * nslots + 8 * ng;
        const uint64_t length = items_base + it;
        char *d_out = (char *)parts_dev + part_offsets[p];
        kern_data_store *kh = (kern_data_store *)head.data();
        kh->length = length;
        kh->usage = it;
        kh->nitems = (uint32_t)ng;
        kh->format = KDS_FORMAT_HASH;
        kh->hash_nslots = (uint32_t)nslots;
        cudaMemcpyAsync(d_out, head.data(), head_len, cudaMemcpyHostToDevice, st);
        cudaMemsetAsync(d_out + head_len, 0, length - head_len, st);
        fa.kds_final = d_out;
        fa.items_base = items_base;
        fa.length = length;
        fa.nslots = (uint32_t)nslots;
        xb_final_write<<<grid, XB_BLOCK, 0, st>>>(fa);
        /* the host header copy must outlive the copy: wait per part */
        if (cudaStreamSynchronize(st) != cudaSuccess) {
            cleanup();
            return XB_ERR(err, ERRCODE_DEVICE_FATAL, "FinalParts: %s", cudaGetErrorString(cudaGetLastError()));
        }
    }
    cleanup();
    return 0;
}

extern "C" int
xpuB200InnerRebuild(xpuB200Device *dev, kern_data_store *kds_dst, const kern_data_store *kds_src,
                    uint32_t hash_divisor, uint32_t hash_remainder, uint64_t *p_required, kern_errorbuf *err)
{
    xb_clear_error(err);
    if (!dev || !kds_dst || !kds_src || (hash_divisor >= 2 && hash_remainder >= hash_divisor))
        return XB_ERR(err, ERRCODE_DEVICE_ERROR, "invalid InnerRebuild arguments");
    if (((uintptr_t)kds_dst & 7) != 0 || ((uintptr_t)kds_src & 7) != 0)
        return XB_ERR(err, ERRCODE_DEVICE_ERROR, "InnerRebuild buffers must be 8-byte aligned");
    XB_CUDA(cudaSetDevice(dev->dindex), err);
    kern_data_store hd, hs;
    XB_CUDA(cudaMemcpy(&hd, kds_dst, offsetof(kern_data_store, colmeta), cudaMemcpyDeviceToHost), err);
    XB_CUDA(cudaMemcpy(&hs, kds_src, offsetof(kern_data_store, colmeta), cudaMemcpyDeviceToHost), err);
    if (hd.format != KDS_FORMAT_HASH || hd.hash_nslots == 0 || hd.nr_colmeta > 4096 ||
        (hd.length & 7) != 0 || (hd.usage & 7) != 0 ||
        KDS_HEAD_LENGTH(&hd) + 8ULL * ((uint64_t)hd.hash_nslots + hd.nitems) + hd.usage > hd.length)
        return XB_ERR(err, ERRCODE_DEVICE_ERROR, "InnerRebuild destination is not a KDS_FORMAT_HASH buffer");
    if ((hs.format != KDS_FORMAT_HASH && hs.format != KDS_FORMAT_ROW) || hs.nr_colmeta > 4096 ||
        (hs.length & 7) != 0)
        return XB_ERR(err, ERRCODE_DEVICE_ERROR, "InnerRebuild source must be KDS_FORMAT_HASH or _ROW");
    if (hd.ncols != hs.ncols)
        return XB_ERR(err, ERRCODE_DEVICE_ERROR, "InnerRebuild source has %u columns, destination %u",
                      hs.ncols, hd.ncols);
    const uint64_t src_rowidx = KDS_HEAD_LENGTH(&hs) + (hs.format == KDS_FORMAT_HASH ? 8ULL * hs.hash_nslots : 0);
    if (src_rowidx + 8ULL * hs.nitems > hs.length)
        return XB_ERR(err, ERRCODE_DEVICE_ERROR, "InnerRebuild source row index is out of the buffer");
    if (hs.nitems == 0) {
        if (p_required)
            *p_required = KDS_HEAD_LENGTH(&hd) + 8ULL * (hd.hash_nslots + hd.nitems) + hd.usage;
        return 0;
    }
    cudaStream_t st = xb_get_stream(dev);
    if (!st)
        return XB_ERR(err, ERRCODE_DEVICE_FATAL, "no stream");
    uint32_t *d_flag = nullptr;
    int rc = 0;
    if (cudaMallocAsync((void **)&d_flag, sizeof(uint32_t), st) != cudaSuccess) {
        xb_put_stream(dev, st);
        return XB_ERR(err, ERRCODE_DEVICE_FATAL, "out of device memory");
    }
    cudaMemsetAsync(d_flag, 0, sizeof(uint32_t), st);
    XbRebuildArgs ra;
    ra.dst = kds_dst;
    ra.src = kds_src;
    ra.dst_head = KDS_HEAD_LENGTH(&hd);
    ra.src_rowidx = src_rowidx;
    ra.divisor = hash_divisor;
    ra.remainder = hash_remainder;
    ra.overflow = d_flag;
    int grid = (int)((hs.nitems + XB_BLOCK - 1) / XB_BLOCK);
    if (grid > dev->nsm * 8) grid = dev->nsm * 8;
    xb_inner_rebuild<<<grid, XB_BLOCK, 0, st>>>(ra);
    uint32_t flag = 0;
    cudaMemcpyAsync(&flag, d_flag, sizeof(uint32_t), cudaMemcpyDeviceToHost, st);
    cudaMemcpyAsync(&hd, kds_dst, offsetof(kern_data_store, colmeta), cudaMemcpyDeviceToHost, st);
    cudaFreeAsync(d_flag, st);
    if (cudaStreamSynchronize(st) != cudaSuccess)
        rc = XB_ERR(err, ERRCODE_DEVICE_FATAL, "InnerRebuild: %s", cudaGetErrorString(cudaGetLastError()));
    xb_put_stream(dev, st);
    if (rc)
        return rc;
    const uint64_t required = KDS_HEAD_LENGTH(&hd) + 8ULL * (hd.hash_nslots + hd.nitems) + hd.usage;
    if (p_required)
        *p_required = required;
    if (flag & 2u)
        return XB_ERR(err, ERRCODE_DEVICE_ERROR, "InnerRebuild source has a broken row");
    /* rows claimed concurrently fit only when all of them do */
    if ((flag & 1u) || required > hd.length)
        return XB_ERR(err, ERRCODE_SUSPEND_NO_SPACE, "InnerRebuild destination needs %llu bytes (buffer %llu)",
                      (unsigned long long)required, (unsigned long long)hd.length);
    return 0;
}

