/*
 * xb_direct.cpp
 *
 * Chunk ingest from storage straight into device memory: the pages of a
 * relation (or Arrow) file that an I/O vector names are read into a device
 * buffer with the public cuFile API (GPUDirect Storage), the way the GPU
 * service fills a KDS_FORMAT_BLOCK chunk from the file before the kernel
 * runs (__gpuservLoadKdsCommon, gpu_service.c:3415-3466, through
 * gpuDirectFileReadIOV, extra.c:569-630, whose cuFile reader lives in the
 * closed heterodb_extra library).  libcufile is bound at run time; where
 * it is absent or its driver cannot open, and for pages cuFile does not
 * read, the pages go through a pinned bounce buffer (the VFS path of the
 * reference, __fallbackFileReadIOV, extra.c:490-566).
 */
#include <cuda_runtime.h>
#include <dlfcn.h>
#include <fcntl.h>
#include <unistd.h>
#include <cstdio>
#include <cstdlib>
#include <cstring>
#include <mutex>
#include <string>
#include "xpu_b200.h"

namespace {

/* the cuFile entry points used here (cufile.h), bound with dlsym */
typedef struct { int err; int cu_err; } xb_cufile_error;
typedef struct {
    int type;                       /* CU_FILE_HANDLE_TYPE_OPAQUE_FD = 1 */
    union { int fd; void *handle; } handle;
    const void *fs_ops;
} xb_cufile_descr;

struct CuFile {
    bool tried = false;
    bool ok = false;
    std::string why;
    xb_cufile_error (*driver_open)(void) = nullptr;
    xb_cufile_error (*handle_register)(void **, xb_cufile_descr *) = nullptr;
    void (*handle_deregister)(void *) = nullptr;
    ssize_t (*read)(void *, void *, size_t, off_t, off_t) = nullptr;
};
CuFile g_cf;
std::mutex g_cf_lock;

void cufile_bind_locked()
{
    if (g_cf.tried)
        return;
    g_cf.tried = true;
    /* libcufile is entered only where the host asks for it: on hosts without
     * the nvidia-fs driver a cuFile read was seen not to return at all */
    const char *on = getenv("XPU_B200_CUFILE");
    if (!on || strcmp(on, "1") != 0) {
        g_cf.why = "cuFile is not enabled (XPU_B200_CUFILE=1)";
        return;
    }
    void *h = nullptr;
    for (const char *l : {"libcufile.so.0", "libcufile.so", "/usr/local/cuda/lib64/libcufile.so.0"})
        if ((h = dlopen(l, RTLD_NOW | RTLD_LOCAL)) != nullptr)
            break;
    if (!h) {
        g_cf.why = "libcufile is not available";
        return;
    }
    g_cf.driver_open = (xb_cufile_error (*)(void))dlsym(h, "cuFileDriverOpen");
    g_cf.handle_register = (xb_cufile_error (*)(void **, xb_cufile_descr *))dlsym(h, "cuFileHandleRegister");
    g_cf.handle_deregister = (void (*)(void *))dlsym(h, "cuFileHandleDeregister");
    g_cf.read = (ssize_t (*)(void *, void *, size_t, off_t, off_t))dlsym(h, "cuFileRead");
    if (!g_cf.driver_open || !g_cf.handle_register || !g_cf.handle_deregister || !g_cf.read) {
        g_cf.why = "libcufile lacks an expected symbol";
        return;
    }
    const xb_cufile_error e = g_cf.driver_open();
    if (e.err != 0) {
        g_cf.why = "cuFileDriverOpen failed (error " + std::to_string(e.err) + ")";
        return;
    }
    g_cf.ok = true;
}

}   /* namespace */

/* the device's index, for the calls below (xb_exec.cu) */
extern "C" int xb_device_index(const xpuB200Device *dev);

extern "C" int
xpuB200ChunkReadDirect(xpuB200Device *dev, const char *pathname,
                       const kern_data_store *kds_head, uint64_t base_offset,
                       const xpuB200IoChunk *ioc, uint32_t nr_chunks,
                       void *kds_dev, uint64_t kds_dev_sz, int try_direct,
                       uint32_t *p_npages_direct, uint32_t *p_npages_vfs, kern_errorbuf *err)
{
    auto fail = [&](uint32_t code, const std::string &m) {
        if (err) {
            memset(err, 0, sizeof(*err));
            err->errcode = code;
            snprintf(err->funcname, sizeof(err->funcname), "%s", "xpuB200ChunkReadDirect");
            snprintf(err->message, sizeof(err->message), "%s", m.c_str());
        }
        return (int)code;
    };
    if (err)
        memset(err, 0, sizeof(*err));
    if (!dev || !pathname || !kds_dev || (!ioc && nr_chunks) || (!kds_head && base_offset))
        return fail(ERRCODE_DEVICE_ERROR, "invalid ChunkReadDirect arguments");
    if (base_offset > kds_dev_sz)
        return fail(ERRCODE_DEVICE_ERROR, "the chunk header does not fit the device buffer");
    for (uint32_t i = 0; i < nr_chunks; i++)
        if (base_offset + ioc[i].m_offset + (uint64_t)ioc[i].nr_pages * XPU_B200_IO_PAGE > kds_dev_sz)
            return fail(ERRCODE_DEVICE_ERROR, "an I/O chunk reaches past the device buffer");
    if (cudaSetDevice(xb_device_index(dev)) != cudaSuccess)
        return fail(ERRCODE_DEVICE_FATAL, "cudaSetDevice failed");
    /* the header and block numbers from host memory */
    if (base_offset && cudaMemcpy(kds_dev, kds_head, base_offset, cudaMemcpyHostToDevice) != cudaSuccess)
        return fail(ERRCODE_DEVICE_FATAL, "header copy failed");
    const int fd = open(pathname, O_RDONLY);
    if (fd < 0)
        return fail(ERRCODE_DEVICE_ERROR, std::string("cannot open ") + pathname);
    uint32_t npages_direct = 0, npages_vfs = 0;
    void *fh = nullptr;
    if (try_direct) {
        std::lock_guard<std::mutex> g(g_cf_lock);
        cufile_bind_locked();
        if (g_cf.ok) {
            xb_cufile_descr d;
            memset(&d, 0, sizeof(d));
            d.type = 1;
            d.handle.fd = fd;
            if (g_cf.handle_register(&fh, &d).err != 0)
                fh = nullptr;
        }
    }
    char *bounce = nullptr;
    const size_t bounce_sz = 8ULL << 20;
    int rc = 0;
    for (uint32_t i = 0; i < nr_chunks && rc == 0; i++) {
        const uint64_t nbytes = (uint64_t)ioc[i].nr_pages * XPU_B200_IO_PAGE;
        const off_t fpos = (off_t)ioc[i].fchunk_id * XPU_B200_IO_PAGE;
        char *dst = (char *)kds_dev + base_offset + ioc[i].m_offset;
        if (fh) {
            const ssize_t got = g_cf.read(fh, dst, nbytes, fpos, 0);
            if (got == (ssize_t)nbytes) {
                npages_direct += ioc[i].nr_pages;
                continue;
            }
        }
        /* through a pinned bounce buffer */
        if (!bounce && cudaMallocHost((void **)&bounce, bounce_sz) != cudaSuccess) {
            rc = fail(ERRCODE_DEVICE_FATAL, "cannot pin a bounce buffer");
            break;
        }
        for (uint64_t done = 0; done < nbytes && rc == 0;) {
            const size_t n = nbytes - done < bounce_sz ? (size_t)(nbytes - done) : bounce_sz;
            const ssize_t got = pread(fd, bounce, n, fpos + (off_t)done);
            if (got != (ssize_t)n) {
                rc = fail(ERRCODE_DEVICE_ERROR, std::string("short read from ") + pathname);
                break;
            }
            if (cudaMemcpy(dst + done, bounce, n, cudaMemcpyHostToDevice) != cudaSuccess)
                rc = fail(ERRCODE_DEVICE_FATAL, "bounce copy failed");
            done += n;
        }
        if (rc == 0)
            npages_vfs += ioc[i].nr_pages;
    }
    if (fh)
        g_cf.handle_deregister(fh);
    if (bounce)
        cudaFreeHost(bounce);
    close(fd);
    if (p_npages_direct) *p_npages_direct = npages_direct;
    if (p_npages_vfs) *p_npages_vfs = npages_vfs;
    return rc;
}
