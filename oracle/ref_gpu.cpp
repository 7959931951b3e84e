/*
 * ref_gpu.cpp -- TEST INFRASTRUCTURE ONLY.
 *
 * Runs PG-Strom's own device executor, kern_gpujoin_main
 * (src/cuda_gpujoin.cu:1050-1279), built for sm_100a from the reference
 * sources by oracle/Makefile "ref_gpu" (_ref/pgstrom_sm100a.fatbin), over
 * the same sessions, inner relations and chunks the CUDA path of this
 * repository consumes.  Around the kernel it does what PG-Strom's GPU
 * service does for one client on one GPU:
 *
 *   gpuservSetupGpuModule (gpu_service.c:6231-6319): load the module, read
 *     the type / function / encoding catalogs (:6111-6225), set the kernel's
 *     dynamic shared-memory limit (opt-in maximum - static - 8 KB);
 *   __resolveDevicePointers (:3156-3317): patch fn_dptr / expr_ops of every
 *     kern_expression and vs_ops of every kvars slot of a session copy;
 *   expandCudaStackLimit (:3066-3108): the context's stack size;
 *   __setupGpuQueryJoinInnerBuffer (:2198-2354): kern_multirels in device
 *     memory with kds_in of each depth pointing into it;
 *   __setupGpuQueryFinalResultsBuffer (:2357-2412): kds_final, of the length
 *     and hash slots pgstromBuildSessionInfo gives a GROUP BY (executor.c:
 *     660-700), its head copied from the session;
 *   __gpuservLaunchGpuTaskExecKernel (:3760-4003): block size from the
 *     occupancy API capped at 512 (gpuOptimalBlockSize, gpu_device.c:
 *     1121-1140), the prep-function buffer (:3673-3716), kern_gputask, one
 *     launch and one stream synchronisation per chunk, and on
 *     SUSPEND_NO_SPACE the expansion of kds_final (:2418-2495) and a resume
 *     launch.
 *
 * The session's groupby_prepfn_bufsz is set as the reference planner sets
 * it: the sum of the partial-state sizes of its aggregate actions
 * (gpu_preagg.c:1190-1260, :1687).  The driver API is bound at run time
 * (libcuda.so.1).  Compiled against the reference headers; never part of
 * the product, and nothing of the product calls it.
 */
#include <dlfcn.h>
#include <cstdio>
#include <cstring>
#include <string>
#include <vector>
#include <map>
#include "xpu_common.h"
#include "cuda_common.h"

namespace {

typedef int CUresult;
typedef int CUdevice;
typedef unsigned long long CUdeviceptr;
typedef struct CUctx_st *CUcontext;
typedef struct CUmod_st *CUmodule;
typedef struct CUfunc_st *CUfunction;
typedef struct CUstream_st *CUstream;
typedef struct CUevent_st *CUevent;

enum {
    XCU_FUNC_ATTRIBUTE_SHARED_SIZE_BYTES = 1,
    XCU_FUNC_ATTRIBUTE_LOCAL_SIZE_BYTES = 3,
    XCU_FUNC_ATTRIBUTE_NUM_REGS = 4,
    XCU_FUNC_ATTRIBUTE_MAX_DYNAMIC_SHARED_SIZE_BYTES = 8,
    XCU_DEVICE_ATTRIBUTE_MULTIPROCESSOR_COUNT = 16,
    XCU_DEVICE_ATTRIBUTE_MAX_SHARED_MEMORY_PER_BLOCK_OPTIN = 97,
    XCU_LIMIT_STACK_SIZE = 0,
    XCU_STREAM_NON_BLOCKING = 1,
};

struct Drv {
    bool ok = false;
    std::string why;
    CUresult (*init)(unsigned);
    CUresult (*device_get)(CUdevice *, int);
    CUresult (*primary_retain)(CUcontext *, CUdevice);
    CUresult (*ctx_set_current)(CUcontext);
    CUresult (*ctx_set_limit)(int, size_t);
    CUresult (*ctx_get_limit)(size_t *, int);
    CUresult (*dev_attr)(int *, int, CUdevice);
    CUresult (*module_load)(CUmodule *, const char *);
    CUresult (*module_unload)(CUmodule);
    CUresult (*module_global)(CUdeviceptr *, size_t *, CUmodule, const char *);
    CUresult (*module_function)(CUfunction *, CUmodule, const char *);
    CUresult (*func_get_attr)(int *, int, CUfunction);
    CUresult (*func_set_attr)(CUfunction, int, int);
    CUresult (*occupancy)(int *, int *, CUfunction, void *, size_t, int);
    CUresult (*mem_alloc)(CUdeviceptr *, size_t);
    CUresult (*mem_free)(CUdeviceptr);
    CUresult (*memset8)(CUdeviceptr, unsigned char, size_t);
    CUresult (*htod)(CUdeviceptr, const void *, size_t);
    CUresult (*dtoh)(void *, CUdeviceptr, size_t);
    CUresult (*dtod)(CUdeviceptr, CUdeviceptr, size_t);
    CUresult (*launch)(CUfunction, unsigned, unsigned, unsigned, unsigned, unsigned, unsigned, unsigned,
                       CUstream, void **, void **);
    CUresult (*stream_create)(CUstream *, unsigned);
    CUresult (*stream_destroy)(CUstream);
    CUresult (*stream_sync)(CUstream);
    CUresult (*event_create)(CUevent *, unsigned);
    CUresult (*event_destroy)(CUevent);
    CUresult (*event_record)(CUevent, CUstream);
    CUresult (*event_sync)(CUevent);
    CUresult (*event_elapsed)(float *, CUevent, CUevent);
    CUresult (*error_string)(CUresult, const char **);
};
Drv g;

template <typename F>
bool bind(void *h, F &f, const char *name)
{
    f = (F)dlsym(h, name);
    return f != nullptr;
}

bool drv_bind(std::string &err)
{
    if (g.ok)
        return true;
    void *h = dlopen("libcuda.so.1", RTLD_NOW | RTLD_GLOBAL);
    if (!h) {
        err = "libcuda.so.1 is not available";
        return false;
    }
    bool ok = bind(h, g.init, "cuInit") && bind(h, g.device_get, "cuDeviceGet") &&
              bind(h, g.primary_retain, "cuDevicePrimaryCtxRetain") &&
              bind(h, g.ctx_set_current, "cuCtxSetCurrent") && bind(h, g.ctx_set_limit, "cuCtxSetLimit") &&
              bind(h, g.ctx_get_limit, "cuCtxGetLimit") && bind(h, g.dev_attr, "cuDeviceGetAttribute") &&
              bind(h, g.module_load, "cuModuleLoad") && bind(h, g.module_unload, "cuModuleUnload") &&
              bind(h, g.module_global, "cuModuleGetGlobal_v2") &&
              bind(h, g.module_function, "cuModuleGetFunction") &&
              bind(h, g.func_get_attr, "cuFuncGetAttribute") && bind(h, g.func_set_attr, "cuFuncSetAttribute") &&
              bind(h, g.occupancy, "cuOccupancyMaxPotentialBlockSize") &&
              bind(h, g.mem_alloc, "cuMemAlloc_v2") && bind(h, g.mem_free, "cuMemFree_v2") &&
              bind(h, g.memset8, "cuMemsetD8_v2") && bind(h, g.htod, "cuMemcpyHtoD_v2") &&
              bind(h, g.dtoh, "cuMemcpyDtoH_v2") && bind(h, g.dtod, "cuMemcpyDtoD_v2") &&
              bind(h, g.launch, "cuLaunchKernel") && bind(h, g.stream_create, "cuStreamCreate") &&
              bind(h, g.stream_destroy, "cuStreamDestroy_v2") && bind(h, g.stream_sync, "cuStreamSynchronize") &&
              bind(h, g.event_create, "cuEventCreate") && bind(h, g.event_destroy, "cuEventDestroy_v2") &&
              bind(h, g.event_record, "cuEventRecord") && bind(h, g.event_sync, "cuEventSynchronize") &&
              bind(h, g.event_elapsed, "cuEventElapsedTime") && bind(h, g.error_string, "cuGetErrorString");
    if (!ok) {
        err = "libcuda.so.1 lacks an expected symbol";
        return false;
    }
    g.ok = true;
    return true;
}

std::string cuerr(const char *what, CUresult rc)
{
    const char *s = nullptr;
    if (g.error_string)
        g.error_string(rc, &s);
    return std::string(what) + ": " + (s ? s : "error " + std::to_string(rc));
}

/* the reference module on one device */
struct Module {
    int dindex = -1;
    CUcontext ctx = nullptr;
    CUmodule mod = nullptr;
    CUfunction fn_main = nullptr;
    std::map<int, CUdeviceptr> types;       /* TypeOpCode -> xpu_datum_operators (device) */
    std::map<int, CUdeviceptr> funcs;       /* FuncOpCode -> device function */
    std::vector<xpu_encode_info> encodes;
    int shmem_limit = 0;
    int nsm = 0;
    size_t stack_limit = 0;
    int nregs = 0;
    int local_bytes = 0;
};
Module *g_mod = nullptr;

/* the lengths of cuda_common.h:116-177 for run-time depths (the macros use
 * offsetof with a variable index, which C accepts and C++ does not) */
size_t warp_basesz(uint32_t nd)
{
    return TYPEALIGN(CUDA_L1_CACHELINE_SZ,
                     offsetof(kern_warp_context, pos) + nd * sizeof(((kern_warp_context *)0)->pos[0]));
}

size_t gputask_head(uint32_t n)
{
    return offsetof(kern_gputask, stats) + n * sizeof(((kern_gputask *)0)->stats[0]);
}

size_t gputask_length(uint32_t nd, uint32_t bufsz, uint64_t grid, uint64_t block)
{
    const size_t warp_len = warp_basesz(nd) + nd * TYPEALIGN(CUDA_L1_CACHELINE_SZ, bufsz);
    return TYPEALIGN(CUDA_L1_CACHELINE_SZ, gputask_head(nd)) + warp_len * grid +
           MAXALIGN(sizeof(uint64_t) * grid * block * nd) + MAXALIGN(sizeof(bool) * grid * block * nd);
}

struct Sess {
    std::vector<char> h_sess;               /* the session with device pointers resolved */
    kern_session_info *session = nullptr;
    CUdeviceptr d_sess = 0;
    CUdeviceptr d_kmrels = 0;
    uint32_t n_rels = 0;
    CUdeviceptr d_final = 0;
    size_t final_len = 0;
    CUdeviceptr d_task = 0;
    size_t task_len = 0;
    int grid = 0, block = 0;
    unsigned shmem = 0;
    unsigned prepfn_nbufs = 0;
    CUstream st = nullptr;
    CUevent ev0 = nullptr, ev1 = nullptr;
    CUevent evk0 = nullptr, evk1 = nullptr;     /* around each launch */
    double kernel_ms = 0.0;                     /* launches' device time, summed */
    uint64_t nitems_raw = 0, nitems_in = 0, nitems_out = 0;
    uint32_t suspends = 0, expands = 0;
};

bool resolve_type(Sess *s, const xpu_datum_operators **p_ops, int code, std::string &err)
{
    (void)s;
    auto it = g_mod->types.find(code);
    if (it == g_mod->types.end()) {
        err = "type opcode " + std::to_string(code) + " is not in the device catalog";
        return false;
    }
    *p_ops = (const xpu_datum_operators *)it->second;
    return true;
}

/* __resolveDevicePointersWalker, gpu_service.c:3156-3250 */
bool resolve_walk(Sess *s, kern_expression *kexp, std::string &err)
{
    auto f = g_mod->funcs.find(kexp->opcode);
    if (f == g_mod->funcs.end()) {
        err = "function opcode " + std::to_string(kexp->opcode) + " is not in the device catalog";
        return false;
    }
    kexp->fn_dptr = (xpu_function_t)f->second;
    if (!resolve_type(s, &kexp->expr_ops, kexp->exptype, err))
        return false;
    kern_expression *karg;
    switch (kexp->opcode) {
    case FuncOpCode__CaseWhenExpr:
        if (kexp->u.casewhen.case_comp) {
            karg = (kern_expression *)((char *)kexp + kexp->u.casewhen.case_comp);
            if (!__KEXP_IS_VALID(kexp, karg) || !resolve_walk(s, karg, err))
                goto corrupt;
        }
        if (kexp->u.casewhen.case_else) {
            karg = (kern_expression *)((char *)kexp + kexp->u.casewhen.case_else);
            if (!__KEXP_IS_VALID(kexp, karg) || !resolve_walk(s, karg, err))
                goto corrupt;
        }
        break;
    case FuncOpCode__Projection:
        if (kexp->u.proj.hash) {
            karg = (kern_expression *)((char *)kexp + kexp->u.proj.hash);
            if (!__KEXP_IS_VALID(kexp, karg) || !resolve_walk(s, karg, err))
                goto corrupt;
        }
        break;
    case FuncOpCode__SortKeys:
        for (int i = 0; i < kexp->u.sort.nkeys; i++) {
            kern_sortkey_desc *sd = &kexp->u.sort.desc[i];
            if (!resolve_type(s, &sd->key_ops, sd->key_type_code, err))
                return false;
        }
        break;
    case FuncOpCode__HashedArrayOp:
        if (!resolve_type(s, &kexp->u.haop.elem_ops, kexp->u.haop.elem_type, err))
            return false;
        break;
    default:
        break;
    }
    karg = KEXP_FIRST_ARG(kexp);
    for (int i = 0; i < kexp->nr_args; i++, karg = KEXP_NEXT_ARG(karg)) {
        if (!__KEXP_IS_VALID(kexp, karg))
            goto corrupt;
        if (!resolve_walk(s, karg, err))
            return false;
    }
    return true;
corrupt:
    if (err.empty())
        err = "XPU code corruption at kexp (" + std::to_string(kexp->opcode) + ")";
    return false;
}

/* __resolveDevicePointers, gpu_service.c:3252-3317 */
bool resolve_session(Sess *s, std::string &err)
{
    kern_session_info *session = s->session;
    kern_expression *kx[12] = {
        SESSION_KEXP_LOAD_VARS(session, -1), SESSION_KEXP_MOVE_VARS(session, -1),
        SESSION_KEXP_SCAN_QUALS(session), SESSION_KEXP_JOIN_QUALS(session, -1),
        SESSION_KEXP_HASH_VALUE(session, -1), SESSION_KEXP_GIST_EVALS(session, -1),
        SESSION_KEXP_PROJECTION(session), SESSION_KEXP_GROUPBY_KEYHASH(session),
        SESSION_KEXP_GROUPBY_KEYLOAD(session), SESSION_KEXP_GROUPBY_KEYCOMP(session),
        SESSION_KEXP_GROUPBY_ACTIONS(session), SESSION_KEXP_GPUSORT_KEYDESC(session)};
    for (kern_expression *k : kx)
        if (k && !resolve_walk(s, k, err))
            return false;
    kern_varslot_desc *vs = SESSION_KVARS_SLOT_DESC(session);
    for (uint32_t i = 0; i < session->kcxt_kvars_nslots; i++)
        if (!resolve_type(s, &vs[i].vs_ops, vs[i].vs_type_code, err))
            return false;
    xpu_encode_info *enc = SESSION_ENCODE(session);
    if (enc) {
        for (size_t i = 0;; i++) {
            if (i >= g_mod->encodes.size() || !g_mod->encodes[i].enc_mblen || g_mod->encodes[i].enc_maxlen < 1) {
                err = std::string("encode [") + enc->encname + "] was not found";
                return false;
            }
            if (strcmp(enc->encname, g_mod->encodes[i].encname) == 0) {
                enc->enc_maxlen = g_mod->encodes[i].enc_maxlen;
                enc->enc_mblen = g_mod->encodes[i].enc_mblen;
                break;
            }
        }
    }
    return true;
}

/* the partial-state bytes of an action (gpu_preagg.c:1190-1260) */
size_t partfn_bufsz(int action)
{
    switch (action & ~__KAGG_ACTION__USE_FILTER) {
    case KAGG_ACTION__NROWS_ANY: case KAGG_ACTION__NROWS_COND:
        return sizeof(int64_t);
    case KAGG_ACTION__PMIN_INT32: case KAGG_ACTION__PMIN_INT64:
    case KAGG_ACTION__PMAX_INT32: case KAGG_ACTION__PMAX_INT64:
        return sizeof(kagg_state__pminmax_int64_packed);
    case KAGG_ACTION__PMIN_FP64: case KAGG_ACTION__PMAX_FP64:
        return sizeof(kagg_state__pminmax_fp64_packed);
    case KAGG_ACTION__PAVG_INT: case KAGG_ACTION__PSUM_INT:
        return sizeof(kagg_state__psum_int_packed);
    case KAGG_ACTION__PAVG_FP: case KAGG_ACTION__PSUM_FP:
        return sizeof(kagg_state__psum_fp_packed);
    case KAGG_ACTION__PAVG_INT64: case KAGG_ACTION__PSUM_INT64:
    case KAGG_ACTION__PAVG_NUMERIC: case KAGG_ACTION__PSUM_NUMERIC:
        return sizeof(kagg_state__psum_numeric_packed);
    case KAGG_ACTION__STDDEV:
        return sizeof(kagg_state__stddev_packed);
    case KAGG_ACTION__COVAR:
        return sizeof(kagg_state__covar_packed);
    default:
        return 0;
    }
}

void set_err(char *buf, size_t len, const std::string &m)
{
    if (buf && len)
        snprintf(buf, len, "%s", m.c_str());
}

void sess_free(Sess *s)
{
    if (!s)
        return;
    if (s->d_sess) g.mem_free(s->d_sess);
    if (s->d_kmrels) g.mem_free(s->d_kmrels);
    if (s->d_final) g.mem_free(s->d_final);
    if (s->d_task) g.mem_free(s->d_task);
    if (s->ev0) g.event_destroy(s->ev0);
    if (s->ev1) g.event_destroy(s->ev1);
    if (s->evk0) g.event_destroy(s->evk0);
    if (s->evk1) g.event_destroy(s->evk1);
    if (s->st) g.stream_destroy(s->st);
    delete s;
}

/* kds_final expanded as __expandGpuQueryGroupByBuffer does (gpu_service.c:
 * 2418-2495): at least 1 GB more, head / slots / row index and the tail
 * ('usage' bytes) copied into the new buffer */
bool expand_final(Sess *s, std::string &err)
{
    kern_data_store head;
    CUresult rc = g.dtoh(&head, s->d_final, sizeof(head));
    if (rc) { err = cuerr("cuMemcpyDtoH", rc); return false; }
    const size_t length = head.length + (head.length > (1UL << 30) ? head.length : (1UL << 30));
    CUdeviceptr d_new = 0;
    if ((rc = g.mem_alloc(&d_new, length))) { err = cuerr("cuMemAlloc", rc); return false; }
    const size_t head_len = KDS_HEAD_LENGTH(&head);
    size_t sz = head_len + sizeof(uint64_t) * ((size_t)head.nitems + head.hash_nslots);
    rc = g.dtod(d_new, s->d_final, sz);
    if (!rc) rc = g.htod(d_new + offsetof(kern_data_store, length), &length, sizeof(size_t));
    if (!rc) rc = g.dtod(d_new + length - head.usage, s->d_final + head.length - head.usage, head.usage);
    if (rc) { g.mem_free(d_new); err = cuerr("cuMemcpyDtoD", rc); return false; }
    g.mem_free(s->d_final);
    s->d_final = d_new;
    s->final_len = length;
    s->expands++;
    return true;
}

/* one chunk: launch, synchronise, resume on SUSPEND_NO_SPACE */
int exec_chunk(Sess *s, CUdeviceptr d_kds, std::string &err)
{
    const kern_session_info *session = s->session;
    const size_t hsz = gputask_head(s->n_rels > 0 ? s->n_rels : 1);
    std::vector<char> hbuf(hsz);
    kern_gputask *kt = (kern_gputask *)hbuf.data();
    memset(kt, 0, hsz);
    kt->grid_sz = s->grid;
    kt->block_sz = s->block;
    kt->kvars_nslots = session->kcxt_kvars_nslots;
    kt->kvecs_bufsz = session->kcxt_kvecs_bufsz;
    kt->kvecs_ndims = session->kcxt_kvecs_ndims;
    kt->n_rels = s->n_rels;
    kt->groupby_prepfn_nbufs = s->prepfn_nbufs;
    kt->cuda_dindex = g_mod->dindex;
    kt->cuda_stack_limit = (uint32_t)g_mod->stack_limit;
    kt->partition_divisor = -1;
    kt->partition_reminder = -1;
    kt->right_outer_depth = 0;
    CUresult rc = g.htod(s->d_task, kt, hsz);
    if (rc) { err = cuerr("cuMemcpyHtoD", rc); return ERRCODE_DEVICE_FATAL; }
    for (int round = 0;; round++) {
        if (round > 64) { err = "kds_final kept running out of space"; return ERRCODE_DEVICE_ERROR; }
        CUdeviceptr kmrels = s->d_kmrels, extra = 0, fallback = 0, dst = s->d_final;
        void *args[7] = {&s->d_sess, &s->d_task, &kmrels, &d_kds, &extra, &dst, &fallback};
        g.event_record(s->evk0, s->st);
        rc = g.launch(g_mod->fn_main, s->grid, 1, 1, s->block, 1, 1, s->shmem, s->st, args, nullptr);
        if (rc) { err = cuerr("cuLaunchKernel", rc); return ERRCODE_DEVICE_FATAL; }
        g.event_record(s->evk1, s->st);
        if ((rc = g.stream_sync(s->st))) { err = cuerr("cuStreamSynchronize", rc); return ERRCODE_DEVICE_FATAL; }
        {
            float kms = 0.0f;
            if (g.event_elapsed(&kms, s->evk0, s->evk1) == 0)
                s->kernel_ms += kms;
        }
        if ((rc = g.dtoh(kt, s->d_task, hsz))) { err = cuerr("cuMemcpyDtoH", rc); return ERRCODE_DEVICE_FATAL; }
        if (kt->kerror.errcode == ERRCODE_STROM_SUCCESS) {
            s->nitems_raw += kt->nitems_raw;
            s->nitems_in += kt->nitems_in;
            s->nitems_out += kt->nitems_out;
            return 0;
        }
        if (kt->kerror.errcode == ERRCODE_SUSPEND_NO_SPACE) {
            s->suspends++;
            if (!expand_final(s, err))
                return ERRCODE_DEVICE_FATAL;
            kt->kerror.errcode = 0;
            kt->resume_context = true;
            if ((rc = g.htod(s->d_task, kt, hsz))) { err = cuerr("cuMemcpyHtoD", rc); return ERRCODE_DEVICE_FATAL; }
            continue;
        }
        char msg[512];
        snprintf(msg, sizeof(msg), "kernel error %u at %s:%d (%s): %s", kt->kerror.errcode, kt->kerror.filename,
                 kt->kerror.lineno, kt->kerror.funcname, kt->kerror.message);
        err = msg;
        return (int)kt->kerror.errcode;
    }
}

}   /* namespace */

extern "C" {

/* load the reference module on device dindex (once per process) */
int rg_open(const char *fatbin, int dindex, char *errbuf, size_t errlen)
{
    std::string err;
    if (g_mod) {
        if (g_mod->dindex == dindex)
            return 0;
        set_err(errbuf, errlen, "the reference module is loaded on another device");
        return -1;
    }
    if (!drv_bind(err)) { set_err(errbuf, errlen, err); return -1; }
    CUresult rc;
    Module *m = new Module();
    m->dindex = dindex;
    CUdevice dev;
    if ((rc = g.init(0)) || (rc = g.device_get(&dev, dindex)) || (rc = g.primary_retain(&m->ctx, dev)) ||
        (rc = g.ctx_set_current(m->ctx))) {
        set_err(errbuf, errlen, cuerr("context", rc));
        delete m;
        return -1;
    }
    if ((rc = g.module_load(&m->mod, fatbin))) {
        set_err(errbuf, errlen, cuerr("cuModuleLoad", rc));
        delete m;
        return -1;
    }
    /* catalogs (gpu_service.c:6111-6225) */
    CUdeviceptr dp;
    size_t nb;
    if ((rc = g.module_global(&dp, &nb, m->mod, "builtin_xpu_types_catalog"))) {
        set_err(errbuf, errlen, cuerr("types catalog", rc));
        return -1;
    }
    std::vector<xpu_type_catalog_entry> tc(nb / sizeof(xpu_type_catalog_entry));
    g.dtoh(tc.data(), dp, tc.size() * sizeof(xpu_type_catalog_entry));
    for (auto &e : tc) {
        if (e.type_opcode == TypeOpCode__Invalid) break;
        m->types[e.type_opcode] = (CUdeviceptr)e.type_ops;
    }
    if ((rc = g.module_global(&dp, &nb, m->mod, "builtin_xpu_functions_catalog"))) {
        set_err(errbuf, errlen, cuerr("functions catalog", rc));
        return -1;
    }
    std::vector<xpu_function_catalog_entry> fc(nb / sizeof(xpu_function_catalog_entry));
    g.dtoh(fc.data(), dp, fc.size() * sizeof(xpu_function_catalog_entry));
    for (auto &e : fc) {
        if (e.func_opcode == FuncOpCode__Invalid) break;
        m->funcs[e.func_opcode] = (CUdeviceptr)e.func_dptr;
    }
    if ((rc = g.module_global(&dp, &nb, m->mod, "xpu_encode_catalog")) == 0) {
        m->encodes.resize(nb / sizeof(xpu_encode_info));
        g.dtoh(m->encodes.data(), dp, m->encodes.size() * sizeof(xpu_encode_info));
    }
    if ((rc = g.module_function(&m->fn_main, m->mod, "kern_gpujoin_main"))) {
        set_err(errbuf, errlen, cuerr("kern_gpujoin_main", rc));
        return -1;
    }
    int st_sz = 0, optin = 0;
    g.func_get_attr(&st_sz, XCU_FUNC_ATTRIBUTE_SHARED_SIZE_BYTES, m->fn_main);
    g.func_get_attr(&m->nregs, XCU_FUNC_ATTRIBUTE_NUM_REGS, m->fn_main);
    g.func_get_attr(&m->local_bytes, XCU_FUNC_ATTRIBUTE_LOCAL_SIZE_BYTES, m->fn_main);
    g.dev_attr(&optin, XCU_DEVICE_ATTRIBUTE_MAX_SHARED_MEMORY_PER_BLOCK_OPTIN, dev);
    g.dev_attr(&m->nsm, XCU_DEVICE_ATTRIBUTE_MULTIPROCESSOR_COUNT, dev);
    m->shmem_limit = optin - (int)TYPEALIGN(1024, st_sz) - 8192;
    if ((rc = g.func_set_attr(m->fn_main, XCU_FUNC_ATTRIBUTE_MAX_DYNAMIC_SHARED_SIZE_BYTES, m->shmem_limit))) {
        set_err(errbuf, errlen, cuerr("cuFuncSetAttribute", rc));
        return -1;
    }
    g.ctx_get_limit(&m->stack_limit, XCU_LIMIT_STACK_SIZE);
    g_mod = m;
    return 0;
}

/*
 * Open a session: the session blob and kern_multirels (or NULL) as the CUDA
 * path receives them.  kds_final is given at least final_min bytes (the
 * reference's planner asks for 1 GB or more for a GROUP BY).
 */
void *rg_session(const void *session_blob, size_t session_sz, const void *kmrels, size_t kmrels_sz,
                 size_t final_min, char *errbuf, size_t errlen)
{
    std::string err;
    if (!g_mod) { set_err(errbuf, errlen, "rg_open first"); return nullptr; }
    g.ctx_set_current(g_mod->ctx);
    Sess *s = new Sess();
    s->h_sess.assign((const char *)session_blob, (const char *)session_blob + session_sz);
    s->session = (kern_session_info *)s->h_sess.data();
    kern_session_info *session = s->session;
    CUresult rc;
    /* the prep-function buffer size the planner gives (gpu_preagg.c:1687) */
    kern_expression *acts = SESSION_KEXP_GROUPBY_ACTIONS(session);
    if (acts && acts->opcode == FuncOpCode__AggFuncs) {
        size_t bufsz = 0;
        for (int i = 0; i < acts->u.pagg.nattrs; i++)
            bufsz += partfn_bufsz(acts->u.pagg.desc[i].action);
        session->groupby_prepfn_bufsz = (uint32_t)bufsz;
    }
    /* kds_final as pgstromBuildSessionInfo sizes it for a GROUP BY */
    if (session->groupby_kds_final) {
        kern_data_store *kf = (kern_data_store *)((char *)session + session->groupby_kds_final);
        if (session->xpucode_groupby_keyhash) {
            const uint64_t nrows = (uint64_t)(session->groupby_ngroups_estimation > 1.0
                                              ? session->groupby_ngroups_estimation : 1.0);
            const uint64_t nslots = KDS_GET_HASHSLOT_WIDTH(nrows);
            kf->format = KDS_FORMAT_HASH;
            kf->hash_nslots = (uint32_t)nslots;
            kf->length = final_min > (1UL << 30) ? final_min : (1UL << 30);
        } else {
            kf->format = KDS_FORMAT_ROW;
            kf->hash_nslots = 0;
            kf->length = 4UL << 20;
        }
        kf->nitems = 0;
        kf->usage = 0;
    }
    if (!resolve_session(s, err)) { set_err(errbuf, errlen, err); sess_free(s); return nullptr; }
    /* the stack the planner would ask for (estimate_cuda_stack_size,
     * codegen.c:4569-4600): a working area, the kern_context with its
     * variable-length buffer, the kvars slot pointers and each slot's
     * datum (sizes read from the device's type catalog), plus 8 KB for the
     * expressions' own frames, which the planner counts while it emits
     * them and this session does not carry */
    {
        size_t sz = 3200 + TYPEALIGN(16, offsetof(kern_context, vlbuf) +
                                           (session->kcxt_extra_bufsz > 512 ? session->kcxt_extra_bufsz : 512));
        sz += TYPEALIGN(16, sizeof(void *) * session->kcxt_kvars_nslots);
        const kern_varslot_desc *vs = SESSION_KVARS_SLOT_DESC(session);
        for (uint32_t i = 0; i < session->kcxt_kvars_nslots; i++) {
            xpu_datum_operators ops;
            if ((rc = g.dtoh(&ops, (CUdeviceptr)vs[i].vs_ops, sizeof(ops)))) {
                set_err(errbuf, errlen, cuerr("type catalog entry", rc));
                sess_free(s);
                return nullptr;
            }
            sz += TYPEALIGN(16, ops.xpu_type_sizeof);
        }
        sz += 8192;
        if (sz > session->cuda_stack_size)
            session->cuda_stack_size = (uint32_t)sz;
    }
    /* the stack the session asks for (expandCudaStackLimit) */
    if (session->cuda_stack_size > g_mod->stack_limit) {
        const size_t lim = TYPEALIGN(1024, session->cuda_stack_size);
        if ((rc = g.ctx_set_limit(XCU_LIMIT_STACK_SIZE, lim))) {
            set_err(errbuf, errlen, cuerr("cuCtxSetLimit", rc));
            sess_free(s);
            return nullptr;
        }
        g_mod->stack_limit = lim;
    }
    if ((rc = g.stream_create(&s->st, XCU_STREAM_NON_BLOCKING)) || (rc = g.event_create(&s->ev0, 0)) ||
        (rc = g.event_create(&s->ev1, 0)) || (rc = g.event_create(&s->evk0, 0)) ||
        (rc = g.event_create(&s->evk1, 0))) {
        set_err(errbuf, errlen, cuerr("stream", rc));
        sess_free(s);
        return nullptr;
    }
    if ((rc = g.mem_alloc(&s->d_sess, session_sz)) || (rc = g.htod(s->d_sess, s->h_sess.data(), session_sz))) {
        set_err(errbuf, errlen, cuerr("session", rc));
        sess_free(s);
        return nullptr;
    }
    if (kmrels && kmrels_sz) {
        std::vector<char> km((const char *)kmrels, (const char *)kmrels + kmrels_sz);
        kern_multirels *h = (kern_multirels *)km.data();
        if ((rc = g.mem_alloc(&s->d_kmrels, kmrels_sz))) {
            set_err(errbuf, errlen, cuerr("kmrels", rc));
            sess_free(s);
            return nullptr;
        }
        for (uint32_t d = 0; d < h->num_inner_rels; d++) {
            if (h->chunks[d].pinned_buffer || !h->chunks[d].kds_offset || h->chunks[d].kds_offset >= kmrels_sz) {
                set_err(errbuf, errlen, "inner relation without a KDS inside kern_multirels");
                sess_free(s);
                return nullptr;
            }
            h->chunks[d].kds_in = (kern_data_store *)(s->d_kmrels + h->chunks[d].kds_offset);
        }
        s->n_rels = h->num_inner_rels;
        if ((rc = g.htod(s->d_kmrels, km.data(), kmrels_sz))) {
            set_err(errbuf, errlen, cuerr("kmrels copy", rc));
            sess_free(s);
            return nullptr;
        }
    }
    if (session->groupby_kds_final) {
        const kern_data_store *kf = (const kern_data_store *)((char *)session + session->groupby_kds_final);
        s->final_len = kf->length;
        if ((rc = g.mem_alloc(&s->d_final, s->final_len)) || (rc = g.memset8(s->d_final, 0, s->final_len)) ||
            (rc = g.htod(s->d_final, kf, KDS_HEAD_LENGTH(kf)))) {
            set_err(errbuf, errlen, cuerr("kds_final", rc));
            sess_free(s);
            return nullptr;
        }
    }
    /* launch shape (__gpuservLaunchGpuTaskExecKernel) */
    unsigned shmem = (unsigned)warp_basesz(session->kcxt_kvecs_ndims);
    if ((rc = g.occupancy(&s->grid, &s->block, g_mod->fn_main, nullptr, shmem, 0))) {
        set_err(errbuf, errlen, cuerr("cuOccupancyMaxPotentialBlockSize", rc));
        sess_free(s);
        return nullptr;
    }
    if (s->block > CUDA_MAXTHREADS_PER_BLOCK)
        s->block = CUDA_MAXTHREADS_PER_BLOCK;
    {
        /* __expand_gpupreagg_prepfunc_buffer (gpu_service.c:3673-3716) */
        size_t sz = TYPEALIGN(1024, shmem);
        const size_t limit = (size_t)g_mod->shmem_limit;
        s->prepfn_nbufs = 0;
        if (session->groupby_prepfn_bufsz && sz < limit) {
            if (session->xpucode_groupby_keyhash && session->xpucode_groupby_keyload &&
                session->xpucode_groupby_keycomp) {
                size_t nbufs = 2 * (size_t)session->groupby_ngroups_estimation + 100;
                if (sz + (size_t)session->groupby_prepfn_bufsz * nbufs > limit)
                    nbufs = (limit - sz) / session->groupby_prepfn_bufsz;
                s->prepfn_nbufs = (unsigned)nbufs;
                shmem = (unsigned)(sz + session->groupby_prepfn_bufsz * nbufs);
            } else if (session->xpucode_groupby_actions && sz + session->groupby_prepfn_bufsz <= limit) {
                s->prepfn_nbufs = 1;
                shmem = (unsigned)(sz + session->groupby_prepfn_bufsz);
            }
        }
    }
    s->shmem = shmem;
    s->task_len = gputask_length(session->kcxt_kvecs_ndims, session->kcxt_kvecs_bufsz, s->grid, s->block);
    if ((rc = g.mem_alloc(&s->d_task, s->task_len))) {
        set_err(errbuf, errlen, cuerr("kern_gputask", rc));
        sess_free(s);
        return nullptr;
    }
    return s;
}

/* the chunks (device addresses) one after the other, as the GPU service
 * runs one task per chunk; with p_ms: device milliseconds of the launches
 * (from the first launch to the end of the last, host synchronisations
 * between them included, as the service has them) */
int rg_exec(void *h, const uint64_t *kds_dev, uint32_t nchunks, double *p_ms, char *errbuf, size_t errlen)
{
    Sess *s = (Sess *)h;
    std::string err;
    g.ctx_set_current(g_mod->ctx);
    if (p_ms) g.event_record(s->ev0, s->st);
    for (uint32_t i = 0; i < nchunks; i++) {
        const int rc = exec_chunk(s, (CUdeviceptr)kds_dev[i], err);
        if (rc) { set_err(errbuf, errlen, err); return rc; }
    }
    if (p_ms) {
        g.event_record(s->ev1, s->st);
        g.event_sync(s->ev1);
        float ms = 0.0f;
        g.event_elapsed(&ms, s->ev0, s->ev1);
        *p_ms = ms;
    }
    return 0;
}

/* kds_final copied out compacted (head, hash slots and row index, then the
 * tuples; item offsets count from the end, so they stay valid).  Returns the
 * bytes it takes; copies only when out_sz is large enough. */
int64_t rg_final(void *h, void *out, size_t out_sz, char *errbuf, size_t errlen)
{
    Sess *s = (Sess *)h;
    g.ctx_set_current(g_mod->ctx);
    if (!s->d_final) return 0;
    kern_data_store head;
    CUresult rc = g.dtoh(&head, s->d_final, sizeof(head));
    if (rc) { set_err(errbuf, errlen, cuerr("cuMemcpyDtoH", rc)); return -1; }
    const size_t head_len = KDS_HEAD_LENGTH(&head);
    const size_t front = head_len + sizeof(uint64_t) * ((size_t)head.hash_nslots + head.nitems);
    const size_t need = front + head.usage;
    if (!out || out_sz < need)
        return (int64_t)need;
    char *o = (char *)out;
    if ((rc = g.dtoh(o, s->d_final, front)) ||
        (head.usage && (rc = g.dtoh(o + front, s->d_final + head.length - head.usage, head.usage)))) {
        set_err(errbuf, errlen, cuerr("cuMemcpyDtoH", rc));
        return -1;
    }
    ((kern_data_store *)o)->length = need;
    return (int64_t)need;
}

/* launch shape and counters, as text */
int rg_info(void *h, char *buf, size_t len)
{
    Sess *s = (Sess *)h;
    snprintf(buf, len,
             "{\"grid\": %d, \"block\": %d, \"shmem\": %u, \"prepfn_nbufs\": %u, \"prepfn_bufsz\": %u, "
             "\"registers\": %d, \"local_bytes\": %d, \"stack_limit\": %zu, \"nitems_raw\": %llu, "
             "\"nitems_in\": %llu, \"nitems_out\": %llu, \"suspends\": %u, \"final_expands\": %u, "
             "\"kds_final_length\": %zu, \"kernel_ms\": %.4f}",
             s->grid, s->block, s->shmem, s->prepfn_nbufs, s->session->groupby_prepfn_bufsz, g_mod->nregs,
             g_mod->local_bytes, g_mod->stack_limit, (unsigned long long)s->nitems_raw,
             (unsigned long long)s->nitems_in, (unsigned long long)s->nitems_out, s->suspends, s->expands,
             s->final_len, s->kernel_ms);
    return 0;
}

void rg_close(void *h)
{
    if (!g_mod) return;
    g.ctx_set_current(g_mod->ctx);
    sess_free((Sess *)h);
}

/* device memory for the reference's own copies of the chunks */
uint64_t rg_upload(const void *src, size_t sz)
{
    if (!g_mod) return 0;
    g.ctx_set_current(g_mod->ctx);
    CUdeviceptr d = 0;
    if (g.mem_alloc(&d, sz) || g.htod(d, src, sz)) {
        if (d) g.mem_free(d);
        return 0;
    }
    return (uint64_t)d;
}

void rg_free(uint64_t d)
{
    if (g_mod && d) {
        g.ctx_set_current(g_mod->ctx);
        g.mem_free((CUdeviceptr)d);
    }
}

}   /* extern "C" */
