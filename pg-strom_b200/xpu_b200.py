"""
Python binding of the C ABI in include/xpu_b200.h (ctypes).

The product is libxpu_b200.so; this module only marshals buffers for tests
and the benchmark.  Loading fails loudly when the library is missing: there
is no fallback implementation.
"""
import ctypes
import os
import struct

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
LIB_PATH = os.path.join(HERE, "libxpu_b200.so")

ERRCODE = {0: "SUCCESS", ord("E"): "DEVICE_ERROR", ord("F"): "DEVICE_FATAL",
           ord("d"): "SUSPEND_NO_SPACE", ord("f"): "SUSPEND_FALLBACK"}


class KernErrorbuf(ctypes.Structure):
    _fields_ = [("errcode", ctypes.c_uint32), ("lineno", ctypes.c_int32),
                ("filename", ctypes.c_char * 33), ("funcname", ctypes.c_char * 65),
                ("message", ctypes.c_char * 201)]


class XpuB200Error(RuntimeError):
    def __init__(self, rc, ebuf):
        self.errcode = rc
        self.message = ebuf.message.decode(errors="replace")
        super().__init__(f"[{ERRCODE.get(rc, rc)}] {ebuf.funcname.decode()}:{ebuf.lineno} {self.message}")


_LIB = None


def lib():
    global _LIB
    if _LIB is None:
        if not os.path.exists(LIB_PATH):
            raise RuntimeError(f"{LIB_PATH} is missing: build it with pg-strom_b200/build.py")
        L = ctypes.CDLL(LIB_PATH)
        P, U64, I = ctypes.c_void_p, ctypes.c_uint64, ctypes.c_int
        EB = ctypes.POINTER(KernErrorbuf)
        L.xpuB200Init.argtypes = [I, U64, ctypes.POINTER(P), EB]
        L.xpuB200Shutdown.argtypes = [P]
        L.xpuB200OpenSession.argtypes = [P, P, U64, P, U64, ctypes.POINTER(P), EB]
        L.xpuB200ExecTask.argtypes = [P, P, I, P, EB]
        L.xpuB200ExecTaskDst.argtypes = [P, P, I, P, U64, I, ctypes.POINTER(U64), P, EB]
        L.xpuB200Final.argtypes = [P, P, U64, ctypes.POINTER(U64), P, EB]
        L.xpuB200MergeFinal.argtypes = [P, P, I, EB]
        L.xpuB200InnerCacheConfig.argtypes = [P, U64, ctypes.POINTER(U64), EB]
        L.xpuB200InnerRebuild.argtypes = [P, P, P, ctypes.c_uint32, ctypes.c_uint32, ctypes.POINTER(U64), EB]
        L.xpuB200CloseSession.argtypes = [P]
        L.xpuB200HandleCommand.argtypes = [P, ctypes.POINTER(P), P, P, U64, P, U64]
        L.xpuB200DeviceAlloc.argtypes = [P, U64, ctypes.POINTER(P)]
        L.xpuB200DeviceFree.argtypes = [P, P]
        L.xpuB200CopyToDevice.argtypes = [P, P, P, U64]
        L.xpuB200CopyToHost.argtypes = [P, P, P, U64]
        L.xpuB200TimeExecTask.argtypes = [P, P, I, ctypes.POINTER(ctypes.c_double), EB]
        L.xpuB200BatchCreate.argtypes = [P, P, ctypes.c_uint32, ctypes.POINTER(P), EB]
        L.xpuB200BatchExec.argtypes = [P, P, EB]
        L.xpuB200BatchTime.argtypes = [P, I, ctypes.POINTER(ctypes.c_double), EB]
        L.xpuB200BatchTune.argtypes = [P, ctypes.c_uint32, ctypes.c_char_p, U64, EB]
        L.xpuB200BatchDestroy.argtypes = [P]
        L.xpuB200Submit.argtypes = [P, P, I, ctypes.POINTER(U64), EB]
        L.xpuB200Poll.argtypes = [P, U64, I, ctypes.POINTER(I), P, EB]
        L.xpuB200ServeConfig.argtypes = [P, U64, ctypes.c_uint32, EB]
        L.xpuB200MemInfo.argtypes = [P, ctypes.POINTER(U64), ctypes.POINTER(U64), ctypes.POINTER(U64)]
        L.xpuB200FinalParts.argtypes = [P, ctypes.c_uint32, P, U64, ctypes.POINTER(U64), ctypes.POINTER(U64), EB]
        L.xpuB200ChunkCachePut.argtypes = [P, U64, ctypes.c_uint32, P, I, ctypes.POINTER(P), EB]
        L.xpuB200ChunkCacheGet.argtypes = [P, U64, ctypes.c_uint32, ctypes.POINTER(P)]
        L.xpuB200ChunkCacheRelease.argtypes = [P, P]
        L.xpuB200ChunkCacheConfig.argtypes = [P, U64, ctypes.POINTER(U64), EB]
        L.xpuB200ChunkReadDirect.argtypes = [P, ctypes.c_char_p, P, U64, P, ctypes.c_uint32, P, U64, I,
                                             ctypes.POINTER(ctypes.c_uint32), ctypes.POINTER(ctypes.c_uint32), EB]
        L.xpuB200MixCreate.argtypes = [P, ctypes.c_uint32, P, P, ctypes.POINTER(P), EB]
        L.xpuB200MixExec.argtypes = [P, P, P]
        L.xpuB200MixTime.argtypes = [P, I, ctypes.POINTER(ctypes.c_double), EB]
        L.xpuB200MixInfo.argtypes = [P, ctypes.POINTER(U64), ctypes.POINTER(U64),
                                     ctypes.POINTER(ctypes.c_uint32), ctypes.POINTER(ctypes.c_uint32),
                                     ctypes.POINTER(ctypes.c_uint32)]
        L.xpuB200MixDestroy.argtypes = [P]
        L.xpuB200SessionInfo.argtypes = [P, ctypes.c_char_p, U64]
        L.xpuB200HashBytes.argtypes = [P, ctypes.c_uint32]
        L.xpuB200HashBytes.restype = ctypes.c_uint32
        _LIB = L
    return _LIB


def _ptr(buf):
    if isinstance(buf, np.ndarray):
        return ctypes.c_void_p(buf.ctypes.data)
    if isinstance(buf, (bytes, bytearray)):
        return ctypes.cast(ctypes.c_char_p(bytes(buf)), ctypes.c_void_p)
    raise TypeError(type(buf))


def results_buffer(nrels):
    return np.zeros(96 + 12 * (nrels + 1) + 16, dtype=np.uint8)


def parse_results(buf):
    b = bytes(buf)
    nraw, nin, nout, nrels = struct.unpack_from("<IIII", b, 80)
    stats = [struct.unpack_from("<III", b, 96 + 12 * i)[2] for i in range(nrels)]
    final_nitems, = struct.unpack_from("<I", b, 24)
    return {"nitems_raw": nraw, "nitems_in": nin, "nitems_out": nout, "num_rels": nrels,
            "depth_out": stats, "final_nitems": final_nitems}


ADMIT_FREE_HBM = (1 << 64) - 1          # XPU_B200_ADMIT_FREE_HBM


class Device:
    def __init__(self, dindex=0, hbm_budget=0):
        self.h = ctypes.c_void_p()
        e = KernErrorbuf()
        rc = lib().xpuB200Init(dindex, hbm_budget, ctypes.byref(self.h), ctypes.byref(e))
        if rc:
            raise XpuB200Error(rc, e)

    def alloc(self, nbytes):
        p = ctypes.c_void_p()
        if lib().xpuB200DeviceAlloc(self.h, nbytes, ctypes.byref(p)):
            raise MemoryError(f"device allocation of {nbytes} bytes failed")
        return p.value

    def free(self, dptr):
        lib().xpuB200DeviceFree(self.h, ctypes.c_void_p(dptr))

    def inner_cache(self, max_bytes=None):
        """Set the budget of inner relations kept across sessions
        (xpuB200InnerCacheConfig); returns the bytes cached now."""
        e = KernErrorbuf()
        got = ctypes.c_uint64()
        rc = lib().xpuB200InnerCacheConfig(self.h, (1 << 64) - 1 if max_bytes is None else max_bytes,
                                           ctypes.byref(got), ctypes.byref(e))
        if rc:
            raise XpuB200Error(rc, e)
        return got.value

    def inner_rebuild(self, dst, src, divisor=0, remainder=0):
        """Append the rows of the device chunk src (HASH or ROW, tuples
        carrying their hash) into the device KDS_FORMAT_HASH buffer dst
        (xpuB200InnerRebuild); with divisor >= 2 only the rows whose hash %
        divisor == remainder.  Returns the bytes dst's rows take."""
        e = KernErrorbuf()
        req = ctypes.c_uint64()
        rc = lib().xpuB200InnerRebuild(self.h, ctypes.c_void_p(dst), ctypes.c_void_p(src), divisor, remainder,
                                       ctypes.byref(req), ctypes.byref(e))
        if rc:
            raise XpuB200Error(rc, e)
        return req.value

    def download(self, dptr, nbytes):
        """Copy nbytes of device memory at dptr into a new uint8 array."""
        out = np.zeros(nbytes, dtype=np.uint8)
        if lib().xpuB200CopyToHost(self.h, _ptr(out), ctypes.c_void_p(dptr), nbytes):
            raise RuntimeError("download failed")
        return out

    def upload(self, arr: np.ndarray, align_pages=True):
        """Copy a KDS chunk into device memory; heap pages land 16B aligned."""
        shift = 0
        if align_pages and arr.size > 48:
            fmt = bytes(arr[24:25])
            if fmt == b"b":
                block_offset = int(np.frombuffer(arr[44:48].tobytes(), dtype=np.uint32)[0])
                shift = (16 - (block_offset & 15)) & 15
        base = self.alloc(arr.nbytes + 256)
        if lib().xpuB200CopyToDevice(self.h, ctypes.c_void_p(base + shift), _ptr(arr), arr.nbytes):
            raise RuntimeError("upload failed")
        return base, base + shift

    def chunk_put(self, table, chunk_no, kds, on_device=False):
        """xpuB200ChunkCachePut: the device address of chunk chunk_no of
        table (placed now, or found resident), pinned until chunk_release."""
        p = ctypes.c_void_p()
        e = KernErrorbuf()
        src = ctypes.c_void_p(kds) if on_device else _ptr(kds)
        rc = lib().xpuB200ChunkCachePut(self.h, table, chunk_no, src, 1 if on_device else 0,
                                        ctypes.byref(p), ctypes.byref(e))
        if rc:
            raise XpuB200Error(rc, e)
        return p.value

    def chunk_get(self, table, chunk_no):
        """The device address of a resident chunk (pinned), or None."""
        p = ctypes.c_void_p()
        return p.value if lib().xpuB200ChunkCacheGet(self.h, table, chunk_no, ctypes.byref(p)) == 0 else None

    def chunk_release(self, dptr):
        return lib().xpuB200ChunkCacheRelease(self.h, ctypes.c_void_p(dptr)) == 0

    def chunk_cache(self, max_bytes=None):
        """Set the chunk cache's budget; returns the bytes held now."""
        got = ctypes.c_uint64()
        e = KernErrorbuf()
        rc = lib().xpuB200ChunkCacheConfig(self.h, (1 << 64) - 1 if max_bytes is None else max_bytes,
                                           ctypes.byref(got), ctypes.byref(e))
        if rc:
            raise XpuB200Error(rc, e)
        return got.value

    def read_direct(self, path, kds_head, base_offset, io_chunks, dptr, dsize, try_direct=True):
        """xpuB200ChunkReadDirect: the first base_offset bytes of kds_head,
        then the file pages of io_chunks ((m_offset, fchunk_id, nr_pages)
        of XPU_B200_IO_PAGE-byte pages) into device memory at dptr.
        Returns (pages read by cuFile, pages read through the bounce
        buffer)."""
        ioc = np.array(list(io_chunks), dtype=[("m_offset", "<u8"), ("fchunk_id", "<u4"), ("nr_pages", "<u4")])
        nd, nv = ctypes.c_uint32(), ctypes.c_uint32()
        e = KernErrorbuf()
        rc = lib().xpuB200ChunkReadDirect(self.h, os.fsencode(path), _ptr(kds_head), base_offset,
                                          _ptr(ioc) if len(ioc) else None, len(ioc),
                                          ctypes.c_void_p(dptr), dsize, 1 if try_direct else 0,
                                          ctypes.byref(nd), ctypes.byref(nv), ctypes.byref(e))
        if rc:
            raise XpuB200Error(rc, e)
        return nd.value, nv.value

    def mem_info(self):
        """(free, total, reserve) bytes of device memory (xpuB200MemInfo)."""
        fr, tot, res = ctypes.c_uint64(), ctypes.c_uint64(), ctypes.c_uint64()
        lib().xpuB200MemInfo(self.h, ctypes.byref(fr), ctypes.byref(tot), ctypes.byref(res))
        return fr.value, tot.value, res.value

    def serve_config(self, admit_bytes=0, alone_units=0):
        """Admission budget (ADMIT_FREE_HBM: by free device memory) and
        the size at which a command runs alone (0 keeps a value)."""
        e = KernErrorbuf()
        rc = lib().xpuB200ServeConfig(self.h, admit_bytes, alone_units, ctypes.byref(e))
        if rc:
            raise XpuB200Error(rc, e)

    def submit(self, sess, kds, on_device=False):
        """Queue one chunk command of sess; returns its ticket.  A host
        chunk must stay alive until the ticket is polled done."""
        t = ctypes.c_uint64()
        e = KernErrorbuf()
        p = ctypes.c_void_p(kds) if on_device else _ptr(kds)
        rc = lib().xpuB200Submit(sess.h, p, 1 if on_device else 0, ctypes.byref(t), ctypes.byref(e))
        if rc:
            raise XpuB200Error(rc, e)
        return t.value

    def poll(self, ticket, nrels=0, wait=True):
        """Results of a submitted command (None while it runs, wait=False)."""
        res = results_buffer(nrels)
        struct.pack_into("<I", res, 92, nrels)
        done = ctypes.c_int()
        e = KernErrorbuf()
        rc = lib().xpuB200Poll(self.h, ticket, 1 if wait else 0, ctypes.byref(done), _ptr(res), ctypes.byref(e))
        if rc:
            raise XpuB200Error(rc, e)
        return parse_results(res) if done.value else None

    def close(self):
        if self.h:
            lib().xpuB200Shutdown(self.h)
            self.h = ctypes.c_void_p()


class Session:
    def __init__(self, dev: Device, session: bytes, kmrels: np.ndarray = None, nrels=0):
        self.dev = dev
        self.nrels = nrels
        self.h = ctypes.c_void_p()
        self._session = np.frombuffer(session, dtype=np.uint8).copy()
        self._kmrels = kmrels
        e = KernErrorbuf()
        rc = lib().xpuB200OpenSession(dev.h, _ptr(self._session), self._session.nbytes,
                                      _ptr(kmrels) if kmrels is not None else None,
                                      kmrels.nbytes if kmrels is not None else 0,
                                      ctypes.byref(self.h), ctypes.byref(e))
        if rc:
            raise XpuB200Error(rc, e)

    def exec(self, kds, on_device=False):
        res = results_buffer(self.nrels)
        struct.pack_into("<I", res, 92, self.nrels)
        e = KernErrorbuf()
        p = ctypes.c_void_p(kds) if on_device else _ptr(kds)
        rc = lib().xpuB200ExecTask(self.h, p, 1 if on_device else 0, _ptr(res), ctypes.byref(e))
        if rc:
            raise XpuB200Error(rc, e)
        return parse_results(res)

    def exec_dst(self, kds, dst_size=1 << 20, on_device=False):
        """Run one chunk of a projection session.  Returns (kds_dst bytes,
        results, retried): kds_dst is dst_size bytes, or the size the
        library asked for when the rows did not fit (SUSPEND_NO_SPACE,
        then the chunk runs again)."""
        retried = False
        while True:
            res = results_buffer(self.nrels)
            struct.pack_into("<I", res, 92, self.nrels)
            e = KernErrorbuf()
            req = ctypes.c_uint64()
            dst = np.zeros(dst_size, dtype=np.uint8)
            p = ctypes.c_void_p(kds) if on_device else _ptr(kds)
            rc = lib().xpuB200ExecTaskDst(self.h, p, 1 if on_device else 0, _ptr(dst), dst.nbytes, 0,
                                          ctypes.byref(req), _ptr(res), ctypes.byref(e))
            if rc == ord("d") and not retried:
                dst_size = (req.value + 7) & ~7
                retried = True
                continue
            if rc:
                raise XpuB200Error(rc, e)
            return dst, parse_results(res), retried

    def time_exec(self, dptr, niters):
        ms = ctypes.c_double()
        e = KernErrorbuf()
        rc = lib().xpuB200TimeExecTask(self.h, ctypes.c_void_p(dptr), niters, ctypes.byref(ms), ctypes.byref(e))
        if rc:
            raise XpuB200Error(rc, e)
        return ms.value

    def final(self, out=None):
        """kds_final (and the results).  With 'out' (a uint8 array, e.g. of
        pinned memory) large enough, kds_final is written there in one call
        and a view of it is returned."""
        req = ctypes.c_uint64()
        res = results_buffer(self.nrels)
        struct.pack_into("<I", res, 92, self.nrels)
        e = KernErrorbuf()
        if out is not None:
            rc = lib().xpuB200Final(self.h, _ptr(out), out.nbytes, ctypes.byref(req), _ptr(res), ctypes.byref(e))
            if rc == 0:
                return (out[:req.value] if req.value else None), parse_results(res)
            if rc != ord("d"):
                raise XpuB200Error(rc, e)
        rc = lib().xpuB200Final(self.h, None, 0, ctypes.byref(req), _ptr(res), ctypes.byref(e))
        if rc:
            raise XpuB200Error(rc, e)
        if req.value == 0:
            return None, parse_results(res)
        buf = np.zeros(req.value, dtype=np.uint8)
        rc = lib().xpuB200Final(self.h, _ptr(buf), buf.nbytes, ctypes.byref(req), _ptr(res), ctypes.byref(e))
        if rc:
            raise XpuB200Error(rc, e)
        return buf, parse_results(res)

    def final_parts(self, nparts, out_dptr=None, out_size=0):
        """xpuB200FinalParts: the groups split into nparts hash partitions,
        written back to back into device memory at out_dptr (out_size
        bytes).  Returns the nparts + 1 part offsets (the last: the bytes
        needed); with out_dptr None only the offsets are computed."""
        offs = (ctypes.c_uint64 * (nparts + 1))()
        req = ctypes.c_uint64()
        e = KernErrorbuf()
        rc = lib().xpuB200FinalParts(self.h, nparts, ctypes.c_void_p(out_dptr) if out_dptr else None,
                                     out_size if out_dptr else 0, offs, ctypes.byref(req), ctypes.byref(e))
        if rc:
            raise XpuB200Error(rc, e)
        return list(offs)

    def merge_final(self, kds, on_device=False):
        """Merge another session's kds_final (a uint8 array from final(), or
        a device address with on_device) into this session's groups."""
        e = KernErrorbuf()
        p = ctypes.c_void_p(kds) if on_device else _ptr(kds)
        rc = lib().xpuB200MergeFinal(self.h, p, 1 if on_device else 0, ctypes.byref(e))
        if rc:
            raise XpuB200Error(rc, e)

    def batch(self, dptrs):
        return Batch(self, dptrs)

    def info(self):
        import json
        b = ctypes.create_string_buffer(4096)
        lib().xpuB200SessionInfo(self.h, b, 4096)
        return json.loads(b.value.decode())

    def close(self):
        if self.h:
            lib().xpuB200CloseSession(self.h)
            self.h = ctypes.c_void_p()


class Batch:
    """Many device-resident chunks executed by one persistent launch."""

    def __init__(self, sess: Session, dptrs):
        self.sess = sess
        arr = (ctypes.c_void_p * len(dptrs))(*dptrs)
        self.h = ctypes.c_void_p()
        e = KernErrorbuf()
        rc = lib().xpuB200BatchCreate(sess.h, arr, len(dptrs), ctypes.byref(self.h), ctypes.byref(e))
        if rc:
            raise XpuB200Error(rc, e)

    def exec(self):
        res = results_buffer(self.sess.nrels)
        struct.pack_into("<I", res, 92, self.sess.nrels)
        e = KernErrorbuf()
        rc = lib().xpuB200BatchExec(self.h, _ptr(res), ctypes.byref(e))
        if rc:
            raise XpuB200Error(rc, e)
        return parse_results(res)

    def time(self, niters):
        ms = ctypes.c_double()
        e = KernErrorbuf()
        rc = lib().xpuB200BatchTime(self.h, niters, ctypes.byref(ms), ctypes.byref(e))
        if rc:
            raise XpuB200Error(rc, e)
        return ms.value

    def tune(self):
        """Measure the session's launch shapes on this batch and keep the
        fastest (xpuB200BatchTune); returns the report (a dict)."""
        import json
        b = ctypes.create_string_buffer(8192)
        e = KernErrorbuf()
        rc = lib().xpuB200BatchTune(self.h, 0, b, 8192, ctypes.byref(e))
        if rc:
            raise XpuB200Error(rc, e)
        return json.loads(b.value.decode())

    def close(self):
        if self.h:
            lib().xpuB200BatchDestroy(self.h)
            self.h = ctypes.c_void_p()


class Mix:
    """Chunk commands of many sessions run as one persistent launch (a
    captured CUDA graph, replayed by every run)."""

    def __init__(self, dev: Device, sessions, dptrs):
        self.dev = dev
        self.sessions = list(sessions)
        n = len(self.sessions)
        self.h = ctypes.c_void_p()
        hs = (ctypes.c_void_p * n)(*[s.h.value for s in self.sessions])
        ks = (ctypes.c_void_p * n)(*dptrs)
        e = KernErrorbuf()
        rc = lib().xpuB200MixCreate(dev.h, n, hs, ks, ctypes.byref(self.h), ctypes.byref(e))
        if rc:
            raise XpuB200Error(rc, e)

    def exec(self):
        """Returns [(results dict or None, error message or None)] per command."""
        n = len(self.sessions)
        bufs = []
        for s in self.sessions:
            r = results_buffer(s.nrels)
            struct.pack_into("<I", r, 92, s.nrels)
            bufs.append(r)
        ptrs = (ctypes.c_void_p * n)(*[b.ctypes.data for b in bufs])
        errs = (KernErrorbuf * n)()
        lib().xpuB200MixExec(self.h, ptrs, errs)
        out = []
        for b, e in zip(bufs, errs):
            if e.errcode:
                out.append((None, XpuB200Error(e.errcode, e)))
            else:
                out.append((parse_results(b), None))
        return out

    def time(self, niters):
        ms = ctypes.c_double()
        e = KernErrorbuf()
        rc = lib().xpuB200MixTime(self.h, niters, ctypes.byref(ms), ctypes.byref(e))
        if rc:
            raise XpuB200Error(rc, e)
        return ms.value

    def info(self):
        b, u = ctypes.c_uint64(), ctypes.c_uint64()
        it, nl, ns = ctypes.c_uint32(), ctypes.c_uint32(), ctypes.c_uint32()
        lib().xpuB200MixInfo(self.h, ctypes.byref(b), ctypes.byref(u), ctypes.byref(it), ctypes.byref(nl),
                             ctypes.byref(ns))
        return {"bytes": b.value, "units": u.value, "items": it.value, "launches": nl.value,
                "specialised": ns.value}

    def close(self):
        if self.h:
            lib().xpuB200MixDestroy(self.h)
            self.h = ctypes.c_void_p()
