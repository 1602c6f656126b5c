"""ctypes access to the reference correlator's own CPU hot path, compiled from
the reference sources into oracle/_ref/libdifxref.so by oracle/Makefile.ref
(harness: oracle/ref_harness.cpp).

Oracle test infrastructure: used to pin the C restatement (oracle/fxoracle.c),
to generate golden fixtures, and as the timed CPU baseline.
"""
from __future__ import annotations

import ctypes
import os
import tempfile
from typing import List, Optional, Sequence, Tuple

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
LIB_PATH = os.path.join(HERE, "_ref", "libdifxref.so")

_lib = None


def available() -> bool:
    return os.path.exists(LIB_PATH)


def lib():
    global _lib
    if _lib is None:
        L = ctypes.CDLL(LIB_PATH)
        vp, ip, fp, dp = ctypes.c_void_p, ctypes.POINTER(ctypes.c_int), ctypes.POINTER(ctypes.c_float), ctypes.POINTER(ctypes.c_double)
        L.dref_open.restype = vp
        L.dref_open.argtypes = [ctypes.c_char_p, ctypes.c_int]
        L.dref_close.argtypes = [vp]
        L.dref_info.argtypes = [vp, ip]
        L.dref_layout.argtypes = [vp, ip]
        L.dref_process_subint.argtypes = [vp, ctypes.c_int, ctypes.POINTER(ctypes.c_void_p), ip, ip, ip, ip,
                                          ctypes.POINTER(ctypes.c_void_p), ctypes.c_int, ctypes.c_int, ctypes.c_int, fp]
        L.dref_mode_fft.argtypes = [vp, ctypes.c_int, ctypes.c_void_p, ctypes.c_int, ctypes.c_int, ctypes.c_int, ctypes.c_int,
                                    ctypes.c_void_p, ctypes.c_int, ctypes.c_int, ctypes.c_int, ctypes.c_int, fp, fp, fp]
        L.dref_interpolator.argtypes = [vp, ctypes.c_int, ctypes.c_int, ctypes.c_int, ctypes.c_int, dp]
        L.dref_unpack.argtypes = [ctypes.c_char_p, ctypes.c_void_p, ctypes.c_int, ctypes.c_int, fp]
        L.dref_visibility_write.argtypes = [vp, ctypes.POINTER(fp), ctypes.c_int]
        L.dref_vdif_mux.argtypes = [ctypes.c_void_p, ctypes.c_int, ctypes.c_int, ip, ctypes.c_int, ctypes.c_int,
                                    ctypes.c_int, ctypes.c_void_p]
        _lib = L
    return _lib


def _fptr(a: np.ndarray):
    return a.ctypes.data_as(ctypes.POINTER(ctypes.c_float))


def _iarr(v: Sequence[int]):
    return (ctypes.c_int * len(v))(*v)


class RefCorrelator:
    """The reference Configuration + Mode objects for one job (config 0)."""

    def __init__(self, job, nthreads: int = 1, workdir: Optional[str] = None, **input_kw):
        from difxinput import write_job_files
        self._tmp = None
        if workdir is None:
            self._tmp = tempfile.TemporaryDirectory(prefix="fxref_")
            workdir = self._tmp.name
        self.job = job
        self.input_path = write_job_files(job, workdir, **input_kw)
        self.h = lib().dref_open(self.input_path.encode(), nthreads)
        if not self.h:
            raise RuntimeError("reference rejected the job (set ORACLE_REF_VERBOSE=1 for its alerts)")
        info = (ctypes.c_int * 6)()
        lib().dref_info(self.h, info)
        self.corelen, self.blockspersend, self.numds, self.numbl, self.nbuffered, self.maxproducts = list(info)

    def close(self):
        if self.h:
            lib().dref_close(self.h)
            self.h = None
        if self._tmp is not None:
            self._tmp.cleanup()
            self._tmp = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    def visibility_write(self, subint_results: List[np.ndarray]) -> bytes:
        """The reference Visibility: addData of each subint core result, then
        writedata; returns the bytes of the SWIN file it wrote."""
        import glob
        outdir = os.path.splitext(self.input_path)[0] + ".difx"
        os.makedirs(outdir, exist_ok=True)
        for f in glob.glob(os.path.join(outdir, "DIFX_*")) + glob.glob(os.path.join(outdir, "PCAL_*")):
            os.remove(f)
        arrs = [np.ascontiguousarray(r, dtype=np.float32) for r in subint_results]
        ptrs = (ctypes.POINTER(ctypes.c_float) * len(arrs))(*[_fptr(a) for a in arrs])
        rc = lib().dref_visibility_write(self.h, ptrs, len(arrs))
        if rc != 0:
            raise RuntimeError("reference Visibility not configured")
        self.pcal_files = {}
        for name in glob.glob(os.path.join(outdir, "PCAL_*")):
            with open(name, "rb") as f:
                self.pcal_files[os.path.basename(name)] = f.read()
        files = glob.glob(os.path.join(outdir, "DIFX_*"))
        if not files:
            return b""
        with open(files[0], "rb") as f:
            return f.read()

    # ---- the integration flow (oracle/fxb_config_adapter.cpp)
    def fxb_desc_address(self, xmac_kind: int = 0) -> int:
        """Address of the fxb_job_desc that fxb_desc_from_configuration builds
        from this job's stock Configuration (kept alive by the library)."""
        L = lib()
        L.dref_fxb_desc.restype = ctypes.c_void_p
        L.dref_fxb_desc.argtypes = [ctypes.c_void_p, ctypes.c_int, ctypes.c_char_p, ctypes.c_int]
        err = ctypes.create_string_buffer(256)
        p = L.dref_fxb_desc(self.h, xmac_kind, err, 256)
        if not p:
            raise RuntimeError("adapter: " + err.value.decode())
        return p

    def fxb_interpolators(self, scan: int, sec: int, ns: int) -> Tuple[np.ndarray, int]:
        L = lib()
        L.dref_fxb_interpolators.argtypes = [ctypes.c_void_p, ctypes.c_int, ctypes.c_int, ctypes.c_int,
                                             ctypes.POINTER(ctypes.c_double)]
        out = np.zeros(3 * self.numds, dtype=np.float64)
        missing = L.dref_fxb_interpolators(self.h, scan, sec, ns, out.ctypes.data_as(ctypes.POINTER(ctypes.c_double)))
        return out.reshape(self.numds, 3), missing

    def fxb_correlate(self, libpath: str, subints, xmac_kind: int = 0) -> np.ndarray:
        """The adapter's integration flow against the product library at
        libpath: subints = [(inputs, sec, ns)] with inputs per datastream
        (bytes, datasec, datans); returns the product's core result."""
        L = lib()
        L.dref_fxb_correlate.restype = ctypes.c_int
        L.dref_fxb_correlate.argtypes = [ctypes.c_void_p, ctypes.c_char_p, ctypes.c_int, ctypes.c_int,
                                         ctypes.POINTER(ctypes.c_void_p), ctypes.POINTER(ctypes.c_longlong),
                                         ctypes.POINTER(ctypes.c_int), ctypes.POINTER(ctypes.c_int),
                                         ctypes.POINTER(ctypes.c_int), ctypes.POINTER(ctypes.c_int),
                                         ctypes.POINTER(ctypes.c_float), ctypes.c_longlong, ctypes.c_char_p,
                                         ctypes.c_int]
        keep = [np.ascontiguousarray(b) for inputs, _, _ in subints for b, _, _ in inputs]
        bufs = (ctypes.c_void_p * len(keep))(*[k.ctypes.data for k in keep])
        nb = (ctypes.c_longlong * len(keep))(*[k.size for k in keep])
        dsec = _iarr([x for inputs, _, _ in subints for _, x, _ in inputs])
        dns = _iarr([x for inputs, _, _ in subints for _, _, x in inputs])
        sec = _iarr([s for _, s, _ in subints])
        ns = _iarr([n for _, _, n in subints])
        out = np.zeros(2 * self.corelen, dtype=np.float32)
        err = ctypes.create_string_buffer(512)
        rc = L.dref_fxb_correlate(self.h, libpath.encode(), xmac_kind, len(subints), bufs, nb, dsec, dns, sec, ns,
                                  _fptr(out), out.size, err, 512)
        if rc != 0:
            raise RuntimeError("integration flow: " + err.value.decode())
        return out

    def datastream(self, ds: int, factor: int, nseg: int) -> "RefRing":
        """The reference's VDIF datastream ds with nseg segments of
        factor / nseg times the largest subint's bytes."""
        L = lib()
        L.dref_ds_create.restype = ctypes.c_void_p
        L.dref_ds_create.argtypes = [ctypes.c_void_p, ctypes.c_int, ctypes.c_int, ctypes.c_int,
                                     ctypes.POINTER(ctypes.c_int)]
        out = (ctypes.c_int * 6)()
        d = L.dref_ds_create(self.h, ds, factor, nseg, out)
        ring = RefRing(d, *list(out))
        ring.parent = self          # the datastream reads the job's configuration
        return ring

    def layout(self) -> np.ndarray:
        nf = len(self.job.freqs)
        n = 2 * nf * self.numbl + 3 * self.numds
        out = np.zeros(n, dtype=np.int32)
        lib().dref_layout(self.h, out.ctypes.data_as(ctypes.POINTER(ctypes.c_int)))
        return out

    def process_subint(self, inputs: List[Tuple[np.ndarray, int, int]], validflags: List[np.ndarray],
                       scan: int, sec: int, ns: int, coreresult: Optional[np.ndarray] = None,
                       nthreads: int = 1) -> np.ndarray:
        if coreresult is None:
            coreresult = np.zeros(2 * self.corelen, dtype=np.float32)
        n = len(inputs)
        bufs = (ctypes.c_void_p * n)(*[b.ctypes.data for b, _, _ in inputs])
        vflags = (ctypes.c_void_p * n)(*[v.ctypes.data for v in validflags])
        lib().dref_process_subint(self.h, nthreads, bufs, _iarr([b.size for b, _, _ in inputs]),
                                  _iarr([0] * n), _iarr([s for _, s, _ in inputs]), _iarr([x for _, _, x in inputs]),
                                  vflags, scan, sec, ns, _fptr(coreresult))
        return coreresult

    def mode_fft(self, ds: int, buf: np.ndarray, dsec: int, dns: int, validflags: np.ndarray,
                 sec: int, ns: int, fftindex: int):
        st = self.job.stations[ds]
        nchan = self.job.station_nchan(ds)
        spec = np.zeros((st.nband, nchan, 2), dtype=np.float32)
        ac = np.zeros((st.nband, nchan, 2), dtype=np.float32)
        w = np.zeros(1, dtype=np.float32)
        lib().dref_mode_fft(self.h, ds, buf.ctypes.data, buf.size, 0, dsec, dns, validflags.ctypes.data,
                            0, sec, ns, fftindex, _fptr(spec), _fptr(w), _fptr(ac))
        return spec[..., 0] + 1j * spec[..., 1], float(w[0]), ac[..., 0] + 1j * ac[..., 1]

    def interpolator(self, ds: int, sec: int, ns: int) -> np.ndarray:
        c = (ctypes.c_double * 3)()
        rc = lib().dref_interpolator(self.h, ds, 0, sec, ns, c)
        if rc != 0:
            raise RuntimeError("no delay model for that time")
        return np.array(list(c))


def unpack(formatname: str, data: np.ndarray, offsetsamples: int, nsamp: int, nchan: int):
    out = np.zeros((nchan, nsamp), dtype=np.float32)
    good = lib().dref_unpack(formatname.encode(), data.ctypes.data, offsetsamples, nsamp, _fptr(out))
    return out, good


def vdif_mux(data: np.ndarray, nthreads: int, thread_ids: Sequence[int], framebytes: int, fps: int,
             nbits: int) -> bytes:
    """The reference VDIFMuxer on one read: the single-thread frames it writes."""
    data = np.ascontiguousarray(data, dtype=np.uint8)
    nout = (data.size // framebytes) // nthreads
    out = np.zeros(max(1, nout * ((framebytes - 32) * nthreads + 32)), dtype=np.uint8)
    n = lib().dref_vdif_mux(data.ctypes.data, data.size, nthreads, _iarr(list(thread_ids)), framebytes, fps, nbits,
                            out.ctypes.data)
    if n < 0:
        raise RuntimeError("reference VDIF muxer rejected the read")
    return out[:n].tobytes()


class RefRing:
    """DataStream control blocks from the stock VDIFDataStream code."""

    def __init__(self, d, readbytes, bufferbytes, nsinc, sendbytes, controllength, guard_ns):
        self.d = d
        self.readbytes, self.bufferbytes, self.nsinc = readbytes, bufferbytes, nsinc
        self.sendbytes, self.controllength, self.guard_ns = sendbytes, controllength, guard_ns

    def control(self, segs, at: int, keep: bool, lastvalid: int, scan: int, sec: int, ns: int):
        """segs: per segment (scan, seconds, ns, readto, validbytes).  Returns
        (bufferindex, atsegment, control words [scan, sec, ns, flags...])."""
        L = lib()
        L.dref_ds_control.restype = ctypes.c_int
        L.dref_ds_control.argtypes = [ctypes.c_void_p, ctypes.POINTER(ctypes.c_longlong), ctypes.c_int, ctypes.c_int,
                                      ctypes.c_int, ctypes.c_int, ctypes.c_int, ctypes.c_int,
                                      ctypes.POINTER(ctypes.c_int), ctypes.c_int]
        arr = np.ascontiguousarray(np.array(segs, dtype=np.int64).reshape(-1))
        out = (ctypes.c_int * 256)()
        n = L.dref_ds_control(self.d, arr.ctypes.data_as(ctypes.POINTER(ctypes.c_longlong)), at, int(keep),
                              lastvalid, scan, sec, ns, out, 256)
        if n < 0:
            raise RuntimeError("control buffer too small")
        return out[0], out[1], list(out[2:n])
