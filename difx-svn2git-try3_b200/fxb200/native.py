"""ctypes binding of the product library (libfxb200.so, C ABI in
include/fxb200.h) and the struct builder for a job description.

The library must exist: on import of :func:`lib` a missing or unloadable
libfxb200.so raises -- there is no CPU fallback.
"""
from __future__ import annotations

import ctypes
import os
from typing import List, Optional, Sequence, Tuple

import numpy as np

from .job import Job

PKG_DIR = os.path.dirname(os.path.abspath(__file__))
LIB_PATH = os.path.join(os.path.dirname(PKG_DIR), "csrc", "libfxb200.so")

FXB_STATUS = {
    0: "FXB_OK", 1: "FXB_ERR_ARG", 2: "FXB_ERR_UNSUPPORTED", 3: "FXB_ERR_CUDA", 4: "FXB_ERR_NOMEM",
    5: "FXB_ERR_STATE", 6: "FXB_ERR_TIMEOUT", 7: "FXB_ERR_BUSY", 8: "FXB_ERR_DATA",
}
XMAC_KIND = {"fp32": 0, "bf16": 1, "fp8": 2, "fp16": 3}


class FxbFreq(ctypes.Structure):
    _fields_ = [("freq_mhz", ctypes.c_double), ("bw_mhz", ctypes.c_double), ("nchan", ctypes.c_int32),
                ("lower_sideband", ctypes.c_int32), ("chans_to_avg", ctypes.c_int32), ("reserved", ctypes.c_int32)]


class FxbStation(ctypes.Structure):
    _fields_ = [("nbits", ctypes.c_int32), ("payload_bytes", ctypes.c_int32), ("header_bytes", ctypes.c_int32),
                ("nband", ctypes.c_int32), ("band_freq", ctypes.POINTER(ctypes.c_int32)),
                ("band_pol", ctypes.c_char_p), ("nzoom", ctypes.c_int32), ("mux_threads", ctypes.c_int32),
                ("zoom_freq", ctypes.POINTER(ctypes.c_int32)), ("zoom_pol", ctypes.c_char_p),
                ("pcal_interval_mhz", ctypes.c_double), ("pcal_base_mhz", ctypes.c_double),
                ("band_clock_us", ctypes.POINTER(ctypes.c_double)),
                ("band_clock_delta_us", ctypes.POINTER(ctypes.c_double)),
                ("band_phase_deg", ctypes.POINTER(ctypes.c_double)),
                ("band_lo_offset_hz", ctypes.POINTER(ctypes.c_double)),
                ("mux_raw", ctypes.c_int32), ("mux_thread_ids", ctypes.POINTER(ctypes.c_int32)),
                ("complex_sampling", ctypes.c_int32)]


class FxbBaseline(ctypes.Structure):
    _fields_ = [("ds1", ctypes.c_int32), ("ds2", ctypes.c_int32), ("nprod", ctypes.c_int32),
                ("prod_freq", ctypes.POINTER(ctypes.c_int32)), ("prod_band1", ctypes.POINTER(ctypes.c_int32)),
                ("prod_band2", ctypes.POINTER(ctypes.c_int32))]


class FxbJobDesc(ctypes.Structure):
    _fields_ = [("nfreq", ctypes.c_int32), ("freqs", ctypes.POINTER(FxbFreq)),
                ("nstation", ctypes.c_int32), ("stations", ctypes.POINTER(FxbStation)),
                ("nbaseline", ctypes.c_int32), ("baselines", ctypes.POINTER(FxbBaseline)),
                ("subint_ns", ctypes.c_int64), ("fringe_rot_order", ctypes.c_int32),
                ("write_autocorrs", ctypes.c_int32), ("xmac_kind", ctypes.c_int32),
                ("max_subints_in_flight", ctypes.c_int32)]


class DescHolder:
    """Owns every ctypes array the descriptor points into."""

    def __init__(self, job: Job, xmac: str = "fp32", inflight: int = 2):
        job.validate()
        self.keep = []
        fr = (FxbFreq * len(job.freqs))()
        for i, f in enumerate(job.freqs):
            fr[i] = FxbFreq(f.freq_mhz, f.bw_mhz, f.nchan, 1 if f.sideband == "L" else 0, f.chans_to_avg, 0)
        st = (FxbStation * len(job.stations))()
        for i, s in enumerate(job.stations):
            bf = (ctypes.c_int32 * s.nband)(*[b[0] for b in s.bands])
            bp = ctypes.create_string_buffer("".join(b[1] for b in s.bands).encode(), s.nband + 1)
            nz = len(s.zoom_bands)
            zf = (ctypes.c_int32 * max(nz, 1))(*[b[0] for b in s.zoom_bands])
            zp = ctypes.create_string_buffer("".join(b[1] for b in s.zoom_bands).encode(), nz + 1)
            self.keep += [bf, bp, zf, zp]
            corr = [None] * 4
            if s.freq_corr:
                for q in range(4):
                    arr = (ctypes.c_double * s.nband)(*[s.band_corr(k)[q] for k in range(s.nband)])
                    self.keep.append(arr)
                    corr[q] = ctypes.cast(arr, ctypes.POINTER(ctypes.c_double))
            tids = None
            if s.mux_threads and s.mux_thread_ids:
                arr = (ctypes.c_int32 * s.mux_threads)(*s.mux_thread_ids)
                self.keep.append(arr)
                tids = ctypes.cast(arr, ctypes.POINTER(ctypes.c_int32))
            st[i] = FxbStation(s.nbits, s.payload_bytes, s.header_bytes, s.nband,
                               ctypes.cast(bf, ctypes.POINTER(ctypes.c_int32)), ctypes.cast(bp, ctypes.c_char_p),
                               nz, s.mux_threads, ctypes.cast(zf, ctypes.POINTER(ctypes.c_int32)),
                               ctypes.cast(zp, ctypes.c_char_p), s.pcal_interval_mhz, s.pcal_base_mhz, *corr,
                               1 if s.mux_raw else 0, tids, 1 if s.complex_sampling else 0)
        bl = (FxbBaseline * len(job.baselines))()
        for i, b in enumerate(job.baselines):
            pf, p1, p2 = [], [], []
            for f, pp in b.products:
                for x1, x2 in pp:
                    pf.append(f); p1.append(x1); p2.append(x2)
            a = (ctypes.c_int32 * len(pf))(*pf)
            c1 = (ctypes.c_int32 * len(pf))(*p1)
            c2 = (ctypes.c_int32 * len(pf))(*p2)
            self.keep += [a, c1, c2]
            bl[i] = FxbBaseline(b.ds1, b.ds2, len(pf), ctypes.cast(a, ctypes.POINTER(ctypes.c_int32)),
                                ctypes.cast(c1, ctypes.POINTER(ctypes.c_int32)),
                                ctypes.cast(c2, ctypes.POINTER(ctypes.c_int32)))
        self.keep += [fr, st, bl]
        self.desc = FxbJobDesc(len(job.freqs), ctypes.cast(fr, ctypes.POINTER(FxbFreq)),
                               len(job.stations), ctypes.cast(st, ctypes.POINTER(FxbStation)),
                               len(job.baselines), ctypes.cast(bl, ctypes.POINTER(FxbBaseline)),
                               job.subint_ns, job.fringe_rot_order, 1 if job.write_autocorrs else 0,
                               XMAC_KIND[xmac], inflight)

    def ptr(self):
        return ctypes.byref(self.desc)


class FxbSegment(ctypes.Structure):
    _fields_ = [("scan", ctypes.c_int32), ("sec", ctypes.c_int32), ("ns", ctypes.c_int32), ("readto", ctypes.c_int32),
                ("validbytes", ctypes.c_int64)]


class FxbRing(ctypes.Structure):
    _fields_ = [("nseg", ctypes.c_int32), ("readbytes", ctypes.c_int32), ("atsegment", ctypes.c_int32),
                ("keepreading", ctypes.c_int32), ("lastvalid", ctypes.c_int32), ("guard_ns", ctypes.c_int32),
                ("seg", ctypes.POINTER(FxbSegment))]


INVALID_SUBINT = -99999999


def _ring(segs, readbytes, at, keep, lastvalid, guard_ns):
    arr = (FxbSegment * len(segs))(*[FxbSegment(int(a), int(b), int(c), int(d), int(e)) for a, b, c, d, e in segs])
    return FxbRing(len(segs), readbytes, at, int(keep), lastvalid, guard_ns,
                   ctypes.cast(arr, ctypes.POINTER(FxbSegment))), arr


def job_datastream_control(job: Job, station: int, segs, readbytes: int, at: int, keep: bool, lastvalid: int,
                           scan: int, sec: int, ns: int, guard_ns: int = 0, delays=None):
    """DataStream control block of subint (scan, sec, ns) for a station, on
    a ring of segments (scan, seconds, ns, readto, validbytes) of readbytes
    each: (offset, nbytes, datasec, datans, validflags, atsegment), datasec
    INVALID_SUBINT when the ring has no data for the subint."""
    holder = DescHolder(job)
    npoly, order, p0, interval, coeffs = poly_arrays(job, station)
    ring, keep_alive = _ring(segs, readbytes, at, keep, lastvalid, guard_ns)
    T = job.blocks_per_send()
    flags = np.zeros(T // 30 + 1, dtype=np.int32)
    off, nb = ctypes.c_int64(), ctypes.c_int32()
    dsec, dns = ctypes.c_int32(), ctypes.c_int32()
    d = None if delays is None else (ctypes.c_double * 2)(*delays)
    check(lib().fxb_job_datastream_control(holder.ptr(), station, npoly, order, p0, interval,
                                           coeffs.ctypes.data_as(ctypes.POINTER(ctypes.c_double)), ctypes.byref(ring),
                                           scan, sec, ns, d, ctypes.byref(off), ctypes.byref(nb), ctypes.byref(dsec),
                                           ctypes.byref(dns), flags.ctypes.data_as(ctypes.POINTER(ctypes.c_int32)),
                                           flags.size), None, "job_datastream_control")
    return off.value, nb.value, dsec.value, dns.value, flags, ring.atsegment


def poly_arrays(job: Job, s: int) -> Tuple[int, int, float, int, np.ndarray]:
    """(npoly, order, poly0_sec, interval_s, coeffs) of station s, padded to
    a common order, in the form fxb_set_delay_poly takes."""
    polys = job.stations[s].polys
    order = max(len(p.coeffs) for p in polys) - 1
    coeffs = np.zeros((len(polys), order + 1))
    for i, p in enumerate(polys):
        coeffs[i, :len(p.coeffs)] = p.coeffs
        coeffs[i, 0] += job.stations[s].clock_us
    return len(polys), order, polys[0].start_sec, polys[0].interval_s, np.ascontiguousarray(coeffs.reshape(-1))


# ---------------------------------------------------------------- library
_lib = None


class FxbError(RuntimeError):
    pass


class FxbMemberSubint(ctypes.Structure):
    _fields_ = [("bufs", ctypes.POINTER(ctypes.c_void_p)), ("nbytes", ctypes.POINTER(ctypes.c_int64)),
                ("datasec", ctypes.POINTER(ctypes.c_int32)), ("datans", ctypes.POINTER(ctypes.c_int32)),
                ("validflags", ctypes.POINTER(ctypes.c_void_p))]


def lib():
    """Load libfxb200.so; raises when it is missing (no fallback)."""
    global _lib
    if _lib is not None:
        return _lib
    if not os.path.exists(LIB_PATH):
        raise FxbError("libfxb200.so not built at %s: run __graft_entry__.build()" % LIB_PATH)
    L = ctypes.CDLL(LIB_PATH)
    vp, i32, i64 = ctypes.c_void_p, ctypes.c_int32, ctypes.c_int64
    i32p, i64p, fp, dp = (ctypes.POINTER(ctypes.c_int32), ctypes.POINTER(ctypes.c_int64),
                          ctypes.POINTER(ctypes.c_float), ctypes.POINTER(ctypes.c_double))
    L.fxb_create.restype = vp
    L.fxb_create.argtypes = [ctypes.POINTER(FxbJobDesc), i32p]
    L.fxb_destroy.argtypes = [vp]
    L.fxb_last_error.restype = ctypes.c_char_p
    L.fxb_last_error.argtypes = [vp]
    L.fxb_set_delay_poly.argtypes = [vp, i32, i32, i32, ctypes.c_double, i32, dp]
    L.fxb_submit_subint.argtypes = [vp, ctypes.POINTER(ctypes.c_void_p), i64p, i32p, i32p,
                                    ctypes.POINTER(ctypes.c_void_p), i32, i32]
    L.fxb_submit_subint_device.argtypes = L.fxb_submit_subint.argtypes
    L.fxb_sync.argtypes = [vp]
    L.fxb_core_result_length.argtypes = [vp, i64p]
    L.fxb_layout.argtypes = [vp, i32p, ctypes.c_size_t]
    L.fxb_read_results.argtypes = [vp, fp, ctypes.c_size_t]
    L.fxb_reset.argtypes = [vp]
    L.fxb_last_timing.argtypes = [vp, fp, fp, fp]
    L.fxb_read_spectra.argtypes = [vp, i32, fp, ctypes.c_size_t, i32p, i32p]
    L.fxb_read_fft_weights.argtypes = [vp, fp, ctypes.c_size_t]
    L.fxb_vdif_unpack.argtypes = [ctypes.c_void_p, i64, i32, i32, i32, i32, i64, i32, fp, i32p]
    L.fxb_job_layout.argtypes = [ctypes.POINTER(FxbJobDesc), i32p, ctypes.c_size_t, i64p]
    L.fxb_job_datastream_control.argtypes = [ctypes.POINTER(FxbJobDesc), i32, i32, i32, ctypes.c_double, i32, dp,
                                             ctypes.POINTER(FxbRing), i32, i32, i32, dp, i64p, i32p, i32p, i32p, i32p,
                                             ctypes.c_size_t]
    L.fxb_datastream_control.argtypes = [vp, i32, ctypes.POINTER(FxbRing), i32, i32, i32, dp, i64p, i32p, i32p, i32p,
                                         i32p, ctypes.c_size_t]
    L.fxb_timing_enable.argtypes = [vp, i32]
    L.fxb_timing_read.argtypes = [vp, i32p, dp, dp, dp]
    L.fxb_get_stream.argtypes = [vp, ctypes.POINTER(ctypes.c_void_p)]
    L.fxb_read_results_device.argtypes = [vp, ctypes.c_void_p, ctypes.c_size_t]
    L.fxb_set_graphs.argtypes = [vp, i32]
    L.fxb_set_graphs.restype = ctypes.c_int
    L.fxb_autotune.argtypes = [vp, i32]
    L.fxb_autotune.restype = ctypes.c_int
    L.fxb_tuning_report.argtypes = [vp, ctypes.c_char_p, ctypes.c_size_t, ctypes.POINTER(ctypes.c_size_t)]
    L.fxb_tuning_report.restype = ctypes.c_int
    L.fxb_batch_autotune.argtypes = [vp, i32]
    L.fxb_batch_autotune.restype = ctypes.c_int
    L.fxb_batch_create.restype = vp
    L.fxb_batch_create.argtypes = [ctypes.POINTER(vp), i32, i32p]
    L.fxb_batch_submit.argtypes = [vp, ctypes.POINTER(FxbMemberSubint), i32, i32]
    L.fxb_batch_submit_device.argtypes = [vp, ctypes.POINTER(FxbMemberSubint), i32, i32]
    L.fxb_batch_submit_device.restype = ctypes.c_int
    L.fxb_batch_sync.argtypes = [vp]
    L.fxb_batch_set_graphs.argtypes = [vp, i32]
    L.fxb_batch_set_fused.argtypes = [vp, i32, ctypes.POINTER(i32)]
    L.fxb_batch_set_fused.restype = i32
    for name in ("fxb_batch_submit", "fxb_batch_sync", "fxb_batch_set_graphs"):
        getattr(L, name).restype = ctypes.c_int
    L.fxb_batch_get_stream.argtypes = [vp, ctypes.POINTER(ctypes.c_void_p)]
    L.fxb_batch_get_stream.restype = ctypes.c_int
    L.fxb_batch_last_error.restype = ctypes.c_char_p
    L.fxb_batch_last_error.argtypes = [vp]
    L.fxb_batch_destroy.argtypes = [vp]
    L.fxb_vdif_mux.argtypes = [vp, i64, i32, i32p, i32, i32, i32, vp, i64, i64p, vp]
    L.fxb_vdif_mux.restype = ctypes.c_int
    L.fxb_host_alloc.restype = vp
    L.fxb_host_alloc.argtypes = [ctypes.c_size_t, i32p]
    L.fxb_host_free.argtypes = [vp]
    for name in ("fxb_set_delay_poly", "fxb_submit_subint", "fxb_submit_subint_device", "fxb_sync",
                 "fxb_core_result_length", "fxb_layout", "fxb_read_results", "fxb_reset", "fxb_last_timing",
                 "fxb_read_spectra", "fxb_read_fft_weights", "fxb_vdif_unpack", "fxb_job_layout",
                 "fxb_timing_enable", "fxb_timing_read", "fxb_get_stream", "fxb_read_results_device"):
        getattr(L, name).restype = ctypes.c_int
    _lib = L
    return L


class _PinnedBlock:
    """A page-locked host allocation (fxb_host_alloc), freed with its last view."""

    def __init__(self, nbytes: int):
        st = ctypes.c_int32(0)
        self.ptr = lib().fxb_host_alloc(max(nbytes, 1), ctypes.byref(st))
        if not self.ptr:
            raise FxbError("fxb_host_alloc(%d) failed: %s" % (nbytes, FXB_STATUS.get(st.value, st.value)))
        self.nbytes = nbytes

    def __del__(self):
        if getattr(self, "ptr", None):
            lib().fxb_host_free(self.ptr)
            self.ptr = None


class PinnedArray(np.ndarray):
    """ndarray over page-locked host memory; views keep the block alive."""
    _block = None


def pinned_empty(nbytes: int) -> PinnedArray:
    """nbytes of page-locked host memory as a uint8 array (station buffers in
    this memory are copied to the device asynchronously)."""
    blk = _PinnedBlock(nbytes)
    raw = (ctypes.c_uint8 * max(nbytes, 1)).from_address(blk.ptr)
    a = np.frombuffer(raw, dtype=np.uint8, count=nbytes).view(PinnedArray)
    a._block = blk
    return a


def check(rc: int, ctx=None, what: str = "") -> None:
    if rc != 0:
        msg = ""
        try:
            m = lib().fxb_last_error(ctx)
            msg = m.decode() if m else ""
        except Exception:
            pass
        raise FxbError("%s failed: %s %s" % (what, FXB_STATUS.get(rc, rc), msg))


def _fptr(a: np.ndarray):
    return a.ctypes.data_as(ctypes.POINTER(ctypes.c_float))


class Correlator:
    """Python view of one fxb_ctx (the product path)."""

    def __init__(self, job: Job, xmac: str = "fp32", inflight: int = 2):
        self.job = job
        self.holder = DescHolder(job, xmac=xmac, inflight=inflight)
        st = ctypes.c_int32(0)
        self.ctx = lib().fxb_create(self.holder.ptr(), ctypes.byref(st))
        if not self.ctx:
            err = lib().fxb_last_error(None)
            raise FxbError("fxb_create: %s %s" % (FXB_STATUS.get(st.value, st.value), err.decode() if err else ""))
        n = ctypes.c_int64(0)
        check(lib().fxb_core_result_length(self.ctx, ctypes.byref(n)), self.ctx, "core_result_length")
        self.corelen = n.value
        for s in range(len(job.stations)):
            npoly, order, p0, interval, coeffs = poly_arrays(job, s)
            check(lib().fxb_set_delay_poly(self.ctx, s, npoly, order, p0, interval,
                                           coeffs.ctypes.data_as(ctypes.POINTER(ctypes.c_double))),
                  self.ctx, "set_delay_poly")

    def close(self):
        if getattr(self, "ctx", None):
            lib().fxb_destroy(self.ctx)
            self.ctx = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    def layout(self) -> np.ndarray:
        nf, nb, ns = len(self.job.freqs), len(self.job.baselines), len(self.job.stations)
        out = np.zeros(2 * nf * nb + 3 * ns, dtype=np.int32)
        check(lib().fxb_layout(self.ctx, out.ctypes.data_as(ctypes.POINTER(ctypes.c_int32)), out.size),
              self.ctx, "layout")
        return out

    def _submit(self, fn, ptrs: Sequence[int], nbytes: Sequence[int], dsec, dns, validflags, sec, ns):
        n = len(ptrs)
        bufs = (ctypes.c_void_p * n)(*ptrs)
        nb = (ctypes.c_int64 * n)(*nbytes)
        ds = (ctypes.c_int32 * n)(*dsec)
        dn = (ctypes.c_int32 * n)(*dns)
        if validflags is None:
            vf = None
        else:
            vf = (ctypes.c_void_p * n)(*[v.ctypes.data if v is not None else None for v in validflags])
        check(fn(self.ctx, bufs, nb, ds, dn, vf, sec, ns), self.ctx, "submit_subint")

    def submit(self, inputs: List[Tuple[np.ndarray, int, int]], sec: int, ns: int,
               validflags: Optional[List[np.ndarray]] = None) -> None:
        self._submit(lib().fxb_submit_subint, [b.ctypes.data for b, _, _ in inputs], [b.size for b, _, _ in inputs],
                     [s for _, s, _ in inputs], [x for _, _, x in inputs], validflags, sec, ns)

    def submit_device(self, ptrs: Sequence[int], nbytes: Sequence[int], dsec, dns, sec: int, ns: int,
                      validflags=None) -> None:
        self._submit(lib().fxb_submit_subint_device, ptrs, nbytes, dsec, dns, validflags, sec, ns)

    def submit_ptrs(self, ptrs: Sequence[int], nbytes: Sequence[int], dsec, dns, sec: int, ns: int,
                    validflags=None) -> None:
        """Submit from host memory given raw pointers (e.g. pinned buffers)."""
        self._submit(lib().fxb_submit_subint, ptrs, nbytes, dsec, dns, validflags, sec, ns)

    def set_graphs(self, on: bool = True):
        """Replay each slot's subint kernels as a CUDA graph (default) or launch them one by one."""
        check(lib().fxb_set_graphs(self.ctx, 1 if on else 0), self.ctx, "set_graphs")

    def autotune(self, rounds: int = 2):
        """Time the scheduling candidates over the next subints and keep the fastest (fxb_autotune)."""
        check(lib().fxb_autotune(self.ctx, rounds), self.ctx, "autotune")

    def tuning_report(self) -> str:
        need = ctypes.c_size_t(0)
        check(lib().fxb_tuning_report(self.ctx, None, 0, ctypes.byref(need)), self.ctx, "tuning_report")
        buf = ctypes.create_string_buffer(need.value)
        check(lib().fxb_tuning_report(self.ctx, buf, need.value, None), self.ctx, "tuning_report")
        return buf.value.decode()

    def results_into(self, out: np.ndarray) -> np.ndarray:
        check(lib().fxb_read_results(self.ctx, _fptr(out), out.size), self.ctx, "read_results")
        return out

    def sync(self):
        check(lib().fxb_sync(self.ctx), self.ctx, "sync")

    def results(self) -> np.ndarray:
        out = np.zeros(2 * self.corelen, dtype=np.float32)
        check(lib().fxb_read_results(self.ctx, _fptr(out), out.size), self.ctx, "read_results")
        return out

    def reset(self):
        check(lib().fxb_reset(self.ctx), self.ctx, "reset")

    def timing(self):
        a, b, c = ctypes.c_float(), ctypes.c_float(), ctypes.c_float()
        check(lib().fxb_last_timing(self.ctx, ctypes.byref(a), ctypes.byref(b), ctypes.byref(c)), self.ctx, "timing")
        return a.value, b.value, c.value

    def timing_enable(self, on: bool = True):
        check(lib().fxb_timing_enable(self.ctx, 1 if on else 0), self.ctx, "timing_enable")

    def timing_read(self):
        n = ctypes.c_int32(0)
        p, f, x = ctypes.c_double(), ctypes.c_double(), ctypes.c_double()
        check(lib().fxb_timing_read(self.ctx, ctypes.byref(n), ctypes.byref(p), ctypes.byref(f), ctypes.byref(x)),
              self.ctx, "timing_read")
        return n.value, p.value, f.value, x.value

    def stream(self) -> int:
        v = ctypes.c_void_p(0)
        check(lib().fxb_get_stream(self.ctx, ctypes.byref(v)), self.ctx, "get_stream")
        return v.value or 0

    def results_device(self, dev_ptr: int, nfloats: int):
        check(lib().fxb_read_results_device(self.ctx, ctypes.c_void_p(dev_ptr), nfloats), self.ctx,
              "read_results_device")

    def spectra(self, freq: int) -> np.ndarray:
        T = self.job.blocks_per_send()
        nchan = self.job.freqs[freq].nchan
        # rows: the recorded and zoom bands on this frequency (at most)
        rows = sum(1 for st in self.job.stations for f, _ in st.bands + st.zoom_bands if f == freq)
        out = np.zeros(T * nchan * max(rows, 1) * 2, dtype=np.float32)
        nt, nr = ctypes.c_int32(), ctypes.c_int32()
        check(lib().fxb_read_spectra(self.ctx, freq, _fptr(out), out.size, ctypes.byref(nt), ctypes.byref(nr)),
              self.ctx, "read_spectra")
        x = out[:nt.value * nr.value * nchan * 2].reshape(nt.value, nr.value, nchan, 2)
        return x[..., 0] + 1j * x[..., 1]

    def fft_weights(self) -> np.ndarray:
        T = self.job.blocks_per_send()
        out = np.zeros(len(self.job.stations) * T, dtype=np.float32)
        check(lib().fxb_read_fft_weights(self.ctx, _fptr(out), out.size), self.ctx, "read_fft_weights")
        return out.reshape(len(self.job.stations), T)


def vdif_unpack(data: np.ndarray, payload: int, header: int, nchan: int, nbits: int,
                offsetsamples: int, nsamp: int) -> Tuple[np.ndarray, int]:
    out = np.zeros((nchan, nsamp), dtype=np.float32)
    good = ctypes.c_int32(0)
    check(lib().fxb_vdif_unpack(data.ctypes.data, data.size, payload, header, nchan, nbits, offsetsamples,
                                nsamp, _fptr(out), ctypes.byref(good)), None, "vdif_unpack")
    return out, good.value


def job_layout(job: Job) -> Tuple[np.ndarray, int]:
    """Core-result offsets and length from the job alone (no GPU needed)."""
    holder = DescHolder(job)
    nf, nb, ns = len(job.freqs), len(job.baselines), len(job.stations)
    out = np.zeros(2 * nf * nb + 3 * ns, dtype=np.int32)
    n = ctypes.c_int64(0)
    check(lib().fxb_job_layout(holder.ptr(), out.ctypes.data_as(ctypes.POINTER(ctypes.c_int32)), out.size,
                               ctypes.byref(n)), None, "job_layout")
    return out, n.value


class Batch:
    """An fxb_batch: member Correlators whose subints are submitted together
    and run as one CUDA graph launch per subint."""

    def __init__(self, members: Sequence[Correlator]):
        self.members = list(members)
        arr = (ctypes.c_void_p * len(self.members))(*[m.ctx for m in self.members])
        st = ctypes.c_int32(0)
        self.b = lib().fxb_batch_create(arr, len(self.members), ctypes.byref(st))
        if not self.b:
            raise FxbError("fxb_batch_create: %s" % FXB_STATUS.get(st.value, st.value))

    def _check(self, rc, what):
        if rc != 0:
            m = lib().fxb_batch_last_error(self.b)
            raise FxbError("%s failed: %s %s" % (what, FXB_STATUS.get(rc, rc), m.decode() if m else ""))

    def _records(self, member_ptrs):
        keep, recs = [], (FxbMemberSubint * len(self.members))()
        for i, (ptrs, nbytes, dsec, dns) in enumerate(member_ptrs):
            n = len(ptrs)
            bufs = (ctypes.c_void_p * n)(*ptrs)
            nb = (ctypes.c_int64 * n)(*nbytes)
            ds = (ctypes.c_int32 * n)(*dsec)
            dn = (ctypes.c_int32 * n)(*dns)
            keep += [bufs, nb, ds, dn]
            recs[i].bufs, recs[i].nbytes, recs[i].datasec, recs[i].datans = bufs, nb, ds, dn
            recs[i].validflags = None
        return keep, recs

    def submit(self, member_inputs: Sequence[List[Tuple[np.ndarray, int, int]]], sec: int, ns: int) -> None:
        """member_inputs[i]: member i's [(buffer, datasec, datans)] per station."""
        keep, recs = self._records([([b.ctypes.data for b, _, _ in inp], [b.size for b, _, _ in inp],
                                     [x for _, x, _ in inp], [x for _, _, x in inp]) for inp in member_inputs])
        self._check(lib().fxb_batch_submit(self.b, recs, sec, ns), "batch_submit")

    def submit_device(self, member_ptrs, sec: int, ns: int) -> None:
        """member_ptrs[i]: (device pointers, nbytes, datasec, datans) of member i's stations."""
        keep, recs = self._records(member_ptrs)
        self._check(lib().fxb_batch_submit_device(self.b, recs, sec, ns), "batch_submit_device")

    def sync(self):
        self._check(lib().fxb_batch_sync(self.b), "batch_sync")

    def set_graphs(self, on: bool = True):
        self._check(lib().fxb_batch_set_graphs(self.b, 1 if on else 0), "batch_set_graphs")

    def set_fused(self, on: bool = True) -> bool:
        """Fused launches (one persistent F launch and one XMAC launch for
        all members) where the members allow them; returns whether the next
        subints run fused."""
        f = ctypes.c_int32(0)
        self._check(lib().fxb_batch_set_fused(self.b, 1 if on else 0, ctypes.byref(f)), "batch_set_fused")
        return bool(f.value)

    def autotune(self, rounds: int = 2):
        self._check(lib().fxb_batch_autotune(self.b, rounds), "batch_autotune")

    def stream(self) -> int:
        v = ctypes.c_void_p(0)
        self._check(lib().fxb_batch_get_stream(self.b, ctypes.byref(v)), "batch_get_stream")
        return v.value or 0

    def close(self):
        if getattr(self, "b", None):
            lib().fxb_batch_destroy(self.b)
            self.b = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass


def vdif_mux_device(dev_in: int, inbytes: int, thread_ids: Sequence[int], framebytes: int, fps: int, nbits: int,
                    dev_out: int, outcap: int, stream: int = 0) -> int:
    """fxb_vdif_mux on device pointers (one read of multi-thread VDIF to
    single-thread frames); returns the output bytes."""
    n = len(thread_ids)
    ids = (ctypes.c_int32 * n)(*thread_ids)
    out = ctypes.c_int64(0)
    rc = lib().fxb_vdif_mux(dev_in, inbytes, n, ids, framebytes, fps, nbits, dev_out, outcap, ctypes.byref(out),
                            stream or None)
    check(rc, None, "vdif_mux")
    return out.value
