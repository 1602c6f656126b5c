"""ctypes wrapper of the FP64 C restatement (oracle/fxoracle.c).

Oracle test infrastructure: the checker for the product's CUDA path.  The
shared library is compiled on first use (gcc is on every machine this runs on)
into oracle/_build/.
"""
from __future__ import annotations

import ctypes
import os
import subprocess
from typing import List, Optional, Tuple

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
SRC = os.path.join(HERE, "fxoracle.c")
LIB = os.path.join(HERE, "_build", "libfxoracle.so")

_lib = None


HDR = os.path.join(os.path.dirname(HERE), "include", "fxb200.h")


def build(force: bool = False) -> str:
    # the restatement reads the job description through the C ABI's structs:
    # rebuilt when either the source or the header is newer
    newest = max(os.path.getmtime(SRC), os.path.getmtime(HDR) if os.path.exists(HDR) else 0.0)
    if force or not os.path.exists(LIB) or os.path.getmtime(LIB) < newest:
        os.makedirs(os.path.dirname(LIB), exist_ok=True)
        # built under a private name and renamed into place, so that a
        # concurrent test process never loads a half-written library
        tmp = "%s.%d.tmp" % (LIB, os.getpid())
        subprocess.check_call(["gcc", "-O2", "-ffp-contract=off", "-fPIC", "-shared", "-o", tmp, SRC, "-lm"])
        os.replace(tmp, LIB)
    return LIB


def lib():
    global _lib
    if _lib is None:
        L = ctypes.CDLL(build())
        vp = ctypes.c_void_p
        L.fxo_create.restype = vp
        L.fxo_create.argtypes = [vp]
        L.fxo_destroy.argtypes = [vp]
        L.fxo_core_result_length.restype = ctypes.c_int64
        L.fxo_core_result_length.argtypes = [vp]
        L.fxo_blocks_per_send.argtypes = [vp]
        L.fxo_layout.argtypes = [vp, ctypes.POINTER(ctypes.c_int32)]
        L.fxo_set_delay_poly.argtypes = [vp, ctypes.c_int, ctypes.c_int, ctypes.c_int, ctypes.c_double, ctypes.c_int,
                                         ctypes.POINTER(ctypes.c_double)]
        L.fxo_interpolator.argtypes = [vp, ctypes.c_int, ctypes.c_int, ctypes.c_int, ctypes.POINTER(ctypes.c_double)]
        L.fxo_process_subint.argtypes = [vp, ctypes.POINTER(ctypes.c_void_p), ctypes.POINTER(ctypes.c_int64),
                                         ctypes.POINTER(ctypes.c_int32), ctypes.POINTER(ctypes.c_int32),
                                         ctypes.POINTER(ctypes.c_void_p), ctypes.c_int, ctypes.c_int,
                                         ctypes.POINTER(ctypes.c_double), ctypes.POINTER(ctypes.c_float)]
        L.fxo_mode_fft.argtypes = [vp, ctypes.c_int, ctypes.c_void_p, ctypes.c_int64, ctypes.c_int, ctypes.c_int,
                                   ctypes.c_void_p, ctypes.c_int, ctypes.c_int, ctypes.c_int,
                                   ctypes.POINTER(ctypes.c_double), ctypes.POINTER(ctypes.c_float),
                                   ctypes.POINTER(ctypes.c_int)]
        L.fxo_vdif_unpack.argtypes = [ctypes.c_void_p, ctypes.c_int64, ctypes.c_int, ctypes.c_int, ctypes.c_int,
                                      ctypes.c_int, ctypes.c_int64, ctypes.c_int, ctypes.POINTER(ctypes.c_float)]
        _lib = L
    return _lib


class OracleCorrelator:
    def __init__(self, job):
        from fxb200.native import DescHolder, poly_arrays
        self.job = job
        self.holder = DescHolder(job)
        self.h = lib().fxo_create(ctypes.addressof(self.holder.desc))
        self.corelen = lib().fxo_core_result_length(self.h)
        self.blockspersend = lib().fxo_blocks_per_send(self.h)
        for s in range(len(job.stations)):
            npoly, order, p0, interval, coeffs = poly_arrays(job, s)
            lib().fxo_set_delay_poly(self.h, s, npoly, order, p0, interval,
                                     coeffs.ctypes.data_as(ctypes.POINTER(ctypes.c_double)))

    def close(self):
        if self.h:
            lib().fxo_destroy(self.h)
            self.h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    def layout(self) -> np.ndarray:
        nf, nb, ns = len(self.job.freqs), len(self.job.baselines), len(self.job.stations)
        out = np.zeros(2 * nf * nb + 3 * ns, dtype=np.int32)
        lib().fxo_layout(self.h, out.ctypes.data_as(ctypes.POINTER(ctypes.c_int32)))
        return out

    def interpolator(self, s: int, sec: int, ns: int) -> np.ndarray:
        c = (ctypes.c_double * 3)()
        if lib().fxo_interpolator(self.h, s, sec, ns, c) != 0:
            raise RuntimeError("no delay model for that time")
        return np.array(list(c))

    def process_subint(self, inputs: List[Tuple[np.ndarray, int, int]], sec: int, ns: int,
                       validflags: Optional[List[np.ndarray]] = None, coreresult: Optional[np.ndarray] = None):
        if coreresult is None:
            coreresult = np.zeros(2 * self.corelen, dtype=np.float64)
        n = len(inputs)
        bufs = (ctypes.c_void_p * n)(*[b.ctypes.data for b, _, _ in inputs])
        nb = (ctypes.c_int64 * n)(*[b.size for b, _, _ in inputs])
        ds = (ctypes.c_int32 * n)(*[s for _, s, _ in inputs])
        dn = (ctypes.c_int32 * n)(*[x for _, _, x in inputs])
        vf = None if validflags is None else (ctypes.c_void_p * n)(*[v.ctypes.data for v in validflags])
        w = np.zeros(n * self.blockspersend, dtype=np.float32)
        lib().fxo_process_subint(self.h, bufs, nb, ds, dn, vf, sec, ns,
                                 coreresult.ctypes.data_as(ctypes.POINTER(ctypes.c_double)),
                                 w.ctypes.data_as(ctypes.POINTER(ctypes.c_float)))
        self.last_weights = w.reshape(n, self.blockspersend)
        return coreresult

    def mode_fft(self, s: int, buf: np.ndarray, dsec: int, dns: int, sec: int, ns: int, fftindex: int,
                 validflags: Optional[np.ndarray] = None):
        st = self.job.stations[s]
        nchan = self.job.station_nchan(s)
        spec = np.zeros((st.nband, nchan, 2))
        w = ctypes.c_float(0)
        nearest = ctypes.c_int(0)
        lib().fxo_mode_fft(self.h, s, buf.ctypes.data, buf.size, dsec, dns,
                           None if validflags is None else validflags.ctypes.data, sec, ns, fftindex,
                           spec.ctypes.data_as(ctypes.POINTER(ctypes.c_double)), ctypes.byref(w), ctypes.byref(nearest))
        return spec[..., 0] + 1j * spec[..., 1], w.value, nearest.value


def vdif_unpack(data: np.ndarray, payload: int, header: int, nchan: int, nbits: int, offsetsamples: int, nsamp: int):
    out = np.zeros((nchan, nsamp), dtype=np.float32)
    good = lib().fxo_vdif_unpack(data.ctypes.data, data.size, payload, header, nchan, nbits, offsetsamples, nsamp,
                                 out.ctypes.data_as(ctypes.POINTER(ctypes.c_float)))
    return out, good
