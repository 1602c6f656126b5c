"""Integration output: amplitude calibration of an integrated core result,
SWIN ``.difx`` records and phase-cal files (fxb_vis_calibrate /
fxb_vis_write_swin / fxb_vis_write_pcal of include/fxb200.h, the reference's
Visibility::writedata and writedifx, mpifxcorr/src/visibility.cpp:104-135,
348-990), plus a reader for the records.

An integration on the device is: ``Correlator.reset()``, submit its subints,
``Correlator.results()`` -- the sum the reference's Visibility::addData
forms -- then :func:`calibrate` and :func:`write_swin` on that buffer.
"""
from __future__ import annotations

import ctypes
import dataclasses
import struct
from typing import List, Optional, Sequence

import numpy as np

from .job import Job
from .native import DescHolder, FxbError, FxbJobDesc, FXB_STATUS, lib

_c = ctypes

SYNC_WORD = 0xFF00FF00
# sync, version, baseline, MJD, seconds, config, source, freq, pol pair,
# pulsar bin, weight, u, v, w (Visibility::writeDiFXHeader): 74 bytes
HEADER = struct.Struct("<Iiiidiiiccidddd")


class FxbVisParams(_c.Structure):
    _fields_ = [("int_time_s", _c.c_double), ("start_mjd", _c.c_int32), ("start_sec", _c.c_int32),
                ("scan_start_sec", _c.c_int32), ("int_start_sec", _c.c_int32), ("int_start_ns", _c.c_int32),
                ("config_index", _c.c_int32), ("source_index", _c.c_int32),
                ("tsys", _c.POINTER(_c.c_double)), ("telescope", _c.POINTER(_c.c_int32)),
                ("uvw", _c.POINTER(_c.c_double)), ("names", _c.POINTER(_c.c_char_p))]


@dataclasses.dataclass
class VisParams:
    int_time_s: float
    start_mjd: int = 0
    start_sec: int = 0
    scan_start_sec: int = 0
    int_start_sec: int = 0
    int_start_ns: int = 0
    config_index: int = 0
    source_index: int = 0
    tsys: Optional[Sequence[float]] = None
    telescope: Optional[Sequence[int]] = None
    uvw: Optional[np.ndarray] = None        # [nbaseline, 3]
    names: Optional[Sequence[str]] = None   # station names (PCAL files)

    @staticmethod
    def for_job(job: Job, **kw) -> "VisParams":
        """The job's own start, integration time and station names."""
        kw.setdefault("names", [st.name for st in job.stations])
        return VisParams(int_time_s=job.duration_s, start_mjd=job.start_mjd, start_sec=job.start_sec, **kw)

    def native(self):
        keep = []
        p = FxbVisParams(self.int_time_s, self.start_mjd, self.start_sec, self.scan_start_sec, self.int_start_sec,
                         self.int_start_ns, self.config_index, self.source_index, None, None, None, None)
        if self.names is not None:
            a = (_c.c_char_p * len(self.names))(*[n.encode() for n in self.names])
            keep.append(a)
            p.names = _c.cast(a, _c.POINTER(_c.c_char_p))
        if self.tsys is not None:
            a = np.ascontiguousarray(self.tsys, dtype=np.float64)
            keep.append(a)
            p.tsys = a.ctypes.data_as(_c.POINTER(_c.c_double))
        if self.telescope is not None:
            a = np.ascontiguousarray(self.telescope, dtype=np.int32)
            keep.append(a)
            p.telescope = a.ctypes.data_as(_c.POINTER(_c.c_int32))
        if self.uvw is not None:
            a = np.ascontiguousarray(self.uvw, dtype=np.float64).reshape(-1)
            keep.append(a)
            p.uvw = a.ctypes.data_as(_c.POINTER(_c.c_double))
        return p, keep


def _bind():
    L = lib()
    if not getattr(L, "_vis_bound", False):
        L.fxb_vis_calibrate.argtypes = [_c.POINTER(FxbJobDesc), _c.POINTER(FxbVisParams), _c.POINTER(_c.c_float)]
        L.fxb_vis_calibrate.restype = _c.c_int
        L.fxb_vis_write_swin.argtypes = [_c.POINTER(FxbJobDesc), _c.POINTER(FxbVisParams), _c.POINTER(_c.c_float),
                                         _c.c_char_p]
        L.fxb_vis_write_swin.restype = _c.c_int
        L.fxb_vis_write_pcal.argtypes = [_c.POINTER(FxbJobDesc), _c.POINTER(FxbVisParams), _c.POINTER(_c.c_float),
                                         _c.c_char_p]
        L.fxb_vis_write_pcal.restype = _c.c_int
        L._vis_bound = True
    return L


def _check(rc, what):
    if rc != 0:
        m = lib().fxb_last_error(None)
        raise FxbError("%s failed: %s %s" % (what, FXB_STATUS.get(rc, rc), m.decode() if m else ""))


def calibrate(job: Job, params: VisParams, coreresult: np.ndarray) -> np.ndarray:
    """A calibrated copy of an integrated core result (float32 pairs)."""
    out = np.array(coreresult, dtype=np.float32, copy=True)
    d = DescHolder(job)
    p, keep = params.native()
    _check(_bind().fxb_vis_calibrate(d.ptr(), _c.byref(p), out.ctypes.data_as(_c.POINTER(_c.c_float))),
           "vis_calibrate")
    return out


def write_swin(job: Job, params: VisParams, calibrated: np.ndarray, outdir: str) -> None:
    """Append the calibrated integration's SWIN records to outdir/DIFX_<mjd>_<sec>.s0000.b0000."""
    a = np.ascontiguousarray(calibrated, dtype=np.float32)
    d = DescHolder(job)
    p, keep = params.native()
    _check(_bind().fxb_vis_write_swin(d.ptr(), _c.byref(p), a.ctypes.data_as(_c.POINTER(_c.c_float)),
                                      outdir.encode()), "vis_write_swin")


def write_pcal(job: Job, params: VisParams, calibrated: np.ndarray, outdir: str) -> None:
    """Append the calibrated integration's phase-cal tones to
    outdir/PCAL_<mjd>_<sec>_<station> of every station extracting them."""
    a = np.ascontiguousarray(calibrated, dtype=np.float32)
    d = DescHolder(job)
    p, keep = params.native()
    _check(_bind().fxb_vis_write_pcal(d.ptr(), _c.byref(p), a.ctypes.data_as(_c.POINTER(_c.c_float)),
                                      outdir.encode()), "vis_write_pcal")


@dataclasses.dataclass
class SwinRecord:
    baseline: int
    mjd: int
    seconds: float
    config_index: int
    source_index: int
    freq_index: int
    polpair: str
    pulsar_bin: int
    weight: float
    uvw: tuple
    vis: np.ndarray          # complex64 [nchan]


def read_swin(data: bytes, nchan_of_freq) -> List[SwinRecord]:
    """Parse SWIN records; nchan_of_freq(freq_index) gives each record's
    channel count (output channels after averaging)."""
    out, off = [], 0
    while off < len(data):
        (sync, ver, bl, mjd, sec, cfg, src, fq, p0, p1, pbin, w, u, v, ww) = HEADER.unpack_from(data, off)
        if sync != SYNC_WORD or ver != 1:
            raise ValueError("bad SWIN sync word or version at byte %d" % off)
        off += HEADER.size
        n = nchan_of_freq(fq)
        vis = np.frombuffer(data, dtype=np.complex64, count=n, offset=off).copy()
        off += 8 * n
        out.append(SwinRecord(bl, mjd, sec, cfg, src, fq, (p0 + p1).decode(), pbin, w, (u, v, ww), vis))
    return out
