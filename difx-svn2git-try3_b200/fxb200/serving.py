"""Serving: the fxb_server_* request loop (include/fxb200.h) from Python, and
the seeded job stream of the serving workload.

A server owns one worker thread on one GPU.  Jobs (a job description, the
stations' delay models and the host VDIF of every subint) are queued with
:meth:`Server.submit`, admitted in arrival order against the HBM budget,
and run concurrently, each on its own stream; :meth:`Server.wait` returns the
core result.  Every array a request points into is kept alive by its
:class:`ServedJob` until the job has completed.
"""
from __future__ import annotations

import ctypes
import time
from typing import List, Sequence, Tuple

import numpy as np

from . import synth
from .job import Freq, Job, full_job
from .native import DescHolder, FxbError, FxbJobDesc, FXB_STATUS, lib, pinned_empty, poly_arrays

_c = ctypes


class FxbJobRequest(_c.Structure):
    _fields_ = [("desc", _c.POINTER(FxbJobDesc)), ("poly_npoly", _c.POINTER(_c.c_int32)),
                ("poly_order", _c.POINTER(_c.c_int32)), ("poly0_sec", _c.POINTER(_c.c_double)),
                ("poly_interval", _c.POINTER(_c.c_int32)), ("poly_coeffs", _c.POINTER(_c.POINTER(_c.c_double))),
                ("nsubint", _c.c_int32), ("bufs", _c.POINTER(_c.c_void_p)), ("nbytes", _c.POINTER(_c.c_int64)),
                ("datasec", _c.POINTER(_c.c_int32)), ("datans", _c.POINTER(_c.c_int32)),
                ("subsec", _c.POINTER(_c.c_int32)), ("subns", _c.POINTER(_c.c_int32)),
                ("coreresult", _c.POINTER(_c.c_float))]


_bound = False


def _bind():
    global _bound
    L = lib()
    if _bound:
        return L
    vp, i32, szt, dp = _c.c_void_p, _c.c_int32, _c.c_size_t, _c.POINTER(_c.c_double)
    L.fxb_job_footprint.argtypes = [_c.POINTER(FxbJobDesc), _c.POINTER(szt)]
    L.fxb_server_create.restype = vp
    L.fxb_server_create.argtypes = [i32, szt, i32, _c.POINTER(i32)]
    L.fxb_server_submit.argtypes = [vp, _c.POINTER(FxbJobRequest), _c.POINTER(_c.c_uint64)]
    L.fxb_server_poll.argtypes = [vp, _c.c_uint64, _c.POINTER(i32), dp]
    L.fxb_server_wait.argtypes = [vp, _c.c_uint64, _c.c_double]
    L.fxb_server_stats.argtypes = [vp, _c.POINTER(i32), dp, dp, dp, dp]
    L.fxb_server_job_times.argtypes = [vp, _c.c_uint64, dp]
    L.fxb_server_last_error.restype = _c.c_char_p
    L.fxb_server_last_error.argtypes = [vp]
    L.fxb_server_destroy.argtypes = [vp]
    for name in ("fxb_job_footprint", "fxb_server_submit", "fxb_server_poll", "fxb_server_wait", "fxb_server_stats",
                 "fxb_server_job_times"):
        getattr(L, name).restype = _c.c_int
    _bound = True
    return L


def job_footprint(job: Job, xmac: str = "fp16", inflight: int = 2) -> int:
    d = DescHolder(job, xmac, inflight)
    out = _c.c_size_t(0)
    rc = _bind().fxb_job_footprint(_c.byref(d.desc), _c.byref(out))
    if rc != 0:
        raise FxbError("fxb_job_footprint failed: %s" % FXB_STATUS.get(rc, rc))
    return out.value


class ServedJob:
    """A queued job: owns every array its request borrows, and its result."""

    def __init__(self, job: Job, subints: Sequence[Tuple[list, int, int]], xmac: str, inflight: int):
        self.job = job
        S = len(job.stations)
        self.holder = DescHolder(job, xmac, inflight)
        ncomplex = _c.c_int64(0)
        rc = lib().fxb_job_layout(_c.byref(self.holder.desc), None, 0, _c.byref(ncomplex))
        if rc != 0:
            raise FxbError("fxb_job_layout failed: %s" % FXB_STATUS.get(rc, rc))
        self.corelen = ncomplex.value
        self.result = np.zeros(2 * self.corelen, dtype=np.float32)
        polys = [poly_arrays(job, s) for s in range(S)]
        self.npoly = np.array([p[0] for p in polys], dtype=np.int32)
        self.order = np.array([p[1] for p in polys], dtype=np.int32)
        self.p0 = np.array([p[2] for p in polys], dtype=np.float64)
        self.interval = np.array([p[3] for p in polys], dtype=np.int32)
        self.coeffs = [np.ascontiguousarray(p[4], dtype=np.float64) for p in polys]
        self.coeff_ptrs = (_c.POINTER(_c.c_double) * S)(*[c.ctypes.data_as(_c.POINTER(_c.c_double))
                                                           for c in self.coeffs])
        n = len(subints)
        self.bufs = [np.ascontiguousarray(b) for inputs, _, _ in subints for b, _, _ in inputs]
        self.buf_ptrs = (_c.c_void_p * (n * S))(*[b.ctypes.data for b in self.bufs])
        self.nbytes = np.array([b.size for b in self.bufs], dtype=np.int64)
        self.datasec = np.array([x for inputs, _, _ in subints for _, x, _ in inputs], dtype=np.int32)
        self.datans = np.array([x for inputs, _, _ in subints for _, _, x in inputs], dtype=np.int32)
        self.subsec = np.array([sec for _, sec, _ in subints], dtype=np.int32)
        self.subns = np.array([ns for _, _, ns in subints], dtype=np.int32)
        i32p, i64p = _c.POINTER(_c.c_int32), _c.POINTER(_c.c_int64)
        self.req = FxbJobRequest(
            _c.pointer(self.holder.desc), self.npoly.ctypes.data_as(i32p), self.order.ctypes.data_as(i32p),
            self.p0.ctypes.data_as(_c.POINTER(_c.c_double)), self.interval.ctypes.data_as(i32p), self.coeff_ptrs,
            n, self.buf_ptrs, self.nbytes.ctypes.data_as(i64p), self.datasec.ctypes.data_as(i32p),
            self.datans.ctypes.data_as(i32p), self.subsec.ctypes.data_as(i32p), self.subns.ctypes.data_as(i32p),
            self.result.ctypes.data_as(_c.POINTER(_c.c_float)))
        self.id = None
        self.data_seconds = n * job.subint_ns * 1e-9


class Server:
    """One fxb_server: a worker thread on `device` with an HBM budget."""

    def __init__(self, budget_bytes: int, max_active: int = 4, device: int = 0):
        L = _bind()
        st = _c.c_int32(0)
        self.srv = L.fxb_server_create(device, budget_bytes, max_active, _c.byref(st))
        if not self.srv:
            raise FxbError("fxb_server_create failed: %s" % FXB_STATUS.get(st.value, st.value))
        self.jobs: List[ServedJob] = []

    def _check(self, rc, what):
        if rc != 0:
            msg = _bind().fxb_server_last_error(self.srv)
            raise FxbError("%s failed: %s %s" % (what, FXB_STATUS.get(rc, rc), msg.decode() if msg else ""))

    def submit(self, job: Job, subints: Sequence[Tuple[list, int, int]], xmac: str = "fp16",
               inflight: int = 2) -> ServedJob:
        sj = ServedJob(job, subints, xmac, inflight)
        jid = _c.c_uint64(0)
        self._check(_bind().fxb_server_submit(self.srv, _c.byref(sj.req), _c.byref(jid)), "server_submit")
        sj.id = jid.value
        self.jobs.append(sj)
        return sj

    def poll(self, sj: ServedJob):
        state, lat = _c.c_int32(0), _c.c_double(0.0)
        self._check(_bind().fxb_server_poll(self.srv, sj.id, _c.byref(state), _c.byref(lat)), "server_poll")
        return state.value, lat.value

    def wait(self, sj: ServedJob, timeout_s: float = 120.0) -> np.ndarray:
        self._check(_bind().fxb_server_wait(self.srv, sj.id, timeout_s), "server_wait")
        return sj.result

    def job_times(self, sj: ServedJob) -> dict:
        """Phases of a done job's latency (ms)."""
        out = (_c.c_double * 5)()
        self._check(_bind().fxb_server_job_times(self.srv, sj.id, out), "server_job_times")
        return dict(zip(("queued", "create", "submit", "drain", "release"), list(out)))

    def stats(self) -> dict:
        n = _c.c_int32(0)
        p50, p99, ds, ws = _c.c_double(0), _c.c_double(0), _c.c_double(0), _c.c_double(0)
        self._check(_bind().fxb_server_stats(self.srv, _c.byref(n), _c.byref(p50), _c.byref(p99), _c.byref(ds),
                                             _c.byref(ws)), "server_stats")
        return {"completed": n.value, "p50_ms": p50.value, "p99_ms": p99.value, "data_seconds": ds.value,
                "wall_seconds": ws.value, "rtf": ds.value / ws.value if ws.value > 0 else 0.0}

    def close(self):
        if getattr(self, "srv", None):
            _bind().fxb_server_destroy(self.srv)
            self.srv = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass


# ---------------------------------------------------------------- workload
def _subint_ns_near(nchan: int, bw_mhz: float, target_ns: int = 8_000_000) -> int:
    fft_ns = int(round(nchan * 1000.0 / bw_mhz))     # 2 nchan samples at 2 bw Ms/s
    return max(1, int(round(target_ns / fft_ns))) * fft_ns


def serving_job(rng: np.random.Generator, seed: int, stations=(4, 32), subbands=(1, 16),
                bws=(8.0, 16.0, 32.0, 64.0), nchans=(256, 512, 1024, 2048, 4096, 8192),
                seconds=(0.1, 2.0)) -> Tuple[Job, int]:
    """One job of the serving stream: station count, subbands, bandwidth,
    channels and duration drawn from the given ranges (one bandwidth and
    channel count per job), dual polarisation with cross hands; returns the
    job and its number of subints."""
    nst = int(rng.integers(stations[0], stations[1] + 1))
    nsb = int(rng.integers(subbands[0], subbands[1] + 1))
    bw = float(rng.choice(bws))
    nchan = int(rng.choice(nchans))
    # the VDIF channel count of a station must be a power of two
    while (2 * nsb) & (2 * nsb - 1):
        nsb += 1
    freqs = [Freq(8400.0 + bw * k, bw, nchan) for k in range(nsb)]
    job = full_job(nst, freqs, full_pol=True, subint_ns=_subint_ns_near(nchan, bw))
    synth.make_delay_polys(job, seed=seed)
    job.validate()
    dur = float(rng.uniform(seconds[0], seconds[1]))
    nsub = max(1, int(round(dur * 1e9 / job.subint_ns)))
    return job, nsub


def job_subints(job: Job, nsub: int, seed: int, rho: float = 0.0, pinned: bool = False,
                pool: int = 0) -> List[Tuple[list, int, int]]:
    """Host VDIF of nsub consecutive subints (starting one subint in): the bulk
    code-statistics generator for rho = 0, the correlated sky + noise model
    otherwise.  pinned=True places every buffer in one page-locked block, as
    a datastream's receive ring would be.

    pool > 0 generates only `pool` distinct subints of bytes (each as long as
    the longest window of the job) and lets subint k reuse those of subint
    k % pool, with its own data time and window length: a job of 2 s of a
    32-station, 16 x 64 MHz array (66 GB of VDIF) then holds a few subints of
    host memory, as a receive ring of a few segments does.  Every subint
    still has its own time, delay interpolator and FFT windows; only the
    sample values repeat."""
    times = []
    for k in range(nsub):
        t = (k + 1) * job.subint_ns
        times.append((t // 1_000_000_000, t % 1_000_000_000))
    S = len(job.stations)
    windows = [[synth.subint_window(job, s, sec, ns) for s in range(S)] for sec, ns in times]
    ndistinct = nsub if pool <= 0 else min(pool, nsub)
    longest = [max(w[s][1] for w in windows) for s in range(S)]
    distinct = []
    for k in range(ndistinct):
        sec, ns = times[k]
        if rho == 0.0:
            bufs = []
            for s in range(S):
                f0, nf, _, _ = windows[k][s]
                bufs.append(synth.bulk_station_frames(job, s, f0, longest[s] if pool > 0 else nf, seed))
        else:
            bufs = [synth.gen_station_frames(job, s, windows[k][s][0], longest[s] if pool > 0 else windows[k][s][1],
                                             rho, seed) for s in range(S)]
        distinct.append(bufs)
    if pinned:
        total = sum(b.nbytes for bufs in distinct for b in bufs)
        block = pinned_empty(total)
        off = 0
        for bufs in distinct:
            for s, b in enumerate(bufs):
                v = block[off:off + b.nbytes]
                v[:] = np.frombuffer(np.ascontiguousarray(b).data, dtype=np.uint8)
                bufs[s] = v
                off += b.nbytes
    out = []
    for k, (sec, ns) in enumerate(times):
        bufs = distinct[k % ndistinct]
        inputs = []
        for s in range(S):
            _, nf, dsec, dns = windows[k][s]
            inputs.append((bufs[s][:nf * job.frame_bytes(s)] if pool > 0 else bufs[s], dsec, dns))
        out.append((inputs, sec, ns))
    return out


def poisson_arrivals(rng: np.random.Generator, n: int, rate_hz: float) -> np.ndarray:
    return np.cumsum(rng.exponential(1.0 / rate_hz, size=n))


def run_stream(server: Server, jobs: Sequence[Tuple[Job, list]], arrivals: Sequence[float], xmac: str = "fp16",
               timeout_s: float = 600.0) -> dict:
    """Submit each job at its arrival time (seconds from now), wait for all,
    return the server's statistics."""
    t0 = time.perf_counter()
    handles = []
    for (job, subints), at in zip(jobs, arrivals):
        delay = at - (time.perf_counter() - t0)
        if delay > 0:
            time.sleep(delay)
        handles.append(server.submit(job, subints, xmac=xmac))
    for h in handles:
        server.wait(h, timeout_s)
    return server.stats()
