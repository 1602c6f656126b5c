"""Correlating a datastream's receive ring: each station's continuous VDIF
fills a ring of read segments; the control block of every subint
(fxb_datastream_control) gives the bytes to submit, their time and the
valid-FFT flags; the GPU result of those windows matches the FP64 oracle on
the same windows.  A gap in one station's data (frames never recorded) is
flagged there rather than correlated."""
import ctypes

import numpy as np
import pytest

from fxb200 import synth
from fxb200.native import INVALID_SUBINT, Correlator, FxbRing, FxbSegment, check, lib
from helpers import compare_core, small_job

import fxoracle

pytestmark = pytest.mark.gpu

NSEG, SEGFRAMES, FIRST = 4, 120, 2000        # 4 segments of 120 frames from frame 2000 (1 s of data in)


def _ring_data(job, s, gap=None):
    """Ring bytes of station s (segments in time order from slot 0) and its
    segment table; gap = (first frame, frames) left out of the data."""
    fb, fps = job.frame_bytes(s), job.frames_per_sec(s)
    frames = []
    segs = []
    f = FIRST
    for k in range(NSEG):
        if gap and k == 2:
            f += gap                               # the reader skips what was never recorded
        data = synth.gen_station_frames(job, s, f, SEGFRAMES, rho=0.05, seed=21)
        frames.append(data)
        t_ns = f * 10**9 // fps
        segs.append((0, t_ns // 10**9, t_ns % 10**9, 1, SEGFRAMES * fb))
        f += SEGFRAMES
    return np.concatenate(frames), segs


def _control(corr, s, segs, readbytes, sec, ns, nflag):
    arr = (FxbSegment * len(segs))(*[FxbSegment(*x) for x in segs])
    ring = FxbRing(len(segs), readbytes, 0, 0, len(segs) - 1, 0, ctypes.cast(arr, ctypes.POINTER(FxbSegment)))
    off, nb = ctypes.c_int64(), ctypes.c_int32()
    dsec, dns = ctypes.c_int32(), ctypes.c_int32()
    flags = np.zeros(nflag, dtype=np.int32)
    check(lib().fxb_datastream_control(corr.ctx, s, ctypes.byref(ring), 0, sec, ns, None, ctypes.byref(off),
                                       ctypes.byref(nb), ctypes.byref(dsec), ctypes.byref(dns),
                                       flags.ctypes.data_as(ctypes.POINTER(ctypes.c_int32)), nflag), corr.ctx,
          "datastream_control")
    return off.value, nb.value, dsec.value, dns.value, flags


@pytest.mark.parametrize("gap", [None, 30])
def test_ring_windows_correlate_like_the_oracle(gap):
    job = small_job(nstation=3, full_pol=True)
    fps = job.frames_per_sec(0)
    readbytes = SEGFRAMES * job.frame_bytes(0)
    rings = [_ring_data(job, s, gap if s == 1 else None) for s in range(len(job.stations))]
    corr = Correlator(job)
    orc = fxoracle.OracleCorrelator(job)
    T = job.blocks_per_send()
    ref = None
    nsub = 0
    flagged = 0
    t0 = (FIRST + 2 * SEGFRAMES - 20) * 10**9 // fps     # 10 ms before the gap, which the subints then cross
    for k in range(6):
        t = t0 + k * job.subint_ns
        sec, ns = t // 10**9, t % 10**9
        inputs, vflags = [], []
        for s, (data, segs) in enumerate(rings):
            off, nb, dsec, dns, flags = _control(corr, s, segs, readbytes, sec, ns, T // 30 + 1)
            if dsec == INVALID_SUBINT:
                inputs.append((np.zeros(0, dtype=np.uint8), 0, 0))
            else:
                assert off + nb <= data.size
                inputs.append((np.ascontiguousarray(data[off:off + nb]), dsec, dns))
            flagged += int(dsec == INVALID_SUBINT or not all(
                (flags[i // 30] >> (i % 30)) & 1 for i in range(T)))
            vflags.append(flags)
        corr.submit(inputs, sec, ns, validflags=vflags)
        ref = orc.process_subint(inputs, sec, ns, validflags=vflags, coreresult=ref)
        nsub += 1
    got, layout, n = corr.results(), corr.layout(), corr.corelen
    corr.close()
    compare_core(job, layout, n, got, ref)
    if gap:
        assert flagged > 0
    else:
        assert flagged == 0
