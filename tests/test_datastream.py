"""DataStream control blocks (fxb_job_datastream_control) against the stock
VDIFDataStream::calculateControlParams of the reference, compiled into
oracle/_ref, on seeded rings of read segments: whole and short reads, gaps in
the data, segments not yet read, the end of the data, requests before, inside
and after the ring.  Byte offset, data time, valid-FFT words, the segment the
ring advances to and the byte count are compared exactly.  Host arithmetic:
no GPU."""
import random

import numpy as np
import pytest

from fxb200.native import INVALID_SUBINT, FxbError, job_datastream_control
from helpers import small_job

import refcorr

JOBS = {
    "2bit_2ch_256": dict(nstation=2),
    "2bit_16ch_1024": dict(nstation=2, nchan=1024, bw=32.0, nfreq=8, full_pol=True, subint_ns=2_048_000),
    "8bit_1ch_256": dict(nstation=2, nbits=8),
}


def scenario(rng, ring, job, nseg):
    """A ring filled in time order from a random slot, and one request."""
    frame_ns = int(round(1e9 / job.frames_per_sec(0)))
    fb, rb = job.frame_bytes(0), ring.readbytes
    t0 = rng.randint(2, 40) * 10**9 + rng.randrange(0, 10**9, frame_ns)
    start = rng.randrange(nseg)
    nfilled = rng.choice([nseg, nseg, nseg - 1, nseg - 2, rng.randint(1, nseg)])
    segs = [None] * nseg
    t = t0
    for k in range(nseg):
        i = (start + k) % nseg
        if rng.random() < 0.1:
            t += rng.randint(1, 50) * frame_ns                 # a gap in the data
        valid = rb if rng.random() >= 0.1 else rng.randrange(0, rb // fb + 1) * fb   # a short read
        readto = int(k < nfilled)
        segs[i] = (0, t // 10**9, t % 10**9, readto, valid if readto else 0)
        t += ring.nsinc
    keep = rng.random() < 0.7
    lastvalid = (start + nfilled - 1) % nseg
    at = (start + rng.choice([0, 0, 1, 2])) % nseg
    # while the reader is active the reference waits for data past the newest
    # segment: ask only up to its start then
    last = segs[lastvalid][1] * 10**9 + segs[lastvalid][2]
    hi = (last - t0) if keep else (nseg + 1) * ring.nsinc
    tr = t0 + rng.randint(-ring.nsinc, max(hi, 0))
    tr -= tr % 1000
    return segs, at, keep, lastvalid, tr // 10**9, tr % 10**9


@pytest.mark.skipif(not refcorr.available(), reason="reference build oracle/_ref absent")
@pytest.mark.parametrize("name", sorted(JOBS))
@pytest.mark.parametrize("nseg,factor", [(8, 32), (4, 8)])
def test_control_blocks_match_reference(name, nseg, factor):
    job = small_job(**JOBS[name])
    ring = refcorr.RefCorrelator(job).datastream(0, factor, nseg)
    rng = random.Random(hash((name, nseg)) & 0xFFFF)
    nvalid = 0
    for _ in range(300):
        segs, at, keep, lastvalid, sec, ns = scenario(rng, ring, job, nseg)
        rbi, rat, ctl = ring.control(segs, at, keep, lastvalid, 0, sec, ns)
        off, nb, dsec, dns, flags, pat = job_datastream_control(job, 0, segs, ring.readbytes, at, keep, lastvalid, 0,
                                                                sec, ns, guard_ns=ring.guard_ns)
        assert dsec == ctl[1], (segs, at, keep, sec, ns)
        if dsec == INVALID_SUBINT:
            continue
        nvalid += 1
        assert (off, dns, pat, nb) == (rbi, ctl[2], rat, ring.sendbytes)
        assert list(flags[:len(ctl) - 3]) == ctl[3:]
    assert nvalid > 50


def test_ring_that_does_not_reach_the_subint_asks_to_read_more():
    job = small_job(nstation=2)
    fb = job.frame_bytes(0)
    readbytes = 40 * fb
    nsinc = int(40 * 1e9 / job.frames_per_sec(0) + 0.5)
    segs = [(0, 10, k * nsinc, 1, readbytes) for k in range(4)]
    with pytest.raises(FxbError, match="STATE"):
        job_datastream_control(job, 0, segs, readbytes, 0, True, 3, 0, 20, 0)
    # once the reader has stopped, the same request is simply not in the data
    off, nb, dsec, dns, flags, at = job_datastream_control(job, 0, segs, readbytes, 0, False, 3, 0, 20, 0)
    assert dsec == INVALID_SUBINT and nb == 0 and not flags.any()
