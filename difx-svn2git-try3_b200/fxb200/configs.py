"""The workload configurations the path is measured and tested on.

c0: 4 stations, one 16 MHz band, dual polarisation (parallel hands), 2-bit
    VDIF (8000-byte payload, 2 channels), 256 channels (nFFT 512), 8 ms subints.
c1: 10 stations, eight 32 MHz bands, dual polarisation with full cross hands,
    2-bit VDIF (16 channels per frame), 1024 channels (nFFT 2048), 8 ms subints.
c2: c1 with the XMAC operand in BF16 / FP8 e4m3 (precision variant).
c3: 20 stations, 16 subbands of seeded width (4, 16, 64 MHz), channel count
    (128, 1024, 4096) and sample size (2, 8 bits), dual polarisation with
    full cross hands, 8.192 ms subints (a whole number of FFTs at every
    width and channel count), as a batch of jobs: one per run of subbands
    sharing (width, channels, bits), since one VDIF stream carries one
    sample rate and sample size.
"""
from __future__ import annotations

from typing import List, Tuple

import numpy as np

from . import synth
from .job import Freq, Job, full_job


def c0(seed: int = 1, subint_ns: int = 8_000_000) -> Job:
    job = full_job(4, [Freq(8400.0, 16.0, 256)], full_pol=False, subint_ns=subint_ns)
    synth.make_delay_polys(job, seed=seed)
    job.validate()
    return job


def c1(seed: int = 1, nstation: int = 10, subint_ns: int = 8_000_000) -> Job:
    freqs = [Freq(8400.0 + 32.0 * k, 32.0, 1024) for k in range(8)]
    job = full_job(nstation, freqs, full_pol=True, subint_ns=subint_ns)
    synth.make_delay_polys(job, seed=seed)
    job.validate()
    return job


C3_WIDTHS = (4.0, 16.0, 64.0)
C3_NCHANS = (128, 1024, 4096)
C3_BITS = (2, 8)


def c3_subbands(seed: int = 3, nsub: int = 16) -> List[Tuple[float, int, int]]:
    """Seeded (width MHz, channels, bits) of each of the nsub subbands."""
    rng = np.random.default_rng(seed)
    return [(float(rng.choice(C3_WIDTHS)), int(rng.choice(C3_NCHANS)), int(rng.choice(C3_BITS))) for _ in range(nsub)]


def c3(seed: int = 3, nstation: int = 20, nsub: int = 16, subint_ns: int = 8_192_000,
       full_pol: bool = True) -> List[Job]:
    """The c3 batch: one job per group of subbands with equal (width,
    channels, bits), split so that each job's VDIF stream has a power-of-two
    channel count within the decoder's limit (64 channels at 2 bits, 4 at 8
    bits).  Sky frequencies run on from 8400 MHz in subband order."""
    subs = c3_subbands(seed, nsub)
    edges, f = [], 8400.0
    for bw, _, _ in subs:
        edges.append(f)
        f += bw
    groups = {}
    for k, key in enumerate(subs):
        groups.setdefault(key, []).append(k)
    jobs = []
    for gi, (key, members) in enumerate(sorted(groups.items())):
        bw, nchan, bits = key
        cap = 32 if bits == 2 else 2           # subbands per stream (two pols each)
        rest = list(members)
        while rest:
            take = 1
            while take * 2 <= min(len(rest), cap):
                take *= 2
            chunk, rest = rest[:take], rest[take:]
            freqs = [Freq(edges[k], bw, nchan) for k in chunk]
            job = full_job(nstation, freqs, full_pol=full_pol, subint_ns=subint_ns, nbits=bits)
            synth.make_delay_polys(job, seed=seed * 100 + len(jobs))
            job.validate()
            jobs.append(job)
    return jobs


CONFIGS = {"c0": c0, "c1": c1}
