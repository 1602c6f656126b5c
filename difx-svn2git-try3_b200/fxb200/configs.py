"""The workload configurations the path is measured and tested on.

c0: 4 stations, one 16 MHz band, dual polarisation (parallel hands), 2-bit
    VDIF (8000-byte payload, 2 channels), 256 channels (nFFT 512), 8 ms subints.
c1: 10 stations, eight 32 MHz bands, dual polarisation with full cross hands,
    2-bit VDIF (16 channels per frame), 1024 channels (nFFT 2048), 8 ms subints.
c2: c1 with the XMAC operand in BF16 / FP8 e4m3 (precision variant).
"""
from __future__ import annotations

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


CONFIGS = {"c0": c0, "c1": c1}
