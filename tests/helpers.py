"""Shared job builders and comparison helpers for the parity tests."""
from __future__ import annotations

import numpy as np

from fxb200 import synth
from fxb200.job import Freq, Job, full_job

# FP32 form vs the FP64 oracle: relative visibility tolerance (north star)
FP32_TOL = 1e-5


def small_job(nstation=4, nchan=256, bw=16.0, nfreq=1, full_pol=False, nbits=2, subint_ns=4_000_000,
              order=1, lsb=False, freq0=8400.0, avg=1, seed=1) -> Job:
    freqs = [Freq(freq0 + k * bw, bw, nchan, "L" if lsb else "U", avg) for k in range(nfreq)]
    job = full_job(nstation, freqs, full_pol=full_pol, subint_ns=subint_ns, nbits=nbits, fringe_rot_order=order)
    synth.make_delay_polys(job, seed=seed)
    job.validate()
    return job


def regions(job: Job, layout: np.ndarray, corelen: int):
    """(name, float slice) of the core result: cross, bweights, autos, acweights."""
    nf, nb, ns = len(job.freqs), len(job.baselines), len(job.stations)
    bl = layout[:nf * nb]
    bw = layout[nf * nb:2 * nf * nb]
    ac = layout[2 * nf * nb:2 * nf * nb + ns]
    acw = layout[2 * nf * nb + ns:]
    bw_valid = bw[bw >= 0]
    xc_end = int(bw_valid.min()) if bw_valid.size else int(ac.min())
    return [("cross", slice(0, 2 * xc_end)), ("bweight", slice(2 * xc_end, 2 * int(ac.min()))),
            ("auto", slice(2 * int(ac.min()), 2 * int(acw.min()))), ("acweight", slice(2 * int(acw.min()), 2 * corelen))]


def rel_err(a: np.ndarray, b: np.ndarray) -> float:
    nb = np.linalg.norm(b)
    if nb == 0:
        return float(np.linalg.norm(a))
    return float(np.linalg.norm(a - b) / nb)


def compare_core(job, layout, corelen, got, ref, tol=FP32_TOL, weights_exact=True):
    out = {}
    for name, sl in regions(job, layout, corelen):
        g, r = got[sl], ref[sl]
        if name in ("bweight", "acweight"):
            if weights_exact:
                assert np.array_equal(g.astype(np.float32), r.astype(np.float32)), (name, g[:8], r[:8])
            else:
                assert np.allclose(g, r, rtol=1e-6, atol=1e-6), name
        else:
            e = rel_err(g, r)
            out[name] = e
            assert e <= tol, "%s relative error %.3g > %.3g" % (name, e, tol)
            scale = np.max(np.abs(r)) if r.size else 1.0
            if scale > 0:
                m = float(np.max(np.abs(g - r)) / scale)
                assert m <= 10 * tol, "%s max error %.3g" % (name, m)
    return out
