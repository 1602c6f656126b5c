"""Zoom bands on the GPU (fxb_station.zoom_freq / zoom_pol).

A zoom band is a channel window of a recorded band correlated as a frequency
of its own (mode.cpp:169-208, core.cpp:1266-1363).  The product gathers each
zoom band's spectra rows from its parent's after the F stage and correlates
the zoom frequency with the ordinary XMAC.  Checked here: parity with the FP64
oracle (itself pinned to the compiled reference on the same jobs) in the FP32,
BF16 and FP8 forms; zoom spectra that are the parent's channels exactly; and
zoom results that do not depend on whether the parents are correlated too.
"""
import numpy as np
import pytest

from fxb200 import synth
from fxb200.native import Correlator, job_layout
from helpers import compare_core, mixed_bw_zoom_job, zoom_job
from test_gpu_tc import FP8_TOL, tc_errors
from helpers import assert_tc_gate

import fxoracle

pytestmark = pytest.mark.gpu

SUBINTS = [(0, 1_024_000), (0, 3_072_000)]
JOBS = {
    "zoom": lambda: zoom_job(),
    "zoom_only": lambda: zoom_job(keep_parents=False),
    "zoom_avg4": lambda: zoom_job(avg=4),
    "zoom_mixed_bw": lambda: mixed_bw_zoom_job(),
}


def _run(job, xmac, subints=SUBINTS, oracle=True):
    corr = Correlator(job, xmac=xmac)
    orc = fxoracle.OracleCorrelator(job) if oracle else None
    ref = None
    for sec, ns in subints:
        inputs = synth.subint_inputs(job, sec, ns, rho=0.05, seed=11)
        corr.submit(inputs, sec, ns)
        if orc:
            ref = orc.process_subint(inputs, sec, ns, coreresult=ref)
    got, layout, n = corr.results(), corr.layout(), corr.corelen
    corr.close()
    if orc:
        assert np.array_equal(layout, orc.layout())
    return got, ref, layout, n


@pytest.mark.parametrize("name", sorted(JOBS))
def test_zoom_fp32_matches_oracle(name):
    job = JOBS[name]()
    got, ref, layout, n = _run(job, "fp32")
    compare_core(job, layout, n, got, ref)


@pytest.mark.parametrize("name", sorted(JOBS))
def test_zoom_fp16_matches_oracle(name):
    job = JOBS[name]()
    got, ref, layout, n = _run(job, "fp16")
    assert_tc_gate(tc_errors(job, layout, n, got, ref))


def test_zoom_fp8_matches_oracle():
    job = zoom_job()
    got, ref, layout, n = _run(job, "fp8")
    e = tc_errors(job, layout, n, got, ref)
    assert e["ccu"] <= FP8_TOL and e["auto_rel"] <= FP8_TOL, e


@pytest.mark.parametrize("xmac", ["fp32", "fp16"])
def test_zoom_spectra_are_parent_channels(xmac):
    # zoom frequency 2 is channels 64..127 of frequency 0 (4 MHz in, 62.5 kHz
    # channels); every station zooms both polarisations, so zoom row r is
    # parent row r
    job = zoom_job()
    corr = Correlator(job, xmac=xmac)
    sec, ns = SUBINTS[0]
    corr.submit(synth.subint_inputs(job, sec, ns, rho=0.05, seed=11), sec, ns)
    parent, zoom = corr.spectra(0), corr.spectra(2)
    corr.close()
    assert zoom.shape == (parent.shape[0], parent.shape[1], 64)
    assert np.array_equal(zoom, parent[:, :, 64:128])
    assert np.abs(zoom).max() > 0


def _zoom_region(job, layout, f):
    nf, nb = len(job.freqs), len(job.baselines)
    bl = layout[:nf * nb].reshape(nf, nb)[f]
    nprod = [sum(len(pp) for ff, pp in b.products if ff == f) for b in job.baselines]
    chans = job.freqs[f].nchan // job.freqs[f].chans_to_avg
    return np.concatenate([np.arange(2 * o, 2 * (o + k * chans)) for o, k in zip(bl, nprod) if o >= 0])


@pytest.mark.parametrize("xmac", ["fp32", "fp16"])
def test_zoom_results_independent_of_parents(xmac):
    # the same zoom windows correlated with and without their parents'
    # products give bit-identical zoom visibilities
    with_parents, only = zoom_job(), zoom_job(keep_parents=False)
    a, _, la, _ = _run(with_parents, xmac, oracle=False)
    b, _, lb, _ = _run(only, xmac, oracle=False)
    for f in range(2, len(with_parents.freqs)):
        ia, ib = _zoom_region(with_parents, la, f), _zoom_region(only, lb, f)
        assert ia.size == ib.size > 0
        assert np.array_equal(a[ia], b[ib]), f


def test_zoom_layout_is_the_hosts():
    job = mixed_bw_zoom_job()
    corr = Correlator(job)
    lay, n = job_layout(job)
    assert np.array_equal(corr.layout(), lay) and corr.corelen == n
    corr.close()
