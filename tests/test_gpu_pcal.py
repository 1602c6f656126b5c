"""Phase-cal extraction on the GPU (fxb_station.pcal_interval_mhz).

The device folds every valid FFT window's unpacked samples into bins by
sample number modulo the extractor's period and takes the DFT at the tone
bins when the result is read (pcal.cpp:927-1105, core.cpp:1124-1150).
Checked against the FP64 oracle, itself pinned to the compiled reference on
the same jobs: integer LOs (32 bins, register sums), a fractional LO (3200
bins, shared-memory bins), 8-bit samples, a band without a tone and a 5 MHz
comb; invalid frames and several subints; reset.
"""
import numpy as np
import pytest

from fxb200 import synth
from fxb200.native import Correlator
from helpers import PCAL_JOBS, compare_core, pcal_job, regions

import fxoracle

pytestmark = pytest.mark.gpu

SUBINTS = [(0, 1_024_000), (0, 3_072_000), (0, 5_120_000)]


def _run(job, xmac="fp32", invalid=None, subints=SUBINTS):
    corr = Correlator(job, xmac=xmac)
    orc = fxoracle.OracleCorrelator(job)
    ref = None
    for sec, ns in subints:
        inputs = synth.subint_inputs(job, sec, ns, rho=0.05, seed=13, invalid=invalid)
        corr.submit(inputs, sec, ns)
        ref = orc.process_subint(inputs, sec, ns, coreresult=ref)
    got, layout, n = corr.results(), corr.layout(), corr.corelen
    corr.close()
    assert np.array_equal(layout, orc.layout())
    return got, ref, layout, n


@pytest.mark.parametrize("name", sorted(PCAL_JOBS))
def test_pcal_matches_oracle(name):
    job = PCAL_JOBS[name]()
    got, ref, layout, n = _run(job)
    errs = compare_core(job, layout, n, got, ref)
    assert "pcal" in errs


def test_pcal_with_invalid_frames_and_tensor_core_form():
    job = PCAL_JOBS["pcal_frac_lo"]()
    f0 = synth.subint_window(job, 0, *SUBINTS[0])[0]
    got, ref, layout, n = _run(job, xmac="fp16", invalid={0: [f0 + 1, f0 + 5], 2: [f0 + 2]})
    pc = dict(regions(job, layout, n))["pcal"]
    e = np.linalg.norm(got[pc] - ref[pc]) / np.linalg.norm(ref[pc])
    assert e < 1e-5, e


def test_pcal_reset_starts_again():
    job = PCAL_JOBS["pcal_int_lo"]()
    corr = Correlator(job)
    sec, ns = SUBINTS[0]
    inputs = synth.subint_inputs(job, sec, ns, rho=0.05, seed=13)
    corr.submit(inputs, sec, ns)
    first = corr.results()
    corr.reset()
    corr.submit(inputs, sec, ns)
    again = corr.results()
    corr.close()
    pc = dict(regions(job, _layout(job), len(first) // 2))["pcal"]
    assert np.abs(first[pc]).max() > 0
    assert np.array_equal(first[pc], again[pc])


def _layout(job):
    from fxb200.native import job_layout
    return job_layout(job)[0]


def test_pcal_long_subint_fine_bins():
    """16000 FFT windows per subint and 32000 bins per band on 5 stations:
    one chunk of FFTs per launch would need a 320 KB FFT table in shared
    memory, so the windows are split into chunks that fit."""
    job = pcal_job(nstation=5, nfreq=2, nchan=64, freq0=8400.001, subint_ns=64_000_000)
    assert job.blocks_per_send() == 16000
    got, ref, layout, n = _run(job, subints=[(0, 0)])
    errs = compare_core(job, layout, n, got, ref)
    assert "pcal" in errs
