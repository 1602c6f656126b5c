"""INTERLACEDVDIF stations on the GPU (fxb_station.mux_threads): per-band data
weights (mk5mode.cpp:145-166), bands blanked by the frames' EDV4 validity
masks (format_vdif.c:4699-4780) in the F stage, baseline and
autocorrelation weights from the per-band weights (core.cpp:1032,
mode.cpp:1300-1303).  Checked against the FP64 oracle (weights exact), with
invalid frames on one station and two EDV4 mask lengths."""
import numpy as np
import pytest

from fxb200 import synth
from fxb200.native import Correlator
from helpers import compare_core, edv4_inputs, mux_job

import fxoracle

pytestmark = pytest.mark.gpu


@pytest.mark.parametrize("masklength,xmac", [(4, "fp32"), (2, "fp32"), (4, "fp16")])
def test_interlaced_vdif_matches_oracle(masklength, xmac):
    job = mux_job(masklength=masklength)
    corr = Correlator(job, xmac=xmac)
    orc = fxoracle.OracleCorrelator(job)
    ref = None
    for k, (sec, ns) in enumerate([(0, 1_024_000), (0, 3_072_000)]):
        f0 = synth.subint_window(job, 0, sec, ns)[0]
        inputs = edv4_inputs(job, synth.subint_inputs(job, sec, ns, rho=0.05, seed=13 + k,
                                                      invalid={0: [f0 + 1, f0 + 6]}), seed=k)
        corr.submit(inputs, sec, ns)
        ref = orc.process_subint(inputs, sec, ns, coreresult=ref)
    got, layout, n = corr.results(), corr.layout(), corr.corelen
    corr.close()
    assert np.array_equal(layout, orc.layout())
    if xmac == "fp32":
        compare_core(job, layout, n, got, ref)
    else:
        compare_core(job, layout, n, got, ref, tol=1e-3)
