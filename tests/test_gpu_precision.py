"""Precision sweep of the cross-multiply operand on the c1 workload shape
(10 stations, eight 32 MHz bands, 1024 channels, full cross hands): the F
output in FP32 (plain form), FP16 (the tensor-core form), BF16 and FP8 e4m3
with a per-(channel, station) scale, over correlation coefficients 1e-4,
1e-3 and 1e-2, each against the FP64 oracle on the same seeded samples.

Reported per (dtype, rho), with the figures of ``helpers.vis_errors``:
norm-wise relative cross and autocorrelation errors, per-visibility relative
amplitude and phase (radians) errors (rms and 99th percentile), the error in
correlation-coefficient units, and the band-averaged amplitude and phase
errors of each (baseline, product, band), where the common sky signal
dominates.  Gates (the stated tolerances): the FP32 form within 1e-5 norm-wise, the
FP16 tensor-core form within 1e-3 (``helpers.assert_tc_gate``).  With
FXB_REPORT_DIR set the table is written there as precision_c2.json."""
import json
import os

import numpy as np
import pytest

from fxb200 import configs, synth
from fxb200.native import Correlator, FxbError
from helpers import TC_REL_TOL, assert_tc_gate, regions, vis_errors

import fxoracle

pytestmark = pytest.mark.gpu

RHOS = (1e-4, 1e-3, 1e-2)
DTYPES = ("fp32", "fp16", "bf16", "fp8")
SUBINT_NS = 2_048_000
SUBINTS = ((0, SUBINT_NS), (0, 2 * SUBINT_NS))


def _complex(a):
    return a[0::2].astype(np.float64) + 1j * a[1::2].astype(np.float64)


def _errors(job, layout, n, got, ref):
    out = vis_errors(job, layout, n, got, ref)
    xc = dict(regions(job, layout, n))["cross"]
    v, r = _complex(got[xc]), _complex(ref[xc])
    # band averages: every baseline product holds nchan consecutive channels
    nchan = job.freqs[0].nchan
    va, ra = v.reshape(-1, nchan).mean(axis=1), r.reshape(-1, nchan).mean(axis=1)
    out["avg_amp"] = float(np.sqrt(np.mean(((np.abs(va) - np.abs(ra)) / np.abs(ra)) ** 2)))
    out["avg_phase"] = float(np.sqrt(np.mean(np.angle(va * np.conj(ra)) ** 2)))
    return out


@pytest.fixture(scope="module")
def sweep_inputs():
    job = configs.c1(subint_ns=SUBINT_NS)
    data = {}
    for k, rho in enumerate(RHOS):
        orc = fxoracle.OracleCorrelator(job)
        ref, subs = None, []
        for sec, ns in SUBINTS:
            inputs = synth.subint_inputs(job, sec, ns, rho=rho, seed=40 + k)
            ref = orc.process_subint(inputs, sec, ns, coreresult=ref)
            subs.append((inputs, sec, ns))
        data[rho] = (subs, ref)
    return job, data


def test_precision_sweep(sweep_inputs):
    job, data = sweep_inputs
    table = []
    for dtype in DTYPES:
        for rho in RHOS:
            subs, ref = data[rho]
            try:
                corr = Correlator(job, xmac=dtype)
            except FxbError as e:
                table.append({"dtype": dtype, "rho": rho, "unsupported": str(e)})
                continue
            for inputs, sec, ns in subs:
                corr.submit(inputs, sec, ns)
            got = corr.results()
            layout, n = corr.layout(), corr.corelen
            corr.close()
            row = {"dtype": dtype, "rho": rho}
            row.update(_errors(job, layout, n, got, ref))
            table.append(row)
    report = {"workload": "c1 shape: 10 stations, 8 x 32 MHz, 1024 channels, full cross hands, 2 x 2.048 ms subints",
              "oracle": "FP64 restatement of Mode::process + XMAC on the same seeded samples",
              "gates": {"fp32": "cross_rel, auto_rel <= 1e-5", "fp16": "cross_rel, auto_rel, amp_rms, phase_rms <= %g" % TC_REL_TOL},
              "rows": table}
    if os.environ.get("FXB_REPORT_DIR"):
        with open(os.path.join(os.environ["FXB_REPORT_DIR"], "precision_c2.json"), "w") as f:
            json.dump(report, f, indent=1)
    for row in table:
        print(row)
        if row["dtype"] == "fp32":
            assert row["cross_rel"] <= 1e-5 and row["auto_rel"] <= 1e-5, row
        elif row["dtype"] == "fp16":
            assert "unsupported" not in row, row
            assert_tc_gate(row)
