"""Precision sweep of the cross-multiply operand on the c1 workload shape
(10 stations, eight 32 MHz bands, 1024 channels, full cross hands): the F
output in FP32 (plain form), BF16 and FP8 e4m3 with a per-(channel, station)
scale (tensor-core forms), over correlation coefficients 1e-4, 1e-3 and 1e-2,
each against the FP64 oracle on the same seeded samples.

Reported per (dtype, rho), over every cross visibility:
  ccu_err    rms error in correlation-coefficient units (error of V_ab over
             the autocorrelation scale sqrt(A_aa A_bb)), the gated figure;
  amp_rms / amp_p99    relative amplitude error (|V| - |V64|) / |V64|;
  phase_rms / phase_p99  phase error arg(V conj(V64)) in degrees;
  avg_amp / avg_phase    the same for the band-averaged visibility of each
             (baseline, product, band), where the common sky signal dominates.
Visibilities with |V64| below a tenth of the median are left out of the
relative figures (their count is reported).  Gates: FP32 <= 1e-5 and BF16
<= 1e-3 in correlation-coefficient units.  With FXB_REPORT_DIR set the table
is written there as precision_c2.json."""
import json
import os

import numpy as np
import pytest

from fxb200 import configs, synth
from fxb200.native import Correlator, FxbError
from helpers import regions

import fxoracle

pytestmark = pytest.mark.gpu

RHOS = (1e-4, 1e-3, 1e-2)
DTYPES = ("fp32", "bf16", "fp8")
GATES = {"fp32": 1e-5, "bf16": 1e-3}
SUBINT_NS = 2_048_000
SUBINTS = ((0, SUBINT_NS), (0, 2 * SUBINT_NS))


def _complex(a):
    return a[0::2].astype(np.float64) + 1j * a[1::2].astype(np.float64)


def _errors(job, layout, n, got, ref):
    reg = dict(regions(job, layout, n))
    xc, ac = reg["cross"], reg["auto"]
    auto_rms = np.sqrt(np.mean(ref[ac][0::2] ** 2))
    out = {"ccu_err": float(np.sqrt(np.mean((got[xc] - ref[xc]) ** 2)) / auto_rms)}
    v, r = _complex(got[xc]), _complex(ref[xc])
    keep = np.abs(r) >= 0.1 * np.median(np.abs(r))
    amp = (np.abs(v[keep]) - np.abs(r[keep])) / np.abs(r[keep])
    ph = np.degrees(np.angle(v[keep] * np.conj(r[keep])))
    out.update(amp_rms=float(np.sqrt(np.mean(amp ** 2))), amp_p99=float(np.quantile(np.abs(amp), 0.99)),
               phase_rms=float(np.sqrt(np.mean(ph ** 2))), phase_p99=float(np.quantile(np.abs(ph), 0.99)),
               left_out=int((~keep).sum()), visibilities=int(keep.size))
    # band averages: every baseline product holds nchan consecutive channels
    nchan = job.freqs[0].nchan
    va, ra = v.reshape(-1, nchan).mean(axis=1), r.reshape(-1, nchan).mean(axis=1)
    out["avg_amp"] = float(np.sqrt(np.mean(((np.abs(va) - np.abs(ra)) / np.abs(ra)) ** 2)))
    out["avg_phase"] = float(np.sqrt(np.mean(np.degrees(np.angle(va * np.conj(ra))) ** 2)))
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
              "oracle": "FP64 restatement of Mode::process + XMAC on the same seeded samples", "rows": table}
    if os.environ.get("FXB_REPORT_DIR"):
        with open(os.path.join(os.environ["FXB_REPORT_DIR"], "precision_c2.json"), "w") as f:
            json.dump(report, f, indent=1)
    for row in table:
        print(row)
        gate = GATES.get(row["dtype"])
        if gate is not None:
            assert "unsupported" not in row, row
            assert row["ccu_err"] <= gate, row
