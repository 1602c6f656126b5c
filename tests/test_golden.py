"""The oracle restatement against golden outputs of the reference's own code
(tests/golden/*.npz, made by tests/golden/make_golden.py from oracle/_ref):
VDIF samples and good-sample counts bit-exact, core result within the
reference's FP32 rounding, layout and delay interpolators exact."""
import glob
import os
import sys

import numpy as np
import pytest

from helpers import compare_core

import fxoracle

GOLD = os.path.join(os.path.dirname(os.path.abspath(__file__)), "golden")
sys.path.insert(0, GOLD)
from make_golden import small_job  # noqa: E402


@pytest.mark.parametrize("path", sorted(glob.glob(os.path.join(GOLD, "unpack_*.npz"))))
def test_oracle_unpack_matches_golden(path):
    z = np.load(path)
    for i, (off, n) in enumerate(zip(z["offsets"], z["nsamp"])):
        out, good = fxoracle.vdif_unpack(z["data"], int(z["payload"]), int(z["header"]), int(z["nchan"]),
                                         int(z["nbits"]), int(off), int(n))
        assert good == int(z["good"][i])
        assert np.array_equal(out, z["samples_%d" % i])


def load_corr():
    z = np.load(os.path.join(GOLD, "corr_small.npz"))
    job = small_job()
    inputs = [(z["buf_%d" % s], int(z["datasec"][s]), int(z["datans"][s])) for s in range(len(job.stations))]
    return job, z, inputs


def test_oracle_correlation_matches_golden():
    job, z, inputs = load_corr()
    orc = fxoracle.OracleCorrelator(job)
    # the fixture predates the phase-cal offsets: a job without phase cal has -1 there
    lay = orc.layout()
    assert np.array_equal(lay[:len(z["layout"])], z["layout"]) and (lay[len(z["layout"]):] == -1).all()
    for s in range(len(job.stations)):
        assert np.array_equal(orc.interpolator(s, int(z["sec"]), int(z["ns"])), z["interp"][s])
    got = orc.process_subint(inputs, int(z["sec"]), int(z["ns"]))
    compare_core(job, lay, orc.corelen, z["core"].astype(np.float64), got, tol=2e-6)
