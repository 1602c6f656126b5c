"""The CUDA path directly against golden outputs of the reference's own code
(tests/golden): GPU VDIF decoding bit-exact against mark5access, and the
core result of a small job within 1e-5 of the reference."""
import glob
import os
import sys

import numpy as np
import pytest

from fxb200 import native
from fxb200.native import Correlator
from helpers import compare_core

pytestmark = pytest.mark.gpu

GOLD = os.path.join(os.path.dirname(os.path.abspath(__file__)), "golden")
sys.path.insert(0, GOLD)
from make_golden import small_job  # noqa: E402


@pytest.mark.parametrize("path", sorted(glob.glob(os.path.join(GOLD, "unpack_*.npz"))))
def test_gpu_unpack_matches_reference(path):
    z = np.load(path)
    for i, (off, n) in enumerate(zip(z["offsets"], z["nsamp"])):
        out, good = native.vdif_unpack(z["data"], int(z["payload"]), int(z["header"]), int(z["nchan"]),
                                       int(z["nbits"]), int(off), int(n))
        assert good == int(z["good"][i])
        assert np.array_equal(out, z["samples_%d" % i])


@pytest.mark.parametrize("xmac,tol", [("fp32", 1e-5)])
def test_gpu_correlation_matches_reference(xmac, tol):
    z = np.load(os.path.join(GOLD, "corr_small.npz"))
    job = small_job()
    inputs = [(z["buf_%d" % s], int(z["datasec"][s]), int(z["datans"][s])) for s in range(len(job.stations))]
    corr = Correlator(job, xmac=xmac)
    # the fixture predates the phase-cal offsets: a job without phase cal has -1 there
    lay = corr.layout()
    assert np.array_equal(lay[:len(z["layout"])], z["layout"]) and (lay[len(z["layout"]):] == -1).all()
    corr.submit(inputs, int(z["sec"]), int(z["ns"]))
    got = corr.results()
    corr.close()
    compare_core(job, lay, len(got) // 2, got.astype(np.float64), z["core"].astype(np.float64), tol=tol)
