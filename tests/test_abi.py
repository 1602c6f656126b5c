"""The C-ABI library loads without a GPU and exports every entry point that
include/fxb200.h declares; the GPU-free layout entry point agrees with the
oracle's restatement of Configuration::populateResultLengths."""
import os
import re

import numpy as np
import pytest

from fxb200 import native
from helpers import small_job

import fxoracle

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


def declared_symbols():
    text = open(os.path.join(ROOT, "include", "fxb200.h")).read()
    return sorted(set(re.findall(r"FXB_API[^;(]*?\b(fxb_\w+)\s*\(", text)))


def test_header_declares_entry_points():
    syms = declared_symbols()
    assert "fxb_create" in syms and "fxb_submit_subint" in syms and "fxb_read_results" in syms
    assert len(syms) >= 15


def test_library_exports_every_declared_symbol():
    L = native.lib()
    missing = [s for s in declared_symbols() if not hasattr(L, s)]
    assert not missing, missing


@pytest.mark.parametrize("kw", [dict(), dict(full_pol=True), dict(nfreq=4, full_pol=True, avg=4),
                                dict(nstation=7, nfreq=2), dict(nbits=8, nstation=2)])
def test_layout_matches_oracle(kw):
    job = small_job(**kw)
    lay, n = native.job_layout(job)
    orc = fxoracle.OracleCorrelator(job)
    assert n == orc.corelen
    assert np.array_equal(lay, orc.layout())


def test_job_rejections():
    job = small_job()
    job.subint_ns = 4_000_100          # not a whole number of FFTs
    with pytest.raises(Exception):
        native.job_layout(job)
    job = small_job()
    job.stations[0].nbits = 4
    with pytest.raises(Exception):
        native.job_layout(job)
