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


@pytest.mark.parametrize("name", ["zoom", "zoom_only", "zoom_avg4", "zoom_mixed_bw"])
def test_zoom_layout_matches_oracle(name):
    from helpers import mixed_bw_zoom_job, zoom_job
    job = {"zoom": lambda: zoom_job(), "zoom_only": lambda: zoom_job(keep_parents=False),
           "zoom_avg4": lambda: zoom_job(avg=4), "zoom_mixed_bw": mixed_bw_zoom_job}[name]()
    lay, n = native.job_layout(job)
    orc = fxoracle.OracleCorrelator(job)
    assert n == orc.corelen
    assert np.array_equal(lay, orc.layout())


def test_zoom_rejections():
    from fxb200.job import Freq
    from helpers import zoom_job
    # one polarisation of a dual-polarisation parent while cross-hand
    # autocorrelations are written: the reference would output the parent's
    # cross-hand spectrum for it, which a single zoom band cannot form
    job = zoom_job(zooms=[(0, 4.0, 4.0)])
    job.stations[0].zoom_bands = job.stations[0].zoom_bands[:1]
    job.baselines = [b for b in job.baselines if b.ds1 != 0]
    with pytest.raises(native.FxbError, match="UNSUPPORTED"):
        native.job_layout(job)
    # a zoom band outside every recorded band
    job = zoom_job(zooms=[(0, 4.0, 4.0)])
    job.freqs[-1] = Freq(9000.0, 4.0, 64)
    with pytest.raises(Exception):
        native.job_layout(job)
    # zoom averaging that differs from the station's
    job = zoom_job(zooms=[(0, 4.0, 4.0)])
    job.freqs[-1].chans_to_avg = 2
    with pytest.raises(native.FxbError, match="UNSUPPORTED"):
        native.job_layout(job)


@pytest.mark.parametrize("name", ["pcal_int_lo", "pcal_frac_lo", "pcal_8bit", "pcal_no_tone", "pcal_5mhz",
                                  "pcal_1024_bins", "pcal_lsb", "pcal_lsb_frac", "pcal_shifting"])
def test_pcal_layout_matches_oracle(name):
    from helpers import PCAL_JOBS
    job = PCAL_JOBS[name]()
    lay, n = native.job_layout(job)
    orc = fxoracle.OracleCorrelator(job)
    assert n == orc.corelen
    assert np.array_equal(lay, orc.layout())


def test_pcal_rejections():
    from helpers import pcal_job
    # a phase-cal base that puts the first tone on the LO needs the trivial
    # extractor, whose tone count then differs from the configuration's
    job = pcal_job(1.0, base=-1.0, nstation=2)
    with pytest.raises(native.FxbError, match="UNSUPPORTED"):
        native.job_layout(job)


def test_job_rejections():
    job = small_job()
    job.subint_ns = 4_000_100          # not a whole number of FFTs
    with pytest.raises(Exception):
        native.job_layout(job)
    job = small_job()
    job.stations[0].nbits = 4
    with pytest.raises(Exception):
        native.job_layout(job)


def test_band_corrections_accepted_and_checked():
    # per-frequency clock / phase / LO offsets leave the layout as it is; bands
    # of one frequency must agree on them
    from helpers import corr_job
    job = corr_job()
    lay, n = native.job_layout(job)
    plain = small_job(nstation=3, full_pol=True, nfreq=2, order=1)
    lay0, n0 = native.job_layout(plain)
    assert n == n0 and np.array_equal(lay, lay0)
    holder = native.DescHolder(job)
    st = holder.desc.stations[1]
    st.band_clock_us[1] = st.band_clock_us[0] + 0.001      # bands 0 and 1 record the same frequency
    out = np.zeros(64, dtype=np.int32)
    rc = native.lib().fxb_job_layout(holder.ptr(), out.ctypes.data_as(native.ctypes.POINTER(native.ctypes.c_int32)),
                                     out.size, native.ctypes.byref(native.ctypes.c_int64(0)))
    assert rc == 1                      # FXB_ERR_ARG
