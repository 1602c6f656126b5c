"""Integration output against the reference's own Visibility (compiled from
mpifxcorr/src/visibility.cpp into oracle/_ref): for the same integrated
core result, the calibrated SWIN records written by fxb_vis_calibrate +
fxb_vis_write_swin are byte-identical to what Visibility::writedata writes --
headers (baseline number, time, indices, polarisation pair, weight, uvw) and
data -- with correlation-coefficient scaling and with a-priori Tsys.  Runs on
the CPU (no GPU: calibration needs only the job layout)."""
import os

import numpy as np
import pytest

from fxb200 import synth, visibility
from helpers import mixed_bw_zoom_job, small_job, zoom_job

import refcorr

pytestmark = pytest.mark.skipif(not refcorr.available(), reason="reference build oracle/_ref absent")

CASES = {
    "fullpol": (dict(nstation=3, full_pol=True), None),
    "fullpol_tsys": (dict(nstation=3, full_pol=True), [40.0, 55.0, 70.0]),
    "parallel_8bit_tsys": (dict(nstation=3, nbits=8), [30.0, 30.0, 45.0]),
    "avg4_two_freqs": (dict(nstation=3, full_pol=True, avg=4, nfreq=2), None),
}


def _subints(job, ref, n=2):
    out = []
    for k in range(n):
        sec, ns = 0, (k + 1) * job.subint_ns
        inputs = synth.subint_inputs(job, sec, ns, rho=0.05, seed=11 + k)
        vf = [synth.valid_flags(job) for _ in job.stations]
        out.append(ref.process_subint(inputs, vf, 0, sec, ns))
    return out


ZOOM_CASES = {
    "zoom": (lambda: zoom_job(), None),
    "zoom_only": (lambda: zoom_job(keep_parents=False), None),
    "zoom_mixed_bw": (lambda: mixed_bw_zoom_job(), None),
    "zoom_parallel_tsys": (lambda: zoom_job(full_pol=False), [40.0, 55.0, 70.0]),
}


def _job(name):
    if name in CASES:
        kw, tsys = CASES[name]
        return small_job(**kw), tsys
    build, tsys = ZOOM_CASES[name]
    return build(), tsys


@pytest.mark.parametrize("name", sorted(CASES) + sorted(ZOOM_CASES))
def test_swin_records_match_reference_visibility(name, tmp_path):
    job, tsys = _job(name)
    ref = refcorr.RefCorrelator(job, tsys=tsys)
    subs = _subints(job, ref)
    expect = ref.visibility_write(subs)
    ref.close()
    integ = np.zeros_like(subs[0])
    for s in subs:
        integ += s                                  # Visibility::addData, in order
    params = visibility.VisParams.for_job(job, tsys=tsys)
    cal = visibility.calibrate(job, params, integ)
    visibility.write_swin(job, params, cal, str(tmp_path))
    with open(os.path.join(str(tmp_path), "DIFX_%05d_%06d.s0000.b0000" % (job.start_mjd, job.start_sec)), "rb") as f:
        got = f.read()
    assert len(expect) > 0
    assert got == expect
    nch = {f: fr.nchan // fr.chans_to_avg for f, fr in enumerate(job.freqs)}
    recs = visibility.read_swin(got, nch.__getitem__)
    nprod = sum(len(pp) for b in job.baselines for _, pp in b.products)
    assert sum(1 for r in recs if r.baseline % 257) == nprod
    assert all(r.weight > 0 for r in recs)


def test_records_append_per_integration(tmp_path):
    job = small_job(nstation=2, full_pol=False)
    ref = refcorr.RefCorrelator(job)
    integ = sum(_subints(job, ref))
    ref.close()
    p0 = visibility.VisParams.for_job(job)
    p1 = visibility.VisParams.for_job(job, int_start_sec=1)
    cal = visibility.calibrate(job, p0, integ)
    visibility.write_swin(job, p0, cal, str(tmp_path))
    visibility.write_swin(job, p1, cal, str(tmp_path))
    path = os.path.join(str(tmp_path), "DIFX_%05d_%06d.s0000.b0000" % (job.start_mjd, job.start_sec))
    nch = {f: fr.nchan for f, fr in enumerate(job.freqs)}
    with open(path, "rb") as f:
        recs = visibility.read_swin(f.read(), nch.__getitem__)
    half = len(recs) // 2
    assert half > 0 and len(recs) == 2 * half
    assert all(abs(r.seconds - (job.duration_s / 2)) < 1e-9 for r in recs[:half])
    assert all(abs(r.seconds - (1 + job.duration_s / 2)) < 1e-9 for r in recs[half:])


def test_tsys_with_zoom_cross_hand_autos_is_refused():
    # the reference's opposite-hand lookup for a zoom band reads past its
    # zoom band tables (configuration.cpp:907-922): no defined result
    job = zoom_job()
    params = visibility.VisParams.for_job(job, tsys=[40.0, 55.0, 70.0])
    from fxb200.native import FxbError
    with pytest.raises(FxbError, match="UNSUPPORTED"):
        visibility.calibrate(job, params, np.zeros(2 * _corelen(job), dtype=np.float32))


def _corelen(job):
    from fxb200.native import job_layout
    return job_layout(job)[1]


@pytest.mark.parametrize("name", ["pcal_int_lo", "pcal_frac_lo", "pcal_lsb", "pcal_shifting", "pcal_no_tone"])
def test_pcal_files_match_reference_visibility(name, tmp_path):
    # phase-cal tones scaled by their band's data weight (visibility.cpp:586-609)
    # and written as one line per station to PCAL_<mjd>_<sec>_<station> after
    # the reference's header (visibility.cpp:104-135, 928-990)
    from helpers import PCAL_JOBS
    job = PCAL_JOBS[name]()
    ref = refcorr.RefCorrelator(job)
    subs = _subints(job, ref)
    expect = ref.visibility_write(subs)
    expect_pcal = dict(ref.pcal_files)
    ref.close()
    integ = np.zeros_like(subs[0])
    for s in subs:
        integ += s
    params = visibility.VisParams.for_job(job)
    cal = visibility.calibrate(job, params, integ)
    visibility.write_swin(job, params, cal, str(tmp_path))
    visibility.write_pcal(job, params, cal, str(tmp_path))
    with open(os.path.join(str(tmp_path), "DIFX_%05d_%06d.s0000.b0000" % (job.start_mjd, job.start_sec)), "rb") as f:
        assert f.read() == expect
    got_pcal = {}
    for fn in os.listdir(str(tmp_path)):
        if fn.startswith("PCAL_"):
            with open(os.path.join(str(tmp_path), fn), "rb") as f:
                got_pcal[fn] = f.read()
    # a station's file exists in the reference from its header alone
    for fn, data in expect_pcal.items():
        if data.count(b"\n") > 5:
            assert got_pcal.get(fn) == data, fn
        else:
            assert fn not in got_pcal, fn
    assert any(d.count(b"\n") > 5 for d in expect_pcal.values()) or name == "pcal_no_tone"
