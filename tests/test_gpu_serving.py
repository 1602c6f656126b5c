"""Serving loop on the GPU (fxb_server_* through the C ABI): jobs of
different shapes submitted while others run give the same core result as
each job run alone, admission against a small HBM budget still completes
every job, and a served job matches the FP64 oracle."""
import numpy as np
import pytest

from fxb200 import serving
from fxb200.native import Correlator
from helpers import small_job
from test_gpu_tc import tc_errors
from helpers import assert_tc_gate

import fxoracle

pytestmark = pytest.mark.gpu


def _jobs():
    # three shapes: stations, subbands, channels and bits differ
    specs = [dict(nstation=3, nchan=256, bw=16.0, nfreq=2, full_pol=True, seed=2),
             dict(nstation=4, nchan=1024, bw=32.0, nfreq=1, full_pol=True, subint_ns=2_048_000, seed=3),
             dict(nstation=2, nchan=128, bw=8.0, nfreq=2, full_pol=True, nbits=8, subint_ns=2_048_000, seed=4)]
    out = []
    for k, kw in enumerate(specs):
        job = small_job(**kw)
        out.append((job, serving.job_subints(job, 3, seed=20 + k, rho=0.05)))
    return out


def _alone(job, subints, xmac):
    c = Correlator(job, xmac=xmac)
    for inputs, sec, ns in subints:
        c.submit(inputs, sec, ns)
    r = c.results()
    c.close()
    return r


@pytest.mark.parametrize("xmac", ["fp16", "fp32"])
def test_results_same_alone_and_in_the_mix(xmac):
    jobs = _jobs()
    alone = [_alone(j, s, xmac) for j, s in jobs]
    srv = serving.Server(budget_bytes=8 << 30, max_active=3)
    handles = [srv.submit(j, s, xmac=xmac) for j, s in jobs]
    for h, ref in zip(handles, alone):
        got = srv.wait(h, 120.0)
        assert np.array_equal(got, ref)
    st = srv.stats()
    srv.close()
    assert st["completed"] == 3 and st["p99_ms"] >= st["p50_ms"] > 0


def test_admission_under_a_small_budget_completes_every_job():
    jobs = _jobs()
    need = max(serving.job_footprint(j) for j, _ in jobs)
    srv = serving.Server(budget_bytes=need, max_active=3)     # one job at a time fits
    handles = [srv.submit(j, s) for j, s in jobs]
    for h in handles:
        srv.wait(h, 120.0)
        assert srv.poll(h)[0] == 2
    assert srv.stats()["completed"] == 3
    srv.close()


def test_served_job_matches_oracle():
    job, subints = _jobs()[1]
    srv = serving.Server(budget_bytes=4 << 30, max_active=2)
    h = srv.submit(job, subints)
    got = srv.wait(h, 120.0)
    srv.close()
    orc = fxoracle.OracleCorrelator(job)
    ref = None
    for inputs, sec, ns in subints:
        ref = orc.process_subint(inputs, sec, ns, coreresult=ref)
    c = Correlator(job, xmac="fp16")
    layout, n = c.layout(), c.corelen
    c.close()
    assert_tc_gate(tc_errors(job, layout, n, got, ref))


def test_pinned_buffers_give_the_same_result_and_phases_add_up():
    jobs = _jobs()
    pinned = []
    for k, (job, _) in enumerate(jobs):
        pinned.append((job, serving.job_subints(job, 3, seed=20 + k, rho=0.05, pinned=True)))
    alone = [_alone(j, s, "fp16") for j, s in jobs]
    srv = serving.Server(budget_bytes=8 << 30, max_active=3)
    handles = [srv.submit(j, s) for j, s in pinned]
    for h, ref in zip(handles, alone):
        assert np.array_equal(srv.wait(h, 120.0), ref)
        t = srv.job_times(h)
        lat = srv.poll(h)[1]
        assert all(v >= 0 for v in t.values())
        assert abs(sum(t.values()) - lat) < 1e-3 * max(lat, 1.0) + 1e-3
    srv.close()


def test_a_failing_job_is_reported_and_the_others_complete():
    import ctypes
    from fxb200.native import FxbError
    jobs = _jobs()
    srv = serving.Server(budget_bytes=8 << 30, max_active=3)
    good = srv.submit(*jobs[0])
    job, subints = jobs[1]
    bad = serving.ServedJob(job, subints, "fp16", 2)
    bad.nbytes[len(job.stations)] = -1            # second subint, first station: rejected by the host check
    jid = ctypes.c_uint64(0)
    assert serving._bind().fxb_server_submit(srv.srv, ctypes.byref(bad.req), ctypes.byref(jid)) == 0
    bad.id = jid.value
    srv.jobs.append(bad)
    last = srv.submit(*jobs[2])
    with pytest.raises(FxbError):
        srv.wait(bad, 120.0)
    assert srv.poll(bad)[0] == 3
    for h in (good, last):
        srv.wait(h, 120.0)
        assert srv.poll(h)[0] == 2
    assert "bad station buffer" in serving._bind().fxb_server_last_error(srv.srv).decode()
    srv.close()


def test_zoom_and_pcal_jobs_served_in_the_mix():
    # a zoom job and a phase-cal job (fractional LO: 3200 bins) served beside
    # a plain one give each job's own result bit for bit
    from helpers import PCAL_JOBS, zoom_job
    jobs = [zoom_job(), PCAL_JOBS["pcal_frac_lo"](), _jobs()[0][0]]
    jobs = [(j, serving.job_subints(j, 3, seed=60 + k, rho=0.05)) for k, j in enumerate(jobs)]
    alone = [_alone(j, s, "fp16") for j, s in jobs]
    srv = serving.Server(budget_bytes=8 << 30, max_active=3)
    handles = [srv.submit(j, s, xmac="fp16") for j, s in jobs]
    for h, ref in zip(handles, alone):
        assert np.array_equal(srv.wait(h, 120.0), ref)
    srv.close()


def test_long_jobs_served_beside_short_ones():
    """The serving workload's 0.1-2 s range: a 2 s job (500 subints of 4 ms,
    three distinct subints of VDIF cycled with their own times) and a 1 s job
    served beside a 0.1 s one give each job's own result bit for bit."""
    short = small_job(nstation=3, nchan=256, bw=16.0, nfreq=2, full_pol=True, seed=2)
    long_ = small_job(nstation=4, nchan=256, bw=16.0, nfreq=1, full_pol=True, seed=5)
    mid = small_job(nstation=2, nchan=512, bw=32.0, nfreq=2, full_pol=True, nbits=8, subint_ns=2_048_000, seed=6)
    jobs = [(long_, serving.job_subints(long_, 500, seed=71, pinned=True, pool=3)),
            (short, serving.job_subints(short, 25, seed=72, pool=3)),
            (mid, serving.job_subints(mid, 488, seed=73, pool=3))]
    assert abs(len(jobs[0][1]) * long_.subint_ns * 1e-9 - 2.0) < 1e-9
    alone = [_alone(j, s, "fp16") for j, s in jobs]
    srv = serving.Server(budget_bytes=8 << 30, max_active=3)
    handles = [srv.submit(j, s, xmac="fp16") for j, s in jobs]
    for h, ref in zip(handles, alone):
        assert np.array_equal(srv.wait(h, 300.0), ref)
    st = srv.stats()
    srv.close()
    assert st["completed"] == 3 and st["data_seconds"] > 3.0
