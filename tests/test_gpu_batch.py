"""CUDA graphs and batches (fxb_set_graphs, fxb_batch_*).

A context's subints replayed as per-slot CUDA graphs give exactly the result
of launching the kernels one by one.  A batch of contexts with uneven
subband shapes (width, channels, bits), run as one graph launch per subint,
gives every member exactly the result it has alone, matches the FP64 oracle,
and keeps doing so after a reset; so does the fused form (one persistent F
launch and one XMAC launch over all members)."""
import numpy as np
import pytest

from fxb200 import synth
from fxb200.job import Freq, full_job
from fxb200.native import Batch, Correlator
from helpers import compare_core, small_job
from test_gpu_tc import tc_errors
from helpers import assert_tc_gate

import fxoracle

pytestmark = pytest.mark.gpu

SUBINT_NS = 2_048_000
SUBINTS = [(0, SUBINT_NS), (0, 2 * SUBINT_NS), (0, 3 * SUBINT_NS)]
# (width MHz, channels, bits): FFTs of 32, 64 and 4 us, all dividing the subint
SHAPES = [(4.0, 128, 2), (16.0, 1024, 8), (64.0, 256, 2)]


def _uneven_jobs(nstation=3):
    jobs = []
    for k, (bw, nchan, bits) in enumerate(SHAPES):
        job = full_job(nstation, [Freq(8400.0 + 100.0 * k, bw, nchan)], full_pol=True, subint_ns=SUBINT_NS,
                       nbits=bits)
        synth.make_delay_polys(job, seed=30 + k)
        job.validate()
        jobs.append(job)
    return jobs


def _inputs(job, k, sec, ns):
    return synth.subint_inputs(job, sec, ns, rho=0.05, seed=60 + k)


def _alone(job, k, xmac, graphs=True):
    c = Correlator(job, xmac=xmac)
    c.set_graphs(graphs)
    for sec, ns in SUBINTS:
        c.submit(_inputs(job, k, sec, ns), sec, ns)
    r = c.results()
    c.close()
    return r


@pytest.mark.parametrize("xmac", ["fp32", "fp16"])
def test_graph_replay_matches_eager_launches(xmac):
    job = small_job(nstation=4, nchan=256, bw=16.0, nfreq=2, full_pol=True, subint_ns=SUBINT_NS)
    eager = _alone(job, 0, xmac, graphs=False)
    graph = _alone(job, 0, xmac, graphs=True)
    assert np.array_equal(graph, eager)


@pytest.mark.parametrize("xmac", ["fp32", "fp16"])
def test_batch_members_match_each_job_alone(xmac):
    jobs = _uneven_jobs()
    alone = [_alone(j, k, xmac) for k, j in enumerate(jobs)]
    members = [Correlator(j, xmac=xmac) for j in jobs]
    batch = Batch(members)
    for sec, ns in SUBINTS:
        batch.submit([_inputs(j, k, sec, ns) for k, j in enumerate(jobs)], sec, ns)
    batch.sync()
    got = [m.results() for m in members]
    # after a reset the batch starts again from zero
    for m in members:
        m.reset()
    for sec, ns in SUBINTS:
        batch.submit([_inputs(j, k, sec, ns) for k, j in enumerate(jobs)], sec, ns)
    again = [m.results() for m in members]
    batch.close()
    for m in members:
        m.close()
    for g, a, r in zip(got, again, alone):
        assert np.array_equal(g, r)
        assert np.array_equal(a, r)


# beside SHAPES: 8192-point FFTs (whole-CTA units of the persistent F launch)
# and 2-bit 2048-point FFTs (the tensor-core FFT kernel)
FUSED_SHAPES = SHAPES + [(4.0, 4096, 8), (16.0, 1024, 2)]


@pytest.mark.parametrize("fused", [True, False])
def test_fused_batch_matches_each_job_alone(fused):
    # one persistent F launch and one XMAC launch for all members, or every
    # member as its own graph branch: either way each member's result is the
    # one it has alone, bit for bit
    jobs = []
    for k, (bw, nchan, bits) in enumerate(FUSED_SHAPES):
        job = full_job(3, [Freq(8400.0 + 100.0 * k, bw, nchan)], full_pol=True, subint_ns=SUBINT_NS, nbits=bits)
        synth.make_delay_polys(job, seed=30 + k)
        job.validate()
        jobs.append(job)
    alone = [_alone(j, k, "fp16") for k, j in enumerate(jobs)]
    members = [Correlator(j, xmac="fp16") for j in jobs]
    batch = Batch(members)
    assert batch.set_fused(fused) == fused
    for graphs in (True, False):
        batch.set_graphs(graphs)
        for m in members:
            m.reset()
        for sec, ns in SUBINTS:
            batch.submit([_inputs(j, k, sec, ns) for k, j in enumerate(jobs)], sec, ns)
        batch.sync()
        got = [m.results() for m in members]
        for k, (g, a) in enumerate(zip(got, alone)):
            assert np.array_equal(g, a), (graphs, FUSED_SHAPES[k])
    batch.close()
    for m in members:
        m.close()


def test_fused_batch_refused_for_fp32_members():
    jobs = _uneven_jobs()
    members = [Correlator(j, xmac="fp32") for j in jobs]
    batch = Batch(members)
    assert not batch.set_fused(True)
    batch.close()
    for m in members:
        m.close()


@pytest.mark.parametrize("xmac", ["fp32", "fp16"])
def test_batch_matches_oracle(xmac):
    jobs = _uneven_jobs()
    members = [Correlator(j, xmac=xmac) for j in jobs]
    batch = Batch(members)
    refs = [None] * len(jobs)
    orcs = [fxoracle.OracleCorrelator(j) for j in jobs]
    for sec, ns in SUBINTS:
        ins = [_inputs(j, k, sec, ns) for k, j in enumerate(jobs)]
        batch.submit(ins, sec, ns)
        for k in range(len(jobs)):
            refs[k] = orcs[k].process_subint(ins[k], sec, ns, coreresult=refs[k])
    batch.sync()
    for k, (job, m) in enumerate(zip(jobs, members)):
        got, layout, n = m.results(), m.layout(), m.corelen
        if xmac == "fp32":
            compare_core(job, layout, n, got, refs[k])
        else:
            assert_tc_gate(tc_errors(job, layout, n, got, refs[k]))
    batch.close()
    for m in members:
        m.close()


def test_member_refuses_its_own_submit_while_batched():
    from fxb200.native import FxbError
    jobs = _uneven_jobs()[:2]
    members = [Correlator(j, xmac="fp16") for j in jobs]
    batch = Batch(members)
    sec, ns = SUBINTS[0]
    with pytest.raises(FxbError):
        members[0].submit(_inputs(jobs[0], 0, sec, ns), sec, ns)
    batch.close()
    members[0].submit(_inputs(jobs[0], 0, sec, ns), sec, ns)      # free again once the batch is gone
    members[0].sync()
    for m in members:
        m.close()


@pytest.mark.parametrize("graphs", [True, False])
def test_kernel_timing_counts_every_subint(graphs):
    job = small_job(nstation=4, nchan=256, bw=16.0, nfreq=2, full_pol=True, subint_ns=SUBINT_NS)
    c = Correlator(job, xmac="fp16")
    c.set_graphs(graphs)
    c.timing_enable(True)
    for sec, ns in SUBINTS:
        c.submit(_inputs(job, 0, sec, ns), sec, ns)
    n, prep, fst, xm = c.timing_read()
    f_last, x_last, total = c.timing()
    c.close()
    assert n == len(SUBINTS)
    assert prep > 0 and fst > 0 and xm > 0
    assert 0 < f_last <= total and 0 < x_last <= total


def _many(job, k, c, n):
    for j in range(n):
        sec, ns = 0, (j + 1) * SUBINT_NS
        c.submit(_inputs(job, k, sec, ns), sec, ns)


@pytest.mark.parametrize("xmac", ["fp32", "fp16", "fp8"])
def test_autotuned_result_is_identical(xmac):
    # the tuner tries up to 9 candidates per round: 2 rounds take 18 subints
    job = small_job(nstation=4, nchan=256, bw=16.0, nfreq=2, full_pol=True, subint_ns=SUBINT_NS)
    plain = Correlator(job, xmac=xmac)
    _many(job, 0, plain, 20)
    ref = plain.results()
    plain.close()
    tuned = Correlator(job, xmac=xmac)
    tuned.autotune(2)
    _many(job, 0, tuned, 20)
    got = tuned.results()
    report = tuned.tuning_report()
    tuned.close()
    assert np.array_equal(got, ref)
    assert "fstage N=512" in report and " ms" in report
    if xmac != "fp32":
        assert "xmac group 0" in report and "rings" in report


def test_batch_autotune_keeps_results():
    jobs = _uneven_jobs()
    alone = []
    for k, j in enumerate(jobs):
        c = Correlator(j, xmac="fp16")
        _many(j, k, c, 20)
        alone.append(c.results())
        c.close()
    members = [Correlator(j, xmac="fp16") for j in jobs]
    batch = Batch(members)
    batch.autotune(2)
    for n in range(20):
        sec, ns = 0, (n + 1) * SUBINT_NS
        batch.submit([_inputs(j, k, sec, ns) for k, j in enumerate(jobs)], sec, ns)
    batch.sync()
    got = [m.results() for m in members]
    reports = [m.tuning_report() for m in members]
    batch.close()
    for m in members:
        m.close()
    for g, r in zip(got, alone):
        assert np.array_equal(g, r)
    assert all(" ms" in rp for rp in reports)


@pytest.mark.parametrize("xmac", ["fp32", "fp16"])
def test_batch_of_zoom_and_pcal_jobs_matches_each_alone(xmac):
    # zoom gather and phase-cal binning run inside the batch graph like the
    # other kernels: every member's result is bit-identical to its own run
    from helpers import PCAL_JOBS, zoom_job
    jobs = [zoom_job(), PCAL_JOBS["pcal_frac_lo"](), PCAL_JOBS["pcal_int_lo"]()]
    subs = [(0, 2_048_000 * (k + 1)) for k in range(3)]

    def inputs(k, job, sec, ns):
        return synth.subint_inputs(job, sec, ns, rho=0.05, seed=40 + k)

    alone = []
    for k, job in enumerate(jobs):
        c = Correlator(job, xmac=xmac)
        for sec, ns in subs:
            c.submit(inputs(k, job, sec, ns), sec, ns)
        alone.append(c.results())
        c.close()
    members = [Correlator(j, xmac=xmac) for j in jobs]
    batch = Batch(members)
    for sec, ns in subs:
        batch.submit([inputs(k, j, sec, ns) for k, j in enumerate(jobs)], sec, ns)
    batch.sync()
    got = [m.results() for m in members]
    batch.close()
    for m in members:
        m.close()
    for g, a in zip(got, alone):
        assert np.array_equal(g, a)
