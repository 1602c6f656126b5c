"""Tensor-core forms against the FP64 oracle.

The headline tensor-core form keeps the F stage's spectra in FP16 (11-bit
significands, ~2^-12 relative rounding per value) and accumulates in FP32.
Its gate is the stated relative visibility tolerance of the tensor-core form, 1e-3
(``helpers.TC_REL_TOL``): norm-wise over the cross and autocorrelations and
as the rms of the per-visibility relative amplitude and phase errors.  BF16
spectra (8-bit significands) are kept as a measured alternative: a value's
rounding is ~8 times coarser, so they are held to correlation-coefficient
units (the error of V_ab over sqrt(A_aa A_bb)), not to the relative gate.
Weights and layout are exact in every form."""
import numpy as np
import pytest

from fxb200 import configs, synth
from fxb200.native import Correlator
from helpers import assert_tc_gate, regions, rel_err, small_job, vis_errors

import fxoracle

pytestmark = pytest.mark.gpu

BF16_CCU_TOL = 1e-3


def run_tc(job, subints, rho=0.05, seed=5, xmac="fp16"):
    corr = Correlator(job, xmac=xmac)
    orc = fxoracle.OracleCorrelator(job)
    ref = None
    for (sec, ns) in subints:
        inputs = synth.subint_inputs(job, sec, ns, rho=rho, seed=seed)
        corr.submit(inputs, sec, ns)
        ref = orc.process_subint(inputs, sec, ns, coreresult=ref)
    got = corr.results()
    layout = corr.layout()
    n = corr.corelen
    corr.close()
    return got, ref, layout, n


def tc_errors(job, layout, n, got, ref):
    reg = dict(regions(job, layout, n))
    for name in ("bweight", "acweight"):
        assert np.array_equal(got[reg[name]].astype(np.float32), ref[reg[name]].astype(np.float32)), name
    return vis_errors(job, layout, n, got, ref)


@pytest.mark.parametrize("kw", [dict(nstation=4, full_pol=True),
                                dict(nstation=10, full_pol=True, nchan=256),
                                dict(nstation=3, nchan=1024, bw=32.0, nfreq=8, full_pol=True, subint_ns=2_048_000),
                                dict(nstation=4, nchan=512, bw=16.0, nfreq=2, full_pol=True, nbits=8,
                                     subint_ns=2_048_000),
                                # one band per work item (the one-band persistent F kernel)
                                dict(nstation=4, nchan=256, bw=16.0, nfreq=2, full_pol=False)])
def test_fp16_tensor_core_vs_fp64(kw):
    job = small_job(**kw)
    got, ref, layout, n = run_tc(job, [(0, 1_024_000), (0, 3_072_000)])
    e = tc_errors(job, layout, n, got, ref)
    print(kw, e)
    assert_tc_gate(e)


def test_fp16_c1_ten_stations_vs_fp64():
    """The c1 shape (10 stations, eight 32 MHz subbands, 1024 channels, full
    cross hands), two 2.048 ms subints."""
    job = configs.c1(subint_ns=2_048_000)
    got, ref, layout, n = run_tc(job, [(0, 0), (0, 2_048_000)], rho=0.01, seed=21)
    e = tc_errors(job, layout, n, got, ref)
    print(e)
    assert_tc_gate(e)


@pytest.mark.parametrize("bw,nchan,nbits", [(16.0, 1024, 8), (64.0, 4096, 2), (4.0, 128, 8)])
def test_fp16_c3_shapes_twenty_stations_vs_fp64(bw, nchan, nbits):
    """Subband shapes of the c3 batch (widths 4..64 MHz, 128..4096 channels,
    2- and 8-bit samples) at its 20 stations, one 8.192 ms subint."""
    job = small_job(nstation=20, nchan=nchan, bw=bw, nfreq=1, full_pol=True, nbits=nbits, subint_ns=8_192_000)
    got, ref, layout, n = run_tc(job, [(0, 0)], rho=0.01, seed=23)
    e = tc_errors(job, layout, n, got, ref)
    print(bw, nchan, nbits, e)
    assert_tc_gate(e)


@pytest.mark.parametrize("kw", [dict(nstation=4, full_pol=True),
                                dict(nstation=3, nchan=1024, bw=32.0, nfreq=8, full_pol=True, subint_ns=2_048_000)])
def test_bf16_tensor_core_vs_fp64(kw):
    job = small_job(**kw)
    got, ref, layout, n = run_tc(job, [(0, 1_024_000), (0, 3_072_000)], xmac="bf16")
    e = tc_errors(job, layout, n, got, ref)
    assert e["ccu"] <= BF16_CCU_TOL, e
    assert e["auto_rel"] <= 1e-3, e


@pytest.mark.parametrize("xmac,tol", [("fp16", 2e-3), ("bf16", 8e-3)])
def test_tc_spectra_readback_matches_oracle(xmac, tol):
    job = small_job(nstation=2, full_pol=True)
    sec, ns = 0, 1_000_000
    inputs = synth.subint_inputs(job, sec, ns, rho=0.05, seed=9)
    corr = Correlator(job, xmac=xmac)
    corr.submit(inputs, sec, ns)
    spec = corr.spectra(0)
    corr.close()
    orc = fxoracle.OracleCorrelator(job)
    buf, dsec, dns = inputs[0]
    for t in (0, 5, 100):
        ref, _, _ = orc.mode_fft(0, buf, dsec, dns, sec, ns, t)
        for b in range(2):
            assert rel_err(spec[t, b], ref[b]) < tol


def _tc_fft_job(lsb=False, order=1, nfreq=2, nstation=3):
    # 1024 channels -> 2048-point FFTs of 2-bit samples: the F stage runs its
    # FFT on the tensor cores (the default where the layout allows it)
    return small_job(nstation=nstation, nchan=1024, bw=32.0, nfreq=nfreq, full_pol=True, subint_ns=2_048_000, lsb=lsb,
                     order=order)


@pytest.mark.parametrize("lsb,order,nfreq", [(False, 1, 2), (True, 1, 2), (False, 0, 2), (False, 1, 1),
                                              (False, 1, 8), (False, 1, 16)])
def test_tensor_core_fft_spectra_match_oracle(lsb, order, nfreq):
    """Spectra of the tensor-core FFT (FP16 operands, FP32 accumulation, FP16
    out) against the FP64 oracle's Mode FFT output: both sidebands, fringe
    rotation orders 0 and 1, stations of 2 to 32 bands (4 to 64 bits per
    time; one subband leaves a work unit with one subband)."""
    job = _tc_fft_job(lsb=lsb, order=order, nfreq=nfreq, nstation=2 if nfreq > 8 else 3)
    sec, ns = 0, 1_024_000
    inputs = synth.subint_inputs(job, sec, ns, rho=0.05, seed=11)
    corr = Correlator(job, xmac="fp16")
    corr.submit(inputs, sec, ns)
    spec = corr.spectra(0)
    corr.close()
    orc = fxoracle.OracleCorrelator(job)
    buf, dsec, dns = inputs[0]
    for t in (0, 7, 31):
        ref, _, _ = orc.mode_fft(0, buf, dsec, dns, sec, ns, t)
        for b in range(2):
            assert rel_err(spec[t, b], ref[b]) < 6e-4, (t, b)


def test_tensor_core_fft_matches_cuda_core_fstage(monkeypatch):
    """The same subints through the tensor-core FFT (the default) and through
    the CUDA-core FP32 F stage (FXB_TC_FFT=0): both within the tensor-core
    relative tolerance of the FP64 oracle and of each other."""
    job = _tc_fft_job()
    subints = [(0, 1_024_000), (0, 3_072_000)]
    got_tc, ref, layout, n = run_tc(job, subints)
    monkeypatch.setenv("FXB_TC_FFT", "0")
    got_cc, _, _, _ = run_tc(job, subints)
    for got in (got_tc, got_cc):
        assert_tc_gate(tc_errors(job, layout, n, got, ref))
    reg = dict(regions(job, layout, n))
    assert rel_err(got_tc[reg["auto"]], got_cc[reg["auto"]]) < 2e-3


# FP8 e4m3 keeps 3 mantissa bits: a value's rounding error is ~3.6 % rms, so a
# visibility averaged over N products carries ~sqrt(2) * 0.036 / sqrt(N) in
# correlation-coefficient units.  Gate: well inside that for the test sizes,
# and far below what a wrong scale or layout would give (order 1).
FP8_TOL = 2e-2


@pytest.mark.parametrize("kw", [dict(nstation=4, full_pol=True),
                                dict(nstation=5, nchan=512, bw=32.0, nfreq=2, full_pol=True, subint_ns=2_048_000),
                                dict(nstation=10, full_pol=True, nchan=256)])
def test_fp8_tensor_core_vs_fp64(kw):
    job = small_job(**kw)
    got, ref, layout, n = run_tc(job, [(0, 1_024_000), (0, 3_072_000)], xmac="fp8")
    e = tc_errors(job, layout, n, got, ref)
    assert e["ccu"] <= FP8_TOL, e
    assert e["auto_rel"] <= FP8_TOL, e


@pytest.mark.parametrize("nchan", [2048, 4096, 8192])
def test_fp16_long_ffts_vs_fp64(nchan):
    # 4096..16384-point FFTs: the longest transforms of the serving workload
    job = small_job(nstation=3, nchan=nchan, bw=16.0, nfreq=2, full_pol=True, subint_ns=8_192_000)
    got, ref, layout, n = run_tc(job, [(0, 8_192_000), (0, 16_384_000)])
    e = tc_errors(job, layout, n, got, ref)
    print(nchan, e)
    assert_tc_gate(e)


@pytest.mark.parametrize("kw", [dict(order=1, nchan=1024, bw=32.0, nfreq=4, subint_ns=2_048_000),
                                dict(order=0, nchan=1024, bw=32.0, nfreq=2, subint_ns=2_048_000),
                                dict(order=1, nchan=256),
                                dict(order=2, nchan=512, seed=3)])
def test_fp16_band_corrections_vs_fp64(kw):
    """Clock, phase and LO offsets in the tensor-core form: the 2048-point
    kinds run the tensor-core FFT (k_fstage_tc), the others the CUDA-core F
    stage with FP16 output; both within the relative gate."""
    from helpers import corr_job
    job = corr_job(**kw)
    got, ref, layout, n = run_tc(job, [(1, 500_000_000), (1, 502_048_000 if kw.get("subint_ns") else 504_000_000)])
    e = tc_errors(job, layout, n, got, ref)
    print(kw, e)
    assert_tc_gate(e)


@pytest.mark.parametrize("kw", [dict(), dict(lsb=True, nbits=8, nfreq=1)])
def test_fp16_complex_sampling_vs_fp64(kw):
    """Complex-sampled stations in the tensor-core form (CUDA-core complex FFT,
    FP16 spectra) within the relative gate."""
    from helpers import cplx_job
    job = cplx_job(**kw)
    got, ref, layout, n = run_tc(job, [(0, 1_000_000), (0, 5_000_000)])
    e = tc_errors(job, layout, n, got, ref)
    print(kw, e)
    assert_tc_gate(e)
