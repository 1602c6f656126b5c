"""Tensor-core (BF16 tcgen05) form against the FP64 oracle.

BF16 spectra carry ~2^-9 relative rounding per value, so a noise-dominated
cross-correlation differs from the FP64 result by ~1e-3 of its own (noise)
amplitude.  The meaningful error of a correlator output is in correlation-
coefficient units: the error of V_ab relative to sqrt(A_aa A_bb), the
autocorrelation scale.  Gates: cross-correlation error <= 1e-3 in those units,
autocorrelations within 1e-3 relative, weights and layout exact."""
import numpy as np
import pytest

from fxb200 import synth
from fxb200.native import Correlator
from helpers import regions, rel_err, small_job

import fxoracle

pytestmark = pytest.mark.gpu

TC_TOL = 1e-3


def run_tc(job, subints, rho=0.05, seed=5, xmac="bf16"):
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
    xc, ac = reg["cross"], reg["auto"]
    # correlation-coefficient units: cross error over the autocorrelation scale
    auto_rms = np.sqrt(np.mean(ref[ac][0::2] ** 2))
    cross_err = np.sqrt(np.mean((got[xc] - ref[xc]) ** 2)) / auto_rms
    auto_err = rel_err(got[ac], ref[ac])
    for name in ("bweight", "acweight"):
        assert np.array_equal(got[reg[name]].astype(np.float32), ref[reg[name]].astype(np.float32)), name
    return cross_err, auto_err


@pytest.mark.parametrize("kw", [dict(nstation=4, full_pol=True),
                                dict(nstation=10, full_pol=True, nchan=256),
                                dict(nstation=3, nchan=1024, bw=32.0, nfreq=8, full_pol=True, subint_ns=2_048_000)])
def test_bf16_tensor_core_vs_fp64(kw):
    job = small_job(**kw)
    got, ref, layout, n = run_tc(job, [(0, 1_024_000), (0, 3_072_000)])
    cross_err, auto_err = tc_errors(job, layout, n, got, ref)
    assert cross_err <= TC_TOL, cross_err
    assert auto_err <= TC_TOL, auto_err


def test_bf16_spectra_readback_matches_oracle():
    job = small_job(nstation=2, full_pol=True)
    sec, ns = 0, 1_000_000
    inputs = synth.subint_inputs(job, sec, ns, rho=0.05, seed=9)
    corr = Correlator(job, xmac="bf16")
    corr.submit(inputs, sec, ns)
    spec = corr.spectra(0)
    corr.close()
    orc = fxoracle.OracleCorrelator(job)
    buf, dsec, dns = inputs[0]
    for t in (0, 5, 100):
        ref, _, _ = orc.mode_fft(0, buf, dsec, dns, sec, ns, t)
        for b in range(2):
            assert rel_err(spec[t, b], ref[b]) < 8e-3


def _tc_fft_job(lsb=False, order=1):
    # 1024 channels -> 2048-point FFTs: the F stage runs its FFT on the tensor cores
    return small_job(nstation=3, nchan=1024, bw=32.0, nfreq=2, full_pol=True, subint_ns=2_048_000, lsb=lsb, order=order)


@pytest.mark.parametrize("lsb,order", [(False, 1), (True, 1), (False, 0)])
def test_tensor_core_fft_spectra_match_oracle(lsb, order, monkeypatch):
    """Spectra of the tensor-core FFT (FXB_TC_FFT=1: FP16 operands, FP32
    accumulation, BF16 out) against the FP64 oracle's Mode FFT output, both
    sidebands."""
    monkeypatch.setenv("FXB_TC_FFT", "1")
    job = _tc_fft_job(lsb=lsb, order=order)
    sec, ns = 0, 1_024_000
    inputs = synth.subint_inputs(job, sec, ns, rho=0.05, seed=11)
    corr = Correlator(job, xmac="bf16")
    corr.submit(inputs, sec, ns)
    spec = corr.spectra(0)
    corr.close()
    orc = fxoracle.OracleCorrelator(job)
    buf, dsec, dns = inputs[0]
    for t in (0, 7, 31):
        ref, _, _ = orc.mode_fft(0, buf, dsec, dns, sec, ns, t)
        for b in range(2):
            assert rel_err(spec[t, b], ref[b]) < 8e-3, (t, b)


def test_tensor_core_fft_matches_cuda_core_fstage(monkeypatch):
    """The same subints through the tensor-core FFT (FXB_TC_FFT=1) and through
    the default CUDA-core FP16 F stage: both within the tensor-core tolerance
    of the FP64 oracle and of each other."""
    job = _tc_fft_job()
    subints = [(0, 1_024_000), (0, 3_072_000)]
    got_cc, ref, layout, n = run_tc(job, subints)
    monkeypatch.setenv("FXB_TC_FFT", "1")
    got_tc, _, _, _ = run_tc(job, subints)
    for got in (got_tc, got_cc):
        cross_err, auto_err = tc_errors(job, layout, n, got, ref)
        assert cross_err <= TC_TOL, cross_err
        assert auto_err <= TC_TOL, auto_err
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
    cross_err, auto_err = tc_errors(job, layout, n, got, ref)
    assert cross_err <= FP8_TOL, cross_err
    assert auto_err <= FP8_TOL, auto_err


@pytest.mark.parametrize("nchan", [2048, 4096, 8192])
def test_bf16_long_ffts_vs_fp64(nchan):
    # the FP16 FFT's rounding over 12..14 radix stages averages down with the
    # number of FFTs integrated: 8.192 ms subints give 8..32 per subint (a 1 s
    # integration has 60..250 times more)
    job = small_job(nstation=3, nchan=nchan, bw=16.0, nfreq=2, full_pol=True, subint_ns=8_192_000)
    got, ref, layout, n = run_tc(job, [(0, 8_192_000), (0, 16_384_000)])
    cross_err, auto_err = tc_errors(job, layout, n, got, ref)
    assert cross_err <= TC_TOL, cross_err
    assert auto_err <= TC_TOL, auto_err
