"""GPU parity of the product path (libfxb200.so through the C ABI) against
the FP64 oracle restatement (oracle/fxoracle.c), on seeded synthetic VDIF.

Tolerances: cross- and auto-correlations within 1e-5 relative (2-norm over
the region, and max error within 1e-4 of the region's peak); per-FFT data
weights, baseline weights and autocorrelation weights bit-exact; layout,
channel order and sample selection exact.
"""
import numpy as np
import pytest

from fxb200 import synth
from fxb200.native import Correlator, job_layout
from helpers import FP32_TOL, compare_core, small_job

import fxoracle

pytestmark = pytest.mark.gpu


def run_both(job, subints, rho=0.05, seed=5, invalid=None, fill=None, validflags=None):
    corr = Correlator(job)
    orc = fxoracle.OracleCorrelator(job)
    ref = None
    for (sec, ns) in subints:
        inputs = synth.subint_inputs(job, sec, ns, rho=rho, seed=seed, invalid=invalid, fill=fill)
        corr.submit(inputs, sec, ns, validflags=validflags)
        ref = orc.process_subint(inputs, sec, ns, validflags=validflags, coreresult=ref)
    got = corr.results()
    w = corr.fft_weights()
    layout = corr.layout()
    assert np.array_equal(layout, orc.layout())
    corelen = corr.corelen
    corr.close()
    return got, ref, layout, corelen, w, orc.last_weights


def test_c0_parallel_hands_two_subints():
    job = small_job(nstation=4, full_pol=False)
    got, ref, layout, n, w, wref = run_both(job, [(0, 1_000_000), (0, 5_000_000)])
    errs = compare_core(job, layout, n, got, ref)
    assert np.array_equal(w, wref)
    assert errs["cross"] < FP32_TOL


def test_full_pol_cross_hand_autos():
    job = small_job(nstation=3, full_pol=True)
    got, ref, layout, n, w, wref = run_both(job, [(0, 2_000_000)])
    compare_core(job, layout, n, got, ref)
    assert np.array_equal(w, wref)


@pytest.mark.parametrize("order", [0, 1, 2])
def test_fringe_rotation_orders(order):
    job = small_job(nstation=3, full_pol=False, order=order, seed=3)
    got, ref, layout, n, w, wref = run_both(job, [(0, 1_000_000)])
    compare_core(job, layout, n, got, ref)


def test_lower_sideband_and_fractional_lo():
    job = small_job(nstation=3, full_pol=True, lsb=True, freq0=8400.25)
    got, ref, layout, n, w, wref = run_both(job, [(0, 1_000_000)])
    compare_core(job, layout, n, got, ref)


def test_invalid_frames_fill_and_flags():
    job = small_job(nstation=3, full_pol=False)
    sec, ns = 0, 1_000_000
    f0 = synth.subint_window(job, 0, sec, ns)[0]
    invalid = {0: [f0 + 2], 2: [f0 + 4, f0 + 5]}
    fill = {1: [f0 + 3]}
    vf = [synth.valid_flags(job) for _ in job.stations]
    vf[1] = synth.valid_flags(job, invalid_ffts=[0, 7, 31, 100])
    got, ref, layout, n, w, wref = run_both(job, [(sec, ns)], invalid=invalid, fill=fill, validflags=vf)
    compare_core(job, layout, n, got, ref)
    assert np.array_equal(w, wref)
    assert (w < 1.0).any() and (w == 0.0).any()


def test_eight_bit_blanking():
    job = small_job(nstation=3, full_pol=False, nbits=8)
    sec, ns = 0, 1_000_000
    f0 = synth.subint_window(job, 1, sec, ns)[0]
    got, ref, layout, n, w, wref = run_both(job, [(sec, ns)], invalid={1: [f0 + 1]})
    compare_core(job, layout, n, got, ref)
    assert np.array_equal(w, wref)


def test_data_before_buffer_start_is_zeroed():
    # subint at t=0: stations with positive delay need samples before the
    # first frame; Mode::process zeroes those FFTs (mode.cpp:703-716)
    job = small_job(nstation=4, full_pol=False)
    got, ref, layout, n, w, wref = run_both(job, [(0, 0)])
    compare_core(job, layout, n, got, ref)
    assert np.array_equal(w, wref)


def test_channel_averaging():
    job = small_job(nstation=3, full_pol=True, avg=4)
    got, ref, layout, n, w, wref = run_both(job, [(0, 1_000_000)])
    compare_core(job, layout, n, got, ref)


def test_sixteen_channel_vdif_1024_channels():
    # config-1 shape (16 VDIF channels = 8 x 32 MHz x 2 pol, 1024 channels),
    # 3 stations, one 2.048 ms subint
    job = small_job(nstation=3, nchan=1024, bw=32.0, nfreq=8, full_pol=True, subint_ns=2_048_000)
    got, ref, layout, n, w, wref = run_both(job, [(0, 1_024_000)], rho=0.02)
    compare_core(job, layout, n, got, ref)
    assert np.array_equal(w, wref)


def test_spectra_match_mode_process():
    job = small_job(nstation=2, full_pol=True)
    sec, ns = 0, 1_000_000
    inputs = synth.subint_inputs(job, sec, ns, rho=0.05, seed=9)
    corr = Correlator(job)
    corr.submit(inputs, sec, ns)
    spec = corr.spectra(0)                  # [t][row][chan]
    corr.close()
    orc = fxoracle.OracleCorrelator(job)
    for s in range(2):
        buf, dsec, dns = inputs[s]
        for t in (0, 1, 17, job.blocks_per_send() - 1):
            ref, wref, _ = orc.mode_fft(s, buf, dsec, dns, sec, ns, t)
            for b in range(job.stations[s].nband):
                g = spec[t, s * 2 + b]
                e = np.linalg.norm(g - ref[b]) / np.linalg.norm(ref[b])
                assert e < 2e-6, (s, t, b, e)


def test_layout_without_gpu_matches_context():
    job = small_job(nstation=5, full_pol=True, nfreq=2)
    lay, n = job_layout(job)
    corr = Correlator(job)
    assert np.array_equal(lay, corr.layout()) and n == corr.corelen
    corr.close()


@pytest.mark.parametrize("nchan", [2048, 4096, 8192])
def test_long_ffts(nchan):
    # 4096-, 8192- and 16384-point FFTs: several butterflies per thread, one
    # band per work item in the FP32 form
    job = small_job(nstation=3, nchan=nchan, bw=16.0, nfreq=2, full_pol=True, subint_ns=2_048_000)
    got, ref, layout, n, w, wref = run_both(job, [(0, 2_048_000), (0, 4_096_000)])
    compare_core(job, layout, n, got, ref)
    assert np.array_equal(w, wref)


@pytest.mark.parametrize("xmac", ["fp32", "fp16"])
def test_adjacent_station_buffers_give_the_same_result(xmac):
    # station buffers one after the other in one block take one copy per subint
    job = small_job(nstation=4, full_pol=True, nfreq=2)
    subs = [(0, 1_000_000), (0, 5_000_000)]
    res = []
    for adjacent in (False, True):
        corr = Correlator(job, xmac=xmac)
        for sec, ns in subs:
            inputs = synth.subint_inputs(job, sec, ns, rho=0.05, seed=13)
            if adjacent:
                blk = np.concatenate([b for b, _, _ in inputs])
                offs = np.cumsum([0] + [b.size for b, _, _ in inputs])
                assert all(o % 16 == 0 for o in offs)
                inputs = [(blk[offs[i]:offs[i + 1]], d, n) for i, (_, d, n) in enumerate(inputs)]
            corr.submit(inputs, sec, ns)
        res.append(corr.results())
        corr.close()
    assert np.array_equal(res[0], res[1])


@pytest.mark.parametrize("name,kw", [("order1", dict(order=1)), ("order0", dict(order=0)),
                                     ("order2", dict(order=2, seed=3)),
                                     ("lsb_fraclo", dict(order=1, lsb=True, freq0=8400.25)),
                                     ("clock_large", dict(order=1, looff=False, phase=False)),
                                     ("2048pt_8bands", dict(order=1, nchan=1024, bw=32.0, nfreq=4,
                                                            subint_ns=2_048_000))])
def test_band_corrections(name, kw):
    """Per-frequency clock offsets with R/L deltas, phase offsets and LO offsets
    (mode.cpp:870-1145, 1296-1347) on a subint 1.5 s into the job, against the
    oracle (itself pinned to the compiled reference on the same corrections)."""
    from helpers import corr_job
    job = corr_job(**kw)
    if name == "clock_large":
        # offsets of several microseconds: tens of turns across the band
        for st in job.stations:
            for f in st.freq_corr:
                clk, dclk, ph, lo = st.freq_corr[f]
                st.freq_corr[f] = (clk * 25.0, dclk, ph, lo)
    got, ref, layout, n, w, wref = run_both(job, [(1, 500_000_000)])
    compare_core(job, layout, n, got, ref)
    assert np.array_equal(w, wref)


@pytest.mark.parametrize("kw", [dict(), dict(lsb=True), dict(nbits=8, nfreq=1), dict(order=2),
                                dict(nchan=1024, bw=32.0, subint_ns=2_048_000)])
def test_complex_sampling(kw):
    """Single-sideband complex sampling (nchan-point complex FFTs, VDIFC
    decoding), with an invalid frame (the complex 8-bit decoders stop
    advancing in it; the first frame of a complex unpack is checked for fill
    pattern only), against the oracle pinned to the compiled reference."""
    from helpers import cplx_job
    job = cplx_job(**kw)
    sec, ns = 1, 500_000_000
    f0 = synth.subint_window(job, 0, sec, ns)[0]
    got, ref, layout, n, w, wref = run_both(job, [(sec, ns)], invalid={0: [f0 + 2]})
    compare_core(job, layout, n, got, ref)
    assert np.array_equal(w, wref)
