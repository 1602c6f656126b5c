"""Pins the oracle restatement to the reference's own compiled CPU code
(oracle/_ref, built from the reference sources by oracle/Makefile.ref):
layout, delay interpolator and data weights exact, VDIF decoding bit-exact
against mark5access, spectra and core results within the FP32 rounding of
the reference.  Skipped where the reference build is absent."""
import numpy as np
import pytest

from fxb200 import synth
from helpers import (PCAL_JOBS, compare_core, edv4_inputs, mixed_bw_zoom_job, mux_job, regions, rel_err, small_job,
                     zoom_job)

import fxoracle
import refcorr

pytestmark = pytest.mark.skipif(not refcorr.available(), reason="reference build oracle/_ref absent")

JOBS = {
    "c0": dict(nstation=4),
    "fullpol": dict(nstation=3, full_pol=True),
    "order0": dict(nstation=3, order=0),
    "order2": dict(nstation=3, order=2, seed=3),
    "lsb_fraclo": dict(nstation=3, full_pol=True, lsb=True, freq0=8400.25),
    "8bit": dict(nstation=3, nbits=8),
    "avg4": dict(nstation=3, full_pol=True, avg=4),
    "16ch_1024": dict(nstation=3, nchan=1024, bw=32.0, nfreq=8, full_pol=True, subint_ns=2_048_000),
}


@pytest.mark.parametrize("name", sorted(JOBS))
def test_subint_matches_reference(name):
    job = small_job(**JOBS[name])
    ref = refcorr.RefCorrelator(job)
    orc = fxoracle.OracleCorrelator(job)
    assert np.array_equal(ref.layout(), orc.layout())
    sec, ns = 0, 1_024_000
    f0 = synth.subint_window(job, 0, sec, ns)[0]
    invalid = {0: [f0 + 1]} if name in ("c0", "8bit") else None
    inputs = synth.subint_inputs(job, sec, ns, rho=0.05, seed=7, invalid=invalid)
    vf = [synth.valid_flags(job) for _ in job.stations]
    r = ref.process_subint(inputs, vf, 0, sec, ns)
    o = orc.process_subint(inputs, sec, ns, validflags=vf)
    for s in range(len(job.stations)):
        assert np.array_equal(ref.interpolator(s, sec, ns), orc.interpolator(s, sec, ns))
    compare_core(job, orc.layout(), orc.corelen, r.astype(np.float64), o, tol=2e-6)


ZOOM_JOBS = {
    "zoom": lambda: zoom_job(),
    "zoom_only": lambda: zoom_job(keep_parents=False),
    "zoom_avg4": lambda: zoom_job(avg=4),
    "zoom_mixed_bw": lambda: mixed_bw_zoom_job(),
}


@pytest.mark.parametrize("name", sorted(ZOOM_JOBS))
def test_zoom_subint_matches_reference(name):
    # zoom bands: windows of recorded bands correlated as frequencies of their
    # own, with or without their parents, averaged, and across stations that
    # record different bandwidths (mode.cpp:169-208, core.cpp:1266-1363)
    job = ZOOM_JOBS[name]()
    ref = refcorr.RefCorrelator(job)
    orc = fxoracle.OracleCorrelator(job)
    assert np.array_equal(ref.layout(), orc.layout())
    sec, ns = 0, 1_024_000
    inputs = synth.subint_inputs(job, sec, ns, rho=0.05, seed=7)
    vf = [synth.valid_flags(job) for _ in job.stations]
    r = ref.process_subint(inputs, vf, 0, sec, ns)
    o = orc.process_subint(inputs, sec, ns, validflags=vf)
    compare_core(job, orc.layout(), orc.corelen, r.astype(np.float64), o, tol=2e-6)


@pytest.mark.parametrize("name", sorted(PCAL_JOBS))
def test_pcal_subint_matches_reference(name):
    # phase-cal tones of the implicit-shift extractor (pcal.cpp:927-1105) and
    # of bands without a tone, copied band by band (core.cpp:1124-1150)
    job = PCAL_JOBS[name]()
    ref = refcorr.RefCorrelator(job)
    orc = fxoracle.OracleCorrelator(job)
    assert np.array_equal(ref.layout(), orc.layout())
    sec, ns = 0, 1_024_000
    inputs = synth.subint_inputs(job, sec, ns, rho=0.05, seed=7)
    vf = [synth.valid_flags(job) for _ in job.stations]
    r = ref.process_subint(inputs, vf, 0, sec, ns)
    o = orc.process_subint(inputs, sec, ns, validflags=vf)
    errs = compare_core(job, orc.layout(), orc.corelen, r.astype(np.float64), o, tol=2e-6)
    assert "pcal" in errs


@pytest.mark.parametrize("masklength", [4, 2])
def test_interlaced_vdif_per_band_weights_match_reference(masklength):
    # INTERLACEDVDIF stations: per-band data weights (mk5mode.cpp:145-166) from
    # the frames' EDV4 validity masks (format_vdif.c:4699-4780), baseline and
    # autocorrelation weights from them (core.cpp:1032, mode.cpp:1300-1303); one station also has invalid frames.
    job = mux_job(masklength=masklength)
    ref = refcorr.RefCorrelator(job)
    orc = fxoracle.OracleCorrelator(job)
    assert np.array_equal(ref.layout(), orc.layout())
    sec, ns = 0, 1_024_000
    f0 = synth.subint_window(job, 0, sec, ns)[0]
    inputs = edv4_inputs(job, synth.subint_inputs(job, sec, ns, rho=0.05, seed=7, invalid={0: [f0 + 2, f0 + 9]}))
    vf = [synth.valid_flags(job) for _ in job.stations]
    r = ref.process_subint(inputs, vf, 0, sec, ns)
    o = orc.process_subint(inputs, sec, ns, validflags=vf)
    reg = dict(regions(job, orc.layout(), orc.corelen))
    for name in ("bweight", "acweight"):
        assert np.array_equal(o[reg[name]].astype(np.float32), r[reg[name]]), name
    plain = fxoracle.OracleCorrelator(job_without_mux(job)).process_subint(inputs, sec, ns, validflags=vf)
    assert not np.array_equal(o[reg["acweight"]], plain[reg["acweight"]])
    compare_core(job, orc.layout(), orc.corelen, r.astype(np.float64), o, tol=2e-6)


def test_interlaced_vdif_full_masks_match_reference():
    # EDV4 headers whose masks keep every band: the whole subint as the reference's
    job = mux_job()
    ref = refcorr.RefCorrelator(job)
    orc = fxoracle.OracleCorrelator(job)
    sec, ns = 0, 1_024_000
    inputs = edv4_inputs(job, synth.subint_inputs(job, sec, ns, rho=0.05, seed=7))
    for s in (0, 2):
        inputs[s][0].reshape(-1, job.frame_bytes(s))[:, 24:32] = np.frombuffer(np.uint64(15).tobytes(), np.uint8)
    vf = [synth.valid_flags(job) for _ in job.stations]
    r = ref.process_subint(inputs, vf, 0, sec, ns)
    o = orc.process_subint(inputs, sec, ns, validflags=vf)
    compare_core(job, orc.layout(), orc.corelen, r.astype(np.float64), o, tol=2e-6)


def job_without_mux(job):
    import copy
    j = copy.deepcopy(job)
    for st in j.stations:
        st.mux_threads = 0
    return j


def test_mode_spectra_match_reference():
    job = small_job(nstation=2, full_pol=True)
    ref = refcorr.RefCorrelator(job)
    orc = fxoracle.OracleCorrelator(job)
    sec, ns = 0, 1_000_000
    inputs = synth.subint_inputs(job, sec, ns, rho=0.05, seed=9)
    vf = synth.valid_flags(job)
    for s in range(2):
        buf, dsec, dns = inputs[s]
        for t in (0, 3, 100, job.blocks_per_send() - 1):
            rs, rw, _ = ref.mode_fft(s, buf, dsec, dns, vf, sec, ns, t)
            os_, ow, _ = orc.mode_fft(s, buf, dsec, dns, sec, ns, t, validflags=vf)
            assert rw == ow
            assert rel_err(os_, rs) < 1e-6


@pytest.mark.parametrize("nchan,nbits", [(1, 2), (2, 2), (4, 2), (8, 2), (16, 2), (32, 2), (64, 2),
                                         (1, 8), (2, 8), (4, 8)])
def test_vdif_decode_matches_mark5access(nchan, nbits):
    from fxb200.job import Freq, Job, Station
    st = Station("A", [(0, "R")] * nchan, nbits=nbits, payload_bytes=1024)
    job = Job([Freq(1000.0, 1.024, 16)], [st], [], subint_ns=62_500)
    synth.make_delay_polys(job, 1)
    fs = job.frame_samples(0)
    data = synth.gen_station_frames(job, 0, 0, 8, rho=0.1, seed=nchan + nbits, invalid=[3], fill=[5])
    fmt = "VDIF_1024-%d-%d-%d" % (job.mbps(0), nchan, nbits)
    for off, n in [(0, fs), (fs - 3, 10), (2 * fs + 1, fs + 5), (3 * fs - 7, 2 * fs)]:
        gran = max(1, 8 // (nchan * nbits))
        off -= off % gran
        n -= n % gran
        r, rgood = refcorr.unpack(fmt, data, off, n, nchan)
        o, ogood = fxoracle.vdif_unpack(data, 1024, 32, nchan, nbits, off, n)
        assert rgood == ogood, (off, n, rgood, ogood)
        assert np.array_equal(r, o), (off, n)


CORR_JOBS = {
    "corr_order1": dict(order=1),
    "corr_order0": dict(order=0),
    "corr_order2": dict(order=2, seed=3),
    "corr_lsb_fraclo": dict(order=1, lsb=True, freq0=8400.25),
    "corr_looff_only": dict(order=1, clock=False, delta=False, phase=False),
    "corr_clock_only_8bit": dict(order=1, looff=False, phase=False, delta=False, nbits=8),
}


@pytest.mark.parametrize("name", sorted(CORR_JOBS))
def test_corrections_subint_matches_reference(name):
    # per-frequency clock offsets and R/L deltas in the fractional-sample
    # rotation, LO offsets in the fringe rotation and phase offsets of the
    # non-R band (mode.cpp:870-1145, 1296-1347, 435-460), on a subint that
    # starts 1.5 s into the job so that the wall-clock terms matter
    from helpers import corr_job
    job = corr_job(**CORR_JOBS[name])
    ref = refcorr.RefCorrelator(job)
    orc = fxoracle.OracleCorrelator(job)
    sec, ns = 1, 500_000_000
    inputs = synth.subint_inputs(job, sec, ns, rho=0.05, seed=17)
    vf = [synth.valid_flags(job) for _ in job.stations]
    r = ref.process_subint(inputs, vf, 0, sec, ns)
    o = orc.process_subint(inputs, sec, ns, validflags=vf)
    compare_core(job, orc.layout(), orc.corelen, r.astype(np.float64), o, tol=2e-6)


CPLX_JOBS = {
    "cplx_usb": dict(),
    "cplx_lsb": dict(lsb=True),
    "cplx_8bit_invalid": dict(nbits=8, nfreq=1),
    "cplx_order2": dict(order=2),
    "cplx_4band_1024": dict(nfreq=2, nchan=1024, bw=32.0, subint_ns=2_048_000),
}


@pytest.mark.parametrize("name", sorted(CPLX_JOBS))
def test_complex_sampling_matches_reference(name):
    # single-sideband complex sampling (mode.cpp:51-59, 889-905, 1182-1234;
    # VDIFC decoders format_vdif.c:2369-2955), with an invalid frame (the
    # complex 8-bit decoders stop advancing in it) and per-frequency
    # corrections on a subint 1.5 s in
    from helpers import cplx_job
    job = cplx_job(**CPLX_JOBS[name])
    rng = np.random.default_rng(5)
    for st in job.stations[1:]:
        for f in st.recorded_freqs():
            st.freq_corr[f] = (float(rng.uniform(-0.1, 0.1)), 0.0, float(rng.uniform(-30, 30)),
                               float(rng.uniform(-900, 900)))
    ref = refcorr.RefCorrelator(job)
    orc = fxoracle.OracleCorrelator(job)
    assert np.array_equal(ref.layout(), orc.layout())
    sec, ns = 1, 500_000_000
    f0 = synth.subint_window(job, 0, sec, ns)[0]
    inputs = synth.subint_inputs(job, sec, ns, rho=0.05, seed=7, invalid={0: [f0 + 2]})
    vf = [synth.valid_flags(job) for _ in job.stations]
    r = ref.process_subint(inputs, vf, 0, sec, ns)
    o = orc.process_subint(inputs, sec, ns, validflags=vf)
    compare_core(job, orc.layout(), orc.corelen, r.astype(np.float64), o, tol=2e-6)
