"""The Configuration -> fxb200 adapter (oracle/fxb_config_adapter.cpp), the
code an integration into mpifxcorr compiles beside Core.

It parses nothing itself: the stock Configuration reads the generated
.input/.calc/.im, fxb_desc_from_configuration maps the parsed tables (and,
through the datastreams' Modes, the per-frequency corrections and the
fringe-rotation order) onto an fxb_job_desc, and fxb_interpolators_from_model
asks the stock Model for each subint's delay interpolators as
Mode::setOffsets does.

CPU: the adapter's descriptor equals the one the job model describes, field
by field, its core-result layout (computed by the product library, no GPU)
equals the reference's, and its interpolators equal the reference Mode's.
GPU: the whole flow (descriptor -> fxb_create -> fxb_submit_subint_interp
per subint -> fxb_read_results) run by the harness in C++ against the
product library gives the reference's core result within 1e-5."""
import ctypes

import numpy as np
import pytest

from fxb200 import native, synth
from helpers import FP32_TOL, compare_core, corr_job, cplx_job, pcal_job, small_job, zoom_job

import refcorr

pytestmark = pytest.mark.skipif(not refcorr.available(), reason="reference build oracle/_ref absent")

JOBS = {
    "c0": lambda: small_job(nstation=4),
    "corrections_order1": lambda: corr_job(order=1),
    "corrections_order0_lsb": lambda: corr_job(order=0, lsb=True, freq0=8400.25),
    "zoom": lambda: zoom_job(),
    "pcal": lambda: pcal_job(),
    "8bit_order2": lambda: small_job(nstation=3, nbits=8, order=2, seed=3),
    "complex_lsb": lambda: cplx_job(lsb=True),
}


def _adapter_desc(ref):
    return ctypes.cast(ref.fxb_desc_address(), ctypes.POINTER(native.FxbJobDesc)).contents


def _arr(p, n, zero=0):
    return [p[i] for i in range(n)] if p else [zero] * n


@pytest.mark.parametrize("name", sorted(JOBS))
def test_adapter_descriptor_matches_job(name):
    job = JOBS[name]()
    ref = refcorr.RefCorrelator(job)
    got = _adapter_desc(ref)
    want = native.DescHolder(job).desc
    for k in ("nfreq", "nstation", "nbaseline", "subint_ns", "fringe_rot_order", "write_autocorrs"):
        assert getattr(got, k) == getattr(want, k), k
    for f in range(want.nfreq):
        a, b = got.freqs[f], want.freqs[f]
        assert (a.freq_mhz, a.bw_mhz, a.nchan, a.lower_sideband, a.chans_to_avg) == \
               (b.freq_mhz, b.bw_mhz, b.nchan, b.lower_sideband, b.chans_to_avg), f
    for s in range(want.nstation):
        a, b = got.stations[s], want.stations[s]
        for k in ("nbits", "payload_bytes", "header_bytes", "nband", "nzoom", "mux_threads", "complex_sampling"):
            assert getattr(a, k) == getattr(b, k), (s, k)
        assert (np.float32(a.pcal_interval_mhz), np.float32(a.pcal_base_mhz)) == \
               (np.float32(b.pcal_interval_mhz), np.float32(b.pcal_base_mhz))
        assert _arr(a.band_freq, b.nband) == _arr(b.band_freq, b.nband)
        assert a.band_pol[:b.nband] == b.band_pol[:b.nband]
        assert _arr(a.zoom_freq, b.nzoom) == _arr(b.zoom_freq, b.nzoom)
        if b.nzoom:
            assert a.zoom_pol[:b.nzoom] == b.zoom_pol[:b.nzoom]
        for k in ("band_clock_us", "band_clock_delta_us", "band_phase_deg", "band_lo_offset_hz"):
            # the .input carries the values to 9 decimals
            assert np.allclose(_arr(getattr(a, k), b.nband, 0.0), _arr(getattr(b, k), b.nband, 0.0),
                               rtol=0, atol=1e-9), (s, k)
    for i in range(want.nbaseline):
        a, b = got.baselines[i], want.baselines[i]
        assert (a.ds1, a.ds2, a.nprod) == (b.ds1, b.ds2, b.nprod), i
        for k in ("prod_freq", "prod_band1", "prod_band2"):
            assert _arr(getattr(a, k), b.nprod) == _arr(getattr(b, k), b.nprod), (i, k)


@pytest.mark.parametrize("name", sorted(JOBS))
def test_adapter_layout_and_interpolators_match_reference(name):
    job = JOBS[name]()
    ref = refcorr.RefCorrelator(job)
    got = _adapter_desc(ref)
    nf, nb, ns = got.nfreq, got.nbaseline, got.nstation
    out = np.zeros(2 * nf * nb + 3 * ns, dtype=np.int32)
    n = ctypes.c_int64(0)
    native.check(native.lib().fxb_job_layout(ctypes.byref(got), out.ctypes.data_as(ctypes.POINTER(ctypes.c_int32)),
                                             out.size, ctypes.byref(n)), None, "job_layout")
    assert n.value == ref.corelen
    assert np.array_equal(out, ref.layout())
    for sec, nsec in ((0, 0), (0, 4_000_000), (1, 500_000_000)):
        interp, missing = ref.fxb_interpolators(0, sec, nsec)
        assert missing == 0
        for s in range(ns):
            assert np.array_equal(interp[s], ref.interpolator(s, sec, nsec))


@pytest.mark.gpu
@pytest.mark.parametrize("name", ["c0", "corrections_order1", "zoom", "pcal", "complex_lsb"])
def test_adapter_flow_through_product_matches_reference(name):
    job = JOBS[name]()
    ref = refcorr.RefCorrelator(job)
    subints = []
    want = None
    vf = [synth.valid_flags(job) for _ in job.stations]
    for k, (sec, ns) in enumerate(((0, 4_000_000), (1, 500_000_000))):
        inputs = synth.subint_inputs(job, sec, ns, rho=0.05, seed=31 + k)
        subints.append((inputs, sec, ns))
        r = ref.process_subint(inputs, vf, 0, sec, ns)
        want = r.astype(np.float64) if want is None else want + r
    got = ref.fxb_correlate(native.LIB_PATH, subints)
    lay = ref.layout()
    compare_core(job, lay, ref.corelen, got.astype(np.float64), want, tol=FP32_TOL)
