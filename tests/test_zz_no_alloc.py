"""The no-allocation per-station F stage (fxb_station_fstage_noalloc) against
the context entry point (fxb_submit_subint + fxb_read_spectra), through the C
ABI, on two calls in a row with different subints.

The variant exists for callers that cannot allocate device memory; the test
owns every buffer (torch allocations made by the caller) and checks that the
spectra agree within the FP32 tolerance of the other parity tests and that
the per-FFT weights agree exactly.  Collected last on purpose."""
import ctypes

import numpy as np
import pytest

from fxb200 import native, synth
from fxb200.native import Correlator, DescHolder, poly_arrays
from helpers import FP32_TOL, small_job

pytestmark = pytest.mark.gpu


def _bind():
    L = native.lib()
    f = L.fxb_station_fstage_noalloc
    f.restype = ctypes.c_int
    f.argtypes = [ctypes.POINTER(native.FxbFreq), ctypes.c_int32, ctypes.POINTER(native.FxbStation),
                  ctypes.c_int32, ctypes.c_int64, ctypes.c_int32, ctypes.c_int32, ctypes.c_double, ctypes.c_int32,
                  ctypes.POINTER(ctypes.c_double), ctypes.c_void_p, ctypes.c_int64, ctypes.c_int32,
                  ctypes.c_int32, ctypes.c_void_p, ctypes.c_int32, ctypes.c_int32, ctypes.c_void_p,
                  ctypes.c_void_p, ctypes.c_void_p]
    return f


def test_noalloc_fstage_matches_context_path_twice():
    torch = pytest.importorskip("torch")
    fn = _bind()
    job = small_job(nstation=2, full_pol=True, seed=4)
    T = job.blocks_per_send()
    nchan = job.station_nchan(0)
    holder = DescHolder(job)
    desc = holder.desc
    npoly, order, p0, interval, coeffs = poly_arrays(job, 0)
    for (sec, ns) in [(0, 1_000_000), (0, 5_000_000)]:
        inputs = synth.subint_inputs(job, sec, ns, rho=0.05, seed=21 + ns // 1_000_000)
        corr = Correlator(job)
        corr.submit(inputs, sec, ns)
        ref = np.stack([corr.spectra(0)[:, 0], corr.spectra(0)[:, 1]], axis=1)   # station 0 rows: [t][band][c]
        wref = corr.fft_weights()[0]
        corr.close()

        buf, dsec, dns = inputs[0]
        d_in = torch.from_numpy(buf).cuda()
        d_spec = torch.empty(T * job.stations[0].nband * nchan * 2, dtype=torch.float32, device="cuda")
        d_w = torch.empty(T, dtype=torch.float32, device="cuda")
        torch.cuda.synchronize()
        rc = fn(desc.freqs, desc.nfreq, desc.stations, job.fringe_rot_order, job.subint_ns, npoly, order, p0,
                interval, coeffs.ctypes.data_as(ctypes.POINTER(ctypes.c_double)), d_in.data_ptr(), buf.size,
                dsec, dns, None, sec, ns, d_spec.data_ptr(), d_w.data_ptr(), None)
        assert rc == 0, native.FXB_STATUS.get(rc, rc)
        got = d_spec.cpu().numpy().reshape(T, job.stations[0].nband, nchan, 2)
        got = got[..., 0] + 1j * got[..., 1]
        err = np.linalg.norm(got - ref) / np.linalg.norm(ref)
        assert err <= FP32_TOL, err
        assert np.array_equal(d_w.cpu().numpy(), wref)


def test_noalloc_rejects_oversized_subint():
    torch = pytest.importorskip("torch")
    fn = _bind()
    job = small_job(nstation=2, subint_ns=200_000_000)     # 12500 FFTs > 8192
    holder = DescHolder(job)
    desc = holder.desc
    npoly, order, p0, interval, coeffs = poly_arrays(job, 0)
    d = torch.zeros(1 << 20, dtype=torch.uint8, device="cuda")
    out = torch.zeros(16, dtype=torch.float32, device="cuda")
    rc = fn(desc.freqs, desc.nfreq, desc.stations, 1, job.subint_ns, npoly, order, p0, interval,
            coeffs.ctypes.data_as(ctypes.POINTER(ctypes.c_double)), d.data_ptr(), d.numel(), 0, 0, None,
            0, 0, out.data_ptr(), None, None)
    assert rc == 2      # FXB_ERR_UNSUPPORTED, nothing launched
