"""The no-allocation per-station F stage (fxb_station_fstage_noalloc) against
the context entry point (fxb_submit_subint + fxb_read_spectra), through the C
ABI, on two calls in a row with different subints.

The variant exists for callers that cannot allocate device memory (a process
whose device memory is all pre-assigned to its own pool, a real-time
pipeline that allocates nothing after set-up); the test owns every buffer
(torch allocations made by the caller) and checks that the spectra agree
within the FP32 tolerance of the other parity tests and that the per-FFT
weights agree exactly.  The GPU cases cover the documented limits: 4096
channels (the legacy F-stage kernel's 64 KiB shared-memory opt-in), 8-bit
samples (the constant level table and the sticky blanking of 2-channel
streams), caller-supplied valid-FFT flags, and a subint at the 8192-FFT
limit.  The refusals (INTERLACEDVDIF stations, buffers too small for the
result) are decided before any CUDA call and run without a GPU.  Collected
last on purpose."""
import ctypes

import numpy as np
import pytest

from fxb200 import native, synth
from fxb200.native import Correlator, DescHolder, poly_arrays
from helpers import FP32_TOL, small_job

FXB_ERR_ARG, FXB_ERR_UNSUPPORTED = 1, 2


def _bind():
    L = native.lib()
    f = L.fxb_station_fstage_noalloc
    f.restype = ctypes.c_int
    f.argtypes = [ctypes.POINTER(native.FxbFreq), ctypes.c_int32, ctypes.POINTER(native.FxbStation),
                  ctypes.c_int32, ctypes.c_int64, ctypes.c_int32, ctypes.c_int32, ctypes.c_double, ctypes.c_int32,
                  ctypes.POINTER(ctypes.c_double), ctypes.c_void_p, ctypes.c_int64, ctypes.c_int32,
                  ctypes.c_int32, ctypes.c_void_p, ctypes.c_int32, ctypes.c_int32, ctypes.c_void_p, ctypes.c_size_t,
                  ctypes.c_void_p, ctypes.c_size_t, ctypes.POINTER(ctypes.c_int32), ctypes.c_void_p]
    return f


def _call(fn, job, holder, d_in, nbytes, dsec, dns, vflags, sec, ns, spec_ptr, spec_cap, w_ptr, w_cap):
    desc = holder.desc
    npoly, order, p0, interval, coeffs = poly_arrays(job, 0)
    nfft = ctypes.c_int32(-1)
    rc = fn(desc.freqs, desc.nfreq, desc.stations, job.fringe_rot_order, job.subint_ns, npoly, order, p0,
            interval, coeffs.ctypes.data_as(ctypes.POINTER(ctypes.c_double)), d_in, nbytes, dsec, dns,
            vflags.ctypes.data if vflags is not None else None, sec, ns, spec_ptr, spec_cap, w_ptr, w_cap,
            ctypes.byref(nfft), None)
    return rc, nfft.value


CASES = {
    "2bit_256ch": dict(kw=dict(nstation=2, full_pol=True, seed=4), subints=[(0, 1_000_000), (0, 5_000_000)]),
    "2bit_4096ch": dict(kw=dict(nstation=2, nchan=4096, bw=16.0, full_pol=True, seed=5, subint_ns=8_192_000),
                        subints=[(0, 0), (0, 8_192_000)]),
    "8bit_2ch": dict(kw=dict(nstation=2, nbits=8, full_pol=False, seed=6), subints=[(0, 1_000_000), (0, 5_000_000)],
                     invalid=True),
    "validflags": dict(kw=dict(nstation=2, full_pol=True, seed=7), subints=[(0, 1_000_000), (0, 5_000_000)],
                       flags=[0, 7, 31, 100, 249]),
    "8192_ffts": dict(kw=dict(nstation=2, nchan=16, bw=16.0, full_pol=True, seed=8, subint_ns=8_192_000),
                      subints=[(0, 0), (0, 8_192_000)]),
}


@pytest.mark.gpu
@pytest.mark.parametrize("case", sorted(CASES))
def test_noalloc_fstage_matches_context_path_twice(case):
    torch = pytest.importorskip("torch")
    fn = _bind()
    c = CASES[case]
    job = small_job(**c["kw"])
    T = job.blocks_per_send()
    nchan = job.station_nchan(0)
    nband = job.stations[0].nband
    holder = DescHolder(job)
    for k, (sec, ns) in enumerate(c["subints"]):
        invalid = None
        if c.get("invalid"):
            f0 = synth.subint_window(job, 0, sec, ns)[0]
            invalid = {0: [f0 + 1 + k, f0 + 3]}
        inputs = synth.subint_inputs(job, sec, ns, rho=0.05, seed=21 + k, invalid=invalid)
        vf = None
        if c.get("flags"):
            vf = [synth.valid_flags(job, invalid_ffts=c["flags"]) for _ in job.stations]
        corr = Correlator(job)
        corr.submit(inputs, sec, ns, validflags=vf)
        spec = corr.spectra(0)
        ref = np.stack([spec[:, b] for b in range(nband)], axis=1)          # station 0 rows: [t][band][c]
        wref = corr.fft_weights()[0]
        corr.close()

        buf, dsec, dns = inputs[0]
        d_in = torch.from_numpy(buf).cuda()
        d_spec = torch.empty(T * nband * nchan * 2, dtype=torch.float32, device="cuda")
        d_w = torch.empty(T, dtype=torch.float32, device="cuda")
        torch.cuda.synchronize()
        rc, nfft = _call(fn, job, holder, d_in.data_ptr(), buf.size, dsec, dns, vf[0] if vf else None, sec, ns,
                         d_spec.data_ptr(), d_spec.numel(), d_w.data_ptr(), d_w.numel())
        assert rc == 0, native.FXB_STATUS.get(rc, rc)
        assert nfft == T
        got = d_spec.cpu().numpy().reshape(T, nband, nchan, 2)
        got = got[..., 0] + 1j * got[..., 1]
        err = np.linalg.norm(got - ref) / np.linalg.norm(ref)
        assert err <= FP32_TOL, err
        assert np.array_equal(d_w.cpu().numpy(), wref)
        if c.get("flags"):
            assert np.all(wref[c["flags"]] == 0) and np.all(np.abs(got[c["flags"]]) == 0)


@pytest.mark.gpu
def test_noalloc_rejects_oversized_subint():
    torch = pytest.importorskip("torch")
    fn = _bind()
    job = small_job(nstation=2, subint_ns=200_000_000)     # 12500 FFTs > 8192
    holder = DescHolder(job)
    d = torch.zeros(1 << 20, dtype=torch.uint8, device="cuda")
    out = torch.zeros(16, dtype=torch.float32, device="cuda")
    rc, _ = _call(fn, job, holder, d.data_ptr(), d.numel(), 0, 0, None, 0, 0, out.data_ptr(), out.numel(), None, 0)
    assert rc == FXB_ERR_UNSUPPORTED      # nothing launched


# The refusals below return before the entry point makes any CUDA call, so
# they run without a GPU; the device pointers are placeholders that are
# never dereferenced.
FAKE_DEV = 1 << 40


def test_noalloc_refuses_interlaced_station_without_cuda():
    from fxb200.job import Freq, full_job
    job = full_job(2, [Freq(8400.0, 16.0, 256)], full_pol=True, subint_ns=4_000_000)
    synth.make_delay_polys(job, seed=3)
    job.stations[0].mux_threads = 2
    holder = DescHolder(job)
    rc, _ = _call(_bind(), job, holder, FAKE_DEV, 1 << 20, 0, 0, None, 0, 0, FAKE_DEV, 1 << 30, None, 0)
    assert rc == FXB_ERR_UNSUPPORTED


@pytest.mark.parametrize("short", ["spectra", "weights"])
def test_noalloc_refuses_short_output_buffers_without_cuda(short):
    job = small_job(nstation=2, full_pol=True)
    T = job.blocks_per_send()
    need = T * job.stations[0].nband * job.station_nchan(0) * 2
    holder = DescHolder(job)
    spec_cap = need - 1 if short == "spectra" else need
    w_cap = T - 1 if short == "weights" else T
    rc, nfft = _call(_bind(), job, holder, FAKE_DEV, 1 << 20, 0, 0, None, 0, 0, FAKE_DEV, spec_cap, FAKE_DEV, w_cap)
    assert rc == FXB_ERR_ARG
    assert nfft == T
