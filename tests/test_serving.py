"""Serving workload and admission sizing on the CPU (no GPU): the seeded job
stream draws valid jobs in the stated ranges, and the device footprint used
for admission (fxb_job_footprint, C ABI) grows with the job."""
import numpy as np

from fxb200 import serving


def test_job_stream_shapes_are_valid_and_seeded():
    rng = np.random.default_rng(7)
    seen = []
    for k in range(12):
        job, nsub = serving.serving_job(rng, seed=k, stations=(4, 32), subbands=(1, 16), seconds=(0.1, 2.0))
        job.validate()
        nst = len(job.stations)
        assert 4 <= nst <= 32
        assert 1 <= len(job.freqs) <= 16
        f = job.freqs[0]
        assert f.bw_mhz in (8.0, 16.0, 32.0, 64.0) and 256 <= f.nchan <= 8192
        fft_ns = f.nchan * 1000.0 / f.bw_mhz
        assert job.subint_ns % int(round(fft_ns)) == 0
        assert 0.05 <= nsub * job.subint_ns * 1e-9 <= 2.1
        seen.append((nst, len(job.freqs), f.nchan))
    rng2 = np.random.default_rng(7)
    again = [(len(j.stations), len(j.freqs), j.freqs[0].nchan)
             for j, _ in (serving.serving_job(rng2, seed=k) for k in range(12))]
    assert seen == again


def test_footprint_grows_with_the_job():
    rng = np.random.default_rng(3)
    small, _ = serving.serving_job(rng, seed=1, stations=(4, 4), subbands=(1, 1), nchans=(256,), bws=(16.0,))
    big, _ = serving.serving_job(rng, seed=2, stations=(16, 16), subbands=(8, 8), nchans=(1024,), bws=(32.0,))
    fs, fb = serving.job_footprint(small), serving.job_footprint(big)
    assert 0 < fs < fb
    # FP32 spectra take twice the bytes of the tensor-core form's bf16x2
    assert serving.job_footprint(big, xmac="fp32") > fb


def test_poisson_arrivals_are_increasing():
    t = serving.poisson_arrivals(np.random.default_rng(1), 50, rate_hz=20.0)
    assert np.all(np.diff(t) > 0) and 1.0 < t[-1] < 5.0
