"""GPU VDIF decoding (fxb_vdif_unpack) against the oracle's restatement of
mark5_unpack_with_offset: samples and good-sample counts bit-exact, over
every supported channel count and bit width, frame boundaries, invalid and
fill-pattern frames, and the 8-bit 2/4-channel blanking semantics."""
import numpy as np
import pytest

from fxb200 import native, synth
from fxb200.job import Freq, Station, Job, Baseline

import fxoracle

pytestmark = pytest.mark.gpu


def vdif_job(nchan, nbits, payload=1024):
    bands = [(0, "R")] * nchan
    st = Station("A", bands, nbits=nbits, payload_bytes=payload)
    job = Job([Freq(1000.0, 1.024, 16)], [st], [], subint_ns=62_500)
    synth.make_delay_polys(job, 1)
    return job


@pytest.mark.parametrize("nchan,nbits", [(1, 2), (2, 2), (4, 2), (8, 2), (16, 2), (32, 2), (64, 2),
                                         (1, 8), (2, 8), (4, 8)])
def test_unpack_bit_exact(nchan, nbits):
    job = vdif_job(nchan, nbits)
    fs = job.frame_samples(0)
    data = synth.gen_station_frames(job, 0, 0, 8, rho=0.1, seed=nchan * 10 + nbits, invalid=[3], fill=[5])
    rng = np.random.default_rng(nchan + nbits)
    cases = [(0, fs), (fs - 3, 10), (2 * fs + 1, fs + 5), (3 * fs - 7, 2 * fs), (int(rng.integers(0, fs)), 3 * fs)]
    for off, n in cases:
        g, ggood = native.vdif_unpack(data, 1024, 32, nchan, nbits, off, n)
        r, rgood = fxoracle.vdif_unpack(data, 1024, 32, nchan, nbits, off, n)
        assert ggood == rgood, (off, n, ggood, rgood)
        assert np.array_equal(g, r), (off, n)
