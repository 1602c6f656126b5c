"""Generate the golden fixtures of tests/golden from the reference's own
compiled CPU code (oracle/_ref, built by oracle/Makefile.ref from the
reference sources).  Run in a checkout where the reference build exists:

    python tests/golden/make_golden.py

Fixtures (small, committed):
  unpack_<nchan>ch_<nbits>bit.npz : VDIF bytes (with an invalid frame and a
      fill-pattern frame), the decode window, and mark5access's samples and
      good-sample count.
  corr_small.npz : a 3-station, 2-polarisation, 64-channel job's VDIF input
      for one 1.024 ms subint, and the reference's core result, layout and
      delay interpolators.
"""
import json
import os
import sys

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(os.path.dirname(HERE))
sys.path[:0] = [os.path.join(ROOT, "difx-svn2git-try3_b200"), os.path.join(ROOT, "oracle")]

from fxb200 import synth  # noqa: E402
from fxb200.job import Freq, Job, Station, full_job  # noqa: E402
import refcorr  # noqa: E402  (only loaded when generating)

# (channels, bits, payload bytes, bandwidth MHz): whole frames per second and
# an integral Mbit/s, as a real VDIF mode has
UNPACK_CASES = [(1, 2, 1000, 1.0), (2, 2, 1000, 1.0), (4, 2, 1000, 1.0), (16, 2, 1000, 1.0), (64, 2, 1024, 2.0),
                (1, 8, 1000, 1.0), (2, 8, 1000, 1.0), (4, 8, 1000, 1.0)]


def unpack_fixture(nchan, nbits, payload, bw):
    st = Station("A", [(0, "R")] * nchan, nbits=nbits, payload_bytes=payload)
    job = Job([Freq(1000.0, bw, 16)], [st], [], subint_ns=64_000)
    synth.make_delay_polys(job, 1)
    fs = job.frame_samples(0)
    data = synth.gen_station_frames(job, 0, 0, 6, rho=0.1, seed=100 + nchan * 10 + nbits, invalid=[2], fill=[4])
    fmt = "VDIF_%d-%d-%d-%d" % (payload, job.mbps(0), nchan, nbits)
    gran = max(1, 8 // (nchan * nbits))
    windows = []
    for off, n in [(0, fs), (fs - 2 * gran, 4 * gran), (fs + gran, 2 * fs), (3 * fs - 4 * gran, 2 * fs + 8 * gran)]:
        off -= off % gran
        n -= n % gran
        out, good = refcorr.unpack(fmt, data, off, n, nchan)
        windows.append((off, n, out, good))
    np.savez_compressed(os.path.join(HERE, "unpack_%dch_%dbit.npz" % (nchan, nbits)), data=data,
                        payload=payload, header=32, nchan=nchan, nbits=nbits,
                        offsets=np.array([w[0] for w in windows]), nsamp=np.array([w[1] for w in windows]),
                        good=np.array([w[3] for w in windows]),
                        **{"samples_%d" % i: w[2] for i, w in enumerate(windows)})


def small_job():
    job = full_job(3, [Freq(8400.0, 4.0, 64)], full_pol=True, subint_ns=1_024_000)
    for s in job.stations:
        s.payload_bytes = 1000
    synth.make_delay_polys(job, seed=12)
    job.validate()
    return job


def corr_fixture():
    job = small_job()
    ref = refcorr.RefCorrelator(job)
    sec, ns = 0, 2_048_000
    inputs = synth.subint_inputs(job, sec, ns, rho=0.1, seed=31)
    vf = [synth.valid_flags(job) for _ in job.stations]
    core = ref.process_subint(inputs, vf, 0, sec, ns)
    interp = np.array([ref.interpolator(s, sec, ns) for s in range(len(job.stations))])
    arrays = {"buf_%d" % s: b for s, (b, _, _) in enumerate(inputs)}
    np.savez_compressed(os.path.join(HERE, "corr_small.npz"), core=core, layout=ref.layout(), interp=interp,
                        datasec=np.array([x for _, x, _ in inputs]), datans=np.array([x for _, _, x in inputs]),
                        sec=sec, ns=ns, **arrays)
    ref.close()


if __name__ == "__main__":
    if not refcorr.available():
        sys.exit("reference build oracle/_ref missing: make -f oracle/Makefile.ref")
    for case in UNPACK_CASES:
        unpack_fixture(*case)
    corr_fixture()
    print(json.dumps(sorted(f for f in os.listdir(HERE) if f.endswith(".npz"))))
