"""The c3 batch on the CPU: the seeded subband draw covers every subband
exactly once, each member job is valid (one VDIF stream with a power-of-two
channel count within the decoder's limit, a whole number of FFTs per subint)
and the split is reproducible."""
from fxb200 import configs


def test_c3_members_cover_every_subband_once():
    subs = configs.c3_subbands()
    jobs = configs.c3()
    seen = []
    for job in jobs:
        job.validate()
        assert len(job.stations) == 20
        st = job.stations[0]
        nb = len(st.bands)
        assert nb & (nb - 1) == 0 and nb <= (64 if st.nbits == 2 else 4)
        for f in job.freqs:
            assert job.subint_ns % round(f.nchan * 1000.0 / f.bw_mhz) == 0
            seen.append((f.bw_mhz, f.nchan, st.nbits, f.freq_mhz))
    assert sorted((b, n, k) for b, n, k, _ in seen) == sorted(subs)
    assert len({f for _, _, _, f in seen}) == len(subs)          # distinct sky frequencies


def test_c3_is_seeded():
    a = [(len(j.freqs), j.freqs[0].bw_mhz, j.freqs[0].nchan, j.stations[0].nbits) for j in configs.c3(seed=3)]
    b = [(len(j.freqs), j.freqs[0].bw_mhz, j.freqs[0].nchan, j.stations[0].nbits) for j in configs.c3(seed=3)]
    assert a == b
    assert configs.c3_subbands(seed=3) != configs.c3_subbands(seed=4)
