"""Shared job builders and comparison helpers for the parity tests."""
from __future__ import annotations

import numpy as np

from fxb200 import synth
from fxb200.job import Freq, Job, full_job

# FP32 form vs the FP64 oracle: relative visibility tolerance of the FP32 form
FP32_TOL = 1e-5
# tensor-core form (FP16 spectra, FP32 accumulation) vs the FP64 oracle:
# relative visibility tolerance of the tensor-core forms, applied norm-wise to the cross
# and autocorrelations and as the rms of the per-visibility relative
# amplitude and phase (radians) errors
TC_REL_TOL = 1e-3


def small_job(nstation=4, nchan=256, bw=16.0, nfreq=1, full_pol=False, nbits=2, subint_ns=4_000_000,
              order=1, lsb=False, freq0=8400.0, avg=1, seed=1) -> Job:
    freqs = [Freq(freq0 + k * bw, bw, nchan, "L" if lsb else "U", avg) for k in range(nfreq)]
    job = full_job(nstation, freqs, full_pol=full_pol, subint_ns=subint_ns, nbits=nbits, fringe_rot_order=order)
    synth.make_delay_polys(job, seed=seed)
    job.validate()
    return job


def regions(job: Job, layout: np.ndarray, corelen: int):
    """(name, float slice) of the core result: cross, bweights, autos,
    acweights and (with phase cal) the phase-cal tones."""
    nf, nb, ns = len(job.freqs), len(job.baselines), len(job.stations)
    bl = layout[:nf * nb]
    bw = layout[nf * nb:2 * nf * nb]
    ac = layout[2 * nf * nb:2 * nf * nb + ns]
    acw = layout[2 * nf * nb + ns:2 * nf * nb + 2 * ns]
    pc = layout[2 * nf * nb + 2 * ns:2 * nf * nb + 3 * ns]
    pc_valid = pc[pc >= 0]
    acw_end = int(pc_valid.min()) if pc_valid.size else corelen
    bw_valid = bw[bw >= 0]
    xc_end = int(bw_valid.min()) if bw_valid.size else int(ac.min())
    out = [("cross", slice(0, 2 * xc_end)), ("bweight", slice(2 * xc_end, 2 * int(ac.min()))),
           ("auto", slice(2 * int(ac.min()), 2 * int(acw.min()))), ("acweight", slice(2 * int(acw.min()), 2 * acw_end))]
    if pc_valid.size:
        out.append(("pcal", slice(2 * acw_end, 2 * corelen)))
    return out


def rel_err(a: np.ndarray, b: np.ndarray) -> float:
    nb = np.linalg.norm(b)
    if nb == 0:
        return float(np.linalg.norm(a))
    return float(np.linalg.norm(a - b) / nb)


def _cplx(a):
    return a[0::2].astype(np.float64) + 1j * a[1::2].astype(np.float64)


def vis_errors(job, layout, corelen, got, ref):
    """Errors of a core result against the FP64 oracle's, over the cross
    visibilities (and norm-wise over the autocorrelations):
      cross_rel / auto_rel   ||V - V64|| / ||V64||;
      amp_rms / amp_p99      per-visibility (|V| - |V64|) / |V64|;
      phase_rms / phase_p99  per-visibility arg(V conj V64), radians;
      ccu                    rms cross error over the autocorrelation scale
                             (correlation-coefficient units).
    The per-visibility figures leave out visibilities with |V64| under a
    tenth of the median (noise-dominated visibilities near zero, whose
    relative error is unbounded; `left_out` counts them)."""
    reg = dict(regions(job, layout, corelen))
    xc, ac = reg["cross"], reg["auto"]
    v, r = _cplx(got[xc]), _cplx(ref[xc])
    auto_rms = np.sqrt(np.mean(ref[ac][0::2].astype(np.float64) ** 2))
    keep = np.abs(r) >= 0.1 * np.median(np.abs(r))
    amp = (np.abs(v[keep]) - np.abs(r[keep])) / np.abs(r[keep])
    ph = np.angle(v[keep] * np.conj(r[keep]))
    return {"cross_rel": float(np.linalg.norm(v - r) / np.linalg.norm(r)),
            "auto_rel": rel_err(got[ac], ref[ac]),
            "amp_rms": float(np.sqrt(np.mean(amp ** 2))), "amp_p99": float(np.quantile(np.abs(amp), 0.99)),
            "phase_rms": float(np.sqrt(np.mean(ph ** 2))), "phase_p99": float(np.quantile(np.abs(ph), 0.99)),
            "ccu": float(np.sqrt(np.mean((got[xc].astype(np.float64) - ref[xc]) ** 2)) / auto_rms),
            "left_out": int((~keep).sum()), "visibilities": int(keep.size)}


def assert_tc_gate(e, tol=TC_REL_TOL):
    """The tensor-core form's relative gate on vis_errors' figures."""
    for k in ("cross_rel", "auto_rel", "amp_rms", "phase_rms"):
        assert e[k] <= tol, (k, e)


def compare_core(job, layout, corelen, got, ref, tol=FP32_TOL, weights_exact=True):
    out = {}
    for name, sl in regions(job, layout, corelen):
        g, r = got[sl], ref[sl]
        if name in ("bweight", "acweight"):
            if weights_exact:
                assert np.array_equal(g.astype(np.float32), r.astype(np.float32)), (name, g[:8], r[:8])
            else:
                assert np.allclose(g, r, rtol=1e-6, atol=1e-6), name
        else:
            e = rel_err(g, r)
            out[name] = e
            assert e <= tol, "%s relative error %.3g > %.3g" % (name, e, tol)
            scale = np.max(np.abs(r)) if r.size else 1.0
            if scale > 0:
                m = float(np.max(np.abs(g - r)) / scale)
                assert m <= 10 * tol, "%s max error %.3g" % (name, m)
    return out


# zoom windows of the two 16 MHz subbands of small_job(nfreq=2):
# (parent freq, offset MHz, width MHz)
ZOOMS = [(0, 4.0, 4.0), (1, 0.0, 8.0), (1, 12.0, 4.0)]


def zoom_job(keep_parents=True, nstation=3, avg=1, zooms=ZOOMS, full_pol=True, **kw) -> Job:
    """small_job with two 16 MHz subbands, dual polarisation with cross hands,
    and zoom windows correlated on every baseline (optionally without the
    parent subbands' own products)."""
    from fxb200.job import add_zoom_bands
    kw.setdefault("subint_ns", 2_048_000)
    job = small_job(nstation=nstation, nchan=256, bw=16.0, nfreq=2, full_pol=full_pol, avg=avg, **kw)
    add_zoom_bands(job, zooms, keep_parents=keep_parents, chans_to_avg=avg)
    job.validate()
    return job


def mixed_bw_zoom_job(seed=4) -> Job:
    """Stations 0 and 1 record 16 MHz at 8400 MHz (256 channels), station 2
    records 8 MHz at 8404 MHz (128 channels: the same channel width and FFT
    duration).  Stations 0 and 1 zoom their band onto station 2's, so every
    baseline correlates 8404-8412 MHz, and 0-1 also the full 16 MHz."""
    from fxb200.job import Baseline, Station
    freqs = [Freq(8400.0, 16.0, 256), Freq(8404.0, 8.0, 128)]
    wide = lambda n: Station(n, [(0, "R"), (0, "L")], zoom_bands=[(1, "R"), (1, "L")])
    st = [wide("A"), wide("B"), Station("C", [(1, "R"), (1, "L")])]
    par = [(0, 0), (0, 1), (1, 0), (1, 1)]       # RR, RL, LR, LL
    zz = [(2 + a, 2 + b) for a, b in par]
    zr = [(2 + a, b) for a, b in par]
    bls = [Baseline(0, 1, [(0, par), (1, zz)]), Baseline(0, 2, [(1, zr)]), Baseline(1, 2, [(1, zr)])]
    job = Job(freqs, st, bls, subint_ns=2_048_000)
    synth.make_delay_polys(job, seed=seed)
    job.validate()
    return job


def pcal_job(interval=1.0, base=0.0, **kw) -> Job:
    """small_job with phase-cal extraction on every station."""
    job = small_job(**kw)
    for st in job.stations:
        st.pcal_interval_mhz = interval
        st.pcal_base_mhz = base
    return job


# integer LOs (32 bins), a fractional LO (3200 bins), 8-bit samples, a comb
# whose spacing exceeds the band (one zero tone), a 5 MHz comb, and 1024 bins
PCAL_JOBS = {
    "pcal_int_lo": lambda: pcal_job(nstation=3, nfreq=2, full_pol=True, subint_ns=2_048_000),
    "pcal_frac_lo": lambda: pcal_job(nstation=3, nfreq=2, full_pol=True, freq0=8400.01, subint_ns=2_048_000),
    "pcal_8bit": lambda: pcal_job(nstation=2, nbits=8, freq0=8400.25),
    "pcal_no_tone": lambda: pcal_job(20.0, nstation=2, freq0=8401.0),
    "pcal_5mhz": lambda: pcal_job(5.0, nstation=2, freq0=8402.0),
    # first tone 31.25 kHz above the LO: 1024 bins, fewer than the 4096
    # samples of a window
    "pcal_1024_bins": lambda: pcal_job(nstation=2, nchan=2048, freq0=8400.96875, subint_ns=4_096_000),
    # a 5 MHz comb over 8400-8432 MHz: the second subband's first tone is 4 MHz
    # above its LO, whose period is not a multiple of the comb's (shifting
    # extractor)
    "pcal_shifting": lambda: pcal_job(5.0, nstation=2, nfreq=2, full_pol=True, subint_ns=2_048_000),
    # lower-sideband bands, LO on the comb and 10 kHz off it
    "pcal_lsb": lambda: pcal_job(nstation=2, nfreq=2, full_pol=True, lsb=True, subint_ns=2_048_000),
    "pcal_lsb_frac": lambda: pcal_job(nstation=2, lsb=True, freq0=8400.01),
}


def mux_job(masklength=None, **kw) -> Job:
    """small_job whose stations 0 and 2 are INTERLACEDVDIF (one band per
    thread, muxed frames handed over); masklength: the EDV4 mask length that
    edv4_inputs writes (default: one bit per band)."""
    kw = dict(dict(nstation=3, nfreq=2, full_pol=True, subint_ns=2_048_000), **kw)
    job = small_job(**kw)
    for s in (0, 2):
        job.stations[s].mux_threads = job.stations[s].nband
    job.edv4_masklength = masklength or job.stations[0].nband
    return job


def edv4_inputs(job: Job, inputs, seed=5):
    """Write EDV4 headers (version 4, the job's mask length, sync word, a
    validity mask per frame: mostly complete, some frames missing one or two
    bit groups) into the frames of the INTERLACEDVDIF stations."""
    rng = np.random.default_rng(seed)
    out = []
    for s, (buf, dsec, dns) in enumerate(inputs):
        st = job.stations[s]
        if not st.mux_threads:
            out.append((buf, dsec, dns))
            continue
        fb = st.payload_bytes + st.header_bytes
        fr = buf.copy().reshape(-1, fb)
        ml = job.edv4_masklength
        full = (1 << ml) - 1
        masks = np.full(len(fr), full, dtype=np.uint64)
        for k in rng.choice(len(fr), size=max(1, len(fr) // 3), replace=False):
            drop = rng.choice(ml, size=int(rng.integers(1, 3)), replace=False)
            masks[k] = full & ~int(sum(1 << int(b) for b in drop))
        words = fr[:, :32].copy().view(np.uint32)
        words[:, 4] = (4 << 24) | (ml << 16)
        words[:, 5] = 0xACABFEED
        fr[:, :32] = words.view(np.uint8)
        fr[:, 24:32] = masks.reshape(-1, 1).view(np.uint8)
        out.append((fr.reshape(-1), dsec, dns))
    return out


def corr_job(order=1, clock=True, delta=True, phase=True, looff=True, seed=9, **kw) -> Job:
    """A full-polarisation job whose stations carry per-frequency clock
    offsets, R/L clock deltas, phase offsets and LO offsets (the datastream
    table's CLK OFFSET offset:delta:phase and FREQ OFFSET), seeded; the first
    station's first frequency keeps a zero clock offset, as the reference asks
    of a telescope's first band."""
    kw.setdefault("nstation", 3)
    kw.setdefault("full_pol", True)
    kw.setdefault("nfreq", 2)
    job = small_job(order=order, **kw)
    rng = np.random.default_rng(seed)
    for s, st in enumerate(job.stations):
        for f in st.recorded_freqs():
            clk = 0.0 if (s == 0 and f == st.bands[0][0]) or not clock else float(rng.uniform(-0.2, 0.2))
            dclk = float(rng.uniform(-0.02, 0.02)) if delta else 0.0
            ph = float(rng.uniform(-60.0, 60.0)) if phase else 0.0
            lo = float(rng.uniform(-2500.0, 2500.0)) if looff else 0.0
            st.freq_corr[f] = (clk, dclk, ph, lo)
    return job


def raw_read(job: Job, s: int, buf: np.ndarray, rng, drop_frac: float = 0.05, lead_extra: bool = True):
    """synth.raw_read with a fraction of thread frames left out and an
    unwanted thread's frame leading the read (see there)."""
    return synth.raw_read(job, s, buf, rng, drop_frac=drop_frac, lead_extra=lead_extra)


def cplx_job(lsb=False, nbits=2, nstation=3, nfreq=2, nchan=256, bw=16.0, order=1, **kw) -> Job:
    """A full-polarisation job of complex-sampled (single-sideband) stations:
    bw complex samples per second per band, nchan-point complex FFTs."""
    job = full_job(nstation, [Freq(8400.0 + k * bw, bw, nchan, "L" if lsb else "U") for k in range(nfreq)],
                   full_pol=True, subint_ns=kw.pop("subint_ns", 4_000_000), nbits=nbits, fringe_rot_order=order)
    for st in job.stations:
        st.complex_sampling = True
    synth.make_delay_polys(job, seed=kw.pop("seed", 4))
    job.validate()
    return job
