"""Seeded synthetic VLBI baseband: correlated sky + station noise, quantised
and packed into VDIF frames.

Signal model (the stand-in for recorded data; no dataset is used):

* one common real Gaussian sky signal per (frequency, polarisation), unit
  variance, shared by all stations, delayed per station by its delay model;
* independent unit-variance Gaussian noise per (station, band);
* station voltage = sqrt(rho) * delayed sky + sqrt(1 - rho) * noise;
* quantised to 2 bits with thresholds +-0.98 sigma (codes 0..3 =
  {x < -t, -t <= x < 0, 0 <= x < t, x >= t}, the order of the decoder table
  {-HiMag, -1, +1, +HiMag}, libraries/mark5access/mark5access/format_vdif.c:78)
  or to 8-bit offset binary b = clip(round(x * 10) + 128, 0, 255) (decoded as
  (b - 128)/3.3, format_vdif.c:122);
* packed LSB-first into single-thread VDIF frames (32-byte header, all bands
  interleaved as VDIF channels, libraries/vdifio/src/vdifio.h:42-58).

The delay is applied in the frequency domain per block of ``BLOCK`` samples
(a phase ramp exp(-2 pi i (f_LO + f) tau) on the block's spectrum), so every
block is reproducible from the seed alone and any window of frames can be
generated independently of any other.
"""
from __future__ import annotations

import hashlib
from typing import Dict, Iterable, Optional, Sequence

import numpy as np

from .job import DelayPoly, Job

BLOCK = 1 << 14
THRESH = 0.98
VDIF_HEADER = 32


def _rng(*key) -> np.random.Generator:
    h = hashlib.blake2b(repr(key).encode(), digest_size=16).digest()
    return np.random.default_rng(np.frombuffer(h, dtype=np.uint64))


def make_delay_polys(job: Job, seed: int, interval_s: int = 120, max_offset_us: float = 5.0,
                     max_rate_us_s: float = 1.0, max_quad_us_s2: float = 1e-4) -> None:
    """Seeded quadratic delay polynomial per station: offset U(+-5 us), rate
    U(+-1 us/s), small quadratic term.  Stored in the .im convention."""
    r = _rng("delay", seed)
    for st in job.stations:
        c0 = r.uniform(-max_offset_us, max_offset_us)
        c1 = r.uniform(-max_rate_us_s, max_rate_us_s)
        c2 = r.uniform(-max_quad_us_s2, max_quad_us_s2)
        st.polys = [DelayPoly(start_sec=0.0, interval_s=interval_s, coeffs=(c0, c1, c2))]


def station_delay_us(job: Job, s: int, t_sec) -> np.ndarray:
    """Evaluate the station's delay polynomial (us) at job-relative time t."""
    st = job.stations[s]
    t = np.asarray(t_sec, dtype=np.float64)
    out = np.zeros_like(t)
    for p in st.polys:
        dt = t - p.start_sec
        sel = (dt >= 0) & (dt <= p.interval_s)
        v = np.zeros_like(t)
        for k, c in enumerate(p.coeffs):
            v = v + c * dt ** k
        out = np.where(sel, v, out)
    return out + st.clock_us


def _band_block(job: Job, s: int, band: int, blk: int, rho: float, seed: int) -> np.ndarray:
    """Real voltage samples of one band of one station for one BLOCK."""
    st = job.stations[s]
    f, pol = st.bands[band]
    fr = job.freqs[f]
    fs = 2.0 * fr.bw_mhz                       # Ms/s
    sky = _rng("sky", seed, f, pol, blk).standard_normal(BLOCK)
    spec = np.fft.rfft(sky)
    fb = np.arange(spec.size) * (fs / BLOCK)   # baseband frequency, MHz
    tmid = (blk + 0.5) * BLOCK / (fs * 1e6)
    tau = float(station_delay_us(job, s, tmid))
    if fr.sideband == "U":
        ph = -2.0 * np.pi * (fr.freq_mhz + fb) * tau
    else:
        ph = 2.0 * np.pi * (fr.freq_mhz - fb) * tau
    skyd = np.fft.irfft(spec * np.exp(1j * ph), n=BLOCK)
    noise = _rng("noise", seed, s, band, blk).standard_normal(BLOCK)
    return np.sqrt(rho) * skyd + np.sqrt(1.0 - rho) * noise


def _band_block_complex(job: Job, s: int, band: int, blk: int, rho: float, seed: int) -> np.ndarray:
    """Complex voltage samples of one band for one BLOCK (complex sampling at
    bw samples per second): a complex sky signal per (frequency, polarisation)
    whose baseband frequency f in [0, bw) is sky frequency LO + f, delayed per
    station (phase exp(-2 pi i (LO + f) tau)), plus complex station noise."""
    st = job.stations[s]
    f, pol = st.bands[band]
    fr = job.freqs[f]
    fs = fr.bw_mhz                             # M complex samples / s
    r = _rng("csky", seed, f, pol, blk)
    sky = (r.standard_normal(BLOCK) + 1j * r.standard_normal(BLOCK)) / np.sqrt(2.0)
    spec = np.fft.fft(sky)
    fb = np.arange(BLOCK) * (fs / BLOCK)       # baseband frequency in [0, bw), MHz
    tmid = (blk + 0.5) * BLOCK / (fs * 1e6)
    tau = float(station_delay_us(job, s, tmid))
    skyd = np.fft.ifft(spec * np.exp(-2j * np.pi * (fr.freq_mhz + fb) * tau))
    q = _rng("cnoise", seed, s, band, blk)
    noise = (q.standard_normal(BLOCK) + 1j * q.standard_normal(BLOCK)) / np.sqrt(2.0)
    return np.sqrt(rho) * skyd + np.sqrt(1.0 - rho) * noise


def band_samples(job: Job, s: int, band: int, n0: int, n: int, rho: float, seed: int) -> np.ndarray:
    """Voltage samples [n0, n0+n) (job-relative sample index) of one band."""
    b0, b1 = n0 // BLOCK, (n0 + n - 1) // BLOCK
    blockfn = _band_block_complex if job.stations[s].complex_sampling else _band_block
    parts = [blockfn(job, s, band, b, rho, seed) for b in range(b0, b1 + 1)]
    x = np.concatenate(parts)
    off = n0 - b0 * BLOCK
    return x[off:off + n]


def quantise(x: np.ndarray, nbits: int) -> np.ndarray:
    if nbits == 2:
        t = THRESH
        return (np.where(x < -t, 0, np.where(x < 0.0, 1, np.where(x < t, 2, 3)))).astype(np.uint8)
    if nbits == 8:
        return np.clip(np.rint(x * 10.0) + 128, 0, 255).astype(np.uint8)
    raise ValueError(nbits)


def pack_payload(codes: np.ndarray, nbits: int) -> np.ndarray:
    """codes [nchan][nsamp] -> VDIF payload bytes, fields LSB-first in
    (time, channel) order."""
    nchan, nsamp = codes.shape
    fields = codes.T.reshape(-1)               # q = t*nchan + c
    if nbits == 8:
        return fields.astype(np.uint8)
    per = 8 // nbits
    f = fields.reshape(-1, per).astype(np.uint16)
    out = np.zeros(f.shape[0], dtype=np.uint16)
    for i in range(per):
        out |= f[:, i] << (nbits * i)
    return out.astype(np.uint8)


def vdif_header(job: Job, s: int, frame_global: int, invalid: bool = False, station_id: int = 0) -> np.ndarray:
    st = job.stations[s]
    fps = job.frames_per_sec(s)
    sec = frame_global // fps
    fnum = frame_global % fps
    w = np.zeros(8, dtype=np.uint32)
    w[0] = (int(sec) & 0x3FFFFFFF) | ((1 << 31) if invalid else 0)
    w[1] = (fnum & 0xFFFFFF)
    log2ch = int(np.log2(st.nband)) if st.nband & (st.nband - 1) == 0 else 0
    w[2] = (1 << 29) | (log2ch << 24) | ((job.frame_bytes(s) // 8) & 0xFFFFFF)
    w[3] = ((st.nbits - 1) << 26) | (station_id & 0xFFFF) | ((1 << 31) if st.complex_sampling else 0)
    return w.view(np.uint8)


FILL_WORD = np.frombuffer(bytes.fromhex("4433221144332211")[::-1], dtype=np.uint8)  # 0x1122334411223344 little-endian


def gen_station_frames(job: Job, s: int, frame0: int, nframes: int, rho: float, seed: int,
                       invalid: Iterable[int] = (), fill: Iterable[int] = ()) -> np.ndarray:
    """nframes VDIF frames of station s starting at job-relative frame index
    frame0.  ``invalid`` / ``fill`` list job-relative frame indices to mark
    with the header invalid bit / to overwrite with fill pattern."""
    st = job.stations[s]
    fsamp = job.frame_samples(s)
    fb = job.frame_bytes(s)
    inv = set(invalid)
    fil = set(fill)
    n0 = frame0 * fsamp
    n = nframes * fsamp
    if st.complex_sampling:
        # real and imaginary fields side by side, per (time, channel)
        # (the complex VDIF decoders' order, format_vdif.c:2369-2410, 2868-2907)
        # (rows 2 c + part: the payload's field order is (time, channel, part))
        x = [band_samples(job, s, b, n0, n, rho, seed) for b in range(st.nband)]
        codes = np.stack([q for v in x for q in (quantise(v.real, st.nbits), quantise(v.imag, st.nbits))])
    else:
        codes = np.stack([quantise(band_samples(job, s, b, n0, n, rho, seed), st.nbits) for b in range(st.nband)])
    out = np.empty(nframes * fb, dtype=np.uint8)
    for k in range(nframes):
        g = frame0 + k
        payload = pack_payload(codes[:, k * fsamp:(k + 1) * fsamp], st.nbits)
        out[k * fb:k * fb + VDIF_HEADER] = vdif_header(job, s, g, invalid=g in inv, station_id=s)
        out[k * fb + VDIF_HEADER:(k + 1) * fb] = payload
        if g in fil:
            out[k * fb + VDIF_HEADER:(k + 1) * fb] = np.resize(FILL_WORD, st.payload_bytes)
    return out


def subint_window(job: Job, s: int, sec: int, ns: int, margin_us: float = 20.0):
    """Frame range that a DataStream would deliver for the subintegration
    starting at (sec, ns): from the frame holding (start - margin) to the frame
    holding (end + margin).  Returns (frame0, nframes, datasec, datans)."""
    fps = job.frames_per_sec(s)
    t0 = sec + ns * 1e-9 - margin_us * 1e-6
    t1 = sec + ns * 1e-9 + job.subint_ns * 1e-9 + margin_us * 1e-6
    f0 = int(np.floor(t0 * fps))
    f1 = int(np.floor(t1 * fps)) + 1
    f0 = max(f0, 0)
    dsec = f0 // fps
    dns = int(round((f0 % fps) * 1e9 / fps))
    return f0, f1 - f0, dsec, dns


def subint_inputs(job: Job, sec: int, ns: int, rho: float, seed: int,
                  invalid: Optional[Dict[int, Sequence[int]]] = None,
                  fill: Optional[Dict[int, Sequence[int]]] = None):
    """Per-station (bytes, datasec, datans) for one subintegration."""
    out = []
    for s in range(len(job.stations)):
        f0, nf, dsec, dns = subint_window(job, s, sec, ns)
        buf = gen_station_frames(job, s, f0, nf, rho, seed,
                                 invalid=(invalid or {}).get(s, ()), fill=(fill or {}).get(s, ()))
        out.append((buf, dsec, dns))
    return out


def valid_flags(job: Job, all_valid: bool = True, invalid_ffts: Sequence[int] = ()) -> np.ndarray:
    """Valid-FFT bitfield as the DataStream control block carries it: 30 flags
    per int32 (mpifxcorr/src/mpifxcorr.h:39, FLAGS_PER_INT)."""
    bps = job.blocks_per_send()
    n = (bps + 29) // 30
    v = np.zeros(n, dtype=np.int32)
    for i in range(bps):
        if all_valid and i not in invalid_ffts:
            v[i // 30] |= (1 << (i % 30))
    return v


# ---------------------------------------------------------------- bulk data
def _code_byte_table(nbits: int) -> np.ndarray:
    """65536-entry table whose uniform sampling yields payload bytes with the
    code statistics of the quantiser on unit-variance Gaussian input: for
    2-bit, four independent fields with P(outer) = 2*Phi(-0.98) each."""
    from math import erf, sqrt
    if nbits == 2:
        p0 = 0.5 * (1.0 + erf(-THRESH / sqrt(2.0)))       # P(x < -0.98)
        pc = np.array([p0, 0.5 - p0, 0.5 - p0, p0])
        probs = np.ones(256)
        for b in range(256):
            for i in range(4):
                probs[b] *= pc[(b >> (2 * i)) & 3]
    else:
        x = (np.arange(256) - 128) / 10.0
        probs = np.exp(-0.5 * x * x)
        probs /= probs.sum()
    counts = np.floor(probs * 65536).astype(np.int64)
    short = 65536 - counts.sum()
    order = np.argsort(-(probs * 65536 - counts))
    counts[order[:short]] += 1
    return np.repeat(np.arange(256, dtype=np.uint8), counts)


_CODE_POOL = {}


def _code_pool(nbits: int) -> np.ndarray:
    """32 MiB of payload bytes with the quantiser's code statistics (seeded)."""
    if nbits not in _CODE_POOL:
        table = _code_byte_table(nbits)
        rng = _rng("codepool", nbits)
        _CODE_POOL[nbits] = table[rng.integers(0, 65536, size=32 << 20, dtype=np.uint16)]
    return _CODE_POOL[nbits]


def bulk_station_frames(job: Job, s: int, frame0: int, nframes: int, seed: int) -> np.ndarray:
    """nframes VDIF frames with valid headers whose payload bytes follow the
    quantiser's code statistics: the bulk stand-in input for throughput
    measurement.  Payloads are runs of a seeded 32 MiB pool of code bytes
    taken at seeded offsets (per station and block of frames), so that
    gigabytes are produced at memory speed."""
    st = job.stations[s]
    fb = job.frame_bytes(s)
    pool = _code_pool(st.nbits)
    rng = _rng("bulk", seed, s, frame0)
    out = np.empty((nframes, fb), dtype=np.uint8)
    per = max(1, (len(pool) // 2) // st.payload_bytes)          # frames per block
    for i in range(0, nframes, per):
        n = min(per, nframes - i)
        off = int(rng.integers(0, len(pool) - n * st.payload_bytes + 1))
        out[i:i + n, VDIF_HEADER:] = pool[off:off + n * st.payload_bytes].reshape(n, st.payload_bytes)
    fps = job.frames_per_sec(s)
    g = frame0 + np.arange(nframes, dtype=np.int64)
    h = np.zeros((nframes, 8), dtype=np.uint32)
    h[:, 0] = (g // fps).astype(np.uint32) & 0x3FFFFFFF
    h[:, 1] = (g % fps).astype(np.uint32) & 0xFFFFFF
    log2ch = int(np.log2(st.nband)) if st.nband & (st.nband - 1) == 0 else 0
    h[:, 2] = (1 << 29) | (log2ch << 24) | ((fb // 8) & 0xFFFFFF)
    h[:, 3] = ((st.nbits - 1) << 26) | (s & 0xFFFF)
    out[:, :VDIF_HEADER] = h.view(np.uint8)
    return out.reshape(-1)


def vdif_header_words(seconds: int, frame: int, epoch: int, framebytes: int, nchan: int, nbits: int,
                      threadid: int, stationid: int = 0, invalid: bool = False) -> np.ndarray:
    """The 8 words of a VDIF header (vdifio.h:58-80)."""
    logch = 0
    while (1 << logch) < nchan:
        logch += 1
    w = np.zeros(8, dtype=np.uint32)
    w[0] = (seconds & 0x3FFFFFFF) | (int(invalid) << 31)
    w[1] = (frame & 0xFFFFFF) | ((epoch & 0x3F) << 24)
    w[2] = ((framebytes // 8) & 0xFFFFFF) | (logch << 24)
    w[3] = (stationid & 0xFFFF) | ((threadid & 0x3FF) << 16) | (((nbits - 1) & 0x1F) << 26)
    return w


def interlaced_vdif(nthreads: int, nframes: int, payload: int = 8000, nbits: int = 2, fps: int = 4000,
                    seconds0: int = 1000, frame0: int = 0, epoch: int = 35, seed: int = 0, thread_ids=None,
                    shuffle: bool = True, drop=(), extra_thread: bool = False, duplicate=()) -> np.ndarray:
    """A multi-thread VDIF stream: nframes frame times of nthreads single-channel
    threads (random payload bytes), each time's frames in a seeded random
    thread order.  drop: (time, thread index) frames left out (thread index
    None: every thread of that time); duplicate: (time, thread index) frames
    sent twice with different payloads; extra_thread adds one more thread
    nobody asks for."""
    rng = np.random.default_rng(seed)
    ids = list(thread_ids) if thread_ids is not None else list(range(nthreads))
    fb = payload + 32
    dropped = set(drop)
    frames = []
    for t in range(nframes):
        fr = frame0 + t
        sec = seconds0 + fr // fps
        order = list(range(nthreads)) + ([nthreads] if extra_thread else [])
        if shuffle:
            rng.shuffle(order)
        for j in order:
            if (t, j) in dropped or (t, None) in dropped:
                continue
            tid = ids[j] if j < nthreads else max(ids) + 1
            reps = 2 if (t, j) in duplicate else 1
            for _ in range(reps):
                h = vdif_header_words(sec, fr % fps, epoch, fb, 1, nbits, tid)
                body = rng.integers(0, 256, size=payload, dtype=np.uint8)
                frames.append(np.concatenate([h.view(np.uint8), body]))
    return np.concatenate(frames) if frames else np.zeros(0, dtype=np.uint8)


def raw_read(job: Job, s: int, buf: np.ndarray, rng, drop_frac: float = 0.0, lead_extra: bool = False):
    """The raw multi-thread read a DataStream would hold for station s's
    muxed frames `buf` (one band per thread): every muxed frame split into its
    threads' frames (thread t: band t's samples in time order, the muxed
    header with one channel, the thread's frame size and id t), each time's
    thread frames in a seeded random order, a fraction of thread frames left
    out (incomplete slots), and -- with lead_extra -- a frame of a thread
    nobody asks for one frame time earlier at the front, so that the read's
    first slot is empty and the muxed stream starts one frame in.  Returns the
    bytes and the number of leading frame times (0 or 1)."""
    st = job.stations[s]
    nt, nbits = st.mux_threads, st.nbits
    fb = st.payload_bytes + st.header_bytes
    tp = st.payload_bytes // nt                      # thread payload bytes
    frames = buf.reshape(-1, fb)
    out = []
    lead = 0
    if lead_extra:
        h = frames[0, :32].copy().view(np.uint32)
        secs, fr = int(h[0] & 0x3FFFFFFF), int(h[1] & 0xFFFFFF)
        fps = int(round(2 * job.station_bw(s) * 1e6 / (tp * 8 // nbits)))
        fr -= 1
        if fr < 0:
            fr += fps
            secs -= 1
        e = h.copy()
        e[0] = (e[0] & 0xC0000000) | (secs & 0x3FFFFFFF)
        e[1] = (e[1] & ~np.uint32(0xFFFFFF)) | np.uint32(fr)
        e[2] = (e[2] & ~np.uint32(0x1F << 24) & ~np.uint32(0xFFFFFF)) | np.uint32((tp + 32) // 8)
        e[3] = (e[3] & ~np.uint32(0x3FF << 16)) | np.uint32(nt << 16)      # thread id nt: not wanted
        out.append(np.concatenate([e.view(np.uint8), rng.integers(0, 256, size=tp, dtype=np.uint8)]))
        lead = 1
    per_word = 32 // nbits
    for f in frames:
        h = f[:32].copy().view(np.uint32)
        words = f[32:].view(np.uint32)
        # codes[n, c]: sample n of channel c (LSB-first fields, channels fastest)
        shifts = (np.arange(per_word, dtype=np.uint32) * nbits)
        codes = ((words[:, None] >> shifts[None, :]) & ((1 << nbits) - 1)).reshape(-1, nt)
        order = rng.permutation(nt)
        for t in order:
            if rng.random() < drop_frac:
                continue
            c = codes[:, t].reshape(-1, per_word).astype(np.uint32)
            tw = np.bitwise_or.reduce(c << shifts[None, :], axis=1).astype(np.uint32)
            th = h.copy()
            th[2] = (th[2] & ~np.uint32(0x1F << 24) & ~np.uint32(0xFFFFFF)) | np.uint32((tp + 32) // 8)
            th[3] = (th[3] & ~np.uint32(0x3FF << 16)) | np.uint32(t << 16)
            out.append(np.concatenate([th.view(np.uint8), tw.view(np.uint8)]))
    return np.concatenate(out), lead
