"""Correlation job description.

A job mirrors the tables that the reference reads from a DiFX ``.input`` file
(mpifxcorr/src/configuration.cpp: FREQ TABLE :1982-2052, DATASTREAM TABLE
:1433-1800, BASELINE TABLE :1059-1120, CONFIGURATIONS :1349-1430) for the one
configuration this hot path correlates:

* ``freqs``     -- the frequency table (sky frequency of the band edge, width,
                   sideband, channel count);
* ``stations``  -- one datastream per station: VDIF framing, bits per sample,
                   recorded bands (frequency-table index and polarisation) in
                   VDIF channel order, delay model;
* ``baselines`` -- station pairs with, per frequency, the list of
                   (band of station A, band of station B) polarisation products.

The product library receives this as the plain C struct declared in
include/fxb200.h (built by :func:`Job.to_native`).
"""
from __future__ import annotations

import dataclasses
import math
from typing import List, Sequence, Tuple


@dataclasses.dataclass
class Freq:
    freq_mhz: float          # sky frequency of the band edge (LO), MHz
    bw_mhz: float            # bandwidth, MHz
    nchan: int               # output channels (FFT length is 2*nchan)
    sideband: str = "U"      # 'U' or 'L'
    chans_to_avg: int = 1


@dataclasses.dataclass
class DelayPoly:
    """Per-station delay polynomial in the ``.im`` convention
    (mpifxcorr/src/model.cpp:229-299): delay(us) = sum_k c[k] * dt**k with dt
    the seconds since ``start_sec`` (seconds after the job start), valid for
    ``interval_s`` seconds.  A station may carry several consecutive polys."""
    start_sec: float
    interval_s: int
    coeffs: Tuple[float, ...]


@dataclasses.dataclass
class Station:
    name: str
    bands: List[Tuple[int, str]]      # (freq index, pol) in VDIF channel order
    nbits: int = 2
    payload_bytes: int = 8000
    header_bytes: int = 32
    polys: List[DelayPoly] = dataclasses.field(default_factory=list)
    clock_us: float = 0.0             # constant clock offset folded into the model
    # zoom bands (freq index, pol): channel windows of a recorded band of the
    # same polarisation; a baseline names zoom band z as band nband + z
    zoom_bands: List[Tuple[int, str]] = dataclasses.field(default_factory=list)
    # phase-cal comb: tones every pcal_interval_mhz (0: no extraction),
    # shifted by pcal_base_mhz
    pcal_interval_mhz: float = 0.0
    pcal_base_mhz: float = 0.0
    # INTERLACEDVDIF: threads of one band each muxed into the frames (0: plain
    # VDIF); data weights are then per band, and EDV4 validity masks in the
    # frame headers blank absent bands
    mux_threads: int = 0
    # per recorded frequency (freq index -> (clock offset us, R/L clock delta
    # us, phase offset degrees, LO offset Hz)): the datastream table's
    # "CLK OFFSET n (us)" = offset[:delta[:phase]] and "FREQ OFFSET n (Hz)"
    freq_corr: dict = dataclasses.field(default_factory=dict)
    # INTERLACEDVDIF: the buffers are the raw reads (the threads' own frames,
    # placed and read inside the F stage) rather than the muxer's output;
    # thread id of each band's thread (empty: 0, 1, ..)
    mux_raw: bool = False
    mux_thread_ids: List[int] = dataclasses.field(default_factory=list)
    # complex (single-sideband) sampling: bw complex samples per second per
    # band, real and imaginary fields side by side (DATA SAMPLING COMPLEX)
    complex_sampling: bool = False

    def band_corr(self, b: int) -> Tuple[float, float, float, float]:
        """(clock us, clock delta us, phase deg, LO offset Hz) of band b's frequency."""
        return tuple(self.freq_corr.get(self.bands[b][0], (0.0, 0.0, 0.0, 0.0)))

    def recorded_freqs(self) -> List[int]:
        seen: List[int] = []
        for f, _ in self.bands:
            if f not in seen:
                seen.append(f)
        return seen

    @property
    def nband(self) -> int:
        return len(self.bands)

    def band(self, b: int) -> Tuple[int, str]:
        """(freq index, pol) of band b: recorded bands, then zoom bands."""
        return self.bands[b] if b < len(self.bands) else self.zoom_bands[b - len(self.bands)]


@dataclasses.dataclass
class Baseline:
    ds1: int
    ds2: int
    # per frequency index: list of (band index in ds1, band index in ds2)
    products: List[Tuple[int, List[Tuple[int, int]]]]


@dataclasses.dataclass
class Job:
    freqs: List[Freq]
    stations: List[Station]
    baselines: List[Baseline]
    subint_ns: int
    start_mjd: int = 58000
    start_sec: int = 0
    fringe_rot_order: int = 1
    num_buffered_ffts: int = 10
    write_autocorrs: bool = True
    duration_s: float = 1.0

    # ---- derived quantities -------------------------------------------------
    def station_bw(self, s: int) -> float:
        return self.freqs[self.stations[s].bands[0][0]].bw_mhz

    def station_nchan(self, s: int) -> int:
        return self.freqs[self.stations[s].bands[0][0]].nchan

    def fft_ns(self) -> float:
        f = self.freqs[self.stations[0].bands[0][0]]
        return 2 * f.nchan * 1e3 / (2 * f.bw_mhz)

    def blocks_per_send(self) -> int:
        n = self.subint_ns / self.fft_ns()
        if abs(n - round(n)) > 1e-9:
            raise ValueError("subint must hold a whole number of FFTs")
        return int(round(n))

    def samples_per_sec(self, s: int) -> int:
        k = 1 if self.stations[s].complex_sampling else 2
        return int(round(k * 1e6 * self.station_bw(s)))

    def frame_samples(self, s: int) -> int:
        st = self.stations[s]
        k = 2 if st.complex_sampling else 1
        return st.payload_bytes * 8 // (st.nbits * st.nband * k)

    def frame_bytes(self, s: int) -> int:
        st = self.stations[s]
        return st.payload_bytes + st.header_bytes

    def frames_per_sec(self, s: int) -> int:
        return self.samples_per_sec(s) // self.frame_samples(s)

    def mbps(self, s: int) -> int:
        st = self.stations[s]
        k = 2 if st.complex_sampling else 1
        return int(round(self.samples_per_sec(s) * st.nbits * st.nband * k / 1e6))

    def vdif_format(self, s: int) -> str:
        st = self.stations[s]
        return "VDIF%s_%d-%d-%d-%d" % ("C" if st.complex_sampling else "", st.payload_bytes, self.mbps(s), st.nband,
                                        st.nbits)

    def max_products(self) -> int:
        return max(len(pp) for b in self.baselines for _, pp in b.products)

    def used_freqs(self) -> List[int]:
        used = set()
        for b in self.baselines:
            for f, _ in b.products:
                used.add(f)
        return sorted(used)

    def station_mhz_per_sec(self) -> float:
        """N_station x sum of recorded band widths (each polarisation counted),
        i.e. the station.MHz processed per second of data."""
        return sum(self.freqs[f].bw_mhz for st in self.stations for f, _ in st.bands)

    def packed_bytes_per_sec(self) -> float:
        tot = 0.0
        for s in range(len(self.stations)):
            tot += self.frames_per_sec(s) * self.frame_bytes(s)
        return tot

    def validate(self) -> None:
        nfft = None
        for s, st in enumerate(self.stations):
            bws = {self.freqs[f].bw_mhz for f, _ in st.bands}
            nch = {self.freqs[f].nchan for f, _ in st.bands}
            if len(bws) != 1 or len(nch) != 1:
                raise ValueError("all bands of one station share bandwidth and channel count")
            if st.nbits not in (2, 8):
                raise ValueError("2-bit and 8-bit VDIF are supported")
            if (st.payload_bytes * 8) % (st.nbits * st.nband):
                raise ValueError("payload must hold whole samples")
            if self.samples_per_sec(s) % self.frame_samples(s):
                raise ValueError("whole frames per second required")
            for f, pol in st.zoom_bands:
                if self.zoom_parent(s, f, pol) is None:
                    raise ValueError("zoom band outside every recorded band of its polarisation")
        for b in self.baselines:
            for f, pp in b.products:
                for b1, b2 in pp:
                    if self.stations[b.ds1].band(b1)[0] != f or self.stations[b.ds2].band(b2)[0] != f:
                        raise ValueError("product bands must record the baseline frequency")
        self.blocks_per_send()

    def zoom_parent(self, s: int, f: int, pol: str):
        """(recorded band index, channel offset) of station s's zoom band on
        frequency f in pol: the last recorded frequency whose range contains
        the zoom band, its band of the same polarisation, and the offset of the
        zoom band edge in parent channels (configuration.cpp:1734-1754)."""
        st = self.stations[s]
        z = self.freqs[f]
        lo = z.freq_mhz - (z.bw_mhz if z.sideband == "L" else 0.0)
        parent = None
        for rf in st.recorded_freqs():
            p = self.freqs[rf]
            plo = p.freq_mhz - (p.bw_mhz if p.sideband == "L" else 0.0)
            if lo + z.bw_mhz <= plo + p.bw_mhz and lo >= plo:
                parent = rf
        if parent is None:
            return None
        r0 = self.freqs[st.bands[0][0]]
        p = self.freqs[parent]
        plo = p.freq_mhz - (p.bw_mhz if p.sideband == "L" else 0.0)
        off = int((lo - plo) / r0.bw_mhz * r0.nchan + 0.5)
        for k, (ff, pp) in enumerate(st.bands):
            if ff == parent and pp == pol:
                return k, off
        return None


def full_job(nstation: int, freqs: Sequence[Freq], pols: str = "RL", full_pol: bool = True,
             subint_ns: int = 8_000_000, nbits: int = 2, **kw) -> Job:
    """All stations record every frequency in every polarisation; every station
    pair forms a baseline with parallel hands (and cross hands when full_pol).
    Product order per frequency follows vex2difx: RR, RL, LR, LL."""
    stations = []
    for s in range(nstation):
        bands = [(f, p) for f in range(len(freqs)) for p in pols]
        stations.append(Station(name="S%02d" % s, bands=bands, nbits=nbits))
    baselines = []
    for a in range(nstation):
        for b in range(a + 1, nstation):
            prods = []
            for f in range(len(freqs)):
                idx = {p: i for i, (ff, p) in enumerate(stations[a].bands) if ff == f}
                pp = []
                for p1 in pols:
                    for p2 in pols:
                        if p1 == p2 or full_pol:
                            pp.append((idx[p1], idx[p2]))
                # vex2difx order: parallel hands first, then cross hands
                par = [x for x in pp if stations[a].bands[x[0]][1] == stations[b].bands[x[1]][1]]
                cross = [x for x in pp if x not in par]
                if full_pol and len(pols) == 2:
                    pp = [par[0], cross[0], cross[1], par[1]]
                else:
                    pp = par + cross
                prods.append((f, pp))
            baselines.append(Baseline(ds1=a, ds2=b, products=prods))
    return Job(freqs=list(freqs), stations=stations, baselines=baselines, subint_ns=subint_ns, **kw)


def ceil_div(a: int, b: int) -> int:
    return -(-a // b)


def gcd_list(v: Sequence[int]) -> int:
    g = 0
    for x in v:
        g = math.gcd(g, x)
    return g


def add_zoom_bands(job: Job, zooms: Sequence[Tuple[int, float, float]], keep_parents: bool = True,
                   chans_to_avg: int = 1) -> Job:
    """Append zoom frequencies to a job, as vex2difx writes them.

    Each (parent freq index, offset MHz, width MHz) becomes a frequency-table
    entry after the recorded ones, with the parent's channel width.  Every
    station that records the parent gets one zoom band per recorded
    polarisation, in the parent bands' order.  Every baseline correlates the
    zoom frequency with the parent frequency's products mapped onto the zoom
    bands.  Without keep_parents the parents' own products are dropped, so
    that only the zoom windows are correlated."""
    nrec = len(job.freqs)
    zfreqs = []
    for parent, off, bw in zooms:
        p = job.freqs[parent]
        nchan = int(round(bw / p.bw_mhz * p.nchan))
        job.freqs.append(Freq(p.freq_mhz + off, bw, nchan, p.sideband, chans_to_avg))
        zfreqs.append((parent, len(job.freqs) - 1))
    zindex = []                      # per station: {(parent, band): zoom band index}
    for st in job.stations:
        m = {}
        for parent, zf in zfreqs:
            for k, (f, pol) in enumerate(st.bands):
                if f == parent:
                    m[(parent, zf, k)] = st.nband + len(st.zoom_bands)
                    st.zoom_bands.append((zf, pol))
        zindex.append(m)
    for b in job.baselines:
        prods = [x for x in b.products if keep_parents or x[0] >= nrec]
        for parent, zf in zfreqs:
            for f, pp in b.products:
                if f == parent:
                    prods.append((zf, [(zindex[b.ds1][(parent, zf, b1)], zindex[b.ds2][(parent, zf, b2)])
                                       for b1, b2 in pp]))
        b.products = prods
    return job
