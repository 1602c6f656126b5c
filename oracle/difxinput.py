"""Writer of DiFX job files (.input, .calc, .im, .threads) for a
:class:`fxb200.job.Job`, so that the reference's own parser
(mpifxcorr/src/configuration.cpp:1051-2100, model.cpp:367-856) builds the
same correlation that the product library is given as a C struct.

Oracle test infrastructure.  Section order and keys follow what
Configuration::parseConfiguration reads (configuration.cpp:206-290) and the
format of the job files the reference ships as examples
(sites/MPIfR/oneoff/difx2difx_testset/ma008_1.{input,calc,im}).
"""
from __future__ import annotations

import os

from fxb200.job import Job


def _kv(key: str, val) -> str:
    key = key + ":"
    return "%-20s%s\n" % (key, val)


def write_job_files(job: Job, outdir: str, name: str = "job",
                    xmac_stride: int = 0, array_stride: int = 0,
                    ac_avg_ns: int = 2_000_000_000, uvshift_ns: int = 2_000_000_000,
                    scan_dur_s: int = 100, tsys=None) -> str:
    job.validate()
    os.makedirs(outdir, exist_ok=True)
    base = os.path.join(os.path.abspath(outdir), name)
    nds = len(job.stations)
    nbl = len(job.baselines)
    poly_interval = job.stations[0].polys[0].interval_s if job.stations[0].polys else 120

    # ---------------------------------------------------------------- .input
    s = []
    s.append("# COMMON SETTINGS ##!\n")
    s.append(_kv("CALC FILENAME", base + ".calc"))
    s.append(_kv("CORE CONF FILENAME", base + ".threads"))
    s.append(_kv("EXECUTE TIME (SEC)", scan_dur_s))
    s.append(_kv("START MJD", job.start_mjd))
    s.append(_kv("START SECONDS", job.start_sec))
    s.append(_kv("ACTIVE DATASTREAMS", nds))
    s.append(_kv("ACTIVE BASELINES", nbl))
    s.append(_kv("VIS BUFFER LENGTH", 80))
    s.append(_kv("OUTPUT FORMAT", "SWIN"))
    s.append(_kv("OUTPUT FILENAME", base + ".difx"))
    s.append("\n# CONFIGURATIONS ###!\n")
    s.append(_kv("NUM CONFIGURATIONS", 1))
    s.append(_kv("CONFIG NAME", "fxcfg"))
    s.append(_kv("INT TIME (SEC)", "%.6f" % job.duration_s))
    s.append(_kv("SUBINT NANOSECONDS", job.subint_ns))
    s.append(_kv("GUARD NANOSECONDS", 0))
    s.append(_kv("FRINGE ROTN ORDER", job.fringe_rot_order))
    s.append(_kv("ARRAY STRIDE LENGTH", array_stride))
    s.append(_kv("XMAC STRIDE LENGTH", xmac_stride))
    s.append(_kv("NUM BUFFERED FFTS", job.num_buffered_ffts))
    s.append(_kv("WRITE AUTOCORRS", "TRUE" if job.write_autocorrs else "FALSE"))
    s.append(_kv("PULSAR BINNING", "FALSE"))
    s.append(_kv("PHASED ARRAY", "FALSE"))
    for i in range(nds):
        s.append(_kv("DATASTREAM %d INDEX" % i, i))
    for i in range(nbl):
        s.append(_kv("BASELINE %d INDEX" % i, i))
    s.append("\n# RULES ############!\n")
    s.append(_kv("NUM RULES", 1))
    s.append(_kv("RULE 0 CONFIG NAME", "fxcfg"))
    s.append("\n# FREQ TABLE #######!\n")
    s.append(_kv("FREQ ENTRIES", len(job.freqs)))
    for i, f in enumerate(job.freqs):
        s.append(_kv("FREQ (MHZ) %d" % i, "%.11f" % f.freq_mhz))
        s.append(_kv("BW (MHZ) %d" % i, "%.11f" % f.bw_mhz))
        s.append(_kv("SIDEBAND %d" % i, f.sideband))
        s.append(_kv("NUM CHANNELS %d" % i, f.nchan))
        s.append(_kv("CHANS TO AVG %d" % i, f.chans_to_avg))
        s.append(_kv("OVERSAMPLE FAC. %d" % i, 1))
        s.append(_kv("DECIMATION FAC. %d" % i, 1))
        s.append(_kv("PHASE CALS %d OUT" % i, 0))
    s.append("\n# TELESCOPE TABLE ##!\n")
    s.append(_kv("TELESCOPE ENTRIES", nds))
    for i, st in enumerate(job.stations):
        s.append(_kv("TELESCOPE NAME %d" % i, st.name))
        s.append(_kv("CLOCK REF MJD %d" % i, "%.10f" % job.start_mjd))
        s.append(_kv("CLOCK POLY ORDER %d" % i, 1))
        s.append(_kv("CLOCK COEFF %d/0" % i, "%.15e" % 0.0))
        s.append(_kv("CLOCK COEFF %d/1" % i, "%.15e" % 0.0))
    s.append("\n# DATASTREAM TABLE #!\n")
    s.append(_kv("DATASTREAM ENTRIES", nds))
    s.append(_kv("DATA BUFFER FACTOR", 32))
    s.append(_kv("NUM DATA SEGMENTS", 8))
    for i, st in enumerate(job.stations):
        s.append(_kv("TELESCOPE INDEX", i))
        ts = 0.0 if tsys is None else (tsys[i] if hasattr(tsys, "__len__") else tsys)
        s.append(_kv("TSYS", "%.6f" % ts))
        if st.mux_threads:
            # the frames handed to the Mode are the muxer's; the .input names
            # the threads and their own frame size (configuration.cpp:1517-1525, 1001-1009)
            s.append(_kv("DATA FORMAT", "INTERLACEDVDIF/" + ":".join(str(k) for k in range(st.mux_threads))))
            s.append(_kv("QUANTISATION BITS", st.nbits))
            s.append(_kv("DATA FRAME SIZE", st.payload_bytes // st.mux_threads + st.header_bytes))
        else:
            s.append(_kv("DATA FORMAT", "VDIF"))
            s.append(_kv("QUANTISATION BITS", st.nbits))
            s.append(_kv("DATA FRAME SIZE", st.payload_bytes + st.header_bytes))
        s.append(_kv("DATA SAMPLING", "COMPLEX" if st.complex_sampling else "REAL"))
        s.append(_kv("DATA SOURCE", "FILE"))
        s.append(_kv("FILTERBANK USED", "FALSE"))
        s.append(_kv("PHASE CAL INT (MHZ)", ("%.6f" % st.pcal_interval_mhz) if st.pcal_interval_mhz else 0))
        if st.pcal_base_mhz:
            s.append(_kv("PHASE CAL BASE(MHZ)", "%.6f" % st.pcal_base_mhz))
        rf = st.recorded_freqs()
        s.append(_kv("NUM RECORDED FREQS", len(rf)))
        for j, f in enumerate(rf):
            npol = sum(1 for ff, _ in st.bands if ff == f)
            s.append(_kv("REC FREQ INDEX %d" % j, f))
            clk, dclk, ph, looff = st.freq_corr.get(f, (0.0, 0.0, 0.0, 0.0))
            if dclk or ph:
                s.append(_kv("CLK OFFSET %d (us)" % j, "%.9f:%.9f:%.9f" % (clk, dclk, ph)))
            else:
                s.append(_kv("CLK OFFSET %d (us)" % j, "%.9f" % clk))
            s.append(_kv("FREQ OFFSET %d (Hz)" % j, "%.9f" % looff))
            s.append(_kv("NUM REC POLS %d" % j, npol))
        for k, (f, pol) in enumerate(st.bands):
            s.append(_kv("REC BAND %d POL" % k, pol))
            s.append(_kv("REC BAND %d INDEX" % k, rf.index(f)))
        zf = []
        for f, _ in st.zoom_bands:
            if f not in zf:
                zf.append(f)
        s.append(_kv("NUM ZOOM FREQS", len(zf)))
        for j, f in enumerate(zf):
            s.append(_kv("ZOOM FREQ INDEX %d" % j, f))
            s.append(_kv("NUM ZOOM POLS %d" % j, sum(1 for ff, _ in st.zoom_bands if ff == f)))
        for k, (f, pol) in enumerate(st.zoom_bands):
            s.append(_kv("ZOOM BAND %d POL" % k, pol))
            s.append(_kv("ZOOM BAND %d INDEX" % k, zf.index(f)))
    s.append("\n# BASELINE TABLE ###!\n")
    s.append(_kv("BASELINE ENTRIES", nbl))
    for i, b in enumerate(job.baselines):
        s.append(_kv("D/STREAM A INDEX %d" % i, b.ds1))
        s.append(_kv("D/STREAM B INDEX %d" % i, b.ds2))
        s.append(_kv("NUM FREQS %d" % i, len(b.products)))
        for j, (f, pp) in enumerate(b.products):
            s.append(_kv("POL PRODUCTS %d/%d" % (i, j), len(pp)))
            for k, (b1, b2) in enumerate(pp):
                s.append(_kv("D/STREAM A BAND %d" % k, b1))
                s.append(_kv("D/STREAM B BAND %d" % k, b2))
    s.append("\n# DATA TABLE #######!\n")
    for i in range(nds):
        s.append(_kv("D/STREAM %d FILES" % i, 1))
        s.append(_kv("FILE %d/0" % i, "/dev/null"))
    with open(base + ".input", "w") as fh:
        fh.write("".join(s))

    # -------------------------------------------------------------- .threads
    with open(base + ".threads", "w") as fh:
        fh.write("NUMBER OF CORES:    1\n1\n")

    # ----------------------------------------------------------------- .calc
    mjd = job.start_mjd
    c = []
    c.append(_kv("JOB ID", 1))
    c.append(_kv("JOB START TIME", "%.7f" % (mjd + job.start_sec / 86400.0)))
    c.append(_kv("JOB STOP TIME", "%.7f" % (mjd + (job.start_sec + scan_dur_s) / 86400.0)))
    c.append(_kv("DUTY CYCLE", "1.000"))
    c.append(_kv("OBSCODE", "FXB200"))
    c.append(_kv("DIFX VERSION", "oracle"))
    c.append(_kv("SUBJOB ID", 0))
    c.append(_kv("SUBARRAY ID", 0))
    c.append(_kv("START MJD", "%.7f" % (mjd + job.start_sec / 86400.0)))
    c.append(_kv("START YEAR", 2017))
    c.append(_kv("START MONTH", 9))
    c.append(_kv("START DAY", 4))
    c.append(_kv("START HOUR", job.start_sec // 3600))
    c.append(_kv("START MINUTE", (job.start_sec // 60) % 60))
    c.append(_kv("START SECOND", job.start_sec % 60))
    c.append(_kv("SPECTRAL AVG", 1))
    c.append(_kv("TAPER FUNCTION", "UNIFORM"))
    c.append(_kv("NUM TELESCOPES", nds))
    for i, st in enumerate(job.stations):
        c.append(_kv("TELESCOPE %d NAME" % i, st.name))
        c.append(_kv("TELESCOPE %d MOUNT" % i, "AZEL"))
        c.append(_kv("TELESCOPE %d OFFSET (m)" % i, "0.000000"))
        c.append(_kv("TELESCOPE %d X (m)" % i, "%.6f" % (4000000.0 + 1000.0 * i)))
        c.append(_kv("TELESCOPE %d Y (m)" % i, "%.6f" % (500000.0 + 1000.0 * i)))
        c.append(_kv("TELESCOPE %d Z (m)" % i, "%.6f" % 4900000.0))
        c.append(_kv("TELESCOPE %d SHELF" % i, "NONE"))
    c.append(_kv("NUM SOURCES", 1))
    c.append(_kv("SOURCE 0 NAME", "SRC"))
    c.append(_kv("SOURCE 0 RA", " 3.3867508046241599"))
    c.append(_kv("SOURCE 0 DEC", "-0.1010425645421680"))
    c.append(_kv("SOURCE 0 CALCODE", " "))
    c.append(_kv("SOURCE 0 QUAL", 0))
    c.append(_kv("NUM SCANS", 1))
    c.append(_kv("SCAN 0 IDENTIFIER", "No0001"))
    c.append(_kv("SCAN 0 START (S)", 0))
    c.append(_kv("SCAN 0 DUR (S)", scan_dur_s))
    c.append(_kv("SCAN 0 OBS MODE NAME", "fxcfg"))
    c.append(_kv("SCAN 0 UVSHIFT INTERVAL (NS)", uvshift_ns))
    c.append(_kv("SCAN 0 AC AVG INTERVAL (NS)", ac_avg_ns))
    c.append(_kv("SCAN 0 POINTING SRC", 0))
    c.append(_kv("SCAN 0 NUM PHS CTRS", 1))
    c.append(_kv("SCAN 0 PHS CTR 0", 0))
    c.append(_kv("NUM EOPS", 0))
    c.append(_kv("NUM SPACECRAFT", 0))
    c.append(_kv("IM FILENAME", base + ".im"))
    c.append(_kv("FLAG FILENAME", base + ".flag"))
    with open(base + ".calc", "w") as fh:
        fh.write("".join(c))
    with open(base + ".flag", "w") as fh:
        fh.write("0\n")

    # ------------------------------------------------------------------- .im
    npoly_per_scan = max(1, -(-scan_dur_s // poly_interval))
    order = 5
    m = []
    m.append(_kv("CALC SERVER", "none"))
    m.append(_kv("CALC PROGRAM", -1))
    m.append(_kv("CALC VERSION", -1))
    m.append(_kv("START YEAR", 2017))
    m.append(_kv("START MONTH", 9))
    m.append(_kv("START DAY", 4))
    m.append(_kv("START HOUR", job.start_sec // 3600))
    m.append(_kv("START MINUTE", (job.start_sec // 60) % 60))
    m.append(_kv("START SECOND", job.start_sec % 60))
    m.append(_kv("POLYNOMIAL ORDER", order))
    m.append(_kv("INTERVAL (SECS)", poly_interval))
    m.append(_kv("ABERRATION CORR", "EXACT"))
    m.append(_kv("NUM TELESCOPES", nds))
    for i, st in enumerate(job.stations):
        m.append(_kv("TELESCOPE %d NAME" % i, st.name))
    m.append(_kv("NUM SCANS", 1))
    m.append(_kv("SCAN 0 POINTING SRC", "SRC"))
    m.append(_kv("SCAN 0 NUM PHS CTRS", 1))
    m.append(_kv("SCAN 0 PHS CTR 0 SRC", "SRC"))
    m.append(_kv("SCAN 0 NUM POLY", npoly_per_scan))

    def row(vals):
        return "\t".join("% .16e" % v for v in vals)

    for j in range(npoly_per_scan):
        t0 = j * poly_interval
        m.append(_kv("SCAN 0 POLY %d MJD" % j, mjd))
        m.append(_kv("SCAN 0 POLY %d SEC" % j, job.start_sec + t0))
        for src in range(2):
            for i, st in enumerate(job.stations):
                coeffs = _poly_for(st, t0, order)
                m.append(_kv("SRC %d ANT %d DELAY (us)" % (src, i), row(coeffs)))
                m.append(_kv("SRC %d ANT %d U (m)" % (src, i), row([0.0] * (order + 1))))
                m.append(_kv("SRC %d ANT %d V (m)" % (src, i), row([0.0] * (order + 1))))
                m.append(_kv("SRC %d ANT %d W (m)" % (src, i), row([0.0] * (order + 1))))
    with open(base + ".im", "w") as fh:
        fh.write("".join(m))
    return base + ".input"


def _poly_for(st, t0: float, order: int):
    """Coefficients (order+1) of the station polynomial re-expanded about t0."""
    for p in st.polys:
        if p.start_sec <= t0 < p.start_sec + p.interval_s or len(st.polys) == 1:
            # shift p(t) = sum c_k (t - s)^k to q(u) = p(u + t0), u = t - t0
            import math
            d = t0 - p.start_sec
            out = [0.0] * (order + 1)
            for k, ck in enumerate(p.coeffs):
                for r in range(k + 1):
                    if r <= order:
                        out[r] += ck * math.comb(k, r) * d ** (k - r)
            out[0] += st.clock_us
            return out
    raise ValueError("no polynomial covers t0")
