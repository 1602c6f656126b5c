#!/usr/bin/env python
"""Throughput of the FX hot path on the 10-station production workload.

Workload (config c1): 10 stations, eight 32 MHz bands, dual polarisation with
full cross hands, 2-bit VDIF (8000-byte payload, 16 channels per frame),
1024 channels (2048-point FFTs), 8 ms subintegrations, fringe rotation order 1.
One step = 125 subintegrations = 1 s of data for every station.

  python bench.py [--gpus N] [--steps K] [--warmup W] [--impl fxb|reference]

Prints one JSON line: value = station.MHz/s processed (whole job, all GPUs)
by the headline form -- by default the tensor-core form (FP16 FFT, BF16
spectra, tcgen05 XMAC with FP32 accumulation; --xmac fp32 selects the plain
FP32 form) -- with the real-time factor, the other form measured beside it on
the same workload (other_form, tc_vs_fp32), the end-to-end figure through the
C ABI with host buffers (host->device copies of the raw VDIF and the
device->host read of the core result inside the timed region), the rooflines
of the F stage (HBM) and of the XMAC (tensor pipe), the reference CPU baseline
and the SM clocks seen during the timed region.

Inputs: a pool of 16 distinct subintegrations per station (bulk synthetic
VDIF with the 2-bit quantiser's code statistics, 327 MB in device memory,
larger than the 126 MB L2) cycled through in every step.
"""
from __future__ import annotations

import argparse
import csv
import io
import json
import os
import statistics
import subprocess
import sys
import tempfile
import time

ROOT = os.path.dirname(os.path.abspath(__file__))
for p in (os.path.join(ROOT, "difx-svn2git-try3_b200"), os.path.join(ROOT, "oracle")):
    if p not in sys.path:
        sys.path.insert(0, p)

import numpy as np  # noqa: E402

from fxb200 import configs, shard, synth  # noqa: E402

METRIC = "real-time factor & station.MHz/s (FX: unpack + fringe rotation + FFT + frac-sample + XMAC)"
UNIT = "station.MHz/s"
POOL = 16


def parse():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=5)
    ap.add_argument("--warmup", type=int, default=3)
    ap.add_argument("--impl", default="fxb", choices=["fxb", "reference"])
    ap.add_argument("--xmac", default="fp16", choices=["fp32", "fp16", "bf16"],
                    help="headline form: fp16 = tensor-core form (FP16 spectra, tcgen05 XMAC with FP32 "
                         "accumulation), bf16 = the same with BF16 spectra, fp32 = the plain FP32 form; the "
                         "other form (FP32, or fp16 when the headline is FP32) is measured beside it")
    ap.add_argument("--no-other-form", "--no-tc-form", dest="no_other_form", action="store_true",
                    help="skip measuring the other form beside the headline")
    ap.add_argument("--subints-per-step", type=int, default=125)
    ap.add_argument("--no-cpu-baseline", action="store_true")
    ap.add_argument("--no-serving", action="store_true", help="skip the serving leg (p50/p99 job latency)")
    ap.add_argument("--no-c3", action="store_true", help="skip the batched uneven-subband leg")
    ap.add_argument("--no-mux", action="store_true", help="skip the INTERLACEDVDIF muxing leg")
    ap.add_argument("--no-features", action="store_true", help="skip the phase-cal and zoom-band legs")
    ap.add_argument("--serving-jobs", type=int, default=12)
    ap.add_argument("--c3-only", choices=["branches", "fused", "per-job"], default=None,
                    help="profiling aid: run only the c3 batch in one form for --warmup + --steps subints "
                         "(no timing) and print one record")
    return ap.parse_args()


def c3_only(args):
    """The c3 leg in one form, for launch lists and captures of its kernels."""
    import torch
    from fxb200.native import Batch, Correlator
    jobs = configs.c3()
    pools = [make_pool(j, 1, seed=7 + m) for m, j in enumerate(jobs)]
    dev = [[torch.from_numpy(b).to("cuda") for b, _, _ in pool[0][1]] for pool in pools]
    meta = [([t.data_ptr() for t in dev[m]], [b.size for b, _, _ in pools[m][0][1]],
             [x for _, x, _ in pools[m][0][1]], [x for _, _, x in pools[m][0][1]]) for m in range(len(jobs))]
    when = pools[0][0][0]
    members = [Correlator(j, xmac="fp16", inflight=3) for j in jobs]
    batch = None if args.c3_only == "per-job" else Batch(members)
    fused = batch.set_fused(args.c3_only == "fused") if batch is not None else False
    for _ in range(args.warmup + args.steps):
        if batch is not None:
            batch.submit_device(meta, *when)
        else:
            for m, c in enumerate(members):
                c.submit_device(*meta[m], *when)
    if batch is not None:
        batch.sync()
        batch.close()
    for m in members:
        m.sync()
        m.close()
    print(json.dumps({"c3_only": args.c3_only, "fused": fused, "subints": args.warmup + args.steps}))


def subint_time(job, k):
    ns_total = k * job.subint_ns
    return ns_total // 1_000_000_000, ns_total % 1_000_000_000


def make_pool(job, npool, seed=1):
    """Per pool entry: per station (bytes, datasec, datans) and the subint time."""
    pool = []
    for k in range(npool):
        sec, ns = subint_time(job, k + 1)          # start one subint in: delays need earlier data
        inputs = []
        for s in range(len(job.stations)):
            f0, nf, dsec, dns = synth.subint_window(job, s, sec, ns)
            inputs.append((synth.bulk_station_frames(job, s, f0, nf, seed), dsec, dns))
        pool.append(((sec, ns), inputs))
    return pool


# ---------------------------------------------------------------- clocks
class ClockSampler:
    FIELDS = ("index,clocks.sm,clocks.max.sm,power.draw,utilization.gpu,clocks_event_reasons.active,"
              "clocks_event_reasons.hw_slowdown,clocks_event_reasons.hw_thermal_slowdown,"
              "clocks_event_reasons.sw_thermal_slowdown,clocks_event_reasons.sw_power_cap")

    def __init__(self, index):
        self.index = index
        self.proc = None
        self.path = None

    def start(self):
        try:
            fd, self.path = tempfile.mkstemp(suffix=".csv")
            os.close(fd)
            self.fh = open(self.path, "w")
            self.proc = subprocess.Popen(["nvidia-smi", "-i", str(self.index), "--query-gpu=" + self.FIELDS,
                                          "--format=csv,noheader,nounits", "-lms", "200"],
                                         stdout=self.fh, stderr=subprocess.DEVNULL)
        except Exception:
            self.proc = None

    def stop(self):
        if self.proc is None:
            return None
        self.proc.terminate()
        try:
            self.proc.wait(timeout=5)
        except Exception:
            self.proc.kill()
        self.fh.close()
        rows = []
        with open(self.path) as fh:
            for r in csv.reader(fh):
                if len(r) >= 10:
                    rows.append([x.strip() for x in r])
        os.unlink(self.path)
        if not rows:
            return None

        def num(x):
            try:
                return float(x)
            except ValueError:
                return float("nan")
        load = [r for r in rows if num(r[4]) >= 50.0] or rows
        sm = [num(r[1]) for r in load if num(r[1]) == num(r[1])]
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        reasons = sorted({names[i] for r in load for i in range(4) if r[6 + i].lower().startswith("active")})
        return {"sm_mhz": statistics.median(sm) if sm else None, "sm_max_mhz": num(rows[0][2]),
                "samples": len(rows), "samples_under_load": len(load), "reasons": reasons,
                "power_w_max": max(num(r[3]) for r in rows)}


# ---------------------------------------------------------------- reference CPU path
# One CPU sample definition for both arms: CPU_SAMPLE_SUBINTS consecutive
# subints of the workload (cycling a pool of distinct subints) through one
# reference correlator that has already processed one untimed subint.
CPU_SAMPLE_SUBINTS = 24


class CpuReference:
    """The reference's own compiled CPU path (oracle/_ref) -- or, where it was
    not built, the oracle's C restatement on one thread -- set up once for
    the workload."""

    def __init__(self, job, pool, nthreads):
        import refcorr
        self.job, self.pool = job, pool
        self.vf = [synth.valid_flags(job) for _ in job.stations]
        if refcorr.available():
            self.ref = refcorr.RefCorrelator(job, nthreads=nthreads)
            self.kind, self.cores, self.nthreads = "reference", nthreads, nthreads
            self.out = np.zeros(2 * self.ref.corelen, dtype=np.float32)
        else:
            import fxoracle
            self.ref = fxoracle.OracleCorrelator(job)
            self.kind, self.cores, self.nthreads = "port", 1, 1
        self.k = 0
        self.one()                       # untimed: first-call set-up

    def one(self):
        (sec, ns), inputs = self.pool[self.k % len(self.pool)]
        self.k += 1
        if self.kind == "reference":
            self.ref.process_subint(inputs, self.vf, 0, sec, ns, coreresult=self.out, nthreads=self.nthreads)
        else:
            self.ref.process_subint(inputs, sec, ns, validflags=self.vf)

    def sample(self, nsub=CPU_SAMPLE_SUBINTS):
        """Seconds of wall time for nsub subints, and the per-subint times."""
        per = []
        t0 = time.perf_counter()
        for _ in range(nsub):
            t1 = time.perf_counter()
            self.one()
            per.append(time.perf_counter() - t1)
        return time.perf_counter() - t0, per

    def close(self):
        if self.kind == "reference":
            self.ref.close()

    def describe(self, nsub, dt, per):
        data_s = nsub * self.job.subint_ns * 1e-9
        return ("%d consecutive subints x %.0f ms of the workload (%.3f s of data) through one reference "
                "correlator after one untimed subint, %d host threads: %.2f s wall; per subint min/median/max "
                "%.0f/%.0f/%.0f ms" % (nsub, self.job.subint_ns / 1e6, data_s, self.nthreads, dt,
                                        1e3 * min(per), 1e3 * statistics.median(per), 1e3 * max(per)))


def cpu_reference(job, pool, nthreads):
    """One CPU sample; returns (station.MHz/s, cores, sample text, kind)."""
    cr = CpuReference(job, pool, nthreads)
    dt, per = cr.sample()
    cr.close()
    data_s = CPU_SAMPLE_SUBINTS * job.subint_ns * 1e-9
    return job.station_mhz_per_sec() * data_s / dt, cr.cores, cr.describe(CPU_SAMPLE_SUBINTS, dt, per), cr.kind


def reference_arm(args, job):
    """The reference's CPU implementation of the path on all host threads:
    each step is one CPU sample (CPU_SAMPLE_SUBINTS subints of the workload,
    the same definition as the GPU arm's cpu_baseline); ms_per_step is the
    measured wall time of a step."""
    rank = int(os.environ.get("RANK", "0"))
    if rank != 0:
        return
    pool = make_pool(job, 8)
    nthreads = os.cpu_count() or 1
    cr = CpuReference(job, pool, nthreads)
    for _ in range(args.warmup):
        cr.sample()
    dts, per_all = [], []
    for _ in range(args.steps):
        dt, per = cr.sample()
        dts.append(dt)
        per_all += per
    cr.close()
    data_step = CPU_SAMPLE_SUBINTS * job.subint_ns * 1e-9
    value = job.station_mhz_per_sec() * data_step * len(dts) / sum(dts)
    rtf = value / job.station_mhz_per_sec()
    sample = cr.describe(CPU_SAMPLE_SUBINTS * len(dts), sum(dts), per_all)
    line = {
        "metric": METRIC, "value": value, "unit": UNIT, "impl": "reference", "n_gpus": args.gpus,
        "steps": args.steps, "warmup": args.warmup, "ms_per_step": 1e3 * sum(dts) / len(dts),
        "higher_is_better": True, "scaling": "weak", "vs_baseline": None, "dtype": "f32",
        "data": "synthetic", "rtf": rtf, "data_seconds_per_step": data_step,
        "config": workload_config(job),
        "cpu_baseline": {"value": value, "unit": UNIT, "cores": cr.cores, "kind": cr.kind, "sample": sample},
        "e2e": {"value": value, "unit": UNIT, "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0},
    }
    print(json.dumps(line), flush=True)


def workload_config(job):
    return {"workload": "c1: 10 stations x 8 x 32 MHz x 2 pol (full cross hands), 2-bit VDIF 16ch, "
                        "1024 channels, 8 ms subints (GPU arm: 1 s of data per step; reference arm: "
                        "%d subints per step)" % CPU_SAMPLE_SUBINTS,
            "stations": len(job.stations), "subbands": len(job.freqs), "bw_mhz": job.freqs[0].bw_mhz,
            "nchan": job.freqs[0].nchan, "fringe_rot_order": job.fringe_rot_order,
            "subint_ms": job.subint_ns / 1e6, "l2": "inputs larger than L2 (327 MB pool cycled)",
            "parallelism": "time-sharded subints, one process per GPU"}


def load_traffic(kernel):
    path = os.path.join(ROOT, "profiles", "traffic.json")
    try:
        with open(path) as fh:
            return json.load(fh).get(kernel)
    except Exception:
        return None


def h2d_link_gbs(blocks=None):
    """Host-to-device copy bandwidth from page-locked memory, the ceiling of
    the end-to-end figure: the given page-locked blocks (the end-to-end path's
    own subint blocks, one copy each) or 256 MB copied as 16 MB pieces, back
    to back on one stream; best of 10 after an untimed round that maps the
    buffers."""
    import torch
    if blocks is None:
        n, piece = 256 << 20, 16 << 20
        src = torch.empty(n, dtype=torch.uint8).pin_memory()
        blocks = [src[o:o + piece] for o in range(0, n, piece)]
    dst = torch.empty(max(b.numel() for b in blocks), dtype=torch.uint8, device="cuda")
    total = sum(b.numel() for b in blocks)

    def once():
        for b in blocks:
            dst[:b.numel()].copy_(b, non_blocking=True)

    once()
    torch.cuda.synchronize()
    best = 0.0
    for _ in range(10):
        e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        e0.record()
        once()
        e1.record()
        e1.synchronize()
        best = max(best, total / (e0.elapsed_time(e1) * 1e-3) / 1e9)
    del dst
    return best


def load_peaks():
    """(HBM GB/s, burst dense bf16 TFLOP/s, sustained dense bf16 TFLOP/s, source)."""
    try:
        with open(os.path.join(ROOT, "MEASURED_PEAKS.json")) as fh:
            p = json.load(fh)
        return (float(p["hbm_gbs"]), float(p["bf16_tflops"]), float(p.get("bf16_tflops_sustained", 0.0)) or None,
                "measured")
    except Exception:
        return 6650.0, 1590.0, 1400.0, "fallback"


# ---------------------------------------------------------------- serving leg
def serving_leg(args):
    """p50/p99 job latency and sustained throughput of the serving loop on a
    seeded Poisson stream of jobs drawn from the serving workload's ranges
    (4-32 stations, 1-16 subbands of 8-64 MHz, 256-8192 channels, 0.1-2 s
    integrations, dual polarisation with cross hands).  Each job's subints
    cycle three distinct subints of page-locked VDIF with their own times
    (serving.job_subints pool=3), so that a 2 s job of the largest shape
    (66 GB of VDIF) needs under 1 GB of host memory; every byte is still
    copied to the device per subint."""
    from fxb200 import serving
    rng = np.random.default_rng(11)
    jobs = []
    for k in range(args.serving_jobs):
        job, nsub = serving.serving_job(rng, seed=100 + k, stations=(4, 32), subbands=(1, 16),
                                        bws=(8.0, 16.0, 32.0, 64.0), nchans=(256, 512, 1024, 2048, 4096, 8192),
                                        seconds=(0.1, 2.0))
        jobs.append((job, serving.job_subints(job, nsub, seed=100 + k, pinned=True, pool=3)))
    rate = 20.0
    arrivals = serving.poisson_arrivals(rng, len(jobs), rate)
    srv = serving.Server(budget_bytes=96 << 30, max_active=4)
    st = serving.run_stream(srv, jobs, arrivals, xmac=args.xmac)
    phases = [srv.job_times(h) for h in srv.jobs]
    srv.close()
    phase_p50 = {k: float(np.median([p[k] for p in phases])) for k in phases[0]} if phases else {}
    smhz = sum(job.station_mhz_per_sec() * len(subs) * job.subint_ns * 1e-9 for job, subs in jobs)
    h2d = sum(b.nbytes for _, subs in jobs for inputs, _, _ in subs for b, _, _ in inputs)
    shapes = [(len(j.stations), len(j.freqs), j.freqs[0].bw_mhz, j.freqs[0].nchan,
               round(len(subs) * j.subint_ns * 1e-9, 3)) for j, subs in jobs]
    link = h2d_link_gbs()
    h2d_gbs = h2d / 1e9 / st["wall_seconds"] if st["wall_seconds"] > 0 else None
    return {"jobs": st["completed"], "p50_ms": st["p50_ms"], "p99_ms": st["p99_ms"],
            "rtf": st["rtf"], "station_mhz_per_s": smhz / st["wall_seconds"] if st["wall_seconds"] > 0 else None,
            "arrival_rate_hz": rate, "max_active": 4, "hbm_budget_gb": 96, "xmac": args.xmac,
            "phase_ms_p50": phase_p50, "h2d_gb": h2d / 1e9, "h2d_gbs": h2d_gbs, "h2d_link_gbs": link,
            "h2d_link_frac": (h2d_gbs / link) if (h2d_gbs and link) else None,
            "data_seconds": st["data_seconds"], "shapes": shapes,
            "sample": "%d seeded jobs, Poisson arrivals at %.0f/s; 4-32 stations, 1-16 subbands of 8-64 MHz, "
                      "256-8192 channels, 0.1-2 s each, dual pol with cross hands; station buffers in "
                      "page-locked host memory (three distinct subints per job, cycled with their own times); "
                      "latency = submit to core result in host memory" % (len(jobs), rate)}


# ---------------------------------------------------------------- batched uneven subbands
def c3_leg(args):
    """The c3 batch (20 stations, 16 subbands of mixed width, channels and
    bits as 12 jobs) with device-resident inputs: the tensor-core form as one
    batch (one CUDA graph launch per subint), the tensor-core form job by job
    and the plain FP32 form job by job (kernels launched one by one), each
    timed with CUDA events that bracket every stream involved."""
    import torch
    from fxb200.native import Batch, Correlator
    jobs = configs.c3()
    npool, nsub = 3, 16
    pools = [make_pool(j, npool, seed=7 + m) for m, j in enumerate(jobs)]
    dev = [[[torch.from_numpy(b).to("cuda") for b, _, _ in inputs] for (_, inputs) in pool] for pool in pools]
    meta = [[([t.data_ptr() for t in dev[m][k]], [b.size for b, _, _ in pools[m][k][1]],
              [x for _, x, _ in pools[m][k][1]], [x for _, _, x in pools[m][k][1]]) for k in range(npool)]
            for m in range(len(jobs))]
    times = [t for (t, _) in pools[0]]
    smhz = sum(j.station_mhz_per_sec() for j in jobs)
    data_s = args.steps * nsub * jobs[0].subint_ns * 1e-9

    def run(form, batched, fused=True):
        members = [Correlator(j, xmac=form, inflight=3) for j in jobs]
        batch = Batch(members) if batched else None
        is_fused = batch.set_fused(fused) if batched else False
        # scheduling tuned online during the warm-up subints (results unchanged)
        for m in members:
            m.autotune(2)
        # a batch's XMACs may run on a second stream; the members' streams
        # are ordered after every batch launch
        streams = ([torch.cuda.ExternalStream(batch.stream())] if batched else []) + \
            [torch.cuda.ExternalStream(m.stream()) for m in members]

        def step():
            for j in range(nsub):
                k = j % npool
                if batched:
                    batch.submit_device([meta[m][k] for m in range(len(jobs))], *times[k])
                else:
                    for m, c in enumerate(members):
                        c.submit_device(*meta[m][k], *times[k])
        for _ in range(args.warmup):
            step()
        torch.cuda.synchronize()
        for m in members:
            m.timing_enable(True)
        e0 = torch.cuda.Event(enable_timing=True)
        e1 = torch.cuda.Event(enable_timing=True)
        cur = torch.cuda.current_stream()
        e0.record(cur)
        for st in streams:
            st.wait_event(e0)
        for _ in range(args.steps):
            step()
        for st in streams:
            ev = torch.cuda.Event()
            ev.record(st)
            cur.wait_event(ev)
        e1.record(cur)
        e1.synchronize()
        ms = e0.elapsed_time(e1)
        kern = [0.0, 0.0, 0.0]
        for m in members:
            n, p, f, x = m.timing_read()
            kern = [kern[0] + p, kern[1] + f, kern[2] + x]
        tuning = [m.tuning_report() for m in members] if batched else None
        if batch is not None:
            batch.close()
        for m in members:
            m.close()
        nrun = args.steps * nsub
        out = {"value": smhz * data_s / (ms * 1e-3), "unit": UNIT, "rtf": data_s / (ms * 1e-3),
               "ms_per_subint": ms / nrun,
               "kernel_ms_per_subint_summed": {"prep": kern[0] / nrun, "fstage": kern[1] / nrun, "xmac": kern[2] / nrun}}
        if batched:
            out["fused"] = is_fused
        if tuning:
            out["tuning"] = [line for rp in tuning for line in rp.strip().split("\n") if "|" in line]
        return out

    out = {"workload": "c3: 20 stations, 16 subbands (seeded widths 4/16/64 MHz, 128/1024/4096 channels, "
                       "2/8-bit), dual pol with full cross hands, 8.192 ms subints, as %d jobs" % len(jobs),
           "station_mhz": smhz, "subints_timed": args.steps * nsub,
           "l2": "inputs larger than L2 (%d MB pool cycled)" % int(sum(sum(x[1]) for mm in meta for x in mm) / 1e6)}
    tcf = args.xmac if args.xmac != "fp32" else "fp16"
    out["tc_batched_graph"] = run(tcf, True, fused=False)
    out["tc_batched_fused"] = run(tcf, True, fused=True)
    out["tc_per_job"] = run(tcf, False)
    out["fp32_per_job"] = run("fp32", False)
    out["tc_batched_vs_fp32"] = out["tc_batched_graph"]["rtf"] / out["fp32_per_job"]["rtf"]
    out["note"] = "every form runs its subints as CUDA graphs (per job, or one per batch)"
    del dev
    torch.cuda.empty_cache()
    return out


# ---------------------------------------------------------------- INTERLACEDVDIF muxing
def mux_leg(args):
    """fxb_vdif_mux on one station of the c1 shape recorded as 16 single-channel
    VDIF threads (2-bit, 64 Ms/s each, 8000-byte payloads, 2000 frames/s per
    thread), one read of 0.5 s (128 MB, larger than L2) resident on the device;
    bytes moved = read + written, against the measured HBM copy bandwidth."""
    import torch
    from fxb200.native import vdif_mux_device
    nthr, payload, fps, nt = 16, 8000, 2000, 1000
    data = synth.interlaced_vdif(nthr, nt, payload=payload, nbits=2, fps=fps, seed=5)
    fb = payload + 32
    din = torch.from_numpy(data).cuda()
    cap = (data.size // fb) // nthr * (payload * nthr + 32)
    dout = torch.empty(cap, dtype=torch.uint8, device="cuda")
    ids = list(range(nthr))
    for _ in range(args.warmup):
        vdif_mux_device(din.data_ptr(), data.size, ids, fb, fps, 2, dout.data_ptr(), cap)
    torch.cuda.synchronize()
    e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    n = 0
    e0.record()
    for _ in range(args.steps):
        n = vdif_mux_device(din.data_ptr(), data.size, ids, fb, fps, 2, dout.data_ptr(), cap)
    e1.record()
    e1.synchronize()
    ms = e0.elapsed_time(e1) / args.steps
    hbm_peak, _, _, src = load_peaks()
    gbs = (data.size + n) / (ms * 1e-3) / 1e9
    return {"workload": "16 threads x 1 channel, 2-bit, 64 Ms/s, 8000-byte payloads, one 0.5 s read (%d MB)"
                        % (data.size // 1000000),
            "ms_per_read": ms, "rtf": 0.5 / (ms * 1e-3), "bytes_in": int(data.size), "bytes_out": int(n),
            "achieved_gbs": gbs, "hbm_peak_gbs": hbm_peak, "frac": gbs / hbm_peak, "peak_source": src,
            "note": "three launches per read (placement, headers, corner turn) plus one 8-byte status read"}


def mux_fused_leg(args):
    """c1 with every station recorded as INTERLACEDVDIF (16 single-channel
    threads of 8000-byte payloads, 2-bit, 64 Ms/s each; 128000-byte muxed
    frames), device-resident raw reads of 3 distinct subints cycled: (a) the
    reads muxed by fxb_vdif_mux and the muxed frames correlated, (b) the raw
    reads correlated directly (fxb_station.mux_raw: placement inside the
    context, each band read from its thread's frame in the F stage, no muxed
    copy).  Both on the headline form; CUDA events on the context stream."""
    import copy

    import torch
    from fxb200.native import Correlator, vdif_mux_device
    job = configs.c1()
    for st in job.stations:
        st.payload_bytes = 8000 * 16
        st.mux_threads = 16
    job.validate()
    raw_job = copy.deepcopy(job)
    for st in raw_job.stations:
        st.mux_raw = True
    npool, nsub = 3, 16
    rng = np.random.default_rng(5)
    tp = 8000
    fps = int(round(2 * job.station_bw(0) * 1e6 / (tp * 8 // 2)))
    raw_dev, raw_meta, mux_out = [], [], []
    for k in range(npool):
        sec, ns = subint_time(job, k + 1)
        bufs, nb, ds, dn, outs = [], [], [], [], []
        for s in range(len(job.stations)):
            f0, nf, dsec, dns = synth.subint_window(job, s, sec, ns)
            muxed = synth.bulk_station_frames(job, s, f0, nf, seed=3 + k)
            rb, _ = synth.raw_read(job, s, muxed, rng)
            t = torch.from_numpy(rb).cuda()
            bufs.append(t)
            nb.append(rb.size)
            ds.append(dsec)
            dn.append(dns)
            outs.append(torch.empty(muxed.size, dtype=torch.uint8, device="cuda"))
        raw_dev.append(bufs)
        raw_meta.append((nb, ds, dn, (sec, ns)))
        mux_out.append(outs)

    def run(fused):
        c = Correlator(raw_job if fused else job, xmac=args.xmac, inflight=3)
        st = torch.cuda.ExternalStream(c.stream())

        def step():
            for j in range(nsub):
                k = j % npool
                nb, ds, dn, (sec, ns) = raw_meta[k]
                if fused:
                    c.submit_device([t.data_ptr() for t in raw_dev[k]], nb, ds, dn, sec, ns)
                else:
                    nout = [vdif_mux_device(raw_dev[k][s].data_ptr(), nb[s], list(range(16)), tp + 32, fps, 2,
                                            mux_out[k][s].data_ptr(), mux_out[k][s].numel())
                            for s in range(len(job.stations))]
                    c.submit_device([t.data_ptr() for t in mux_out[k]], nout, ds, dn, sec, ns)
        for _ in range(args.warmup):
            step()
        c.sync()
        e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        e0.record(st)
        for _ in range(args.steps):
            step()
        e1.record(st)
        e1.synchronize()
        ms = e0.elapsed_time(e1) / (args.steps * nsub)
        r = c.results()
        c.close()
        return ms, r

    ms_mux, r_mux = run(False)
    ms_raw, r_raw = run(True)
    data_ms = job.subint_ns * 1e-6
    return {"workload": "c1 as INTERLACEDVDIF: 10 stations x 16 threads x 1 channel, 2-bit, 8000-byte thread "
                        "payloads; raw reads of 3 distinct subints cycled (%d MB per subint)"
                        % (sum(raw_meta[0][0]) // 1000000),
            "mux_then_correlate_ms_per_subint": ms_mux, "fused_ms_per_subint": ms_raw,
            "fused_speedup": ms_mux / ms_raw, "fused_rtf": data_ms / ms_raw,
            "identical_results": bool(np.array_equal(r_mux, r_raw)),
            "note": "(a) fxb_vdif_mux per station read (placement, headers, corner turn, status read) then the "
                    "muxed frames correlated; (b) the raw reads correlated with no muxed copy"}


# ---------------------------------------------------------------- GPU arm
def features_leg(args, job, plain_value, step_device, max_over_ranks, data_s):
    """The headline workload correlated with a 1 MHz phase-cal comb on every
    station (integer LOs: 64 bins per band, register sums; LOs 10 kHz off the
    comb: 6400 bins per band) and with two 8 MHz zoom windows per 32 MHz
    subband correlated beside it; each on the headline's device-resident
    subints, timed with CUDA events like the headline."""
    import copy

    import torch
    from fxb200.job import add_zoom_bands
    from fxb200.native import Correlator

    def pcal(v, shift):
        for st in v.stations:
            st.pcal_interval_mhz = 1.0
        for f in v.freqs:
            f.freq_mhz += shift

    variants = [
        ("pcal_1mhz_comb_int_lo", lambda v: pcal(v, 0.0),
         "1 MHz comb on every station, LOs on the comb: 32 tones and 64 bins per band"),
        ("pcal_1mhz_comb_frac_lo", lambda v: pcal(v, 0.01),
         "1 MHz comb on every station, LOs 10 kHz off the comb: 32 tones and 6400 bins per band"),
        ("zoom_2x8mhz_per_subband", lambda v: add_zoom_bands(v, [(f, off, 8.0) for f in range(len(v.freqs))
                                                                 for off in (4.0, 20.0)]),
         "two 8 MHz zoom windows (256 channels) per 32 MHz subband, correlated beside the subbands"),
    ]
    out = {}
    for name, mod, desc in variants:
        v = copy.deepcopy(job)
        mod(v)
        v.validate()
        c = Correlator(v, xmac=args.xmac, inflight=3)
        c.autotune(2)
        for _ in range(args.warmup):
            step_device(c)
        c.sync()
        torch.cuda.synchronize()
        c.timing_enable(True)
        st = torch.cuda.ExternalStream(c.stream())
        e0 = torch.cuda.Event(enable_timing=True)
        e1 = torch.cuda.Event(enable_timing=True)
        e0.record(st)
        for _ in range(args.steps):
            step_device(c)
        e1.record(st)
        e1.synchronize()
        c.sync()
        n, p, f, x = c.timing_read()
        ms = max_over_ranks(e0.elapsed_time(e1))
        val = v.station_mhz_per_sec() * data_s / (ms * 1e-3)
        out[name] = {"desc": desc, "value": val, "unit": UNIT, "rtf": data_s / (ms * 1e-3),
                     "vs_headline": val / plain_value,
                     "kernel_ms_per_subint": {"prep": p / max(n, 1), "fstage_pcal_zoom": f / max(n, 1),
                                              "xmac": x / max(n, 1)}}
        c.close()
    return out


def gpu_arm(args, job):
    import torch
    import torch.distributed as dist
    from fxb200.native import Correlator

    world = int(os.environ.get("WORLD_SIZE", "1"))
    rank = int(os.environ.get("RANK", "0"))
    local = int(os.environ.get("LOCAL_RANK", "0"))
    torch.cuda.set_device(local)
    if world > 1:
        import datetime
        dist.init_process_group("nccl", timeout=datetime.timedelta(seconds=120))

    pool = make_pool(job, POOL, seed=1 + rank)
    S = len(job.stations)
    dev = []        # [k][s] device tensors
    host = []       # [k][s] pinned host tensors
    blocks = []                       # the page-locked subint blocks (the link probe copies them too)
    for (_, inputs) in pool:
        dev.append([torch.from_numpy(b).to("cuda") for b, _, _ in inputs])
        # the subint's station buffers one after the other in one page-locked
        # block, as a datastream's receive ring holds them: one copy per subint
        blk = torch.from_numpy(np.concatenate([b for b, _, _ in inputs])).pin_memory()
        blocks.append(blk)
        offs = np.cumsum([0] + [b.size for b, _, _ in inputs])
        host.append([blk[int(offs[i]):int(offs[i + 1])] for i in range(len(inputs))])
    nbytes = [[b.size for b, _, _ in inputs] for (_, inputs) in pool]
    dsec = [[x for _, x, _ in inputs] for (_, inputs) in pool]
    dns = [[x for _, _, x in inputs] for (_, inputs) in pool]
    times = [t for (t, _) in pool]

    corr = Correlator(job, xmac=args.xmac, inflight=3)
    corr.autotune(2)                  # scheduling tuned online during the warm-up (results unchanged)
    ext = torch.cuda.ExternalStream(corr.stream())
    nsub = args.subints_per_step
    core_dev = torch.zeros(2 * corr.corelen, dtype=torch.float32, device="cuda")

    def step_device(c=None):
        c = c or corr
        for j in range(nsub):
            k = j % POOL
            c.submit_device([t.data_ptr() for t in dev[k]], nbytes[k], dsec[k], dns[k], times[k][0], times[k][1])
        if world > 1:
            # integration end: sum the ranks' core results (time-sharded subints)
            c.results_device(core_dev.data_ptr(), core_dev.numel())
            with torch.cuda.stream(torch.cuda.ExternalStream(c.stream())):
                shard.reduce_core_result(core_dev, dst=0)

    host_result = np.zeros(2 * corr.corelen, dtype=np.float32)

    def step_host():
        for j in range(nsub):
            k = j % POOL
            corr.submit_ptrs([t.data_ptr() for t in host[k]], nbytes[k], dsec[k], dns[k], times[k][0], times[k][1])
        if world > 1:
            corr.results_device(core_dev.data_ptr(), core_dev.numel())
            with torch.cuda.stream(ext):
                shard.reduce_core_result(core_dev, dst=0)
        corr.results_into(host_result)

    def barrier():
        if world > 1:
            dist.barrier()
        torch.cuda.synchronize()
        corr.sync()

    def max_over_ranks(x):
        if world == 1:
            return x
        t = torch.tensor([x], dtype=torch.float64, device="cuda")
        dist.all_reduce(t, op=dist.ReduceOp.MAX)
        return float(t.item())

    # ---- device-resident throughput (value)
    for _ in range(args.warmup):
        step_device()
    barrier()
    clocks = ClockSampler(local)
    clocks.start()
    corr.timing_enable(True)
    ev0 = torch.cuda.Event(enable_timing=True)
    ev1 = torch.cuda.Event(enable_timing=True)
    barrier()
    ev0.record(ext)
    for _ in range(args.steps):
        step_device()
    ev1.record(ext)
    ev1.synchronize()
    barrier()
    ms = ev0.elapsed_time(ev1)
    nrec, prep_ms, f_ms, x_ms = corr.timing_read()
    tuning = [line for line in corr.tuning_report().strip().split("\n")]
    corr.timing_enable(False)
    clk = clocks.stop()
    ms = max_over_ranks(ms)
    data_s = args.steps * nsub * job.subint_ns * 1e-9 * world
    value = job.station_mhz_per_sec() * data_s / (ms * 1e-3)
    rtf = data_s / (ms * 1e-3)

    # ---- end-to-end through the C ABI with host buffers
    corr.reset()
    for _ in range(max(1, args.warmup // 2)):
        step_host()
    barrier()
    t0 = time.perf_counter()
    for _ in range(args.steps):
        step_host()
    barrier()
    e2e_ms = max_over_ranks((time.perf_counter() - t0) * 1e3)
    e2e_value = job.station_mhz_per_sec() * data_s / (e2e_ms * 1e-3)
    h2d = sum(nbytes[j % POOL][s] for j in range(nsub) for s in range(S))
    d2h = 2 * corr.corelen * 4

    # ---- the other form on the same workload (device-resident)
    other = None
    other_name = "fp32" if args.xmac != "fp32" else "fp16"
    if not args.no_other_form:
        ctc = Correlator(job, xmac=other_name, inflight=3)
        ctc.autotune(2)
        for _ in range(args.warmup):
            step_device(ctc)
        ctc.sync()
        barrier()
        ctc.timing_enable(True)
        ext2 = torch.cuda.ExternalStream(ctc.stream())
        e0 = torch.cuda.Event(enable_timing=True)
        e1 = torch.cuda.Event(enable_timing=True)
        e0.record(ext2)
        for _ in range(args.steps):
            step_device(ctc)
        e1.record(ext2)
        e1.synchronize()
        ctc.sync()
        n2, p2, f2, x2 = ctc.timing_read()
        tms = max_over_ranks(e0.elapsed_time(e1))
        tval = job.station_mhz_per_sec() * data_s / (tms * 1e-3)
        other = {"xmac": other_name, "value": tval, "unit": UNIT, "rtf": data_s / (tms * 1e-3),
                 "ms_per_step": tms / args.steps,
                 "kernel_ms_per_subint": {"prep": p2 / max(n2, 1), "fstage": f2 / max(n2, 1), "xmac": x2 / max(n2, 1)}}
        ctc.close()
        barrier()
    if other is not None:
        tc_v, fp_v = (value, other["value"]) if args.xmac != "fp32" else (other["value"], value)
        tc_vs_fp32 = tc_v / fp_v
    else:
        tc_vs_fp32 = None

    # ---- the headline workload with phase-cal extraction or zoom bands, on
    # the same device-resident inputs (rank 0, N=1)
    feats = None
    if rank == 0 and world == 1 and not args.no_features:
        feats = features_leg(args, job, value, step_device, max_over_ranks, data_s)

    # ---- rooflines: F stage against HBM (its design bound); XMAC against the
    # tensor pipe (burst and sustained peaks) and against HBM (its spectra read)
    hbm_peak, tf_peak, tf_sus, peak_src = load_peaks()
    T = job.blocks_per_send()
    rows = sum(st.nband for st in job.stations)
    in_bytes = sum(nbytes[k][s] for k in range(POOL) for s in range(S)) / POOL
    s_out = 4 if args.xmac != "fp32" else 8
    spec_bytes = T * rows * job.freqs[0].nchan * s_out
    f_avg = f_ms / max(nrec, 1)
    x_avg = x_ms / max(nrec, 1)
    tcfft = args.xmac != "fp32" and any("tensor-core FFT" in t for t in tuning)
    fname = "k_fstage_tc" if tcfft else "k_fstage"
    alg = in_bytes + spec_bytes
    achieved = alg / (f_avg * 1e-3) / 1e9
    roofline = {"bound": "hbm", "kernel": fname, "achieved": achieved, "peak": hbm_peak, "unit": "GB/s",
                "frac": achieved / hbm_peak, "traffic": load_traffic(fname + "_c1_" + args.xmac),
                "peak_source": peak_src, "algorithmic_bytes_per_launch": alg,
                "note": "achieved = (packed VDIF bytes read + spectra bytes written) per 8 ms subint / F-stage "
                        "event time per subint (F-stage launches only)",
                "kernel_ms_per_subint": {"prep": prep_ms / max(nrec, 1), "fstage": f_avg, "xmac": x_avg}}
    # useful XMAC flops: 8 per Hermitian-unique input pair, channel and FFT
    useful = 0
    for f in range(len(job.freqs)):
        I = sum(1 for st in job.stations for fb, _ in st.bands if fb == f)
        useful += 8 * (I * (I + 1) // 2) * job.freqs[f].nchan * T
    tcx = args.xmac != "fp32"
    xname = "k_xmac_tc" if tcx else "k_xmac_fp32v2"
    xach = useful / (x_avg * 1e-3) / 1e12
    xmac_roofline = {"bound": "tensor" if tcx else "fp32 pipe", "kernel": xname, "achieved": xach, "unit": "TFLOP/s",
                     "peak_burst": tf_peak if tcx else None, "frac_burst": xach / tf_peak if tcx else None,
                     "peak_sustained": tf_sus if tcx else None,
                     "frac_sustained": xach / tf_sus if (tcx and tf_sus) else None,
                     "hbm_bound": {"spectra_bytes_read": spec_bytes, "achieved_gbs": spec_bytes / (x_avg * 1e-3) / 1e9,
                                   "frac": spec_bytes / (x_avg * 1e-3) / 1e9 / hbm_peak},
                     "useful_flops_per_subint": useful,
                     "note": "useful flops only (8 per Hermitian-unique pair); the time includes the weights kernel; "
                             "at 20 inputs the contraction carries ~21 useful flops per spectra byte, so HBM bounds it"}

    # ---- CPU baseline (rank 0, N=1 only)
    cpu = None
    if rank == 0 and world == 1 and not args.no_cpu_baseline:
        v, cores, sample, kind = cpu_reference(job, pool, os.cpu_count() or 1)
        cpu = {"value": v, "unit": UNIT, "cores": cores, "kind": kind, "sample": sample}

    serve = None
    if rank == 0 and world == 1 and not args.no_serving:
        serve = serving_leg(args)
    c3 = None
    if rank == 0 and world == 1 and not args.no_c3:
        c3 = c3_leg(args)
    mux = None
    muxf = None
    if rank == 0 and world == 1 and not args.no_mux:
        mux = mux_leg(args)
        muxf = mux_fused_leg(args)

    # per subint: interpolators and frame validity (one launch), FFT
    # parameters, one F-stage launch per FFT length (the workload's are
    # tensor-core FFT kinds), one XMAC launch per group of equally shaped
    # subbands, weights
    shapes = {(sum(1 for st in job.stations for fb, _ in st.bands if fb == f), job.freqs[f].nchan)
              for f in range(len(job.freqs)) if any(fb == f for st in job.stations for fb, _ in st.bands)}
    flens = {2 * job.freqs[st.bands[0][0]].nchan for st in job.stations}
    launches_per_subint = 2 + len(flens) + len(shapes) + 1
    if rank == 0:
        link = h2d_link_gbs(blocks) if world == 1 else None
        e2e_gbs = h2d / (e2e_ms / args.steps * 1e-3) / 1e9
        # the full record first, then the headline line (last, compact) carrying
        # the secondary figures
        detail = {"bench_detail": True, "tuning": tuning, "serving": serve, "batched_c3": c3, "vdif_mux": mux,
                  "vdif_mux_fused": muxf,
                  "features": feats, "other_form": other, "roofline": roofline, "xmac_roofline": xmac_roofline,
                  "cpu_baseline": cpu, "clocks": clk}
        print(json.dumps(detail), flush=True)
        line = {
            "metric": METRIC, "value": value, "unit": UNIT, "n_gpus": world, "steps": args.steps,
            "warmup": args.warmup, "ms_per_step": ms / args.steps, "higher_is_better": True, "scaling": "weak",
            "vs_baseline": None, "dtype": {"fp32": "f32", "fp16": "f16", "bf16": "bf16"}[args.xmac],
            "data": "synthetic", "rtf": rtf, "xmac": args.xmac,
            "config": workload_config(job),
            "e2e": {"value": e2e_value, "unit": UNIT, "rtf": e2e_value / job.station_mhz_per_sec(),
                    "h2d_bytes_per_step": h2d, "d2h_bytes_per_step": d2h, "ms_per_step": e2e_ms / args.steps,
                    "h2d_gbs": e2e_gbs, "h2d_link_gbs": link, "link_frac": (e2e_gbs / link) if link else None},
            "roofline": {k: roofline[k] for k in ("bound", "kernel", "achieved", "peak", "unit", "frac", "traffic",
                                                  "peak_source", "kernel_ms_per_subint")},
            "xmac_roofline": {k: xmac_roofline[k] for k in ("kernel", "achieved", "unit", "frac_burst",
                                                            "frac_sustained", "hbm_bound")},
            "cpu_baseline": cpu, "clocks": clk,
            "other_form": None if other is None else {k: other[k] for k in ("xmac", "value", "rtf",
                                                                            "kernel_ms_per_subint")},
            "tc_vs_fp32": tc_vs_fp32,
            "serving": None if serve is None else {k: serve[k] for k in ("jobs", "p50_ms", "p99_ms", "rtf",
                                                                          "station_mhz_per_s", "h2d_link_frac")
                                                   if k in serve},
            "batched_c3": None if c3 is None else {"tc_batched_vs_fp32": c3["tc_batched_vs_fp32"],
                                                   "tc_batched_rtf": c3["tc_batched_graph"]["rtf"],
                                                   "tc_batched_fused_rtf": c3["tc_batched_fused"]["rtf"],
                                                   "tc_per_job_rtf": c3["tc_per_job"]["rtf"],
                                                   "fp32_per_job_rtf": c3["fp32_per_job"]["rtf"]},
            "vdif_mux_frac": None if mux is None else mux["frac"],
            "vdif_mux_fused": None if muxf is None else {k: muxf[k] for k in ("fused_ms_per_subint",
                                                                              "mux_then_correlate_ms_per_subint",
                                                                              "fused_speedup", "identical_results")},
            "gpu_launches": launches_per_subint * nsub * args.steps,
        }
        print(json.dumps(line), flush=True)
    corr.close()
    if world > 1:
        dist.destroy_process_group()


def main():
    args = parse()
    job = configs.c1()
    if args.c3_only:
        c3_only(args)
    elif args.impl == "reference":
        reference_arm(args, job)
    else:
        gpu_arm(args, job)


if __name__ == "__main__":
    main()
