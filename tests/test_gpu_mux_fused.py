"""INTERLACEDVDIF stations fed the raw multi-thread reads (fxb_station.mux_raw):
the context places the threads' frames and reads each band from its thread's
frame inside the F stage, with no muxed copy.  The result must equal, bit for
bit, that of the same stations fed fxb_vdif_mux's output of the same reads
(itself byte-identical to the reference VDIFMuxer), with thread frames in
random order, some missing (incomplete slots, invalid muxed frames), EDV4
validity masks, an unwanted thread's frame leading the read (the muxed
stream starts one frame in) and invalid frames; and that result matches the
FP64 oracle on the muxed frames."""
import copy

import numpy as np
import pytest

from fxb200 import synth
from fxb200.native import Correlator, vdif_mux_device
from helpers import compare_core, edv4_inputs, mux_job, raw_read

import fxoracle

pytestmark = pytest.mark.gpu


def _muxed_and_raw(job, sec, ns, k, rng):
    f0 = synth.subint_window(job, 0, sec, ns)[0]
    base = edv4_inputs(job, synth.subint_inputs(job, sec, ns, rho=0.05, seed=13 + k,
                                                invalid={0: [f0 + 1, f0 + 6]}), seed=k)
    import torch
    muxed, raw = [], []
    for s, (buf, dsec, dns) in enumerate(base):
        st = job.stations[s]
        if not st.mux_threads:
            muxed.append((buf, dsec, dns))
            raw.append((buf, dsec, dns))
            continue
        rb, lead = raw_read(job, s, buf, rng, lead_extra=(s == 0))
        tp = st.payload_bytes // st.mux_threads
        fps = int(round(2 * job.station_bw(s) * 1e6 / (tp * 8 // st.nbits)))
        din = torch.from_numpy(rb).cuda()
        cap = (rb.size // (tp + 32)) // st.mux_threads * (st.payload_bytes + 32)
        dout = torch.zeros(cap, dtype=torch.uint8, device="cuda")
        n = vdif_mux_device(din.data_ptr(), rb.size, list(range(st.mux_threads)), tp + 32, fps, st.nbits,
                            dout.data_ptr(), cap)
        torch.cuda.synchronize()
        muxed.append((dout[:n].cpu().numpy(), dsec, dns))
        # the raw read's first frame is `lead` frame times before the muxed stream
        t = dsec * 1_000_000_000 + dns - lead * (1_000_000_000 // fps)
        raw.append((rb, t // 1_000_000_000, t % 1_000_000_000))
    return muxed, raw


@pytest.mark.parametrize("masklength,xmac,kw", [(4, "fp32", {}), (2, "fp16", {}),
                                                # one band per work item; 8192-point FFTs (the
                                                # persistent F kernels' other raw-read classes)
                                                (2, "fp16", dict(full_pol=False)),
                                                (2, "fp16", dict(nchan=4096, bw=16.0))])
def test_fused_raw_reads_equal_muxed_frames(masklength, xmac, kw):
    job = mux_job(masklength=masklength, **kw)
    fused = copy.deepcopy(job)
    for st in fused.stations:
        if st.mux_threads:
            st.mux_raw = True
    c_mux = Correlator(job, xmac=xmac)
    c_raw = Correlator(fused, xmac=xmac)
    orc = fxoracle.OracleCorrelator(job)
    rng = np.random.default_rng(7)
    ref = None
    for k, (sec, ns) in enumerate([(0, 1_024_000), (0, 3_072_000)]):
        muxed, raw = _muxed_and_raw(job, sec, ns, k, rng)
        c_mux.submit(muxed, sec, ns)
        c_raw.submit(raw, sec, ns)
        ref = orc.process_subint(muxed, sec, ns, coreresult=ref)
    a, b = c_raw.results(), c_mux.results()
    wa, wb = c_raw.fft_weights(), c_mux.fft_weights()
    layout, n = c_mux.layout(), c_mux.corelen
    c_raw.close()
    c_mux.close()
    assert np.array_equal(wa, wb)
    assert np.array_equal(a, b)
    compare_core(job, layout, n, b, ref, tol=1e-5 if xmac == "fp32" else 1e-3)
