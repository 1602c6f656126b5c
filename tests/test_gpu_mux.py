"""INTERLACEDVDIF on the device (fxb_vdif_mux) against the reference's own
VDIFMuxer (mpifxcorr/src/datamuxer.cpp, compiled into oracle/_ref): for one
read of multi-thread VDIF -- threads in random order, a thread nobody asked
for, a frame missing from one thread, a time missing from every thread, a
frame sent twice -- every output header is bit-identical and every valid
output frame's payload (the corner turn) is byte-identical.  Invalid frames'
payloads are not compared: the reference leaves them unwritten."""
import zlib

import numpy as np
import pytest
import torch

from fxb200 import synth
from fxb200.native import vdif_mux_device

import refcorr

pytestmark = [pytest.mark.gpu,
              pytest.mark.skipif(not refcorr.available(), reason="reference build oracle/_ref absent")]

CASES = {
    "2thr_2bit": dict(nthreads=2, nbits=2),
    "4thr_2bit_gaps": dict(nthreads=4, nbits=2, drop=[(3, 1), (5, None)], extra_thread=True, duplicate=[(7, 2)]),
    "8thr_2bit": dict(nthreads=8, nbits=2, drop=[(2, 7)]),
    "16thr_2bit": dict(nthreads=16, nbits=2, payload=8192),
    "2thr_8bit": dict(nthreads=2, nbits=8, drop=[(0, 1)]),
    "4thr_4bit_ids": dict(nthreads=4, nbits=4, thread_ids=[3, 9, 1, 12]),
}


def _mux_gpu(data, nthreads, ids, framebytes, fps, nbits):
    din = torch.from_numpy(data).cuda()
    nout = (data.size // framebytes) // nthreads
    cap = max(1, nout * ((framebytes - 32) * nthreads + 32))
    dout = torch.full((cap,), 0xAB, dtype=torch.uint8, device="cuda")
    n = vdif_mux_device(din.data_ptr(), data.size, ids, framebytes, fps, nbits, dout.data_ptr(), cap)
    return dout[:n].cpu().numpy().tobytes()


@pytest.mark.parametrize("name", sorted(CASES))
def test_mux_matches_reference(name):
    kw = dict(CASES[name])
    nthreads, nbits = kw["nthreads"], kw["nbits"]
    payload = kw.pop("payload", 8000)
    ids = kw.get("thread_ids") or list(range(nthreads))
    fps = 64_000_000 * nbits // (8 * payload) if payload == 8000 else 1000
    data = synth.interlaced_vdif(nframes=24, payload=payload, fps=fps, seed=zlib.crc32(name.encode()), **kw)
    fb = payload + 32
    ref = refcorr.vdif_mux(data, nthreads, ids, fb, fps, nbits)
    got = _mux_gpu(data, nthreads, ids, fb, fps, nbits)
    assert len(got) == len(ref) > 0
    ofb = payload * nthreads + 32
    nvalid = 0
    for k in range(len(ref) // ofb):
        g, r = got[k * ofb:(k + 1) * ofb], ref[k * ofb:(k + 1) * ofb]
        assert g[:32] == r[:32], (name, k)
        if not (r[3] & 0x80):
            assert g[32:] == r[32:], (name, k)
            nvalid += 1
    assert nvalid > 0
