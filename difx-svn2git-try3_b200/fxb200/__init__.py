"""fxb200: B200-native FX correlator hot path (DiFX Mode::process + Core XMAC).

Python side of the product: the job description (job.py), the seeded
synthetic VDIF generator used by tests and the bench (synth.py), the
workload configurations (configs.py) and the ctypes binding of the C ABI
(native.py).  All correlation work happens in libfxb200.so on the GPU.
"""
from .job import Baseline, DelayPoly, Freq, Job, Station, full_job  # noqa: F401
