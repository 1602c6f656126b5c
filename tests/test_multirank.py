"""The multi-process (time-sharded) path on CPU: two gloo ranks correlate
alternate subints of one integration and reduce their core results; the sum
equals the single-process integration.  The per-rank correlation here is the
FP64 oracle standing in for each rank's GPU (no GPU in this test); the
sharding and reduction code is the product's (fxb200.shard)."""
import os
import socket

import numpy as np
import pytest
import torch
import torch.distributed as dist
import torch.multiprocessing as mp

from fxb200 import shard, synth
from helpers import rel_err, small_job


def _free_port():
    s = socket.socket()
    s.bind(("127.0.0.1", 0))
    p = s.getsockname()[1]
    s.close()
    return p


def _job():
    return small_job(nstation=3, full_pol=True, subint_ns=1_024_000, seed=8)


def _worker(rank, world, port, out_path):
    import fxoracle
    os.environ["MASTER_ADDR"] = "127.0.0.1"
    os.environ["MASTER_PORT"] = str(port)
    dist.init_process_group("gloo", rank=rank, world_size=world,
                            timeout=__import__("datetime").timedelta(seconds=60))
    job = _job()
    subints = shard.integration_subints(job, 0, 1_024_000, 6 * job.subint_ns * 1e-9)
    mine = shard.subints_for_rank(subints, rank, world)
    orc = fxoracle.OracleCorrelator(job)
    acc = np.zeros(2 * orc.corelen, dtype=np.float64)
    for sec, ns in mine:
        inputs = synth.subint_inputs(job, sec, ns, rho=0.05, seed=3)
        orc.process_subint(inputs, sec, ns, coreresult=acc)
    buf = torch.from_numpy(acc.astype(np.float32))
    shard.reduce_core_result(buf, dst=0)
    if rank == 0:
        np.save(out_path, buf.numpy())
    dist.barrier()
    dist.destroy_process_group()


def test_round_robin_assignment():
    subints = [(0, k) for k in range(7)]
    parts = [shard.subints_for_rank(subints, r, 3) for r in range(3)]
    assert sorted(sum(parts, [])) == subints
    assert parts[0] == [(0, 0), (0, 3), (0, 6)]
    with pytest.raises(ValueError):
        shard.subints_for_rank(subints, 3, 3)


def test_two_rank_integration_equals_single_process(tmp_path):
    import fxoracle
    out = str(tmp_path / "r0.npy")
    mp.start_processes(_worker, args=(2, _free_port(), out), nprocs=2, join=True, start_method="spawn")
    got = np.load(out)
    job = _job()
    orc = fxoracle.OracleCorrelator(job)
    ref = np.zeros(2 * orc.corelen, dtype=np.float64)
    for sec, ns in shard.integration_subints(job, 0, 1_024_000, 6 * job.subint_ns * 1e-9):
        inputs = synth.subint_inputs(job, sec, ns, rho=0.05, seed=3)
        orc.process_subint(inputs, sec, ns, coreresult=ref)
    assert rel_err(got.astype(np.float64), ref) < 1e-6
