"""The N>1 bench path on CPU: two gloo ranks, replicas only (no data-path collective).

Every rank factors and solves its own copy of the workload (here through the oracle, on the
64x64 / L=4 case); ranks meet only at the barriers around the timed region and in the maximum of
their timings, from which rank 0 reports the whole-job rate.
"""
import os
import socket
import subprocess
import sys

import numpy as np
import pytest
import torch.multiprocessing as mp

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


def _free_port():
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        return s.getsockname()[1]


def _rank_main(rank, world, port, out):
    os.environ.update(MASTER_ADDR="127.0.0.1", MASTER_PORT=str(port), RANK=str(rank),
                      WORLD_SIZE=str(world), LOCAL_RANK=str(rank))
    sys.path.insert(0, ROOT)
    sys.path.insert(0, os.path.join(ROOT, "tests"))
    from helpers import oracle_run
    from robinsolver_b200 import workloads as W
    from robinsolver_b200.replicas import Replicas

    rep = Replicas("gloo", timeout_s=60)
    rep.barrier()
    _, U = oracle_run(W.make_workload(1))          # this rank's replica of the whole workload
    rep.barrier()
    # every replica computed the same thing: the checksum's max and min over ranks agree
    chk = float(np.sum(np.abs(U)))
    hi, lo = rep.max(chk), -rep.max(-chk)
    # rank r pretends its timed region took 10*(r+1) ms for 4 steps of 8 right-hand sides
    value, ms = rep.rate(4 * 8, 10.0 * (rank + 1))
    out[rank] = (rep.world, rep.leader, hi, lo, chk, value, ms)
    rep.close()


def test_two_gloo_replicas_agree_and_report_the_slowest_rank():
    world, port = 2, _free_port()
    mgr = mp.Manager()
    out = mgr.dict()
    mp.spawn(_rank_main, args=(world, port, out), nprocs=world, join=True)
    res = dict(out)
    assert sorted(res) == [0, 1]
    for r, (w, leader, hi, lo, chk, value, ms) in res.items():
        assert w == 2 and leader == (r == 0)
        assert hi == lo == chk                      # replicas are bit-identical
        assert ms == 20.0                           # the slower rank's time
        assert value == pytest.approx(2 * 32 / 0.020)  # whole-job units / slowest time


def test_reference_arm_runs_on_rank_zero_only():
    env = dict(os.environ, RANK="1", WORLD_SIZE="2", LOCAL_RANK="1")
    p = subprocess.run([sys.executable, os.path.join(ROOT, "bench.py"), "--impl", "reference", "--config", "1",
                        "--steps", "1", "--warmup", "0"], env=env, capture_output=True, text=True, timeout=120)
    assert p.returncode == 0, p.stderr
    assert p.stdout.strip() == ""
