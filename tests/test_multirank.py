"""The multi-GPU path of bench.py on CPU: two gloo ranks.

Each rank converges its own 64-point isotherm (weak scaling, no collective on the data
path); the only collectives are the barrier and the max over ranks of the device time.
These tests run that logic with the gloo backend on the host."""
import os
import socket

import pytest
import torch.multiprocessing as mp


def _free_port():
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        return s.getsockname()[1]


def _rank_main(rank, world, port, out):
    import sys
    import datetime
    import torch.distributed as dist
    root = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
    sys.path.insert(0, root)
    import bench
    os.environ.update(MASTER_ADDR="127.0.0.1", MASTER_PORT=str(port), RANK=str(rank), WORLD_SIZE=str(world))
    dist.init_process_group("gloo", rank=rank, world_size=world, timeout=datetime.timedelta(seconds=60))
    specs = bench.isotherm_specs(rank)
    # each rank times a different amount of work; the job time is the slowest rank's
    local_ms = 10.0 * (rank + 1)
    ms = bench.max_over_ranks(local_ms, dist, "cpu")
    rate = bench.whole_job_rate(len(specs), world, ms)
    out[rank] = (specs, ms, rate)
    dist.destroy_process_group()


def test_two_ranks_shard_state_points_and_take_the_max_time():
    world = 2
    port = _free_port()
    with mp.Manager() as mgr:
        out = mgr.dict()
        mp.spawn(_rank_main, args=(world, port, out), nprocs=world, join=True)
        res = dict(out)
    (s0, ms0, r0), (s1, ms1, r1) = res[0], res[1]
    assert len(s0) == len(s1) == 64
    # distinct state points per rank (pressures shifted by 0.1 % per rank), same grids
    assert all(a[2] == b[2] and a[0] == b[0] for a, b in zip(s0, s1))
    assert all(abs(b[1] / a[1] - 1.001) < 1e-12 for a, b in zip(s0, s1))
    # every rank reports the slowest rank's time and the whole-job rate
    assert ms0 == ms1 == 20.0
    assert r0 == r1 == pytest.approx(128 / 0.020)
