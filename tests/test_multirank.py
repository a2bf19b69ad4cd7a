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


def _partition_main(rank, world, port, out):
    """One rank: converge its LPT share of a small isotherm with the CPU stand-in for
    converge! (the oracle's C++ restatement), then gather (adsorption, Omega_ex, errcode,
    rho) to rank 0 -- the data path has no collective."""
    import sys
    import datetime
    import torch.distributed as dist
    root = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
    for p in (root, os.path.join(root, "cdft.jl_b200"), os.path.join(root, "tests")):
        sys.path.insert(0, p)
    from cdft_b200 import shard
    os.environ.update(MASTER_ADDR="127.0.0.1", MASTER_PORT=str(port), RANK=str(rank), WORLD_SIZE=str(world))
    dist.init_process_group("gloo", rank=rank, world_size=world, timeout=datetime.timedelta(seconds=120))
    specs, systems = _small_isotherm()
    costs = [shard.estimated_cost(N) for _, _, N in specs]
    parts = shard.lpt_partition(costs, world)
    mine = parts[rank]
    records = _converge_records([systems[i] for i in mine])
    allrec = shard.gather_results(dist, rank, world, mine, records, len(specs))
    if rank == 0:
        out["records"] = allrec
        out["parts"] = parts
    dist.destroy_process_group()


def _small_isotherm():
    from golden import make_fixtures as mf
    from oracle import functional as fn
    specs = [s for k, s in enumerate(mf.isotherm_specs()) if k % 8 in (0, 5)][:8]   # 8 points, uneven grids
    om = mf.oracle_model(["methane"])
    s = om.sigma[0]
    systems = []
    for H, p, N in specs:
        rb = mf.stable_bulk_density(om, p, 150.0)
        systems.append(fn.DFTSystem(om, fn.Structure((p, 150.0), [rb], [(0.7 * s, H - 0.7 * s)], (N,)),
                                    [fn.SteeleWall.graphite(H)]))
    return specs, systems


def _converge_records(systems):
    import numpy as np
    from oracle import cpu
    rhos = [np.ascontiguousarray(so.initialize_profiles()) for so in systems]
    res, _ = cpu.batch_converge(systems, rhos, nthreads=1, beta=0.1, tol=1e-10, anderson_m=5)
    return [(float(so.adsorption(r)[0]), float(so.surface_tension(r)), int(x.errcode), r)
            for so, r, x in zip(systems, rhos, res)]


def test_two_ranks_partition_one_isotherm_and_gather():
    """An isotherm's state points split by LPT over two gloo ranks and gathered on rank 0
    equal the single-rank result bit for bit (each state point converges independently)."""
    import sys
    import numpy as np
    root = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
    for p in (root, os.path.join(root, "cdft.jl_b200")):
        sys.path.insert(0, p)
    from cdft_b200 import shard
    from oracle import cpu
    cpu.build()
    world = 2
    port = _free_port()
    with mp.Manager() as mgr:
        out = mgr.dict()
        mp.spawn(_partition_main, args=(world, port, out), nprocs=world, join=True)
        res = dict(out)
    parts = res["parts"]
    assert sorted(parts[0] + parts[1]) == list(range(8)) and parts[0] and parts[1]
    specs, systems = _small_isotherm()
    costs = [shard.estimated_cost(N) for _, _, N in specs]
    assert shard.balance(parts, costs) < 1.25
    single = _converge_records(systems)
    for (a0, o0, e0, r0), (a1, o1, e1, r1) in zip(single, res["records"]):
        assert e0 == e1 == 0 and a0 == a1 and o0 == o1 and np.array_equal(r0, r1)


def test_lpt_partition_properties():
    from cdft_b200 import shard
    costs = [shard.estimated_cost(n) for n in (100, 143, 186, 229, 271, 314, 357, 400)] * 8
    for world in (1, 2, 3, 4, 8):
        parts = shard.lpt_partition(costs, world)
        assert sorted(i for p in parts for i in p) == list(range(len(costs)))
        assert shard.balance(parts, costs) < 1.1
    assert shard.lpt_partition([5.0], 3) == [[0], [], []]
