"""The multi-GPU path of bench.py on CPU: world-size-2 gloo process groups.
Each rank of a weak-scaling run times its own sweep; the step time is the
largest over the ranks, and only rank 0 prints."""
import json
import os
import socket
import subprocess
import sys

import pytest
import torch.multiprocessing as mp

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


def _free_port():
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        return s.getsockname()[1]


def _rank_main(rank, world, port, out):
    import datetime

    import torch.distributed as dist
    sys.path.insert(0, ROOT)
    import bench
    os.environ["MASTER_ADDR"] = "127.0.0.1"
    os.environ["MASTER_PORT"] = str(port)
    dist.init_process_group("gloo", rank=rank, world_size=world, timeout=datetime.timedelta(seconds=60))
    try:
        # rank r's step took 10 (r + 1) ms: the job's step is the slowest one
        got = bench.max_over_ranks_of(dist, 10.0 * (rank + 1), "cpu")
        out.put((rank, got))
    finally:
        dist.destroy_process_group()


def test_max_over_ranks_gloo_world_2():
    ctx = mp.get_context("spawn")
    out = ctx.Queue()
    port = _free_port()
    procs = [ctx.Process(target=_rank_main, args=(r, 2, port, out)) for r in range(2)]
    for p in procs:
        p.start()
    for p in procs:
        p.join(120)
        assert p.exitcode == 0
    got = dict(out.get(timeout=10) for _ in range(2))
    assert got == {0: 20.0, 1: 20.0}


def test_max_over_ranks_single_rank_is_identity():
    sys.path.insert(0, ROOT)
    import bench
    assert bench.max_over_ranks_of(None, 12.5, "cpu") == 12.5


@pytest.mark.timeout(600)
def test_reference_arm_under_torchrun_world_2():
    """bench.py --impl reference under torchrun with two ranks, as a two-GPU
    run launches it: both ranks join a gloo group, rank 0 alone prints one
    JSON line."""
    env = dict(os.environ, OMP_NUM_THREADS="2")
    cmd = [sys.executable, "-m", "torch.distributed.run", "--nnodes=1", "--nproc-per-node", "2",
           "--master-addr", "127.0.0.1", "--master-port", str(_free_port()),
           os.path.join(ROOT, "bench.py"), "--impl", "reference", "--gpus", "2", "--steps", "1", "--warmup", "0",
           "--count", "2", "--cpu-sample", "1", "--ref-chunks", "1"]
    r = subprocess.run(cmd, cwd=ROOT, env=env, capture_output=True, text=True, timeout=560)
    assert r.returncode == 0, r.stderr[-2000:]
    lines = [json.loads(l) for l in r.stdout.splitlines() if l.startswith("{")]
    assert len(lines) == 1
    line = lines[0]
    assert line["impl"] == "reference" and line["n_gpus"] == 2 and line["value"] > 0


def _shard_main(rank, world, port, out):
    """One rank of a sharded sweep: its LPT part, computed with the oracle on
    small matrices (the CPU stand-in for the device), gathered on rank 0."""
    import datetime

    import torch.distributed as dist
    sys.path.insert(0, ROOT)
    import bench
    from csharp_linearalgebra_b200.sweep import expm_cost_estimate, gather_to_rank0, lpt_partition
    from oracle import oracle
    os.environ["MASTER_ADDR"] = "127.0.0.1"
    os.environ["MASTER_PORT"] = str(port)
    dist.init_process_group("gloo", rank=rank, world_size=world, timeout=datetime.timedelta(seconds=60))
    try:
        count, seed = 12, 7
        orders, omegas = bench.sweep_spec(count, seed)
        orders = [8 + n % 40 for n in orders]  # small orders: the oracle finishes at once
        costs = [expm_cost_estimate(n, w) for n, w in zip(orders, omegas)]
        parts, loads = lpt_partition(costs, world)
        mine = parts[rank]
        results = [oracle.expm(bench.sweep_matrix(k, orders[k], omegas[k], seed))[0] for k in mine]
        gathered = gather_to_rank0(dist, rank, world, mine, results)
        out.put((rank, mine, loads, gathered))
    finally:
        dist.destroy_process_group()


def test_lpt_sharded_sweep_gathers_the_single_rank_result():
    """A sweep partitioned over two gloo ranks by LPT: the parts are
    disjoint and cover the sweep, the loads balance to within the largest
    single cost, and the results gathered on rank 0 equal, bit for bit, the
    same sweep computed by one rank."""
    sys.path.insert(0, ROOT)
    import numpy as np

    import bench
    from csharp_linearalgebra_b200.sweep import expm_cost_estimate
    from oracle import oracle
    ctx = mp.get_context("spawn")
    out = ctx.Queue()
    port = _free_port()
    procs = [ctx.Process(target=_shard_main, args=(r, 2, port, out)) for r in range(2)]
    for p in procs:
        p.start()
    got = {}
    for _ in range(2):
        rank, mine, loads, gathered = out.get(timeout=120)
        got[rank] = (mine, loads, gathered)
    for p in procs:
        p.join(60)
        assert p.exitcode == 0
    count, seed = 12, 7
    orders, omegas = bench.sweep_spec(count, seed)
    orders = [8 + n % 40 for n in orders]
    parts = [got[0][0], got[1][0]]
    assert sorted(parts[0] + parts[1]) == list(range(count)) and not set(parts[0]) & set(parts[1])
    costs = [expm_cost_estimate(n, w) for n, w in zip(orders, omegas)]
    loads = got[0][1]
    assert abs(loads[0] - loads[1]) <= max(costs)
    assert got[1][2] is None
    single = [oracle.expm(bench.sweep_matrix(k, orders[k], omegas[k], seed))[0] for k in range(count)]
    assert len(got[0][2]) == count
    assert all(np.array_equal(a, b) for a, b in zip(got[0][2], single))


def test_lpt_partition_properties():
    sys.path.insert(0, ROOT)
    from csharp_linearalgebra_b200.sweep import lpt_partition
    costs = [5.0, 3.0, 3.0, 2.0, 2.0, 2.0, 1.0]
    parts, loads = lpt_partition(costs, 3)
    assert sorted(i for p in parts for i in p) == list(range(len(costs)))
    assert loads == [sum(costs[i] for i in p) for p in parts]
    assert max(loads) - min(loads) <= max(costs)
    # one rank takes everything, in order
    assert lpt_partition(costs, 1)[0] == [list(range(len(costs)))]
    with pytest.raises(ValueError):
        lpt_partition(costs, 0)
