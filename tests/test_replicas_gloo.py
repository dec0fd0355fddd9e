"""The multi-GPU form of bench.py (independent replicas, one per rank) on
CPU ranks: two gloo processes agree on the whole-job rate (every rank's
cells over the slowest rank's time) and the reference arm runs on rank 0
only."""
import os
import socket
import sys
from pathlib import Path

import pytest

ROOT = Path(__file__).resolve().parents[1]
torch = pytest.importorskip("torch")


def _free_port():
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        return s.getsockname()[1]


def _rank_main(rank, world, port, out):
    import datetime
    import torch.distributed as dist
    sys.path.insert(0, str(ROOT))
    os.environ.update(MASTER_ADDR="127.0.0.1", MASTER_PORT=str(port))
    dist.init_process_group("gloo", rank=rank, world_size=world, timeout=datetime.timedelta(seconds=60))
    import bench
    value, ms = bench.job_rate(10.0 + 5.0 * rank, 1000, 4, world)
    out[rank] = (value, ms)
    # the reference arm: ranks other than 0 return at once, without work
    class Args:
        n, steps, warmup, case, gpus = 64, 1, 0, "sod", world
    if rank != 0:
        assert bench.run_reference(Args, world, rank) is None
    dist.barrier()
    dist.destroy_process_group()


def test_two_replicas_agree_on_the_job_rate():
    import torch.multiprocessing as mp
    world = 2
    port = _free_port()
    with mp.Manager() as m:
        out = m.dict()
        mp.spawn(_rank_main, args=(world, port, out), nprocs=world, join=True)
        res = dict(out)
    slowest = 15.0
    expect = world * 1000 * 4 / (slowest * 1e-3) / 1e9
    for rank in range(world):
        value, ms = res[rank]
        assert ms == slowest
        assert value == pytest.approx(expect, rel=1e-12)


def test_single_rank_rate_needs_no_process_group():
    sys.path.insert(0, str(ROOT))
    import bench
    value, ms = bench.job_rate(2.0, 500, 10, 1)
    assert ms == 2.0 and value == pytest.approx(500 * 10 / 2e-3 / 1e9)


def test_reference_arm_line_keeps_the_contract(capsys):
    """The reference arm (the CPU restatement on the host cores) prints one
    JSON line with our arm's metric, unit and workload, a cpu_baseline block
    and an e2e block without host transfers."""
    import json
    sys.path.insert(0, str(ROOT))
    import bench

    class Args:
        n, steps, warmup, case, gpus = 16, 2, 1, "sod", 1
    bench.run_reference(Args, 1, 0)
    lines = [ln for ln in capsys.readouterr().out.splitlines() if ln.startswith("{")]
    assert len(lines) == 1
    d = json.loads(lines[0])
    assert d["impl"] == "reference" and d["metric"] == bench.METRIC and d["unit"] == bench.UNIT
    assert d["higher_is_better"] is True and d["steps"] == 2 and d["warmup"] == 1 and d["n_gpus"] == 1
    assert d["config"]["workload"] == bench.workload_name("sod", 16) and d["config"]["grid"] == [16, 16, 16]
    assert d["value"] > 0 and d["cpu_baseline"]["value"] == d["value"]
    assert d["cpu_baseline"]["kind"] == "port" and d["cpu_baseline"]["cores"] >= 1
    assert d["e2e"] == {"value": d["value"], "unit": bench.UNIT, "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0}
