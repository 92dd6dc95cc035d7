"""The multi-rank plumbing of bench.py on CPU: two gloo ranks on 127.0.0.1 run the
rank barrier and the max-over-ranks reduction the timed region uses, and the
reference arm does no work on ranks other than 0."""
import os
import socket

import pytest
import torch.distributed as dist
import torch.multiprocessing as mp


def _free_port() -> int:
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        return s.getsockname()[1]


def _rank_main(rank, world, port, q):
    import datetime

    import bench
    os.environ.update(MASTER_ADDR="127.0.0.1", MASTER_PORT=str(port))
    dist.init_process_group("gloo", rank=rank, world_size=world, timeout=datetime.timedelta(seconds=60))
    try:
        bench.rank_barrier(dist, cuda=False)
        ms = 10.0 * (rank + 1)  # each rank's own elapsed time
        worst = bench.rank_max(ms, dist, device="cpu")
        bench.rank_barrier(dist, cuda=False)
        q.put((rank, worst))
    finally:
        dist.destroy_process_group()


def test_two_gloo_ranks_take_the_slowest_time():
    world, port = 2, _free_port()
    ctx = mp.get_context("spawn")
    q = ctx.Queue()
    procs = [ctx.Process(target=_rank_main, args=(r, world, port, q)) for r in range(world)]
    for p in procs:
        p.start()
    for p in procs:
        p.join(120)
        assert p.exitcode == 0
    got = dict(q.get(timeout=10) for _ in range(world))
    assert got == {0: 20.0, 1: 20.0}


def test_reference_arm_is_rank0_only(capsys):
    import argparse

    import bench
    args = argparse.Namespace(steps=1, warmup=0, workload="mri", gpus=2)
    bench.run_reference(args, rank=1)
    assert capsys.readouterr().out == ""


def test_single_process_max_is_identity():
    import bench
    assert bench.rank_max(3.5, None) == 3.5


def test_reference_arm_loads_no_product_library():
    """The reference arm runs the oracle alone: its initial state comes from the oracle's own
    problem set-up, so libdumses_gpu.so is never mapped into the process."""
    import json
    import pathlib
    import subprocess
    import sys
    root = pathlib.Path(__file__).resolve().parents[1]
    code = ("import argparse, bench; bench.run_reference(argparse.Namespace(steps=1, warmup=1, workload='mri', gpus=1, "
            "n=16, nu=0.0, eta=0.0), 0); print('MAPS', open('/proc/self/maps').read().count('libdumses_gpu'), "
            "open('/proc/self/maps').read().count('liboracle'))")
    out = subprocess.run([sys.executable, "-c", code], cwd=root, capture_output=True, text=True, timeout=300)
    assert out.returncode == 0, out.stderr
    line = json.loads(out.stdout.splitlines()[0])
    assert line["impl"] == "reference" and line["value"] > 0 and line["config"]["grid"] == [16, 16, 16]
    maps = out.stdout.splitlines()[-1].split()
    assert maps[0] == "MAPS" and int(maps[1]) == 0 and int(maps[2]) > 0
