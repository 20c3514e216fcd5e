"""The multi-process path of bench.py on CPU (gloo, world size 2).

bench.py --gpus N runs one replica of the workload per rank (particles are
independent, so there is no collective on the data path).  Its host logic is
what these tests cover without a GPU: the rank environment, the maximum of the
timed region over ranks (the job is as slow as its slowest rank), the
whole-job throughput, and the reference arm's ranks other than 0 exiting
without work.
"""
from __future__ import annotations

import json
import os
import socket
import subprocess
import sys
from pathlib import Path

import pytest

ROOT = Path(__file__).resolve().parents[1]


def _free_port() -> int:
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        return s.getsockname()[1]


def _rank_main(rank: int, world: int, port: int, out_dir: str) -> None:
    import datetime

    import torch.distributed as dist

    sys.path.insert(0, str(ROOT))
    os.environ.update(RANK=str(rank), WORLD_SIZE=str(world), LOCAL_RANK=str(rank))
    import bench

    dist.init_process_group("gloo", init_method=f"tcp://127.0.0.1:{port}", rank=rank, world_size=world,
                            timeout=datetime.timedelta(seconds=60))
    try:
        w, r, local = bench._dist()
        # each replica "times" its region; rank 1 is the slow one
        dist.barrier()
        mine = [0.25, 1.75][rank]
        slowest = bench.max_over_ranks(dist, mine, "cpu")
        dist.barrier()
        units = 1.0e10  # particle-steps of one replica
        rate = bench.whole_job_rate(w, units, slowest)
        Path(out_dir, f"rank{rank}.json").write_text(json.dumps(
            {"world": w, "rank": r, "local": local, "mine": mine, "slowest": slowest, "rate": rate}))
    finally:
        dist.destroy_process_group()


def test_two_rank_reduction_gloo(tmp_path):
    import torch.multiprocessing as mp

    port = _free_port()
    ctx = mp.get_context("spawn")
    procs = [ctx.Process(target=_rank_main, args=(k, 2, port, str(tmp_path))) for k in range(2)]
    for p in procs:
        p.start()
    for p in procs:
        p.join(120)
    for p in procs:
        if p.is_alive():
            p.kill()
            pytest.fail("a rank did not finish")
        assert p.exitcode == 0
    res = [json.loads((tmp_path / f"rank{k}.json").read_text()) for k in range(2)]
    for k, r in enumerate(res):
        assert (r["world"], r["rank"], r["local"]) == (2, k, k)
        assert r["slowest"] == 1.75                   # every rank sees the max
        assert r["rate"] == pytest.approx(2 * 1.0e10 / 1.75)


def test_single_process_has_no_collective():
    sys.path.insert(0, str(ROOT))
    import bench

    assert bench.max_over_ranks(None, 0.5, "cpu") == 0.5
    assert bench.whole_job_rate(1, 3.0e9, 1.5) == pytest.approx(2.0e9)


def test_reference_arm_other_ranks_exit_without_work():
    env = dict(os.environ, RANK="1", WORLD_SIZE="2", LOCAL_RANK="1")
    r = subprocess.run([sys.executable, str(ROOT / "bench.py"), "--impl", "reference", "--gpus", "2",
                        "--steps", "1", "--warmup", "3"], cwd=ROOT, env=env, capture_output=True, text=True,
                       timeout=120)
    assert r.returncode == 0
    assert r.stdout.strip() == ""
