"""The multi-rank host logic of bench.py with two gloo ranks on CPU.

A run on N GPUs is one process per GPU: every rank solves its own scenes
(no collective on the data path), the job's time is the maximum of the
ranks' device times, and the whole-job rate counts every rank's scenes
over that time.  The reference arm prints from rank 0 only.
"""

import json
import os
import socket
import subprocess
import sys
from pathlib import Path

import pytest

torch = pytest.importorskip("torch")
import torch.distributed as dist  # noqa: E402
import torch.multiprocessing as mp  # noqa: E402

REPO = Path(__file__).resolve().parents[1]


def _free_port() -> int:
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        return s.getsockname()[1]


def _worker(rank: int, world: int, port: int, out_dir: str) -> None:
    sys.path.insert(0, str(REPO))
    import bench

    os.environ.update(MASTER_ADDR="127.0.0.1", MASTER_PORT=str(port))
    dist.init_process_group("gloo", rank=rank, world_size=world)
    try:
        seeds = list(bench.shard_seeds(rank, 4))
        gathered = [None] * world
        dist.all_gather_object(gathered, seeds)
        my_ms = 10.0 + 5.0 * rank  # rank 1 is the slow one
        job = bench.max_over_ranks(my_ms, dist, torch.device("cpu"))
        rate = bench.job_rate(4, 3, world, job)
        Path(out_dir, f"r{rank}.json").write_text(json.dumps({"seeds": gathered, "job": job, "rate": rate}))
        dist.barrier()
    finally:
        dist.destroy_process_group()


def test_two_gloo_ranks_shard_scenes_and_time_the_slowest(tmp_path):
    world = 2
    mp.start_processes(_worker, args=(world, _free_port(), str(tmp_path)), nprocs=world, start_method="spawn")
    res = [json.loads((tmp_path / f"r{r}.json").read_text()) for r in range(world)]
    seeds = res[0]["seeds"]
    assert res[1]["seeds"] == seeds
    flat = [s for part in seeds for s in part]
    assert sorted(flat) == list(range(8)) and len(set(flat)) == 8  # disjoint, complete
    for r in res:
        assert r["job"] == 15.0  # the maximum over ranks, on every rank
        assert r["rate"] == pytest.approx(4 * 3 * 2 / 0.015)


def test_reference_arm_prints_from_rank_zero_only():
    env = dict(os.environ, RANK="1", WORLD_SIZE="2", PYTHONPATH=str(REPO))
    r = subprocess.run([sys.executable, str(REPO / "bench.py"), "--impl", "reference", "--steps", "1",
                        "--warmup", "1"], capture_output=True, text=True, env=env, timeout=300)
    assert r.returncode == 0
    assert r.stdout.strip() == ""
