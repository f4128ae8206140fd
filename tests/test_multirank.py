"""The multi-rank host logic of the benchmark on CPU: two gloo ranks set up through the same
environment torchrun gives (RANK, WORLD_SIZE, MASTER_ADDR 127.0.0.1), the job time reduced as the
maximum over ranks, and the reference arm run by rank 0 alone while the other rank exits without
work.  The GPU replicas themselves share no data (independent frequency units, no collective)."""

from __future__ import annotations

import json
import os
import socket
import sys
from pathlib import Path

import pytest

ROOT = Path(__file__).resolve().parents[1]


def _free_port():
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        return s.getsockname()[1]


def _rank_main(rank, world, port, out_dir, mode):
    os.environ.update({"RANK": str(rank), "LOCAL_RANK": str(rank), "WORLD_SIZE": str(world),
                       "MASTER_ADDR": "127.0.0.1", "MASTER_PORT": str(port)})
    sys.path.insert(0, str(ROOT))
    import argparse

    import bench

    world_, rank_, local, pg = bench.dist_setup()
    try:
        if mode == "reduce":
            res = bench.reduce_max(pg, [rank + 1.0, 5.0 - rank])
        else:
            bench.CASE = "tiny"
            args = argparse.Namespace(steps=1, warmup=0)
            res = bench.cpu_reference(args, world_, rank_, pg)
        Path(out_dir, f"rank{rank}.json").write_text(json.dumps(res))
    finally:
        pg.destroy_process_group()


def _spawn(mode, tmp_path, world=2):
    import torch.multiprocessing as mp

    port = _free_port()
    mp.spawn(_rank_main, args=(world, port, str(tmp_path), mode), nprocs=world, join=True)
    return [json.loads(Path(tmp_path, f"rank{r}.json").read_text()) for r in range(world)]


def test_job_time_is_the_max_over_two_gloo_ranks(tmp_path):
    pytest.importorskip("torch")
    out = _spawn("reduce", tmp_path)
    assert out[0] == out[1] == [2.0, 5.0]


def test_reference_arm_runs_on_rank_zero_only(tmp_path):
    pytest.importorskip("torch")
    out = _spawn("reference", tmp_path)
    line, other = out
    assert other is None
    assert line["impl"] == "reference" and line["n_gpus"] == 2
    assert line["value"] > 0 and line["cpu_baseline"]["kind"] == "port"
    assert line["e2e"]["h2d_bytes_per_step"] == 0
