"""The split of independent (body, frequency) units over ranks (hydrobem_b200.partition): every unit in
exactly one run, the modelled cost balanced on the 64-body configuration, and the partitioned result --
two gloo ranks on CPU, each solving its runs with a stand-in solver, gathered on rank 0 -- equal to the
result of one rank solving everything."""

from __future__ import annotations

import json
import os
import socket
import sys
from pathlib import Path

import numpy as np
import pytest

from hydrobem_b200 import partition as pt

ROOT = Path(__file__).resolve().parents[1]


def c3_sizes():
    """Panel and frequency counts of the 64-body configuration, drawn as meshes.uneven_bodies draws its
    bodies (seed 20261203: cylinders with n_phi (n_z + n_r) panels, n_r = n_z, or hemispheres with
    n_theta n_phi panels; N ~ U[800, 6000] rounded to those grids; 16 frequencies each)."""
    rng = np.random.default_rng(20261203)
    out = []
    for _ in range(64):
        rng.uniform(0.5, 3.0), rng.uniform(0.3, 2.0)
        n = int(rng.uniform(800, 6000))
        if rng.uniform() < 0.5:
            nphi = max(8, int(round(np.sqrt(n) / 4)) * 4)
            nz = max(2, int(round(n / (2 * nphi))))
            panels = 2 * nphi * nz
        else:
            nphi = max(8, int(round(np.sqrt(2 * n) / 4)) * 4)
            panels = max(2, int(round(n / nphi))) * nphi
        rng.uniform(0.1, 10.0, 16)
        out.append((panels, 16))
    return out


def test_c3_sizes_follow_the_generators():
    """The counts above are those of the meshes the GPU tests build (a few bodies checked)."""
    from hydrobem_b200 import meshes

    sizes = c3_sizes()
    bodies = meshes.uneven_bodies(64)
    assert [(len(v), len(om)) for v, om in bodies] == sizes


def test_plan_covers_every_unit_once():
    sizes = [(1000, 7), (4096, 40), (300, 1), (2500, 16), (800, 0)]
    for world in (1, 2, 3, 4, 8, 64):
        runs = pt.plan(sizes, world)
        assert len(runs) == world
        seen = [np.zeros(f, int) for _, f in sizes]
        for rs in runs:
            for r in rs:
                assert 0 <= r.f0 < r.f1 <= sizes[r.body][1]
                seen[r.body][r.f0:r.f1] += 1
        assert all((s == 1).all() for s in seen), world


@pytest.mark.parametrize("world", [2, 4, 8])
def test_plan_balances_the_64_body_configuration(world):
    sizes = c3_sizes()
    runs = pt.plan(sizes, world)
    loads = pt.rank_loads(sizes, runs)
    assert max(loads) <= 1.05 * (sum(loads) / world), loads
    # statics repeated only where a body is cut: at most world - 1 cuts
    assert sum(len(rs) for rs in runs) - len(sizes) <= world - 1


class _B:
    def __init__(self, n, F, seed):
        self.vertices = np.zeros((n, 4, 3))
        self.omegas = np.linspace(0.5, 2.0, F) + seed


def _fake_solver(bodies):
    """A deterministic stand-in for the GPU solve: per-frequency arrays that depend on (body, omega)."""
    def solve(runs):
        out = []
        for r in runs:
            om = bodies[r.body].omegas[r.f0:r.f1]
            A = np.stack([np.full((6, 6), r.body + w) + np.eye(6) * w for w in om])
            X = np.stack([np.exp(1j * w * np.arange(12)).reshape(2, 6) * (r.body + 1) for w in om])
            out.append({"A": A, "X": X})
        return out
    return solve


def _bodies():
    return [_B(100 * (b + 1), 3 + 2 * b, 0.1 * b) for b in range(5)]


def _free_port():
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        return s.getsockname()[1]


def _rank_main(rank, world, port, out_dir):
    os.environ.update({"RANK": str(rank), "LOCAL_RANK": str(rank), "WORLD_SIZE": str(world),
                       "MASTER_ADDR": "127.0.0.1", "MASTER_PORT": str(port)})
    sys.path.insert(0, str(ROOT))
    import datetime

    import torch.distributed as dist

    from hydrobem_b200 import partition as p

    dist.init_process_group("gloo", timeout=datetime.timedelta(seconds=60))
    try:
        bodies = _bodies()
        res = p.solve_partitioned(bodies, _fake_solver(bodies), rank, world, dist)
        if rank == 0:
            enc = [{k: [np.real(v).tolist(), np.imag(v).tolist()] for k, v in r.items()} for r in res]
            Path(out_dir, "rank0.json").write_text(json.dumps(enc))
        else:
            Path(out_dir, f"rank{rank}.json").write_text(json.dumps(res))
    finally:
        dist.destroy_process_group()


def test_partitioned_result_equals_one_rank(tmp_path):
    pytest.importorskip("torch")
    import torch.multiprocessing as mp

    bodies = _bodies()
    one = pt.solve_partitioned(bodies, _fake_solver(bodies))
    mp.spawn(_rank_main, args=(2, _free_port(), str(tmp_path)), nprocs=2, join=True)
    got = json.loads(Path(tmp_path, "rank0.json").read_text())
    assert json.loads(Path(tmp_path, "rank1.json").read_text()) is None
    for b, r in enumerate(one):
        for k, v in r.items():
            g = np.array(got[b][k][0]) + 1j * np.array(got[b][k][1])
            assert np.array_equal(g, v), (b, k)


def test_a_missing_unit_is_an_error():
    bodies = _bodies()

    def bad(runs):
        out = _fake_solver(bodies)(runs)
        out[0]["A"] = out[0]["A"]
        return out[:-1]
    with pytest.raises(RuntimeError):
        pt.solve_partitioned(bodies, bad)
