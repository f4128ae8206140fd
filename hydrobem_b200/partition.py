"""Independent (body, frequency) units over the GPUs of a node, one process per GPU.

The reference runs the frequencies of a solve on separate workers with disjoint outputs: the next free
worker takes the next frequency (``crates/hydrobem/src/solve_driver.rs:275-282``,
``parallel.rs:59-97``).  Across GPUs the same independence holds with no exchange step, so the units are
split statically before the solve and nothing crosses NVLink on the data path:

- a unit (body b, frequency f) costs about ``N_b^3`` (its LU) plus ``c N_b^2`` (its assembly and
  right-hand sides); a body's statics cost ``s N_b^2`` once on every rank that takes any of its
  frequencies (they are replicated, never shipped);
- the units are laid out body by body, heaviest body first, and cut into ``world`` contiguous runs of
  about equal cost (the statics of each body a run touches included): a body is split over at most a
  few neighbouring ranks, so little statics work is repeated;
- each rank solves its runs through the library's batched entry (``hbg_solve_batch``: one problem per
  body run, frequencies batched on the device) and the outputs -- a few kB per unit -- are gathered on
  rank 0 by ``torch.distributed`` (``gather_object``) and put back in body and frequency order.

The planner and the gather are plain host code; ``solve_partitioned`` takes the solve as a function so
that the same logic runs on CPU ranks (gloo) with a stand-in solver in the tests.
"""

from __future__ import annotations

from dataclasses import dataclass

import numpy as np

# relative costs per unit and per body (panels N): the LU (8/3 N^3 flops on the tensor cores) against
# the assembly (N^2 pair kernels, ~1e3 flop-equivalents each) and the statics (N^2 closed forms, ~3e3)
ASSEMBLY_WEIGHT = 1.0e3
STATICS_WEIGHT = 3.0e3


def unit_cost(n_panels: int) -> float:
    n = float(n_panels)
    return n ** 3 + ASSEMBLY_WEIGHT * n * n


def statics_cost(n_panels: int) -> float:
    n = float(n_panels)
    return STATICS_WEIGHT * n * n


@dataclass(frozen=True)
class Run:
    """Frequencies f0 .. f1 - 1 of body ``body``."""

    body: int
    f0: int
    f1: int


def plan(sizes, world: int) -> list[list[Run]]:
    """Runs of every rank for bodies of ``sizes`` = [(n_panels, n_frequencies), ...].

    The bodies in order of decreasing total cost, their units one after the other, cut where a rank's
    running cost reaches total / world; a cut inside a body makes both sides pay its statics.  Every
    unit is in exactly one run; ranks past the last unit get none."""
    if world < 1:
        raise ValueError("world must be at least 1")
    cost = [f * unit_cost(n) + statics_cost(n) if f > 0 else 0.0 for n, f in sizes]
    order = sorted(range(len(sizes)), key=lambda b: -cost[b])
    target = sum(cost) / world
    out: list[list[Run]] = [[] for _ in range(world)]
    rank, load = 0, 0.0
    for b in order:
        n, F = sizes[b]
        f = 0
        while f < F:
            if rank < world - 1 and load >= target * 0.999:
                rank, load = rank + 1, 0.0
            load += statics_cost(n)
            u = unit_cost(n)
            # the frequencies of this body that fit the rank's share (at least one; the last rank all)
            room = max(1, int(round((target - load) / u))) if rank < world - 1 else F - f
            f1 = min(F, f + room)
            out[rank].append(Run(b, f, f1))
            load += (f1 - f) * u
            f = f1
            if f < F:  # the rank's share is used up inside this body: the rest goes to the next rank
                rank, load = rank + 1, 0.0
    return out


def rank_loads(sizes, runs: list[list[Run]]) -> list[float]:
    """The modelled cost of each rank's runs (statics of every run included)."""
    return [sum(statics_cost(sizes[r.body][0]) + (r.f1 - r.f0) * unit_cost(sizes[r.body][0]) for r in rs)
            for rs in runs]


def solve_partitioned(bodies, solve_runs, rank: int = 0, world: int = 1, pg=None):
    """Solve ``bodies`` (objects with ``vertices`` [P][4][3] and ``omegas``) split over ``world`` ranks.

    ``solve_runs(runs)`` solves this rank's runs and returns one dict of per-frequency arrays per run
    (leading axis: the run's frequencies).  Rank 0 returns, per body, the dict of arrays over all its
    frequencies; the other ranks return None.  ``pg`` is ``torch.distributed`` (initialised) or None
    for one process."""
    sizes = [(len(b.vertices), len(b.omegas)) for b in bodies]
    runs = plan(sizes, world)[rank]
    mine = solve_runs(runs)
    if len(mine) != len(runs):
        raise RuntimeError("the solver returned a different number of runs than it was given")
    payload = [(r.body, r.f0, r.f1, res) for r, res in zip(runs, mine)]
    if pg is None or world == 1:
        gathered = [payload]
    else:
        gathered = [None] * world if rank == 0 else None
        pg.gather_object(payload, gathered, dst=0)
    if rank != 0:
        return None
    out: list[dict | None] = [None] * len(bodies)
    filled = [np.zeros(len(b.omegas), dtype=bool) for b in bodies]
    for part in gathered:
        for b, f0, f1, res in part:
            if out[b] is None:
                F = len(bodies[b].omegas)
                out[b] = {k: np.zeros((F,) + np.asarray(v).shape[1:], dtype=np.asarray(v).dtype) for k, v in res.items()}
            if filled[b][f0:f1].any():
                raise RuntimeError(f"body {b}: frequencies {f0}..{f1 - 1} solved twice")
            for k, v in res.items():
                out[b][k][f0:f1] = v
            filled[b][f0:f1] = True
    for b, m in enumerate(filled):
        if not m.all():
            raise RuntimeError(f"body {b}: frequencies {np.flatnonzero(~m).tolist()} were not solved")
    return out


def gpu_solve_runs(bodies, **options):
    """The ``solve_runs`` of a GPU rank: one problem per run (the body with the run's frequencies) in
    one ``hbg_solve_batch`` call on this process's device; returns A, B, X, FK, SC, HK per run."""
    from . import native as nv

    def solve(runs):
        probs = []
        for r in runs:
            b = bodies[r.body]
            probs.append(nv.Body(b.vertices, np.asarray(b.omegas)[r.f0:r.f1], b.headings, b.kinds, b.panel_body,
                                 b.centers, b.symmetry))
        if not probs:
            return []
        res = nv.solve_batch(probs, **options)
        return [{k: r[k] for k in ("A", "B", "X", "FK", "SC", "HK")} for r in res]

    return solve
