"""Replica scheduler for parameter sweeps over several GPUs.

A phase-diagram sweep is many independent instances (the reference runs one
per process).  Here the instances are dealt out to the ranks of a
torch.distributed group (one process per GPU) so that every rank gets about
the same number of grid-point steps, each rank advances its share as one
batch (fortress_b200.Batch: one CUDA graph launch per group of steps), and
the per-instance results come back to every rank in the original order.
There is no data-path collective: the only exchange is the final gather of
small per-instance records.
"""
from __future__ import annotations

import numpy as np


def instance_cost(p):
    """Relative cost of one step of an instance: grid points x components."""
    return int(np.prod(p["n"])) * (2 * p["spin"] + 1)


def partition(costs, world):
    """Longest-processing-time-first assignment: instances sorted by cost
    (ties by index) go one by one to the least-loaded rank (ties to the lowest
    rank).  Returns one list of instance indices per rank, each in ascending
    order, and the per-rank loads."""
    order = sorted(range(len(costs)), key=lambda i: (-costs[i], i))
    load = [0] * world
    parts = [[] for _ in range(world)]
    for i in order:
        r = min(range(world), key=lambda q: (load[q], q))
        parts[r].append(i)
        load[r] += costs[i]
    return [sorted(p) for p in parts], load


def run(instances, work, rank=0, world=1, group=None):
    """Run work(my_instances, my_indices) -> list of per-instance records on
    this rank's share and gather all records on every rank, in the order of
    `instances`.  With world == 1 nothing is communicated."""
    parts, _ = partition([instance_cost(p) for p in instances], world)
    mine = parts[rank]
    recs = work([instances[i] for i in mine], mine)
    if len(recs) != len(mine):
        raise ValueError("work returned a different number of records than instances")
    if world == 1:
        return list(recs)
    import torch.distributed as dist
    gathered = [None] * world
    dist.all_gather_object(gathered, (mine, list(recs)), group=group)
    out = [None] * len(instances)
    for idx, rr in gathered:
        for i, r in zip(idx, rr):
            out[i] = r
    return out


def imaginary_time_work(steps, guess, with_state=False):
    """A `work` callable for run(): one Batch of the rank's instances, the
    guess(p) initial states normalised, `steps` imaginary-time steps, then
    per instance {en, mu, mz, rms, norm} (and the state if asked)."""
    def work(insts, idx):
        from .batch import Batch
        if not insts:
            return []
        b = Batch(insts)
        try:
            for i, p in enumerate(insts):
                b[i].set_state(guess(p))
                b[i].normt()
            b.step(steps)
            obs = b.observables(with_conv=False)
            recs = []
            for i, o in enumerate(obs):
                r = {k: (v.tolist() if hasattr(v, "tolist") else float(v)) for k, v in o.items() if k != "conv"}
                if with_state:
                    r["state"] = b[i].state()
                recs.append(r)
            return recs
        finally:
            b.close()
    return work
