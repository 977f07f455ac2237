"""Launch-shape autotuner for the sweep.

The sweep's kernels are grid-stride loops over device lists, and the spatial pass
tests several candidate draws of a contact in parallel lanes.  Neither choice
changes results (every list is read order-independently and each draw has its own
fixed random numbers), so the tuner may pick whatever runs fastest: it times a
short throwaway realisation, seeded heavily so that the sweeps carry load, under
each candidate and keeps the best.
"""
import itertools

import numpy as np

from . import abi

GRIDS_PER_SM = (2, 4, 8, 16)
LANES = (2, 4, 8, 16)


def autotune(simulation, n_sm=148, grids_per_sm=GRIDS_PER_SM, lanes=LANES, steps=24, seed_frac=0.02, seed=4040):
    """Time `steps` timesteps of a realisation seeded with `seed_frac` of the
    population under each (grid, lanes) setting; apply and return the fastest as
    {"grid": blocks, "spatial_lanes": lanes, "ms": {setting: ms}}."""
    import torch
    be = simulation.backend
    P = simulation.params
    n_seed = max(1, int(simulation.pop.n_people * seed_frac))
    seeds = simulation.choose_seeds(seed, n_seed)
    stream = torch.cuda.ExternalStream(be.stream())
    timings = {}
    for g, ln in itertools.product(grids_per_sm, lanes):
        be.set_grid(n_sm * g)
        be.set_spatial_lanes(ln)
        be.begin_run(seed, seeds)
        for k in range(4):                          # capture the step graph, warm up
            be.step(k * P.ModelTimeStep, 0)
        e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        e0.record(stream)
        for k in range(4, 4 + steps):
            be.step(k * P.ModelTimeStep, 0)
        e1.record(stream)
        be.sync()
        timings[(g, ln)] = e0.elapsed_time(e1)
    (g, ln) = min(timings, key=timings.get)
    be.set_grid(n_sm * g)
    be.set_spatial_lanes(ln)
    return {"grid": n_sm * g, "spatial_lanes": ln,
            "ms": {"%dx%d" % k: round(v, 3) for k, v in sorted(timings.items())}}


def autotune_batch(batch, n_sm=148, grids_per_sm=(1, 2, 4, 8), lanes=(2, 4, 8), steps=12, seed_frac=0.02, seed=4040):
    """autotune for a sim.Batch: every member starts a throwaway realisation
    seeded with `seed_frac` of its population; each (grid, lanes) setting is timed
    over `steps` batched timesteps and the fastest is applied."""
    import torch
    stream = torch.cuda.ExternalStream(batch.stream())
    dt = batch.sims[0].params.ModelTimeStep
    timings = {}
    for g, ln in itertools.product(grids_per_sm, lanes):
        batch.set_grid(n_sm * g)
        batch.set_spatial_lanes(ln)
        for k, s in enumerate(batch.sims):
            n_seed = max(1, int(s.pop.n_people * seed_frac))
            s.backend.begin_run(seed + k, s.choose_seeds(seed + k, n_seed))
        for k in range(3):
            batch.step(k * dt)
        e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        e0.record(stream)
        for k in range(3, 3 + steps):
            batch.step(k * dt)
        e1.record(stream)
        batch.sync()
        timings[(g, ln)] = e0.elapsed_time(e1)
    (g, ln) = min(timings, key=timings.get)
    batch.set_grid(n_sm * g)
    batch.set_spatial_lanes(ln)
    return {"grid": n_sm * g, "spatial_lanes": ln,
            "ms": {"%dx%d" % k: round(v, 3) for k, v in sorted(timings.items())}}
