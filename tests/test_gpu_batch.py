"""Realisations stepped together: replicas sharing one population's static device
arrays, batches stepping several members with one graph per timestep, and the
launch-shape setting the tuner varies.  Each must give, state for state, what a
lone context (itself bit-exact to the oracle) gives for the same seed."""
import ctypes as C

import numpy as np
import pytest

from covidsim_b200 import abi, sim
import oracle_py
from tests.helpers import tiny_world, snapshot, STATE_FIELDS

pytestmark = pytest.mark.gpu


def _same(a, b, where):
    for k in STATE_FIELDS:
        assert np.array_equal(a[k], b[k]), "%s: %s differs at %d entries" % (where, k, int(np.sum(a[k] != b[k])))


def _steps(s, n, t0=0):
    for k in range(t0, t0 + n):
        s.backend.step(k * s.params.ModelTimeStep, 0)


def test_replica_matches_oracle():
    pop, P, lk, hr = tiny_world()
    base = sim.Simulation(pop, P, lk, hr)
    rep = base.replica()
    o = sim.Simulation(pop, P, lk, hr, backend=oracle_py.OracleBackend)
    seeds = base.choose_seeds(77, 20)
    # the base runs too, so the two realisations use the shared arrays side by side
    base.backend.begin_run(78, seeds)
    rep.backend.begin_run(77, seeds)
    o.backend.begin_run(77, seeds)
    for k in range(50):
        t = k * P.ModelTimeStep
        base.backend.step(t, 0)
        rep.backend.step(t, 0)
        o.backend.step(t, 0)
        if k == 30:
            rep.backend.update_probs(0)
            o.backend.update_probs(0)
    _same(snapshot(rep.backend, pop), snapshot(o.backend, pop), "replica vs oracle")
    ca, cb = abi.counters_to_dict(rep.backend.counters()), abi.counters_to_dict(o.backend.counters())
    assert ca == cb
    # destroying the base leaves the replica's shared arrays alive
    base.close()
    _steps(rep, 10, 50)
    o_more = o
    for k in range(50, 60):
        o_more.backend.step(k * P.ModelTimeStep, 0)
    _same(snapshot(rep.backend, pop), snapshot(o.backend, pop), "after the base was destroyed")
    rep.close()
    o.close()


def test_batch_matches_lone_contexts():
    w1 = tiny_world()
    w2 = tiny_world(n_people=12000, seed=4711)
    a = sim.Simulation(*w1)
    P2 = abi.cs_params.from_buffer_copy(w1[1])
    P2.LocalBeta = w1[1].LocalBeta * 1.3          # a member with its own parameters
    b = a.replica(P2)
    c = sim.Simulation(*w2)
    members = [a, b, c]
    seeds = [11, 12, 13]
    batch = sim.Batch(members)
    got = batch.run(seeds, days=12, n_seed=25)
    snaps = [snapshot(m.backend, m.pop) for m in members]
    batch.close()
    # the same realisations, each on a lone context
    lone = [sim.Simulation(*w1), sim.Simulation(w1[0], P2, w1[2], w1[3]), sim.Simulation(*w2)]
    for k, (m, seed) in enumerate(zip(lone, seeds)):
        ref = m.run(seed, days=12, n_seed=25)
        for key in ref:
            assert np.array_equal(ref[key], got[k][key]), "member %d series %s" % (k, key)
        _same(snapshot(m.backend, m.pop), snaps[k], "member %d" % k)
        m.close()
    # members work on their own again once the batch is gone
    _steps(a, 4, 48)
    for m in members:
        m.close()


def test_launch_shape_does_not_change_results():
    pop, P, lk, hr = tiny_world()
    ref = sim.Simulation(pop, P, lk, hr)
    ref.run(31, days=15, n_seed=20)
    want = snapshot(ref.backend, pop)
    for grid, lanes in ((148 * 2, 8), (148 * 8, 4), (148 * 16, 16), (148 * 4, 2)):
        alt = ref.replica()
        alt.backend.set_grid(grid)
        alt.backend.set_spatial_lanes(lanes)
        alt.run(31, days=15, n_seed=20)
        _same(snapshot(alt.backend, pop), want, "grid %d, %d spatial lanes" % (grid, lanes))
        alt.close()
    ref.close()


def test_autotuner_picks_a_setting_and_keeps_results():
    from covidsim_b200 import tune
    pop, P, lk, hr = tiny_world()
    s = sim.Simulation(pop, P, lk, hr)
    s.run(41, days=10, n_seed=20)
    want = snapshot(s.backend, pop)
    best = tune.autotune(s, steps=8)
    assert best["grid"] % 148 == 0 and best["spatial_lanes"] in (2, 4, 8, 16) and len(best["ms"]) == 16
    s.run(41, days=10, n_seed=20)
    _same(snapshot(s.backend, pop), want, "after tuning")
    s.close()


def test_ensemble_split_by_realisation_gives_the_same_members():
    """The multi-GPU ensemble split (bench.py ensemble_share: every world-th member to
    each rank) on one GPU: two batches, one per rank's share, yield each member's
    daily series exactly as one batch holding every member does, so gathering the
    ranks' series reproduces the single-process ensemble."""
    import importlib.util
    import os
    spec = importlib.util.spec_from_file_location("_bench", os.path.join(os.path.dirname(os.path.dirname(
        os.path.abspath(__file__))), "bench.py"))
    bench = importlib.util.module_from_spec(spec)
    spec.loader.exec_module(bench)
    pop, P, lk, hr = tiny_world()
    n, world, days = 5, 2, 25
    seeds = [3100 + 7 * k for k in range(n)]
    policy = sim.InterventionPolicy(threshold=2, duration=10.0)

    def members(idx):
        base = sim.Simulation(pop, P, lk, hr)
        return [base] + [base.replica() for _ in idx[1:]]
    everyone = members(list(range(n)))
    whole = sim.Batch(everyone).run(seeds, days, n_seed=20, policy=policy)
    shares = [bench.ensemble_share(n, r, world) for r in range(world)]
    got = [None] * n
    for share in shares:
        ms = members(share)
        out = sim.Batch(ms).run([seeds[k] for k in share], days, n_seed=20, policy=policy)
        for k, ser in zip(share, out):
            got[k] = ser
        for m in ms:
            m.close()
    for k in range(n):
        for key in whole[k]:
            assert np.array_equal(whole[k][key], got[k][key]), "member %d: %s differs" % (k, key)
    assert sorted(sum(shares, [])) == list(range(n))
    assert max(int(whole[k]["cumI"][-1]) for k in range(n)) > 500
    for m in everyone:
        m.close()
