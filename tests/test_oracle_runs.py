"""The CPU oracle on its own: conservation, cell-list invariants, determinism."""
import numpy as np

from covidsim_b200 import sim
import oracle_py
from tests.helpers import tiny_world, snapshot, check_lists


def _run(seed, steps, n_seed=20, world=None):
    pop, P, lk, hr = world or tiny_world()
    s = sim.Simulation(pop, P, lk, hr, backend=oracle_py.OracleBackend)
    be = s.backend
    be.begin_run(seed, s.choose_seeds(seed, n_seed))
    out = []
    for k in range(steps):
        be.step(k * P.ModelTimeStep, 0)
        out.append(abi_counts(be.counters()))
    return s, be, out


def abi_counts(c):
    return (c.S, c.L, c.I, c.R, c.D, c.cumI, c.cumC, c.cumDC, c.Critical, c.cumCritical)


def test_conservation_and_lists():
    pop, P, lk, hr = tiny_world()
    s, be, out = _run(7, 160)
    for row in out:
        assert sum(row[:5]) == pop.n_people
    assert out[-1][5] > 200          # the epidemic took off
    snap = snapshot(be, pop)
    check_lists(snap, pop)
    assert (snap["inf"] != 0).sum() == out[-1][5]


def test_deterministic_per_seed():
    _, _, a = _run(11, 80)
    _, _, b = _run(11, 80)
    _, _, c = _run(12, 80)
    assert a == b
    assert a != c


def test_update_probs_renormalises():
    pop, P, lk, hr = tiny_world()
    s, be, out = _run(3, 200)
    be.update_probs(0)
    snap = snapshot(be, pop)
    S0 = snap["cell_S"] + snap["cell_L"] + snap["cell_I"]
    assert np.array_equal(snap["cell_S0"], S0)
    tp = snap["cell_tot_prob"]
    assert np.all((tp > 0) & (tp <= 1.0))
    assert tp.min() < 1.0
