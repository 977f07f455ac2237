"""GPU sweep against the CPU oracle at the size of the 1M-person workload (1,000,000
people on 240 x 240 cells of 10 x 10 microcells), state for state.

The GPU advances the epidemic to its peak region (a few hundred timesteps the oracle
would take minutes for); its full state is then handed to the oracle and back to
the GPU through the state-transfer entry points, so both continue from the same
state with the same seed.  Over the next 40 timesteps -- the busiest of the run,
with interventions (case isolation, household quarantine, social distancing and
school/university closure) switched on a quarter of the way in -- every per-person
field, cell list and counter must stay identical."""
import numpy as np
import pytest

from covidsim_b200 import abi, params as prm, population, sim
import oracle_py
from tests.helpers import snapshot, STATE_FIELDS

pytestmark = pytest.mark.gpu


def _compare(pop, g, o, where):
    a, b = snapshot(g.backend, pop), snapshot(o.backend, pop)
    for k in STATE_FIELDS:
        if not np.array_equal(a[k], b[k]):
            bad = np.nonzero(a[k] != b[k])[0]
            raise AssertionError("%s: field %s differs at %d entries, first %s" % (where, k, len(bad), bad[:5]))
    ca, cb = abi.counters_to_dict(g.backend.counters()), abi.counters_to_dict(o.backend.counters())
    assert ca == cb, "%s: counters differ" % where
    return a


def test_parity_at_one_million_people_around_the_peak():
    pop = population.preset("c0")
    P, lk, hr = prm.build_params(pop.grid)
    P.LocalBeta, _ = sim.calibrate_local_beta(pop, P, 2.4)
    g = sim.Simulation(pop, P, lk, hr)
    seed = 5151
    g.backend.begin_run(seed, g.choose_seeds(seed, 100))
    # to the peak region on the GPU alone: the first day-end on which prevalence falls
    step, I_prev = 0, -1
    while step < 4 * 200:
        g.backend.step(step * P.ModelTimeStep, 0)
        step += 1
        if step % 4 == 0:
            c = g.backend.counters()
            if c.I < I_prev and c.I > 0.02 * pop.n_people:
                break
            I_prev = c.I
    assert step < 4 * 200, "no epidemic peak within 200 days"
    arrs, view = sim.state_arrays(pop.n_people, pop.n_cells)
    g.backend.download(view)
    o = sim.Simulation(pop, P, lk, hr, backend=oracle_py.OracleBackend)
    for s in (g, o):
        s.backend.upload(seed, view)
    _compare(pop, g, o, "after the hand-over at step %d" % step)
    socd = [np.zeros(pop.n_mcells, dtype=np.uint8) for _ in range(2)]
    for k in range(40):
        t = (step + k) * P.ModelTimeStep
        if k == 10:
            for s, sd in zip((g, o), socd):
                s._switch_interventions(t, sim.InterventionPolicy(duration=30.0), True, sd)
        for s in (g, o):
            s.backend.step(t, 0)
        if k % 10 == 9:
            _compare(pop, g, o, "step %d (%d after the hand-over)" % (step + k, k + 1))
    c = g.backend.counters()
    assert c.I > 0.02 * pop.n_people and c.cumHQ > 0 and c.cumDC > 0
    g.close()
    o.close()
