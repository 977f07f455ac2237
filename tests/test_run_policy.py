"""The run loop's intervention policy on the host, with the oracle as the sweep:
the global trigger and the per-admin-unit triggers (staggered switches), and the
conversion of a policy to the cs_run_policy the device run loop takes."""
import numpy as np

from covidsim_b200 import abi, sim
import oracle_py
from tests.helpers import tiny_world


def _record_windows(s, n_adunits):
    """Each set_interventions call's per-admin-unit case isolation starts."""
    calls = []
    orig = s.backend.set_interventions

    def rec(iv):
        if iv.adunit_CaseIsolationTimeStart:
            arr = (abi.C.c_double * n_adunits).from_address(iv.adunit_CaseIsolationTimeStart)
            calls.append(np.ctypeslib.as_array(arr).copy())
        else:
            calls.append(np.full(n_adunits, iv.CaseIsolationTimeStart))
        orig(iv)
    s.backend.set_interventions = rec
    return calls


def test_per_adunit_triggers_switch_units_on_their_own_days():
    pop, P, lk, hr = tiny_world(adunit_grid=3)
    assert pop.n_adunits == 9
    o = sim.Simulation(pop, P, lk, hr, backend=oracle_py.OracleBackend)
    calls = _record_windows(o, pop.n_adunits)
    pol = sim.InterventionPolicy(threshold=1, window=7, duration=12.0, per_adunit=True)
    o.run(505, 60, n_seed=20, policy=pol)
    on = np.array([c < 1e9 for c in calls])            # [switch call, admin unit]
    assert len(calls) >= 3
    # units switch on at different days: the first call does not turn on every unit
    assert 0 < on[0].sum() < pop.n_adunits
    starts = {}
    for c in calls:
        for a in np.nonzero(c < 1e9)[0]:
            starts.setdefault(int(a), float(c[a]))
    assert len(set(starts.values())) > 1
    # a unit's window starts the day after its trigger fired and stays on for the duration
    for c_prev, c in zip(calls, calls[1:]):
        off = (c_prev < 1e9) & (c >= 1e9)
        for a in np.nonzero(off)[0]:
            assert starts[int(a)] + pol.duration <= 60 + 1
    o.close()


def test_global_and_per_unit_policies_differ_and_repeat():
    pop, P, lk, hr = tiny_world(adunit_grid=3)
    o = sim.Simulation(pop, P, lk, hr, backend=oracle_py.OracleBackend)
    a = o.run(606, 50, n_seed=20, policy=sim.InterventionPolicy(threshold=2, duration=10.0))
    b = o.run(606, 50, n_seed=20, policy=sim.InterventionPolicy(threshold=2, duration=10.0, per_adunit=True))
    b2 = o.run(606, 50, n_seed=20, policy=sim.InterventionPolicy(threshold=2, duration=10.0, per_adunit=True))
    assert not np.array_equal(a["cumI"], b["cumI"])
    for k in b:
        assert np.array_equal(b[k], b2[k])
    o.close()


def test_run_policy_conversion():
    pol = sim.InterventionPolicy(threshold=40, window=5, duration=30.0, close_place_types=(0, 2, 7),
                                 social_distancing=False, per_adunit=True)
    p = sim.run_policy(pol, 4, probs_every_step=True)
    assert (p.icu_trigger, p.icu_threshold, p.icu_window) == (1, 40, 5)
    assert (p.case_isolation, p.household_quarantine, p.social_distancing) == (1, 1, 0)
    assert p.close_place_types == 0b101 and p.per_adunit == 1 and p.probs_every_step == 1
    assert p.duration == 30.0
    q = sim.run_policy(None, 4)
    assert q.icu_trigger == 0 and q.probs_every_step == 0
