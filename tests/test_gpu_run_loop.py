"""The run loop on the device (cs_gpu_run): the logic between timesteps (day-end
counters, the UpdateProbs test on the susceptible fraction, the critical-care
trigger switching interventions on and off) evaluated by kernels in one graph per
day.  Day for day and state for state it must give what the same logic gives on
the host, and what the oracle gives under that host logic."""
import numpy as np
import pytest

from covidsim_b200 import abi, sim
import oracle_py
from tests.helpers import tiny_world, snapshot, STATE_FIELDS

pytestmark = pytest.mark.gpu

DAYS = 60


def _policy():
    # fires early in the tiny world's epidemic and switches off again inside the run
    return sim.InterventionPolicy(threshold=3, window=7, duration=12.0)


def _same_state(a, b, where):
    for k in STATE_FIELDS:
        assert np.array_equal(a[k], b[k]), "%s: %s differs at %d entries" % (where, k, int(np.sum(a[k] != b[k])))


def _same_series(a, b, where):
    for k in sim.SERIES:
        assert np.array_equal(np.asarray(a[k]), np.asarray(b[k])), "%s: series %s differs" % (where, k)


def _word_field(w):
    """The cs_counters field holding int64 word w of the block."""
    for name, t in abi.cs_counters._fields_:
        f = getattr(abi.cs_counters, name)
        if f.offset // 8 <= w < (f.offset + f.size) // 8:
            return name
    return "?"


def _instrument(s):
    """Record the host loop's UpdateProbs calls and intervention switches."""
    log = {"update": 0, "switch": []}
    up = s.backend.update_probs

    def update_probs(do_place=0):
        log["update"] += 1
        up(do_place)
    s.backend.update_probs = update_probs
    sw = s._switch_interventions

    def switch(t, policy, on, socd):
        log["switch"].append((t, on))
        sw(t, policy, on, socd)
    s._switch_interventions = switch
    return log


@pytest.mark.parametrize("every_step", [False, True])
def test_device_loop_matches_host_loop(every_step):
    pop, P, lk, hr = tiny_world()
    host = sim.Simulation(pop, P, lk, hr)
    log = _instrument(host)
    want, want_blocks = host.run(505, DAYS, n_seed=20, policy=_policy(), probs_every_step=every_step,
                                 device_loop=False, blocks=True)
    want_state = snapshot(host.backend, pop)
    # the run exercised what the loop decides
    assert log["update"] >= 1, log
    assert [on for _, on in log["switch"]] == [True, False], log
    dev = host.replica()
    got, got_blocks = dev.run(505, DAYS, n_seed=20, policy=_policy(), probs_every_step=every_step,
                              device_loop=True, blocks=True)
    _same_series(got, want, "device loop")
    # every counter of the block, at t = 0 and every day's end
    assert got_blocks.shape == want_blocks.shape == (DAYS + 1, abi.C.sizeof(abi.cs_counters) // 8)
    bad = np.nonzero((got_blocks != want_blocks).any(axis=0))[0]
    assert bad.size == 0, "counters differ: %s" % sorted({_word_field(w) for w in bad})
    _same_state(snapshot(dev.backend, pop), want_state, "device loop")
    # a second run on the same context replays the same graph from a fresh start
    again = dev.run(505, DAYS, n_seed=20, policy=_policy(), probs_every_step=every_step)
    _same_series(again, want, "second device run")
    _same_state(snapshot(dev.backend, pop), want_state, "second device run")
    dev.close()
    host.close()


def test_device_loop_matches_oracle():
    pop, P, lk, hr = tiny_world()
    o = sim.Simulation(pop, P, lk, hr, backend=oracle_py.OracleBackend)
    log = _instrument(o)
    g = sim.Simulation(pop, P, lk, hr)
    want = o.run(606, DAYS, n_seed=20, policy=_policy(), probs_every_step=True)
    assert log["update"] >= 1 and [on for _, on in log["switch"]] == [True, False], log
    got = g.run(606, DAYS, n_seed=20, policy=_policy(), probs_every_step=True)
    _same_series(got, want, "device loop vs oracle")
    _same_state(snapshot(g.backend, pop), snapshot(o.backend, pop), "device loop vs oracle")
    assert abi.counters_to_dict(g.backend.counters()) == abi.counters_to_dict(o.backend.counters())
    g.close()
    o.close()


def test_graph_and_eager_day_loops_agree():
    pop, P, lk, hr = tiny_world()
    a = sim.Simulation(pop, P, lk, hr)
    b = a.replica()
    b.backend.lib.cs_gpu_use_graphs(b.backend.ctx, 0)
    n0 = a.backend.launches()
    ra = a.run(707, 30, n_seed=20, policy=_policy())
    per_day_graph = (a.backend.launches() - n0) / 30
    n0 = b.backend.launches()
    rb = b.run(707, 30, n_seed=20, policy=_policy())
    per_day_eager = (b.backend.launches() - n0) / 30
    _same_series(ra, rb, "graph vs eager")
    _same_state(snapshot(a.backend, pop), snapshot(b.backend, pop), "graph vs eager")
    # both count the same kernels: four timesteps, the totals, the gated UpdateProbs,
    # the trigger, the flags and one closure kernel per place type
    assert per_day_graph == per_day_eager > 4 * 10
    b.close()
    a.close()


def test_run_loop_errors():
    pop, P, lk, hr = tiny_world()
    s = sim.Simulation(pop, P, lk, hr)
    with pytest.raises(abi.CovidSimError):
        s.backend.run_device(3, sim.run_policy(None, pop.num_place_types))   # before begin_run
    s.backend.begin_run(1, s.choose_seeds(1, 10))
    bad = sim.run_policy(_policy(), pop.num_place_types)
    bad.icu_window = 0
    with pytest.raises(abi.CovidSimError):
        s.backend.run_device(3, bad)
    # a run of no days does nothing
    assert s.backend.run_device(0, sim.run_policy(None, pop.num_place_types)).shape[0] == 0
    s.close()


@pytest.mark.parametrize("every_step", [[False, False, False], [False, True, False]])
def test_batch_device_loop_matches_lone_host_loops(every_step):
    w1 = tiny_world()
    w2 = tiny_world(n_people=12000, seed=4711)
    a = sim.Simulation(*w1)
    P2 = abi.cs_params.from_buffer_copy(w1[1])
    P2.LocalBeta = w1[1].LocalBeta * 1.3
    b = a.replica(P2)
    c = sim.Simulation(*w2)
    members = [a, b, c]
    policies = [_policy(), None, sim.InterventionPolicy(threshold=2, window=5, duration=8.0, close_place_types=(1, 3))]
    seeds = [21, 22, 23]
    batch = sim.Batch(members)
    got = batch.run(seeds, DAYS, n_seed=20, policy=policies, probs_every_step=every_step)
    snaps = [snapshot(m.backend, m.pop) for m in members]
    # the batch graph is kept and replayed by a second run
    again = batch.run(seeds, DAYS, n_seed=20, policy=policies, probs_every_step=every_step)
    batch.close()
    lone = [sim.Simulation(*w1), sim.Simulation(w1[0], P2, w1[2], w1[3]), sim.Simulation(*w2)]
    for k, (m, seed) in enumerate(zip(lone, seeds)):
        log = _instrument(m)
        want = m.run(seed, DAYS, n_seed=20, policy=policies[k], probs_every_step=every_step[k], device_loop=False)
        if policies[k] is not None:
            assert log["switch"], "member %d: the trigger never fired" % k
        _same_series(got[k], want, "member %d" % k)
        _same_series(again[k], want, "member %d, second run" % k)
        _same_state(snapshot(m.backend, m.pop), snaps[k], "member %d" % k)
        m.close()
    for m in members:
        m.close()


def _unit_policy():
    # staggered: each of the 9 admin units fires on its own admissions
    return sim.InterventionPolicy(threshold=1, window=7, duration=12.0, per_adunit=True)


@pytest.mark.parametrize("every_step", [False, True])
def test_per_adunit_device_loop_matches_host_loop_and_oracle(every_step):
    pop, P, lk, hr = tiny_world(adunit_grid=3)
    host = sim.Simulation(pop, P, lk, hr)
    calls = []
    orig = host.backend.set_interventions
    host.backend.set_interventions = lambda iv: (calls.append(1), orig(iv))
    want = host.run(505, DAYS, n_seed=20, policy=_unit_policy(), probs_every_step=every_step, device_loop=False)
    want_state = snapshot(host.backend, pop)
    assert len(calls) >= 3, "the admin units' triggers did not switch on different days"
    dev = host.replica()
    got = dev.run(505, DAYS, n_seed=20, policy=_unit_policy(), probs_every_step=every_step, device_loop=True)
    _same_series(got, want, "per admin unit, device loop")
    _same_state(snapshot(dev.backend, pop), want_state, "per admin unit, device loop")
    if every_step:
        o = sim.Simulation(pop, P, lk, hr, backend=oracle_py.OracleBackend)
        ow = o.run(505, DAYS, n_seed=20, policy=_unit_policy(), probs_every_step=True)
        _same_series(got, ow, "per admin unit, device loop vs oracle")
        _same_state(snapshot(dev.backend, pop), snapshot(o.backend, pop), "per admin unit, device loop vs oracle")
        o.close()
    dev.close()
    host.close()


def test_batch_with_per_adunit_member():
    pop, P, lk, hr = tiny_world(adunit_grid=3)
    a = sim.Simulation(pop, P, lk, hr)
    b = a.replica()
    policies = [_unit_policy(), sim.InterventionPolicy(threshold=3, window=7, duration=12.0)]
    batch = sim.Batch([a, b])
    got = batch.run([31, 32], DAYS, n_seed=20, policy=policies)
    snaps = [snapshot(m.backend, pop) for m in (a, b)]
    batch.close()
    for k, seed in enumerate([31, 32]):
        m = sim.Simulation(pop, P, lk, hr)
        want = m.run(seed, DAYS, n_seed=20, policy=policies[k], device_loop=False)
        _same_series(got[k], want, "member %d" % k)
        _same_state(snapshot(m.backend, pop), snaps[k], "member %d" % k)
        m.close()
    a.close()
    b.close()


def test_batch_blocks_match_lone_runs():
    """A batch's counter blocks (t = 0 and every day's end), member by member, equal
    lone runs' blocks under the host loop; the summary table averages them."""
    from covidsim_b200 import output
    pop, P, lk, hr = tiny_world()
    a = sim.Simulation(pop, P, lk, hr)
    b = a.replica()
    batch = sim.Batch([a, b])
    _, got = batch.run([41, 42], 20, n_seed=20, policy=_policy(), blocks=True)
    batch.close()
    for k, seed in enumerate([41, 42]):
        m = sim.Simulation(pop, P, lk, hr)
        _, want = m.run(seed, 20, n_seed=20, policy=_policy(), device_loop=False, blocks=True)
        assert np.array_equal(got[k], want), "member %d" % k
        m.close()
    a.close()
    b.close()
