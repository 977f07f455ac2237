"""Place closures and microcell status handed over by a host's own TreatSweep
(cs_gpu_place_events, cs_gpu_set_mcell_status).

The CPU tests pin the oracle's member loops to a direct restatement of the
reference's DoPlaceClose (src/Update.cpp:1196-1240, DoAnyway = 1), UpdateHostClosure
(src/Update.cpp:1243-1258) and DoPlaceOpen (src/Update.cpp:1260-1294), written
here over the downloaded state.  The GPU test holds the library to the oracle, state
for state, while events and microcell status changes arrive between steps."""
import numpy as np
import pytest

from covidsim_b200 import abi, sim
import oracle_py
from tests.helpers import tiny_world, snapshot, STATE_FIELDS


def _world(attending):
    pop, P, lk, hr = tiny_world()
    P2 = type(P).from_buffer_copy(P)
    for t, a in enumerate(attending):
        P2.PlaceClosePropAttending[t] = a
    P2.CaseAbsentChildPropAdultCarers = 0.6
    return pop, P2, lk, hr


def _advance(sims, P, k0, k1, policy_at=None):
    for k in range(k0, k1):
        t = k * P.ModelTimeStep
        if policy_at is not None and k == policy_at:
            for s in sims:   # case isolation and household quarantine, so some people are quarantined
                s._switch_interventions(t, sim.InterventionPolicy(duration=60.0, close_place_types=()), True,
                                        np.zeros(s.pop.n_mcells, dtype=np.uint8))
        for s in sims:
            s.backend.step(t, 0)


def _events(pop, rng, ts, kind, frac, types, members=None, window=None):
    out = []
    for pt in types:
        n = len(pop.places[pt]["mcell"])
        for l in np.nonzero(rng.random(n) < frac)[0]:
            e = abi.cs_place_event()
            e.place, e.place_type, e.kind, e.ts = int(l), pt, kind, ts
            if kind == abi.CS_PLACE_EV_CLOSE:
                e.members = int(rng.random() < 0.8) if members is None else members
                e.win_start, e.win_stop = window
                e.close_start, e.close_end = (window if e.members else (window[1], window[1]))
            elif kind == abi.CS_PLACE_EV_HOLIDAY:
                e.win_start, e.win_stop = window
            out.append(e)
    return out


class _Ref:
    """The reference's member loops over a state snapshot (TEST RESTATEMENT)."""

    def __init__(self, pop, P, snap):
        self.pop, self.P, self.s = pop, P, snap
        self.close_end = {}

    def quarantined(self, x, ts):
        s = self.s
        comply = (int(s["flags"][x]) & 0x0C) >> 2
        return comply == 1 and int(s["quar_start_time"][x]) + self.P.usHQuarantineHouseDuration > ts and \
            s["quar_start_time"][x] <= ts

    def absent(self, x, ts):
        return self.s["absent_start_time"][x] <= ts and self.s["absent_stop_time"][x] > ts

    def alive(self, x):
        return abs(int(self.s["inf"][x])) != 5

    def household(self, x):
        h = self.pop.person_hh[x]
        return range(self.pop.hh_first[h], self.pop.hh_first[h] + self.pop.hh_nh[h])

    def adult_home(self, x, ts):
        P, wp = self.P, self.P.PlaceTypeNoAirNum - 1
        return any(self.alive(j) and self.pop.person_age[j] >= P.CaseAbsentChildAgeCutoff and
                   (self.pop.person_place[wp][j] < 0 or self.quarantined(j, ts)) for j in self.household(x))

    def members(self, pt, l):
        pl = self.pop.places[pt]
        return pl["members"][pl["member_ofs"][l]:pl["member_ofs"][l + 1]]

    def close(self, e, queue):
        P, s = self.P, self.s
        self.close_end[(e.place_type, e.place)] = e.close_end
        if not e.members:
            return
        att = P.PlaceClosePropAttending[e.place_type]
        for w in self.members(e.place_type, e.place):
            if not (att == 0 or s["ProbAbsent"][w] >= att):
                continue
            if (not self.absent(w, e.ts)) and (not self.quarantined(w, e.ts)) and \
                    self.pop.person_age[w] < P.CaseAbsentChildAgeCutoff:
                if s["ProbCare"][w] < P.CaseAbsentChildPropAdultCarers and not self.adult_home(w, e.ts):
                    for j in self.household(w):
                        if self.pop.person_age[j] >= P.CaseAbsentChildAgeCutoff and self.alive(j):
                            queue.append((j, e.win_start, e.win_stop))
                            break
            s["absent_start_time"][w] = min(s["absent_start_time"][w], e.win_start)
            s["absent_stop_time"][w] = max(s["absent_stop_time"][w], e.win_stop)

    def open(self, e):
        P, s = self.P, self.s
        ce = self.close_end.get((e.place_type, e.place), 0)
        if not e.ts < ce:
            return
        for ai in self.members(e.place_type, e.place):
            if s["absent_stop_time"][ai] == ce:
                s["absent_stop_time"][ai] = e.ts
            if s["ProbCare"][ai] < P.CaseAbsentChildPropAdultCarers:
                if self.pop.person_age[ai] < P.CaseAbsentChildAgeCutoff and not self.quarantined(ai, e.ts):
                    if not self.adult_home(ai, e.ts):
                        for l in self.household(ai):
                            if self.pop.person_age[l] >= P.CaseAbsentChildAgeCutoff and self.alive(l) and \
                                    self.absent(l, e.ts) and s["absent_stop_time"][l] == ce:
                                s["absent_stop_time"][l] = e.ts
        self.close_end[(e.place_type, e.place)] = e.ts

    def holiday(self, e):
        """IncubRecoverySweep's holiday loop for one chosen place (src/Sweep.cpp:
        904-913): the place's window and every member's absence widen."""
        s = self.s
        self.close_end[(e.place_type, e.place)] = max(self.close_end.get((e.place_type, e.place), 0), e.win_stop)
        for w in self.members(e.place_type, e.place):
            if s["absent_start_time"][w] > e.win_start:
                s["absent_start_time"][w] = e.win_start
            if s["absent_stop_time"][w] < e.win_stop:
                s["absent_stop_time"][w] = e.win_stop

    def apply(self, events):
        rank = {abi.CS_PLACE_EV_OPEN: 0, abi.CS_PLACE_EV_CLOSE: 1}
        order = sorted(range(len(events)), key=lambda i: (rank.get(events[i].kind, 2), events[i].place_type, i))
        queue = []
        for i in order:
            e = events[i]
            if e.kind == abi.CS_PLACE_EV_OPEN:
                self.open(e)
            elif e.kind == abi.CS_PLACE_EV_CLOSE:
                self.close(e, queue)
        for j, a, b in queue:   # UpdateHostClosure
            self.s["absent_start_time"][j] = min(self.s["absent_start_time"][j], a)
            self.s["absent_stop_time"][j] = max(self.s["absent_stop_time"][j], b)
        for i in order:
            if events[i].kind == abi.CS_PLACE_EV_HOLIDAY:
                self.holiday(events[i])
        return len(queue)


def test_oracle_place_events_follow_reference():
    pop, P, lk, hr = _world((0.0, 0.5, 0.0, 0.0))
    o = sim.Simulation(pop, P, lk, hr, backend=oracle_py.OracleBackend)
    o.backend.begin_run(77, o.choose_seeds(77, 40))
    _advance([o], P, 0, 130, policy_at=60)
    rng = np.random.default_rng(5)
    ts = 130
    closes = _events(pop, rng, ts, abi.CS_PLACE_EV_CLOSE, 0.5, (0, 1, 2), window=(ts, ts + 200))
    ref = _Ref(pop, P, snapshot(o.backend, pop))
    assert any(ref.quarantined(x, ts) for x in range(pop.n_people)), "no quarantined people: weak test"
    n_carers = ref.apply(closes)
    assert n_carers > 0, "no child needed a carer: weak test"
    o.backend.place_events(closes)
    got = snapshot(o.backend, pop)
    for k in ("absent_start_time", "absent_stop_time"):
        assert np.array_equal(got[k], ref.s[k]), k
    # openings later in the closure, and closures of other places, in one call
    ts2 = ts + 40
    opens = [e for e in closes if e.members and rng.random() < 0.6]
    opens = [abi.cs_place_event(place=e.place, place_type=e.place_type, kind=abi.CS_PLACE_EV_OPEN, ts=ts2) for e in opens]
    more = _events(pop, rng, ts2, abi.CS_PLACE_EV_CLOSE, 0.2, (3,), members=1, window=(ts2, ts2 + 120))
    batch = more + opens      # opens are applied first whatever the order given
    ref.s = snapshot(o.backend, pop)
    ref.apply(batch)
    o.backend.place_events(batch)
    got = snapshot(o.backend, pop)
    for k in ("absent_start_time", "absent_stop_time"):
        assert np.array_equal(got[k], ref.s[k]), k
    assert np.any(got["absent_stop_time"] == ts2), "no absence ended with an opening: weak test"
    o.close()


def test_oracle_close_places_follows_reference():
    """cs_cpu_close_places (the Python host's and device run loop's closure) runs the
    same member loop at its start time, carers included."""
    pop, P, lk, hr = _world((0.0, 0.0, 0.3, 0.0))
    o = sim.Simulation(pop, P, lk, hr, backend=oracle_py.OracleBackend)
    o.backend.begin_run(78, o.choose_seeds(78, 40))
    _advance([o], P, 0, 120, policy_at=50)
    ts, stop = 120, 300
    ref = _Ref(pop, P, snapshot(o.backend, pop))
    o.backend.close_places(0, None, ts, stop)
    got = snapshot(o.backend, pop)
    # which places closed depends on their ProbClose, which the state view does not
    # carry: every place of type 0 closes when its efficacy is 0
    assert P.Efficacies[abi.CS_NPI_PLACE_CLOSURE][0] == 0
    closes = [abi.cs_place_event(place=l, place_type=0, kind=abi.CS_PLACE_EV_CLOSE, members=1, ts=ts,
                                 close_start=ts, close_end=stop, win_start=ts, win_stop=stop)
              for l in range(len(pop.places[0]["mcell"]))]
    assert ref.apply(closes) > 0
    for k in ("absent_start_time", "absent_stop_time"):
        assert np.array_equal(got[k], ref.s[k]), k
    o.close()


def test_oracle_holidays_follow_reference():
    """Holiday closures (CS_PLACE_EV_HOLIDAY) against the reference's holiday loop
    restated over the state, mixed with closures in one call (holidays after the
    closures' carers)."""
    pop, P, lk, hr = _world((0.0, 0.0, 0.0, 0.0))
    o = sim.Simulation(pop, P, lk, hr, backend=oracle_py.OracleBackend)
    o.backend.begin_run(79, o.choose_seeds(79, 40))
    _advance([o], P, 0, 100, policy_at=40)
    rng = np.random.default_rng(8)
    ts = 100
    hol = _events(pop, rng, ts, abi.CS_PLACE_EV_HOLIDAY, 0.7, (0, 1, 2, 3), window=(ts + 1, ts + 57))
    closes = _events(pop, rng, ts, abi.CS_PLACE_EV_CLOSE, 0.3, (0, 1), window=(ts, ts + 120))
    ref = _Ref(pop, P, snapshot(o.backend, pop))
    ref.apply(hol + closes)
    o.backend.place_events(hol + closes)
    got = snapshot(o.backend, pop)
    for k in ("absent_start_time", "absent_stop_time"):
        assert np.array_equal(got[k], ref.s[k]), k
    assert np.sum(got["absent_start_time"] == ts + 1) > 1000, "few members on holiday: weak test"
    o.close()


@pytest.mark.gpu
def test_gpu_place_events_match_oracle():
    pop, P, lk, hr = _world((0.0, 0.5, 0.0, 0.0))
    g = sim.Simulation(pop, P, lk, hr)
    o = sim.Simulation(pop, P, lk, hr, backend=oracle_py.OracleBackend)
    seeds = g.choose_seeds(91, 40)
    for s in (g, o):
        s.backend.begin_run(91, seeds)
    _advance([g, o], P, 0, 100, policy_at=40)
    rng = np.random.default_rng(9)
    nm = pop.n_mcells
    done = 100
    for round_, (ts_close, ts_open) in enumerate(((100, None), (150, 150), (200, 230))):
        _advance([g, o], P, done, ts_close)
        done = ts_close
        ev = _events(pop, rng, ts_close, abi.CS_PLACE_EV_CLOSE, 0.3, (0, 1, 2, 3), window=(ts_close, ts_close + 160))
        if round_ == 1:   # holidays among the closures and openings
            ev += _events(pop, rng, ts_close, abi.CS_PLACE_EV_HOLIDAY, 0.5, (0, 1, 3), window=(ts_close + 1, ts_close + 41))
        if ts_open is not None:
            ev += [abi.cs_place_event(place=int(l), place_type=pt, kind=abi.CS_PLACE_EV_OPEN, ts=ts_open)
                   for pt in (0, 1) for l in np.nonzero(rng.random(len(pop.places[pt]["mcell"])) < 0.3)[0]]
        m = np.nonzero(rng.random(nm) < 0.25)[0].astype(np.int32)
        sd = rng.integers(0, 4, len(m)).astype(np.uint8)
        mr = rng.integers(0, 3, len(m)).astype(np.uint8)
        for s in (g, o):
            s.backend.place_events(ev)
            s.backend.set_mcell_status(m, sd, mr if round_ else None)
        a, b = snapshot(g.backend, pop), snapshot(o.backend, pop)
        for k in STATE_FIELDS:
            assert np.array_equal(a[k], b[k]), "after events %d: %s" % (round_, k)
    _advance([g, o], P, done, done + 80)
    a, b = snapshot(g.backend, pop), snapshot(o.backend, pop)
    for k in STATE_FIELDS:
        assert np.array_equal(a[k], b[k]), "after the steps: %s" % k
    ca, cb = abi.counters_to_dict(g.backend.counters()), abi.counters_to_dict(o.backend.counters())
    assert ca == cb
    assert ca["cumI"] > 500
    g.close()
    o.close()
