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


def _bound_dominates(world, n_pairs=60000, seed=3):
    """For household pairs in every kind of block pair (same, adjacent, far), the
    tabulated proposal bound of their blocks is at least the FP32 kernel value at
    their distance: the acceptance probability K(d)/bound of the spatial pass never
    exceeds 1, so the rejection sampler draws exactly in proportion to K(d)."""
    import ctypes as C
    pop, P, lk, hr = world
    s = sim.Simulation(pop, P, lk, hr, backend=oracle_py.OracleBackend)
    lib = oracle_py.load()
    geo = np.zeros(4, np.int32)
    lib.cs_cpu_block_geometry(s.backend.ctx, geo.ctypes.data)
    bs, nbx, nby, tab = (int(v) for v in geo)
    assert tab == 1
    lk32, hr32 = lk.astype(np.float32), hr.astype(np.float32)
    cx = np.floor(pop.hh_x / P.cell_width).astype(np.int64)
    cy = np.floor(pop.hh_y / P.cell_height).astype(np.int64)
    blk = (cx // bs) * nby + (cy // bs)
    rng = np.random.default_rng(seed)
    a = rng.integers(0, len(blk), n_pairs)
    # half the partners from the same or a neighbouring block, where the bound is tight
    near = np.nonzero(rng.random(n_pairs) < 0.5)[0]
    b = rng.integers(0, len(blk), n_pairs)
    order = np.argsort(blk, kind="stable")
    first = np.searchsorted(blk[order], np.arange(nbx * nby))
    last = np.searchsorted(blk[order], np.arange(nbx * nby), side="right")
    worst = 0.0
    for k in near:
        bx, by = divmod(int(blk[a[k]]), nby)
        tx = min(max(bx + int(rng.integers(-1, 2)), 0), nbx - 1)
        ty = min(max(by + int(rng.integers(-1, 2)), 0), nby - 1)
        t = tx * nby + ty
        if last[t] > first[t]:
            b[k] = order[rng.integers(first[t], last[t])]
    for i, j in zip(a, b):
        d2 = lib.cs_cpu_dist2_raw(C.byref(P), float(pop.hh_x[i]), float(pop.hh_y[i]), float(pop.hh_x[j]),
                                  float(pop.hh_y[j]))
        kf = lib.cs_cpu_kernel_num_f32(lk32.ctypes.data, hr32.ctypes.data, P.kernel_size, P.kernel_expansion,
                                       P.kernel_delta, d2)
        bound = lib.cs_cpu_block_bound(s.backend.ctx, int(blk[i]), int(blk[j]))
        worst = max(worst, kf / bound)
    s.close()
    assert 0.5 < worst <= 1.0, worst


def test_spatial_bound_dominates_kernel_utm():
    _bound_dominates(tiny_world())


def test_spatial_bound_dominates_kernel_planar():
    _bound_dominates(tiny_world(utm=0))


def test_infection_radii_follow_their_definition():
    """The oracle's radius counters against the definition restated here: every
    infection but a seed's adds (int)(r^2 * 2^32), r the distance in degrees from
    its household to the last seed's (src/Update.cpp:116-127, src/CovidSim.cpp:
    1358-1359), and the largest r^2 is kept."""
    pop, P, lk, hr = tiny_world()
    s, be, out = _run(21, 120)
    snap = snapshot(be, pop)
    seeds = s.choose_seeds(21, 20)
    o = np.array([pop.hh_x[pop.person_hh[seeds[-1]]], pop.hh_y[pop.person_hh[seeds[-1]]]], np.float64)
    inf = np.nonzero((snap["inf"] != 0) & (snap["infector"] != -2))[0]
    h = pop.person_hh[inf]
    r2 = (pop.hh_x[h].astype(np.float64) - o[0]) ** 2 + (pop.hh_y[h].astype(np.float64) - o[1]) ** 2
    c = be.counters()
    assert len(inf) > 300
    assert c.sumRad2_q == int(np.sum((r2 * 4294967296.0).astype(np.int64)))
    assert np.array([c.maxRad2_bits], np.int64).view(np.float64)[0] == r2.max()


def test_blanket_movement_restrictions_cut_long_contacts():
    """Blanket movement restrictions (src/Sweep.cpp:300-301): with the effect 0 and a
    radius of a few hundred metres, contacts beyond the radius cannot infect while
    the restriction lasts, so the epidemic grows more slowly than without it and
    the infections in the window stay near their infectors."""
    pop, P, lk, hr = tiny_world()
    Q = type(P).from_buffer_copy(P)
    Q.DoBlanketMoveRestr = 1
    Q.MoveRestrTimeStart, Q.MoveRestrDuration = 10.0, 20.0
    Q.MoveRestrRadius2 = 500.0 ** 2          # dist2 is in square metres
    Q.MoveRestrEffect = 0.0
    _, be0, a = _run(31, 120, world=(pop, P, lk, hr))
    _, be1, b = _run(31, 120, world=(pop, Q, lk, hr))
    assert a[39] == b[39]                    # identical until the restriction starts
    assert b[-1][5] < 0.8 * a[-1][5]         # fewer infections by day 30


def test_false_positives_are_counted_and_detected():
    """False positives (src/Sweep.cpp:2046, src/Update.cpp:896-905): a fraction of
    the entries that would infect become false cases instead, every one counted in
    cumFC and, with ControlPropCasesId 1, detected (cumDC) and so isolated when case
    isolation is on; the infections fall by about that fraction."""
    pop, P, lk, hr = tiny_world()
    Q = type(P).from_buffer_copy(P)
    Q.FalsePositiveRate = 0.3
    Q.ControlPropCasesId = 1.0
    _, be0, a = _run(41, 80, world=(pop, P, lk, hr))
    _, be1, b = _run(41, 80, world=(pop, Q, lk, hr))
    c0, c1 = be0.counters(), be1.counters()
    assert c0.cumFC == 0 and c1.cumFC > 100
    assert c1.cumDC >= c1.cumFC            # every false case detected, besides the real ones
    # the transmission rate is scaled by 1 / (1 - rate) (src/Sweep.cpp:295), so the
    # infections per generation stay about the same
    assert 0.5 * c0.cumI < c1.cumI < 2.0 * c0.cumI
