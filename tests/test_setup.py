"""Population set-up on the GPU (cs_gpu_setup_run) against its sequential
restatement in the oracle (cs_cpu_setup_run): integer membership (households,
microcells, cells, places, groups, member lists) and the float locations are
compared array for array (bit-exact).  The set-up's own structure is checked on
its own: every person in one household of one microcell, cells and microcells in
the reference's order (src/SetupModel.cpp:1163-1185), households within their
microcell, place links and member lists that agree, groups that partition each
place; and its distributions against the host generator's (the same rules)."""
import numpy as np
import pytest

from covidsim_b200 import population


def _grid(width, cell_deg, nmcl):
    return population.make_grid(width_deg=width, height_deg=width, cell_deg=cell_deg, nmcl=nmcl)


WORLDS = {
    "tiny": (20000, dict(width=0.2, cell_deg=1.0 / 120, nmcl=10), dict()),
    "blobs_adunits": (60000, dict(width=0.5, cell_deg=1.0 / 60, nmcl=4),
                      dict(sigma=1.5, blobs=5, blob_share=0.4, adunit_grid=3)),
    "sparse": (4000, dict(width=0.2, cell_deg=1.0 / 120, nmcl=2), dict(sigma=2.0, seed=77)),
}


def check_structure(pop):
    """Invariants of a set-up's output (any backend)."""
    N = pop.n_people
    g = pop.grid
    th = g["nch"] * g["nmcl"]
    # households: consecutive people, sizes >= 1, one microcell each
    assert pop.hh_first[0] == 0
    assert np.array_equal(pop.hh_first[1:], pop.hh_first[:-1] + pop.hh_nh[:-1].astype(np.int64))
    assert int(pop.hh_first[-1]) + int(pop.hh_nh[-1]) == N
    assert pop.hh_nh.min() >= 1 and pop.hh_nh.max() <= 10
    assert np.array_equal(pop.person_hh, np.repeat(np.arange(pop.n_households, dtype=np.int32), pop.hh_nh))
    mc_of_hh = pop.person_mcell[pop.hh_first]
    assert np.array_equal(pop.person_mcell, np.repeat(mc_of_hh, pop.hh_nh))
    # household locations inside their microcell
    mcw, mch = g["cell_width"] / g["nmcl"], g["cell_height"] / g["nmcl"]
    j = pop.mcell_grid[mc_of_hh]
    fx = pop.hh_x.astype(np.float64) / mcw - (j // th)
    fy = pop.hh_y.astype(np.float64) / mch - (j % th)
    assert fx.min() > -1e-4 and fx.max() < 1 + 1e-4 and fy.min() > -1e-4 and fy.max() < 1 + 1e-4
    # cells: populated, grid order; microcells grouped by cell, x-major within it
    assert np.all(np.diff(pop.cell_grid) > 0)
    assert pop.cell_start[0] == 0 and pop.cell_start[-1] == N and np.all(np.diff(pop.cell_start) > 0)
    nch, nmcl = g["nch"], g["nmcl"]
    mx, my = pop.mcell_grid // th, pop.mcell_grid % th
    cell_of_mc = (mx // nmcl) * nch + (my // nmcl)
    assert np.array_equal(pop.cell_grid[pop.mcell_cell], cell_of_mc)
    key = pop.mcell_cell.astype(np.int64) * (nmcl * nmcl) + (mx % nmcl) * nmcl + (my % nmcl)
    assert np.all(np.diff(key) > 0)
    # people numbered cell by cell, microcell by microcell
    assert np.all(np.diff(pop.person_mcell) >= 0)
    cell_of_person = pop.mcell_cell[pop.person_mcell]
    assert np.array_equal(np.searchsorted(pop.cell_start, np.arange(N), side="right") - 1, cell_of_person)
    # places: one place per person at most; member lists agree with the links
    anyplace = np.zeros(N, dtype=np.int32)
    for t, pl in enumerate(pop.places):
        links = pop.person_place[t]
        npl = len(pl["mcell"])
        assert links.max() < npl
        att = np.nonzero(links >= 0)[0]
        anyplace[att] += 1
        counts = np.bincount(links[att], minlength=npl)
        assert np.array_equal(np.diff(pl["member_ofs"]), counts)
        assert np.array_equal(np.sort(pl["members"]), att)
        assert np.array_equal(links[pl["members"]], np.repeat(np.arange(npl), counts))
        # groups partition each place, members know their group
        ng = np.diff(pl["group_ofs"])
        assert ng.min() >= 1
        gp = np.repeat(np.arange(npl), ng)
        assert np.array_equal(np.bincount(gp, weights=pl["group_size"], minlength=npl).astype(np.int64), counts)
        pos = np.arange(len(pl["members"])) - pl["member_ofs"][links[pl["members"]]]
        grp = pop.person_group[t][pl["members"]]
        gfirst = pl["group_ofs"][links[pl["members"]]] + grp
        assert np.all(pos >= pl["group_start"][gfirst])
        assert np.all(pos < pl["group_start"][gfirst] + pl["group_size"][gfirst])
        # places lie in their microcell
        jp = pop.mcell_grid[pl["mcell"]]
        px = pl["x"].astype(np.float64) / mcw - (jp // th)
        assert px.min() > -1e-4 and px.max() < 1 + 1e-4
    assert anyplace.max() <= 1


def test_oracle_setup_structure():
    import oracle_py
    for name, (n, gk, kw) in WORLDS.items():
        pop = oracle_py.setup_population(n, _grid(**gk), **kw)
        assert pop.n_people == n, name
        check_structure(pop)
        if kw.get("adunit_grid"):
            assert pop.n_adunits == kw["adunit_grid"] ** 2
            assert set(np.unique(pop.mcell_adunit)) <= set(range(pop.n_adunits))


def _reference_household_rule(counts, hh_dist, seed=3):
    """Household sizes by the reference's loop (src/SetupModel.cpp:1224-1253), in
    plain Python on the given microcell populations: a size from the cumulative
    distribution, cut at the microcell's remaining people and at 10."""
    rng = np.random.default_rng(seed)
    cdf = np.cumsum(hh_dist) / np.sum(hh_dist)
    hist = np.zeros(11, dtype=np.int64)
    for n in counts:
        k = 0
        while k < n:
            u = rng.random()
            m = 1
            while u > cdf[m - 1] and k + m < n and m < 10:
                m += 1
            hist[m] += 1
            k += m
    return hist


def test_oracle_setup_distributions_follow_the_reference_rules():
    """Households by the reference's rule; microcell occupancy, ages, attendance and
    place sizes as the host generator draws them (the same rules, other streams):
    1M people on the 240 x 240 grid of the 1M workload."""
    import oracle_py
    grid = population.make_grid(cell_deg=1.0 / 120, nmcl=10)
    a = oracle_py.setup_population(1_000_000, grid)
    b = population.generate(1_000_000, grid)
    # household sizes: the set-up's against the reference's loop on the same microcells
    ref = _reference_household_rule(np.bincount(a.person_mcell), population.HH_SIZE_DIST)
    ha = np.bincount(a.hh_nh, minlength=11)[1:] / a.n_households
    hr = ref[1:] / ref.sum()
    assert abs(a.n_households - ref.sum()) / ref.sum() < 0.005, (a.n_households, ref.sum())
    assert np.abs(ha - hr).max() < 0.003, (ha, hr)
    # people per populated microcell, populated cells
    assert abs(a.n_mcells - b.n_mcells) / b.n_mcells < 0.01
    assert abs(a.n_cells - b.n_cells) / b.n_cells < 0.01
    # ages by band
    aa = np.bincount(a.person_age // 5, minlength=17) / a.n_people
    ab = np.bincount(b.person_age // 5, minlength=17) / b.n_people
    assert np.abs(aa - ab).max() < 0.003
    for t in range(4):
        na, nb = (a.person_place[t] >= 0).sum(), (b.person_place[t] >= 0).sum()
        assert abs(na - nb) / nb < 0.02, (t, na, nb)
        sa = np.diff(a.places[t]["member_ofs"])
        sb = np.diff(b.places[t]["member_ofs"])
        # realised place sizes: means within 15% (capacity rounds leave places a
        # little under their drawn size; slack 1.125)
        assert abs(sa.mean() - sb.mean()) / sb.mean() < 0.15, (t, sa.mean(), sb.mean())
    # the nearest-place choice keeps places local: the median home-to-place distance
    # is within the radius holding the `nearest` places a person chooses among
    # (sqrt(nearest) x the places' typical spacing), and shorter than the host
    # generator's Z-order runs give
    G = grid["ncw"] * grid["nch"]

    def median_cells(pop, t):
        pl = pop.places[t]
        h = pop.person_hh[pl["members"]]
        p = np.repeat(np.arange(len(pl["mcell"])), np.diff(pl["member_ofs"]))
        return np.median(np.hypot(pop.hh_x[h] - pl["x"][p], pop.hh_y[h] - pl["y"][p])) / grid["cell_width"]
    for t in range(4):
        reach = np.sqrt(population.PLACE_NEAREST[t] * G / len(a.places[t]["mcell"]))
        assert median_cells(a, t) < reach, (t, median_cells(a, t), reach)
        assert median_cells(a, t) < median_cells(b, t), t


@pytest.mark.gpu
@pytest.mark.parametrize("name", sorted(WORLDS))
def test_gpu_setup_matches_oracle(name):
    import oracle_py
    n, gk, kw = WORLDS[name]
    grid = _grid(**gk)
    g = population.generate_on_device(n, grid, **kw)
    o = oracle_py.setup_population(n, grid, **kw)
    for k in population._ARRAYS:
        assert np.array_equal(getattr(g, k), getattr(o, k)), "%s: %s differs" % (name, k)
    for t, (pg, po) in enumerate(zip(g.places, o.places)):
        for k in population._PLACE_ARRAYS:
            assert np.array_equal(pg[k], po[k]), "%s: place type %d %s differs" % (name, t, k)
    assert g.setup_info["forced"] == o.setup_info["forced"]
    check_structure(g)


@pytest.mark.gpu
def test_gpu_setup_at_one_million_matches_oracle_and_runs():
    """The 1M-person workload's geography set up on the GPU equals the oracle's, and
    a realisation steps on it (the set-up's output is a valid sweep input)."""
    import oracle_py
    from covidsim_b200 import params as prm, sim
    grid = population.make_grid(cell_deg=1.0 / 120, nmcl=10)
    g = population.generate_on_device(1_000_000, grid)
    o = oracle_py.setup_population(1_000_000, grid)
    for k in population._ARRAYS:
        assert np.array_equal(getattr(g, k), getattr(o, k)), k
    for pg, po in zip(g.places, o.places):
        for k in population._PLACE_ARRAYS:
            assert np.array_equal(pg[k], po[k]), k
    P, lk, hr = prm.build_params(g.grid)
    P.LocalBeta, _ = sim.calibrate_local_beta(g, P, 2.4)
    s = sim.Simulation(g, P, lk, hr, device=0)
    ser = s.run(seed=11, days=30, n_seed=100)
    s.close()
    assert ser["cumI"][-1] > 1000
