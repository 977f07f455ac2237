"""Population files: the .npz cache of a generated population, and the reference's
network file of person-to-place links (src/SetupModel.cpp:2603-2690)."""
import numpy as np
import pytest

from covidsim_b200 import population


def _same(a, b):
    for k in population._ARRAYS:
        assert np.array_equal(getattr(a, k), getattr(b, k)), k
    assert a.n_people == b.n_people and a.n_adunits == b.n_adunits
    assert len(a.places) == len(b.places)
    for pa, pb in zip(a.places, b.places):
        for k in population._PLACE_ARRAYS:
            assert np.array_equal(pa[k], pb[k]), k
    for k in a.grid:
        assert np.array_equal(np.asarray(a.grid[k]), np.asarray(b.grid[k])), k


def test_save_and_load_round_trip(tmp_path):
    pop = population.preset("tiny", n_people=5000, adunit_grid=2)
    path = tmp_path / "pop.npz"
    population.save(pop, path)
    back = population.load(path)
    _same(pop, back)
    assert (back.n_households, back.n_cells, back.n_mcells) == (pop.n_households, pop.n_cells, pop.n_mcells)


def test_network_file_layout_and_round_trip(tmp_path):
    pop = population.preset("tiny", n_people=3000)
    path = tmp_path / "net.bin"
    population.save_network_file(pop, path, 98798150, 729101)
    raw = np.fromfile(path, dtype="<i4")
    npt = len(pop.places)
    assert list(raw[:5]) == [population.NETWORK_FILE_VERSION, npt, pop.n_people, 98798150, 729101]
    assert raw.size == 5 + npt * pop.n_people
    # person-major: person i's links follow one another
    links = np.asarray(pop.person_place).reshape(npt, pop.n_people)
    assert np.array_equal(raw[5:5 + npt], links[:, 0])
    n_places = [len(pl["mcell"]) for pl in pop.places]
    back = population.load_network_file(path, pop.n_people, n_places, 98798150, 729101)
    assert np.array_equal(back, links)


def test_network_file_checks(tmp_path):
    pop = population.preset("tiny", n_people=2000)
    path = tmp_path / "net.bin"
    population.save_network_file(pop, path, 1, 2)
    n_places = [len(pl["mcell"]) for pl in pop.places]
    with pytest.raises(ValueError, match="seeds"):
        population.load_network_file(path, pop.n_people, n_places, 1, 3)
    with pytest.raises(ValueError, match="population size"):
        population.load_network_file(path, pop.n_people + 1, n_places, 1, 2)
    with pytest.raises(ValueError, match="place types"):
        population.load_network_file(path, pop.n_people, n_places[:-1], 1, 2)
    with pytest.raises(ValueError, match="out of bounds"):
        population.load_network_file(path, pop.n_people, [1] * len(n_places), 1, 2)
    raw = np.fromfile(path, dtype="<i4")
    raw[0] = 7
    raw.tofile(path)
    with pytest.raises(ValueError, match="incompatible"):
        population.load_network_file(path, pop.n_people, n_places, 1, 2)


def test_cache_generates_once(tmp_path):
    calls = []

    def make():
        calls.append(1)
        return population.preset("tiny", n_people=1500)
    a = population.cached(str(tmp_path), "tiny1500", make)
    b = population.cached(str(tmp_path), "tiny1500", make)
    assert len(calls) == 1
    _same(a, b)
    assert population.cached(None, "x", make) is not None and len(calls) == 2


def test_network_file_read_by_the_reference(tmp_path):
    """A network file written here is read link for link by the reference's own
    LoadPeopleToPlaces (src/SetupModel.cpp:2603-2659).  The reference's command line
    refuses /L with /S, so the network tool's loader mode runs the reference's
    set-up with LoadPeopleToPlaces on our file in place of the place assignment and
    /S writes back what it loaded (SavePeopleToPlaces); the two files are the same
    bytes.  The file written here carries a network the reference did not make
    (links exchanged among the attendees of each place type), so the match cannot
    come from the reference re-deriving its own.  The stock reference then runs a
    realisation on our file with /L."""
    import os
    import refrun
    if not (os.path.exists(refrun.NETGEN) and os.path.exists(refrun.STOCK)):
        pytest.skip("reference executables not built (needs the reference checkout at build time)")
    grid = population.make_grid(width_deg=0.2, height_deg=0.2, cell_deg=1.0 / 120, nmcl=10)
    pop = population.generate(5000, grid, sigma=1.2, seed=98798150)
    seeds = (98798150, 729101)
    theirs = str(tmp_path / "reference.net")
    refrun.run_reference(pop, 1, nr=1, threads=2, binary=refrun.NETGEN, extra_args=("/S:" + theirs,), timeout=600)
    raw = np.fromfile(theirs, dtype="<i4")
    npt, n = int(raw[1]), int(raw[2])
    assert (raw[0], n, raw[3], raw[4]) == (population.NETWORK_FILE_VERSION, pop.n_people) + seeds
    n_places = [int(raw[5 + t::npt].max()) + 1 for t in range(npt)]
    links = population.load_network_file(theirs, n, n_places, *seeds)
    assert np.array_equal(np.ascontiguousarray(links.T).ravel(), raw[5:])
    # exchange links among each type's attendees (every link stays a valid place)
    rng = np.random.default_rng(5)
    mine = links.copy()
    for t in range(npt):
        att = np.nonzero(mine[t] >= 0)[0]
        mine[t, att] = mine[t, rng.permutation(att)]
    assert not np.array_equal(mine, links)
    ours = str(tmp_path / "ours.net")
    population.save_network_links(mine, n_places, ours, *seeds)
    back = str(tmp_path / "back.net")
    refrun.run_reference(pop, 1, nr=1, threads=2, binary=refrun.NETGEN, extra_args=("/S:" + back,), timeout=600,
                         env={"CS_NETGEN_LOAD": ours})
    assert open(back, "rb").read() == open(ours, "rb").read()
    refrun.run_reference(pop, 1, nr=1, threads=2, binary=refrun.STOCK, extra_args=("/L:" + ours,), timeout=600)
