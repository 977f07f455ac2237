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
