"""cs_gpu_update_probs_static (UpdateProbs on the library's fixed scratch array)
against cs_gpu_update_probs, through the C ABI.

The two must agree bit for bit (tolerance: exact equality) on every per-person
field, cell list and cell value, call after call, including when the fixed array
still holds another population's values from the call before."""
import ctypes as C

import numpy as np
import pytest

from covidsim_b200 import abi, population, params as prm, sim
from tests.helpers import tiny_world, snapshot, STATE_FIELDS

pytestmark = pytest.mark.gpu


def _static(be, do_place=0):
    rc = be.lib.cs_gpu_update_probs_static(be.ctx, do_place)
    assert rc == abi.CONST["CS_OK"], be.lib.cs_gpu_last_error(be.ctx).decode()


def _same(a, b, where):
    for k in STATE_FIELDS:
        assert np.array_equal(a[k], b[k]), "%s: %s differs at %d entries" % (where, k, int(np.sum(a[k] != b[k])))


def _advance(sims, P, k0, k1):
    for k in range(k0, k1):
        for s in sims:
            s.backend.step(k * P.ModelTimeStep, 0)


def _sparse_world():
    """4,000 people on 24 x 24 cells: many grid positions hold no populated cell."""
    grid = population.make_grid(width_deg=0.2, height_deg=0.2, cell_deg=1.0 / 120, nmcl=2)
    pop = population.generate(4000, grid, sigma=2.0, seed=77)
    P, lk, hr = prm.build_params(pop.grid, kernel_size=200000)
    P.LocalBeta, _ = sim.calibrate_local_beta(pop, P, 2.4)
    return pop, P, lk, hr


def test_static_matches_update_probs_call_after_call():
    pop, P, lk, hr = _sparse_world()
    # Another population on the same device fills the fixed array first.  Grid
    # positions it populates and this world leaves empty hold its stale values,
    # which the call must clear.
    other = tiny_world()
    stale = set(other[0].cell_grid.tolist()) - set(pop.cell_grid.tolist())
    assert stale, "the check needs grid positions populated only in the first world"
    so = sim.Simulation(*other)
    so.backend.begin_run(3, so.choose_seeds(3, 30))
    _static(so.backend)          # first call on the device: set-up, before any capture
    _advance([so], other[1], 0, 30)
    _static(so.backend)

    ref = sim.Simulation(pop, P, lk, hr)
    var = sim.Simulation(pop, P, lk, hr)
    seed = 2024
    seeds = ref.choose_seeds(seed, 40)
    for s in (ref, var):
        s.backend.begin_run(seed, seeds)
    done = 0
    for call, steps in enumerate((32, 24)):
        _advance([ref, var], P, done, done + steps)
        done += steps
        ref.backend.update_probs(0)
        _static(var.backend)
        a, b = snapshot(ref.backend, pop), snapshot(var.backend, pop)
        assert not np.all(a["cell_tot_prob"] == 1.0), "epidemic too small to move tot_prob"
        _same(a, b, "call %d" % (call + 1))
    # the sweeps that follow read the recomputed values the same way
    _advance([ref, var], P, done, done + 8)
    _same(snapshot(ref.backend, pop), snapshot(var.backend, pop), "after the calls")
    for s in (ref, var, so):
        s.backend.close()


def test_static_rejects_grids_above_its_limit():
    limit = abi.CONST["CS_STATIC_MAX_GRID_CELLS"]
    side = 4 * int(np.ceil((limit ** 0.5 + 8) / 4))    # side * side > limit
    grid = population.make_grid(width_deg=2.0, height_deg=2.0, cell_deg=2.0 / side, nmcl=1)
    assert grid["ncw"] * grid["nch"] > limit
    pop = population.generate(2000, grid, seed=5)
    P, lk, hr = prm.build_params(pop.grid)
    s = sim.Simulation(pop, P, lk, hr)
    s.backend.begin_run(1, s.choose_seeds(1, 5))
    rc = s.backend.lib.cs_gpu_update_probs_static(s.backend.ctx, 0)
    assert rc == abi.CONST["CS_E_RANGE"]
    assert b"exceed its fixed scratch" in s.backend.lib.cs_gpu_last_error(s.backend.ctx)
    # the context stays usable through the allocating entry point
    s.backend.update_probs(0)
    s.backend.close()
