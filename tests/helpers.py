"""Shared fixtures of the tests: small seeded populations and parameter blocks."""
import functools

import numpy as np

from covidsim_b200 import population, params as prm, sim


@functools.lru_cache(maxsize=None)
def tiny_world(n_people=20000, seed=98798150, kernel_size=200000, r0=2.4, utm=1, adunit_grid=None):
    pop = population.preset("tiny", n_people=n_people, seed=seed, adunit_grid=adunit_grid)
    P, lk, hr = prm.build_params(pop.grid, kernel_size=kernel_size)
    P.DoUTM_coords = utm
    if not utm:
        P, lk, hr = _planar(pop, P, kernel_size)
    beta, _ = sim.calibrate_local_beta(pop, P, r0)
    P.LocalBeta = beta
    return pop, P, lk, hr


def _planar(pop, P, kernel_size):
    P2, lk, hr = prm.build_params(pop.grid, kernel_size=kernel_size, kernel=(5, 0.04, 3.0, 0.0, 0.0))
    P2.DoUTM_coords = 0
    import ctypes as C
    from covidsim_b200 import abi
    lib = abi.load_library()
    d = C.c_double()
    lib.cs_build_kernel_table(5, 0.04, 3.0, 0.0, 0.0, prm.longest_distance2(P2), kernel_size,
                              P2.kernel_expansion, lk.ctypes.data, hr.ctypes.data, C.byref(d))
    P2.kernel_delta = d.value
    return P2, lk, hr


STATE_FIELDS = ("inf", "severity", "flags", "infection_time", "latent_time", "recovery_or_death_time",
                "SARI_time", "Critical_time", "Stepdown_time", "absent_start_time", "absent_stop_time",
                "isolation_start_time", "quar_start_time", "detected_time", "infectiousness", "susc",
                "ProbAbsent", "ProbCare", "infector", "infect_type", "listpos", "cell_slots", "cell_S",
                "cell_L", "cell_I", "cell_R", "cell_D", "cell_S0", "cell_tot_prob")


def snapshot(backend, pop):
    arrs, view = sim.state_arrays(pop.n_people, pop.n_cells)
    backend.download(view)
    return {k: arrs[k].copy() for k in STATE_FIELDS}


def check_lists(snap, pop):
    """Cell-list invariants the reference maintains (src/Update.cpp:1402-1579)."""
    slots, listpos, inf = snap["cell_slots"], snap["listpos"], snap["inf"]
    cs = pop.cell_start
    for c in range(pop.n_cells):
        b0, b1 = cs[c], cs[c + 1]
        seg = slots[b0:b1]
        assert sorted(seg.tolist()) == sorted(pop.cell_members[b0:b1].tolist())
        assert np.all(listpos[seg] == np.arange(b1 - b0))
        S, L, I = snap["cell_S"][c], snap["cell_L"][c], snap["cell_I"][c]
        st = inf[seg]
        assert np.all(st[:S] == 0)
        assert np.all(st[S:S + L] == 1)
        assert np.all(np.isin(st[S + L:S + L + I], (-1, 2, -2)))
        assert np.all(np.isin(st[S + L + I:], (3, -3, 5, -5)))
