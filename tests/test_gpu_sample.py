"""The three ways a host reads what RecordSample needs agree with each other and with
the oracle: cs_gpu_get_sample (32-bit cell counts), cs_gpu_get_sample16 (16-bit) and
cs_gpu_get_sample_packed (the counter block and the 16-bit counts in one buffer,
S..D of the block left 0, also in two halves queued behind a timestep), into
page-locked memory from cs_host_alloc."""
import ctypes as C

import numpy as np
import pytest

from covidsim_b200 import abi, sim
import oracle_py
from tests.helpers import tiny_world, snapshot

pytestmark = pytest.mark.gpu


def test_sample_copies_agree_with_each_other_and_the_oracle():
    pop, P, lk, hr = tiny_world()
    g = sim.Simulation(pop, P, lk, hr)
    o = sim.Simulation(pop, P, lk, hr, backend=oracle_py.OracleBackend)
    seeds = g.choose_seeds(5, 20)
    g.backend.begin_run(5, seeds)
    o.backend.begin_run(5, seeds)
    for k in range(60):
        t = k * P.ModelTimeStep
        for s in (g, o):
            s.backend.infect_sweep(t, 0)
            s.backend.incub_recovery_sweep(t)
    be = g.backend
    lib, ctx = be.lib, be.ctx
    nc = pop.n_cells
    cells32 = np.zeros(5 * nc, np.int32)
    k32 = abi.cs_counters()
    p = cells32.ctypes.data
    assert lib.cs_gpu_get_sample(ctx, p, p + 4 * nc, p + 8 * nc, p + 12 * nc, p + 16 * nc, C.byref(k32)) == 0
    cells16 = np.zeros(5 * nc, np.uint16)
    k16 = abi.cs_counters()
    assert lib.cs_gpu_get_sample16(ctx, cells16.ctypes.data, C.byref(k16)) == 0
    nbytes = lib.cs_gpu_sample_packed_bytes(ctx)
    assert nbytes == C.sizeof(abi.cs_counters) + 2 * 5 * nc
    buf = lib.cs_host_alloc(nbytes)
    assert buf
    try:
        assert lib.cs_gpu_get_sample_packed(ctx, buf, nbytes - 1) != 0   # too small a buffer is refused
        assert lib.cs_gpu_get_sample_packed(ctx, buf, nbytes) == 0
        raw = np.ctypeslib.as_array(C.cast(buf, C.POINTER(C.c_uint8)), shape=(nbytes,)).copy()
        # the two halves, queued behind a timestep: the same bytes as the timestep's
        # own copy afterwards
        C.memset(buf, 0, nbytes)
        t = 60 * P.ModelTimeStep
        be.infect_sweep(t, 0)
        be.incub_recovery_sweep(t)
        assert lib.cs_gpu_sample_packed_begin(ctx, buf, nbytes) == 0
        assert lib.cs_gpu_sample_packed_end(ctx, buf) == 0
        queued = np.ctypeslib.as_array(C.cast(buf, C.POINTER(C.c_uint8)), shape=(nbytes,)).copy()
        assert lib.cs_gpu_get_sample_packed(ctx, buf, nbytes) == 0
        after = np.ctypeslib.as_array(C.cast(buf, C.POINTER(C.c_uint8)), shape=(nbytes,)).copy()
        assert np.array_equal(queued, after)
    finally:
        lib.cs_host_free(buf)
    kp = abi.cs_counters.from_buffer_copy(raw[:C.sizeof(abi.cs_counters)].tobytes())
    cellsp = raw[C.sizeof(abi.cs_counters):].view(np.uint16)
    assert np.array_equal(cells16.astype(np.int32), cells32)
    assert np.array_equal(cellsp, cells16)
    a, b, c = abi.counters_to_dict(k32), abi.counters_to_dict(k16), abi.counters_to_dict(kp)
    for key in a:
        assert a[key] == b[key], key
        if key in ("S", "L", "I", "R", "D"):
            assert c[key] == 0, key
        else:
            assert a[key] == c[key], key
    # the counts are the oracle's
    snap = snapshot(o.backend, pop)
    for j, key in enumerate(("cell_S", "cell_L", "cell_I", "cell_R", "cell_D")):
        assert np.array_equal(cells32[j * nc:(j + 1) * nc], snap[key]), key
    assert a["cumI"] == abi.counters_to_dict(o.backend.counters())["cumI"]
    assert a["cumI"] > 100


def test_state_uploaded_in_slices_equals_whole_upload():
    """cs_gpu_upload_people: the per-person arrays sent ahead in three slices, then
    cs_gpu_upload_state, give the context the same state as one whole upload, and the
    run goes on identically; a slice that does not follow the last one is refused."""
    from covidsim_b200 import sim as simmod
    pop, P, lk, hr = tiny_world()
    g = sim.Simulation(pop, P, lk, hr)
    seeds = g.choose_seeds(9, 20)
    g.backend.begin_run(9, seeds)
    for k in range(40):
        t = k * P.ModelTimeStep
        g.backend.infect_sweep(t, 0)
        g.backend.incub_recovery_sweep(t)
    arrs, view = simmod.state_arrays(pop.n_people, pop.n_cells)
    g.backend.download(view)
    results = []
    lib, ctx = g.backend.lib, g.backend.ctx
    for sliced in (False, True):
        if sliced:
            n = pop.n_people
            cuts = [0, n // 3, (2 * n) // 3, n]
            assert lib.cs_gpu_upload_people(ctx, C.byref(view), 5, 10) != 0   # not from person 0
            for a, b in zip(cuts[:-1], cuts[1:]):
                assert lib.cs_gpu_upload_people(ctx, C.byref(view), a, b - a) == 0
        g.backend.upload(77, view)
        for k in range(40, 60):
            t = k * P.ModelTimeStep
            g.backend.infect_sweep(t, 0)
            g.backend.incub_recovery_sweep(t)
        results.append((snapshot(g.backend, pop), abi.counters_to_dict(g.backend.counters())))
    (a, ca), (b, cb) = results
    for key in a:
        assert np.array_equal(a[key], b[key]), key
    assert ca == cb
