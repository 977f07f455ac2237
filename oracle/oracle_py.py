"""ctypes binding of the CPU oracle (oracle/cs_oracle.c).  TEST INFRASTRUCTURE ONLY:
imported by tests/, the smoke check and bench.py's CPU-baseline leg, never by the
product package.  OracleBackend mirrors covidsim_b200.sim.GpuBackend method for
method, so a Simulation can run on either and the two can be compared."""
import ctypes as C
import os
import subprocess

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
LIB = os.path.join(HERE, "_build", "libcs_oracle.so")


def build():
    subprocess.run(["make", "-s", "-C", HERE, "oracle"], check=True)
    return LIB


_lib = None


def load():
    global _lib
    if _lib is not None:
        return _lib
    src = os.path.join(HERE, "cs_oracle.c")
    if not os.path.exists(LIB) or os.path.getmtime(LIB) < os.path.getmtime(src):
        build()
    from covidsim_b200 import abi
    lib = C.CDLL(LIB)
    P, I, D, V = C.POINTER, C.c_int, C.c_double, C.c_void_p
    sig = {
        "cs_cpu_create": (I, [P(abi.cs_population), P(abi.cs_params), P(V)]),
        "cs_cpu_destroy": (None, [V]),
        "cs_cpu_last_error": (C.c_char_p, [V]),
        "cs_cpu_set_params": (I, [V, P(abi.cs_params)]),
        "cs_cpu_begin_run": (I, [V, C.c_uint64, V, I, I]),
        "cs_cpu_seed_infections": (I, [V, D, V, I]),
        "cs_cpu_infect_sweep": (I, [V, D, I]),
        "cs_cpu_incub_recovery_sweep": (I, [V, D]),
        "cs_cpu_update_probs": (I, [V, I]),
        "cs_cpu_step": (I, [V, D, I]),
        "cs_cpu_set_interventions": (I, [V, P(abi.cs_interventions)]),
        "cs_cpu_close_places": (I, [V, I, V, I, C.c_uint16, C.c_uint16]),
        "cs_cpu_place_events": (I, [V, V, I]),
        "cs_cpu_set_mcell_status": (I, [V, V, V, V, I]),
        "cs_cpu_download_state": (I, [V, P(abi.cs_state_view)]),
        "cs_cpu_get_counters": (I, [V, P(abi.cs_counters)]),
        "cs_cpu_kernel_num": (D, [V, D]),
        "cs_cpu_kernel_num_f32": (D, [V, V, I, I, D, D]),
        "cs_cpu_block_bound": (D, [V, I, I]),
        "cs_cpu_block_geometry": (None, [V, V]),
        "cs_cpu_dist2_raw": (D, [P(abi.cs_params), D, D, D, D]),
        "cs_cpu_dist2_cc_min": (D, [P(abi.cs_params), I, I]),
        "cs_cpu_icdf_choose": (C.c_uint16, [P(abi.cs_icdf), D, D, D]),
        "cs_cpu_philox": (None, [C.c_uint32, C.c_uint32, P(C.c_uint32), P(C.c_uint32)]),
        "cs_cpu_build_kernel_table": (I, [I, D, D, D, D, D, I, I, V, V, P(D)]),
        "cs_cpu_upload_state": (I, [V, C.c_uint64, P(abi.cs_state_view)]),
        "cs_cpu_calc": (D, [V, I, I, I, I, I]),
        "cs_cpu_setup_run": (I, [P(abi.cs_setup_spec), P(abi.cs_params), P(V)]),
        "cs_cpu_setup_sizes": (I, [V, P(abi.cs_setup_out)]),
        "cs_cpu_setup_download": (I, [V, P(abi.cs_setup_out)]),
        "cs_cpu_setup_last_error": (C.c_char_p, [V]),
        "cs_cpu_setup_destroy": (None, [V]),
        "cs_cpu_sample_many": (I, [I, C.c_uint64, D, D, I, V]),
    }
    for name, (res, args) in sig.items():
        fn = getattr(lib, name)
        fn.restype, fn.argtypes = res, args
    _lib = lib
    return lib


class OracleBackend:
    prefix = "cs_cpu_"

    def __init__(self, pop_c, params, device=0):
        from covidsim_b200 import abi
        self.abi = abi
        self.lib = load()
        self.ctx = C.c_void_p()
        rc = self.lib.cs_cpu_create(C.byref(pop_c), C.byref(params), C.byref(self.ctx))
        if rc != 0:
            raise abi.CovidSimError("cs_cpu_create: %s" % self.lib.cs_cpu_last_error(self.ctx).decode())

    def _ck(self, rc, what):
        if rc != 0:
            raise self.abi.CovidSimError("cs_cpu_%s: %s" % (what, self.lib.cs_cpu_last_error(self.ctx).decode()))

    def close(self):
        if self.ctx:
            self.lib.cs_cpu_destroy(self.ctx)
            self.ctx = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    def begin_run(self, seed, seeds):
        s = np.ascontiguousarray(seeds, dtype=np.int32)
        self._ck(self.lib.cs_cpu_begin_run(self.ctx, seed, s.ctypes.data, len(s), 0), "begin_run")

    def seed_infections(self, t, people):
        s = np.ascontiguousarray(people, dtype=np.int32)
        self._ck(self.lib.cs_cpu_seed_infections(self.ctx, t, s.ctypes.data, len(s)), "seed_infections")

    def infect_sweep(self, t, run=0):
        self._ck(self.lib.cs_cpu_infect_sweep(self.ctx, t, run), "infect_sweep")

    def incub_recovery_sweep(self, t):
        self._ck(self.lib.cs_cpu_incub_recovery_sweep(self.ctx, t), "incub_recovery_sweep")

    def step(self, t, run=0):
        self._ck(self.lib.cs_cpu_step(self.ctx, t, run), "step")

    def update_probs(self, do_place=0):
        self._ck(self.lib.cs_cpu_update_probs(self.ctx, do_place), "update_probs")

    def set_params(self, params):
        self._ck(self.lib.cs_cpu_set_params(self.ctx, C.byref(params)), "set_params")

    def set_interventions(self, iv):
        self._ck(self.lib.cs_cpu_set_interventions(self.ctx, C.byref(iv)), "set_interventions")

    def close_places(self, place_type, mcells, start, stop):
        if mcells is None:
            self._ck(self.lib.cs_cpu_close_places(self.ctx, place_type, None, 0, start, stop), "close_places")
        else:
            m = np.ascontiguousarray(mcells, dtype=np.int32)
            self._ck(self.lib.cs_cpu_close_places(self.ctx, place_type, m.ctypes.data, len(m), start, stop), "close_places")

    def place_events(self, events):
        ev = (self.abi.cs_place_event * len(events))(*events)
        self._ck(self.lib.cs_cpu_place_events(self.ctx, ev, len(events)), "place_events")

    def set_mcell_status(self, mcells, socdist=None, moverest=None):
        m = np.ascontiguousarray(mcells, dtype=np.int32)
        sd = None if socdist is None else np.ascontiguousarray(socdist, dtype=np.uint8)
        mr = None if moverest is None else np.ascontiguousarray(moverest, dtype=np.uint8)
        self._ck(self.lib.cs_cpu_set_mcell_status(self.ctx, m.ctypes.data, None if sd is None else sd.ctypes.data,
                                                  None if mr is None else mr.ctypes.data, len(m)), "set_mcell_status")

    def counters(self):
        out = self.abi.cs_counters()
        self._ck(self.lib.cs_cpu_get_counters(self.ctx, C.byref(out)), "get_counters")
        return out

    def download(self, view):
        self._ck(self.lib.cs_cpu_download_state(self.ctx, C.byref(view)), "download_state")

    def sync(self):
        pass

    def upload(self, seed, view):
        self._ck(self.lib.cs_cpu_upload_state(self.ctx, seed, C.byref(view)), "upload_state")

    def calc(self, kind, p, q, pt, ts):
        return self.lib.cs_cpu_calc(self.ctx, kind, p, q, pt, ts)

    def kernel_num(self, r2):
        return self.lib.cs_cpu_kernel_num(self.ctx, r2)


def setup_population(n_people, grid, **kw):
    """The oracle's restatement of the set-up kernels (cs_cpu_setup_run) on the spec
    covidsim_b200.population.generate_on_device builds: a Population to compare
    with the GPU's array for array."""
    from covidsim_b200 import abi, population
    lib = load()
    S, P, keep = population.setup_spec(n_people, grid, **kw)
    h = C.c_void_p()
    rc = lib.cs_cpu_setup_run(C.byref(S), C.byref(P), C.byref(h))
    try:
        if rc != 0:
            raise RuntimeError("cs_cpu_setup_run: %s" % lib.cs_cpu_setup_last_error(h).decode())
        sizes = abi.cs_setup_out()
        lib.cs_cpu_setup_sizes(h, C.byref(sizes))
        pop = population.from_setup(sizes, lambda out: lib.cs_cpu_setup_download(h, C.byref(out)), grid)
    finally:
        lib.cs_cpu_setup_destroy(h)
    del keep
    return pop
