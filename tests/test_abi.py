"""The C-ABI library: loads without a GPU, exports every symbol the header
declares, and its structures match the Python mirror."""
import ast
import ctypes as C
import os
import subprocess
import sys

import numpy as np
import pytest

from covidsim_b200 import abi


def test_library_loads_and_sizes_match():
    lib = abi.load_library()
    assert lib.cs_abi_version() == abi.CS_ABI_VERSION
    assert lib.cs_sizeof_params() == C.sizeof(abi.cs_params)
    assert lib.cs_sizeof_population() == C.sizeof(abi.cs_population)
    assert lib.cs_sizeof_counters() == C.sizeof(abi.cs_counters)


def test_exports_every_declared_symbol():
    abi.load_library()
    out = subprocess.run(["nm", "-D", "--defined-only", abi.LIB_PATH], capture_output=True, text=True, check=True).stdout
    exported = {line.split()[-1] for line in out.splitlines() if line.strip()}
    declared = abi.exported_symbols()
    assert len(declared) >= 25
    missing = [s for s in declared if s not in exported]
    assert not missing, missing


@pytest.mark.gpu
def test_library_runs_sm100_machine_code():
    """The CUDA runtime loads the sweep kernels as sm_100 machine code (not PTX
    compiled at load time for another architecture)."""
    lib = abi.load_library()
    b, p = C.c_int(), C.c_int()
    assert lib.cs_kernel_arch(C.byref(b), C.byref(p)) == 0
    assert b.value == 100, b.value


def test_kernel_table_host_functions():
    lib = abi.load_library()
    n = 100000
    lk, hr = np.empty(n + 1), np.empty(n + 1)
    d = C.c_double()
    rc = lib.cs_build_kernel_table(5, 4000.0, 3.0, 0.0, 0.0, 1e10, n, n // 1600, lk.ctypes.data, hr.ctypes.data, C.byref(d))
    assert rc == 0 and d.value == 1e10 / n
    assert lk[0] == 1.0
    # power_b kernel: 1 / (1 + (d/scale)^shape)
    r2 = 3000.0 ** 2
    v = lib.cs_kernel_num(lk.ctypes.data, hr.ctypes.data, n, n // 1600, d.value, r2)
    assert abs(v - 1.0 / (1.0 + (3000.0 / 4000.0) ** 3)) < 1e-6
    assert np.isnan(lib.cs_kernel_num(lk.ctypes.data, hr.ctypes.data, n, n // 1600, d.value, 2e10))
    assert lib.cs_build_kernel_table(9, 4000.0, 3.0, 0.0, 0.0, 1e10, n, 10, lk.ctypes.data, hr.ctypes.data, C.byref(d)) == abi.CS_E_ARG


_NO_DEVICE_CHILD = r'''
import ctypes as C
from covidsim_b200 import abi, sim
from tests.helpers import tiny_world
lib = abi.load_library()
assert lib.cs_kernel_arch(C.byref(C.c_int()), None) == abi.CONST["CS_E_CUDA"]
pop, P, lk, hr = tiny_world()
try:
    sim.Simulation(pop, P, lk, hr)
except abi.CovidSimError as e:
    assert "cs_gpu_create" in str(e), str(e)
    print("failed cleanly")
'''


def test_create_without_gpu_fails_cleanly():
    """With no device visible, the create call and the architecture query return
    error codes and a message instead of crashing.  Runs in a child process with
    CUDA_VISIBLE_DEVICES empty, so it tests the same path on a GPU machine."""
    root = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
    env = dict(os.environ, CUDA_VISIBLE_DEVICES="",
               PYTHONPATH=os.pathsep.join([root, os.path.join(root, "covid-sim_b200"), os.environ.get("PYTHONPATH", "")]))
    r = subprocess.run([sys.executable, "-c", _NO_DEVICE_CHILD], env=env, cwd=root, capture_output=True, text=True,
                       timeout=300)
    assert r.returncode == 0 and "failed cleanly" in r.stdout, r.stdout + r.stderr[-2000:]


def test_product_does_not_import_oracle():
    """No module of the package imports anything from the oracle, calls its C
    entry points or loads its library."""
    pkg = os.path.join(os.path.dirname(abi.__file__))
    for f in sorted(os.listdir(pkg)):
        if not f.endswith(".py"):
            continue
        src = open(os.path.join(pkg, f)).read()
        for node in ast.walk(ast.parse(src)):
            if isinstance(node, ast.Import):
                names = [a.name for a in node.names]
            elif isinstance(node, ast.ImportFrom):
                names = [node.module or ""]
            else:
                continue
            assert not any(n.split(".")[0].startswith("oracle") for n in names), (f, names)
        assert "cs_cpu_" not in src and "libcs_oracle" not in src, f
