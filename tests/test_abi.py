"""The C-ABI library: loads without a GPU, exports every symbol the header
declares, and its structures match the Python mirror."""
import ctypes as C
import os
import subprocess

import numpy as np

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


def test_library_is_sm100a_only():
    out = subprocess.run(["/usr/local/cuda/bin/cuobjdump", "--list-elf", abi.LIB_PATH], capture_output=True, text=True)
    if out.returncode != 0:
        return  # tool unavailable: nothing to check
    assert "sm_100a" in out.stdout


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


def test_create_without_gpu_fails_cleanly():
    """With no device the create call returns an error code and a message."""
    import torch
    if torch.cuda.is_available():
        return
    from tests.helpers import tiny_world
    from covidsim_b200 import sim
    pop, P, lk, hr = tiny_world()
    try:
        sim.Simulation(pop, P, lk, hr)
    except abi.CovidSimError as e:
        assert "cs_gpu_create" in str(e)
    else:
        raise AssertionError("expected a CUDA error without a device")


def test_product_does_not_import_oracle():
    pkg = os.path.join(os.path.dirname(abi.__file__))
    for f in os.listdir(pkg):
        if f.endswith(".py"):
            src = open(os.path.join(pkg, f)).read()
            assert "oracle" not in src.replace("oracle/", "").split("import")[0] or "import oracle" not in src
            assert "import oracle_py" not in src and "cs_cpu_" not in src
