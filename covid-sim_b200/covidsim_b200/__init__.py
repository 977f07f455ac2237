"""Host side of the B200 sweep of CovidSim: bindings, parameters, synthetic
populations and the run loop.  The compute path is the sm_100a library
lib/libcovidsim_b200.so behind the C ABI of include/covidsim_b200.h; nothing in
this package computes a sweep on the CPU.
"""
from . import abi  # noqa: F401
from .abi import CovidSimError, load_library  # noqa: F401
