"""ctypes view of include/covidsim_b200.h.

The structure layouts are read from the header itself at import time, so the
Python mirror cannot drift from the C declarations; the loaded library's
cs_sizeof_* exports are checked against them before any call.
"""
import ctypes as C
import os
import re

_HERE = os.path.dirname(os.path.abspath(__file__))
PKG_ROOT = os.path.dirname(_HERE)
REPO_ROOT = os.path.dirname(PKG_ROOT)
HEADER = os.path.join(REPO_ROOT, "include", "covidsim_b200.h")
LIB_PATH = os.path.join(PKG_ROOT, "lib", "libcovidsim_b200.so")

_SCALARS = {
    "double": C.c_double, "float": C.c_float, "int32_t": C.c_int32, "int64_t": C.c_int64,
    "uint16_t": C.c_uint16, "uint8_t": C.c_uint8, "int8_t": C.c_int8, "int16_t": C.c_int16,
    "uint32_t": C.c_uint32, "uint64_t": C.c_uint64, "int": C.c_int, "size_t": C.c_size_t,
}


def _read_header():
    with open(HEADER) as f:
        text = f.read()
    text = re.sub(r"/\*.*?\*/", "", text, flags=re.S)
    text = re.sub(r"//[^\n]*", "", text)
    return text


def _defines(text):
    out = {}
    for m in re.finditer(r"^\s*#define\s+(CS_\w+)\s+(.+?)\s*$", text, flags=re.M):
        out[m.group(1)] = m.group(2)
    vals = {}

    def ev(name, depth=0):
        if name in vals:
            return vals[name]
        expr = out[name]
        expr = re.sub(r"\b(CS_\w+)\b", lambda mm: str(ev(mm.group(1), depth + 1)), expr)
        expr = expr.replace("u", "") if re.fullmatch(r"[0-9xXa-fA-F]+u", expr.strip()) else expr
        try:
            vals[name] = int(eval(expr, {"__builtins__": {}}))
        except Exception:
            vals[name] = None
        return vals[name]

    for k in out:
        ev(k)
    return {k: v for k, v in vals.items() if v is not None}


_TEXT = _read_header()
CONST = _defines(_TEXT)
globals().update(CONST)

STRUCTS = {}


def _dim(expr):
    expr = re.sub(r"\b(CS_\w+)\b", lambda m: str(CONST[m.group(1)]), expr)
    return int(eval(expr, {"__builtins__": {}}))


def _build_struct(name, body):
    fields = []
    for stmt in body.split(";"):
        stmt = " ".join(stmt.split())
        if not stmt:
            continue
        m = re.match(r"^(const\s+)?(\w+)\s*(\*?)\s*(.*)$", stmt)
        base, star, rest = m.group(2), m.group(3), m.group(4)
        if base in _SCALARS:
            ctype = _SCALARS[base]
        else:
            ctype = STRUCTS[base]
        for decl in rest.split(","):
            decl = decl.strip()
            ptr = star == "*"
            if decl.startswith("*"):
                ptr, decl = True, decl[1:].strip()
            dm = re.match(r"^(\w+)((?:\[[^\]]+\])*)$", decl)
            fname, dims = dm.group(1), re.findall(r"\[([^\]]+)\]", dm.group(2))
            t = C.c_void_p if ptr else ctype
            for dexpr in reversed(dims):
                t = t * _dim(dexpr)
            fields.append((fname, t))
    return type(name, (C.Structure,), {"_fields_": fields})


for _m in re.finditer(r"typedef\s+struct\s+(\w+)\s*\{(.*?)\}\s*(\w+)\s*;", _TEXT, flags=re.S):
    STRUCTS[_m.group(3)] = _build_struct(_m.group(3), _m.group(2))

cs_icdf = STRUCTS["cs_icdf"]
cs_params = STRUCTS["cs_params"]
cs_population = STRUCTS["cs_population"]
cs_state_view = STRUCTS["cs_state_view"]
cs_interventions = STRUCTS["cs_interventions"]
cs_counters = STRUCTS["cs_counters"]
cs_run_policy = STRUCTS["cs_run_policy"]
cs_place_event = STRUCTS["cs_place_event"]
cs_setup_spec = STRUCTS["cs_setup_spec"]
cs_setup_out = STRUCTS["cs_setup_out"]

COUNTER_FIELDS = [f for f, _ in cs_counters._fields_]

_lib = None


class CovidSimError(RuntimeError):
    pass


def load_library(path=LIB_PATH):
    """Load the sm_100a library, (re)building it first when it is missing or older
    than its sources."""
    global _lib
    if _lib is not None:
        return _lib
    if path == LIB_PATH:
        import importlib.util
        spec = importlib.util.spec_from_file_location("_cs_build", os.path.join(PKG_ROOT, "build.py"))
        mod = importlib.util.module_from_spec(spec)
        spec.loader.exec_module(mod)
        mod.build()
    lib = C.CDLL(path)
    P, I, D, V = C.POINTER, C.c_int, C.c_double, C.c_void_p
    sig = {
        "cs_abi_version": (I, []),
        "cs_sizeof_params": (C.c_size_t, []),
        "cs_sizeof_population": (C.c_size_t, []),
        "cs_sizeof_counters": (C.c_size_t, []),
        "cs_sizeof_interventions": (C.c_size_t, []),
        "cs_sizeof_run_policy": (C.c_size_t, []),
        "cs_kernel_arch": (I, [P(I), P(I)]),
        "cs_build_kernel_table": (I, [I, D, D, D, D, D, I, I, V, V, P(D)]),
        "cs_kernel_num": (D, [V, V, I, I, D, D]),
        "cs_gpu_create": (I, [P(cs_population), P(cs_params), I, P(V)]),
        "cs_gpu_destroy": (None, [V]),
        "cs_gpu_last_error": (C.c_char_p, [V]),
        "cs_gpu_set_params": (I, [V, P(cs_params)]),
        "cs_gpu_begin_run": (I, [V, C.c_uint64, V, I, I]),
        "cs_gpu_upload_state": (I, [V, C.c_uint64, P(cs_state_view)]),
        "cs_gpu_upload_people": (I, [V, P(cs_state_view), C.c_int64, C.c_int64]),
        "cs_gpu_download_state": (I, [V, P(cs_state_view)]),
        "cs_gpu_seed_infections": (I, [V, D, V, I]),
        "cs_gpu_infect_sweep": (I, [V, D, I]),
        "cs_gpu_incub_recovery_sweep": (I, [V, D]),
        "cs_gpu_update_probs": (I, [V, I]),
        "cs_gpu_update_probs_static": (I, [V, I]),
        "cs_gpu_step": (I, [V, D, I]),
        "cs_gpu_use_graphs": (I, [V, I]),
        "cs_gpu_set_grid": (I, [V, I]),
        "cs_gpu_grid": (I, [V]),
        "cs_gpu_set_spatial_lanes": (I, [V, I]),
        "cs_gpu_create_replica": (I, [V, P(V)]),
        "cs_gpu_batch_create": (I, [P(V), I, P(V)]),
        "cs_gpu_batch_step": (I, [V, D, I]),
        "cs_gpu_batch_set_grid": (I, [V, I]),
        "cs_gpu_batch_set_spatial_lanes": (I, [V, I]),
        "cs_gpu_batch_sync": (I, [V]),
        "cs_gpu_batch_stream": (V, [V]),
        "cs_gpu_batch_last_error": (C.c_char_p, [V]),
        "cs_gpu_batch_destroy": (None, [V]),
        "cs_sur_num_params": (C.c_size_t, []),
        "cs_sur_create": (I, [I, I, P(V)]),
        "cs_sur_destroy": (None, [V]),
        "cs_sur_last_error": (C.c_char_p, [V]),
        "cs_sur_set_params": (I, [V, V]),
        "cs_sur_get_params": (I, [V, V]),
        "cs_sur_forward": (I, [V, V, I, V]),
        "cs_sur_loss_grad": (I, [V, V, V, I, P(C.c_float), V]),
        "cs_sur_train_step": (I, [V, V, V, I, C.c_float, C.c_float, P(C.c_float)]),
        "cs_sur_set_gemm": (I, [V, I]),
        "cs_gpu_set_interventions": (I, [V, P(cs_interventions)]),
        "cs_gpu_close_places": (I, [V, I, V, I, C.c_uint16, C.c_uint16]),
        "cs_gpu_place_events": (I, [V, V, I]),
        "cs_gpu_set_mcell_status": (I, [V, V, V, V, I]),
        "cs_gpu_get_counters": (I, [V, P(cs_counters)]),
        "cs_gpu_run": (I, [V, I, P(cs_run_policy), V]),
        "cs_gpu_batch_run": (I, [V, I, V, V]),
        "cs_gpu_get_cell_counts": (I, [V, V, V, V, V, V]),
        "cs_gpu_get_sample": (I, [V, V, V, V, V, V, P(cs_counters)]),
        "cs_gpu_get_sample16": (I, [V, V, P(cs_counters)]),
        "cs_gpu_sample_packed_bytes": (C.c_size_t, [V]),
        "cs_gpu_get_sample_packed": (I, [V, V, C.c_size_t]),
        "cs_gpu_sample_packed_begin": (I, [V, V, C.c_size_t]),
        "cs_gpu_sample_packed_end": (I, [V, V]),
        "cs_host_alloc": (V, [C.c_size_t]),
        "cs_host_free": (None, [V]),
        "cs_gpu_sync": (I, [V]),
        "cs_gpu_stream": (V, [V]),
        "cs_gpu_launch_count": (C.c_int64, [V]),
        "cs_gpu_profile": (I, [V, I]),
        "cs_gpu_profile_entry": (I, [V, I, C.c_char_p, I, P(D), P(C.c_int64)]),
        "cs_sizeof_setup_spec": (C.c_size_t, []),
        "cs_sizeof_setup_out": (C.c_size_t, []),
        "cs_gpu_setup_run": (I, [P(cs_setup_spec), P(cs_params), I, P(V)]),
        "cs_gpu_setup_sizes": (I, [V, P(cs_setup_out)]),
        "cs_gpu_setup_download": (I, [V, P(cs_setup_out)]),
        "cs_gpu_setup_last_error": (C.c_char_p, [V]),
        "cs_gpu_setup_destroy": (None, [V]),
    }
    for name, (res, args) in sig.items():
        fn = getattr(lib, name)
        fn.restype, fn.argtypes = res, args
    if lib.cs_abi_version() != CONST["CS_ABI_VERSION"]:
        raise CovidSimError("library ABI version %d, header %d" % (lib.cs_abi_version(), CONST["CS_ABI_VERSION"]))
    for fn, st in (("cs_sizeof_params", cs_params), ("cs_sizeof_population", cs_population),
                   ("cs_sizeof_counters", cs_counters), ("cs_sizeof_interventions", cs_interventions),
                   ("cs_sizeof_run_policy", cs_run_policy), ("cs_sizeof_setup_spec", cs_setup_spec),
                   ("cs_sizeof_setup_out", cs_setup_out)):
        if getattr(lib, fn)() != C.sizeof(st):
            raise CovidSimError("%s: library %d bytes, Python mirror %d" % (fn, getattr(lib, fn)(), C.sizeof(st)))
    _lib = lib
    return lib


def exported_symbols(header=HEADER):
    """Every function the header declares (used to check the library's exports)."""
    return sorted(set(re.findall(r"^\s*[\w\s\*]+?\b(cs_\w+)\s*\(", _TEXT, flags=re.M)))


def counters_to_dict(c):
    out = {}
    for name, t in cs_counters._fields_:
        v = getattr(c, name)
        out[name] = list(v) if hasattr(v, "__len__") else int(v)
    return out
