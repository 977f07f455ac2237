"""The oracle's leaf arithmetic against golden vectors produced by the reference's
own functions (tests/golden/make_ref_pins.py -> tests/golden/ref_pins.json):
kernel lookup (Kernels.cpp:108-129), great-circle distances (Dist.cpp:23-144),
inverse CDF draws (InverseCdf.cpp:60-74), the infectiousness and susceptibility
products (CalcInfSusc.cpp) -- all bit-exact -- and the random-variate samplers
(Rand.cpp ignpoi_mt / ignbin_mt / gen_gamma_mt) by distribution."""
import ctypes as C
import json
import math
import os

import numpy as np
import pytest

from covidsim_b200 import abi, params as prm, population, sim
import oracle_py

GOLD = json.load(open(os.path.join(os.path.dirname(__file__), "golden", "ref_pins.json")))


def _utm_params(bbox_y, cell, n):
    p = abi.cs_params()
    p.DoUTM_coords = 1
    p.bbox_bottom_left_y = bbox_y
    p.cell_width = p.cell_height = cell
    p.ncw = p.nch = n
    p.width_deg = p.height_deg = n * cell
    sinx, cosx, asin2 = prm.haversine_tables()
    for i in range(361):
        p.sinx[i], p.cosx[i] = sinx[i], cosx[i]
    for i in range(1001):
        p.asin2sqx[i] = asin2[i]
    return p


def test_philox_known_answers():
    """Philox4x32-10 known-answer vectors of the Random123 distribution."""
    lib = oracle_py.load()
    kat = [
        ((0, 0), (0, 0, 0, 0), (0x6627E8D5, 0xE169C58D, 0xBC57AC4C, 0x9B00DBD8)),
        ((0xFFFFFFFF, 0xFFFFFFFF), (0xFFFFFFFF,) * 4, (0x408F276D, 0x41C83B0E, 0xA20BC7C6, 0x6D5451FD)),
        ((0xA4093822, 0x299F31D0), (0x243F6A88, 0x85A308D3, 0x13198A2E, 0x03707344),
         (0xD16CFE09, 0x94FDCCEB, 0x5001E420, 0x24126EA1)),
    ]
    for key, ctr, want in kat:
        c = (C.c_uint32 * 4)(*ctr)
        o = (C.c_uint32 * 4)()
        lib.cs_cpu_philox(key[0], key[1], c, o)
        assert tuple(o) == want


def test_dist2_utm_bit_exact():
    g = GOLD["utm"]
    p = _utm_params(g["bbox_y"], 1.0 / 120, 240)
    lib = oracle_py.load()
    for x1, y1, x2, y2, d in zip(g["x1"], g["y1"], g["x2"], g["y2"], g["d2"]):
        assert lib.cs_cpu_dist2_raw(C.byref(p), x1, y1, x2, y2) == d


def test_dist2_cc_min_bit_exact():
    g = GOLD["cc_min"]
    p = _utm_params(GOLD["utm"]["bbox_y"], g["cell"], g["nch"])
    lib = oracle_py.load()
    for l, m, d in zip(g["l"], g["m"], g["d2"]):
        assert lib.cs_cpu_dist2_cc_min(C.byref(p), int(l), int(m)) == d


@pytest.mark.parametrize("key", ["kernel", "kernel2"])
def test_kernel_lookup_bit_exact(key):
    """Both the product's host table builder and the oracle's reproduce
    KernelLookup::num to the last bit."""
    g = GOLD[key]
    n, e = g["size"], g["expansion"]
    lib = abi.load_library()
    olib = oracle_py.load()
    for builder in (lib.cs_build_kernel_table, olib.cs_cpu_build_kernel_table):
        lk, hr = np.empty(n + 1), np.empty(n + 1)
        d = C.c_double()
        assert builder(g["type"], g["scale"], g["shape"], 0.0, 0.0, g["longest_d2"], n, e, lk.ctypes.data,
                       hr.ctypes.data, C.byref(d)) == 0
        got = [lib.cs_kernel_num(lk.ctypes.data, hr.ctypes.data, n, e, d.value, r2) for r2 in g["r2"]]
        assert got == g["num"]


@pytest.mark.parametrize("key", ["kernel", "kernel2"])
def test_kernel_lookup_fp32_within_1e6(key):
    """The spatial pass's acceptance test reads FP32 copies of the kernel tables:
    within 1e-6 relative of the reference's double KernelLookup::num."""
    g = GOLD[key]
    n, e = g["size"], g["expansion"]
    olib = oracle_py.load()
    lk, hr = np.empty(n + 1), np.empty(n + 1)
    d = C.c_double()
    assert olib.cs_cpu_build_kernel_table(g["type"], g["scale"], g["shape"], 0.0, 0.0, g["longest_d2"], n, e,
                                          lk.ctypes.data, hr.ctypes.data, C.byref(d)) == 0
    lk32, hr32 = lk.astype(np.float32), hr.astype(np.float32)
    got = np.array([olib.cs_cpu_kernel_num_f32(lk32.ctypes.data, hr32.ctypes.data, n, e, d.value, r2) for r2 in g["r2"]])
    want = np.array(g["num"])
    assert np.all(np.abs(got - want) <= 1e-6 * np.abs(want)), np.max(np.abs(got - want) / np.abs(want))


def test_inverse_cdf_bit_exact():
    g = GOLD["icdf"]
    icdf = abi.cs_icdf()
    for i, v in enumerate(g["raw"]):
        icdf.v[i] = math.exp(-v)
    lib = oracle_py.load()
    got = [lib.cs_cpu_icdf_choose(C.byref(icdf), m, u, g["steps_per_day"]) for u, m in zip(g["u"], g["mean"])]
    assert got == [int(v) for v in g["value"]]


def _moments_close(samples, mean, var, n_ref):
    """Sample moments agree with the reference's within 5 standard errors."""
    m, v = samples.mean(), samples.var()
    se_m = math.sqrt(var / len(samples) + var / n_ref)
    assert abs(m - mean) < 5 * se_m + 1e-12, (m, mean)
    # variance of the sample variance ~ 2 var^2 / n for near-normal; generous bound
    se_v = math.sqrt(2 * var * var / len(samples) + 2 * var * var / n_ref) * 2 + 1e-12
    assert abs(v - var) < 5 * se_v, (v, var)


def test_poisson_matches_reference_distribution():
    lib = oracle_py.load()
    for row in GOLD["samplers"]["poisson"]:
        n = 100000
        out = np.empty(n)
        lib.cs_cpu_sample_many(0, 77, row["lambda"], 0.0, n, out.ctypes.data)
        _moments_close(out, row["mean"], row["var"], row["n"])
        # two-sample chi-square on the common histogram
        h = np.zeros(64)
        b = out.astype(int) - row["offset"]
        ok = (b >= 0) & (b < 64)
        np.add.at(h, b[ok], 1)
        r = np.asarray(row["hist"], dtype=float)
        keep = (h + r) >= 20
        chi2 = (((h[keep] - r[keep]) ** 2) / (h[keep] + r[keep])).sum()
        dof = max(1, keep.sum() - 1)
        assert chi2 < dof + 6 * math.sqrt(2 * dof), (row["lambda"], chi2, dof)


def test_binomial_by_geometric_skips_matches_reference():
    lib = oracle_py.load()
    for row in GOLD["samplers"]["binomial"]:
        n = 100000
        out = np.empty(n)
        lib.cs_cpu_sample_many(2, 91, row["trials"], row["p"], n, out.ctypes.data)
        _moments_close(out, row["mean"], row["var"], row["n"])


def test_gamma_matches_reference_distribution():
    lib = oracle_py.load()
    for row in GOLD["samplers"]["gamma"]:
        n = 100000
        out = np.empty(n)
        lib.cs_cpu_sample_many(1, 5, row["shape"], row["shape"], n, out.ctypes.data)
        _moments_close(out, row["mean"], row["var"], row["n"])


def test_calc_inf_susc_bit_exact():
    g = GOLD["calc"]
    N, NH, NM = g["n"], len(g["hh_nhr"]), len(g["mcell_socdist"])
    ts = g["ts"]
    # a one-cell world holding exactly the harness's people
    grid = population.make_grid(width_deg=1.0 / 60, height_deg=1.0 / 60, cell_deg=1.0 / 60, nmcl=2)
    pop = population.Population(
        n_people=N, grid=grid, person_hh=np.array(g["hh"], dtype=np.int32),
        person_mcell=np.array(g["mcell"], dtype=np.int32), person_age=np.array(g["age"], dtype=np.uint8),
        person_flags=(np.array(g["care_home"], dtype=np.uint8) * abi.CS_PF_CARE_HOME_RESIDENT
                      | np.array(g["esocdist"], dtype=np.uint8) * abi.CS_PF_ESOCDIST_COMPLY).astype(np.uint8),
        person_place=np.full((4, N), -1, dtype=np.int32), person_group=np.zeros((4, N), dtype=np.uint16),
        hh_first=np.arange(0, N, 4, dtype=np.int32), hh_nh=np.full(NH, 4, dtype=np.uint16),
        hh_nhr=np.array(g["hh_nhr"], dtype=np.uint16), hh_x=np.zeros(NH, dtype=np.float32),
        hh_y=np.zeros(NH, dtype=np.float32), mcell_cell=np.zeros(NM, dtype=np.int32),
        mcell_adunit=np.zeros(NM, dtype=np.int32), mcell_grid=np.arange(NM), cell_grid=np.zeros(1, dtype=np.int32),
        cell_start=np.array([0, N], dtype=np.int32), cell_members=np.arange(N, dtype=np.int32),
        places=[dict(mcell=np.zeros(1, np.int32), x=np.zeros(1, np.float32), y=np.zeros(1, np.float32),
                     member_ofs=np.array([0, 0], np.int32), members=np.zeros(0, np.int32),
                     group_ofs=np.array([0, 1], np.int32), group_start=np.zeros(1, np.int32),
                     group_size=np.zeros(1, np.int32)) for _ in range(4)])
    P, lk, hr = prm.build_params(grid, kernel_size=20000)
    eff = np.array(g["efficacies"]).reshape(6, abi.CS_NUM_SETTINGS)
    for i in range(6):
        for j in range(abi.CS_NUM_SETTINGS):
            P.Efficacies[i][j] = eff[i, j]
    w = np.array(g["waifw"]).reshape(17, 17)
    for a in range(17):
        for b in range(17):
            P.WAIFW_Matrix[a][b] = w[a, b]
        P.AgeSusceptibility[a] = g["age_susc"][a]
        P.RelativeSpatialContact[a] = g["rel_spatial"][a]
        P.RelativeSpatialContactSusc[a] = g["rel_spatial_susc"][a]
    for i in range(10):
        P.HouseholdDenomLookup[i] = g["hh_denom"][i]
    for i in range(abi.CS_MAX_INFECTIOUS_STEPS):
        P.infectiousness[i] = g["infectiousness_profile"][i] if i < 200 else 0.0
    for t in range(5):
        P.PlaceTypeTrans[t] = g["place_trans"][t]
        P.PlaceTypeGroupSizeParam1[t] = g["group_size_param1"][t]
        P.SymptPlaceTypeContactRate[t] = g["sympt_place_contact"][t]
    P.CareHomeResidentHouseholdScaling = g["care_home_hh_scaling"]
    P.SymptSpatialContactRate = g["sympt_spatial"]
    P.SymptInfectiousness, P.AsymptInfectiousness = g["sympt_inf"], g["asympt_inf"]
    P.NoInfectiousnessSDinHH = 0
    P.usCaseIsolationDelay, P.usCaseIsolationDuration = g["us_iso_delay"], g["us_iso_dur"]
    P.usHQuarantineHouseDuration = g["us_hq_dur"]
    be = oracle_py.OracleBackend(pop.to_c(lk, hr), P)
    be.begin_run(1, [])
    arrs, view = sim.state_arrays(N, 1)
    be.download(view)
    arrs["inf"][:] = np.array(g["inf"], dtype=np.int8)
    arrs["susc"][:] = np.array(g["susc"], dtype=np.float32)
    arrs["infectiousness"][:] = np.array(g["infectiousness"], dtype=np.float32)
    arrs["latent_time"][:] = np.array(g["latent_time"], dtype=np.uint16)
    arrs["isolation_start_time"][:] = np.array(g["isolation_start_time"], dtype=np.uint16)
    arrs["quar_start_time"][:] = np.array(g["quar_start"], dtype=np.uint16)
    arrs["flags"][:] = (np.array(g["quar_comply"], dtype=np.uint8) << abi.CS_DF_QUAR_COMPLY_SHIFT).astype(np.uint8)
    be.upload(1, view)
    iv = abi.cs_interventions()
    iv.CaseIsolationTimeStart = iv.HQuarantineTimeStart = 1e10
    socd = np.array(g["mcell_socdist"], dtype=np.uint8)
    iv.mcell_socdist = socd.ctypes.data
    be.set_interventions(iv)
    for p in range(N):
        q = (p * 5 + 3) % N
        assert be.calc(0, p, q, 0, ts) == g["house_inf"][p], p
        assert be.calc(2, p, q, 0, ts) == g["spatial_inf"][p], p
        assert be.calc(4, p, q, 0, ts) == g["house_susc"][p], p
        assert be.calc(6, p, q, 0, ts) == g["spatial_susc"][p], p
        assert be.calc(7, p, q, 0, ts) == g["person_susc"][p], p
        for pt in range(4):
            assert be.calc(1, p, q, pt, ts) == g["place_inf"][p * 4 + pt], (p, pt)
            assert be.calc(5, p, q, pt, ts) == g["place_susc"][p * 4 + pt], (p, pt)
    be.close()
