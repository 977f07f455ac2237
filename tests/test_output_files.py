"""The reference's output tables (SaveResults, src/CovidSim.cpp:1657-1851) written
from a run's counter blocks, here from a run of the oracle under the host loop."""
import numpy as np

from covidsim_b200 import abi, output, sim
import oracle_py
from tests.helpers import tiny_world

DAYS = 12


def _run(tmp_path):
    pop, P, lk, hr = tiny_world(adunit_grid=2)
    o = sim.Simulation(pop, P, lk, hr, backend=oracle_py.OracleBackend)
    series, blocks = o.run(404, DAYS, n_seed=20, blocks=True)
    base = str(tmp_path / "run")
    ts = output.write_results(base, blocks, P.ModelTimeStep, n_adunits=pop.n_adunits)
    final = abi.counters_to_dict(o.backend.counters())
    o.close()
    return pop, series, blocks, base, ts, final


def test_blocks_match_series_and_final_counters(tmp_path):
    pop, series, blocks, base, ts, final = _run(tmp_path)
    assert blocks.shape == (DAYS + 1, abi.C.sizeof(abi.cs_counters) // 8)
    for k in ("S", "I", "cumI", "Critical"):
        assert np.array_equal(ts[k][1:] if k in ts else output._col(blocks, k)[1:], np.asarray(series[k], float))
    assert output._col(blocks, "cumI")[-1] == final["cumI"]
    # t = 0 is the state after seeding: 20 infections, nobody else touched
    assert ts["incI"][0] == 20 and ts["S"][0] == pop.n_people - 20


def test_main_table(tmp_path):
    pop, series, blocks, base, ts, final = _run(tmp_path)
    lines = open(base + ".xls").read().splitlines()
    head = lines[0].split("\t")
    assert head[:6] == ["t", "S", "L", "I", "R", "D"] and len(head) == 21 and head[-3:] == ["Extinct", "rmsRad", "maxRad"]
    rows = [l.split("\t") for l in lines[1:]]
    assert len(rows) == DAYS + 1
    # the reference's row format joins cumTP and cumV with a 't'
    assert all(len(r) == 20 and "t" in r[15] for r in rows)
    t = np.array([float(r[0]) for r in rows])
    assert np.array_equal(t, np.arange(DAYS + 1))
    SLIRD = np.array([[float(x) for x in r[1:6]] for r in rows])
    assert np.all(SLIRD.sum(axis=1) == pop.n_people)
    incI = np.array([float(r[6]) for r in rows])
    assert incI.sum() == final["cumI"]


def test_severity_and_adunit_tables(tmp_path):
    pop, series, blocks, base, ts, final = _run(tmp_path)
    sev = np.loadtxt(base + ".severity.xls", skiprows=1)
    head = open(base + ".severity.xls").readline().rstrip("\n").split("\t")
    assert len(head) == 31 and sev.shape == (DAYS + 1, 31)
    col = {h: sev[:, i] for i, h in enumerate(head)}
    assert col["cumCritical"][-1] == final["cumCritical"]
    assert np.array_equal(np.cumsum(col["incCritical"]), col["cumCritical"])
    assert col["cumDeath"][-1] == final["D"]
    ad = np.loadtxt(base + ".adunit.xls", skiprows=1)
    na = pop.n_adunits
    assert ad.shape == (DAYS + 1, 1 + 3 * na)
    # the admin units' infections add up to all infections
    assert np.array_equal(ad[:, 1:1 + na].sum(axis=1), ts["incI"])


def _rt_loop(inf, latent_time, infector, infect_type, dt, days):
    """The reference's loop (src/CovidSim.cpp:3882-3915, 3964-3973), person by person."""
    n, M = days + 1, abi.CS_INFECT_TYPE_MASK
    denom = [0.0] * n
    rtype = [[0.0] * M for _ in range(n)]
    for i in range(len(inf)):
        if inf[i] in (abi.CS_INF_SUSCEPTIBLE, abi.CS_INF_IMMUNE_AT_START):
            continue
        if latent_time[i] * dt <= days:
            denom[int(latent_time[i] * dt / 1.0)] += 1
        j = infector[i]
        if j >= 0 and latent_time[j] * dt <= days:
            rtype[int(latent_time[j] * dt / 1.0)][infect_type[i] % M] += 1
    out = []
    for k in range(n):
        d = denom[k] if denom[k] else 1e-10
        s = 0.0
        for t in range(M):
            s += rtype[k][t] / d
        out.append(s)
    return out


def test_reproduction_numbers(tmp_path):
    from tests.helpers import snapshot
    pop, P, lk, hr = tiny_world()
    o = sim.Simulation(pop, P, lk, hr, backend=oracle_py.OracleBackend)
    _, blocks = o.run(505, 40, n_seed=20, blocks=True)
    st = snapshot(o.backend, pop)
    rt = output.reproduction_numbers(st, P.ModelTimeStep, 40)
    want = _rt_loop(st["inf"], st["latent_time"], st["infector"], st["infect_type"], P.ModelTimeStep, 40)
    assert np.array_equal(rt, np.array(want))
    assert rt[:10].max() > 1.0            # a growing epidemic early on (R0 2.4)
    ts = output.write_results(str(tmp_path / "r"), blocks, P.ModelTimeStep, state=st, ages=pop.person_age)
    sev = np.loadtxt(str(tmp_path / "r") + ".severity.xls", skiprows=1)
    assert np.allclose(sev[:, 1], np.round(rt, 10), atol=1e-9)
    # the infection-type table: R is the sum of the Rtype columns, and the Rage
    # columns split the same infections by the infectee's age group
    it = np.loadtxt(str(tmp_path / "r") + ".inftype.xls", skiprows=1)
    M, G = abi.CS_INFECT_TYPE_MASK, abi.CS_NUM_AGE_GROUPS
    assert it.shape == (41, 4 + 2 * M + G)
    assert np.allclose(it[:, 4:4 + M].sum(axis=1), it[:, 1], atol=1e-4)
    assert np.allclose(it[:, 4 + 2 * M:].sum(axis=1), it[:, 1], atol=1e-4)
    assert it[:, 4 + M:4 + 2 * M].sum() == output._col(blocks, "cumI")[-1]
    # the age table: incidence by age group adds up to all infections, and the
    # distribution row to one
    lines = open(str(tmp_path / "r") + ".age.xls").read().splitlines()
    assert lines[-1].startswith("dist")
    age = np.array([[float(x) for x in l.split("\t")] for l in lines[1:-1]])
    assert age.shape == (41, 1 + 3 * G)
    assert np.array_equal(age[:, 1:1 + G].sum(axis=1), ts["incI"])
    assert abs(sum(float(x) for x in lines[-1].split("\t")[1:]) - 1.0) < 1e-8
    o.close()


def test_summary_over_realisations(tmp_path):
    pop, P, lk, hr = tiny_world()
    o = sim.Simulation(pop, P, lk, hr, backend=oracle_py.OracleBackend)
    runs = [o.run(900 + k, 15, n_seed=20, blocks=True)[1] for k in range(3)]
    # a run whose epidemic dies out at once: one infection that cannot spread
    runs.append(o.run(950, 15, n_seed=1, blocks=True)[1])
    o.close()
    series = [output.time_series(b, P.ModelTimeStep) for b in runs]
    ne = [s for s in series if not s["extinct"][-1]]
    base = str(tmp_path / "ens")
    assert output.write_summary(base, runs, P.ModelTimeStep, (0.5, 0.7, 1.2)) == len(ne)
    lines = open(base + ".avNE.xls").read().splitlines()
    head = lines[0].split("\t")
    assert head[:6] == ["t", "S", "L", "I", "R", "D"] and head[32:35] == ["", str(len(ne)), str(len(runs) - len(ne))]
    rows = np.array([[float(x) for x in l.split("\t")] for l in lines[1:]])
    assert rows.shape == (16, 32)
    mean_I = np.mean([s["I"] for s in ne], axis=0)
    var_I = np.var([s["I"] for s in ne], axis=0)
    assert np.allclose(rows[:, 3], mean_I, atol=1e-5) and np.allclose(rows[:, 21], var_I, rtol=1e-9, atol=1e-6)
    assert np.allclose(rows[:, 0], np.arange(16))


def test_summary_peak_statistics_follow_reference(tmp_path):
    """The header's peak statistics from hand-made runs, as RecordInfTypes forms them
    (src/CovidSim.cpp:3962-4016): the running maximum of the case incidence starts
    from the run's last-step Rt, a later equal value does not move the peak, and
    mean and variance are taken over all runs."""
    import ctypes as C
    W = C.sizeof(abi.cs_counters) // 8
    off = {k: getattr(abi.cs_counters, k).offset // 8 for k in ("cumC", "cumI", "S", "I")}

    def blocks(inc_c, infectious=3):
        b = np.zeros((len(inc_c), W), np.int64)
        b[:, off["cumC"]] = np.cumsum(inc_c)
        b[:, off["cumI"]] = np.cumsum(inc_c)
        b[:, off["S"]] = 1000
        b[:, off["I"]] = infectious
        return b

    runs = [blocks([0, 2, 7, 7, 3, 0]),    # peak 7 first reached on day 2
            blocks([0, 1, 1, 2, 9, 4]),    # peak 9 on day 4
            blocks([0, 1, 2, 1, 0, 0])]    # last-step Rt 2.5 is above every day: the peak stays at it
    last_rt = [1.5, 0.0, 2.5]
    base = str(tmp_path / "pk")
    output.write_summary(base, runs, 0.25, (0.0, 0.0, 0.0), last_rt=last_rt)
    head = open(base + ".avNE.xls").readline().rstrip("\n").split("\t")
    h = np.array([7.0, 9.0, 2.5])
    t = np.array([2.0, 4.0, 0.0])
    vals = [float(x) for x in head[-4:]]
    c = 1.0 / 3
    assert np.allclose(vals, [c * h.sum(), c * (h * h).sum() - c * c * h.sum() ** 2,
                              c * t.sum(), c * (t * t).sum() - c * c * t.sum() ** 2], atol=1e-9)


def test_tables_match_the_reference_written_tables(tmp_path):
    """The writers against the reference's own SaveResults / SaveSummaryResults on
    the same realisations: the reference executable with the oracle's sweeps linked
    in (oracle/_ref/CovidSim_oracle, built from the reference's sources) runs two
    realisations of a 20,000-person epidemic with interventions and writes its
    tables; the drop-in dumps the counter blocks RecordSample read
    (CS_DUMP_BLOCKS), and the tables written from them here must be the same bytes:
    `<base>.<run>.xls`, `<base>.<run>.severity.xls` and the data rows and peak
    statistics of `<base>.avNE.xls`."""
    import ctypes as C
    import os

    import pytest

    import ensemble
    import refrun
    binary = os.path.join(os.path.dirname(refrun.DROPIN), "CovidSim_oracle")
    if not os.path.exists(binary):
        pytest.skip("oracle/_ref/CovidSim_oracle not built (needs the reference checkout at build time)")
    days, wd = 200, str(tmp_path)
    refrun.run_reference(ensemble.population("interventions"), days, nr=2, threads=4, binary=binary, series=True,
                         workdir=wd, interventions=True, threshold=5,
                         env={"OMP_WAIT_POLICY": "passive", "CS_DUMP_BLOCKS": os.path.join(wd, "dump")},
                         pre_extra={"OutputNonSeverity": 1})
    small = 100    # "Maximum number of cases defining small outbreak" in the pre-parameters
    W = C.sizeof(abi.cs_counters) // 8
    runs = []
    for r in range(2):
        b = np.fromfile(os.path.join(wd, "dump.%d.blocks" % r), dtype=np.int64).reshape(-1, W)
        # a run whose epidemic died out stops calling the sweeps; RecordSample then
        # records the same state to the end
        assert 1 <= b.shape[0] <= days + 1
        runs.append(np.concatenate([b, np.repeat(b[-1:], days + 1 - b.shape[0], axis=0)]))
        mine = os.path.join(wd, "mine.%d" % r)
        output.write_results(mine, runs[-1], 0.25, small_epidemic_cases=small)
        for suffix in (".xls", ".severity.xls"):
            ref = open(os.path.join(wd, "out.%d%s" % (r, suffix))).read()
            assert open(mine + suffix).read() == ref, "run %d %s differs" % (r, suffix)
    output.write_summary(os.path.join(wd, "mine"), runs, 0.25, small_epidemic_cases=small)
    ref = open(os.path.join(wd, "out.avNE.xls")).read().split("\n")
    mine = open(os.path.join(wd, "mine.avNE.xls")).read().split("\n")
    assert mine[1:] == ref[1:]
    # the header: realisation counts and peak statistics (the R0 parts come from the
    # reference's set-up, not from the counters)
    hr, hm = ref[0].split("\t"), mine[0].split("\t")
    assert hm[:-8] == hr[:-8] and hm[-5:] == hr[-5:], (hm[-11:], hr[-11:])
