"""The reference's time-series output files, made from the counter blocks a run
returns (sim.Simulation.run(..., blocks=True)): the block at t = 0 and at each day's
end.  With the device run loop those come back in one copy at the end of the run,
so there is no per-step host reduction (the reference's RecordSample,
src/CovidSim.cpp:3024-3484, sums per-thread state every sample).

TimeSeries[n] is the state at t = n days (n = 0 .. days), as RecordSample records
it with a one-day output step (src/CovidSim.cpp:1411-1413, 1525); incidences are
differences of cumulative counters between consecutive samples, the first from 0.
Columns for features the sweep does not model (treatment, vaccination, contact
tracing) are written as 0; Rt comes from the final per-person state when it is
given.  Files and formats follow
SaveResults and SaveSummaryResults (src/CovidSim.cpp:1657-2199): `<base>.xls`,
`<base>.severity.xls`, `<base>.age.xls`, `<base>.inftype.xls` and, with admin units,
`<base>.adunit.xls`, tab-separated.
"""
import numpy as np

from . import abi


def _col(blocks, name, k=None):
    off = getattr(abi.cs_counters, name).offset // 8
    return blocks[:, off + (k or 0)].astype(np.float64)


def _inc(x):
    return np.diff(x, prepend=0.0)


def time_series(blocks, model_timestep, small_epidemic_cases=-1, n_adunits=0):
    """TimeSeries fields [days + 1] from counter blocks [days + 1, words]."""
    b = np.asarray(blocks, np.int64)
    n = b.shape[0]
    ts = {"t": np.arange(n, dtype=np.float64)}
    for k in ("S", "L", "I", "R", "D", "Mild", "ILI", "SARI", "Critical", "CritRecov", "cumMild", "cumILI",
              "cumSARI", "cumCritical", "cumCritRecov", "cumDeath_ILI", "cumDeath_SARI", "cumDeath_Critical", "cumDC"):
        ts[k] = _col(b, k)
    for k, src in (("incI", "cumI"), ("incR", "cumR"), ("incFC", "cumFC"), ("incC", "cumC"), ("incDC", "cumDC"),
                   ("incD", "cumD"), ("incMild", "cumMild"), ("incILI", "cumILI"), ("incSARI", "cumSARI"),
                   ("incCritical", "cumCritical"), ("incCritRecov", "cumCritRecov"),
                   ("incDeath_ILI", "cumDeath_ILI"), ("incDeath_SARI", "cumDeath_SARI"),
                   ("incDeath_Critical", "cumDeath_Critical"), ("incHQ", "cumHQ")):
        ts[k] = _inc(_col(b, src))
    # RecordSample reads and zeroes the generation-time sums at every sample
    # (src/CovidSim.cpp:3065-3068, 3141-3146): means over each output step's new
    # infections, from the blocks' cumulative sums
    ntg, tg, si = _inc(_col(b, "nTG")), _inc(_col(b, "cumTG")), _inc(_col(b, "cumSI"))
    with np.errstate(invalid="ignore", divide="ignore"):
        ts["meanTG"] = np.where(ntg > 0, model_timestep * tg / np.maximum(ntg, 1), 0.0)
        ts["meanSI"] = np.where(ntg > 0, model_timestep * si / np.maximum(ntg, 1), 0.0)
    # infection radii as RecordSample forms them (src/CovidSim.cpp:3059-3074, 3107,
    # 3389-3390): it adds each thread's sum of squared radii twice, takes the root
    # mean over all infections, and the largest radius so far
    s2 = _col(b, "sumRad2_q") / 4294967296.0
    cum_i = _col(b, "cumI")
    with np.errstate(invalid="ignore", divide="ignore"):
        ts["rmsRad"] = np.where(cum_i > 0, np.sqrt((s2 + s2) / np.maximum(cum_i, 1.0)), 0.0)
    off = getattr(abi.cs_counters, "maxRad2_bits").offset // 8
    ts["maxRad"] = np.sqrt(np.ascontiguousarray(b[:, off]).view(np.float64))
    small = (ts["R"] <= small_epidemic_cases) if small_epidemic_cases >= 0 else np.ones(n, bool)
    ts["extinct"] = (small & (ts["I"] + ts["L"] == 0)).astype(np.float64)
    na = min(n_adunits, abi.CS_MAX_ADUNITS)
    for k, src in (("incI_adunit", "cumI_adunit"), ("incC_adunit", "cumC_adunit"), ("incDC_adunit", "cumDC_adunit")):
        ts[k] = np.stack([_inc(_col(b, src, a)) for a in range(na)], axis=1) if na else np.zeros((n, 0))
    return ts


def infection_breakdown(state, model_timestep, days, ages=None, output_step=1.0):
    """RecordInfTypes at the end of a run (src/CovidSim.cpp:3856-3973): every person
    ever infected (not susceptible, not immune at the start) whose latent period
    ended by the end of the run counts once in the output step of that time
    (Rdenom); every person they infected counts once in the same step of their
    infector, by the infection's type (Rtype) and by the infectee's age group
    (Rage).  Returns (Rt, Rtype [steps, 16], Rage [steps, 17] or None), each
    divided by Rdenom (1e-10 where no one's latent period ended), and Rt the sum
    of Rtype over the types in type order, as the reference forms them.  `state`
    holds the downloaded per-person arrays inf, latent_time, infector and
    infect_type (sim.state_arrays); `ages` the people's ages in years."""
    inf = np.asarray(state["inf"])
    t_lat = np.asarray(state["latent_time"], np.float64) * model_timestep
    infector = np.asarray(state["infector"], np.int64)
    n = int(days) + 1
    ever = (inf != abi.CS_INF_SUSCEPTIBLE) & (inf != abi.CS_INF_IMMUNE_AT_START)
    step = (t_lat / output_step).astype(np.int64)
    own = ever & (t_lat <= days)
    denom = np.bincount(step[own], minlength=n)[:n].astype(np.float64)
    idx = np.nonzero(ever)[0]
    src = infector[idx]
    keep = src >= 0
    idx, src = idx[keep], src[keep]
    keep = t_lat[src] <= days
    idx, src = idx[keep], src[keep]
    bins = step[src]
    denom[denom == 0] = 1e-10
    rtype = np.zeros((n, abi.CS_INFECT_TYPE_MASK))
    if "infect_type" in state:
        types = np.asarray(state["infect_type"], np.int64)[idx] % abi.CS_INFECT_TYPE_MASK
    else:
        types = np.zeros(len(idx), np.int64)
    np.add.at(rtype, (bins, types), 1.0)
    rtype /= denom[:, None]
    rt = np.zeros(n)
    for k in range(abi.CS_INFECT_TYPE_MASK):
        rt += rtype[:, k]
    rage = None
    if ages is not None:
        groups = np.minimum(np.asarray(ages, np.int64)[idx] // 5, abi.CS_NUM_AGE_GROUPS - 1)
        rage = np.zeros((n, abi.CS_NUM_AGE_GROUPS))
        np.add.at(rage, (bins, groups), 1.0)
        rage /= denom[:, None]
    return rt, rtype, rage


def reproduction_numbers(state, model_timestep, days, output_step=1.0):
    """Rt of each output step (infection_breakdown's first result)."""
    return infection_breakdown(state, model_timestep, days, output_step=output_step)[0]


def _write(path, header, columns):
    rows = np.stack(columns, axis=1)
    with open(path, "w") as f:
        f.write(header + "\n")
        for r in rows:
            f.write("\t".join("%.10f" % v for v in r) + "\n")


def write_results(base, blocks, model_timestep, small_epidemic_cases=-1, n_adunits=0, adunit_names=None, state=None,
                  ages=None):
    """Write `<base>.xls`, `<base>.severity.xls`, `<base>.age.xls` and, with admin
    units, `<base>.adunit.xls`; returns the TimeSeries fields.  With `state` (the
    final per-person arrays) the severity table's Rt column is filled (else it is
    0) and `<base>.inftype.xls` is written; `ages` (years) adds the age
    distribution row of the age table and the Rage columns."""
    ts = time_series(blocks, model_timestep, small_epidemic_cases, n_adunits)
    z = np.zeros_like(ts["t"])
    n = len(z)
    if state is not None:
        ts["Rt"], ts["Rtype"], ts["Rage"] = infection_breakdown(state, model_timestep, n - 1, ages)
    else:
        ts["Rt"] = z
    # SaveResults' main table (src/CovidSim.cpp:1665-1677); its format string has
    # "%.10ft%.10f" between cumTP and cumV, reproduced here
    with open(base + ".xls", "w") as f:
        f.write("t\tS\tL\tI\tR\tD\tincI\tincR\tincFC\tincC\tincDC\tincTC\tincCT\tincCC\tcumT\tcumTP\tcumV\tcumVG\t"
                "Extinct\trmsRad\tmaxRad\n")
        cols = [ts["t"], ts["S"], ts["L"], ts["I"], ts["R"], ts["D"], ts["incI"], ts["incR"], ts["incFC"], ts["incC"],
                ts["incDC"], z, z, z, z, z, z, z, ts["extinct"], ts["rmsRad"], ts["maxRad"]]
        for r in np.stack(cols, axis=1):
            v = ["%.10f" % x for x in r]
            f.write("\t".join(v[:15]) + "\t" + v[15] + "t" + "\t".join(v[16:]) + "\n")
    # the severity table (src/CovidSim.cpp:1838-1851)
    _write(base + ".severity.xls",
           "t\tRt\tTG\tSI\tS\tI\tR\tincI\tMild\tILI\tSARI\tCritical\tCritRecov\tincMild\tincILI\tincSARI\t"
           "incCritical\tincCritRecov\tincDeath\tincDeath_ILI\tincDeath_SARI\tincDeath_Critical\tcumMild\tcumILI\t"
           "cumSARI\tcumCritical\tcumCritRecov\tcumDeath\tcumDeath_ILI\tcumDeath_SARI\tcumDeath_Critical",
           [ts["t"], ts["Rt"], ts["meanTG"], ts["meanSI"], ts["S"], ts["I"], ts["R"], ts["incI"], ts["Mild"], ts["ILI"],
            ts["SARI"], ts["Critical"], ts["CritRecov"], ts["incMild"], ts["incILI"], ts["incSARI"], ts["incCritical"],
            ts["incCritRecov"], ts["incD"], ts["incDeath_ILI"], ts["incDeath_SARI"], ts["incDeath_Critical"],
            ts["cumMild"], ts["cumILI"], ts["cumSARI"], ts["cumCritical"], ts["cumCritRecov"], ts["D"],
            ts["cumDeath_ILI"], ts["cumDeath_SARI"], ts["cumDeath_Critical"]])
    # by age group (src/CovidSim.cpp:2035-2061), and by infection type
    # (src/CovidSim.cpp:2184-2199, "%lf" values there)
    b = np.asarray(blocks, np.int64)
    ng = abi.CS_NUM_AGE_GROUPS
    inc_age = {k: np.stack([_inc(_col(b, src, g)) for g in range(ng)], axis=1)
               for k, src in (("I", "cumIa"), ("C", "cumCa"), ("D", "cumDa"))}
    with open(base + ".age.xls", "w") as f:
        f.write("t" + "".join("\t%s%d-%d" % (k, 5 * g, 5 * (g + 1)) for k in ("I", "C", "D") for g in range(ng)) + "\n")
        for r in range(n):
            f.write("%.10f" % ts["t"][r] + "".join("\t%.10f" % inc_age[k][r, g] for k in ("I", "C", "D")
                                                 for g in range(ng)) + "\n")
        if ages is not None:
            dist = np.bincount(np.minimum(np.asarray(ages, np.int64) // 5, ng - 1), minlength=ng)[:ng]
            f.write("dist" + "".join("\t%.10f" % v for v in dist / max(dist.sum(), 1)) + "\n")
    if state is not None:
        inc_type = np.stack([_inc(_col(b, "cumItype", k)) for k in range(abi.CS_INFECT_TYPE_MASK)], axis=1)
        rage = ts["Rage"] if ts["Rage"] is not None else np.zeros((n, ng))
        with open(base + ".inftype.xls", "w") as f:
            f.write("t\tR\tTG\tSI" + "".join("\tRtype_%d" % k for k in range(abi.CS_INFECT_TYPE_MASK)) +
                    "".join("\tincItype_%d" % k for k in range(abi.CS_INFECT_TYPE_MASK)) +
                    "".join("\tRage_%d" % g for g in range(ng)) + "\n")
            for r in range(n):
                vals = [ts["t"][r], ts["Rt"][r], ts["meanTG"][r], ts["meanSI"][r]] + list(ts["Rtype"][r]) + \
                       list(inc_type[r]) + list(rage[r])
                f.write("\t".join("%f" % v for v in vals) + "\n")
    na = ts["incI_adunit"].shape[1]
    if na:
        names = list(adunit_names) if adunit_names is not None else ["%d" % a for a in range(na)]
        header = "t" + "".join("\tI_%s" % m for m in names[:na]) + "".join("\tC_%s" % m for m in names[:na]) + \
                 "".join("\tDC_%s" % m for m in names[:na])
        cols = [ts["t"]] + [ts["incI_adunit"][:, a] for a in range(na)] + [ts["incC_adunit"][:, a] for a in range(na)] \
            + [ts["incDC_adunit"][:, a] for a in range(na)]
        _write(base + ".adunit.xls", header, cols)
    return ts


def write_summary(base, runs, model_timestep, r0_parts=(0.0, 0.0, 0.0), small_epidemic_cases=-1, last_rt=None):
    """`<base>.avNE.xls`: the main table averaged over the non-extinct realisations
    among `runs` (each a run's counter blocks), with per-time-step variances, as
    SaveSummaryResults writes it (src/CovidSim.cpp:1960-1999; the sums over runs as
    src/CovidSim.cpp:3978-4019).  The header line carries the realisation counts
    (non-extinct, extinct), the three R0 parts, and the mean and variance over all
    realisations of the peak daily case incidence and its time.  The reference's
    column names are kept as it writes them (its ninth value is incFC under the
    name incD, and the variance written under vincFC is that of incD).  The peak of
    each realisation is found as RecordInfTypes finds it (src/CovidSim.cpp:3962-
    4016): the running maximum starts from the realisation's last-step Rt (the
    summed Rtype the loop before leaves in it; `last_rt`, one per run, 0 when not
    given) and a step counts when its case incidence exceeds it; the time is that
    step's output time.  When no step exceeds it the reference keeps an
    uninitialised time; 0 is written here.  Returns the number of non-extinct
    realisations."""
    series = [time_series(b, model_timestep, small_epidemic_cases) for b in runs]
    if not series:
        return 0
    n = len(series[0]["t"])
    zero = np.zeros(n)
    ne = [ts for ts in series if not ts["extinct"][-1]]
    n_ne, n_e = len(ne), len(series) - len(ne)
    peaks_h, peaks_t = [], []
    for i, ts in enumerate(series):
        h, t = (float(last_rt[i]) if last_rt is not None else 0.0), 0.0
        for k in range(n):
            if h < ts["incC"][k]:
                h, t = float(ts["incC"][k]), float(ts["t"][k])
        peaks_h.append(h)
        peaks_t.append(t)
    c = 1.0 / len(series)
    ph, pt = np.asarray(peaks_h), np.asarray(peaks_t)
    head = ("t\tS\tL\tI\tR\tD\tincI\tincR\tincD\tincC\tincDC\tincTC\tcumT\tcumTmax\tcumTP\tcumV\tcumVmax\tExtinct\t"
            "rmsRad\tmaxRad\tvS\tvI\tvR\tvD\tvincI\tvincR\tvincFC\tvincC\tvincDC\tvincTC\tvrmsRad\tvmaxRad\t\t%i\t%i\t"
            "%.10f\t%.10f\t%.10f\t\t%.10f\t%.10f\t%.10f\t%.10f\n"
            % (n_ne, n_e, r0_parts[0], r0_parts[1], r0_parts[2], c * ph.sum(), c * (ph * ph).sum() - c * c * ph.sum() ** 2,
               c * pt.sum(), c * (pt * pt).sum() - c * c * pt.sum() ** 2))
    with open(base + ".avNE.xls", "w") as f:
        f.write(head)
        if not n_ne:
            return 0
        c = 1.0 / n_ne

        def mean(k):
            return c * sum(ts.get(k, zero) for ts in ne)

        def var(k):
            s1 = sum(ts.get(k, zero) for ts in ne)
            s2 = sum(ts.get(k, zero) ** 2 for ts in ne)
            return c * s2 - c * c * s1 * s1
        first = ["t", "S", "L", "I", "R", "D", "incI", "incR", "incFC", "incC", "incDC", "incTC", "cumT", "cumTmax",
                 "cumTP", "cumV", "cumVmax", "extinct", "rmsRad", "maxRad"]
        maxed = {"cumTmax", "cumVmax"}    # written as maxima, not scaled by c
        cols1 = [zero if k in maxed else mean(k) for k in first]
        cols2 = [var(k) for k in ("S", "I", "R", "D", "incI", "incR", "incD", "incC", "incDC", "incTC", "rmsRad", "maxRad")]
        for r in range(n):
            f.write("%.10f" % cols1[0][r] + "".join("\t%10f" % col[r] for col in cols1[1:]) + "\t")
            f.write("\t".join("%.10f" % col[r] for col in cols2) + "\n")
    return n_ne
