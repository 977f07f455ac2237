"""Statistical equivalence of whole epidemics: the reference executable against the
same executable with the GPU sweep linked in (oracle/_ref/CovidSim_b200).

TEST INFRASTRUCTURE.  Both binaries read the same parameter and density files, so
the reference's own set-up builds the same population (same set-up seeds) and its
own RecordSample writes the outputs; only the sweeps differ.  Per realisation we
keep the final size (cumulative infections), the peak day of prevalence and the
daily incidence, critical-care and death curves.

Workloads (CONFIGS):
  plain          20,000 people on 24 x 24 cells, 120 days, no interventions;
  medium         200,000 people at the 1M workload's cell density with the
                 interventions, people linked to places by a network file;
  holidays       the plain workload with a 30-day holiday from day 25 that closes
                 every school and university (the drop-in hands the reference's
                 holiday choices to the device);
  interventions  the same world for 200 days with the 10M workload's interventions:
                 the global trigger on critical-care admissions over the last 7 days
                 (above 5 here, the 20,000-person scale of the workload's 100 per
                 10M rounded up to a trigger that fires mid-growth in every run)
                 switches on case isolation, household quarantine, social
                 distancing and place closure for 90 days; the reference's own
                 RecordSample and TreatSweep decide them, the drop-in's sweeps
                 consume them.
"""
import os
import sys

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(HERE)
sys.path.insert(0, os.path.join(ROOT, "covid-sim_b200"))
sys.path.insert(0, HERE)

CONFIGS = {
    "plain": dict(people=20000, width_deg=0.2, cell_deg=1.0 / 120, nmcl=10, sigma=1.2, days=120, realisations=200,
                  setup_seed=98798150),
    "interventions": dict(people=20000, width_deg=0.2, cell_deg=1.0 / 120, nmcl=10, sigma=1.2, days=200,
                          realisations=200, setup_seed=98798150, interventions=True, threshold=5, duration=90.0),
}
# the plain world for 120 days with one 30-day holiday from day 25 that closes every
# school and university (the proportion of places of each type that stays open:
# primary, secondary, university, workplace), src/Sweep.cpp:889-918
CONFIGS["holidays"] = dict(CONFIGS["plain"], admin_extra={
    "Include holidays": 1, "Proportion of places remaining open during holidays by place type": [0.0, 0.0, 0.0, 1.0],
    "Number of holidays": 1, "Holiday start times": [25.0], "Holiday durations": [30.0]})
# 200,000 people at the 1M workload's cell density (1 x 1 degree, 120 x 120 cells of
# 10 x 10 microcells) for 200 days with the interventions (trigger above 20 weekly
# critical-care admissions); people linked to places by a network file (/L) written
# once per thread count by the network tool, so both arms hold the same network
CONFIGS["medium"] = dict(people=200000, width_deg=1.0, cell_deg=1.0 / 120, nmcl=10, sigma=1.2, days=200,
                         realisations=200, setup_seed=98798150, interventions=True, threshold=20, duration=90.0,
                         network=True)
CONFIG = CONFIGS["plain"]
GOLDEN = {"plain": "ref_ensemble.json", "interventions": "ref_ensemble_iv.json", "holidays": "ref_ensemble_hol.json",
          "medium": "ref_ensemble_200k.json"}


def population(config="plain"):
    from covidsim_b200 import population as popmod
    c = CONFIGS[config]
    grid = popmod.make_grid(width_deg=c["width_deg"], height_deg=c["width_deg"], cell_deg=c["cell_deg"], nmcl=c["nmcl"])
    return popmod.generate(c["people"], grid, sigma=c["sigma"], seed=c["setup_seed"])


def run(binary, nr=None, threads=None, config="plain"):
    """Realisations of `binary` on a workload.  A drop-in binary (its sweeps on the
    oracle or the GPU) runs with OpenMP's passive wait policy: its host threads idle
    while the sweep runs, and spinning threads would compete with it for cores."""
    import refrun
    c = CONFIGS[config]
    dropin = os.path.basename(binary) != "CovidSim"
    pop = population(config)
    extra = ()
    if c.get("network"):
        extra = ("/L:" + refrun.network_file(pop, "ensemble_" + config, threads or os.cpu_count()),)
    res = refrun.run_reference(pop, c["days"], nr=nr or c["realisations"], threads=threads, binary=binary, extra_args=extra,
                               series=True, timeout=5400, interventions=c.get("interventions", False),
                               threshold=c.get("threshold", 100), duration=c.get("duration", 90.0),
                               env={"OMP_WAIT_POLICY": "passive"} if dropin else None, admin_extra=c.get("admin_extra"))
    return summarise(res["series"]), res


def summarise(series):
    n = len(series)
    days = len(series[0]["t"])
    cumI = np.array([s["incI"].sum() for s in series])
    peak = np.array([int(np.argmax(s["I"])) for s in series])
    inc = np.stack([s["incI"] for s in series])
    crit = np.stack([s["Critical"] for s in series])
    deaths = np.stack([s["cumDeath"] for s in series])
    return dict(n=n, days=days, final_size=cumI.tolist(), peak_day=peak.tolist(),
                inc_mean=inc.mean(0).tolist(), inc_var=inc.var(0, ddof=1).tolist(),
                crit_mean=crit.mean(0).tolist(), crit_var=crit.var(0, ddof=1).tolist(),
                deaths_mean=deaths.mean(0).tolist(), deaths_var=deaths.var(0, ddof=1).tolist())


def compare(a, b):
    """Two-sample KS on final size and peak day; ensemble means of the daily curves
    within 2 standard errors on at least 90% of days and 4 on all."""
    from scipy import stats
    out = {}
    out["ks_final_size_p"] = float(stats.ks_2samp(a["final_size"], b["final_size"]).pvalue)
    out["ks_peak_day_p"] = float(stats.ks_2samp(a["peak_day"], b["peak_day"]).pvalue)
    for key in ("inc", "crit", "deaths"):
        ma, mb = np.array(a[key + "_mean"]), np.array(b[key + "_mean"])
        se = np.sqrt(np.array(a[key + "_var"]) / a["n"] + np.array(b[key + "_var"]) / b["n"])
        z = np.abs(ma - mb) / np.where(se > 0, se, np.inf)
        live = se > 0
        out[key + "_within_2se"] = float((z[live] <= 2).mean()) if live.any() else 1.0
        out[key + "_max_z"] = float(z[live].max()) if live.any() else 0.0
    return out
