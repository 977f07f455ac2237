"""Run the reference executable on a synthetic workload and time its sweeps.

TEST AND CPU-BASELINE INFRASTRUCTURE: bench.py's reference arm and the statistical parity
tests call this; the product never does.  The workload's population is written in
the reference's input formats (covidsim_b200.refconfig), the reference builds its
own households and places from it, and oracle/_ref/CovidSim_timed (the reference
compiled from its sources with wall-clock timers around InfectSweep and
IncubRecoverySweep, oracle/ref_timing_shim.cpp) runs W + K realisations in one
process (/NR), so set-up is paid once.  person-steps/s = people x timesteps / sweep
wall time, per realisation.
"""
import os
import re
import shutil
import subprocess
import sys
import tempfile
import time

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(HERE)
BIN = os.path.join(HERE, "_ref", "CovidSim_timed")
STOCK = os.path.join(HERE, "_ref", "CovidSim")

# The reference keeps two dense Ncells x Ncells float tables (src/SetupModel.cpp:
# 1207-1216): 8 bytes per cell pair.  Its sample grids are chosen to fit in memory
# and set up in seconds.
SAMPLES = {
    # The 10M-person workload scaled down to what the reference sets up in about a
    # minute: its dense cell tables (8 B x cells^2) rule out the 600x600 grid
    # (1.04 TB) and its set-up time grows with people and with cells^2.  The
    # sample keeps the workload's generator, its 28 people per cell and its
    # interventions, with the ICU trigger scaled per head (100 per 10M).
    "c1": dict(people=115_000, cell_deg=1.0 / 32, days=365, interventions=True, threshold=1,
               note="115k people of the 10M workload's generator on 64x64 cells (28 people per cell, as the "
                    "10M workload), C1 interventions with the ICU trigger scaled per head, 365 d"),
    "c0": dict(people=1_000_000, cell_deg=1.0 / 120, days=120, interventions=False, threshold=100,
               note="1M people, 240x240 cells (26.5 GB of dense cell tables), 120 d"),
}


def parse_timing(stderr):
    rows = []
    for m in re.finditer(r"(?:REF|SWEEP)TIMING run=(\d+) pop=(\d+) threads=(\d+) steps=(\d+) infect_s=([\d.]+) incub_s=([\d.]+)",
                         stderr):
        rows.append(dict(run=int(m.group(1)), pop=int(m.group(2)), threads=int(m.group(3)), steps=int(m.group(4)),
                         infect_s=float(m.group(5)), incub_s=float(m.group(6))))
    return rows


def run_reference(pop, days, nr=1, threads=None, interventions=False, threshold=100, workdir=None,
                  seeds=(98798150, 729101, 17389101, 4797132),
                  binary=BIN, keep=False, timeout=3000, series=False, duration=90.0, env=None, extra_args=()):
    sys.path.insert(0, os.path.join(ROOT, "covid-sim_b200"))
    from covidsim_b200 import refconfig
    threads = threads or os.cpu_count()
    wd = workdir or tempfile.mkdtemp(prefix="csref_")
    try:
        f = refconfig.write_workload(wd, pop, days, interventions=interventions)
        params = refconfig.intervention_params(interventions, duration=duration, threshold=threshold)
        pre = refconfig.pre_params(days, pop.grid, 2.4, 100)
        pre["Number of realisations"] = nr
        pre["Number of non-extinct realisations"] = nr
        if series:  # one .severity.xls per realisation
            pre["OutputNonSummaryResults"] = 1
            pre["OutputSeverity"] = 1
        refconfig.write_params(f["pre"], pre)
        refconfig.write_params(f["params"], params)
        cmd = [binary, "/c:%d" % threads, "/PP:" + f["pre"], "/P:" + f["params"], "/A:" + f["admin"],
               "/D:" + f["density"], "/O:" + os.path.join(wd, "out"), *extra_args, *[str(s) for s in seeds]]
        t0 = time.time()
        r = subprocess.run(cmd, capture_output=True, text=True, timeout=timeout,
                           env=dict(os.environ, **env) if env else None)
        wall = time.time() - t0
        if r.returncode != 0:
            raise RuntimeError("reference exited %d: %s" % (r.returncode, r.stderr[-800:]))
        out = dict(rows=parse_timing(r.stderr), wall=wall, threads=threads, workdir=wd, stderr=r.stderr[-4000:],
                   dropin=[ln[ln.index("GPU sweep:"):].strip() for ln in r.stderr.splitlines() if "GPU sweep:" in ln])
        if series:
            out["series"] = [read_severity(os.path.join(wd, "out.%d.severity.xls" % k) if nr > 1 else
                                           os.path.join(wd, "out.severity.xls")) for k in range(nr)]
        return out
    finally:
        if not keep and workdir is None:
            shutil.rmtree(wd, ignore_errors=True)


def read_severity(path):
    """Daily series of one realisation from the reference's .severity.xls output
    (src/CovidSim.cpp:1838-1850)."""
    import numpy as np
    with open(path) as f:
        head = f.readline().strip().split("\t")
        data = np.array([[float(x) for x in line.split("\t")] for line in f if line.strip()])
    return {k: data[:, i] for i, k in enumerate(head)}


def time_reference(workload, steps=3, warmup=3):
    if not os.path.exists(BIN):
        return {"unavailable": "oracle/_ref/CovidSim_timed not built (the reference checkout was absent at build time)"}
    sys.path.insert(0, os.path.join(ROOT, "covid-sim_b200"))
    from covidsim_b200 import population
    s = SAMPLES[workload]
    grid = population.make_grid(cell_deg=s["cell_deg"], nmcl=10)
    pop = population.generate(s["people"], grid, sigma=1.2, seed=98798150)
    res = run_reference(pop, s["days"], nr=warmup + steps, interventions=s["interventions"], threshold=s["threshold"])
    rows = res["rows"][warmup:warmup + steps]
    if len(rows) < steps:
        return {"unavailable": "reference produced %d timed realisations" % len(rows)}
    person_steps = sum(r["pop"] * r["steps"] for r in rows)
    secs = sum(r["infect_s"] + r["incub_s"] for r in rows)
    return {"value": person_steps / secs, "ms_per_step": 1e3 * secs / steps, "cores": res["threads"],
            "sample": s["note"] + "; %d realisations after %d warm-up, sweep wall time (omp_get_wtime), %d threads"
                      % (steps, warmup, res["threads"]), "rows": rows}
