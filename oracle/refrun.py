"""Run the reference executable on a synthetic workload and time its sweeps.

TEST AND CPU-BASELINE INFRASTRUCTURE: bench.py's reference arm and the statistical parity
tests call this; the product never does.  The workload's population is written in
the reference's input formats (covidsim_b200.refconfig), the reference builds its
own households and places from it, and oracle/_ref/CovidSim_timed (the reference
compiled from its sources with wall-clock timers around InfectSweep and
IncubRecoverySweep, oracle/ref_timing_shim.cpp) runs W + K realisations in one
process (/NR), so set-up is paid once.  person-steps/s = people x timesteps / sweep
wall time, per realisation.

At 10M people the reference's own place assignment alone runs for hours
(single-threaded, one microcell spiral per person), so those workloads load a
network file (/L) that oracle/_ref/CovidSim_netgen wrote once (/S): the reference's
own set-up with a fast place assignment (oracle/ref_network_tool.cpp).  The timed
reference and the drop-in (oracle/_ref/CovidSim_b200, the reference with the GPU
sweep linked in) then load the same file: the same people, households, places and
groups, and the same host code around the sweeps.
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
DROPIN = os.path.join(HERE, "_ref", "CovidSim_b200")
NETGEN = os.path.join(HERE, "_ref", "CovidSim_netgen")
NET_DIR = os.path.join(HERE, "_ref", "net")

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
    # The 10M workload itself on the 240 x 240 grid (the largest grid whose dense cell
    # tables, 26.5 GB, the reference can hold): the same density file, parameters
    # and interventions as the GPU's c1_240 workload, the population set up by the
    # reference from them with its place links from the network file.
    "c1_240": dict(people=10_000_000, preset="c1_240", days=365, interventions=True, threshold=100, network=True,
                   note="10M people on 240x240 cells, C1 interventions (global ICU trigger at 100 weekly admissions), "
                        "365 d; the reference's own set-up with place links loaded from a network file (/L)"),
}


def sample_population(s):
    sys.path.insert(0, os.path.join(ROOT, "covid-sim_b200"))
    from covidsim_b200 import population
    if s.get("preset"):
        return population.preset(s["preset"])
    grid = population.make_grid(cell_deg=s["cell_deg"], nmcl=10)
    return population.generate(s["people"], grid, sigma=1.2, seed=98798150)


def network_file(pop, key, threads):
    """The network file (person-to-place links) of the population `key`, written by
    CovidSim_netgen (/S) when absent; /L runs of the reference and the drop-in load
    it.  It records the population size and the set-up seeds, which /L checks.  The
    people the reference sets up depend on the density file, and its places are
    generated thread by thread with per-thread random streams (src/SetupModel.cpp:
    1520-1530), so a file fits one density file and one thread count: both are in
    its name (the density file by a hash of its bytes, which can differ between
    machines whose floating-point library rounds the generator's draws
    differently)."""
    import hashlib
    sys.path.insert(0, os.path.join(ROOT, "covid-sim_b200"))
    from covidsim_b200 import refconfig
    wd = tempfile.mkdtemp(prefix="csnet_")
    try:
        dens = os.path.join(wd, "density.txt")
        refconfig.write_density(dens, pop)
        h = hashlib.sha256()
        with open(dens, "rb") as f:
            for chunk in iter(lambda: f.read(1 << 24), b""):
                h.update(chunk)
        digest = h.hexdigest()[:12]
    finally:
        shutil.rmtree(wd, ignore_errors=True)
    path = os.path.join(NET_DIR, "%s_%s_t%d.net" % (key, digest, threads))
    if os.path.exists(path):
        return path
    if not os.path.exists(NETGEN):
        raise RuntimeError("oracle/_ref/CovidSim_netgen not built (needs the reference checkout at build time)")
    os.makedirs(NET_DIR, exist_ok=True)
    part = path[:-4] + ".part.net"
    if os.path.exists(part):
        os.remove(part)
    run_reference(pop, 1, nr=1, binary=NETGEN, threads=threads, extra_args=("/S:" + part,), timeout=7200)
    os.replace(part, path)
    return path


def parse_timing(stderr):
    rows = []
    for m in re.finditer(r"(?:REF|SWEEP)TIMING run=(\d+) pop=(\d+) threads=(\d+) steps=(\d+) infect_s=([\d.]+) incub_s=([\d.]+)"
                         r"((?: \w+=[\d.]+)*)", stderr):
        rows.append(dict(run=int(m.group(1)), pop=int(m.group(2)), threads=int(m.group(3)), steps=int(m.group(4)),
                         infect_s=float(m.group(5)), incub_s=float(m.group(6))))
        # the drop-in's parts: state upload, copies back, the wait for the device, the
        # copy into the host's cells, the hand-over after TreatSweep
        for k, v in re.findall(r" (\w+)=([\d.]+)", m.group(7)):
            rows[-1][k] = float(v)
    return rows


def run_reference(pop, days, nr=1, threads=None, interventions=False, threshold=100, workdir=None,
                  seeds=(98798150, 729101, 17389101, 4797132),
                  binary=BIN, keep=False, timeout=3000, series=False, duration=90.0, env=None, extra_args=(),
                  pre_extra=None, admin_extra=None):
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
        pre.update(pre_extra or {})
        refconfig.write_params(f["pre"], pre)
        if admin_extra:
            adm = refconfig.admin_params(pop.n_people, 100)
            adm.update(admin_extra)
            refconfig.write_params(f["admin"], adm)
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


def time_reference(workload, steps=3, warmup=3, binary=BIN, threads=None, env=None, pop=None):
    """Sweep throughput of `binary` on a workload sample: warmup + steps realisations
    in one process, the last `steps` timed (wall time of the sweep calls)."""
    if not os.path.exists(binary):
        return {"unavailable": "oracle/_ref/%s not built (the reference checkout was absent at build time)"
                               % os.path.basename(binary)}
    s = SAMPLES[workload]
    pop = pop if pop is not None else sample_population(s)
    threads = threads or os.cpu_count()
    extra = ("/L:" + network_file(pop, workload, threads),) if s.get("network") else ()
    run = lambda: run_reference(pop, s["days"], nr=warmup + steps, interventions=s["interventions"],
                                threshold=s["threshold"], binary=binary, threads=threads, env=env, extra_args=extra,
                                timeout=7200)
    try:
        res = run()
    except RuntimeError as e:
        # the reference's set-up may place people differently from the run that wrote
        # the cached file (its place generation is threaded): write the file again
        # from this machine's set-up and retry once
        if not extra or not re.search(r"place link|does not match|Incompatible network file", str(e)):
            raise
        os.remove(extra[0][3:])
        extra = ("/L:" + network_file(pop, workload, threads),)
        res = run()
    rows = res["rows"][warmup:warmup + steps]
    if len(rows) < steps:
        return {"unavailable": "reference produced %d timed realisations" % len(rows)}
    person_steps = sum(r["pop"] * r["steps"] for r in rows)
    secs = sum(r["infect_s"] + r["incub_s"] for r in rows)
    # RunModel's time stepping per realisation, the host code between sweeps included
    loop = [r["loop_s"] for r in rows if "loop_s" in r]
    return {"value": person_steps / secs, "ms_per_step": 1e3 * secs / steps, "cores": res["threads"],
            "run_loop_ms_per_step": round(1e3 * sum(loop) / len(loop), 3) if loop else None,
            "sample": s["note"] + "; %d realisations after %d warm-up, sweep wall time (omp_get_wtime), %d threads"
                      % (steps, warmup, res["threads"]), "rows": rows, "wall": res["wall"], "dropin": res.get("dropin"),
            "network_file": os.path.basename(extra[0][3:]) if extra else None}


def time_dropin(workload, steps=3, warmup=1, device=0, threads=None, pop=None):
    """The same as time_reference through the drop-in: the reference executable with
    the GPU sweep linked in, on this process's CUDA device `device` (the drop-in uses
    its device 0, so it is given that one device only)."""
    visible = os.environ.get("CUDA_VISIBLE_DEVICES")
    if visible:
        ids = [x for x in visible.split(",") if x.strip()]
        visible = ids[device] if device < len(ids) else str(device)
    else:
        visible = str(device)
    # OpenMP's wait policy as the reference arm runs with (the runtime's default)
    env = {"CUDA_VISIBLE_DEVICES": visible}
    if os.environ.get("CS_DROPIN_OMP_WAIT_POLICY"):
        env["OMP_WAIT_POLICY"] = os.environ["CS_DROPIN_OMP_WAIT_POLICY"]
    return time_reference(workload, steps=steps, warmup=warmup, binary=DROPIN, threads=threads, env=env, pop=pop)
