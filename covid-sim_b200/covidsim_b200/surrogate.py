"""Scenario surrogate around the GPU simulator (no counterpart in the reference).

A network (library entry points cs_sur_*) maps 8 scenario parameters to 365
daily values of 4 outputs.  It is trained on trajectories the simulator itself
generates (batched realisations, several seeds per scenario), screens large
scenario sweeps in milliseconds, and hands the scenarios it ranks highly back to
the simulator, which re-runs them and measures the surrogate's error against its
own ensemble mean.  The simulator stays the judge and the fallback.
"""
import ctypes as C

import numpy as np

from . import abi, sim

# (name, low, high) of the 8 scenario parameters; the network sees them scaled to [0, 1]
PARAMS = (
    ("R0", 1.5, 3.5),
    ("isolation_compliance", 0.3, 0.9),     # CaseIsolationProp
    ("quarantine_compliance", 0.3, 0.9),    # HQuarantinePropHouseCompliant
    ("distancing_compliance", 0.3, 0.9),    # 1 - residual spatial/work contacts under distancing
    ("icu_trigger", 20.0, 400.0),           # weekly ICU admissions switching interventions on
    ("closure_days", 30.0, 180.0),          # intervention duration
    ("isolation_residual", 0.1, 0.5),       # residual contacts of isolated cases
    ("closure_spatial_rel", 1.0, 1.5),      # relative spatial contacts while places are closed
)
N_PARAMS = len(PARAMS)
OUTPUTS = ("incidence", "hospital", "icu", "deaths")
DAYS = 365
LO = np.array([p[1] for p in PARAMS])
HI = np.array([p[2] for p in PARAMS])


def to_unit(theta):
    return (np.asarray(theta, np.float64) - LO) / (HI - LO)


def from_unit(u):
    return LO + np.asarray(u, np.float64) * (HI - LO)


def sample_scenarios(n, seed):
    return from_unit(np.random.default_rng(seed).random((n, N_PARAMS)))


def scenario_params(P, beta_r24, theta):
    """cs_params and intervention policy of one scenario: a copy of P with the
    transmission coefficient scaled to R0 and the intervention settings replaced."""
    q = abi.cs_params.from_buffer_copy(P)
    r0, iso, hq, sd, trig, dur, iso_res, pc_sp = [float(v) for v in theta]
    q.LocalBeta = beta_r24 * r0 / 2.4      # the calibrated coefficient scales R0 linearly
    q.CaseIsolationProp = iso
    q.HQuarantinePropHouseCompliant = hq
    E = q.Efficacies
    S_SP = abi.CS_SETTING_SPATIAL
    for t in range(abi.CS_MAX_PLACE_TYPES):
        E[abi.CS_NPI_CASE_ISOLATION][t] = iso_res
        if t >= 2:
            E[abi.CS_NPI_SOCIAL_DISTANCING][t] = 1.0 - sd
    E[abi.CS_NPI_CASE_ISOLATION][S_SP] = iso_res
    E[abi.CS_NPI_SOCIAL_DISTANCING][S_SP] = 1.0 - sd
    E[abi.CS_NPI_PLACE_CLOSURE][S_SP] = pc_sp
    policy = sim.InterventionPolicy(threshold=int(round(trig)), duration=dur)
    return q, policy


def outputs_from_series(series, n_people):
    """[365, 4] log1p(daily value per million): new infections, hospital
    occupancy (SARI + critical), critical-care occupancy, new deaths."""
    per_m = 1e6 / n_people
    cum_i = np.asarray(series["cumI"], np.float64)
    inc = np.diff(np.concatenate([[0.0], cum_i]))
    hosp = np.asarray(series["SARI"], np.float64) + np.asarray(series["Critical"], np.float64)
    icu = np.asarray(series["Critical"], np.float64)
    dead = np.asarray(series["D"], np.float64)
    deaths = np.diff(np.concatenate([[0.0], dead]))
    out = np.stack([inc, hosp, icu, deaths], axis=1)[:DAYS] * per_m
    return np.log1p(np.maximum(out, 0.0)).astype(np.float32)


def simulate(pop, P, lk, hr, thetas, seeds_per, days=DAYS, batch_size=64, n_seed=100, seed0=1000, progress=None):
    """Simulator trajectories for each scenario and seed: returns (theta index per
    trajectory, outputs [n, days, 4]).  Realisations run batched on one
    population: replicas with each scenario's parameters, one graph per timestep."""
    beta24, _ = sim.calibrate_local_beta(pop, P, 2.4)
    jobs = [(i, s) for i in range(len(thetas)) for s in range(seeds_per)]
    base = sim.Simulation(pop, P, lk, hr)
    members = [base] + [base.replica() for _ in range(min(batch_size, len(jobs)) - 1)]
    batch = sim.Batch(members)
    idx, outs = [], []
    try:
        for j0 in range(0, len(jobs), len(members)):
            chunk = jobs[j0:j0 + len(members)]
            policies, seeds = [], []
            for m, (i, s) in zip(members, chunk):
                q, pol = scenario_params(P, beta24, thetas[i])
                m.backend.set_params(q)
                m.params = q
                policies.append(pol)
                seeds.append(seed0 + 7919 * i + s)
            active = members[:len(chunk)]
            if len(active) < len(members):      # idle members repeat a finished job; results dropped
                policies += [policies[0]] * (len(members) - len(active))
                seeds += [seeds[0]] * (len(members) - len(active))
            series = batch.run(seeds, days, n_seed=n_seed, policy=policies)
            for (i, s), ser in zip(chunk, series):
                idx.append(i)
                outs.append(outputs_from_series(ser, pop.n_people))
            if progress:
                progress(j0 + len(chunk), len(jobs))
    finally:
        batch.close()
        for m in members:
            m.close()
    return np.asarray(idx), np.stack(outs)


class Surrogate:
    """The cs_sur_* network: FP32 master weights on the device, BF16 tensor-core
    (tcgen05) forward and backward with FP32 accumulation, Adam."""

    def __init__(self, max_batch=256, device=0, seed=0, params=None):
        self.lib = abi.load_library()
        self.h = C.c_void_p()
        rc = self.lib.cs_sur_create(max_batch, device, C.byref(self.h))
        if rc != 0:
            msg = self.lib.cs_sur_last_error(self.h)
            self.lib.cs_sur_destroy(self.h)
            self.h = None
            raise abi.CovidSimError("cs_sur_create: %s" % msg.decode())
        self.max_batch = max_batch
        self.set_params(he_init(seed) if params is None else params)

    def _ck(self, rc, what):
        if rc != 0:
            raise abi.CovidSimError("cs_sur_%s: %s" % (what, self.lib.cs_sur_last_error(self.h).decode()))

    @staticmethod
    def n_params():
        return abi.load_library().cs_sur_num_params()

    def set_gemm(self, impl):
        """Matrix products on tcgen05 ("tcgen05", the default) or mma.sync ("mma.sync")."""
        self._ck(self.lib.cs_sur_set_gemm(self.h, {"tcgen05": 0, "mma.sync": 1}[impl]), "set_gemm")

    def set_params(self, flat):
        f = np.ascontiguousarray(flat, np.float32)
        assert f.size == self.n_params()
        self._ck(self.lib.cs_sur_set_params(self.h, f.ctypes.data), "set_params")

    def get_params(self):
        f = np.empty(self.n_params(), np.float32)
        self._ck(self.lib.cs_sur_get_params(self.h, f.ctypes.data), "get_params")
        return f

    def predict(self, x_unit):
        x = np.ascontiguousarray(x_unit, np.float32)
        y = np.empty((x.shape[0], DAYS, len(OUTPUTS)), np.float32)
        self._ck(self.lib.cs_sur_forward(self.h, x.ctypes.data, x.shape[0], y.ctypes.data), "forward")
        return y

    def loss_grad(self, x_unit, target):
        x = np.ascontiguousarray(x_unit, np.float32)
        t = np.ascontiguousarray(target, np.float32)
        loss = C.c_float()
        g = np.empty(self.n_params(), np.float32)
        self._ck(self.lib.cs_sur_loss_grad(self.h, x.ctypes.data, t.ctypes.data, x.shape[0], C.byref(loss),
                                           g.ctypes.data), "loss_grad")
        return float(loss.value), g

    def train_step(self, x_unit, target, lr, weight_decay=0.0):
        x = np.ascontiguousarray(x_unit, np.float32)
        t = np.ascontiguousarray(target, np.float32)
        loss = C.c_float()
        self._ck(self.lib.cs_sur_train_step(self.h, x.ctypes.data, t.ctypes.data, x.shape[0], lr, weight_decay,
                                            C.byref(loss)), "train_step")
        return float(loss.value)

    def loss(self, x_unit, y):
        """Mean squared error of the predictions (no update)."""
        p = self.predict(x_unit)
        return float(np.mean((p - y) ** 2))

    def fit(self, x_unit, y, epochs=200, lr=1e-3, batch=None, seed=0, lr_final=1e-5, holdout=0.0, check_every=10,
            weight_decay=0.0):
        """Minibatch Adam with a cosine learning-rate decay; returns the epoch losses.
        With `holdout` > 0 that fraction of the samples is kept out of training and
        the weights with the lowest held-out loss (checked every `check_every`
        epochs) are kept at the end."""
        batch = batch or self.max_batch
        rng = np.random.default_rng(seed)
        n_all = x_unit.shape[0]
        perm = rng.permutation(n_all)
        n_val = int(n_all * holdout)
        val, tr = perm[:n_val], perm[n_val:]
        n = len(tr)
        hist = []
        steps = max(1, epochs * ((n + batch - 1) // batch))
        k = 0
        best, best_w = np.inf, None
        self.val_history = []
        for ep in range(epochs):
            order = tr[rng.permutation(n)]
            tot, cnt = 0.0, 0
            for b0 in range(0, n, batch):
                sel = order[b0:b0 + batch]
                lr_k = lr_final + 0.5 * (lr - lr_final) * (1 + np.cos(np.pi * k / steps))
                tot += self.train_step(x_unit[sel], y[sel], lr_k, weight_decay) * len(sel)
                cnt += len(sel)
                k += 1
            hist.append(tot / cnt)
            if n_val and ((ep + 1) % check_every == 0 or ep == epochs - 1):
                v = self.loss(x_unit[val], y[val])
                self.val_history.append((ep + 1, v))
                if v < best:
                    best, best_w = v, self.get_params()
        if best_w is not None:
            self.set_params(best_w)
        return hist

    def close(self):
        if self.h:
            self.lib.cs_sur_destroy(self.h)
            self.h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass


class Ensemble:
    """n Surrogates trained on the same scenarios from different initial weights,
    held-out splits and minibatch orders; their predictions are averaged on the
    natural scale (expm1 of the log1p outputs), which cuts the variance a single
    network shows between neighbouring scenarios."""

    def __init__(self, n, max_batch=256, seed=0):
        self.nets = []
        try:
            for k in range(n):
                self.nets.append(Surrogate(max_batch=max_batch, seed=seed + k))
        except Exception:
            self.close()
            raise

    def fit(self, x_unit, y, **kw):
        """Surrogate.fit for each member (member k splits and shuffles with seed k);
        returns the members' epoch losses."""
        kw.pop("seed", None)
        return [net.fit(x_unit, y, seed=k, **kw) for k, net in enumerate(self.nets)]

    def predict(self, x_unit):
        return np.log1p(np.mean([np.expm1(net.predict(x_unit)) for net in self.nets], axis=0)).astype(np.float32)

    def close(self):
        for net in self.nets:
            net.close()
        self.nets = []

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass


def relative_l2(pred, ref):
    """||pred - ref|| / ||ref|| per scenario, on the natural scale (expm1 of the
    log1p outputs)."""
    p, r = np.expm1(pred), np.expm1(ref)
    num = np.sqrt(((p - r) ** 2).sum(axis=tuple(range(1, p.ndim))))
    den = np.sqrt((r ** 2).sum(axis=tuple(range(1, r.ndim))))
    return num / np.maximum(den, 1e-12)


def he_init(seed):
    """He-uniform weights and zero biases in the flat layout of cs_sur_set_params."""
    rng = np.random.default_rng(seed)
    shapes = [(512, 8), (512, 512), (512, 512), (512, 512), (256, 512), (2944, 256), (64, 320), (32, 320), (4, 160)]
    parts = []
    for o, i in shapes:
        lim = np.sqrt(6.0 / i)
        parts.append(rng.uniform(-lim, lim, size=o * i).astype(np.float32))
        parts.append(np.zeros(o, np.float32))
    return np.concatenate(parts)


def time_training(steps=50, batch=256, sweep=100_000, impl="tcgen05", seed=0):
    """Milliseconds per training step (batch rows, random data) and seconds to screen
    `sweep` scenarios, on the given GEMM path."""
    import time
    rng = np.random.default_rng(seed)
    x = rng.random((batch, N_PARAMS)).astype(np.float32)
    y = rng.normal(0.0, 1.0, (batch, DAYS, len(OUTPUTS))).astype(np.float32)
    net = Surrogate(max_batch=batch, seed=seed)
    try:
        net.set_gemm(impl)
        for _ in range(3):
            net.train_step(x, y, 1e-3, 1e-4)
        t0 = time.perf_counter()
        for _ in range(steps):
            net.train_step(x, y, 1e-3, 1e-4)
        step_ms = (time.perf_counter() - t0) / max(steps, 1) * 1e3
        xs = rng.random((sweep, N_PARAMS)).astype(np.float32)
        t0 = time.perf_counter()
        net.predict(xs)
        screen_s = time.perf_counter() - t0
    finally:
        net.close()
    return step_ms, screen_s


if __name__ == "__main__":
    import argparse
    ap = argparse.ArgumentParser(description="time the surrogate's training step and screening")
    ap.add_argument("--steps", type=int, default=50)
    ap.add_argument("--sweep", type=int, default=100_000)
    ap.add_argument("--gemm", default="tcgen05", choices=["tcgen05", "mma.sync"])
    a = ap.parse_args()
    ms, sc = time_training(a.steps, sweep=a.sweep, impl=a.gemm)
    print("%s: %.3f ms per training step (256 rows), %.3f s to screen %d scenarios" % (a.gemm, ms, sc, a.sweep))
