"""Run loop around the sweep: the host side of RunModel (src/CovidSim.cpp:1383-1543).

`Simulation` owns one device context (cs_gpu_*) and drives it step by step:
InitModel + SeedInfection at the start of a realisation, InfectSweep +
IncubRecoverySweep per timestep, UpdateProbs(0) whenever the susceptible fraction
has fallen by 0.2 since the last update, daily counter samples (RecordSample,
CovidSim.cpp:3024) and, for the intervention configurations, a global trigger on
weekly ICU admissions that switches case isolation, household quarantine, school
and university closure and social distancing on for a fixed duration (the role
TreatSweep plays, Sweep.cpp:1324-2004).

`calibrate_local_beta` restates InitTransmissionCoeffs (src/SetupModel.cpp:640-846):
the spatial transmission coefficient that makes the household + place + spatial
reproduction numbers add up to R0.
"""
import ctypes as C
import math
from dataclasses import dataclass

import numpy as np

from . import abi


class GpuBackend:
    """The cs_gpu_* entry points of the library, as methods."""
    prefix = "cs_gpu_"

    def __init__(self, pop_c, params, device=0):
        self.lib = abi.load_library()
        self.ctx = C.c_void_p()
        rc = self.lib.cs_gpu_create(C.byref(pop_c), C.byref(params), device, C.byref(self.ctx))
        if rc != 0:
            msg = self.lib.cs_gpu_last_error(self.ctx)
            self.lib.cs_gpu_destroy(self.ctx)
            self.ctx = None
            raise abi.CovidSimError("cs_gpu_create: %s" % (msg.decode() if msg else rc))

    @classmethod
    def replica(cls, base):
        """Another realisation of base's population, sharing its static device arrays."""
        self = cls.__new__(cls)
        self.lib = base.lib
        self.ctx = C.c_void_p()
        rc = self.lib.cs_gpu_create_replica(base.ctx, C.byref(self.ctx))
        if rc != 0:
            msg = self.lib.cs_gpu_last_error(self.ctx)
            self.lib.cs_gpu_destroy(self.ctx)
            self.ctx = None
            raise abi.CovidSimError("cs_gpu_create_replica: %s" % (msg.decode() if msg else rc))
        return self

    def set_grid(self, blocks):
        self._ck(self.lib.cs_gpu_set_grid(self.ctx, blocks), "set_grid")

    def set_spatial_lanes(self, lanes):
        self._ck(self.lib.cs_gpu_set_spatial_lanes(self.ctx, lanes), "set_spatial_lanes")

    def _ck(self, rc, what):
        if rc != 0:
            raise abi.CovidSimError("%s%s: %s" % (self.prefix, what, self.lib.cs_gpu_last_error(self.ctx).decode()))

    def close(self):
        if self.ctx:
            self.lib.cs_gpu_destroy(self.ctx)
            self.ctx = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    def begin_run(self, seed, seeds):
        s = np.ascontiguousarray(seeds, dtype=np.int32)
        self._ck(self.lib.cs_gpu_begin_run(self.ctx, seed, s.ctypes.data, len(s), 0), "begin_run")

    def seed_infections(self, t, people):
        s = np.ascontiguousarray(people, dtype=np.int32)
        self._ck(self.lib.cs_gpu_seed_infections(self.ctx, t, s.ctypes.data, len(s)), "seed_infections")

    def infect_sweep(self, t, run=0):
        self._ck(self.lib.cs_gpu_infect_sweep(self.ctx, t, run), "infect_sweep")

    def incub_recovery_sweep(self, t):
        self._ck(self.lib.cs_gpu_incub_recovery_sweep(self.ctx, t), "incub_recovery_sweep")

    def step(self, t, run=0):
        self._ck(self.lib.cs_gpu_step(self.ctx, t, run), "step")

    def update_probs(self, do_place=0):
        self._ck(self.lib.cs_gpu_update_probs(self.ctx, do_place), "update_probs")

    def update_probs_static(self, do_place=0):
        """UpdateProbs with the library's fixed scratch array (no device allocation)."""
        self._ck(self.lib.cs_gpu_update_probs_static(self.ctx, do_place), "update_probs_static")

    def set_params(self, params):
        self._ck(self.lib.cs_gpu_set_params(self.ctx, C.byref(params)), "set_params")

    def set_interventions(self, iv):
        self._ck(self.lib.cs_gpu_set_interventions(self.ctx, C.byref(iv)), "set_interventions")

    def close_places(self, place_type, mcells, start, stop):
        if mcells is None:
            self._ck(self.lib.cs_gpu_close_places(self.ctx, place_type, None, 0, start, stop), "close_places")
        else:
            m = np.ascontiguousarray(mcells, dtype=np.int32)
            self._ck(self.lib.cs_gpu_close_places(self.ctx, place_type, m.ctypes.data, len(m), start, stop), "close_places")

    def place_events(self, events):
        """Outcomes of a host TreatSweep's DoPlaceClose / DoPlaceOpen calls (a list of
        abi.cs_place_event)."""
        ev = (abi.cs_place_event * len(events))(*events)
        self._ck(self.lib.cs_gpu_place_events(self.ctx, ev, len(events)), "place_events")

    def set_mcell_status(self, mcells, socdist=None, moverest=None):
        """Microcell social-distancing / movement-restriction status (TreatStat) for
        the listed microcells."""
        m = np.ascontiguousarray(mcells, dtype=np.int32)
        sd = None if socdist is None else np.ascontiguousarray(socdist, dtype=np.uint8)
        mr = None if moverest is None else np.ascontiguousarray(moverest, dtype=np.uint8)
        self._ck(self.lib.cs_gpu_set_mcell_status(self.ctx, m.ctypes.data, None if sd is None else sd.ctypes.data,
                                                  None if mr is None else mr.ctypes.data, len(m)), "set_mcell_status")

    def counters(self):
        out = abi.cs_counters()
        self._ck(self.lib.cs_gpu_get_counters(self.ctx, C.byref(out)), "get_counters")
        return out

    def run_device(self, days, policy):
        """cs_gpu_run: `days` days from t = 0 with the run loop's logic on the device
        (policy: a cs_run_policy); returns the day-end counter blocks as an int64
        array [days, sizeof(cs_counters) / 8]."""
        out = np.empty((days, C.sizeof(abi.cs_counters) // 8), np.int64)   # every field is int64
        self._ck(self.lib.cs_gpu_run(self.ctx, days, C.byref(policy), out.ctypes.data), "run")
        return out

    def download(self, view):
        self._ck(self.lib.cs_gpu_download_state(self.ctx, C.byref(view)), "download_state")

    def sync(self):
        self._ck(self.lib.cs_gpu_sync(self.ctx), "sync")

    def stream(self):
        return self.lib.cs_gpu_stream(self.ctx)

    def launches(self):
        return self.lib.cs_gpu_launch_count(self.ctx)

    def upload(self, seed, view):
        self._ck(self.lib.cs_gpu_upload_state(self.ctx, seed, C.byref(view)), "upload_state")

    def profile(self, enable):
        self._ck(self.lib.cs_gpu_profile(self.ctx, enable), "profile")

    def profile_entries(self):
        """{kernel name: (total ms, launches)} recorded since profiling was enabled."""
        out = {}
        buf = C.create_string_buffer(128)
        ms, n = C.c_double(), C.c_int64()
        i = 0
        while self.lib.cs_gpu_profile_entry(self.ctx, i, buf, 128, C.byref(ms), C.byref(n)) == 0:
            out[buf.value.decode()] = (ms.value, n.value)
            i += 1
        return out


def state_arrays(n_people, n_cells):
    """Host arrays for every field of cs_state_view, and the view over them."""
    spec = dict(inf=np.int8, severity=np.uint8, flags=np.uint8, infection_time=np.uint16, latent_time=np.uint16,
                recovery_or_death_time=np.uint16, SARI_time=np.uint16, Critical_time=np.uint16,
                Stepdown_time=np.uint16, absent_start_time=np.uint16, absent_stop_time=np.uint16,
                isolation_start_time=np.uint16, quar_start_time=np.uint16, detected_time=np.uint16,
                infectiousness=np.float32, susc=np.float32, ProbAbsent=np.float32, ProbCare=np.float32,
                infector=np.int32, infect_type=np.int16, listpos=np.int32, cell_slots=np.int32)
    cell_spec = dict(cell_S=np.int32, cell_L=np.int32, cell_I=np.int32, cell_R=np.int32, cell_D=np.int32,
                     cell_S0=np.int32, cell_tot_prob=np.float64)
    arrs = {k: np.zeros(n_people, dtype=v) for k, v in spec.items()}
    arrs.update({k: np.zeros(n_cells, dtype=v) for k, v in cell_spec.items()})
    view = abi.cs_state_view()
    for k, a in arrs.items():
        setattr(view, k, a.ctypes.data)
    return arrs, view


# ------------------------------------------------------------ calibration
def calibrate_local_beta(pop, p, R0, seed=1, sample=400_000):
    """P.LocalBeta from InitTransmissionCoeffs (src/SetupModel.cpp:640-846), by the
    same per-person expectation over a sample of the population."""
    rng = np.random.default_rng(seed)
    N = pop.n_people
    idx = rng.choice(N, size=min(N, sample), replace=False) if N > sample else np.arange(N)
    n = len(idx)
    dt = p.ModelTimeStep
    ag = np.minimum(pop.person_age[idx] // 5, abi.CS_NUM_AGE_GROUPS - 1)
    k = 1.0 / (p.InfectiousnessSD ** 2) if p.InfectiousnessSD > 0 else None
    infn = np.array([p.AgeInfectiousness[a] for a in range(abi.CS_NUM_AGE_GROUPS)])[ag]
    if k:
        infn = infn * rng.gamma(k, 1.0 / k, n)
    sympt = rng.random(n) < np.array(list(p.ProportionSymptomatic))[ag]
    infn = np.where(sympt, -infn * p.SymptInfectiousness, infn * p.AsymptInfectiousness)
    # recovery time in steps from the infectious-period ICDF (constant exp(-1) with a profile)
    q = rng.random(n) * abi.CS_CDF_RES
    j = np.floor(q).astype(int)
    q -= j
    icdf = np.array(list(p.infectious_icdf.v))
    rec = np.floor(0.5 - (p.InfectiousPeriod * np.log(q * icdf[j + 1] + (1 - q) * icdf[j]) / dt)).astype(int)
    prof = np.array(list(p.infectiousness))
    cum = np.concatenate([[0.0], np.cumsum(prof)])
    lts = min(int(p.LatentToSymptDelay / dt), 10 ** 6)
    pre = np.minimum(np.minimum(rec, lts), rec)
    # household
    hh = pop.person_hh[idx]
    nh = pop.hh_nh[hh].astype(int)
    nhr = pop.hh_nhr[hh].astype(int)
    hinf = np.abs(infn) * dt * p.HouseholdTrans * np.array(list(p.HouseholdDenomLookup))[nhr - 1]
    logs = np.log(np.clip(1.0 - hinf[:, None] * prof[None, :200], 1e-300, None))
    mask = np.arange(200)[None, :] < rec[:, None]
    surv = np.exp(np.where(mask, logs, 0.0).sum(axis=1))
    R0hh = ((1 - surv) * np.array(list(p.AgeSusceptibility))[ag] * (nh - 1)).sum() / n
    # spatial
    rsc = np.array(list(p.RelativeSpatialContact))[ag]
    sinf = np.abs(infn) * rsc * dt
    sp = sinf * cum[pre] + sinf * np.where(infn < 0, p.SymptSpatialContactRate, 1.0) * (cum[rec] - cum[pre])
    R0sp = sp.sum() / n
    # places
    R0pl = 0.0
    for t in range(pop.num_place_types):
        link = pop.person_place[t, idx]
        has = link >= 0
        if not has.any():
            continue
        pl = pop.places[t]
        li = link[has]
        gi = pop.person_group[t, idx][has].astype(int)
        gsz = pl["group_size"][pl["group_ofs"][li] + gi].astype(float)
        npl = np.diff(pl["member_ofs"])[li].astype(float)
        infh = np.abs(infn[has])
        pinf = infh * dt * p.PlaceTypeTrans[t]
        att = np.where(infn[has] < 0, p.SymptPlaceTypeContactRate[t] * (1 - p.SymptPlaceTypeWithdrawalProp[t]), 1.0)
        r, pr = rec[has], pre[has]
        lim = 200
        days = np.arange(lim)[None, :]
        fac = np.where(days < pr[:, None], 1.0, att[:, None])
        live = days < r[:, None]

        def survive(scale):
            v = 1.0 - scale[:, None] * prof[None, :lim] * fac
            return np.exp(np.where(live, np.log(np.clip(v, 1e-300, None)), 0.0).sum(axis=1))

        s_grp = survive(pinf / p.PlaceTypeGroupSizeParam1[t])
        s_btw = survive(p.PlaceTypePropBetweenGroupLinks[t] * pinf / npl)
        ng = gsz - 1
        R0pl += ((1 - s_grp * s_btw) * ng + (1 - s_btw) * (npl - 1 - ng)).sum() / n
    beta = (R0 - R0hh - R0pl) / R0sp if R0sp > 0 else 0.0
    return max(beta, 0.0), dict(R0household=R0hh, R0places=R0pl, SpatialR0=R0sp)


# --------------------------------------------------------------- run loop
@dataclass
class InterventionPolicy:
    """Global ICU trigger (src/CovidSim.cpp:3150-3159 ICU triggers with global
    thresholds): when admissions to critical care over the last `window` days reach
    `threshold`, switch the interventions on for `duration` days."""
    threshold: int = 100
    window: int = 7
    duration: float = 90.0
    close_place_types: tuple = (0, 1, 2)
    social_distancing: bool = True
    case_isolation: bool = True
    household_quarantine: bool = True
    # one trigger per admin unit (the reference's DoAdminTriggers) on the unit's own
    # admissions, firing above the threshold and switching that unit's windows,
    # microcells and places
    per_adunit: bool = False


def run_policy(policy, n_place_types, probs_every_step=False):
    """The cs_run_policy of cs_gpu_run for an InterventionPolicy (or None)."""
    p = abi.cs_run_policy()
    p.probs_every_step = int(bool(probs_every_step))
    if policy is not None:
        p.icu_trigger = 1
        p.icu_threshold = int(policy.threshold)
        p.icu_window = int(policy.window)
        p.case_isolation = int(bool(policy.case_isolation))
        p.household_quarantine = int(bool(policy.household_quarantine))
        p.social_distancing = int(bool(policy.social_distancing))
        p.close_place_types = sum(1 << pt for pt in set(policy.close_place_types) if 0 <= pt < n_place_types)
        p.per_adunit = int(bool(policy.per_adunit))
        p.duration = float(policy.duration)
    return p


class Simulation:
    def __init__(self, pop, params, lookup, hires, backend=None, device=0):
        self.pop = pop
        self.params = params
        self._pop_c = pop.to_c(lookup, hires)
        self.backend = backend(self._pop_c, params) if backend else GpuBackend(self._pop_c, params, device)

    def close(self):
        self.backend.close()

    def replica(self, params=None):
        """A Simulation of another realisation of this population that shares its
        static device arrays; `params` (same geometry) may differ, e.g. in LocalBeta."""
        other = Simulation.__new__(Simulation)
        other.pop = self.pop
        other.params = params if params is not None else self.params
        other._pop_c = self._pop_c
        other.backend = type(self.backend).replica(self.backend)
        if params is not None:
            other.backend.set_params(params)
        return other

    def choose_seeds(self, seed, n_seed):
        """SeedInfection with random locations: uniformly chosen people (the
        reference picks a person, then a member of that person's microcell)."""
        rng = np.random.default_rng(seed ^ 0x5EED)
        return rng.choice(self.pop.n_people, size=n_seed, replace=False).astype(np.int32)

    def run(self, seed, days, n_seed=100, policy=None, sample_every_day=True, callback=None, initial_state=None,
            probs_every_step=False, device_loop=None, blocks=False):
        """One realisation; returns daily time series of the main counters.

        initial_state: a cs_state_view of host arrays holding a prepared start
        (InitModel + SeedInfection already applied); it is copied to the device
        instead of resetting and seeding there.
        probs_every_step: test the susceptible fraction for UpdateProbs after every
        timestep, as the reference does, rather than at day ends.
        device_loop: run the logic between timesteps on the device (cs_gpu_run), one
        host round trip per run; the default uses it whenever the backend has it, the
        run has whole days and there is no per-day callback.  Results are the same.
        blocks: also return the whole counter block at t = 0 and at each day's end
        (int64 [days + 1, sizeof(cs_counters) / 8]), as `(series, blocks)`; the
        reference's output tables are made from them (covidsim_b200.output)."""
        be = self.backend
        if initial_state is not None:
            be.upload(seed, initial_state)
        else:
            be.begin_run(seed, self.choose_seeds(seed, n_seed))
        rs = _RunState(self, days, policy, callback, probs_every_step)
        first = counter_block(be.counters()) if blocks else None
        whole = rs.nsteps == int(days) * rs.spd and float(days) == int(days)
        if device_loop is None:
            device_loop = hasattr(be, "run_device") and callback is None and whole
        if device_loop:
            if not whole or callback is not None:
                raise ValueError("the device run loop takes whole days and no callback")
            daily = be.run_device(int(days), run_policy(policy, self.pop.num_place_types, probs_every_step))
            series = {k: daily[:, _COUNTER_INDEX[k]].copy() for k in SERIES}
            return (series, np.vstack([first[None], daily])) if blocks else series
        rs.keep_blocks = blocks
        for step in range(rs.nsteps):
            be.step(step * self.params.ModelTimeStep, 0)
            rs.after_step(step)
        if blocks:
            return rs.result(), np.vstack([first[None]] + rs.blocks)
        return rs.result()

    def _switch_interventions(self, t, policy, on, socd):
        iv = abi.cs_interventions()
        big = 1e10
        iv.CaseIsolationTimeStart = t if (on and policy.case_isolation) else big
        iv.CaseIsolationPolicyDuration = policy.duration
        iv.HQuarantineTimeStart = t if (on and policy.household_quarantine) else big
        iv.HQuarantinePolicyDuration = policy.duration
        socd[:] = abi.CS_TREAT_TREATED if (on and policy.social_distancing) else abi.CS_TREAT_UNTREATED
        iv.mcell_socdist = socd.ctypes.data
        iv.mcell_moverest = None
        self.backend.set_interventions(iv)
        if on:
            ts = int(t * self.params.TimeStepsPerDay)
            stop = min(65533, ts + int(policy.duration * self.params.TimeStepsPerDay))
            for pt in policy.close_place_types:
                if pt < self.pop.num_place_types:
                    self.backend.close_places(pt, None, ts, stop)


SERIES = ("S", "L", "I", "R", "D", "cumI", "cumC", "cumDC", "Critical", "cumCritical",
          "cumDeath_Critical", "cumDeath_SARI", "cumDeath_ILI", "SARI", "ILI", "Mild")
_COUNTER_INDEX = {k: getattr(abi.cs_counters, k).offset // 8 for k in SERIES}


def counter_block(c):
    """A cs_counters as its int64 words (every field of the block is int64)."""
    return np.frombuffer(bytes(c), dtype=np.int64).copy()


class _RunState:
    """Host side of one realisation between timesteps (src/CovidSim.cpp:1480-1530):
    daily counters, UpdateProbs when the susceptible fraction has fallen by 0.2,
    and the global ICU trigger switching interventions on and off."""

    def __init__(self, sim, days, policy, callback, probs_every_step=False):
        self.sim, self.policy, self.callback = sim, policy, callback
        self.every_step = probs_every_step
        P = sim.params
        self.spd = int(round(P.TimeStepsPerDay))
        self.nsteps = int(days * self.spd)
        self.prev_prop_s = 1.0
        self.series = {k: [] for k in SERIES}
        self.keep_blocks, self.blocks = False, []
        self.iv_on_until = -1.0
        self.iv_started = False
        self.socd = np.zeros(sim.pop.n_mcells, dtype=np.uint8)
        if policy is not None and policy.per_adunit:
            na = min(max(sim.pop.n_adunits, 1), abi.CS_MAX_ADUNITS)
            self.ad_started = np.zeros(na, bool)
            self.ad_on_until = np.full(na, -1.0)
            self.ad_ci = np.full(max(sim.pop.n_adunits, 1), 1e10)
            self.ad_hq = np.full(max(sim.pop.n_adunits, 1), 1e10)
            self.ad_cum = []
            self.ad_mcells = [np.nonzero(sim.pop.mcell_adunit == a)[0].astype(np.int32) for a in range(na)]

    def after_step(self, step):
        day_end = (step + 1) % self.spd == 0 or step == self.nsteps - 1
        if not (day_end or self.every_step):
            return
        sim, be, P, policy = self.sim, self.sim.backend, self.sim.params, self.policy
        series = self.series
        t = step * P.ModelTimeStep
        c = be.counters()
        if day_end:
            for k in series:
                series[k].append(int(getattr(c, k)))
            if self.keep_blocks:
                self.blocks.append(counter_block(c))
        prop_s = c.S / sim.pop.n_people
        if self.prev_prop_s - prop_s > 0.2:
            self.prev_prop_s = prop_s
            be.update_probs(0)
        if not day_end:
            return
        if policy is not None and policy.per_adunit:
            self._per_adunit(c, t + P.ModelTimeStep)
        elif policy is not None:
            day = len(series["cumCritical"])
            w = policy.window
            recent = series["cumCritical"][-1] - (series["cumCritical"][-w - 1] if day > w else 0)
            tn = t + P.ModelTimeStep
            if not self.iv_started and recent >= policy.threshold:
                self.iv_started = True
                self.iv_on_until = tn + policy.duration
                sim._switch_interventions(tn, policy, True, self.socd)
            elif self.iv_started and self.iv_on_until > 0 and tn >= self.iv_on_until:
                self.iv_on_until = -1.0
                sim._switch_interventions(tn, policy, False, self.socd)
        if self.callback:
            self.callback(step, c)

    def _per_adunit(self, c, tn):
        """One trigger per admin unit on its own critical-care admissions over the
        window (src/CovidSim.cpp:3442-3446 trigDC_adunit with ICU triggers), firing
        when they exceed the threshold (src/Sweep.cpp:1478-1482); a switch sets that
        unit's windows and microcells and closes its places."""
        sim, policy, P = self.sim, self.policy, self.sim.params
        na = len(self.ad_started)
        cum = np.array(c.cumCritical_adunit[:na], dtype=np.int64)
        self.ad_cum.append(cum)
        w = policy.window
        recent = cum - (self.ad_cum[-w - 1] if len(self.ad_cum) > w else 0)
        switched, closing = False, []
        for a in range(na):
            sw = -1
            if not self.ad_started[a] and recent[a] > policy.threshold:
                self.ad_started[a] = True
                self.ad_on_until[a] = tn + policy.duration
                sw = 1
            elif self.ad_started[a] and self.ad_on_until[a] > 0 and tn >= self.ad_on_until[a]:
                self.ad_on_until[a] = -1.0
                sw = 0
            if sw < 0:
                continue
            switched = True
            self.ad_ci[a] = tn if (sw and policy.case_isolation) else 1e10
            self.ad_hq[a] = tn if (sw and policy.household_quarantine) else 1e10
            self.socd[self.ad_mcells[a]] = abi.CS_TREAT_TREATED if (sw and policy.social_distancing) else abi.CS_TREAT_UNTREATED
            if sw:
                closing.append(a)
        if not switched:
            return
        iv = abi.cs_interventions()
        iv.CaseIsolationTimeStart = iv.HQuarantineTimeStart = 1e10
        iv.CaseIsolationPolicyDuration = iv.HQuarantinePolicyDuration = policy.duration
        iv.mcell_socdist = self.socd.ctypes.data
        iv.mcell_moverest = None
        iv.adunit_CaseIsolationTimeStart = self.ad_ci.ctypes.data
        iv.adunit_HQuarantineTimeStart = self.ad_hq.ctypes.data
        sim.backend.set_interventions(iv)
        ts = int(tn * P.TimeStepsPerDay)
        stop = min(65533, ts + int(policy.duration * P.TimeStepsPerDay))
        for a in closing:
            for pt in policy.close_place_types:
                if pt < sim.pop.num_place_types:
                    sim.backend.close_places(pt, self.ad_mcells[a], ts, stop)

    def result(self):
        return {k: np.asarray(v) for k, v in self.series.items()}


class Batch:
    """Realisations advanced together: one cs_gpu_batch_step per timestep launches
    one CUDA graph whose kernels each run the step's work of every member.  Members are Simulations (replicas of one population via
    Simulation.replica(), or of different populations); each keeps its own host
    logic (daily counters, UpdateProbs, interventions)."""

    def __init__(self, sims):
        self.sims = list(sims)
        self.lib = abi.load_library()
        ctxs = (C.c_void_p * len(self.sims))(*[s.backend.ctx for s in self.sims])
        self.handle = C.c_void_p()
        rc = self.lib.cs_gpu_batch_create(ctxs, len(self.sims), C.byref(self.handle))
        if rc != 0:
            msg = self.lib.cs_gpu_batch_last_error(self.handle)
            self.lib.cs_gpu_batch_destroy(self.handle)
            self.handle = None
            raise abi.CovidSimError("cs_gpu_batch_create: %s" % msg.decode())

    def _ck(self, rc, what):
        if rc != 0:
            raise abi.CovidSimError("cs_gpu_batch_%s: %s" % (what, self.lib.cs_gpu_batch_last_error(self.handle).decode()))

    def step(self, t, run=0):
        self._ck(self.lib.cs_gpu_batch_step(self.handle, t, run), "step")

    def set_grid(self, blocks):
        self._ck(self.lib.cs_gpu_batch_set_grid(self.handle, blocks), "set_grid")

    def set_spatial_lanes(self, lanes):
        self._ck(self.lib.cs_gpu_batch_set_spatial_lanes(self.handle, lanes), "set_spatial_lanes")

    def sync(self):
        self._ck(self.lib.cs_gpu_batch_sync(self.handle), "sync")

    def stream(self):
        return self.lib.cs_gpu_batch_stream(self.handle)

    def run(self, seeds, days, n_seed=100, policy=None, callback=None, probs_every_step=False, device_loop=None,
            blocks=False):
        """One realisation per member (member k with run seed seeds[k] and, when
        `policy` is a list, policy[k]); returns the members' daily series.
        device_loop as Simulation.run: by default the logic between timesteps runs
        on the device (cs_gpu_batch_run) whenever there is no callback and the run
        has whole days.  probs_every_step may be a list (one flag per member).
        blocks: also return each member's counter blocks at t = 0 and every day's
        end, as `(series, blocks)` (Simulation.run; output.write_summary averages
        them over the members)."""
        states, firsts = [], []
        policies = policy if isinstance(policy, (list, tuple)) else [policy] * len(self.sims)
        every = probs_every_step if isinstance(probs_every_step, (list, tuple)) else [probs_every_step] * len(self.sims)
        for sim, seed, pol, ev in zip(self.sims, seeds, policies, every):
            sim.backend.begin_run(seed, sim.choose_seeds(seed, n_seed))
            if blocks:
                firsts.append(counter_block(sim.backend.counters()))
            cb = (lambda step, c, k=len(states): callback(k, step, c)) if callback else None
            states.append(_RunState(sim, days, pol, cb, ev))
            states[-1].keep_blocks = blocks
        whole = float(days) == int(days) and all(rs.nsteps == int(days) * rs.spd for rs in states)
        if device_loop is None:
            device_loop = callback is None and whole
        if device_loop:
            if not whole or callback is not None:
                raise ValueError("the device run loop takes whole days and no callback")
            n, nd = len(self.sims), int(days)
            pols = (abi.cs_run_policy * n)(*[run_policy(p, s.pop.num_place_types, ev)
                                             for p, s, ev in zip(policies, self.sims, every)])
            out = np.empty((n, max(nd, 1), C.sizeof(abi.cs_counters) // 8), np.int64)
            self._ck(self.lib.cs_gpu_batch_run(self.handle, nd, C.addressof(pols), out.ctypes.data), "run")
            series = [{k: out[j, :nd, _COUNTER_INDEX[k]].copy() for k in SERIES} for j in range(n)]
            if blocks:
                return series, [np.vstack([firsts[j][None], out[j, :nd]]) for j in range(n)]
            return series
        nsteps = max(rs.nsteps for rs in states)
        dt = self.sims[0].params.ModelTimeStep
        for step in range(nsteps):
            self.step(step * dt, 0)
            for rs in states:
                rs.after_step(step)
        series = [rs.result() for rs in states]
        if blocks:
            return series, [np.vstack([f[None]] + rs.blocks) for f, rs in zip(firsts, states)]
        return series

    def close(self):
        if self.handle:
            self.lib.cs_gpu_batch_destroy(self.handle)
            self.handle = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass
