"""Whole epidemics through the reference's own executable: the reference host code
(set-up, InitModel, SeedInfection, RecordSample, TreatSweep, output files) with its
sweeps replaced -- by the CPU oracle (oracle/_ref/CovidSim_oracle) or by the GPU
library (oracle/_ref/CovidSim_b200) -- against 200 realisations of the unmodified
reference (tests/golden/ref_ensemble*.json, made by tests/golden/make_ref_ensemble.py).
Two-sample KS on final size and peak day (p > 0.01); ensemble-mean daily
incidence, critical-care and death curves within 2 standard errors on at least
90% of days.

Three workloads (oracle/ensemble.py): `plain`; `holidays`, the plain one with a
30-day holiday closing every school and university; and `interventions`, where the
reference's own trigger logic and TreatSweep switch case isolation, household
quarantine, social distancing and place closure on and the drop-in's sweeps consume
what they decided.  The drop-in runs with the host thread count the reference ran
with: the reference's host code, which the drop-in keeps, gives thread-count-
dependent results (its per-thread random streams), and with interventions that
moves the final-size distribution measurably (mean 7,797 with 8 threads, 8,108 with
7, over 200 realisations each)."""
import json
import os

import pytest

import ensemble

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


def _gold(config):
    return json.load(open(os.path.join(ROOT, "tests", "golden", ensemble.GOLDEN[config])))


def _run(binary, config, nr=None):
    return ensemble.run(binary, config=config, threads=_gold(config)["threads"], nr=nr)


def _check(summary, config):
    gold = _gold(config)
    assert gold["config"] == ensemble.CONFIGS[config], "golden file of another workload"
    cmp = ensemble.compare(summary, gold)
    assert cmp["ks_final_size_p"] > 0.01, cmp
    assert cmp["ks_peak_day_p"] > 0.01, cmp
    for key in ("inc", "crit", "deaths"):
        assert cmp[key + "_within_2se"] >= 0.90, cmp
    return cmp


def _binary(name):
    path = os.path.join(ROOT, "oracle", "_ref", name)
    if not os.path.exists(path):
        pytest.skip("%s not built (needs the reference checkout at build time)" % name)
    return path


@pytest.mark.slow
def test_oracle_sweep_in_reference_matches_reference():
    summary, _ = _run(_binary("CovidSim_oracle"), "plain")
    _check(summary, "plain")


@pytest.mark.slow
def test_oracle_sweep_with_interventions_matches_reference():
    summary, _ = _run(_binary("CovidSim_oracle"), "interventions")
    _check(summary, "interventions")


@pytest.mark.slow
def test_oracle_sweep_with_holidays_matches_reference():
    summary, _ = _run(_binary("CovidSim_oracle"), "holidays")
    _check(summary, "holidays")


@pytest.mark.gpu
def test_gpu_sweep_in_reference_matches_reference():
    summary, res = _run(_binary("CovidSim_b200"), "plain")
    _check(summary, "plain")
    assert any("people" in ln for ln in res["dropin"]), res["dropin"]


@pytest.mark.gpu
def test_gpu_sweep_with_interventions_matches_reference():
    summary, res = _run(_binary("CovidSim_b200"), "interventions")
    _check(summary, "interventions")
    assert any("people" in ln for ln in res["dropin"]), res["dropin"]


@pytest.mark.gpu
def test_gpu_sweep_with_holidays_matches_reference():
    summary, res = _run(_binary("CovidSim_b200"), "holidays")
    _check(summary, "holidays")
    assert any("people" in ln for ln in res["dropin"]), res["dropin"]


@pytest.mark.gpu
def test_gpu_sweep_at_200k_people_matches_reference():
    """200,000 people at the 1M workload's cell density with the interventions, 100
    realisations against 200 of the reference on the same network file (the
    comparisons' standard errors take each side's count)."""
    summary, res = _run(_binary("CovidSim_b200"), "medium", nr=100)
    _check(summary, "medium")
    assert any("people" in ln for ln in res["dropin"]), res["dropin"]
