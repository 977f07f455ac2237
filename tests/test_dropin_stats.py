"""Whole epidemics through the reference's own executable: the reference host code
(set-up, InitModel, SeedInfection, RecordSample, output files) with its sweeps
replaced -- by the CPU oracle (oracle/_ref/CovidSim_oracle) or by the GPU library
(oracle/_ref/CovidSim_b200) -- against 200 realisations of the unmodified reference
(tests/golden/ref_ensemble.json, made by tests/golden/make_ref_ensemble.py).
Two-sample KS on final size and peak day (p > 0.01); ensemble-mean daily
incidence, critical-care and death curves within 2 standard errors on at least
90% of days."""
import json
import os

import pytest

import ensemble

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
GOLD = json.load(open(os.path.join(ROOT, "tests", "golden", "ref_ensemble.json")))


def _check(summary):
    cmp = ensemble.compare(summary, GOLD)
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
    summary, _ = ensemble.run(_binary("CovidSim_oracle"))
    _check(summary)


@pytest.mark.gpu
def test_gpu_sweep_in_reference_matches_reference():
    summary, res = ensemble.run(_binary("CovidSim_b200"))
    assert "GPU sweep:" in res["stderr"] or summary["n"] == GOLD["n"]
    _check(summary)
