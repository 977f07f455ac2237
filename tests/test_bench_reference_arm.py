"""bench.py's reference arm on the host: it times at most three realisations whatever
K is, says how many it timed, and prints the line the contract asks for (impl,
cpu_baseline, an e2e block with no copies).  The reference run itself is replaced by
a stand-in that records what it was asked for."""
import argparse

import bench


def _args(steps, warmup=3, workload="c1_240"):
    return argparse.Namespace(steps=steps, warmup=warmup, workload=workload, gpus=1)


def test_reference_arm_caps_the_realisations_and_reports_them(monkeypatch):
    import sys
    sys.path.insert(0, bench.os.path.join(bench.ROOT, "oracle"))
    import refrun
    asked = {}

    def fake_time_reference(workload, steps=3, warmup=3, **kw):
        asked.update(workload=workload, steps=steps, warmup=warmup)
        return {"value": 1.4e9, "ms_per_step": 10000.0, "cores": 16, "sample": "stand-in", "rows": [],
                "wall": 60.0, "network_file": "x.net", "run_loop_ms_per_step": 38000.0}

    monkeypatch.setattr(refrun, "time_reference", fake_time_reference)
    monkeypatch.delenv("RANK", raising=False)
    line = bench.run_reference(_args(20))
    assert asked == {"workload": "c1_240", "steps": bench.REF_MAX_STEPS, "warmup": 1}
    assert line["impl"] == "reference" and line["steps"] == bench.REF_MAX_STEPS and line["steps_requested"] == 20
    assert line["value"] == 1.4e9 and line["higher_is_better"] is True
    assert line["cpu_baseline"]["kind"] == "reference" and line["cpu_baseline"]["cores"] == 16
    assert line["e2e"] == {"value": 1.4e9, "unit": bench.METRIC, "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0}
    assert line["config"]["run_loop_ms_per_step"] == 38000.0
    # fewer realisations than the cap are taken as asked
    line = bench.run_reference(_args(2, warmup=0))
    assert asked["steps"] == 2 and asked["warmup"] == 0 and line["steps"] == 2


def test_reference_arm_reports_an_unavailable_reference(monkeypatch):
    import sys
    sys.path.insert(0, bench.os.path.join(bench.ROOT, "oracle"))
    import refrun
    monkeypatch.setattr(refrun, "time_reference", lambda *a, **k: {"unavailable": "not built"})
    monkeypatch.delenv("RANK", raising=False)
    assert bench.run_reference(_args(5)) == {"impl": "reference", "unavailable": "not built"}


def test_other_ranks_print_nothing(monkeypatch):
    monkeypatch.setenv("RANK", "1")
    assert bench.run_reference(_args(5)) is None
