"""Regenerate the golden ensembles: 200 realisations of the reference executable
(oracle/_ref/CovidSim, built from the reference sources) on a workload of
oracle/ensemble.py, summarised as final sizes, peak days and ensemble-mean daily
curves.

    python tests/golden/make_ref_ensemble.py [plain|interventions|holidays|medium]

writes tests/golden/ref_ensemble.json (plain, the default), ref_ensemble_iv.json,
ref_ensemble_hol.json or ref_ensemble_200k.json;
CS_THREADS sets the reference's thread count (default: every core)."""
import json
import os
import sys

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(os.path.dirname(HERE))
sys.path.insert(0, os.path.join(ROOT, "oracle"))


def main():
    import ensemble
    config = sys.argv[1] if len(sys.argv) > 1 else "plain"
    threads = int(os.environ.get("CS_THREADS", "0")) or None
    summary, res = ensemble.run(os.path.join(ROOT, "oracle", "_ref", "CovidSim"), config=config, threads=threads)
    summary["threads"] = res["threads"]
    summary["config"] = ensemble.CONFIGS[config]
    with open(os.path.join(HERE, ensemble.GOLDEN[config]), "w") as f:
        json.dump(summary, f, separators=(",", ":"))
    print("realisations", summary["n"], "mean final size", sum(summary["final_size"]) / summary["n"],
          "wall %.1fs" % res["wall"])


if __name__ == "__main__":
    sys.exit(main())
