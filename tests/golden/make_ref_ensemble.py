"""Regenerate tests/golden/ref_ensemble.json: 200 realisations of the reference
executable (oracle/_ref/CovidSim, built from the reference sources) on the
20,000-person synthetic population of oracle/ensemble.py, summarised as final
sizes, peak days and ensemble-mean daily curves."""
import json
import os
import sys

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(os.path.dirname(HERE))
sys.path.insert(0, os.path.join(ROOT, "oracle"))


def main():
    import ensemble
    summary, res = ensemble.run(os.path.join(ROOT, "oracle", "_ref", "CovidSim"))
    summary["threads"] = res["threads"]
    summary["config"] = ensemble.CONFIG
    with open(os.path.join(HERE, "ref_ensemble.json"), "w") as f:
        json.dump(summary, f, separators=(",", ":"))
    print("realisations", summary["n"], "mean final size", sum(summary["final_size"]) / summary["n"],
          "wall %.1fs" % res["wall"])


if __name__ == "__main__":
    sys.exit(main())
