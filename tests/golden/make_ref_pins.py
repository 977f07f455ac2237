"""Regenerate tests/golden/ref_pins.json from the reference's own functions.

Builds oracle/_ref/ref_pins (oracle/Makefile: the reference's Kernels.cpp,
Dist.cpp, InverseCdf.cpp, CalcInfSusc.cpp, Person.cpp and Rand.cpp compiled from the
reference checkout, plus oracle/ref_pins.cpp) and stores its JSON output.  Needs the
reference checkout, named by the REF environment variable
(REF=<path of the reference checkout> python tests/golden/make_ref_pins.py); the tests
only read the committed JSON.
"""
import json
import os
import subprocess
import sys

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(os.path.dirname(HERE))


def main():
    if not os.environ.get("REF"):
        sys.exit("set REF=<path of the reference checkout>")
    subprocess.run(["make", "-s", "-C", os.path.join(ROOT, "oracle"), "pins", "REF=" + os.environ["REF"]], check=True)
    out = subprocess.run([os.path.join(ROOT, "oracle", "_ref", "ref_pins")], check=True, capture_output=True, text=True).stdout
    data = json.loads(out)
    with open(os.path.join(HERE, "ref_pins.json"), "w") as f:
        json.dump(data, f, separators=(",", ":"))
    print("wrote", os.path.join(HERE, "ref_pins.json"), "keys", sorted(data))


if __name__ == "__main__":
    sys.exit(main())
