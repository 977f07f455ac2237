"""The timing lines the two arms' shims print at exit (oracle/ref_timing_shim.cpp for
the reference's sweeps, covid-sim_b200/shim/cs_sweep_shim.cpp for the drop-in) parse
into the rows bench.py's e2e and reference arms are formed from, and the drop-in's
parts come out per realisation."""
import refrun


REF = ("noise\nREFTIMING run=0 pop=10000000 threads=16 steps=1460 infect_s=7.250000 incub_s=2.600000 "
       "first_t=0.0000 last_t=364.7500 loop_s=38.390403\n"
       "REFTIMING run=1 pop=10000000 threads=16 steps=1417 infect_s=7.000000 incub_s=2.500000 "
       "first_t=0.0000 last_t=354.0000 loop_s=37.000000\n")

DROPIN = ("GPU sweep: 10000000 people, 57600 populated cells on device\n"
          "\nSWEEPTIMING run=1 pop=10000000 threads=16 steps=1417 infect_s=0.128530 incub_s=0.101310 "
          "upload_s=0.028767 copyback_s=0.037214 wait_s=0.064001 scatter_s=0.035796 handover_s=0.040200 "
          "mcell_scans=2 upload_device_s=0.002453 cell_bytes=2 loop_s=34.101217\n")


def test_reference_timing_lines():
    rows = refrun.parse_timing(REF)
    assert [r["run"] for r in rows] == [0, 1]
    assert rows[0]["pop"] == 10_000_000 and rows[0]["threads"] == 16 and rows[0]["steps"] == 1460
    assert abs(rows[0]["infect_s"] + rows[0]["incub_s"] - 9.85) < 1e-9
    assert abs(rows[0]["loop_s"] - 38.390403) < 1e-9
    assert rows[1]["last_t"] == 354.0


def test_dropin_timing_line_carries_its_parts():
    (r,) = refrun.parse_timing(DROPIN)
    assert r["steps"] == 1417
    for k, v in (("upload_s", 0.028767), ("copyback_s", 0.037214), ("wait_s", 0.064001),
                 ("scatter_s", 0.035796), ("handover_s", 0.0402), ("upload_device_s", 0.002453),
                 ("loop_s", 34.101217)):
        assert abs(r[k] - v) < 1e-12, k
    assert r["mcell_scans"] == 2 and r["cell_bytes"] == 2
    # the parts lie inside the sweep calls' time
    assert r["upload_device_s"] <= r["upload_s"] <= r["infect_s"] + r["incub_s"]
    assert r["scatter_s"] <= r["copyback_s"]
    assert r["infect_s"] + r["incub_s"] < r["loop_s"]
