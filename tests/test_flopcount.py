"""The FP64 operation counts per cell update that bench.py's FP-pipe roofline
uses are those of the instrumented build of the oracle (oracle/flopcount.cpp),
and the count follows the reference's operation structure: more ghost-region
work per interior cell at smaller mx, clawpack 5's narrower flux ranges cost
less than clawpack 4.6's."""
import json
import subprocess
import sys
from pathlib import Path

ROOT = Path(__file__).resolve().parents[1]


def _counts():
    subprocess.run(["make", "-s", "-C", str(ROOT / "oracle"), "flopcount"], check=True)
    out = subprocess.run([str(ROOT / "oracle" / "flopcount")], check=True, capture_output=True, text=True).stdout
    return [json.loads(l) for l in out.splitlines() if l.strip()]


def test_bench_constants_match_the_counting_build():
    sys.path.insert(0, str(ROOT))
    import bench

    rows = _counts()
    by = {(r["case"], r["mx"], r["claw_version"]): r for r in rows}
    for (case, mx), ops in bench.FP64_OPS_PER_CELL.items():
        assert abs(by[(case, mx, 4)]["ops_per_cell"] - ops) < 1e-3, (case, mx)


def test_count_structure():
    rows = _counts()
    by = {(r["case"], r["mx"], r["claw_version"]): r for r in rows}
    adv = [by[("advection_swirl_order22", mx, 4)]["ops_per_cell"] for mx in (8, 16, 32)]
    assert adv[0] > adv[1] > adv[2]
    assert by[("advection_swirl_order22", 16, 5)]["ops_per_cell"] < by[("advection_swirl_order22", 16, 4)]["ops_per_cell"]
    eul = [by[("euler4_roe_order22", mx, 4)]["ops_per_cell"] for mx in (8, 16, 32, 64)]
    assert eul == sorted(eul, reverse=True)
    # the Roe solvers take square roots; advection takes none
    assert by[("swe_roe_order22", 32, 4)]["sqrt"] > 0 and by[("advection_swirl_order22", 16, 4)]["sqrt"] == 0
    # every row sums its parts
    for r in rows:
        assert abs(r["ops_per_cell"] - (r["add"] + r["mul"] + r["div"] + r["sqrt"] + r["cmp"])) < 1e-2
