"""Regenerate tests/golden/regression_pins.json from the reference tree.

The reference's regression tests pin three counters per run
(src/fclaw2d_finalize.c:140-197): count_amr_advance, global_num_patches and
count_amr_new_domain.  This script copies those numbers for the runs whose
configuration lies on this path (swirl, quadrants, bump and the periodic
2 x 2 brick with clawpack 4.6 and 5, radialdam example 0 with clawpack 4.6
and 5 and time-sync, filament example 1 (the cart-mapped 2 x 2 brick with
capacity) with clawpack 4.6 and 5), so the tests can check the oracle and the CUDA path without
the reference tree.

Usage: python tests/golden/make_pins.py REFERENCE_ROOT
"""
import csv
import json
import sys
from pathlib import Path


def read_csv(p: Path) -> dict:
    out = {}
    with open(p) as f:
        for row in csv.reader(f):
            if len(row) == 2:
                out[row[0]] = int(row[1])
    return out


RUNS = {
    "swirl": "applications/clawpack/advection/2d/swirl/regression_values_0.csv",
    "swirl_claw5": "applications/clawpack/advection/2d/swirl/regression_values_1.csv",
    "radialdam": "applications/clawpack/shallow/2d/radialdam/regression_values_0.csv",
    "radialdam_claw5": "applications/clawpack/shallow/2d/radialdam/regression_values_1.csv",
    "quadrants": "applications/clawpack/euler/2d/quadrants/regression_values_0.csv",
    "quadrants_claw5": "applications/clawpack/euler/2d/quadrants/regression_values_1.csv",
    "bump": "applications/clawpack/shallow/2d/bump/regression_values_0.csv",
    "bump_claw5": "applications/clawpack/shallow/2d/bump/regression_values_1.csv",
    "periodic": "applications/clawpack/advection/2d/periodic/regression_values_0.csv",
    "periodic_claw5": "applications/clawpack/advection/2d/periodic/regression_values_1.csv",
    "filament": "applications/clawpack/advection/2d/filament/regression_values_0.csv",
    "filament_claw5": "applications/clawpack/advection/2d/filament/regression_values_1.csv",
}


def main(ref: Path):
    pins = {name: {"source": src, "values": read_csv(ref / src)} for name, src in RUNS.items()}
    out = Path(__file__).with_name("regression_pins.json")
    out.write_text(json.dumps(pins, indent=1) + "\n")
    print(out)


if __name__ == "__main__":
    if len(sys.argv) != 2:
        sys.exit(__doc__)
    main(Path(sys.argv[1]))
