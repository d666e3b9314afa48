"""Regenerates tests/golden/d3q19_equilibrium.json from the reference.

Run where the reference tree is available, giving its path
as the argument or in $GPU_SIMS_REFERENCE:

    python tests/golden/make_golden.py <reference tree>

It imports the reference's own D3Q19 verifier
(tools/integrity/integrity/cat3_numerical/d3q19_verify.py), runs its three
verification passes against the reference's committed expected-values file
(d3q19_equilibrium.expected.json, produced by d3q19_verify.py:201-357), and
writes those values (velocity set, weights, opposite index, feq and moment
sums at the four test points) plus a re-evaluation through the verifier's
own feq() as the fixture.  Nothing here is needed at test time.
"""
from __future__ import annotations

import json
import os
import sys
from pathlib import Path

def _reference_root() -> Path:
    """The reference tree: the first argument, else $GPU_SIMS_REFERENCE."""
    arg = sys.argv[1] if len(sys.argv) > 1 else os.environ.get("GPU_SIMS_REFERENCE")
    if not arg:
        raise SystemExit("give the reference tree's path as the argument or in $GPU_SIMS_REFERENCE")
    return Path(arg)
OUT = Path(__file__).resolve().parent / "d3q19_equilibrium.json"


def main() -> int:
    REF = _reference_root()
    sys.path.insert(0, str(REF / "tools" / "integrity"))
    from integrity.cat3_numerical import d3q19_verify as v  # noqa: E402

    payload = v.load_expected_payload()
    errs = v.verify_velocity_set(payload) + v.verify_weights(payload) + v.verify_equilibrium(payload)
    if errs:
        print("reference verifier reports:", *errs, sep="\n  ")
        return 1
    cs = v.build_velocity_set()
    ws = [float(v.weight_for(c)) for c in cs]
    points = []
    for tp in payload["test_points"]:
        ux, uy, uz = tp["u"]
        points.append({
            "name": tp["name"], "rho": tp["rho"], "u": tp["u"],
            "feq": tp["feq"], "sums": tp["sums"],
            "feq_reevaluated": v.feq(tp["rho"], ux, uy, uz, cs, ws),
        })
    out = {
        "generated_by": "tests/golden/make_golden.py",
        "reference_files": [
            "tools/integrity/integrity/cat3_numerical/d3q19_verify.py",
            "tools/integrity/integrity/cat3_numerical/d3q19_equilibrium.expected.json",
        ],
        "tolerance_abs": v.TOL_ABS,
        "velocity_set": [list(c) for c in cs],
        "weights": ws,
        "opposite_index": [v.opposite_index(i, cs) for i in range(19)],
        "test_points": points,
    }
    OUT.write_text(json.dumps(out, indent=1) + "\n")
    print(f"wrote {OUT}")
    return 0


if __name__ == "__main__":
    sys.exit(main())
