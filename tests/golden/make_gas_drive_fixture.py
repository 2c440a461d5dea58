"""Writes tests/golden/gas_drive_case.json from the reference's own three-phase acceptance test.

src/lib/ressim/src/tests/three_phase_acceptance.rs grades the solution-gas-drive depletion case
(`make_gas_drive_acceptance_sim`, PVT rows `gas_drive_pvt_rows`) against an OPM Flow solution
(`OPM_GAS_DRIVE`: time, field pressure, oil rate, cumulative oil, GOR) with the tolerances of
`three_phase_gas_drive_matches_opm_flow_reference`; docs/THREE_PHASE_VALIDATION.md records the
errors the reference's engine printed on that test.  This script reads both as text and stores
those items unchanged as a fixture.

    python tests/golden/make_gas_drive_fixture.py <reference root>
"""
from __future__ import annotations

import json
import os
import re
import sys

sys.path.insert(0, os.path.dirname(os.path.abspath(__file__)))
from make_spe1_fixture import arg, reference_root, split_top  # noqa: E402

OUT = os.path.join(os.path.dirname(os.path.abspath(__file__)), "gas_drive_case.json")


def main() -> None:
    root = reference_root()
    text = open(os.path.join(root, "src/lib/ressim/src/tests/three_phase_acceptance.rs")).read()
    consts = {k: float(v.replace("_", "")) for k, v in re.findall(r"const (\w+): f64 = ([-\d._eE+]+);", text)}
    rows_body = re.search(r"fn gas_drive_pvt_rows\(\).*?const ROWS: \[.*?\] = \[(.*?)\];", text, re.S).group(1)
    pvt = [[float(v) for v in t.split(",")] for t in re.findall(r"\(([^()]*)\)", rows_body)]
    start = text.index("fn make_gas_drive_acceptance_sim()")
    body = text[start:text.index("\nfn ", start + 10)]
    nx, ny, nz, phi = re.search(r"ReservoirSimulator::new\((\d+), (\d+), (\d+), ([\d.]+)\)", body).groups()
    ops = []
    for m in re.finditer(r"\bsim\.(\w+)(?:\((.*?)\)\s*(?:\.unwrap\(\))?|\s*=\s*(.*?));", body, re.S):
        name, call_args, value = m.groups()
        if call_args is not None:
            ops.append(["call", name, [arg(t, consts) for t in split_top(call_args)]])
        else:
            ops.append(["set", name, value.strip()])
    data = re.search(r"const OPM_GAS_DRIVE: \[.*?\] = \[(.*?)\];", text, re.S).group(1)
    series = [[float(v) for v in t.split(",")] for t in re.findall(r"\(([^()]*)\)", data)]
    test = text[text.index("fn three_phase_gas_drive_matches_opm_flow_reference()"):]
    max_dt = float(re.search(r"step_to\(&mut sim, t_days, ([\d.]+)\)", test).group(1))
    # the errors the reference's own engine printed for this test (docs/THREE_PHASE_VALIDATION.md)
    doc = open(os.path.join(root, "docs/THREE_PHASE_VALIDATION.md")).read()
    recorded = []
    for m in re.finditer(r"t=\s*([\d.]+) pressure_err=\s*([\d.]+)% oil_rate_err=\s*([\d.]+%|--) "
                         r"cum_oil_err=\s*([\d.]+)% gor_err=\s*([\d.]+)%", doc):
        t, pe, qe, ce, ge = m.groups()
        recorded.append([float(t), float(pe), None if qe == "--" else float(qe[:-1]), float(ce), float(ge)])
    fixture = {
        "source": "src/lib/ressim/src/tests/three_phase_acceptance.rs",
        "grid": [int(nx), int(ny), int(nz)],
        "porosity": float(phi),
        "pvt_rows": pvt,
        "ops": ops,
        "opm_series": series,
        "series_columns": ["t_days", "pressure_bar", "oil_rate_sc_day", "cumulative_oil_sc", "gor"],
        "max_dt_days": max_dt,
        "recorded_errors_percent": recorded,
        "recorded_columns": ["t_days", "pressure", "oil_rate", "cumulative_oil", "gor"],
        "recorded_source": "docs/THREE_PHASE_VALIDATION.md (the reference engine's printed errors)",
        "scalars": {k: v for k, v in consts.items() if k.startswith("GAS_DRIVE_")},
    }
    with open(OUT, "w") as fh:
        json.dump(fixture, fh, indent=1)
        fh.write("\n")
    print(f"wrote {OUT}: {len(pvt)} PVT rows, {len(ops)} ops, {len(series)} OPM points")


if __name__ == "__main__":
    main()
