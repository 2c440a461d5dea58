"""Writes tests/golden/spe1_case.json from the reference's own SPE1 acceptance test.

The reference grades its black-oil FIM engine against the published SPE1 Case 1 series in
src/lib/ressim/src/tests/spe1_acceptance.rs (series, targets and tolerances) on the deck that
`make_spe1_like_grid_sim` builds in src/lib/ressim/src/lib.rs (PVT rows, SWOF/SGOF rows and
setter calls).  This script reads both files as text and stores what they hold, unchanged, as a
fixture, so that the tests can replay the acceptance check without the reference's sources.

    python tests/golden/make_spe1_fixture.py <reference root>
"""
from __future__ import annotations

import json
import os
import re
import sys

OUT = os.path.join(os.path.dirname(os.path.abspath(__file__)), "spe1_case.json")


def number(tok: str):
    tok = tok.strip().replace("_", "")
    try:
        return float(tok)
    except ValueError:
        return None


def split_top(s: str):
    out, depth, cur = [], 0, ""
    for ch in s:
        if ch in "([{":
            depth += 1
        elif ch in ")]}":
            depth -= 1
        if ch == "," and depth == 0:
            out.append(cur)
            cur = ""
        else:
            cur += ch
    if cur.strip():
        out.append(cur)
    return [a.strip() for a in out]


def arg(tok: str, consts: dict):
    m = re.fullmatch(r"vec!\[(.*)\]", tok, re.S)
    if m:
        return [arg(t, consts) for t in split_top(m.group(1))]
    m = re.fullmatch(r'"([^"]*)"(?:\.to_string\(\))?', tok)
    if m:
        return m.group(1)
    if tok in ("true", "false"):
        return tok == "true"
    if tok in consts:
        return consts[tok]
    v = number(tok)
    return v if v is not None else "$" + tok


def rows(text: str, kind: str, keys):
    out = []
    for body in re.findall(kind + r"\s*\{(.*?)\}", text, re.S):
        kv = dict(re.findall(r"(\w+):\s*(?:Some\()?([-\d._eE+]+)\)?", body))
        out.append([float(kv[k]) for k in keys])
    return out


def reference_root() -> str:
    """The reference checkout's root, the script's one required argument."""
    if len(sys.argv) != 2:
        sys.exit(f"usage: python {os.path.basename(sys.argv[0])} <reference root>")
    return sys.argv[1]


def main() -> None:
    src = os.path.join(reference_root(), "src/lib/ressim/src")
    lib = open(os.path.join(src, "lib.rs")).read()
    start = lib.index("fn make_spe1_like_grid_sim(")
    end = lib.index("fn make_spe1_like_sim(", start)
    helper = lib[start:end]
    consts = {k: float(v) for k, v in re.findall(r"const (\w+): f64 = ([-\d._eE+]+);", helper)}
    nz, phi = re.search(r"ReservoirSimulator::new\(nx, ny, (\d+), ([\d.]+)\)", helper).groups()
    domain = float(re.search(r"let cell_dx = ([\d.]+) / nx", helper).group(1))
    calls = []
    for name, body in re.findall(r"\bsim\.(\w+)\((.*?)\)\s*(?:\.unwrap\(\))?;", helper, re.S):
        calls.append([name, [arg(t, consts) for t in split_top(body)]])
    acc = open(os.path.join(src, "tests/spe1_acceptance.rs")).read()
    series = {}
    for name, body in re.findall(r"const (REF_\w+): \[\(f64, f64\); \d+\] = \[(.*?)\];", acc, re.S):
        series[name] = [[float(a), float(b)] for a, b in re.findall(r"\(([-\d.]+),\s*([-\d.]+)\)", body)]
    scalars = {k: number(v) for k, v in re.findall(r"const (\w+): f64 = ([-\d._eE+]+);", acc)}
    m = re.search(r"make_spe1_like_grid_sim\(\s*nx,\s*nx,\s*nx - 1,\s*nx - 1,\s*vec!\[(.*?)\],\s*([\d.]+),"
                  r"\s*([\d.]+),\s*([\d.]+),?\s*\)", acc, re.S)
    first = re.search(r"fn spe1_first_year_matches_published_reference\(\).*?step_to\(&mut sim, ([\d.]+), ([\d.]+)\)",
                      acc, re.S)
    fixture = {
        "source": ["src/lib/ressim/src/lib.rs (make_spe1_like_grid_sim)",
                   "src/lib/ressim/src/tests/spe1_acceptance.rs"],
        "nz": int(nz),
        "porosity": float(phi),
        "domain_m": domain,
        "pvt_rows": rows(helper, "PvtRow", ("p_bar", "rs_m3m3", "bo_m3m3", "mu_o_cp", "bg_m3m3", "mu_g_cp")),
        "swof": rows(helper, "SwofRow", ("sw", "krw", "krow")),
        "sgof": rows(helper, "SgofRow", ("sg", "krg", "krog")),
        "calls": calls,
        "acceptance_layer_perms_z": [float(v) for v in split_top(m.group(1))],
        "acceptance_stability": [float(m.group(2)), float(m.group(3)), float(m.group(4))],
        "first_year": {"t_days": float(first.group(1)), "max_dt_days": float(first.group(2))},
        "series": series,
        "scalars": scalars,
    }
    with open(OUT, "w") as fh:
        json.dump(fixture, fh, indent=1)
        fh.write("\n")
    print(f"wrote {OUT}: {len(fixture['pvt_rows'])} PVT rows, {len(fixture['swof'])} SWOF, "
          f"{len(fixture['sgof'])} SGOF, {len(calls)} calls, series {sorted(series)}")


if __name__ == "__main__":
    main()
