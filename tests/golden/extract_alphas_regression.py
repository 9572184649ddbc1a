"""Extract the fixture qex_alphas_regression_8x8x8x16.json from QEX's own
regression logs (src/alphas/regression/*/*.log in the QEX source tree).

Those logs are QEX's HISQ HMC (src/alphas/alphas.nim) run on an 8^3 x 16
lattice from a cold start (unit links), m = 0.005 with a Hasenbusch mass of
0.6, action solves to r2 <= 1e-20 |b|^2.  Before any molecular dynamics the
trajectory makes three full-lattice solves (stagSolve.nim:469-557) on the
HISQ-smeared cold field: the ratio pseudofermion's heatbath
(alphas.nim:722-745, D(-0.6)^-1 D(-0.005) eta) and the two terms of the
initial fermion action (alphas.nim:694-707, D(-0.6)^-1 phi and
D(-0.005)^-1 D(-0.6) hphi).  QEX prints each as
"stagSolve: <iterations> <time> <rate> <r2/b2>", then the Hamiltonian's
parts ("kinetic: .. gauge: .. fermion: ..").  This script reads the first
three such lines, the start-of-trajectory gauge and fermion actions and the
run parameters of every log, checks that all logs agree, and writes them
out.

  python tests/golden/extract_alphas_regression.py [QEX source root]
"""
from __future__ import annotations

import json
import re
import sys
from pathlib import Path

HERE = Path(__file__).resolve().parent


def parse(log: Path):
    text = log.read_text(errors="replace")
    geom = re.search(r"#physGeom:@\[([0-9, ]+)\]", text).group(1)
    params = {
        "lattice": [int(v) for v in geom.split(",")],
        "mass": float(re.search(r"^mass: (\S+)", text, re.M).group(1)),
        "hasenbusch_mass": float(re.search(r"^hasenbusch mass: (\S+)", text, re.M).group(1)),
        "gauge_start": re.search(r"^gauge start: (\S+)", text, re.M).group(1),
        "action_r2req": float(re.search(r"minimum squared residual \(action CG solver\): (\S+)", text).group(1)),
        "naik": float(re.search(r"^naik: (\S+)", text, re.M).group(1)),
    }
    # the Hamiltonian's parts at the start of the trajectory (alphas.nim:709-718)
    h0 = re.search(r"^kinetic: (\S+) gauge: (\S+) fermion: (\S+)", text, re.M)
    params["start_gauge_action"] = float(h0.group(2))
    params["start_fermion_action"] = float(h0.group(3))
    solves = re.findall(r"^stagSolve: (\d+)\s+\S+\s+\S+\s+(\S+)", text, re.M)
    # logs of runs over several processes interleave identical lines of
    # every process: keep the first occurrence of each (iterations, r2)
    seen, first = set(), []
    for its, r2 in solves:
        if (its, r2) not in seen:
            seen.add((its, r2))
            first.append({"iterations": int(its), "r2_over_b2": float(r2)})
        if len(first) == 3:
            break
    return params, first


DEFAULT_ROOT = Path("/root/reference")
FIXTURE = HERE / "qex_alphas_regression_8x8x8x16.json"


def extract(root: Path = DEFAULT_ROOT) -> dict:
    """The fixture's content, read from the logs under root."""
    logs = sorted((root / "src/alphas/regression").glob("*/*.log"))
    assert logs, f"no regression logs under {root}"
    runs = [(log, *parse(log)) for log in logs]
    params, solves = runs[0][1], runs[0][2]
    actions = [p.pop("start_fermion_action") for _, p, _ in runs]
    for log, p, s in runs:
        assert p == params, (log, p)
        assert [x["iterations"] for x in s] == [x["iterations"] for x in solves], (log, s)
    # the final residuals differ in the last digits between thread and
    # process counts (summation order): keep their range
    for k, sv in enumerate(solves):
        r2s = [s[k]["r2_over_b2"] for _, _, s in runs]
        sv["r2_over_b2"] = [min(r2s), max(r2s)]
    # S_F = (|psi|^2 + |hpsi|^2) / 2 after those solves (alphas.nim:694-707),
    # equal across the logs up to summation order
    params["start_fermion_action"] = [min(actions), max(actions)]
    out = {
        "source": "QEX src/alphas/regression/*/*.log: the first three stagSolve lines and the "
                  "start-of-trajectory action of each run",
        "logs": [str(log.relative_to(root)) for log in logs],
        "params": params,
        "solves": [
            {"what": "heatbath of the ratio pseudofermion: D(-hmass)^-1 D(-mass) eta (alphas.nim:722-745)",
             **solves[0]},
            {"what": "action, heavy term: D(-hmass)^-1 phi, phi odd half zero (alphas.nim:702)", **solves[1]},
            {"what": "action, ratio term: D(-mass)^-1 D(-hmass) hphi, hphi odd half zero (alphas.nim:701-703)",
             **solves[2]},
        ],
    }
    return out


def main():
    root = Path(sys.argv[1]) if len(sys.argv) > 1 else DEFAULT_ROOT
    out = extract(root)
    FIXTURE.write_text(json.dumps(out, indent=1) + "\n")
    print(FIXTURE, [s["iterations"] for s in out["solves"]])


if __name__ == "__main__":
    main()
