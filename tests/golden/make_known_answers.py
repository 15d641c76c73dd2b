"""Extract the reference's known answers for the model plugins into
tests/golden/known_answers.json (the tests run where the reference tree is
absent).

  analytic  tests/analytic/analytic_test.py: the published total fluxes of
            the five GRRT test problems (Gold et al. 2020) that the
            reference's own test compares with a 2% tolerance, and the run
            parameters of tests/analytic/analytic.par.
  sphere    tests/isothermal_sphere/thermal.txt: total fluxes (polarized and
            unpolarized transfer) of the isothermal sphere at 38 frequency /
            inclination pairs, with the run line of tests/isothermal_sphere/info.

    python tests/golden/make_known_answers.py [reference tree]
"""
from __future__ import annotations

import ast
import json
import os
import re
import sys

HERE = os.path.dirname(os.path.abspath(__file__))


def main(ref: str) -> None:
    src = open(os.path.join(ref, "tests", "analytic", "analytic_test.py")).read()
    published = ast.literal_eval(re.search(r"published\s*=\s*(\[[^\]]*\])", src).group(1))
    tol = float(re.search(r"if err > ([0-9.eE+-]+)", src).group(1))
    par = {}
    for line in open(os.path.join(ref, "tests", "analytic", "analytic.par")):
        t = line.split("#")[0].split()
        if len(t) == 2:
            par[t[0]] = t[1]
    rows = []
    for line in open(os.path.join(ref, "tests", "isothermal_sphere", "thermal.txt")):
        if line.startswith("#") or not line.strip():
            continue
        f, inc, ftot, funpol = (float(x) for x in line.split()[:4])
        rows.append([f, inc, ftot, funpol])
    info = [l.strip() for l in open(os.path.join(ref, "tests", "isothermal_sphere", "info")) if "./ipole" in l][0]
    out = {
        "analytic": {"published_Ftot_unpol": published[1:], "models": list(range(1, len(published))),
                     "tolerance": tol, "par": par, "source": "tests/analytic/analytic_test.py, analytic.par"},
        "sphere_thermal": {"rows": rows, "columns": ["freqcgs", "thetacam", "Ftot", "Ftot_unpol"],
                           "run": info, "source": "tests/isothermal_sphere/thermal.txt, info"},
    }
    with open(os.path.join(HERE, "known_answers.json"), "w") as fp:
        json.dump(out, fp, indent=1)
    print("analytic", published[1:], "tol", tol, "| sphere rows", len(rows))


if __name__ == "__main__":
    if len(sys.argv) < 2:
        raise SystemExit("usage: make_known_answers.py <reference checkout>")
    main(sys.argv[1])
