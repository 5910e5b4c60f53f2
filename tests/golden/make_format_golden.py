"""Golden records for the gfortran edit rules of the output writers.

The reference ships two runs with their outputs (THERMACOND/Ge-example/kappa
and THERMACOND/GeSe-example/kappa, written by its gfortran build).  Their
output files use the record layouts the current writers still use:

* Qvalue.dat       list-directed: INTEGER, INTEGER, REAL(8), REAL(8)
                   (Qandtau, sub.f90:8263)
* RHS_IBZ.dat      list-directed: one REAL(8) per record
* tau_RTA.dat,     format (99(1x,g14.8)) with INTEGERs in fields 2 and 6
  tau_RTAandeff-cg.dat  (write_kappa, sub.f90:1894, 1910)
* kappa_RTA.dat,   (i2,99(1x,g11.4)) per band, list-directed character and
  kappa_direct-cg.dat   REAL(8) records, format (2(3x,2(3(1x,f9.3),2x)))
                   (write_kappa, sub.f90:1862-1874)

This script keeps, verbatim, every record of the kappa files and a selection
of the others: each record showing an edge of the rules (Infinity, NaN, a
three-digit exponent, a dropped leading zero, a zero, an "E+" exponent), at
most 40 per edge and file, and an evenly spaced sample.  The test rebuilds
each record from its own numbers and must get the same bytes.

Run where the reference is mounted:
    python tests/golden/make_format_golden.py <path of the reference checkout>
It writes tests/golden/fortran_records.json.
"""
from __future__ import annotations

import json
import os
import re
import sys

HERE = os.path.dirname(os.path.abspath(__file__))

EDGES = {
    "infinity": re.compile(r"Infinity"),
    "nan": re.compile(r"NaN"),
    "exp3": re.compile(r"\d[+-]\d{3}(\s|$)"),
    "dropped_zero": re.compile(r"(^|\s)-\.\d"),
    "zero": re.compile(r"(^|\s)0\.0+(\s|$)"),
    "eplus": re.compile(r"E\+"),
}
KINDS = {"Qvalue.dat": "qvalue", "RHS_IBZ.dat": "rhs", "tau_RTA.dat": "tau", "tau_RTAandeff-cg.dat": "tau",
         "kappa_RTA.dat": "kappa", "kappa_direct-cg.dat": "kappa"}


def select(lines, n_sample=40, per_edge=40):
    keep = set()
    for rx in EDGES.values():
        hits = [i for i, l in enumerate(lines) if rx.search(l)]
        keep.update(hits[:per_edge])
    step = max(1, len(lines) // n_sample)
    keep.update(range(0, len(lines), step))
    return sorted(keep)


def main(ref: str):
    out = []
    for ex in ("Ge-example", "GeSe-example"):
        d = os.path.join(ref, "THERMACOND", ex, "kappa")
        for name, kind in KINDS.items():
            lines = open(os.path.join(d, name)).read().split("\n")
            if lines and lines[-1] == "":
                lines.pop()
            if kind == "kappa":
                out.append({"source": f"THERMACOND/{ex}/kappa/{name}", "kind": kind, "lines": lines})
                continue
            head = 1 if kind in ("qvalue", "tau") else 0
            body = lines[head:]
            idx = select(body)
            out.append({"source": f"THERMACOND/{ex}/kappa/{name}", "kind": kind,
                        "header": lines[0] if head else None,
                        "lines": [body[i] for i in idx]})
    with open(os.path.join(HERE, "fortran_records.json"), "w") as f:
        json.dump({"records": out}, f, indent=0)
    print(sum(len(r["lines"]) for r in out), "records")


if __name__ == "__main__":
    if len(sys.argv) != 2:
        sys.exit("usage: %s <path of the reference checkout>" % sys.argv[0])
    main(sys.argv[1])
