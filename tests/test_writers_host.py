"""The gfortran edit rules of the output writers, on the CPU.

Golden: records of the output files the reference ships with its Ge and
GeSe examples (tests/golden/fortran_records.json, made by
tests/golden/make_format_golden.py).  Each record is rebuilt from its own
numbers, by the library's formatter (ald_format_value, host code of the
writers) and by the oracle's restatement (oracle/writers.py), and must come
out byte for byte the same.  A random sweep then checks that the two agree
on every edit the writers use.
"""
import json
import math
import os
import re
import sys

import numpy as np
import pytest

from conftest import ROOT

sys.path.insert(0, os.path.join(ROOT, "oracle"))
import writers as OW  # noqa: E402

RECORDS = json.load(open(os.path.join(ROOT, "tests", "golden", "fortran_records.json")))["records"]
EXP3 = re.compile(r"^([+-]?[0-9]*\.[0-9]*)([+-][0-9]{3})$")


def num(t):
    m = EXP3.match(t)
    if m:
        return float(m.group(1) + "e" + m.group(2))
    return float({"Infinity": "inf", "-Infinity": "-inf"}.get(t, t))


class LibFmt:
    """list_record / edit_* on top of the library's ald_format_value."""

    def __init__(self, ald):
        self.f = ald.format_value

    def list_record(self, *items):
        out, prev = "", False
        for it in items:
            c = isinstance(it, str)
            if not (c and prev) or not out:
                out += " "
            out += it if c else self.f("*I" if isinstance(it, int) else "*", it)
            prev = c
        return out

    def edit(self, e, x):
        return self.f(e, x)


class OracleFmt:
    def list_record(self, *items):
        return OW.list_record(*items)

    def edit(self, e, x):
        return OW.format_value(e, x)


def rebuild(F, kind, line):
    t = line.split()
    if kind == "qvalue":
        return F.list_record(int(t[0]), int(t[1]), num(t[2]), num(t[3]))
    if kind == "rhs":
        return F.list_record(*[num(x) for x in t])
    if kind == "tau":
        return "".join(" " + (F.edit("I14", int(x)) if k in (1, 5) else F.edit("G14.8", num(x)))
                       for k, x in enumerate(t))
    # kappa file records
    if line.startswith(" tot_kap="):
        return F.list_record("tot_kap=", num(t[1]))
    if line.strip() == "":
        return F.list_record(" ")
    if re.match(r"^[ 0-9]\d ", line) and len(t) == 7:
        return F.edit("I2", int(t[0])) + "".join(" " + F.edit("G11.4", num(x)) for x in t[1:])
    if len(t) == 3 and line.startswith("   "):
        return "   " + "".join(" " + F.edit("F9.3", num(x)) for x in t)
    return F.list_record(line[1:])  # the character header


def _cases():
    for r in RECORDS:
        lines = list(r["lines"])
        if r.get("header"):
            lines = [r["header"]] + lines
        yield r["source"], r["kind"], lines


@pytest.mark.parametrize("impl", ["oracle", "library"])
def test_records_rebuilt_byte_for_byte(impl, ald_lib):
    F = OracleFmt() if impl == "oracle" else LibFmt(ald_lib)
    n = bad = 0
    first = []
    for src, kind, lines in _cases():
        for k, line in enumerate(lines):
            if k == 0 and kind in ("qvalue", "tau"):
                got = F.list_record(line[1:])
            else:
                got = rebuild(F, kind, line)
            n += 1
            if got != line:
                bad += 1
                if len(first) < 5:
                    first.append((src, line, got))
    assert n > 700
    assert bad == 0, first


def test_golden_covers_the_edges():
    text = "\n".join("\n".join(r["lines"]) for r in RECORDS)
    for edge in ("Infinity", "-.", "E+", "E-", " 0.0000000 "):
        assert edge in text, edge
    assert re.search(r"\d[+-]\d{3}(\s|$)", text)  # Ew.d with a three-digit exponent


def _sweep_values(n=4000, seed=20261203):
    rng = np.random.default_rng(seed)
    mags = 10.0 ** rng.uniform(-320, 300, n)
    vals = list(mags * rng.choice([-1.0, 1.0], n))
    vals += list(rng.uniform(-2, 2, 500))
    # values on and around the G / list-directed switch points and roundings
    for e in range(-3, 19):
        for base in (1.0, 0.99999999995, 0.999999999999999999, 0.5, 9.99995, 0.0999999999):
            vals += [base * 10.0 ** e, -base * 10.0 ** e]
    vals += [0.0, -0.0, math.inf, -math.inf, math.nan, 5e-324, 2.2250738585072014e-308, 1e10, 1e-10, 0.1, 0.05]
    return vals


@pytest.mark.parametrize("edit", ["*", "G14.8", "G11.4", "G25.17", "F9.3", "F20.16", "E11.4", "E14.8"])
def test_library_and_oracle_agree(edit, ald_lib):
    diff = []
    for x in _sweep_values():
        a, b = ald_lib.format_value(edit, x), OW.format_value(edit, x)
        if a != b:
            diff.append((x, a, b))
    assert not diff, diff[:5]


def test_integer_edits(ald_lib):
    for v in [0, 1, -1, 7, 123456, -2147483647, 2147483647]:
        for e in ("I2", "I14", "*I"):
            assert ald_lib.format_value(e, v) == OW.format_value(e, v)
    assert ald_lib.format_value("I2", 123) == "**"
    assert ald_lib.format_value("*I", 1) == "          1"


def test_fortran_rules_by_hand(ald_lib):
    f = ald_lib.format_value
    assert f("G14.8", 300.0) == " 300.00000    "
    assert f("G14.8", -0.55093850) == "-.55093850    "
    assert f("G14.8", 0.0) == " 0.0000000    "
    assert f("G14.8", math.inf) == "      Infinity"
    assert f("G14.8", -math.inf) == "     -Infinity"
    assert f("G14.8", math.nan) == "           NaN"
    assert f("G11.4", 19.7198) == "  19.72    "
    assert f("G11.4", -4.770e-4) == "-0.4770E-03"
    assert f("F9.3", 62.10438) == "   62.104"
    assert f("*", 1.0) == "  1.0000000000000000     "
    assert f("*", 0.1) == " 0.10000000000000001     "
    assert f("*", -1.3169752846541651e-22) == " -1.3169752846541651E-022"
    for bad in ("X3", "G14", "F", "I0", "E9.0"):
        with pytest.raises(ValueError):
            f(bad, 1.0)
