"""The device tetrahedron weights (ald_tet.h, compiled here for the host
with FMA contraction off, as the kernel is) against the oracle's literal
weight_tet (THERMACOND/tetrahedron.f90:188-384): bit-for-bit equal weights
for random corner energies and for every tie pattern."""
import itertools
import os
import subprocess

import numpy as np
import pytest

from conftest import ROOT


@pytest.fixture(scope="module")
def harness(tmp_path_factory):
    exe = str(tmp_path_factory.mktemp("tet") / "tet_harness")
    subprocess.check_call(["g++", "-std=c++17", "-O2", "-ffp-contract=off", "-o", exe,
                           os.path.join(ROOT, "tests", "tet_weight_harness.cpp")])
    return exe


def run(exe, rows):
    inp = "\n".join(" ".join(repr(float(x)) for x in r) for r in rows) + "\n"
    out = subprocess.run([exe], input=inp, capture_output=True, text=True, check=True).stdout
    a = np.array([[float(x) for x in l.split()] for l in out.strip().split("\n")])
    # columns 0-3: per-corner form, 4-7: four-at-once form; both must agree bitwise
    assert np.array_equal(np.nan_to_num(a[:, :4], nan=7.0), np.nan_to_num(a[:, 4:], nan=7.0))
    return a[:, :4]


def test_random_corners_bitwise(harness, oracle_lib):
    rng = np.random.default_rng(11)
    rows = []
    for _ in range(3000):
        w = rng.uniform(-50, 400, size=4)
        e1, e4 = w.min(), w.max()
        rows.append(list(w) + [rng.uniform(e1 - 5, e4 + 5)])
    got = run(harness, rows)
    for r, g in zip(rows, got):
        ref = oracle_lib.weight_tet(np.array(r[:4]), r[4])
        assert np.array_equal(g, ref), (r, g, ref)


def test_tie_patterns_bitwise(harness, oracle_lib):
    vals = [1.25, 2.5, 3.75, 5.0]
    rows = []
    for pat in itertools.product(range(4), repeat=4):
        for e in (1.0, 1.25, 1.9, 2.5, 3.1, 3.75, 4.4, 5.0, 5.5):
            rows.append([vals[p] for p in pat] + [e])
    got = run(harness, rows)
    for r, g in zip(rows, got):
        ref = oracle_lib.weight_tet(np.array(r[:4]), r[4])
        assert np.array_equal(np.nan_to_num(g, nan=7.0), np.nan_to_num(ref, nan=7.0)), (r, g, ref)


def test_tiny_differences_bitwise(harness, oracle_lib):
    """Differences below 1e-10 are replaced by +-1e-10 in FP32 (tetrahedron.f90:314-352)."""
    rng = np.random.default_rng(5)
    rows = []
    for _ in range(500):
        base = rng.uniform(-1e-8, 1e-8)
        w = base + rng.uniform(-3e-11, 3e-11, size=4)
        rows.append(list(w) + [rng.uniform(-2e-8, 2e-8)])
    got = run(harness, rows)
    for r, g in zip(rows, got):
        ref = oracle_lib.weight_tet(np.array(r[:4]), r[4])
        assert np.array_equal(np.nan_to_num(g, nan=7.0), np.nan_to_num(ref, nan=7.0)), (r, g, ref)
