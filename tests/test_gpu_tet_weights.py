"""The tetrahedron weights as the GPU computes them (ald_weight_tet: the
device build of ald_tet.h, compiled with -fmad=false as the delta kernels
are) against the oracle's literal weight_tet
(THERMACOND/tetrahedron.f90:188-384): the FP64 pipeline's form equal to the
reference's value for value (NaN where the reference divides 0 by 0) on
random tetrahedra, every tie pattern and sub-1e-10 differences; the mixed
pipeline's FP32 form within 1e-5 of each weight plus 1e-6 of the largest
weight of its tetrahedron on the random set."""
import itertools

import numpy as np
import pytest

pytestmark = pytest.mark.gpu


def _random_rows(seed=11, n=3000):
    rng = np.random.default_rng(seed)
    rows = []
    for _ in range(n):
        w = rng.uniform(-50, 400, size=4)
        rows.append(list(w) + [rng.uniform(w.min() - 5, w.max() + 5)])
    return rows


def _tie_rows():
    vals = [1.25, 2.5, 3.75, 5.0]
    rows = []
    for pat in itertools.product(range(4), repeat=4):
        for e in (1.0, 1.25, 1.9, 2.5, 3.1, 3.75, 4.4, 5.0, 5.5):
            rows.append([vals[p] for p in pat] + [e])
    return rows


def _tiny_rows(seed=5, n=500):
    rng = np.random.default_rng(seed)
    rows = []
    for _ in range(n):
        base = rng.uniform(-1e-8, 1e-8)
        w = base + rng.uniform(-3e-11, 3e-11, size=4)
        rows.append(list(w) + [rng.uniform(-2e-8, 2e-8)])
    return rows


def _device(ald_lib, rows, fp32=False):
    """weight_tet of each row's tetrahedron at the row's own energy: one
    call per distinct energy, as the reference evaluates all tetrahedra at
    one energy."""
    rows = np.asarray(rows, dtype=float)
    out = np.empty((len(rows), 4))
    for e in np.unique(rows[:, 4]):
        sel = rows[:, 4] == e
        out[sel] = ald_lib.weight_tet(rows[sel, :4], e, fp32=fp32)
    return out


def _oracle(oracle_lib, rows):
    return np.array([oracle_lib.weight_tet(np.array(r[:4]), r[4]) for r in rows])


@pytest.mark.parametrize("kind", ["random", "ties", "tiny"])
def test_device_weights_equal_reference(ald_lib, oracle_lib, kind):
    rows = {"random": _random_rows, "ties": _tie_rows, "tiny": _tiny_rows}[kind]()
    got, ref = _device(ald_lib, rows), _oracle(oracle_lib, rows)
    assert np.array_equal(np.isnan(got), np.isnan(ref))
    bad = ~np.isnan(ref) & (got != ref)
    assert not bad.any(), (np.argwhere(bad)[:5], got[bad][:5], ref[bad][:5])


def test_device_weights_one_energy_many_tetrahedra(ald_lib, oracle_lib):
    """The reference's own call shape: every tetrahedron at one energy
    (100 000 of them, more than one thread per tetrahedron in one pass of
    the grid)."""
    rng = np.random.default_rng(3)
    w = rng.uniform(0, 300, size=(100_000, 4))
    e = 150.0
    got = ald_lib.weight_tet(w, e)
    idx = rng.choice(len(w), 2000, replace=False)
    ref = np.array([oracle_lib.weight_tet(w[i], e) for i in idx])
    assert np.array_equal(got[idx], ref)
    outside = (e < w.min(1)) | (e > w.max(1))
    assert np.all(got[outside] == 0.0)


def test_mixed_fp32_weights_close(ald_lib, oracle_lib):
    rows = _random_rows(seed=23)
    got, ref = _device(ald_lib, rows, fp32=True), _oracle(oracle_lib, rows)
    scale = np.abs(ref).max(axis=1, keepdims=True)
    assert np.all(np.abs(got - ref) <= 1e-5 * np.abs(ref) + 1e-6 * scale)
    # out of range: exactly zero in both forms
    assert np.array_equal(got == 0.0, ref == 0.0)
