"""Three-phonon self-energy at arbitrary q (job=2: make_kp_bs,
function_self_w3/w4, lw-selfenergy files) through the C ABI vs the oracle
(oracle/oracle_self.cpp), GPU.

The mesh eigenpairs of the oracle are injected into the context.  The
eigenpairs at the path points q and at q3 = -q - q2 come from each code's
own eigensolver, so per-mode values are compared as sums over degenerate
groups of la (|omega_i - omega_j| < 1e-6 max omega): a sum over a degenerate
subspace does not depend on the basis chosen in it, and the sums over l3
inside each value are basis-free in the same way.  Acoustic modes at Gamma
(omega0 < 1e-3 max omega) are left out: there omega -> 0 makes the matrix
element 0/0 in both codes.  Values are compared at the path points strictly
inside the segments: at a segment end (Gamma, X, L, all points of the 4^3
mesh, or within 3e-9 of one: make_kp_bs divides by nkdir-1+1e-8) there is a
q2 with q3 = -q - q2 within rounding of Gamma, where om3 and the matrix
element are rounding noise amplified by 1/om3 and n(om3), in the reference as
here.  The files are still checked at every point for their layout.

Tolerance: |gpu - ref| <= 1e-8 |ref| + 1e-9 max|ref| over the compared values
(the orders of the sums differ; the real part of function_self_w3 is a
principal-value sum with cancellations).
"""
import os
import sys

import numpy as np
import pytest

from conftest import ROOT, make_case

sys.path.insert(0, os.path.join(ROOT, "oracle"))
import writers as OW  # noqa: E402

pytestmark = pytest.mark.gpu

CASES = [(1, (4, 4, 4), {}), (0, (4, 4, 4), {})]
NKDIR = 4
KPBS = "0\n%d\n2\nG 0 0 0\nX 0 0 1\nL 0.5 0.5 0.5\n" % NKDIR
INTERIOR = [p for p in range(2 * NKDIR) if 0 < p % NKDIR < NKDIR - 1]
KB, H, CL = 1.3806504e-23, 6.62606896e-34, 2.99792458e+8


@pytest.fixture(scope="module", params=CASES, ids=lambda c: "cfg%d_%d" % (c[0], c[1][0]))
def case(request, oracle_lib, ald_lib, workdir):
    cfg, mesh, kw = request.param
    d = make_case(workdir, cfg, mesh, **kw)
    with open(os.path.join(d, "kpbs.params"), "w") as f:
        f.write(KPBS)
    O = oracle_lib.Oracle(d)
    O.mesh()
    O.phonons()
    ev, vec, vel = O.get_phonons()
    ctx = ald_lib.Context(d)
    ctx.set_phonons(ev, vec, vel)
    yield d, O, ctx
    ctx.close()


def groups(omega):
    """index groups of equal frequencies (degenerate modes)."""
    tol = 1e-6 * max(float(np.max(omega)), 1e-30)
    order = np.argsort(omega)
    out, cur = [], [order[0]]
    for i in order[1:]:
        if abs(omega[i] - omega[cur[-1]]) < tol:
            cur.append(i)
        else:
            out.append(cur)
            cur = [i]
    out.append(cur)
    return out


def grouped(values, omega, skip_below):
    """sums of values over degenerate groups, groups of frequency >= skip_below."""
    return np.array([sum(values[i] for i in g) for g in groups(omega) if omega[g[0]] >= skip_below])


def close(g, r, rtol=1e-8, atol=1e-9):
    g, r = np.asarray(g), np.asarray(r)
    scale = np.abs(r).max() if r.size else 0.0
    return bool(np.all(np.abs(g - r) <= rtol * np.abs(r) + atol * scale)), float(np.abs(g - r).max())


def test_make_kp_bs(case):
    d, O, ctx = case
    kp, dk = ctx.make_kp_bs(d)
    ko, do = O.make_kp_bs(d)
    assert kp.shape == ko.shape == (3, 8)
    assert np.allclose(kp, ko, rtol=1e-14, atol=1e-14)
    assert np.allclose(dk, do, rtol=1e-14, atol=1e-14)
    assert dk[0] == 0.0 and np.all(np.diff(dk) >= 0)


@pytest.mark.parametrize("gauss", [False, True])
def test_function_self_w(case, gauss):
    d, O, ctx = case
    kp, _ = O.make_kp_bs(d)
    ev, _ = O.frequencies_at(kp)
    cnst = O.lattice()["cnst"]
    om0 = np.sqrt(np.abs(ev)) * cnst          # (ndyn, nkp)
    temp = 300.0 * KB / (100 * H * CL)
    n = O.ndyn
    qs = np.repeat(kp, n, axis=1)
    las = np.tile(np.arange(1, n + 1), kp.shape[1])
    oms = om0.T.ravel()
    ns_o, us_o = O.self_w(qs, las, oms, temp, gauss=gauss)
    ns_g, us_g = ctx.function_self_w(qs, las, oms, temp, gauss=gauss)
    skip = 1e-3 * om0.max()
    for part_g, part_o in ((ns_g, ns_o), (us_g, us_o)):
        G, R = [], []
        for p in INTERIOR:
            sl = slice(p * n, (p + 1) * n)
            G.append(grouped(part_g[sl], om0[:, p], skip))
            R.append(grouped(part_o[sl], om0[:, p], skip))
        G, R = np.concatenate(G), np.concatenate(R)
        for comp in (np.real, np.imag):
            ok, worst = close(comp(G), comp(R))
            assert ok, worst
    if gauss:  # function_self_w4 computes the imaginary part only
        assert np.all(np.real(ns_g) == 0) and np.all(np.real(us_g) == 0)
    assert np.any(np.imag(ns_o + us_o) != 0)


def test_self_energy_bs_files(case, tmp_path):
    d, O, ctx = case
    tempk = 300.0
    res = ctx.self_energy_bs(d, tempk, out_dir=str(tmp_path))
    kp, dk = O.make_kp_bs(d)
    ev, _ = O.frequencies_at(kp)
    cnst = O.lattice()["cnst"]
    om0 = np.sqrt(np.abs(ev)) * cnst
    assert np.allclose(res["omega0"], om0, rtol=1e-10, atol=1e-8 * om0.max())
    n, npt = O.ndyn, kp.shape[1]
    temp = tempk * KB / (100 * H * CL)
    ns_o, us_o = O.self_w(np.repeat(kp, n, axis=1), np.tile(np.arange(1, n + 1), npt), om0.T.ravel(), temp)
    ise_o = 2 * np.imag(ns_o + us_o).reshape(npt, n).T
    ise_g = 2 * np.imag(res["nself"] + res["uself"])
    skip = 1e-3 * om0.max()
    G = np.concatenate([grouped(ise_g[:, p], om0[:, p], skip) for p in INTERIOR])
    R = np.concatenate([grouped(ise_o[:, p], om0[:, p], skip) for p in INTERIOR])
    ok, worst = close(G, R)
    assert ok, worst
    # file layout: one lw-selfenergy.dat record per (point, mode), one
    # lw-selfenergy2.dat record per point, list-directed
    L1 = open(tmp_path / "lw-selfenergy.dat").read().splitlines()
    L2 = open(tmp_path / "lw-selfenergy2.dat").read().splitlines()
    assert len(L1) == npt * n and len(L2) == npt
    for p in range(npt):
        for la in range(n):
            t = L1[p * n + la].split()
            assert len(t) == 12 and int(t[1]) == la + 1 and int(t[2]) == p + 1
            assert np.allclose([float(x) for x in t[3:6]], kp[:, p], rtol=1e-13, atol=1e-13)
            ise = np.float64(ise_g[la, p])
            with np.errstate(divide="ignore"):  # IEEE results at a zero linewidth, as in the reference
                tse = np.float64(1e10) / CL / ise
                inv = np.float64(1) / tse
            want = OW.list_record(tempk, la + 1, p + 1, *res["kp_bs"][:, p], res["dk_bs"][p], res["omega0"][la, p],
                                  ise / 2, ise, tse, inv)
            assert L1[p * n + la] == want
        t2 = L2[p].split()
        assert len(t2) == 2 + 2 * n
