"""CUDA path vs the oracle at the benchmark suite's own sizes (GPU).

The stage tests of test_gpu_parity.py run on 4^3 and 6^3 meshes; these run
on the meshes the workloads are quoted on:

  rock-salt Morse, 16^3 (276 IBZ points, tetrahedron delta), the bench
    workload: V3, P1smpi/P2smpi and Q of three IBZ rows against the live
    oracle; the fused pipeline (Q, Q_N, Q_U of every row, the RTA and CG
    kappa) at 100, 300 and 600 K against the oracle's full job=1 run stored
    in tests/golden/nacl_morse_mesh16.npz (make_oracle_fixtures.py);
  LJ argon, 10^3 (85 IBZ points, Gaussian 0.1 THz), every row: the whole
    job=1 sequence against the live oracle;
  LJ argon, 32^3 (1 768 IBZ points, Gaussian 0.05 THz): two IBZ rows of V3
    and of the delta, FP64 and the tensor-core mixed form.

The oracle's eigenpairs are injected into the GPU context so that both
sides start from the same phonons.  Bars (written per test): FP64 stages
|gpu - ref| <= 1e-10 |ref| + 1e-12 max|ref|, kappa tensors with a floor of
1e-10 max|kappa| (components that vanish by symmetry carry cancellation
noise); the mixed path |V3|^2 normwise 1e-4, Q per mode 1e-4 (+1e-8 max|Q|),
kappa 1e-4 of max|kappa|.
"""
import os

import numpy as np
import pytest

from conftest import make_case
from test_gpu_parity import close, gamma_acoustic_mask

pytestmark = pytest.mark.gpu

HERE = os.path.dirname(os.path.abspath(__file__))
FIX16 = os.path.join(HERE, "golden", "nacl_morse_mesh16.npz")
TEMPS = (100.0, 300.0, 600.0)
ROWS16 = (138, 140)  # three IBZ rows of the 16^3 mesh (1-based, inclusive)


def _oracle_phonons(oracle_lib, d):
    O = oracle_lib.Oracle(d)
    O.mesh()
    O.phonons()
    O.tet()
    return O, O.get_phonons()


@pytest.fixture(scope="module")
def nacl16(oracle_lib, ald_lib, workdir):
    d = make_case(workdir, 1, (16, 16, 16))
    O, ph = _oracle_phonons(oracle_lib, d)
    fx = np.load(FIX16)
    ev = ph[0]
    # the fixture was made from these eigenpairs
    assert abs(ev.sum() - fx["ev_sum"]) <= 1e-12 * abs(fx["ev_sum"])
    assert abs((ev * ev).sum() - fx["ev_sumsq"]) <= 1e-12 * abs(fx["ev_sumsq"])
    v33 = O.v3(*ROWS16)
    P1s, P2s = O.fgr(ROWS16[0], ROWS16[1], v33, gauss=False)
    yield d, O, ph, fx, v33, P1s, P2s


def test_rocksalt16_rows_v3_fgr_tau(nacl16, ald_lib):
    d, O, ph, fx, v33, P1s, P2s = nacl16
    ctx = ald_lib.Context(d)
    ctx.set_phonons(*ph)
    v = ctx.calculate_w3_ibz_split_sq(list(ROWS16))
    keep = ~gamma_acoustic_mask(O, ph[0], *ROWS16)
    assert keep.mean() > 0.95
    ok, worst = close(v[keep], v33[keep])
    assert ok, ("V3", worst)
    P1, P2 = ctx.calculate_fgr(list(ROWS16), v33)
    for g, r, name in ((P1, P1s, "P1smpi"), (P2, P2s, "P2smpi")):
        ok, worst = close(g, r)
        assert ok, (name, worst)
    for T in TEMPS:
        O.distribution(T)
        Qr, QNr, QUr, _, _ = O.tau(ROWS16[0], ROWS16[1], T, P1s, P2s, want_p=False)
        Q, QN, QU, _, _ = ctx.calculate_tau_rta(list(ROWS16), T, P1s, P2s, want_p=False)
        for g, r, name in ((Q, Qr, "Q"), (QN, QNr, "QN"), (QU, QUr, "QU")):
            ok, worst = close(g, r)
            assert ok, (T, name, worst)
        # the fixture's full run holds the same rows
        ok, worst = close(Qr, fx["Q_%d" % T][ROWS16[0] - 1:ROWS16[1]])
        assert ok, (T, "fixture", worst)
    ctx.close()


@pytest.mark.parametrize("T", TEMPS)
def test_rocksalt16_pipeline_fp64(nacl16, ald_lib, T):
    d, O, ph, fx, _, _, _ = nacl16
    ctx = ald_lib.Context(d)
    ctx.set_phonons(*ph)
    out = ctx.kappa_pipeline(T)
    t = "%d" % T
    for key in ("Q", "QN", "QU"):
        ok, worst = close(out[key], fx[key + "_" + t])
        assert ok, (key, worst)
    ok, worst = close(out["kappa_rta_modes"], fx["kappa_rta_" + t], atol=1e-10)
    assert ok, ("kappa_rta", worst)
    assert out["cg_iters"] == int(fx["cg_iters_" + t])
    ok, worst = close(out["x"], fx["x_" + t], atol=1e-10)
    assert ok, ("x", worst)
    ok, worst = close(out["kappa_cg_modes"], fx["kappa_cg_" + t], atol=1e-10)
    assert ok, ("kappa_cg", worst)
    ctx.close()


@pytest.mark.parametrize("T", TEMPS)
def test_rocksalt16_mixed(nacl16, ald_lib, T):
    d, O, ph, fx, v33, _, _ = nacl16
    ctx = ald_lib.Context(d, ald_lib.default_options(precision=ald_lib.MIXED, delta=ald_lib.DELTA_TETRA))
    ctx.set_phonons(*ph)
    if T == 300.0:
        v = ctx.calculate_w3_ibz_split_sq(list(ROWS16))
        keep = ~gamma_acoustic_mask(O, ph[0], *ROWS16)
        err = np.linalg.norm(v[keep] - v33[keep]) / np.linalg.norm(v33[keep])
        print("mixed |V3|^2 normwise", err)
        assert err <= 1e-4, err
    out = ctx.kappa_pipeline(T)
    t = "%d" % T
    Qr = fx["Q_" + t]
    eq = np.abs(out["Q"] - Qr) / (np.abs(Qr) + 1e-8 * np.abs(Qr).max())
    print("mixed Q worst", eq.max())
    assert eq.max() <= 1e-4
    for key in ("kappa_rta", "kappa_cg"):
        k, kr = out[key], fx[key + "_" + t].sum(0)
        e = np.abs(k - kr).max() / np.abs(kr).max()
        print("mixed", key, e)
        assert e <= 1e-4, (key, e)
    ctx.close()


def test_argon10_full_job1(oracle_lib, ald_lib, workdir):
    """Configuration 0 as specified: 10^3 mesh, Gaussian 0.1 THz, all 85 rows."""
    d = make_case(workdir, 0, (10, 10, 10))
    ref = oracle_lib.run_job1(d)
    O = ref["O"]
    ph = O.get_phonons()
    ctx = ald_lib.Context(d)
    ctx.set_phonons(*ph)
    v = ctx.calculate_w3_ibz_split_sq([1, ctx.nibz])
    keep = ~gamma_acoustic_mask(O, ph[0], 1, ctx.nibz)
    ok, worst = close(v[keep], ref["v33"][keep])
    assert ok, ("V3", worst)
    P1, P2 = ctx.calculate_fgr([1, ctx.nibz], ref["v33"])
    for g, r in ((P1, ref["P1s"]), (P2, ref["P2s"])):
        ok, worst = close(g, r)
        assert ok, ("FGR", worst)
    out = ctx.kappa_pipeline(ref["tempk"])
    for key in ("Q", "QN", "QU"):
        ok, worst = close(out[key], ref[key])
        assert ok, (key, worst)
    ok, worst = close(out["kappa_rta_modes"], ref["kappa_rta"], atol=1e-10)
    assert ok, ("kappa_rta", worst)
    assert out["cg_iters"] == ref["cg_iters"]
    ok, worst = close(out["x"], ref["x"], atol=1e-10)
    assert ok, ("x", worst)
    ok, worst = close(out["kappa_cg_modes"], ref["kappa_cg"], atol=1e-10)
    assert ok, ("kappa_cg", worst)
    ctx.close()
    # the mixed path on the same inputs
    ctx = ald_lib.Context(d, ald_lib.default_options(precision=ald_lib.MIXED, delta=ald_lib.DELTA_GAUSS))
    ctx.set_phonons(*ph)
    out = ctx.kappa_pipeline(ref["tempk"])
    eq = np.abs(out["Q"] - ref["Q"]) / (np.abs(ref["Q"]) + 1e-8 * np.abs(ref["Q"]).max())
    assert eq.max() <= 1e-4, eq.max()
    for key, rk in (("kappa_rta", "kappa_rta"), ("kappa_cg", "kappa_cg")):
        k, kr = out[key], ref[rk].sum(0)
        assert np.abs(k - kr).max() <= 1e-4 * np.abs(kr).max(), key
    ctx.close()


def test_argon32_rows_fp64_and_tensor_cores(oracle_lib, ald_lib, workdir):
    """Configuration 2's 32^3 mesh: two IBZ rows of |V3|^2 (FP64 and the
    tcgen05 class sums of the mixed path) and of the Gaussian delta."""
    d = make_case(workdir, 2, (32, 32, 32))
    O, ph = _oracle_phonons(oracle_lib, d)
    rows = (884, 885)
    v33 = O.v3(*rows)
    P1s, P2s = O.fgr(rows[0], rows[1], v33, gauss=True)
    keep = ~gamma_acoustic_mask(O, ph[0], *rows)
    ctx = ald_lib.Context(d)
    ctx.set_phonons(*ph)
    v = ctx.calculate_w3_ibz_split_sq(list(rows))
    ok, worst = close(v[keep], v33[keep])
    assert ok, ("V3 fp64", worst)
    P1, P2 = ctx.calculate_fgr(list(rows), v33)
    for g, r in ((P1, P1s), (P2, P2s)):
        ok, worst = close(g, r)
        assert ok, ("FGR", worst)
    ctx.close()
    ctx = ald_lib.Context(d, ald_lib.default_options(precision=ald_lib.MIXED, delta=ald_lib.DELTA_GAUSS))
    ctx.set_phonons(*ph)
    v = ctx.calculate_w3_ibz_split_sq(list(rows))
    err = np.linalg.norm(v[keep] - v33[keep]) / np.linalg.norm(v33[keep])
    print("tensor-core |V3|^2 normwise", err)
    assert err <= 1e-4, err
    ctx.close()
