"""Cells of more than 12 bands on the GPU against the oracle (GPU).

Two cells of the batched benchmark suites:
  * the 8-atom LJ mass superlattice (p = 2, 24 bands; nearest-neighbour
    cutoff 1.2 sigma so that the oracle's term-by-term V3 stays fast),
    2 x 4 x 4 mesh;
  * the 64-atom rock-salt Morse cell (192 bands, 95 040 FC3 terms), 2^3 mesh.
They run the large-cell kernels: the Householder + QL eigensolver (above 64
bands; selected by ALD_EIGENSOLVER=householder below that), V3 as batched
complex GEMMs per pair (ald_v3_dense.cu) and the band-generic delta kernels.
The literal oracle checks the 24-band cell; for 192 bands its V3 loop
(7e11 term iterations per pair) is out of reach and tests/oracle_dense.py,
pinned to it by test_oracle_dense.py, stands in.  Bars as in
test_gpu_parity.py: FP64 |gpu - ref| <= 1e-10 |ref| + 1e-12 max|ref|.
"""
import os

import numpy as np
import pytest

import oracle_dense
from conftest import make_case
from test_gpu_parity import close, degenerate_groups, gamma_acoustic_mask

pytestmark = pytest.mark.gpu


def _phonons(oracle_lib, d):
    O = oracle_lib.Oracle(d)
    O.mesh()
    O.phonons()
    O.tet()
    return O, O.get_phonons()


def _own_phonons(ald_lib, d, householder):
    old = os.environ.get("ALD_EIGENSOLVER")
    if householder:
        os.environ["ALD_EIGENSOLVER"] = "householder"
    try:
        ctx = ald_lib.Context(d)
        ph = ctx.get_frequencies()
    finally:
        if old is None:
            os.environ.pop("ALD_EIGENSOLVER", None)
        else:
            os.environ["ALD_EIGENSOLVER"] = old
    return ctx, ph


def _check_phonons(O, ref, got):
    ev_o, vec_o, vel_o = ref
    ev_g, vec_g, vel_g = got
    n = O.ndyn
    scale = np.abs(ev_o).max()
    assert np.all(np.abs(ev_g - ev_o) <= 1e-10 * np.abs(ev_o) + 1e-13 * scale)
    # floor: 1e-9 of a physical velocity scale (about 1e-5 c here); on meshes of
    # high-symmetry points only (the 2^3 mesh) every velocity is rounding noise
    vs = max(np.abs(vel_o).max(), 1e-6)
    assert np.all(np.abs(vel_g - vel_o) <= 1e-8 * np.abs(vel_o) + 1e-9 * vs)
    for k in range(O.nkc):
        V = vec_g[:, :, k]
        assert np.allclose(V.conj().T @ V, np.eye(n), atol=1e-12)
        w = ev_o[:, k]
        for gr in degenerate_groups(w, 1e-8):
            if abs(w[gr[0]]) < 1e-9 * abs(w).max():
                continue
            Pg = vec_g[:, gr, k] @ vec_g[:, gr, k].conj().T
            Po = vec_o[:, gr, k] @ vec_o[:, gr, k].conj().T
            assert np.abs(Pg - Po).max() < 1e-8


def gamma_acoustic_modes(O, ev):
    """(nibz, ndyn) True for the acoustic modes of the IBZ point at Gamma: their
    eigenvalues are rounding noise, and so are their linewidths (|V3|^2 there
    is 0/0 noise weighted by the delta), in the reference as here."""
    mapinv = O.ibz()["mapinv"] - 1
    w = ev[:, mapinv].T
    return np.abs(w) < 1e-9 * np.abs(ev).max()


def close_q(g, r, O, ev, rtol=1e-10, atol=1e-12):
    """close() over the linewidths of every mode but the Gamma-acoustic ones,
    which must stay below 1e-8 of the largest."""
    ac = gamma_acoustic_modes(O, ev)
    scale = np.abs(r).max()
    assert np.all(np.abs(g[ac]) <= 1e-8 * scale) and np.all(np.abs(r[ac]) <= 1e-8 * scale)
    return close(g[~ac], r[~ac], rtol, atol)


@pytest.fixture(scope="module")
def sl24(oracle_lib, ald_lib, workdir):
    d = make_case(workdir, 3, (2, 4, 4), p=2, rc_sigma=1.2, delta="tetra")
    O, ph = _phonons(oracle_lib, d)
    return d, O, ph


@pytest.mark.parametrize("householder", [False, True], ids=["jacobi", "householder"])
def test_superlattice24_eigensolvers(sl24, ald_lib, householder):
    d, O, ph = sl24
    ctx, got = _own_phonons(ald_lib, d, householder)
    _check_phonons(O, ph, got)
    ctx.close()


@pytest.mark.parametrize("delta", ["tetra", "gauss"])
def test_superlattice24_v3_fgr_tau(sl24, ald_lib, oracle_lib, workdir, delta):
    d0, O, ph = sl24
    d = make_case(workdir, 3, (2, 4, 4), p=2, rc_sigma=1.2, delta=delta)
    rows = (2, 4)
    v33 = O.v3(*rows)
    P1s, P2s = O.fgr(rows[0], rows[1], v33, gauss=delta == "gauss")
    ctx = ald_lib.Context(d)
    ctx.set_phonons(*ph)
    v = ctx.calculate_w3_ibz_split_sq(list(rows))
    keep = ~gamma_acoustic_mask(O, ph[0], *rows)
    ok, worst = close(v[keep], v33[keep])
    assert ok, ("V3", worst)
    P1, P2 = ctx.calculate_fgr(list(rows), v33)
    for g, r in ((P1, P1s), (P2, P2s)):
        ok, worst = close(g, r)
        assert ok, ("FGR", worst)
    T = 300.0
    O.distribution(T)
    Qr, QNr, QUr, _, _ = O.tau(rows[0], rows[1], T, P1s, P2s, want_p=False)
    Q, QN, QU, _, _ = ctx.calculate_tau_rta(list(rows), T, P1s, P2s, want_p=False)
    for g, r in ((Q, Qr), (QN, QNr), (QU, QUr)):
        ok, worst = close(g, r)
        assert ok, ("Q", worst)
    ctx.close()


@pytest.mark.parametrize("delta", ["tetra", "gauss"])
def test_superlattice24_pipeline(ald_lib, oracle_lib, workdir, delta):
    """The fused pipeline (band-generic delta into R1/R2, collision matrix,
    CG) against the oracle's whole job=1 sequence."""
    d = make_case(workdir, 3, (2, 4, 4), p=2, rc_sigma=1.2, delta=delta)
    ref = oracle_lib.run_job1(d)
    O = ref["O"]
    ctx = ald_lib.Context(d)
    ctx.set_phonons(*O.get_phonons())
    out = ctx.kappa_pipeline(ref["tempk"])
    ev = O.get_phonons()[0]
    for key in ("Q", "QN", "QU"):
        ok, worst = close_q(out[key], ref[key], O, ev)
        assert ok, (key, worst)
    ok, worst = close(out["kappa_rta_modes"], ref["kappa_rta"], atol=1e-10)
    assert ok, ("kappa_rta", worst)
    assert out["cg_iters"] == ref["cg_iters"]
    ok, worst = close(out["kappa_cg_modes"], ref["kappa_cg"], atol=1e-10)
    assert ok, ("kappa_cg", worst)
    ctx.close()


@pytest.fixture(scope="module")
def rs192(oracle_lib, ald_lib, workdir):
    d = make_case(workdir, 4, (2, 2, 2))
    O, ph = _phonons(oracle_lib, d)
    return d, O, ph


def test_rocksalt192_householder(rs192, ald_lib):
    d, O, ph = rs192
    assert O.ndyn == 192
    ctx, got = _own_phonons(ald_lib, d, False)  # above 64 bands: Householder + QL
    _check_phonons(O, ph, got)
    ctx.close()


def test_rocksalt192_v3_fgr_pipeline(rs192, ald_lib, oracle_lib):
    d, O, ph = rs192
    rows = (O.nibz, O.nibz)
    v33 = oracle_dense.v3_factorised(O, *rows)
    ctx = ald_lib.Context(d)
    ctx.set_phonons(*ph)
    v = ctx.calculate_w3_ibz_split_sq(list(rows))
    keep = ~gamma_acoustic_mask(O, ph[0], *rows)
    ok, worst = close(v[keep], v33[keep])
    assert ok, ("V3", worst)
    P1s, P2s = O.fgr(rows[0], rows[1], v33, gauss=False)
    P1, P2 = ctx.calculate_fgr(list(rows), v33)
    for g, r in ((P1, P1s), (P2, P2s)):
        ok, worst = close(g, r)
        assert ok, ("FGR", worst)
    del P1, P2
    T = 300.0
    O.distribution(T)
    Qr, _, _, _, _ = O.tau(rows[0], rows[1], T, P1s, P2s, want_p=False)
    out = ctx.kappa_pipeline(T)
    ok, worst = close(out["Q"][rows[0] - 1:rows[1]], Qr)
    assert ok, ("pipeline Q", worst)
    assert np.all(np.isfinite(out["kappa_cg"]))
    ctx.close()


@pytest.fixture(scope="module")
def lj12(oracle_lib, ald_lib, workdir):
    d = make_case(workdir, 3, (4, 4, 4), rc_sigma=1.2, delta="tetra")
    O, ph = _phonons(oracle_lib, d)
    return d, O, ph


@pytest.mark.parametrize("which", ["lj12", "sl24", "rs192"])
def test_large_mixed_tensor_cores(which, lj12, sl24, rs192, ald_lib):
    """ALD_MIXED from 9 bands up: both mode products as split-FP16 tcgen05
    GEMMs (ald_v3_dense_tc.cu) against the FP64 oracle on the same
    eigenpairs; |V3|^2 normwise within 1e-4, and the pipeline's Q per mode
    within 1e-4 (+1e-8 max|Q|) of the FP64 pipeline's."""
    d, O, ph = {"lj12": lj12, "sl24": sl24, "rs192": rs192}[which]
    rows = (O.nibz, O.nibz) if which == "rs192" else (2, 3)
    v33 = oracle_dense.v3_factorised(O, *rows) if which == "rs192" else O.v3(*rows)
    keep = ~gamma_acoustic_mask(O, ph[0], *rows)
    delta = ald_lib.DELTA_TETRA
    ctx = ald_lib.Context(d, ald_lib.default_options(precision=ald_lib.MIXED, delta=delta))
    ctx.set_phonons(*ph)
    v = ctx.calculate_w3_ibz_split_sq(list(rows))
    err = np.linalg.norm(v[keep] - v33[keep]) / np.linalg.norm(v33[keep])
    print(which, "tensor-core |V3|^2 normwise", err)
    assert err <= 1e-4, err
    out = ctx.kappa_pipeline(300.0)
    ctx.close()
    ref = ald_lib.Context(d, ald_lib.default_options(precision=ald_lib.FP64, delta=delta))
    ref.set_phonons(*ph)
    r = ref.kappa_pipeline(300.0)
    ref.close()
    eq = np.abs(out["Q"] - r["Q"]) / (np.abs(r["Q"]) + 1e-8 * np.abs(r["Q"]).max())
    eq = eq[~gamma_acoustic_modes(O, ph[0])]
    print(which, "mixed Q worst", eq.max(), "median", np.median(eq))
    assert eq.max() <= 1e-4
    k, kr = out["kappa_cg"], r["kappa_cg"]
    if which == "rs192":
        # every point of the 2^3 mesh is a high-symmetry point: the group
        # velocities, and with them kappa, vanish to rounding noise
        assert np.abs(kr).max() < 1e-20
    else:
        assert np.abs(k - kr).max() <= 1e-4 * np.abs(kr).max()
