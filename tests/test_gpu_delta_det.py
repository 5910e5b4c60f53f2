"""The pipeline's tetrahedron delta with the deterministic option: run-to-run
reproducibility and agreement with the atomic form (GPU).

With ald_options.deterministic = 1 (the default for the FP64 path) the
pipeline's tetrahedron delta runs twice: the first pass records each R1/R2
entry's largest term, the second adds every term as a 62-bit fixed-point
integer scaled by that bound, so the sums do not depend on the order of the
additions and repeated runs give the same bits (FP64 and mixed paths).  With
deterministic = 0 the terms are added with FP64 atomics in arrival order;
both sum the same terms, so they agree to FP64 rounding:
  Q, Q_N, Q_U, the CG solution and kappa within 1e-12 relative (floor
  1e-14 of the largest value).
Both forms are also held to the oracle at 1e-10 (the FP64 default by the
pipeline tests of test_gpu_parity.py and test_gpu_suite_sizes.py, and
test_deterministic_matches_oracle below).
"""
import numpy as np
import pytest

from conftest import make_case

pytestmark = pytest.mark.gpu

KEYS = ("Q", "QN", "QU", "x", "kappa_rta", "kappa_cg", "kappa_rta_modes", "kappa_cg_modes")

# (configuration, mesh, options): rock-salt (6 bands) on even and odd meshes,
# LJ argon (3 bands) and the 4-atom superlattice cell (12
# bands) with the tetrahedron delta; the crystals are cubic, so their meshes
# are too (other meshes put star arms off the mesh)
CASES = [(1, (6, 6, 6), {}), (1, (5, 5, 5), {}), (1, (3, 3, 3), {}), (1, (4, 4, 4), {}),
         (0, (5, 5, 5), {"delta": "tetra"}), (3, (4, 4, 4), {"delta": "tetra", "rc_sigma": 1.2})]


def run(ald_lib, d, precision, deterministic=0):
    opt = ald_lib.default_options(precision=precision, delta=ald_lib.DELTA_TETRA, deterministic=deterministic)
    with ald_lib.Context(d, opt) as ctx:
        return ctx.kappa_pipeline()


def close(g, r, rtol=1e-12, atol=1e-14):
    g, r = np.asarray(g), np.asarray(r)
    scale = np.abs(r).max() if r.size else 0.0
    return bool(np.all(np.abs(g - r) <= rtol * np.abs(r) + atol * scale)), \
        float((np.abs(g - r) / (np.abs(r) + atol * scale + 1e-300)).max())


@pytest.mark.parametrize("cfg,mesh,kw", CASES, ids=lambda c: str(c) if not isinstance(c, tuple) else "x".join(map(str, c)))
def test_deterministic_matches_default_fp64(ald_lib, workdir, cfg, mesh, kw):
    d = make_case(workdir, cfg, mesh, **kw)
    a = run(ald_lib, d, ald_lib.FP64, 1)
    r = run(ald_lib, d, ald_lib.FP64)
    assert a["cg_iters"] == r["cg_iters"]
    assert np.abs(r["Q"]).max() > 0
    for k in KEYS:
        ok, worst = close(a[k], r[k])
        assert ok, (k, worst)


@pytest.mark.parametrize("precision", ["FP64", "MIXED"])
def test_deterministic_bitwise_repeatable(ald_lib, workdir, precision):
    d = make_case(workdir, 1, (8, 8, 8))
    p = getattr(ald_lib, precision)
    a = run(ald_lib, d, p, 1)
    b = run(ald_lib, d, p, 1)
    for k in KEYS:
        assert np.array_equal(a[k], b[k]), k


def test_deterministic_mixed_matches_default(ald_lib, workdir):
    """The mixed path (FP32 weights and |V3|^2): the same FP64 terms, summed
    in fixed point by the deterministic form and with FP64 atomics by the
    default form; far inside the mixed path's own 1e-4 bars of each other."""
    d = make_case(workdir, 1, (6, 6, 6))
    a = run(ald_lib, d, ald_lib.MIXED, 1)
    r = run(ald_lib, d, ald_lib.MIXED)
    Q, Qr = a["Q"], r["Q"]
    assert np.all(np.abs(Q - Qr) <= 1e-6 * np.abs(Qr) + 1e-10 * np.abs(Qr).max())
    kr = np.abs(r["kappa_cg"]).max()
    assert np.abs(a["kappa_cg"] - r["kappa_cg"]).max() <= 1e-6 * kr


def test_deterministic_matches_oracle(oracle_lib, ald_lib, workdir):
    """The deterministic form against the oracle's job=1 run on the same
    eigenpairs: Q, Q_N, Q_U, kappa RTA and CG at the FP64 bar (1e-10, floor
    1e-12 / 1e-10 of the largest value), the same CG iteration count."""
    d = make_case(workdir, 1, (6, 6, 6))
    ref = oracle_lib.run_job1(d)
    ev, vec, vel = ref["O"].get_phonons()
    opt = ald_lib.default_options(precision=ald_lib.FP64, delta=ald_lib.DELTA_TETRA, deterministic=1)
    with ald_lib.Context(d, opt) as ctx:
        ctx.set_phonons(ev, vec, vel)
        out = ctx.kappa_pipeline(ref["tempk"])
    for k, rk in (("Q", "Q"), ("QN", "QN"), ("QU", "QU")):
        r = ref[rk]
        assert np.all(np.abs(out[k] - r) <= 1e-10 * np.abs(r) + 1e-12 * np.abs(r).max()), k
    kr, kc = ref["kappa_rta"].sum(0), ref["kappa_cg"].sum(0)
    assert np.allclose(out["kappa_rta"], kr, rtol=1e-10, atol=1e-10 * np.abs(kr).max())
    assert out["cg_iters"] == ref["cg_iters"]
    assert np.allclose(out["kappa_cg"], kc, rtol=1e-10, atol=1e-10 * np.abs(kc).max())
