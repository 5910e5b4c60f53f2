"""The mixed-precision V3 path (ALD_MIXED) against the FP64 oracle (GPU).

ALD_MIXED runs the phase-class sums and the two eigenvector mode products of
V3 in FP32 with FP32 accumulation (for 3-band cells the class sums as
split-FP16 tensor-core MMAs); inside the pipeline the tetrahedron and
Gaussian delta weights are FP32 as well.  Eigenvalues, den = sqrt(8
sqrt|l1 l2 l3|), Bose factors, the sums into Q, the collision matrix, CG and
kappa stay FP64.  Tolerances (the targets of the mixed path):
  |V3|^2      normwise relative error <= 1e-4 (Gamma-acoustic 0/0 entries excluded)
  linewidths  |Q - Q_ref| <= 1e-4 |Q_ref| + 1e-8 max|Q_ref| for every mode
  kappa       every component of the RTA and CG tensors within 1e-4 of max|kappa|
The oracle's eigenpairs are injected so that only the V3 arithmetic differs.
"""
import numpy as np
import pytest

from conftest import make_case
from test_gpu_parity import gamma_acoustic_mask

pytestmark = pytest.mark.gpu


@pytest.mark.parametrize("cfg,mesh,kw", [(1, (6, 6, 6), {}), (0, (6, 6, 6), {"delta": "gauss"})],
                         ids=["nacl6_tetra", "lj6_gauss"])
def test_mixed_precision_errors(oracle_lib, ald_lib, workdir, cfg, mesh, kw):
    d = make_case(workdir, cfg, mesh, **kw)
    ref = oracle_lib.run_job1(d)
    O = ref["O"]
    ev, vec, vel = O.get_phonons()
    delta = ald_lib.DELTA_GAUSS if kw.get("delta") == "gauss" else ald_lib.DELTA_TETRA
    ctx = ald_lib.Context(d, ald_lib.default_options(precision=ald_lib.MIXED, delta=delta))
    ctx.set_phonons(ev, vec, vel)
    v = ctx.calculate_w3_ibz_split_sq([1, ctx.nibz])
    keep = ~gamma_acoustic_mask(O, ev, 1, ctx.nibz)
    r = ref["v33"][keep]
    err_v3 = np.linalg.norm(v[keep] - r) / np.linalg.norm(r)
    assert err_v3 <= 1e-4, err_v3
    out = ctx.kappa_pipeline(ref["tempk"])
    Q, Qr = out["Q"], ref["Q"]
    assert np.all(np.abs(Q - Qr) <= 1e-4 * np.abs(Qr) + 1e-8 * np.abs(Qr).max())
    for key, rk in (("kappa_rta", "kappa_rta"), ("kappa_cg", "kappa_cg")):
        k, kr = out[key], ref[rk].sum(0)
        assert np.abs(k - kr).max() <= 1e-4 * np.abs(kr).max(), (key, k, kr)
    ctx.close()


@pytest.mark.parametrize("cfg,mesh,kw", [
    (3, (3, 4, 4), {"p": 2, "rc_sigma": 1.2, "ibz": "none", "delta": "gauss"}),
    (3, (4, 4, 4), {"p": 1, "rc_sigma": 1.2, "delta": "gauss"}),
    (3, (4, 4, 4), {"p": 1, "rc_sigma": 1.2, "delta": "tetra"})],
    ids=["sl24_odd_mesh", "sl12_gauss", "sl12_tetra"])
def test_mixed_near_zero_modes(ald_lib, workdir, cfg, mesh, kw):
    """The mixed path against the FP64 path where modes of vanishing frequency
    enter: on the odd 3x4x4 mesh the reference's Gamma test (indices nc/2+1)
    misses Gamma, so the pairs with q2 or q3 at Gamma carry the acoustic modes'
    cancellation residue into the sums; at q1 = Gamma the acoustic linewidths
    are that residue.  The mixed path forms those pairs in FP64, so the linewidths
    of every other mode and kappa stay within the mixed bars of the FP64 path."""
    d = make_case(workdir, cfg, mesh, **kw)
    delta = ald_lib.DELTA_GAUSS if kw.get("delta") == "gauss" else ald_lib.DELTA_TETRA
    out = {}
    for prec in (ald_lib.FP64, ald_lib.MIXED):
        with ald_lib.Context(d, ald_lib.default_options(precision=prec, delta=delta)) as ctx:
            ev = ctx.get_frequencies()[0]
            mapinv = ctx.get_mesh()["mapinv"] - 1
            out[prec] = ctx.kappa_pipeline(ctx.info.tempk)
    f, m = out[ald_lib.FP64], out[ald_lib.MIXED]
    # linewidths of the IBZ modes whose frequency is not rounding noise
    soft = np.abs(ev[:, mapinv].T) < 1e-9 * np.abs(ev).max()
    Qf, Qm = f["Q"][~soft], m["Q"][~soft]
    assert np.all(np.abs(Qm - Qf) <= 1e-4 * np.abs(Qf) + 1e-8 * np.abs(Qf).max()), np.abs(Qm - Qf).max()
    for key in ("kappa_rta", "kappa_cg"):
        k, kr = m[key], f[key]
        assert np.abs(k - kr).max() <= 1e-4 * np.abs(kr).max(), (key, k, kr)
