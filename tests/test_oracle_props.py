"""Known-answer and property checks of the oracle and the input generators (CPU)."""
import numpy as np
import pytest

from conftest import make_case


@pytest.mark.parametrize("cfg,mesh,nibz", [(0, (10, 10, 10), 85), (1, (16, 16, 16), 276), (2, (32, 32, 32), 1768)])
def test_ibz_sizes_of_the_workloads(oracle_lib, workdir, cfg, mesh, nibz):
    d = make_case(workdir, cfg, mesh)
    O = oracle_lib.Oracle(d)
    assert O.mesh() == nibz
    assert O.npg == 48


@pytest.mark.parametrize("cfg", [0, 1])
def test_acoustic_sum_rule_gamma(oracle_lib, workdir, cfg):
    d = make_case(workdir, cfg, (4, 4, 4))
    O = oracle_lib.Oracle(d)
    ev, _ = O.get_freq(np.zeros(3))
    assert np.all(np.abs(ev[:3]) < 1e-12 * np.abs(ev).max() + 1e-14)
    assert np.all(ev[3:] > 1e-3 * np.abs(ev).max()) if O.ndyn > 3 else True


def test_jacobi_matches_lapack_zheev(oracle_lib, workdir):
    from scipy.linalg import lapack
    d = make_case(workdir, 1, (4, 4, 4))
    O = oracle_lib.Oracle(d)
    O.mesh()
    rng = np.random.default_rng(7)
    kpc = O.kpc()
    for n in rng.choice(O.nkc, 12, replace=False):
        q = kpc[:, n] + rng.normal(scale=1e-2, size=3)
        D = O.dynmat(q)
        H = np.triu(D) + np.triu(D, 1).conj().T
        H[np.diag_indices_from(H)] = D.diagonal().real
        w, v, info = lapack.zheev(H)
        assert info == 0
        ev, vec = O.get_freq(q)
        assert np.allclose(np.sort(np.abs(w)), ev, rtol=1e-12, atol=1e-14 * np.abs(w).max())


def test_weight_tet_corner_map_is_a_permutation(oracle_lib):
    """Every tie pattern of four corner energies assigns all four corners."""
    import itertools
    vals = [1.0, 2.0, 3.0, 4.0]
    before = oracle_lib.weight_tet_nonperm()
    for pat in itertools.product(range(4), repeat=4):
        w = np.array([vals[p] for p in pat])
        for e in (0.5, 1.0, 1.5, 2.5, 3.5, 4.0, 5.0):
            c = oracle_lib.weight_tet(w, e)
            assert not np.any(c == -12345.0)
    assert oracle_lib.weight_tet_nonperm() == before


def test_weight_tet_sum_is_tetrahedron_dos(oracle_lib):
    """sum_k c_k equals the linear-tetrahedron density of states g(e)."""
    rng = np.random.default_rng(3)
    for _ in range(300):
        w = rng.uniform(-5, 5, size=4)
        e1, e2, e3, e4 = np.sort(np.float32(w)).astype(float)
        e = rng.uniform(e1 - 0.2, e4 + 0.2)
        c = oracle_lib.weight_tet(w, e)
        if e < e1 or e > e4:
            g = 0.0
        elif e <= e2:
            g = 3 * (e - e1) ** 2 / ((e2 - e1) * (e3 - e1) * (e4 - e1))
        elif e <= e3:
            g = 3 * ((e2 - e1) + 2 * (e - e2) - (e3 - e1 + e4 - e2) * (e - e2) ** 2 / ((e3 - e2) * (e4 - e2))) / \
                ((e3 - e1) * (e4 - e1))
        else:
            g = 3 * (e4 - e) ** 2 / ((e4 - e1) * (e4 - e2) * (e4 - e3))
        assert abs(c.sum() - g) <= 1e-4 * max(abs(g), 1e-3)


def test_cg_quadratic_solves_spd(oracle_lib):
    rng = np.random.default_rng(1)
    n = 40
    A = rng.normal(size=(n, n))
    A = A @ A.T + n * np.eye(n)
    b = rng.normal(size=n)
    x, fm, it = oracle_lib.Oracle.cg(None, A, b, np.zeros(n), max_iter=200, ndig=6) if False else (None, None, None)
    O = oracle_lib.lib()
    import ctypes as C
    xx = np.zeros(n)
    fmin = C.c_double(0)
    Af = np.asfortranarray(A)
    it = O.orc_cg(n, Af.ctypes.data_as(oracle_lib.dp), np.ascontiguousarray(b).ctypes.data_as(oracle_lib.dp),
                  xx.ctypes.data_as(oracle_lib.dp), C.byref(fmin), 200, 6, 2)
    assert it < 200
    assert np.allclose(A @ xx, b, rtol=1e-5, atol=1e-6)


def test_small_case_end_to_end_is_finite(oracle_lib, workdir):
    d = make_case(workdir, 1, (4, 4, 4))
    r = oracle_lib.run_job1(d)
    assert np.all(np.isfinite(r["kappa_cg"]))
    kd = np.diag(r["kappa_cg"].sum(0))
    assert np.all(kd > 0)
    # cubic crystal: kappa isotropic within the CG tolerance
    assert np.ptp(kd) < 0.05 * kd.mean()


def test_get_k_info_has_no_state_across_oracles(oracle_lib, workdir):
    """get_k_info folds with the dual basis of the State it is given: oracles of
    crystals with different lattice constants, created and freed one after the
    other (so a new State may reuse a freed one's address), keep exact mesh
    index round trips."""
    dirs = [make_case(workdir, 1, (8, 8, 8)), make_case(workdir, 0, (8, 8, 8))]
    kpcs = {}
    for d in dirs:
        O = oracle_lib.Oracle(d)
        O.mesh()
        kpcs[d] = O.kpc()
        del O
    for rep in range(16):
        d = dirs[rep % 2]
        O = oracle_lib.Oracle(d)
        kpc = kpcs[d]
        idx = [O.get_k_info(kpc[:, n])[0] for n in range(kpc.shape[1])]
        assert idx == list(range(1, kpc.shape[1] + 1))
        del O


def _v3_case(oracle_lib, workdir, cfg, mesh, **kw):
    d = make_case(workdir, cfg, mesh, **kw)
    O = oracle_lib.Oracle(d)
    O.mesh()
    R = O.ibz()
    O.phonons()
    ev, _, _ = O.get_phonons()
    v = O.v3(1, O.nibz)
    kpc = O.kpc()
    gam = {q for q in range(O.nkc) if np.abs(kpc[:, q]).max() < 1e-9}
    q3 = np.array([[O.get_k_info(-kpc[:, R["mapinv"][n1] - 1] - kpc[:, q2])[0] - 1 for q2 in range(O.nkc)]
                   for n1 in range(O.nibz)])
    return O, R, ev, v, kpc, gam, q3


def _gamma_acoustic(b, gam, qs):
    """Mask (l1, l2, l3) of the entries with an acoustic mode at Gamma: 0/0
    in exact arithmetic (the reference zeroes them downstream)."""
    m = np.ones((b, b, b), bool)
    for ax, q in enumerate(qs):
        if q in gam:
            idx = [slice(None)] * 3
            idx[ax] = slice(0, 3)
            m[tuple(idx)] = False
    return m


@pytest.mark.parametrize("cfg,mesh", [(1, (4, 4, 4)), (0, (5, 5, 5))])
def test_v3_symmetric_in_q2_q3(oracle_lib, workdir, cfg, mesh):
    """matrix_elt_simplified (sub.f90:5888-6011) with FC3 symmetric in its
    atom/direction pairs gives V3(q1l1, q2l2, q3l3) = V3(q1l1, q3l3, q2l2):
    the oracle's |V3|^2 at (q2, l2, l3) equals that at (q3, l3, l2)."""
    O, R, ev, v, kpc, gam, q3 = _v3_case(oracle_lib, workdir, cfg, mesh)
    b, scale = O.ndyn, np.abs(v).max()
    for n1 in range(O.nibz):
        q1 = R["mapinv"][n1] - 1
        for q2 in range(O.nkc):
            a, c = v[n1, q2], v[n1, q3[n1, q2]].transpose(0, 2, 1)
            m = _gamma_acoustic(b, gam, (q1, q2, q3[n1, q2]))
            assert np.all(np.abs(a - c)[m] <= 1e-9 * np.abs(a)[m] + 1e-12 * scale), (n1, q2)


@pytest.mark.parametrize("cfg", [1, 0])
def test_v3_invariant_under_the_little_group_of_q1(oracle_lib, workdir, cfg):
    """|V3|^2 summed over degenerate groups of modes is a scalar of the
    lattice point group: for every op S with S q1 = q1 (mod G), the group
    sums at (q2, q3) and at (S q2, S q3) agree.  On a 4^3 mesh the reference's
    default-REAL mesh fractions m/4 are exact, so the mesh is exactly
    symmetric and the sums agree to rounding (on meshes such as 6^3 the
    fractions m/6 carry FP32 noise and the sums agree to about 1e-5 only)."""
    O, R, ev, v, kpc, gam, q3 = _v3_case(oracle_lib, workdir, cfg, (4, 4, 4))
    b, scale = O.ndyn, np.abs(v).max()
    tol = 1e-8 * np.abs(ev).max()

    def group_matrix(q):
        w, g, cur = ev[:, q], [], [0]
        for l in range(1, b):
            if abs(w[l] - w[cur[-1]]) <= tol:
                cur.append(l)
            else:
                g.append(cur)
                cur = [l]
        g.append(cur)
        P = np.zeros((len(g), b))
        for i, gg in enumerate(g):
            P[i, gg] = 1.0
        return P, np.array([(q in gam) and gg[0] < 3 for gg in g])

    GM = [group_matrix(q) for q in range(O.nkc)]
    ops = O.op_kmatrix()
    checked = 0
    for n1 in range(O.nibz):
        q1 = R["mapinv"][n1] - 1
        for S in ops:
            if O.get_k_info(S @ kpc[:, q1])[0] - 1 != q1:
                continue
            for q2 in range(O.nkc):
                s2 = O.get_k_info(S @ kpc[:, q2])[0] - 1
                sums = []
                for qa, qb in ((q2, q3[n1, q2]), (s2, q3[n1, s2])):
                    (P1, a1), (P2, a2), (P3, a3) = GM[q1], GM[qa], GM[qb]
                    t = np.einsum("ai,bj,ck,ijk->abc", P1, P2, P3, v[n1, qa])
                    t[a1] = np.nan
                    t[:, a2] = np.nan
                    t[:, :, a3] = np.nan
                    sums.append(t)
                a, c = sums
                m = ~np.isnan(a)
                assert np.array_equal(m, ~np.isnan(c))
                assert np.all(np.abs(a - c)[m] <= 1e-9 * np.abs(a)[m] + 1e-12 * scale), (n1, q2, s2)
                checked += 1
    assert checked > O.nkc * O.nibz  # every row has ops beyond the identity


@pytest.mark.parametrize("cfg", [1, 0])
def test_rta_kappa_diagonal_is_isotropic(oracle_lib, workdir, cfg):
    """Cubic crystals: mode_kappa (sub.f90:1292-1401) sums every IBZ mode over
    its star arms with op_kmatrix, so the three diagonal entries of the RTA
    kappa tensor (summed over bands) agree to rounding.  With the Gaussian
    delta (argon) the off-diagonal entries vanish to rounding too; with the
    tetrahedron delta (rock-salt) they are about 2e-3 of the diagonal, since
    make_kp_reg_tet cuts every mesh cell into six tetrahedra around one cell
    diagonal, which breaks the cubic symmetry of Q.  (The CG kappa is not
    isotropic either way: the reference's stop rule, (num/den)^2 |p|^2/|x|^2
    < 1e-4, leaves the solution about 1 % from converged.)"""
    d = make_case(workdir, cfg, (4, 4, 4))
    r = oracle_lib.run_job1(d)
    K = r["kappa_rta"].sum(0)
    diag = np.diag(K)
    assert np.all(diag > 0)
    assert (diag.max() - diag.min()) <= 1e-12 * diag.mean()
    if cfg == 0:
        assert np.abs(K - np.diag(diag)).max() <= 1e-12 * diag.mean()
