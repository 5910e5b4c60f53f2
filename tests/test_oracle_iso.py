"""The oracle's isotope-scattering restatement (iso=1) on CPU.

cal_g (sub.f90:3766-4693) is checked against the mass-variance formula on
the element data it tabulates; P_iso_split (sub.f90:4825-4961) against a
literal Python loop over n2, l2, every tetrahedron and corner, with the
oracle's own weight_tet, so the folding of the reference's n2 loop (its body
does not use n2) is pinned to the loop as written.
"""
import numpy as np

import oracle_py
from conftest import make_case


def mass_variance(iso):
    m = np.array([x[0] for x in iso])
    f = np.array([x[1] for x in iso])
    mave = (m * f).sum() / 100
    return (f * (1 - m / mave) ** 2).sum() / 100


def test_cal_g(workdir):
    d = make_case(workdir, 1, (4, 4, 4), iso=1)
    O = oracle_py.Oracle(d)
    O.mesh()
    g = O.giso()
    # rock-salt: atom 1 Na (one stable isotope), atom 2 Cl
    assert g[0] == 0.0
    cl = mass_variance([(34.968853, 75.77), (36.965903, 24.23)])
    assert abs(g[1] - cl) <= 1e-15 * cl
    assert 5e-4 < g[1] < 6e-4  # natural chlorine, 5.9e-4


def test_p_iso_literal(workdir):
    d = make_case(workdir, 0, (4, 4, 4), iso=1)
    O = oracle_py.Oracle(d)
    O.mesh()
    O.phonons()
    corners = O.tet()  # (4, 6 nkc), 1-based mesh indices
    g = O.giso()
    assert g[0] > 0
    ev, vec, _ = O.get_phonons()
    freq, _ = O.distribution(300.0)
    Piso = O.p_iso(1, O.nibz, g)
    nkc, ndn = O.nkc, O.ndyn
    mapinv = O.ibz()["mapinv"]
    ref = np.zeros_like(Piso)
    for n1 in range(O.nibz):
        i = mapinv[n1] - 1
        for l1 in range(ndn):
            om1 = freq[i, l1]
            s = 0.0
            for n2 in range(nkc):  # the reference's loop; its body does not use n2
                if n2 > 0:
                    s += body
                    continue
                body = 0.0
                for l2 in range(ndn):
                    for t in range(corners.shape[1]):
                        w = corners[:, t] - 1
                        c = oracle_py.weight_tet(freq[w, l2], om1)
                        for k in range(4):
                            dots = [np.vdot(vec[3 * a:3 * a + 3, l1, i], vec[3 * a:3 * a + 3, l2, w[k]])
                                    for a in range(O.nat0)]
                            gs = sum(g[a] * abs(dots[a]) ** 2 for a in range(O.nat0))
                            body += gs * c[k] / 6.0
                s += body
            ref[n1, l1] = s * om1 ** 2 * np.pi / (2 * nkc)
    big = np.abs(ref) > 1e-12 * np.abs(ref).max()
    assert big.any()
    np.testing.assert_allclose(Piso[big], ref[big], rtol=1e-11)
    assert np.all(np.abs(Piso[~big]) <= 1e-12 * np.abs(ref).max())
