"""The oracle's update_mpi (THERMACOND/sub.f90:2295-2449, restated literally
over IBZ q2 and star arms) against the band-marginal form the GPU kernel
evaluates, on CPU:

    A(q1,l1) = sum_q sum_l R1'(q,l1,l) F(q1+q,l) - R1(q,l1,l) F(q,l)
                         + (R2(q,l1,l) F(q,l) + R2'(q,l1,l) F(q1-q,l)) / 2,

R = sum_l3 P, R' = sum_l2 P, F(q,l) = S_op(q) FFF(ibz(q),l) with op(q) the op
of q's arm in kstarsinfbz1 of its IBZ point.  Equal up to summation order.
Also: the job=3 iteration converges within its 150 steps."""
import numpy as np
import pytest

from conftest import make_case


def marginal_form(O, ref, F):
    nkc, nibz, b = O.nkc, O.nibz, O.ndyn
    I = O.ibz()
    kpc = O.kpc()
    opk = O.op_kmatrix()  # (n, 3, 3) row-major
    full = np.zeros((nkc, b, 3))
    for n in range(nibz):
        st, ops = O.getstar(I["kibz"][:, n], fbz=True)
        for k in range(st.shape[0]):
            q = O.get_k_info(st[k])[0] - 1
            for l in range(b):
                full[q, l] = opk[ops[k] - 1] @ F[n, l]
    P1, P2 = ref["P1"], ref["P2"]
    R1, R1p = P1.sum(axis=4), P1.sum(axis=3)
    R2, R2p = P2.sum(axis=4), P2.sum(axis=3)
    out = np.zeros((nibz, b, 3))
    for n1 in range(nibz):
        q1 = I["mapinv"][n1] - 1
        for q in range(nkc):
            qp = O.get_k_info(kpc[:, q1] + kpc[:, q])[0] - 1
            qm = O.get_k_info(kpc[:, q1] - kpc[:, q])[0] - 1
            for l1 in range(b):
                out[n1, l1] += (R1p[n1, q, l1] @ full[qp] - R1[n1, q, l1] @ full[q] +
                                0.5 * (R2[n1, q, l1] @ full[q] + R2p[n1, q, l1] @ full[qm]))
    return ref["FFF"] + out / ref["Q"][:, :, None]


@pytest.mark.parametrize("cfg,mesh,kw", [(1, (4, 4, 4), {}), (0, (4, 4, 4), {"delta": "gauss"})])
def test_update_mpi_equals_marginal_form(oracle_lib, workdir, cfg, mesh, kw):
    d = make_case(workdir, cfg, mesh, **kw)
    ref = oracle_lib.run_job1(d)
    O = ref["O"]
    rng = np.random.default_rng(3)
    F = ref["FFF"] * (1 + 0.1 * rng.standard_normal(ref["FFF"].shape))
    got = O.update_mpi(1, O.nibz, ref["P1"], ref["P2"], ref["Q"], ref["FFF"], F)
    want = marginal_form(O, ref, F)
    scale = np.abs(want).max()
    assert np.abs(got - want).max() <= 1e-11 * scale


def test_iterative_bte_converges(oracle_lib, workdir):
    d = make_case(workdir, 1, (4, 4, 4))
    ref = oracle_lib.run_job1(d)
    O = ref["O"]
    F, kap, iters, normk = O.iterative(ref["tempk"], ref["P1"], ref["P2"], ref["Q"], ref["FFF"])
    assert 1 <= iters < 150 and normk < 1e-4
    k = np.diag(kap.sum(0))
    assert np.all(np.isfinite(k)) and np.all(k > 0)
