"""Oracle results for the rock-salt Morse crystal on its 16x16x16 mesh.

The benchmark workload (2 atoms, 6 bands, 276 IBZ points, tetrahedron
delta) takes the oracle about 2 CPU-hours: its V3 loops over every FC3 term
for every band triplet, as matrix_elt_simplified does (sub.f90:5888-6011).
That is too slow for a test, so this script runs the whole job=1 sequence
once (V3, FGR, tauRTA, RTA kappa, collision matrix, RHS, cg_quadratic,
mode_kappa_d) at 100, 300 and 600 K and stores the results in
tests/golden/nacl_morse_mesh16.npz:

    T                      the temperatures (K)
    ev_sum, ev_sumsq       checks of the oracle's eigenvalues, so a test can
                           tell that it injects the same eigenpairs
    Q_<T>, QN_<T>, QU_<T>  (nibz, ndyn) linewidth sums of calculate_tauRTA_mpi2
    kappa_rta_<T>          (ndyn, 3, 3) mode_kappa
    kappa_cg_<T>           (ndyn, 3, 3) mode_kappa_d of the CG solution
    x_<T>                  the CG solution, cg_iters_<T> its iteration count

The inputs are the files that tests/conftest.py's make_case writes for
configuration 1 on the 16^3 mesh; the GPU tests recompute the oracle's
eigenpairs (0.2 s) and inject them, so that both sides start from the same
phonons.  Usage (about 15 minutes on 8 threads):

    python tests/golden/make_oracle_fixtures.py [nthreads]
"""
import os
import sys
import tempfile
import time

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(os.path.dirname(HERE))
sys.path.insert(0, os.path.join(ROOT, "tests"))
sys.path.insert(0, os.path.join(ROOT, "anharmonic-lattice-dynamics_b200", "python"))

import oracle_py  # noqa: E402
from conftest import make_case  # noqa: E402

TEMPS = (100.0, 300.0, 600.0)
OUT = os.path.join(HERE, "nacl_morse_mesh16.npz")


def main(nthreads: int = 0):
    oracle_py.build()
    wd = tempfile.mkdtemp()
    d = make_case(wd, 1, (16, 16, 16))
    O = oracle_py.Oracle(d, nthreads)
    O.mesh()
    O.phonons()
    O.tet()
    ev, _, _ = O.get_phonons()
    nibz, b = O.nibz, O.ndyn
    N = 3 * b * nibz
    out = {"T": np.array(TEMPS), "ev_sum": ev.sum(), "ev_sumsq": (ev * ev).sum()}
    Q = {T: np.zeros((nibz, b), order="F") for T in TEMPS}
    QN = {T: np.zeros((nibz, b), order="F") for T in TEMPS}
    QU = {T: np.zeros((nibz, b), order="F") for T in TEMPS}
    CM = {T: np.zeros((N, N), order="F") for T in TEMPS}
    chunk = 8
    t0 = time.time()
    for k1 in range(1, nibz + 1, chunk):
        k2 = min(nibz, k1 + chunk - 1)
        v33 = O.v3(k1, k2)
        P1s, P2s = O.fgr(k1, k2, v33, gauss=False)
        del v33
        for T in TEMPS:
            O.distribution(T)
            q, qn, qu, P1, P2 = O.tau(k1, k2, T, P1s, P2s)
            Q[T][k1 - 1:k2], QN[T][k1 - 1:k2], QU[T][k1 - 1:k2] = q, qn, qu
            CM[T][3 * b * (k1 - 1):3 * b * k2, :] = O.collision(k1, k2, P1, P2)
            del P1, P2
        print("rows %d-%d of %d, %.0f s" % (k1, k2, nibz, time.time() - t0), flush=True)
    for T in TEMPS:
        O.distribution(T)
        FFF, krta = O.rta(T, Q[T])
        RHS = O.rhs(T)
        x0 = np.array([FFF[i, j, k] for i in range(nibz) for j in range(b) for k in range(3)])
        x, _, it = O.cg(CM[T], RHS, x0)
        kd = O.kappa_d(T, x)
        t = "%d" % T
        out.update({"Q_" + t: Q[T], "QN_" + t: QN[T], "QU_" + t: QU[T], "kappa_rta_" + t: krta,
                    "kappa_cg_" + t: kd, "x_" + t: x, "cg_iters_" + t: it})
    np.savez_compressed(OUT, **out)
    print("wrote", OUT, os.path.getsize(OUT), "bytes")


if __name__ == "__main__":
    main(int(sys.argv[1]) if len(sys.argv) > 1 else 0)
