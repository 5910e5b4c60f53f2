"""ctypes access to the C++ oracle (oracle/_build/liboracle.so).

Test infrastructure: the oracle restates the reference's Fortran routines
and is used only as the checker (tests, smoke, bench CPU baseline).
Arrays follow the reference's Fortran layout; numpy arrays are created
with order='F' so indices read like the Fortran source.
"""
from __future__ import annotations

import ctypes as C
import os
import subprocess

import numpy as np

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
LIB = os.path.join(ROOT, "oracle", "_build", "liboracle.so")
_lib = None

dp = C.POINTER(C.c_double)
ip = C.POINTER(C.c_int)


def build():
    subprocess.check_call(["make", "-s", "-C", os.path.join(ROOT, "oracle")])


def lib():
    global _lib
    if _lib is None:
        if not os.path.exists(LIB):
            build()
        L = C.CDLL(LIB)
        L.orc_load.restype = C.c_void_p
        L.orc_load.argtypes = [C.c_char_p, C.c_char_p, C.c_int]
        L.orc_free.argtypes = [C.c_void_p]
        for name in ["orc_sizes", "orc_lattice", "orc_op_kmatrix", "orc_mesh", "orc_get_kpc", "orc_get_ibz",
                     "orc_get_k_info", "orc_getstar", "orc_kstars", "orc_dynmat", "orc_get_freq", "orc_phonons",
                     "orc_get_phonons", "orc_set_phonons", "orc_tet", "orc_v3", "orc_fgr", "orc_distribution",
                     "orc_tau", "orc_rta", "orc_collision", "orc_rhs", "orc_kappa_d", "orc_update_mpi",
                     "orc_iterative", "orc_giso", "orc_p_iso", "orc_collision_iso", "orc_mode_kappa_teff",
                     "orc_kappa_d_teff", "orc_make_kp_bs", "orc_frequencies_at", "orc_self_w",
                     "orc_check_inside_bz", "orc_fc3_terms"]:
            getattr(L, name).restype = C.c_int
        L.orc_weight_tet_nonperm.restype = C.c_long
        _lib = L
    return _lib


def _p(a, t=dp):
    return a.ctypes.data_as(t) if a is not None else None


class Oracle:
    def __init__(self, d: str, nthreads: int = 0):
        L = lib()
        err = C.create_string_buffer(512)
        h = L.orc_load(d.encode(), err, 512)
        if not h:
            raise RuntimeError("oracle load failed: " + err.value.decode())
        self.h = C.c_void_p(h)
        self.nthreads = nthreads or (os.cpu_count() or 1)
        self._sizes()

    def __del__(self):
        try:
            lib().orc_free(self.h)
        except Exception:
            pass

    def _sizes(self):
        s = np.zeros(12, dtype=np.int32)
        lib().orc_sizes(self.h, _p(s, ip))
        (self.ndyn, self.nkc, self.nibz, self.nt2, self.nt3, self.natoms, self.npg,
         n1, n2, n3, self.nat0, self.npos) = [int(x) for x in s]
        self.nc = (n1, n2, n3)

    def lattice(self):
        o = np.zeros(22)
        lib().orc_lattice(self.h, _p(o))
        return {"r": o[0:9].reshape(3, 3), "g": o[9:18].reshape(3, 3), "volume_r": o[18], "volume_g": o[19],
                "const33": o[20], "cnst": o[21]}

    def op_kmatrix(self):
        o = np.zeros((48, 3, 3))
        n = lib().orc_op_kmatrix(self.h, _p(o))
        # stored column-major per op -> transpose to (row, col)
        return np.array([o[i].T for i in range(n)])

    def mesh(self):
        n = lib().orc_mesh(self.h)
        self._sizes()
        return n

    def kpc(self):
        k = np.zeros((3, self.nkc), order="F")
        lib().orc_get_kpc(self.h, _p(k))
        return k

    def ibz(self):
        mapibz = np.zeros(self.nkc, dtype=np.int32)
        mapinv = np.zeros(self.nibz, dtype=np.int32)
        kibz = np.zeros((3, self.nibz), order="F")
        wibz = np.zeros(self.nibz)
        mappos = np.zeros(self.nkc, dtype=np.int32)
        lib().orc_get_ibz(self.h, _p(mapibz, ip), _p(mapinv, ip), _p(kibz), _p(wibz), _p(mappos, ip))
        return {"mapibz": mapibz, "mapinv": mapinv, "kibz": kibz, "wibz": wibz, "mappos": mappos}

    def get_k_info(self, q):
        o = np.zeros(5, dtype=np.int32)
        q = np.ascontiguousarray(q, dtype=float)
        lib().orc_get_k_info(self.h, _p(q), _p(o, ip))
        return tuple(int(x) for x in o)  # nk, i, j, k, inside

    def getstar(self, q, fbz=False):
        st = np.zeros((48, 3))
        ops = np.zeros(48, dtype=np.int32)
        q = np.ascontiguousarray(q, dtype=float)
        f = lib().orc_kstars if fbz else lib().orc_getstar
        n = f(self.h, _p(q), _p(st), _p(ops, ip))
        return st[:n].copy(), ops[:n].copy()

    def dynmat(self, q):
        d = np.zeros((self.ndyn, self.ndyn), dtype=complex, order="F")
        q = np.ascontiguousarray(q, dtype=float)
        lib().orc_dynmat(self.h, _p(q), d.ctypes.data_as(dp))
        return d

    def get_freq(self, q):
        ev = np.zeros(self.ndyn)
        vec = np.zeros((self.ndyn, self.ndyn), dtype=complex, order="F")
        q = np.ascontiguousarray(q, dtype=float)
        lib().orc_get_freq(self.h, _p(q), _p(ev), vec.ctypes.data_as(dp))
        return ev, vec

    def phonons(self):
        lib().orc_phonons(self.h, self.nthreads)

    def get_phonons(self):
        n, nk = self.ndyn, self.nkc
        ev = np.zeros((n, nk), order="F")
        vec = np.zeros((n, n, nk), dtype=complex, order="F")
        vel = np.zeros((3, n, nk), order="F")
        lib().orc_get_phonons(self.h, _p(ev), vec.ctypes.data_as(dp), _p(vel))
        return ev, vec, vel

    def set_phonons(self, ev, vec, vel):
        ev = np.asfortranarray(ev, dtype=float)
        vec = np.asfortranarray(vec, dtype=complex)
        vel = np.asfortranarray(vel, dtype=float)
        lib().orc_set_phonons(self.h, _p(ev), vec.ctypes.data_as(dp), _p(vel))

    def fc3_terms(self):
        """read_fc234's fc3 term list and the supercell atoms (1-based)."""
        nt, na, n0 = self.nt3, self.natoms, self.nat0
        iat = np.zeros((3, nt), dtype=np.int32, order="F")
        ixyz = np.zeros((3, nt), dtype=np.int32, order="F")
        fcs = np.zeros(nt)
        pos = np.zeros((3, na), order="F")
        cell0 = np.zeros(na, dtype=np.int32)
        mass0 = np.zeros(n0)
        lib().orc_fc3_terms(self.h, _p(iat, ip), _p(ixyz, ip), _p(fcs), _p(pos), _p(cell0, ip), _p(mass0))
        return {"iat": iat, "ixyz": ixyz, "fcs": fcs, "atompos": pos, "cell0": cell0, "mass0": mass0}

    def tet(self):
        c = np.zeros((4, 6 * self.nkc), dtype=np.int32, order="F")
        lib().orc_tet(self.h, _p(c, ip))
        return c

    def v3(self, k1, k2):
        n, nk = self.ndyn, self.nkc
        out = np.zeros((k2 - k1 + 1, nk, n, n, n), order="F")
        err = C.create_string_buffer(256)
        r = lib().orc_v3(self.h, k1, k2, _p(out), self.nthreads, err, 256)
        if r:
            raise RuntimeError(err.value.decode())
        return out

    def fgr(self, k1, k2, v33, gauss=False):
        P1 = np.zeros_like(v33, order="F")
        P2 = np.zeros_like(v33, order="F")
        v33 = np.asfortranarray(v33)
        lib().orc_fgr(self.h, k1, k2, _p(v33), _p(P1), _p(P2), int(gauss), self.nthreads)
        return P1, P2

    def distribution(self, tempk):
        f = np.zeros((self.nkc, self.ndyn), order="F")
        d = np.zeros((self.nkc, self.ndyn), order="F")
        e = lib().orc_distribution(self.h, C.c_double(tempk), _p(f), _p(d))
        if e:
            raise RuntimeError("nbe error %d" % e)
        return f, d

    def tau(self, k1, k2, tempk, P1s, P2s, want_p=True):
        ns = k2 - k1 + 1
        Q = np.zeros((ns, self.ndyn), order="F")
        QN = np.zeros_like(Q)
        QU = np.zeros_like(Q)
        P1 = np.zeros_like(P1s, order="F") if want_p else None
        P2 = np.zeros_like(P1s, order="F") if want_p else None
        lib().orc_tau(self.h, k1, k2, C.c_double(tempk), _p(np.asfortranarray(P1s)), _p(np.asfortranarray(P2s)),
                      _p(Q), _p(QN), _p(QU), _p(P1), _p(P2), self.nthreads)
        return Q, QN, QU, P1, P2

    def rta(self, tempk, Q):
        FFF = np.zeros((self.nibz, self.ndyn, 3), order="F")
        kap = np.zeros((self.ndyn, 3, 3), order="F")
        Q = np.asfortranarray(Q)
        e = lib().orc_rta(self.h, C.c_double(tempk), _p(Q), _p(FFF), _p(kap))
        if e:
            raise RuntimeError("nbe error %d" % e)
        return FFF, kap

    def collision(self, k1, k2, P1, P2):
        ns = k2 - k1 + 1
        CM = np.zeros((ns * self.ndyn * 3, self.nibz * self.ndyn * 3), order="F")
        lib().orc_collision(self.h, k1, k2, _p(np.asfortranarray(P1)), _p(np.asfortranarray(P2)), _p(CM),
                            self.nthreads)
        return CM

    def giso(self):
        """cal_giso (sub.f90:4695): g per primitive atom from the element names."""
        g = np.zeros(self.nat0)
        err = C.create_string_buffer(256)
        if lib().orc_giso(self.h, _p(g), err, 256):
            raise RuntimeError(err.value.decode())
        return g

    def p_iso(self, k1, k2, g):
        """P_iso_split (sub.f90:4825): Piso(nk1, ndyn) of rows k1..k2."""
        Piso = np.zeros((k2 - k1 + 1, self.ndyn), order="F")
        lib().orc_p_iso(self.h, k1, k2, _p(np.ascontiguousarray(g, dtype=float)), _p(Piso), self.nthreads)
        return Piso

    def collision_iso(self, P1, P2, Piso):
        """CollisionMatrix_iso (sub.f90:3387) over all IBZ rows."""
        n = self.nibz * self.ndyn * 3
        CM = np.zeros((n, n), order="F")
        f = lambda a: _p(np.asfortranarray(a, dtype=float))
        lib().orc_collision_iso(self.h, f(P1), f(P2), f(Piso), _p(CM), self.nthreads)
        return CM

    def rhs(self, tempk):
        r = np.zeros(self.nibz * self.ndyn * 3)
        lib().orc_rhs(self.h, C.c_double(tempk), _p(r))
        return r

    def cg(self, A, b, x0, max_iter=100, ndig=2):
        A = np.asfortranarray(A, dtype=float)
        x = np.array(x0, dtype=float)
        fmin = C.c_double(0)
        it = lib().orc_cg(A.shape[0], _p(A), _p(np.ascontiguousarray(b, dtype=float)), _p(x), C.byref(fmin),
                          max_iter, ndig, self.nthreads)
        return x, fmin.value, it

    def update_mpi(self, k1, k2, P1, P2, Q, F_RTA, FFF):
        """update_mpi (sub.f90:2295): F2(nk1, ndyn, 3) from Bose-weighted P1/P2 of rows k1..k2."""
        nr = k2 - k1 + 1
        F2 = np.zeros((nr, self.ndyn, 3), order="F")
        f = lambda a: _p(np.asfortranarray(a, dtype=float))
        lib().orc_update_mpi(self.h, k1, k2, f(P1), f(P2), f(Q), f(F_RTA), f(FFF), _p(F2), self.nthreads)
        return F2

    def iterative(self, tempk, P1, P2, Q, F_RTA, max_iter=150, mix=0.4):
        """The job=3 iteration (kappa.f90:1390-1487); returns (F, kappa(ndyn,3,3), iters, normk)."""
        F = np.zeros((self.nibz, self.ndyn, 3), order="F")
        kap = np.zeros((self.ndyn, 3, 3), order="F")
        it = C.c_int(0)
        nk = C.c_double(0)
        f = lambda a: _p(np.asfortranarray(a, dtype=float))
        e = lib().orc_iterative(self.h, C.c_double(tempk), f(P1), f(P2), f(Q), f(F_RTA), max_iter, C.c_double(mix),
                                _p(F), _p(kap), C.byref(it), C.byref(nk), self.nthreads)
        if e:
            raise RuntimeError("nbe error %d" % e)
        return F, kap, it.value, nk.value

    def mode_kappa_teff(self, tempk, FFF, teff=None, keep_all=False):
        """mode_kappa (sub.f90:1292) and the module array tauinv_eff(nibz,ndn)
        as it leaves it: only the last mode keeps its sum (keep_all: every
        mode keeps its own sum)."""
        kap = np.zeros((self.ndyn, 3, 3), order="F")
        t = np.zeros((self.nibz, self.ndyn), order="F") if teff is None else np.array(teff, dtype=float, order="F")
        e = lib().orc_mode_kappa_teff(self.h, C.c_double(tempk), _p(np.asfortranarray(FFF)), _p(kap), _p(t),
                                      int(keep_all))
        if e:
            raise RuntimeError("nbe error %d" % e)
        return kap, t

    def kappa_d_teff(self, tempk, x, teff):
        """mode_kappa_d (sub.f90:1407) adding to tauinv_eff (a copy of teff)."""
        kap = np.zeros((self.ndyn, 3, 3), order="F")
        t = np.array(teff, dtype=float, order="F")
        e = lib().orc_kappa_d_teff(self.h, C.c_double(tempk), _p(np.ascontiguousarray(x, dtype=float)), _p(kap),
                                   _p(t))
        if e:
            raise RuntimeError("nbe error %d" % e)
        return kap, t

    def make_kp_bs(self, d):
        """make_kp_bs (modules.f90:1507) from d/kpbs.params: kp_bs (3,nkp), dk_bs."""
        n = C.c_int(0)
        err = C.create_string_buffer(256)
        if lib().orc_make_kp_bs(self.h, d.encode(), C.byref(n), None, None, 0, err, 256):
            raise RuntimeError(err.value.decode())
        kp = np.zeros((3, n.value), order="F")
        dk = np.zeros(n.value)
        lib().orc_make_kp_bs(self.h, d.encode(), C.byref(n), _p(kp), _p(dk), n.value, err, 256)
        return kp, dk

    def frequencies_at(self, kp):
        """get_frequencies at the points kp (3,np): eival (ndyn,np), eivec."""
        kp = np.asfortranarray(kp, dtype=float)
        np_ = kp.shape[1]
        ev = np.zeros((self.ndyn, np_), order="F")
        vec = np.zeros((self.ndyn, self.ndyn, np_), dtype=complex, order="F")
        lib().orc_frequencies_at(self.h, np_, _p(kp), _p(ev), vec.ctypes.data_as(dp), self.nthreads)
        return ev, vec

    def self_w(self, q, la, omega, temp, gauss=False):
        """function_self_w3 (gauss False) / function_self_w4 (True) per job:
        q (3,n), la (n, 1-based), omega (n) and temp in cm^-1.  Returns
        nself, uself (n,) complex."""
        q = np.asfortranarray(q, dtype=float)
        n = q.shape[1]
        la = np.ascontiguousarray(la, dtype=np.int32)
        om = np.ascontiguousarray(omega, dtype=float)
        out = np.zeros((4, n), order="F")
        e = lib().orc_self_w(self.h, n, _p(q), _p(la, ip), _p(om), C.c_double(temp), int(gauss), _p(out),
                             self.nthreads)
        if e:
            raise RuntimeError("self-energy error %d" % e)
        return out[0] + 1j * out[1], out[2] + 1j * out[3]

    def check_inside_bz(self, q):
        return lib().orc_check_inside_bz(self.h, _p(np.ascontiguousarray(q, dtype=float)))

    def kappa_d(self, tempk, x):
        kap = np.zeros((self.ndyn, 3, 3), order="F")
        e = lib().orc_kappa_d(self.h, C.c_double(tempk), _p(np.ascontiguousarray(x, dtype=float)), _p(kap))
        if e:
            raise RuntimeError("nbe error %d" % e)
        return kap


def weight_tet(w, e):
    c = np.zeros(4)
    w = np.ascontiguousarray(w, dtype=float)
    lib().orc_weight_tet(_p(w), C.c_double(e), _p(c))
    return c


def weight_tet_nonperm() -> int:
    return int(lib().orc_weight_tet_nonperm())


def run_job1(d: str, tempk=None, gauss=None, k1=1, k2=None, phonons=None, nthreads=0):
    """The whole job=1 sequence of kappa.f90:389-871 on the oracle.

    Returns a dict with every intermediate array.  `phonons` =
    (eigenval, eigenvec, veloc) injects eigenpairs in place of the oracle's
    own eigensolver.  `gauss` switches the delta to the Gaussian extension.
    """
    O = Oracle(d, nthreads)
    O.mesh()
    if phonons is None:
        O.phonons()
    else:
        O.set_phonons(*phonons)
    O.tet()
    k2 = k2 or O.nibz
    if tempk is None:
        tempk = float(open(os.path.join(d, "latdyn.params")).read().split("\n")[6].split()[0])
    if gauss is None:
        gauss = False
        bp = os.path.join(d, "b200.params")
        if os.path.exists(bp):
            gauss = "delta gauss" in open(bp).read()
    v33 = O.v3(k1, k2)
    P1s, P2s = O.fgr(k1, k2, v33, gauss=gauss)
    freq, dist = O.distribution(tempk)
    Q, QN, QU, P1, P2 = O.tau(k1, k2, tempk, P1s, P2s)
    out = {"O": O, "v33": v33, "P1s": P1s, "P2s": P2s, "freq": freq, "dist": dist, "Q": Q, "QN": QN, "QU": QU,
           "P1": P1, "P2": P2, "tempk": tempk}
    # iso=1 (latdyn.params line 11): calculate_tauRTA_iso adds Piso to Q, Q_N
    # and Q_U (sub.f90:8311-8549); the collision matrix is CollisionMatrix_iso
    iso = int(open(os.path.join(d, "latdyn.params")).read().split("\n")[10].split()[0]) == 1
    if iso:
        g = O.giso()
        Piso = O.p_iso(k1, k2, g)
        out.update({"giso": g, "Piso": Piso, "Q3": Q.copy()})
        Q, QN, QU = Q + Piso, QN + Piso, QU + Piso
        out.update({"Q": Q, "QN": QN, "QU": QU})
    if k1 == 1 and k2 == O.nibz:
        FFF, krta = O.rta(tempk, Q)
        CM = O.collision_iso(P1, P2, out["Piso"]) if iso else O.collision(k1, k2, P1, P2)
        RHS = O.rhs(tempk)
        x0 = np.array([FFF[i, j, k] for i in range(O.nibz) for j in range(O.ndyn) for k in range(3)])
        x, fmin, it = O.cg(CM, RHS, x0)
        kd = O.kappa_d(tempk, x)
        out.update({"FFF": FFF, "kappa_rta": krta, "CM": CM, "RHS": RHS, "x0": x0, "x": x, "cg_iters": it,
                    "kappa_cg": kd})
    return out
