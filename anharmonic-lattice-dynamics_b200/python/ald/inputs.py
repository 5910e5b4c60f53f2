"""Synthetic THERMACOND inputs written in the reference's own file formats.

The reference reads five positional text files (``latdyn.params``,
``structure.params``, ``lat_fc.dat``, ``fc2.dat``, ``fc3.dat``) plus
``dielectric.params`` and ``kpbs.params``.  The writers below follow the
*readers* of the reference, record by record:

* ``latdyn.params``   -> ``read_params``      THERMACOND/rest.f90:13-51
* ``structure.params``-> ``read_input_fit``   THERMACOND/rest.f90:87-130
* ``lat_fc.dat``      -> ``read_lattice``     THERMACOND/rest.f90:164-289
* ``fc2.dat``/``fc3.dat`` -> ``read_fc234``   THERMACOND/rest.f90:340-401
* ``dielectric.params`` -> ``read_born``      THERMACOND/rest.f90:3587-3598
* ``kpbs.params``     -> ``make_kp_bs``       THERMACOND/modules.f90:1525-1540

Force constants are the analytic second and third derivatives of a
central pair potential (Lennard-Jones or Morse) summed over the listed
neighbour shells, with the on-site blocks fixed by the acoustic sum rule.
Values are written with ``repr`` so the files hold the exact doubles.

Knobs that the reference files do not carry (delta form, precision, IBZ
rule, CG stop rule) go to a separate ``b200.params`` so the reference
files stay byte-compatible.
"""
from __future__ import annotations

import dataclasses
import math
import os
from typing import Callable, Dict, List, Optional, Sequence, Tuple

import numpy as np

THZ_TO_CM = 1e12 / 2.99792458e10  # 1 THz in cm^-1

# ----------------------------------------------------------------------------
# pair potentials: return (V', V'', V''') at distance r (eV, Angstrom)
# ----------------------------------------------------------------------------


def lennard_jones(eps: float, sigma: float) -> Callable[[float], Tuple[float, float, float]]:
    s6 = sigma ** 6
    s12 = s6 * s6

    def d(r: float):
        v1 = 4 * eps * (-12 * s12 / r ** 13 + 6 * s6 / r ** 7)
        v2 = 4 * eps * (156 * s12 / r ** 14 - 42 * s6 / r ** 8)
        v3 = 4 * eps * (-2184 * s12 / r ** 15 + 336 * s6 / r ** 9)
        return v1, v2, v3

    return d


def morse(D: float, alpha: float, r0: float) -> Callable[[float], Tuple[float, float, float]]:
    def d(r: float):
        ea = math.exp(-alpha * (r - r0))
        v1 = 2 * D * alpha * (ea - ea * ea)
        v2 = 2 * D * alpha ** 2 * (2 * ea * ea - ea)
        v3 = 2 * D * alpha ** 3 * (ea - 4 * ea * ea)
        return v1, v2, v3

    return d


def pair_fc2(R: np.ndarray, dv) -> np.ndarray:
    """phi_{i alpha, j beta} for the pair i->j separated by R (j != i)."""
    r = float(np.linalg.norm(R))
    n = R / r
    v1, v2, _ = dv(r)
    return -(v2 * np.outer(n, n) + (v1 / r) * (np.eye(3) - np.outer(n, n)))


def pair_v3(R: np.ndarray, dv) -> np.ndarray:
    """Third derivative tensor d^3 V(|R|)/dR_a dR_b dR_c of a central potential."""
    r = float(np.linalg.norm(R))
    n = R / r
    v1, v2, v3 = dv(r)
    A = v2 - v1 / r
    Ap = v3 - v2 / r + v1 / (r * r)
    d = np.eye(3)
    t = (Ap - 2 * A / r) * np.einsum("a,b,c->abc", n, n, n)
    t += (A / r) * (np.einsum("ab,c->abc", d, n) + np.einsum("ac,b->abc", d, n)
                    + np.einsum("bc,a->abc", d, n))
    return t


# ----------------------------------------------------------------------------
# structure description
# ----------------------------------------------------------------------------


@dataclasses.dataclass
class Structure:
    """A crystal with pairwise interactions.

    conv_abc / prim_in_conv / conv_lattice_parameter follow structure.params:
    latticeparameters (a,b,c,alpha,beta,gamma) are multiplied by
    lattice_parameter; primitivelattice(:,j) is the j-th primitive vector in
    units of the conventional vectors.  Atom positions are reduced
    coordinates of the conventional cell.
    """
    name: str
    conv_abc: Tuple[float, float, float]
    prim_in_conv: np.ndarray            # 3x3, column j = primitive vector j
    lattice_parameter: float
    atom_types: List[int]               # 1-based type per primitive atom
    atom_red_conv: List[Tuple[float, float, float]]
    type_masses: List[float]
    type_names: List[str]
    # list of (type_i, type_j, rmin, rmax, potential-derivative function)
    pairs: List[Tuple[int, int, float, float, Callable]]
    # optional per-atom masses overriding the per-type ones (superlattices)
    atom_masses: Optional[List[float]] = None

    @property
    def conv_to_cart(self) -> np.ndarray:
        a, b, c = (x * self.lattice_parameter for x in self.conv_abc)
        return np.diag([a, b, c])

    @property
    def prim_cart(self) -> np.ndarray:
        """rows: r1, r2, r3 in Cartesian Angstrom."""
        return (self.conv_to_cart @ self.prim_in_conv).T

    def atom_cart(self) -> np.ndarray:
        c = self.conv_to_cart
        return np.array([c @ np.array(p, dtype=float) for p in self.atom_red_conv])


def _interaction(st: Structure, ti: int, tj: int, r: float):
    for (a, b, rmin, rmax, dv) in st.pairs:
        if {a, b} == {ti, tj} and (a == ti and b == tj or a == tj and b == ti):
            if rmin - 1e-6 <= r <= rmax + 1e-6:
                return dv
    return None


def build_force_constants(st: Structure):
    """Enumerate neighbours and compute FC2/FC3 term lists.

    Returns dict with: r (3x3 rows r1..r3), atoms (list of
    (pos, j0, n1, n2, n3)), fc2 terms [(i,a,j,b,val)], fc3 terms
    [(i,a,j,b,k,c,val)], all indices 1-based as in the reference files.
    """
    R = st.prim_cart
    tau = st.atom_cart()
    nat0 = len(tau)
    types = st.atom_types
    rmax = max(p[3] for p in st.pairs) + 1e-6
    # enough cells to cover rmax
    inv = np.linalg.inv(R.T)
    span = int(math.ceil(rmax * max(np.linalg.norm(inv, axis=1)))) + 2
    neigh: Dict[int, List[Tuple[int, Tuple[int, int, int], np.ndarray, Callable]]] = {}
    for i0 in range(nat0):
        lst = []
        for n1 in range(-span, span + 1):
            for n2 in range(-span, span + 1):
                for n3 in range(-span, span + 1):
                    Rv = n1 * R[0] + n2 * R[1] + n3 * R[2]
                    for j0 in range(nat0):
                        d = tau[j0] + Rv - tau[i0]
                        r = float(np.linalg.norm(d))
                        if r < 1e-8 or r > rmax:
                            continue
                        dv = _interaction(st, types[i0], types[j0], r)
                        if dv is None:
                            continue
                        lst.append((j0, (n1, n2, n3), d, dv))
        lst.sort(key=lambda x: (round(float(np.linalg.norm(x[2])), 8), x[0], x[1]))
        neigh[i0] = lst
    # supercell atom list: primitive atoms first, then every neighbour once
    atoms: List[Tuple[np.ndarray, int, int, int, int]] = []
    index: Dict[Tuple[int, Tuple[int, int, int]], int] = {}
    for j0 in range(nat0):
        index[(j0, (0, 0, 0))] = len(atoms) + 1
        atoms.append((tau[j0].copy(), j0 + 1, 0, 0, 0))
    extra = []
    for i0 in range(nat0):
        for (j0, n, d, dv) in neigh[i0]:
            key = (j0, n)
            if key not in index and key not in [e[0] for e in extra]:
                pos = tau[j0] + n[0] * R[0] + n[1] * R[1] + n[2] * R[2]
                extra.append((key, pos))
    extra.sort(key=lambda e: (round(float(np.linalg.norm(e[1])), 8), e[0][0], e[0][1]))
    for key, pos in extra:
        index[key] = len(atoms) + 1
        atoms.append((pos, key[0] + 1, key[1][0], key[1][1], key[1][2]))

    fc2: List[Tuple[int, int, int, int, float]] = []
    fc3: List[Tuple[int, int, int, int, int, int, float]] = []
    for i0 in range(nat0):
        ii = i0 + 1
        onsite2 = np.zeros((3, 3))
        onsite3 = np.zeros((3, 3, 3))
        blocks3 = []
        for (j0, n, d, dv) in neigh[i0]:
            jj = index[(j0, n)]
            phi = pair_fc2(d, dv)
            for a in range(3):
                for b in range(3):
                    v = float(phi[a, b])
                    fc2.append((ii, a + 1, jj, b + 1, v))
                    onsite2[a, b] -= v
            v3 = pair_v3(d, dv)
            blocks3.append((jj, v3))
        for a in range(3):
            for b in range(3):
                fc2.append((ii, a + 1, ii, b + 1, float(onsite2[a, b])))
        for (jj, v3) in blocks3:
            for (sgn, t1, t2) in ((-1.0, jj, jj), (1.0, ii, jj), (1.0, jj, ii)):
                for a in range(3):
                    for b in range(3):
                        for c in range(3):
                            fc3.append((ii, a + 1, t1, b + 1, t2, c + 1, sgn * float(v3[a, b, c])))
            onsite3 -= v3
        for a in range(3):
            for b in range(3):
                for c in range(3):
                    fc3.append((ii, a + 1, ii, b + 1, ii, c + 1, float(onsite3[a, b, c])))
    return {"r": R, "atoms": atoms, "fc2": fc2, "fc3": fc3, "nat0": nat0}


# ----------------------------------------------------------------------------
# writers
# ----------------------------------------------------------------------------


def _f(x: float) -> str:
    return repr(float(x))


@dataclasses.dataclass
class RunParams:
    mesh: Tuple[int, int, int]
    tempk: float = 300.0
    width_cm: float = 0.1 * THZ_TO_CM   # Gaussian width (cm^-1), extension only
    etaz: float = 1.0
    wmesh: int = 200
    wmax: float = 500.0
    job: int = 1
    iso: int = 0
    classical: int = 0
    # b200.params knobs
    delta: str = "tetra"        # tetra | gauss
    precision: str = "fp64"     # fp64 | mixed
    ibz: str = "lattice"        # lattice | none
    cg_stop: str = "reference"  # reference | residual
    cg_tol: float = 1e-8


def write_inputs(st: Structure, rp: RunParams, out_dir: str) -> dict:
    """Write all reference input files for `st` into `out_dir`."""
    os.makedirs(out_dir, exist_ok=True)
    fc = build_force_constants(st)
    R = fc["r"]
    nat0 = fc["nat0"]
    masses = st.atom_masses or [st.type_masses[t - 1] for t in st.atom_types]
    ntypes = len(st.type_masses) if st.atom_masses is None else nat0
    # per-atom masses (superlattices) use one "type" per atom so that the
    # mass check of read_lattice holds exactly
    if st.atom_masses is not None:
        type_of_atom = list(range(1, nat0 + 1))
        tmass = list(st.atom_masses)
        tname = [st.type_names[t - 1] for t in st.atom_types]
    else:
        type_of_atom = list(st.atom_types)
        tmass = list(st.type_masses)
        tname = list(st.type_names)

    with open(os.path.join(out_dir, "latdyn.params"), "w") as f:
        f.write("%d %d %d .false.   mesh, dos_bs_only\n" % tuple(rp.mesh))
        f.write("0 0 0   shift\n")
        f.write("0 0 1   normald\n")
        f.write("%d %s   wmesh, wmax\n" % (rp.wmesh, _f(rp.wmax)))
        f.write("%s %s   width, etaz\n" % (_f(rp.width_cm), _f(rp.etaz)))
        f.write(".false.   verbose\n")
        f.write("%s %s 1   tmin tmax ntemp\n" % (_f(rp.tempk), _f(rp.tempk)))
        f.write("%d   job\n" % rp.job)
        f.write("10   ksub_size\n")
        f.write("./\n")
        f.write("%d   iso\n" % rp.iso)
        f.write("%d   classical\n" % rp.classical)
        f.write("0 0 0 0   calc_cross q_cross\n")
        f.write("1000   lmicron\n")

    with open(os.path.join(out_dir, "structure.params"), "w") as f:
        f.write("%s %s %s 90 90 90   lattice parameters\n" % tuple(_f(x) for x in st.conv_abc))
        pl = st.prim_in_conv
        f.write(" ".join(_f(pl[i, j]) for j in range(3) for i in range(3)) + "   primitive lattice\n")
        f.write("%s   lattice parameter\n" % _f(st.lattice_parameter))
        f.write("1 1 1 0   include_fc\n")
        f.write("1 1 0 0   invariances\n")
        f.write("0 300   temperature weighting\n")
        f.write("1 .false.   number of force files, verbosity\n")
        f.write("%d   natom_type\n" % len(tmass))
        f.write(" ".join(_f(m) for m in tmass) + "   masses\n")
        f.write(" ".join(tname) + "   names\n")
        f.write("%d   natoms0\n" % nat0)
        for _ in range(8):
            f.write("0   shells\n")
        conv = st.conv_to_cart
        for i in range(nat0):
            red = st.atom_red_conv[i]
            f.write("%d %d %s %s %s\n" % (i + 1, type_of_atom[i], _f(red[0]), _f(red[1]), _f(red[2])))

    atoms = fc["atoms"]
    fc2, fc3 = fc["fc2"], fc["fc3"]
    with open(os.path.join(out_dir, "lat_fc.dat"), "w") as f:
        f.write(" lattice and force-constant tables (synthetic %s)\n" % st.name)
        f.write("  Crystal data: translation vectors of the primitive cell\n")
        for k in range(3):
            f.write("  %s %s %s\n" % tuple(_f(x) for x in R[k]))
        f.write("  Crystal-data:atoms-in-primitive-cell\n")
        f.write("  %d\n" % nat0)
        for i in range(nat0):
            p = atoms[i][0]
            f.write("  %d %s %d %s %s %s %s\n" % (i + 1, tname[type_of_atom[i] - 1], type_of_atom[i],
                                                _f(p[0]), _f(p[1]), _f(p[2]), _f(tmass[type_of_atom[i] - 1])))
        f.write("  Included-ranks-of-FCs\n")
        f.write("  1 1 1 0\n")
        for _ in range(8):
            f.write("  shells-record\n")
        f.write("  Number-of-groups\n")
        f.write("  0 %d %d 0\n" % (len(fc2), len(fc3)))
        f.write("  Number-of-FCs-for-each-rank\n")
        f.write("  0 %d %d 0\n" % (len(fc2), len(fc3)))
        f.write("  skipped-record\n")
        f.write("  skipped-record\n")
        f.write("  maxshells,atoms:i,x,y,z,iatomcell0,n1,n2,n3\n")
        f.write("  8 %d\n" % len(atoms))
        for j, (p, j0, n1, n2, n3) in enumerate(atoms):
            f.write("  %d %s %s %s %d %d %d %d\n" % (j + 1, _f(p[0]), _f(p[1]), _f(p[2]), j0, n1, n2, n3))

    with open(os.path.join(out_dir, "fc2.dat"), "w") as f:
        f.write(" # RANK 2 tensors :term,group,(iatom,ixyz)_2\n")
        for t, (i, a, j, b, v) in enumerate(fc2):
            f.write("%d %d %d %d %d %d %s\n" % (t + 1, t + 1, i, a, j, b, _f(v)))
    with open(os.path.join(out_dir, "fc3.dat"), "w") as f:
        f.write(" # RANK 3 tensors :term,group,(iatom,ixyz)_3\n")
        for t, (i, a, j, b, k, c, v) in enumerate(fc3):
            f.write("%d %d %d %d %d %d %d %d %s\n" % (t + 1, t + 1, i, a, j, b, k, c, _f(v)))

    with open(os.path.join(out_dir, "dielectric.params"), "w") as f:
        f.write("0\n1 0 0\n0 1 0\n0 0 1\n")
        for _ in range(nat0):
            f.write("0 0 0\n0 0 0\n0 0 0\n")
    with open(os.path.join(out_dir, "kpbs.params"), "w") as f:
        f.write("0\n20\n2\nG 0 0 0\nX 0 0 1\nL 0.5 0.5 0.5\n")
    with open(os.path.join(out_dir, "b200.params"), "w") as f:
        f.write("delta %s\nprecision %s\nibz %s\ncg_stop %s\ncg_tol %s\nwidth_cm %s\n" % (
            rp.delta, rp.precision, rp.ibz, rp.cg_stop, _f(rp.cg_tol), _f(rp.width_cm)))
    return {"nterms2": len(fc2), "nterms3": len(fc3), "natoms": len(atoms), "nat0": nat0}


# ----------------------------------------------------------------------------
# the workloads
# ----------------------------------------------------------------------------

FCC_PRIM = np.array([[0.0, 0.5, 0.5], [0.5, 0.0, 0.5], [0.5, 0.5, 0.0]]).T  # columns


def lj_argon(a: float = 5.26, mass: float = 39.948, eps: float = 0.0104,
             sigma: float = 3.4, rc_sigma: float = 2.5) -> Structure:
    """fcc Lennard-Jones argon, 1-atom primitive cell, cutoff rc_sigma*sigma."""
    dv = lennard_jones(eps, sigma)
    return Structure(
        name="lj-argon-fcc", conv_abc=(1.0, 1.0, 1.0), prim_in_conv=FCC_PRIM.copy(),
        lattice_parameter=a, atom_types=[1], atom_red_conv=[(0.0, 0.0, 0.0)],
        type_masses=[mass], type_names=["Ar"],
        pairs=[(1, 1, 0.1, rc_sigma * sigma, dv)])


def rocksalt_morse(a: float = 5.64, mA: float = 22.99, mB: float = 35.45,
                   ab=(0.5, 1.2, 2.82), aa=(0.1, 1.0, 3.99), bb=(0.1, 1.0, 3.99)) -> Structure:
    """Rock-salt A-B with Morse pairs on the 1st (A-B) and 2nd (A-A, B-B) shells."""
    d1 = a / 2.0
    d2 = a / math.sqrt(2.0)
    return Structure(
        name="rocksalt-morse", conv_abc=(1.0, 1.0, 1.0), prim_in_conv=FCC_PRIM.copy(),
        lattice_parameter=a, atom_types=[1, 2], atom_red_conv=[(0.0, 0.0, 0.0), (0.5, 0.0, 0.0)],
        type_masses=[mA, mB], type_names=["Na", "Cl"],
        pairs=[(1, 2, d1 - 0.01, d1 + 0.01, morse(*ab)),
               (1, 1, d2 - 0.01, d2 + 0.01, morse(*aa)),
               (2, 2, d2 - 0.01, d2 + 0.01, morse(*bb))])


def lj_superlattice(p: int, seed: int, a: float = 5.26, eps: float = 0.0104,
                    sigma: float = 3.4, rc_sigma: float = 2.5) -> Structure:
    """fcc conventional cell stacked p x 1 x 1, layer masses U[20,80] amu."""
    rng = np.random.default_rng(seed)
    layer_mass = rng.uniform(20.0, 80.0, size=p)
    base = [(0.0, 0.0, 0.0), (0.0, 0.5, 0.5), (0.5, 0.0, 0.5), (0.5, 0.5, 0.0)]
    pos, masses = [], []
    for l in range(p):
        for b in base:
            pos.append(((b[0] + l) / p, b[1], b[2]))
            masses.append(float(layer_mass[l]))
    return Structure(
        name="lj-superlattice-p%d" % p, conv_abc=(float(p), 1.0, 1.0), prim_in_conv=np.eye(3),
        lattice_parameter=a, atom_types=[1] * len(pos), atom_red_conv=pos,
        type_masses=[39.948], type_names=["Ar"],
        pairs=[(1, 1, 0.1, rc_sigma * sigma, lennard_jones(eps, sigma))], atom_masses=masses)


def rocksalt_supercell(seed: int, a: float = 5.64) -> Structure:
    """The rock-salt Morse crystal in its 2x2x2 conventional supercell,
    relabelled as one 64-atom cubic cell (192 bands), with the seeded
    per-structure jitter of the batched benchmark: D +-20 %, alpha +-10 %
    (uniform, per pair type), the two masses uniform in [10, 130] amu."""
    rng = np.random.default_rng(seed)
    mA, mB = (float(x) for x in rng.uniform(10.0, 130.0, size=2))
    jit = lambda D, al, r0: (D * rng.uniform(0.8, 1.2), al * rng.uniform(0.9, 1.1), r0)
    ab, aa, bb = jit(0.5, 1.2, 2.82), jit(0.1, 1.0, 3.99), jit(0.1, 1.0, 3.99)
    fcc = [(0.0, 0.0, 0.0), (0.0, 0.5, 0.5), (0.5, 0.0, 0.5), (0.5, 0.5, 0.0)]
    pos, types = [], []
    for t, shift in ((1, (0.0, 0.0, 0.0)), (2, (0.5, 0.0, 0.0))):
        for i in range(2):
            for j in range(2):
                for k in range(2):
                    for f in fcc:
                        pos.append(((f[0] + shift[0] + i) / 2.0 % 1.0, (f[1] + shift[1] + j) / 2.0 % 1.0,
                                    (f[2] + shift[2] + k) / 2.0 % 1.0))
                        types.append(t)
    d1, d2 = a / 2.0, a / math.sqrt(2.0)
    return Structure(
        name="rocksalt-morse-2x2x2-s%d" % seed, conv_abc=(2.0, 2.0, 2.0), prim_in_conv=np.eye(3),
        lattice_parameter=a, atom_types=types, atom_red_conv=pos, type_masses=[mA, mB], type_names=["Na", "Cl"],
        pairs=[(1, 2, d1 - 0.01, d1 + 0.01, morse(*ab)),
               (1, 1, d2 - 0.01, d2 + 0.01, morse(*aa)),
               (2, 2, d2 - 0.01, d2 + 0.01, morse(*bb))])


# configurations of the benchmark suite (seeded synthetic stand-ins); seeds
# are 20261203 + structure index
BASE_SEED = 20261203


def config(n: int, mesh: Optional[Sequence[int]] = None, tempk: float = 300.0,
           rc_sigma: float = 2.5, p: int = 1, s: int = 0) -> Tuple[Structure, RunParams]:
    if n == 0:
        return lj_argon(), RunParams(mesh=tuple(mesh or (10, 10, 10)), tempk=tempk,
                                     width_cm=0.1 * THZ_TO_CM, delta="gauss")
    if n == 1:
        return rocksalt_morse(), RunParams(mesh=tuple(mesh or (16, 16, 16)), tempk=tempk, delta="tetra")
    if n == 2:
        return lj_argon(), RunParams(mesh=tuple(mesh or (32, 32, 32)), tempk=tempk,
                                     width_cm=0.05 * THZ_TO_CM, delta="gauss", cg_stop="residual",
                                     cg_tol=1e-8)
    if n == 3:
        # one structure of the batched suite: superlattice p (1: the 4-atom
        # conventional cell, 12 bands; up to 8: 96 bands), structure s,
        # mesh (ceil(12/p) >= 2) x 12 x 12
        m = mesh or (max(2, -(-12 // p)), 12, 12)
        return (lj_superlattice(p, seed=BASE_SEED + s, rc_sigma=rc_sigma),
                RunParams(mesh=tuple(m), tempk=tempk, width_cm=0.1 * THZ_TO_CM, delta="gauss"))
    if n == 4:
        # one structure of the batched mixed suite: the 64-atom rock-salt cell
        # (192 bands), structure s, 8 x 8 x 8 mesh, tetrahedron delta
        return (rocksalt_supercell(seed=BASE_SEED + s),
                RunParams(mesh=tuple(mesh or (8, 8, 8)), tempk=tempk, delta="tetra"))
    raise ValueError("unknown configuration %r" % n)
