"""Build golden fixtures from the outputs the reference shipped with its examples.

The reference ships two THERMACOND runs with their outputs:
``THERMACOND/Ge-example/kappa`` (fcc Ge, 2 atoms, 30x30x30 mesh) and
``THERMACOND/GeSe-example/kappa`` (orthorhombic GeSe, 8 atoms, 12x10x4).
Their inputs use an older file layout that the current readers do not
parse (latdyn.params lacks the ``normald`` record; structure.params has 4
shell records instead of 8; lat_fc.dat carries a "groups" record).  This
script re-lays the same numbers out (lattice, atoms, supercell positions,
FC2 terms) and keeps the reference's outputs that depend only on them:

* KPOINT.IBZ          IBZ points and weights (get_weights, modules.f90:2006)
* FBZ_freqs.dat       mesh frequencies (get_frequencies, rest.f90:2230; g11.5)
* RHS_IBZ.dat         the BTE right-hand side (cal_RHS_IBZ, sub.f90:2618),
                      full precision; it folds in frequencies, group
                      velocities (finitedif_vel) and Bose factors at 300 K
* tau_RTA.dat / veloc.dat  omega, n_BE and group velocities per mode

No example ships fc3.dat, so nothing here pins V3 or later stages.

Run in a container that has the reference mounted:
    python tests/golden/make_golden.py <path of the reference checkout>
It writes tests/golden/{ge,gese}_example.npz.
"""
from __future__ import annotations

import os
import sys

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))


def _toks(line):
    return line.replace(",", " ").split()


def _num(s):
    return float(s.replace("d", "e").replace("D", "E"))


def parse_example(d: str, n_shell_lines_old: int):
    sp = [l for l in open(os.path.join(d, "structure.params"))]
    it = iter(sp)
    latp = [_num(x) for x in _toks(next(it))[:6]]
    prim = [_num(x) for x in _toks(next(it))[:9]]
    scale = _num(_toks(next(it))[0])
    next(it)  # include_fc
    for _ in range(3):
        next(it)
    ntype = int(_toks(next(it))[0])
    mass_str = _toks(next(it))[:ntype]
    names = _toks(next(it))[:ntype]
    nat0 = int(_toks(next(it))[0])
    for _ in range(n_shell_lines_old):
        next(it)
    atoms = []
    for _ in range(nat0):
        t = _toks(next(it))
        atoms.append((int(t[0]), int(t[1]), [_num(x) for x in t[2:5]]))
    lf = [l.rstrip("\n") for l in open(os.path.join(d, "lat_fc.dat"))]
    i = [k for k, l in enumerate(lf) if l.startswith("  Crystal data: transl")][0]
    r = np.array([[_num(x) for x in _toks(lf[i + 1 + k])[:3]] for k in range(3)])
    assert int(_toks(lf[i + 5])[0]) == nat0
    prim_atoms = []
    for k in range(nat0):
        t = _toks(lf[i + 6 + k])
        prim_atoms.append((int(t[0]), t[1], int(t[2]), [_num(x) for x in t[3:6]], t[6]))
    j = [k for k, l in enumerate(lf) if "Number of FCs for each rank" in l][0]
    nterms = [int(x) for x in _toks(lf[j + 1])[:4]]
    m = [k for k, l in enumerate(lf) if "maxshells" in l][0]
    natoms2 = int(_toks(lf[m + 1])[1])
    sc = []
    for k in range(natoms2):
        t = _toks(lf[m + 2 + k])
        sc.append((int(t[0]), [_num(x) for x in t[1:4]], int(t[4]), [int(x) for x in t[5:8]]))
    fc2 = []
    with open(os.path.join(d, "fc2.dat")) as f:
        next(f)
        for line in f:
            t = _toks(line)
            if not t:
                continue
            fc2.append((int(t[2]), int(t[3]), int(t[4]), int(t[5]), _num(t[6])))
    assert len(fc2) == nterms[1], (len(fc2), nterms)
    diel = [_toks(l) for l in open(os.path.join(d, "dielectric.params")) if _toks(l)]
    born_flag = int(diel[0][0])
    epsil = np.array([[_num(x) for x in diel[1 + i][:3]] for i in range(3)])
    charge = np.array([[[_num(x) for x in diel[4 + 3 * k + i][:3]] for i in range(3)] for k in range(nat0)])
    ld = [l for l in open(os.path.join(d, "latdyn.params"))]
    mesh = [int(x) for x in _toks(ld[0])[:3]]
    tempk = _num(_toks(ld[5])[0])
    return dict(latp=np.array(latp), prim=np.array(prim), scale=scale, mass_str=np.array(mass_str),
                names=np.array(names), nat0=nat0,
                atom_types=np.array([a[1] for a in atoms]), atom_red=np.array([a[2] for a in atoms]),
                r=r, prim_cart=np.array([a[3] for a in prim_atoms]),
                sc_pos=np.array([s[1] for s in sc]), sc_cell0=np.array([s[2] for s in sc], dtype=np.int32),
                sc_cell=np.array([s[3] for s in sc], dtype=np.int32),
                fc2_idx=np.array([f[:4] for f in fc2], dtype=np.int16), fc2_val=np.array([f[4] for f in fc2]),
                mesh=np.array(mesh), tempk=tempk, born_flag=born_flag, epsil=epsil, charge=charge)


def parse_outputs(d: str, ndyn: int):
    out = {}
    ibz = np.loadtxt(os.path.join(d, "KPOINT.IBZ"), comments="#")
    out["ibz_kcart"] = ibz[:, 1:4]
    out["ibz_w"] = ibz[:, 4]
    out["ibz_kred"] = ibz[:, 5:8]
    out["rhs"] = np.loadtxt(os.path.join(d, "RHS_IBZ.dat"))
    fr = np.loadtxt(os.path.join(d, "FBZ_freqs.dat"))
    out["fbz_freq"] = fr[:, 5:5 + ndyn]
    out["fbz_k"] = fr[:, 2:5]
    tau = []
    with open(os.path.join(d, "tau_RTA.dat")) as f:
        next(f)
        for line in f:
            t = line.split()
            if len(t) < 10:
                continue
            tau.append([float(x) if x.lower() != "infinity" else np.inf for x in
                        [t[1], t[5], t[6], t[7]] + t[-3:]])
    tau = np.array(tau)
    out["tau_ibz"] = tau[:, 0].astype(np.int32)
    out["tau_band"] = tau[:, 1].astype(np.int32)
    out["tau_omega"] = tau[:, 2]
    out["tau_nb0"] = tau[:, 3]
    out["tau_veloc"] = tau[:, 4:7]
    return out


def main(ref_root: str):
    ex = {
        "ge_example": (os.path.join(ref_root, "THERMACOND", "Ge-example", "kappa"), 4),
        "gese_example": (os.path.join(ref_root, "THERMACOND", "GeSe-example", "kappa"), 4),
    }
    for name, (d, nsh) in ex.items():
        inp = parse_example(d, nsh)
        ndyn = 3 * inp["nat0"]
        outp = parse_outputs(d, ndyn)
        fn = os.path.join(HERE, name + ".npz")
        np.savez_compressed(fn, **inp, **{"out_" + k: v for k, v in outp.items()})
        print("wrote", fn, os.path.getsize(fn), "bytes; nibz", len(outp["ibz_w"]), "fc2", len(inp["fc2_val"]))


if __name__ == "__main__":
    if len(sys.argv) != 2:
        sys.exit("usage: %s <path of the reference checkout>" % sys.argv[0])
    main(sys.argv[1])
