"""Write the reference's Ge / GeSe example inputs (from the committed npz
fixtures) in the layout the current THERMACOND readers parse.

The numbers are the ones the reference shipped (lattice, atoms, supercell
positions, FC2 terms); only the record layout changes.  FC3 is switched
off (include_fc(3)=0): no example ships an fc3.dat.
"""
from __future__ import annotations

import os

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))


def load(name: str) -> dict:
    z = np.load(os.path.join(HERE, name + ".npz"))
    return {k: z[k] for k in z.files}


def _f(x) -> str:
    return repr(float(x))


def materialize(name: str, out_dir: str) -> dict:
    z = load(name)
    os.makedirs(out_dir, exist_ok=True)
    nat0 = int(z["nat0"])
    masses = [float(m) for m in z["mass_str"]]
    types = [int(t) for t in z["atom_types"]]
    mesh = [int(x) for x in z["mesh"]]
    with open(os.path.join(out_dir, "latdyn.params"), "w") as f:
        f.write("%d %d %d .false.\n0 0 0\n0 0 1\n300 350\n10 30\n.false.\n" % tuple(mesh))
        f.write("%s %s 1\n1\n2\n./\n0\n0\n0 0 0 0\n100\n" % (_f(z["tempk"]), _f(z["tempk"])))
    with open(os.path.join(out_dir, "structure.params"), "w") as f:
        f.write(" ".join(_f(x) for x in z["latp"]) + "\n")
        f.write(" ".join(_f(x) for x in z["prim"]) + "\n")
        f.write(_f(z["scale"]) + "\n1 1 0 0\n1 1 0 0\n0 300\n1 .false.\n")
        f.write("%d\n" % len(masses) + " ".join(_f(m) for m in masses) + "\n" + " ".join(str(n) for n in z["names"]) + "\n")
        f.write("%d\n" % nat0 + "0\n" * 8)
        for i in range(nat0):
            f.write("%d %d %s\n" % (i + 1, types[i], " ".join(_f(x) for x in z["atom_red"][i])))
    sc = z["sc_pos"]
    with open(os.path.join(out_dir, "lat_fc.dat"), "w") as f:
        f.write(" converted example\n  Crystal data: translation vectors of the primitive cell\n")
        for k in range(3):
            f.write("  " + " ".join(_f(x) for x in z["r"][k]) + "\n")
        f.write("  atoms\n  %d\n" % nat0)
        for i in range(nat0):
            f.write("  %d %s %d %s %s\n" % (i + 1, z["names"][types[i] - 1], types[i],
                                          " ".join(_f(x) for x in z["prim_cart"][i]), _f(masses[types[i] - 1])))
        nt2 = len(z["fc2_val"])
        f.write("  ranks\n  1 1 0 0\n" + "  shells\n" * 8 + "  groups\n  0 %d 0 0\n  nterms\n  0 %d 0 0\n" % (nt2, nt2))
        f.write("  skip\n  skip\n  atoms\n  8 %d\n" % len(sc))
        for j in range(len(sc)):
            c = z["sc_cell"][j]
            f.write("  %d %s %d %d %d %d\n" % (j + 1, " ".join(_f(x) for x in sc[j]), int(z["sc_cell0"][j]),
                                             c[0], c[1], c[2]))
    with open(os.path.join(out_dir, "fc2.dat"), "w") as f:
        f.write(" # rank 2\n")
        idx, val = z["fc2_idx"], z["fc2_val"]
        for t in range(len(val)):
            a = idx[t]
            f.write("%d %d %d %d %d %d %s\n" % (t + 1, t + 1, a[0], a[1], a[2], a[3], _f(val[t])))
    with open(os.path.join(out_dir, "dielectric.params"), "w") as f:
        f.write("%d\n" % int(z["born_flag"]))
        for i in range(3):
            f.write(" ".join(_f(x) for x in z["epsil"][i]) + "\n")
        for k in range(nat0):
            for i in range(3):
                f.write(" ".join(_f(x) for x in z["charge"][k][i]) + "\n")
    return z
