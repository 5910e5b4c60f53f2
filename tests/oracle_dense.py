"""|V3|^2 of large cells on the CPU in factorised form -- test infrastructure.

The literal oracle (oracle/oracle_bte.cpp, calculate_w3_ibz_split_sq)
follows matrix_elt_simplified (THERMACOND/sub.f90:5888-6011) term by term:
for every band triplet it sums all nterms(3) FC3 terms, nkc*b^3*nterms(3)
iterations per IBZ row.  For the 64-atom rock-salt cell (192 bands, 95 040
terms) that is 7e11 per (q1, q2) pair, out of reach for a test.  This module
evaluates the same sum with the terms regrouped:

  Phi(q2,q3)[a,b,c] = sum_{t in channel (a,b,c)} fcs_3(t)/sqrt(mi mj mk) eiqr2(q2,j) eiqr2(q3,k)
  V(l1,l2,l3)       = sum_{a,b,c} e1[a,l1] e2[b,l2] e3[c,l3] Phi[a,b,c]

with channel (a, b, c) = (x1 + 3(i0-1), x2 + 3(j0-1), x3 + 3(k0-1)), eiqr2 of
cal_eiqr2 (sub.f90:6015-6067), q3 = -q1-q2 folded by get_k_info, the
eigenvectors not conjugated and |V|^2 scaled by (const33/sqrt(8 sqrt|l1 l2
l3|))^2 as in the reference.  The regrouping reorders the sums, so results
agree with the literal oracle to FP64 rounding; tests/test_oracle_dense.py
checks that on the 6- and 24-band cells.
"""
from __future__ import annotations

import numpy as np


def v3_factorised(O, k1: int, k2: int, q2s=None) -> np.ndarray:
    """|V3|^2 of IBZ rows k1..k2 (1-based, inclusive) as v33s8(nsub, nkc,
    ndyn, ndyn, ndyn); only the q2 (0-based) of `q2s` are filled when given."""
    T = O.fc3_terms()
    ev, vec, _ = O.get_phonons()
    kpc = O.kpc()
    mapinv = O.ibz()["mapinv"]
    const33 = O.lattice()["const33"]
    n, nk = O.ndyn, O.nkc
    iat, ixyz, fcs = T["iat"], T["ixyz"], T["fcs"]
    cell0, mass0, pos = T["cell0"], T["mass0"], T["atompos"]
    # terms whose first atom is a primitive atom (matrix_elt_simplified skips the rest)
    keep = cell0[iat[0] - 1] == iat[0]
    i3, j, k = iat[0][keep], iat[1][keep], iat[2][keep]
    x1, x2, x3 = ixyz[0][keep] - 1, ixyz[1][keep] - 1, ixyz[2][keep] - 1
    i0, j0, k0 = cell0[i3 - 1], cell0[j - 1], cell0[k - 1]
    w = fcs[keep] / np.sqrt(mass0[i0 - 1] * mass0[j0 - 1] * mass0[k0 - 1])
    chan = ((x1 + 3 * (i0 - 1)) * n + (x2 + 3 * (j0 - 1))) * n + (x3 + 3 * (k0 - 1))
    # eiqr2(q, atom) = exp(i kpc(:,q).(atompos(:,atom) - atompos(:,atom0)))
    rel = pos - pos[:, cell0 - 1]
    eiqr2 = np.exp(1j * (kpc.T @ rel))  # (nkc, natoms)
    out = np.zeros((k2 - k1 + 1, nk, n, n, n), order="F")
    q2s = range(nk) if q2s is None else q2s
    for s, n1 in enumerate(range(k1, k2 + 1)):
        q1 = mapinv[n1 - 1] - 1
        e1 = vec[:, :, q1]
        for q2 in q2s:
            q3 = O.get_k_info(-kpc[:, q1] - kpc[:, q2])[0] - 1
            ph = w * eiqr2[q2, j - 1] * eiqr2[q3, k - 1]
            phi = (np.bincount(chan, weights=ph.real, minlength=n ** 3) +
                   1j * np.bincount(chan, weights=ph.imag, minlength=n ** 3)).reshape(n, n, n)
            t = np.tensordot(e1, phi, axes=([0], [0]))            # (l1, b, c)
            t = np.tensordot(t, vec[:, :, q2], axes=([1], [0]))    # (l1, c, l2)
            v = np.tensordot(t, vec[:, :, q3], axes=([1], [0]))    # (l1, l2, l3)
            den = np.sqrt(8 * np.sqrt(np.abs(ev[:, q1][:, None, None] * ev[:, q2][None, :, None] *
                                             ev[:, q3][None, None, :])))
            vv = v / den * const33
            out[s, q2] = vv.real ** 2 + vv.imag ** 2
    return out
