"""ORACLE -- TEST INFRASTRUCTURE ONLY.  Only tests, smoke() and the bench's
CPU baseline may use this file, and only as the checker.

A pure-Python restatement of the output files of THERMACOND's job=1 run and
of the gfortran edit rules they are written with:

  Qvalue.dat                        Qandtau      THERMACOND/sub.f90:8198-8305
  tau_RTA.dat, kappa_RTA.dat        write_kappa  THERMACOND/sub.f90:1818-1916 (after mode_kappa)
  tau_RTAandeff-cg.dat,             write_kappa  (after mode_kappa_d; kappa.f90:559-870)
  kappa_direct-cg.dat

Parity of the edit rules is pinned by lines of the files the reference
ships with its Ge and GeSe examples (tests/golden/fortran_records.json):
every one of them is reproduced byte for byte from its own numbers.

Rules (gfortran):
* list-directed (`write(u,*)`): each item is preceded by one blank, except a
  character item right after another character item; INTEGER is I11;
  REAL(8) has 17 significant digits in 25 columns: F20.(17-s) plus five
  blanks when 0 <= s <= 17 (s = the decimal exponent of the rounded value,
  0.1 <= |x|/10^s < 1; s = 1 for zero), else 1PE25.16 with "E" and a
  three-digit exponent;
* Iw, Fw.d, Ew.d (two-digit exponent with E, three digits without E above
  99), Gw.d = F(w-4).(d-s) plus four blanks for 0 <= s <= d else Ew.d; an
  INTEGER under G is Iw; the optional leading zero before the decimal point
  is dropped when the field is one short; a number that still does not fit
  is w asterisks; Infinity/Inf/NaN right-justified.
"""
from __future__ import annotations

import math
import os

import numpy as np

# physical constants of modules.f90:4-23 (the values the library uses)
C_LIGHT = 2.99792458e+8


def _stars(w):
    return "*" * w


def _pad(s, w):
    return _stars(w) if len(s) > w else " " * (w - len(s)) + s


def _sig(ax, nd):
    m, e = ("%.*e" % (nd - 1, ax)).split("e")
    return m.replace(".", ""), int(e) + 1


def _special(w, x):
    if math.isnan(x):
        return _pad("NaN", w)
    neg = x < 0
    word = "Infinity" if w - neg >= 8 else "Inf"
    return _pad(("-" if neg else "") + word, w)


def _fit(neg, body, w):
    if len(body) + neg > w and body.startswith("0."):
        body = body[1:]
    return _pad(("-" if neg else "") + body, w)


def edit_I(w, v):
    return _pad(str(int(v)), w)


def edit_F(w, d, x):
    if not math.isfinite(x):
        return _special(w, x)
    body = "%.*f" % (d, abs(x))
    if d == 0:
        body += "."
    return _fit(math.copysign(1.0, x) < 0, body, w)


def edit_E(w, d, x):
    if not math.isfinite(x):
        return _special(w, x)
    if x == 0:
        dig, s = "0" * d, 0
    else:
        dig, s = _sig(abs(x), d)
    ex = ("E%s%02d" if abs(s) <= 99 else "%s%03d") % ("-" if s < 0 else "+", abs(s))
    return _fit(math.copysign(1.0, x) < 0, "0." + dig + ex, w)


def edit_G(w, d, x):
    if not math.isfinite(x):
        return _special(w, x)
    s = 1 if x == 0 else _sig(abs(x), d)[1]
    if s < 0 or s > d:
        return edit_E(w, d, x)
    return edit_F(w - 4, d - s, x) + "    "


def list_real(x):
    if not math.isfinite(x):
        return _special(25, x)
    if x == 0:
        dig, s = "0" * 17, 1
    else:
        dig, s = _sig(abs(x), 17)
    if 0 <= s <= 17:
        return edit_F(20, 17 - s, x) + "     "
    e = s - 1
    body = dig[0] + "." + dig[1:] + "E%s%03d" % ("-" if e < 0 else "+", abs(e))
    return _pad(("-" if x < 0 else "") + body, 25)


def list_int(v):
    return _pad(str(int(v)), 11)


def list_record(*items):
    """write(u,*) items: int -> I11, float -> REAL(8), str -> as is."""
    out, prev_chr = "", False
    for it in items:
        chr_ = isinstance(it, str)
        if not (chr_ and prev_chr) or not out:
            out += " "
        out += it if chr_ else (list_int(it) if isinstance(it, (int, np.integer)) else list_real(float(it)))
        prev_chr = chr_
    return out


def format_value(edit: str, x) -> str:
    """The same edits as the library's ald_format_value."""
    if edit == "*":
        return list_real(float(x))
    if edit == "*I":
        return list_int(x)
    k, spec = edit[0], edit[1:]
    if k == "I":
        return edit_I(int(spec), x)
    w, d = (int(v) for v in spec.split("."))
    return {"F": edit_F, "E": edit_E, "G": edit_G}[k](w, d, float(x))


# ------------------------------------------------------------------ writers
def qandtau(dist, mapinv, Q, QN, QU, path=None):
    """Qandtau (sub.f90:8244-8285).  dist(nkc, ndn); mapinv 1-based;
    Q, QN, QU(nibz, ndn).  Returns tauinv_N, tauinv_U, tauinv_tot."""
    nibz, ndn = Q.shape
    tN = np.zeros((nibz, ndn), order="F")
    tU = np.zeros((nibz, ndn), order="F")
    tT = np.zeros((nibz, ndn), order="F")
    lines = [list_record("nk,la,Q")]
    f64 = np.float64
    with np.errstate(divide="ignore", invalid="ignore", over="ignore"):  # IEEE results, as the Fortran
        for ibz in range(1, nibz + 1):
            for ii in range(1, ndn + 1):
                nb1 = f64(dist[mapinv[ibz - 1] - 1, ii - 1])
                q = f64(Q[ibz - 1, ii - 1])
                lines.append(list_record(ibz, ii, q, q / (nb1 * (nb1 + 1))))
                tN[ibz - 1, ii - 1] = f64(QN[ibz - 1, ii - 1]) / (nb1 * (nb1 + 1)) * f64(C_LIGHT) * 100
                tU[ibz - 1, ii - 1] = f64(QU[ibz - 1, ii - 1]) / (nb1 * (nb1 + 1)) * f64(C_LIGHT) * 100
                tT[ibz - 1, ii - 1] = tN[ibz - 1, ii - 1] + tU[ibz - 1, ii - 1]
    if path:
        with open(path, "w") as f:
            f.write("\n".join(lines) + "\n")
    return tN, tU, tT


def write_kappa(tempk, kappa, freq, dist, veloc, kibz, mapinv, tN, tU, tT, teff, kappa_path, tau_path):
    """write_kappa (sub.f90:1818-1916).  kappa(ndn,3,3); freq, dist(nkc, ndn);
    veloc(3, ndn, nkc); kibz(3, nibz); tN and tU are changed in place (zero
    -> 1e10) as in the reference."""
    ndn = kappa.shape[0]
    nibz = tN.shape[0]
    tot_kap = 0.0
    for j in range(3):
        for jj in range(3):
            for ii in range(ndn):
                if j == jj:
                    tot_kap = tot_kap + float(kappa[ii, j, jj]) / 3
    L = [list_record("la, kxx,kyy,kzz, kxy,kxz,kyz, k_RTA")]
    for ii in range(ndn):
        v = [kappa[ii, 0, 0], kappa[ii, 1, 1], kappa[ii, 2, 2], kappa[ii, 0, 1], kappa[ii, 0, 2], kappa[ii, 1, 2]]
        L.append(edit_I(2, ii + 1) + "".join(" " + edit_G(11, 4, float(x)) for x in v))
    L += [list_record(" "), list_record("tot_kap=", tot_kap), list_record(" ")]
    sums = []
    for j in range(3):
        s = 0.0
        for ii in range(ndn):
            s = s + float(kappa[ii, j, j])
        sums.append(s)
    L.append("   " + "".join(" " + edit_F(9, 3, s) for s in sums))
    with open(kappa_path, "w") as f:
        f.write("\n".join(L) + "\n")
    T = [list_record("tempk,i,kibz(:,i),ii,omega,nb0,1/tauinv_N(i,ii),1/tauinv_U(i,ii),1/tauinv_tot(i,ii),"
                     "1/tauinv_eff(i,ii),veloc(:,ii,mapinv(i))")]
    def inv(v):
        with np.errstate(divide="ignore", over="ignore"):
            return float(np.float64(1.0) / np.float64(v))

    for i in range(1, nibz + 1):
        q = mapinv[i - 1] - 1
        for ii in range(1, ndn + 1):
            m = (i - 1, ii - 1)
            if tU[m] == 0:
                tU[m] = 1.0e10
            if tN[m] == 0:
                tN[m] = 1.0e10
            vals = [("G", tempk), ("I", i)] + [("G", kibz[x, i - 1]) for x in range(3)] + [("I", ii)]
            vals += [("G", freq[q, ii - 1]), ("G", dist[q, ii - 1]), ("G", inv(tN[m])), ("G", inv(tU[m])),
                     ("G", inv(tT[m])), ("G", teff[m])] + [("G", veloc[x, ii - 1, q]) for x in range(3)]
            T.append("".join(" " + (edit_I(14, v) if k == "I" else edit_G(14, 8, float(v))) for k, v in vals))
    with open(tau_path, "w") as f:
        f.write("\n".join(T) + "\n")


def write_job1_files(out_dir, tempk, freq, dist, veloc, kibz, mapinv, Q, QN, QU, kappa_rta, kappa_cg, teff_rta,
                     teff_cg):
    """The five files in kappa_full's order.  teff_rta is tauinv_eff as
    mode_kappa leaves it, teff_cg as mode_kappa_d leaves it."""
    tN, tU, tT = qandtau(dist, mapinv, Q, QN, QU, os.path.join(out_dir, "Qvalue.dat"))
    write_kappa(tempk, kappa_rta, freq, dist, veloc, kibz, mapinv, tN, tU, tT, teff_rta,
                os.path.join(out_dir, "kappa_RTA.dat"), os.path.join(out_dir, "tau_RTA.dat"))
    write_kappa(tempk, kappa_cg, freq, dist, veloc, kibz, mapinv, tN, tU, tT, teff_cg,
                os.path.join(out_dir, "kappa_direct-cg.dat"), os.path.join(out_dir, "tau_RTAandeff-cg.dat"))
