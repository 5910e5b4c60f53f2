"""The job=1 output files (Qvalue.dat, tau_RTA.dat, kappa_RTA.dat,
tau_RTAandeff-cg.dat, kappa_direct-cg.dat) written through the C ABI vs the
oracle's restatement of Qandtau / write_kappa (oracle/writers.py), GPU.

The oracle's eigenpairs are injected into the context (identical inputs, as
in the stage parity tests).  Records must agree in layout (line count, line
lengths, token count, every integer, every non-numeric token) and in value:
equal text, or numbers within one unit of the last printed digit plus
rtol |value| + atol max|column| (rtol 1e-10, atol 1e-12 given the oracle's
results; rtol 1e-8, atol 1e-10 for the files from the library's own
pipeline, the kappa_cg tolerance of the pipeline parity test; there the
1/tauinv columns are compared as rates, since the inverse of a rate near
zero is arbitrarily large).

tauinv_eff of mode_kappa_d divides by |v|^2 of the star-averaged velocity:
where that velocity is rounding noise (|v| < 1e-9 max|v|) both codes return
0/0 or noise/noise, so those entries of tau_RTAandeff-cg.dat are excluded
from the value check (their layout is still checked).
"""
import math
import os
import re
import sys

import numpy as np
import pytest

from conftest import ROOT, make_case

sys.path.insert(0, os.path.join(ROOT, "oracle"))
import writers as OW  # noqa: E402

pytestmark = pytest.mark.gpu

FILES = ["Qvalue.dat", "tau_RTA.dat", "kappa_RTA.dat", "tau_RTAandeff-cg.dat", "kappa_direct-cg.dat"]
CASES = [(1, (4, 4, 4), {}), (0, (6, 6, 6), {"delta": "gauss"})]
NUM = re.compile(r"^([+-]?)(\d*)\.(\d*)(?:E?([+-]\d+))?$")


def num(t):
    m = NUM.match(t)
    if not m:
        return {"Infinity": math.inf, "-Infinity": -math.inf, "NaN": math.nan}[t]
    return float(m.group(1) + (m.group(2) or "0") + "." + (m.group(3) or "0") + "e" + (m.group(4) or "0"))


def last_unit(t):
    m = NUM.match(t)
    return 10.0 ** (-len(m.group(3)) + int(m.group(4) or 0))


def _val(t, inverse):
    v = num(t)
    if inverse:  # 1/rate -> rate
        return 0.0 if math.isinf(v) else 1.0 / v
    return v


def column_scale(lines, inverse=()):
    """max |value| per token column over the finite numbers of a file."""
    sc = {}
    for y in lines:
        for c, v in enumerate(y.split()):
            if NUM.match(v) and "." in v:
                f = abs(_val(v, c in inverse))
                if math.isfinite(f):
                    sc[c] = max(sc.get(c, 0.0), f)
    return sc


def compare(a_path, b_path, rtol, atol, skip=lambda line, col: False, inverse=()):
    """a (library) vs b (oracle): |a - b| <= one unit of b's last digit +
    rtol |b| + atol max|column of b|, or equal text.  Columns in `inverse`
    hold 1/rate and are compared as rates (a rate near zero makes its
    inverse arbitrarily large)."""
    A = open(a_path).read().split("\n")
    B = open(b_path).read().split("\n")
    assert len(A) == len(B), (a_path, len(A), len(B))
    scale = column_scale(B, inverse)
    worst = 0.0
    for k, (x, y) in enumerate(zip(A, B)):
        if x == y:
            continue
        assert len(x) == len(y), (a_path, k, x, y)
        tx, ty = x.split(), y.split()
        assert len(tx) == len(ty), (a_path, k, x, y)
        for c, (u, v) in enumerate(zip(tx, ty)):
            if u == v or skip(k, c):
                continue
            assert NUM.match(u) and NUM.match(v), (a_path, k, c, u, v)
            assert "." in u, (a_path, k, c, u, v)  # integers must match exactly
            inv = c in inverse
            fu, fv = _val(u, inv), _val(v, inv)
            unit = last_unit(v) * (abs(fv) / abs(num(v)) if inv and fv != 0 else 1.0)
            err = abs(fu - fv) - 1.01 * unit - rtol * abs(fv) - atol * scale.get(c, 0.0)
            worst = max(worst, abs(fu - fv) / (abs(fv) + 1e-300))
            assert err <= 0, (a_path, k, c, u, v)
    return worst


@pytest.fixture(scope="module", params=CASES, ids=lambda c: "cfg%d_%s_%s" % (c[0], c[1][0], c[2].get("delta", "")))
def case(request, oracle_lib, ald_lib, workdir):
    cfg, mesh, kw = request.param
    d = make_case(workdir, cfg, mesh, **kw)
    ref = oracle_lib.run_job1(d)
    O = ref["O"]
    ev, vec, vel = O.get_phonons()
    ctx = ald_lib.Context(d)
    ctx.set_phonons(ev, vec, vel)
    yield d, ref, ctx, vel
    ctx.close()


def noise_velocity(vel, mapinv):
    """(nibz, ndn): the mode's velocity at mapinv is rounding noise."""
    v = np.linalg.norm(vel, axis=0)  # (ndn, nkc)
    return (v[:, np.asarray(mapinv) - 1] < 1e-9 * v.max()).T


def oracle_files(out, ref, vel, Q, QN, QU, krta, kcg, x):
    O = ref["O"]
    I = O.ibz()
    FFF, _ = O.rta(ref["tempk"], Q)
    _, trta = O.mode_kappa_teff(ref["tempk"], FFF)
    _, tcg = O.kappa_d_teff(ref["tempk"], x, trta)
    os.makedirs(out, exist_ok=True)
    OW.write_job1_files(out, ref["tempk"], ref["freq"], ref["dist"], vel, I["kibz"], I["mapinv"], Q, QN, QU, krta,
                        kcg, trta, tcg)
    return I["mapinv"]


def test_tau_eff_per_mode(case):
    d, ref, ctx, vel = case
    O = ref["O"]
    noise = noise_velocity(vel, O.ibz()["mapinv"])
    _, t0 = O.mode_kappa_teff(ref["tempk"], ref["FFF"], keep_all=True)
    g0 = ctx.tau_eff(ref["tempk"], ref["FFF"], 0)
    scale = np.abs(t0).max()
    assert np.all(np.abs(g0 - t0) <= 1e-10 * np.abs(t0) + 1e-12 * scale)
    _, t1 = O.kappa_d_teff(ref["tempk"], ref["x"], np.zeros_like(t0))
    g1 = ctx.tau_eff(ref["tempk"], ref["x"], 1)
    ok = ~noise
    assert ok.sum() > 0
    scale = np.abs(t1[ok]).max()
    assert np.all(np.abs(g1[ok] - t1[ok]) <= 1e-9 * np.abs(t1[ok]) + 1e-12 * scale)


def test_qandtau(case, tmp_path):
    d, ref, ctx, vel = case
    tN, tU, tT = ctx.qandtau(ref["tempk"], ref["Q"], ref["QN"], ref["QU"], str(tmp_path / "Qvalue.dat"))
    oN, oU, oT = OW.qandtau(ref["dist"], ref["O"].ibz()["mapinv"], ref["Q"], ref["QN"], ref["QU"],
                            str(tmp_path / "Qvalue_oracle.dat"))
    for g, r in ((tN, oN), (tU, oU), (tT, oT)):
        assert np.allclose(g, r, rtol=1e-12, atol=0)
    compare(str(tmp_path / "Qvalue.dat"), str(tmp_path / "Qvalue_oracle.dat"), 1e-12, 0.0)


def _skip_for(mapinv, vel, ndn):
    noise = noise_velocity(vel, mapinv)

    def skip(line, col):  # tau_eff is token 11 of a tau record; line 0 is the header
        if line == 0 or col != 11:
            return False
        m = line - 1
        return bool(noise[m // ndn, m % ndn])
    return skip


def test_files_given_oracle_results(case, tmp_path):
    """The writers alone: the oracle's Q, Q_N, Q_U, per-band kappas and CG
    solution go into ald_write_job1_files."""
    d, ref, ctx, vel = case
    res = {"Q": ref["Q"], "QN": ref["QN"], "QU": ref["QU"], "kappa_rta_modes": ref["kappa_rta"],
           "kappa_cg_modes": ref["kappa_cg"], "x": ref["x"]}
    lib_dir, orc_dir = str(tmp_path / "lib"), str(tmp_path / "oracle")
    os.makedirs(lib_dir)
    ctx.write_job1_files(lib_dir, ref["tempk"], res)
    mapinv = oracle_files(orc_dir, ref, vel, ref["Q"], ref["QN"], ref["QU"], ref["kappa_rta"], ref["kappa_cg"],
                          ref["x"])
    skip = _skip_for(mapinv, vel, ctx.ndyn)
    for f in FILES:
        compare(os.path.join(lib_dir, f), os.path.join(orc_dir, f), 1e-10, 1e-12,
                skip if f == "tau_RTAandeff-cg.dat" else (lambda line, col: False))
    # the layout of kappa_full's files: one record per IBZ mode plus a header
    n = ref["O"].nibz * ctx.ndyn
    for f in ("Qvalue.dat", "tau_RTA.dat", "tau_RTAandeff-cg.dat"):
        assert len(open(os.path.join(lib_dir, f)).read().splitlines()) == n + 1
    assert len(open(os.path.join(lib_dir, "kappa_RTA.dat")).read().splitlines()) == ctx.ndyn + 5


def test_files_from_pipeline(case, tmp_path):
    """ald_kappa_pipeline's own results written out vs the oracle's job=1."""
    d, ref, ctx, vel = case
    out = ctx.kappa_pipeline(ref["tempk"])
    lib_dir, orc_dir = str(tmp_path / "lib"), str(tmp_path / "oracle")
    os.makedirs(lib_dir)
    ctx.write_job1_files(lib_dir, ref["tempk"], out)
    mapinv = oracle_files(orc_dir, ref, vel, ref["Q"], ref["QN"], ref["QU"], ref["kappa_rta"], ref["kappa_cg"],
                          ref["x"])
    skip = _skip_for(mapinv, vel, ctx.ndyn)
    for f in FILES:
        compare(os.path.join(lib_dir, f), os.path.join(orc_dir, f), 1e-8, 1e-10,
                skip if f == "tau_RTAandeff-cg.dat" else (lambda line, col: False),
                inverse=(8, 9, 10) if f.startswith("tau") else ())
