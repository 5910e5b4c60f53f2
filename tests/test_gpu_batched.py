"""ald_kappa_batched: several structures through the job=1 pipeline at once
(one host thread and one stream per context) must give what each context gives
alone, GPU.  The contexts run the FP64 path with the default options, whose
tetrahedron delta is deterministic: the tetrahedron structures must give the
same bits batched as alone.  The Gaussian structures' delta sums in registers,
also in a fixed order, so they must too.  kappa is also compared to 1e-12
relative (plus 1e-14 of its largest component) and the CG iteration counts
exactly."""
import numpy as np
import pytest

from conftest import make_case

pytestmark = pytest.mark.gpu

CASES = [(1, (4, 4, 4), {}), (0, (6, 6, 6), {"delta": "gauss"}), (1, (6, 6, 6), {}),
         (3, (4, 4, 4), {"delta": "gauss", "width_cm": 5.0, "rc_sigma": 1.2})]


def test_batched_equals_single(ald_lib, workdir):
    dirs = [make_case(workdir, cfg, mesh, **kw) for cfg, mesh, kw in CASES]
    single = []
    for d in dirs:
        ctx = ald_lib.Context(d)
        single.append(ctx.kappa_pipeline(want_modes=False))
        ctx.close()
    ctxs = [ald_lib.Context(d) for d in dirs]
    tempk = [c.info.tempk for c in ctxs]
    for rep in range(2):  # the second pass reuses every context's workspaces and graphs
        out, st = ald_lib.kappa_batched(ctxs, tempk)
        assert st == [0] * len(dirs)
        for o, s in zip(out, single):
            assert o["cg_iters"] == s["cg_iters"]
            for k in ("kappa_rta", "kappa_cg"):
                assert np.allclose(o[k], s[k], rtol=1e-12, atol=1e-14 * np.abs(s[k]).max()), k
                assert np.array_equal(o[k], s[k]), k
            assert o["triplet_bands"] == s["triplet_bands"]
    for c in ctxs:
        c.close()


def test_batched_rejects_a_repeated_context(ald_lib, workdir):
    d = make_case(workdir, 1, (4, 4, 4))
    ctx = ald_lib.Context(d)
    with pytest.raises(RuntimeError):
        ald_lib.kappa_batched([ctx, ctx], 300.0)
    ctx.close()


def test_device_memory_cache_reuse_and_release(ald_lib, workdir):
    """Workspaces freed by one context are reused by the next one of the same
    system; after ald_release_cached_memory a new context still runs, with
    the same results."""
    d = make_case(workdir, 1, (6, 6, 6))
    runs = []
    for release in (False, False, True):
        ctx = ald_lib.Context(d)
        runs.append(ctx.kappa_pipeline(want_modes=False))
        ctx.close()
        if release:
            ald_lib.release_cached_memory()
    ctx = ald_lib.Context(d)
    runs.append(ctx.kappa_pipeline(want_modes=False))
    ctx.close()
    for r in runs[1:]:
        assert r["cg_iters"] == runs[0]["cg_iters"]
        for k in ("kappa_rta", "kappa_cg"):
            assert np.allclose(r[k], runs[0][k], rtol=1e-12, atol=1e-14 * np.abs(runs[0][k]).max())


def test_batched_uneven_sizes_against_oracle(ald_lib, oracle_lib, workdir):
    """Three structures of uneven size in one ald_kappa_batched call -- the
    rock-salt cell (6 bands), the 4-atom LJ cell (12 bands) and the 8-atom
    superlattice (24 bands, the large-cell kernels) -- each against the
    oracle's job=1 run on the same eigenpairs: Q to 1e-10, kappa to 1e-10
    (floor 1e-10 max|kappa|), the same CG iterations."""
    from test_gpu_parity import close
    cases = [(1, (4, 4, 4), {}), (3, (4, 4, 4), {"delta": "gauss", "width_cm": 5.0, "rc_sigma": 1.2}),
             (3, (2, 4, 4), {"p": 2, "rc_sigma": 1.2, "delta": "gauss", "width_cm": 5.0})]
    refs, ctxs = [], []
    for cfg, mesh, kw in cases:
        d = make_case(workdir, cfg, mesh, **kw)
        ref = oracle_lib.run_job1(d)
        ctx = ald_lib.Context(d)
        ctx.set_phonons(*ref["O"].get_phonons())
        refs.append(ref)
        ctxs.append(ctx)
    out, st = ald_lib.kappa_batched(ctxs, [r["tempk"] for r in refs])
    assert st == [0] * len(cases)
    for o, r, c in zip(out, refs, ctxs):
        assert c.ndyn in (6, 12, 24)
        assert o["cg_iters"] == r["cg_iters"]
        for key, rk in (("kappa_rta", "kappa_rta"), ("kappa_cg", "kappa_cg")):
            ok, worst = close(o[key], r[rk].sum(0), atol=1e-10)
            assert ok, (c.ndyn, key, worst)
    for c in ctxs:
        c.close()


def test_release_workspaces_then_rerun(ald_lib, workdir):
    """ald_release_workspaces hands a context's workspaces back; its next
    pipeline call takes new ones and gives the same results."""
    d = make_case(workdir, 1, (6, 6, 6))
    ctx = ald_lib.Context(d)
    a = ctx.kappa_pipeline(want_modes=False)
    ctx.release_workspaces()
    b = ctx.kappa_pipeline(want_modes=False)
    assert a["cg_iters"] == b["cg_iters"]
    for k in ("kappa_rta", "kappa_cg"):
        assert np.allclose(a[k], b[k], rtol=1e-12, atol=1e-14 * np.abs(a[k]).max())
    ctx.close()
