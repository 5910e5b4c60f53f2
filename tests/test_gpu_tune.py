"""The pipeline's autotuner (ald_autotune, no counterpart in the reference)
on the GPU: it times candidate launch shapes, keeps the fastest on the
context and in its cache file, reads the choice back for a context of the
same shape without timing anything, and leaves the results unchanged (its
knobs only change how rows and pairs are grouped into launches)."""
import os

import numpy as np
import pytest

from conftest import make_case

pytestmark = pytest.mark.gpu


@pytest.mark.parametrize("cfg,mesh,kw,prec", [
    (0, (6, 6, 6), {"delta": "gauss"}, "mixed"),    # 3 bands: the tensor-core class sums' knobs
    (1, (6, 6, 6), {}, "fp64"),                     # deterministic FP64 path: bitwise equal
    (3, (2, 4, 4), {"p": 2, "rc_sigma": 1.2, "delta": "gauss"}, "mixed")],  # 24 bands: the GEMM batches
    ids=["lj3_mixed", "nacl6_fp64", "sl24_mixed"])
def test_autotune_cache_and_results(ald_lib, workdir, tmp_path, cfg, mesh, kw, prec):
    d = make_case(workdir, cfg, mesh, **kw)
    delta = ald_lib.DELTA_GAUSS if kw.get("delta") == "gauss" else ald_lib.DELTA_TETRA
    P = ald_lib.MIXED if prec == "mixed" else ald_lib.FP64
    opts = ald_lib.default_options(precision=P, delta=delta)
    cache = str(tmp_path / "tune.txt")
    with ald_lib.Context(d, opts) as ctx:
        ref = ctx.kappa_pipeline(ctx.info.tempk)
        t = ctx.autotune(cache, budget_s=20)
        assert t["from_cache"] == 0 and t["candidates"] >= 2 and t["ms"] > 0
        got = ctx.kappa_pipeline(ctx.info.tempk)
    lines = open(cache).read().splitlines()
    assert len(lines) == 1 and "chunk_bytes=%d " % t["chunk_bytes"] in lines[0]
    for key in ("Q", "kappa_rta", "kappa_cg"):
        a, b = np.asarray(got[key]), np.asarray(ref[key])
        if prec == "fp64":
            assert np.array_equal(a, b), key
        else:  # FP64 atomics in arrival order in the mixed delta
            assert np.allclose(a, b, rtol=1e-10, atol=1e-12 * np.abs(b).max()), key
    # a second context of the same shape reads the choice from the file
    with ald_lib.Context(d, opts) as ctx2:
        t2 = ctx2.autotune(cache)
        assert t2["from_cache"] == 1 and t2["candidates"] == 0
        for k in ("chunk_bytes", "v3_rows_per_cta", "v3_epilogue_wg", "v3_gemm_bytes"):
            assert t2[k] == t[k], k
        got2 = ctx2.kappa_pipeline(ctx2.info.tempk)
    assert np.allclose(got2["kappa_cg"], ref["kappa_cg"], rtol=1e-10, atol=1e-12 * np.abs(ref["kappa_cg"]).max())
    assert len(open(cache).read().splitlines()) == 1
    os.remove(cache)
