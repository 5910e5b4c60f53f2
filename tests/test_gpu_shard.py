"""The row-sharded job=1 against the single-context pipeline (GPU).

Every rank of ald_kappa_pipeline_sharded runs here as a host thread with its
own context on the one GPU of the test machine; the all-gather is an
in-process exchange (a barrier and a shared list).  No kernel of one rank
waits on another rank's: all the waiting is on the host, between launches.
Q, Q_N, Q_U and the RTA kappa come from the same per-row arithmetic as the
single context and must agree to FP64 rounding (1e-12); the CG products are
summed in another order (dot kernels after the exchange instead of the gemv
partials), so the CG kappa and solution carry the CG tolerance of the other
parity tests (1e-8) and the iteration count must match.
"""
import threading

import numpy as np
import pytest

from conftest import make_case
from test_gpu_parity import close

pytestmark = pytest.mark.gpu


class InProcessGather:
    """All-gather among `n` threads: each deposits its block, waits for the
    others, then reads the concatenation in rank order."""

    def __init__(self, n):
        self.n = n
        self.blocks = [None] * n
        self.barrier = threading.Barrier(n, timeout=120)

    def for_rank(self, rank):
        def gather(mine, counts):
            self.blocks[rank] = np.array(mine)
            self.barrier.wait()
            out = np.concatenate([self.blocks[k] for k in range(self.n)])
            self.barrier.wait()  # nobody overwrites a block before everyone has read it
            return out
        return gather


def run_ranks(ald_lib, d, nranks, tempk):
    ctxs = [ald_lib.Context(d) for _ in range(nranks)]
    g = InProcessGather(nranks)
    outs, errs = [None] * nranks, []

    def work(r):
        try:
            outs[r] = ctxs[r].kappa_pipeline_sharded(r, nranks, g.for_rank(r), tempk)
        except Exception as ex:
            errs.append(ex)
            g.barrier.abort()

    th = [threading.Thread(target=work, args=(r,)) for r in range(nranks)]
    for t in th:
        t.start()
    for t in th:
        t.join(timeout=600)
    ranges = [ctxs[r].shard_rows(r, nranks) for r in range(nranks)]
    for c in ctxs:
        c.close()
    if errs:
        raise errs[0]
    return outs, ranges


@pytest.mark.parametrize("cfg,mesh,kw,nranks", [(1, (6, 6, 6), {}, 2), (1, (6, 6, 6), {}, 3),
                                                 (0, (6, 6, 6), {"delta": "gauss"}, 2),
                                                 (0, (4, 4, 4), {"delta": "tetra", "iso": 1}, 3)],
                         ids=["nacl6_2", "nacl6_3", "lj6_gauss_2", "lj4_iso_3"])
def test_sharded_pipeline_matches_single_context(ald_lib, workdir, cfg, mesh, kw, nranks):
    d = make_case(workdir, cfg, mesh, **kw)
    one = ald_lib.Context(d)
    ref = one.kappa_pipeline()
    tempk = one.info.tempk
    nibz = one.nibz
    one.close()
    outs, ranges = run_ranks(ald_lib, d, nranks, tempk)
    assert ranges == [ald_lib.shard_rows(nibz, r, nranks) for r in range(nranks)]
    for o in outs:
        for key in ("Q", "QN", "QU"):
            ok, worst = close(o[key], ref[key], rtol=1e-12, atol=1e-14)
            assert ok, (key, worst)
        ok, worst = close(o["kappa_rta_modes"], ref["kappa_rta_modes"], rtol=1e-12, atol=1e-12)
        assert ok, worst
        assert o["cg_iters"] == ref["cg_iters"]
        ok, worst = close(o["kappa_cg_modes"], ref["kappa_cg_modes"], rtol=1e-8, atol=1e-10)
        assert ok, worst
        ok, worst = close(o["x"], ref["x"], rtol=1e-8, atol=1e-10)
        assert ok, worst
    # the replicated CG gives every rank the same kappa
    for o in outs[1:]:
        assert np.array_equal(o["kappa_cg_modes"], outs[0]["kappa_cg_modes"])
