"""The row-sharded pipeline across processes (GPU).

Two ranks run as two processes on the one GPU of this test, each with its own
context, exchanging Q and the CG products through torch.distributed (gloo):
over host buffers (ald_kappa_pipeline_sharded) and over device buffers
(ald_kappa_pipeline_sharded_dev, the NCCL-style path bench.py takes on
several GPUs).  No kernel of one rank waits on the other: the exchanges run
on the host between launches.  Results against a single context: Q, Q_N,
Q_U to 1e-12, kappa and the CG solution to 1e-10, the same iterations.
"""
import os
import socket
import subprocess
import sys

import numpy as np
import pytest

from conftest import make_case
from test_gpu_parity import close

pytestmark = pytest.mark.gpu

HERE = os.path.dirname(os.path.abspath(__file__))


def _free_port():
    s = socket.socket()
    s.bind(("127.0.0.1", 0))
    p = s.getsockname()[1]
    s.close()
    return p


def _run_ranks(d, mode, out, world=2):
    port = _free_port()
    procs = []
    for r in range(world):
        env = dict(os.environ, RANK=str(r), WORLD_SIZE=str(world), LOCAL_RANK="0", MASTER_ADDR="127.0.0.1",
                   MASTER_PORT=str(port))
        procs.append(subprocess.Popen([sys.executable, os.path.join(HERE, "shard_worker.py"), d, mode, out], env=env,
                                      stdout=subprocess.PIPE, stderr=subprocess.STDOUT, text=True))
    logs = []
    for p in procs:
        try:
            o, _ = p.communicate(timeout=300)
        except subprocess.TimeoutExpired:
            p.kill()
            o, _ = p.communicate()
        logs.append(o)
    for p, o in zip(procs, logs):
        assert p.returncode == 0, o[-3000:]


@pytest.mark.parametrize("mode", ["host", "device"])
@pytest.mark.parametrize("cfg,mesh,kw", [(1, (6, 6, 6), {}), (0, (6, 6, 6), {"delta": "gauss"})],
                         ids=["nacl6", "lj6_gauss"])
def test_sharded_pipeline_two_processes(ald_lib, workdir, tmp_path, cfg, mesh, kw, mode):
    d = make_case(workdir, cfg, mesh, **kw)
    out = str(tmp_path / ("rank0_%s.npz" % mode))
    _run_ranks(d, mode, out)
    got = np.load(out)
    ctx = ald_lib.Context(d)
    ref = ctx.kappa_pipeline()
    ctx.close()
    for key in ("Q", "QN", "QU"):
        ok, worst = close(got[key], ref[key], rtol=1e-12, atol=1e-14)
        assert ok, (key, worst)
    assert int(got["cg_iters"]) == ref["cg_iters"]
    for key in ("kappa_rta_modes", "kappa_cg_modes"):
        ok, worst = close(got[key], ref[key], atol=1e-10)
        assert ok, (key, worst)
    ok, worst = close(got["x"], ref["x"], atol=1e-10)
    assert ok, ("x", worst)
