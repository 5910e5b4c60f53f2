import os
import sys

import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
for p in (os.path.join(ROOT, "anharmonic-lattice-dynamics_b200", "python"), os.path.join(ROOT, "tests"),
          os.path.join(ROOT, "tests", "golden")):
    if p not in sys.path:
        sys.path.insert(0, p)


def pytest_configure(config):
    config.addinivalue_line("markers", "gpu: needs a CUDA device (B200); parity tests of the CUDA path")


@pytest.fixture(scope="session")
def oracle_lib():
    import oracle_py
    oracle_py.build()
    return oracle_py


@pytest.fixture(scope="session")
def ald_lib():
    from ald import build
    build.build()
    import ald
    ald.lib()
    return ald


@pytest.fixture(scope="session")
def workdir(tmp_path_factory):
    return tmp_path_factory.mktemp("ald")


def make_case(workdir, cfg, mesh, **kw):
    """Write one synthetic configuration into workdir and return its path."""
    from ald import inputs as I
    skw = {k: kw.pop(k) for k in ("rc_sigma", "p", "s") if k in kw}
    st, rp = I.config(cfg, mesh=mesh, **skw)
    kw.update({"_" + k: v for k, v in skw.items()})  # part of the directory tag only
    for k, v in kw.items():
        if k.startswith("_"):
            continue
        setattr(rp, k, v)
    tag = "c%d_%s_%s" % (cfg, "x".join(map(str, mesh)), "_".join("%s%s" % kv for kv in sorted(kw.items())))
    d = os.path.join(str(workdir), tag)
    if not os.path.exists(os.path.join(d, "fc3.dat")):
        I.write_inputs(st, rp, d)
    return d
