"""The C ABI library on the CPU: symbols, host-side tables, error codes."""
import os
import re
import shutil

import numpy as np
import pytest

import example_inputs as E
from conftest import ROOT, make_case


def _declared_symbols():
    txt = open(os.path.join(ROOT, "include", "ald.h")).read()
    return sorted(set(re.findall(r"\b(ald_[a-z0-9_]+)\s*\(", txt)))


def test_library_exports_every_declared_symbol(ald_lib):
    import ctypes
    L = ctypes.CDLL(ald_lib.LIB_PATH)
    missing = [s for s in _declared_symbols() if not hasattr(L, s)]
    assert not missing, missing
    assert set(ald_lib.EXPORTS) <= set(_declared_symbols())


@pytest.mark.parametrize("cfg,mesh", [(0, (10, 10, 10)), (1, (16, 16, 16)), (1, (6, 6, 6)), (2, (8, 8, 8))])
def test_host_tables_equal_oracle(ald_lib, oracle_lib, workdir, cfg, mesh):
    d = make_case(workdir, cfg, mesh)
    info, M = ald_lib.read_mesh(d)
    O = oracle_lib.Oracle(d)
    O.mesh()
    R = O.ibz()
    assert info.nibz == O.nibz and info.lattpgcount == O.npg
    assert np.array_equal(M["kpc"], O.kpc())
    assert np.array_equal(M["mapinv"], R["mapinv"])
    assert np.array_equal(M["mapibz"], R["mapibz"])
    assert np.array_equal(M["kibz"], R["kibz"])
    assert np.allclose(M["wibz"], R["wibz"], rtol=0, atol=1e-15)


@pytest.mark.parametrize("name", ["ge_example", "gese_example"])
def test_host_tables_equal_reference_ibz(ald_lib, workdir, name):
    d = os.path.join(str(workdir), "abi_" + name)
    z = E.materialize(name, d)
    info, M = ald_lib.read_mesh(d)
    assert info.nibz == len(z["out_ibz_w"])
    assert np.abs(M["kibz"].T - z["out_ibz_kcart"]).max() < 6e-5
    assert np.abs(M["wibz"] - z["out_ibz_w"]).max() < 1e-8


def test_missing_file_is_an_io_error(ald_lib, workdir):
    d = make_case(workdir, 1, (4, 4, 4))
    bad = os.path.join(str(workdir), "bad_missing")
    shutil.copytree(d, bad, dirs_exist_ok=True)
    os.remove(os.path.join(bad, "fc2.dat"))
    with pytest.raises(ald_lib.AldError) as e:
        ald_lib.read_mesh(bad)
    assert e.value.code == 2


def test_fc3_term_count_mismatch_is_an_io_error(ald_lib, workdir):
    d = make_case(workdir, 1, (4, 4, 4))
    bad = os.path.join(str(workdir), "bad_count")
    shutil.copytree(d, bad, dirs_exist_ok=True)
    lines = open(os.path.join(bad, "fc3.dat")).read().splitlines()
    open(os.path.join(bad, "fc3.dat"), "w").write("\n".join(lines[:-1]) + "\n")
    with pytest.raises(ald_lib.AldError) as e:
        ald_lib.read_mesh(bad)
    assert e.value.code == 2
    assert "READ_FC3" in str(e.value)


def test_incompatible_masses_are_rejected(ald_lib, workdir):
    d = make_case(workdir, 1, (4, 4, 4))
    bad = os.path.join(str(workdir), "bad_mass")
    shutil.copytree(d, bad, dirs_exist_ok=True)
    p = os.path.join(bad, "lat_fc.dat")
    txt = open(p).read().replace(" 22.99\n", " 23.0\n", 1)
    open(p, "w").write(txt)
    with pytest.raises(ald_lib.AldError) as e:
        ald_lib.read_mesh(bad)
    assert "not compatible" in str(e.value)


def test_create_without_device_fails_cleanly(ald_lib, workdir):
    import torch
    if torch.cuda.is_available():
        pytest.skip("a GPU is present")
    d = make_case(workdir, 1, (4, 4, 4))
    with pytest.raises(ald_lib.AldError) as e:
        ald_lib.Context(d)
    assert e.value.code == 7


@pytest.mark.parametrize("cfg,mesh,kw", [(3, (6, 12, 12), {"p": 2}), (3, (3, 12, 12), {"p": 5}),
                                         (4, (4, 4, 4), {}), (1, (5, 5, 5), {})])
def test_host_tables_equal_oracle_large_cells(ald_lib, oracle_lib, workdir, cfg, mesh, kw):
    """The superlattices (point group of 16 ops, an odd mesh edge) and the
    192-band cell (an FC3 file of the size the worker pool parses in
    parallel): mesh, IBZ and weights against the oracle."""
    d = make_case(workdir, cfg, mesh, **kw)
    info, M = ald_lib.read_mesh(d)
    O = oracle_lib.Oracle(d)
    O.mesh()
    R = O.ibz()
    assert info.nibz == O.nibz and info.lattpgcount == O.npg
    assert np.array_equal(M["kpc"], O.kpc())
    assert np.array_equal(M["mapinv"], R["mapinv"])
    assert np.array_equal(M["mapibz"], R["mapibz"])
    assert np.allclose(M["wibz"], R["wibz"], rtol=0, atol=1e-15)


def _fc3_variant(workdir, tag, edit):
    d = make_case(workdir, 1, (4, 4, 4))
    bad = os.path.join(str(workdir), tag)
    shutil.copytree(d, bad, dirs_exist_ok=True)
    p = os.path.join(bad, "fc3.dat")
    lines = open(p).read().splitlines()
    open(p, "w").write("\n".join(edit(lines)) + "\n")
    return bad


def test_fc3_blank_records_are_skipped(ald_lib, workdir):
    """Blank records between terms: a list-directed READ passes over them,
    so the file reads as without them (the same mesh and IBZ)."""
    d = make_case(workdir, 1, (4, 4, 4))
    spaced = _fc3_variant(workdir, "fc3_blank", lambda L: L[:1] + [x for l in L[1:] for x in (l, "   ")])
    a, Ma = ald_lib.read_mesh(d)
    b, Mb = ald_lib.read_mesh(spaced)
    assert (a.nterms3, a.nibz) == (b.nterms3, b.nibz)
    assert np.array_equal(Ma["mapibz"], Mb["mapibz"])


def test_fc3_short_record_is_truncated(ald_lib, workdir):
    """A term record with a value missing: the READ takes the next record's
    values, and the file ends before the last term (the sequential reader's
    error, whichever worker met the short record)."""
    def drop_value(L):
        j = len(L) // 2
        L = list(L)
        L[j] = " ".join(L[j].split()[:-1])
        return L
    bad = _fc3_variant(workdir, "fc3_short", drop_value)
    with pytest.raises(ald_lib.AldError) as e:
        ald_lib.read_mesh(bad)
    assert e.value.code == 2
    assert "truncated" in str(e.value)


def test_fc3_index_out_of_range(ald_lib, workdir):
    def bad_xyz(L):
        L = list(L)
        t = L[-1].split()
        t[3] = "4"  # the first xyz index of the last term
        L[-1] = " ".join(t)
        return L
    bad = _fc3_variant(workdir, "fc3_xyz", bad_xyz)
    with pytest.raises(ald_lib.AldError) as e:
        ald_lib.read_mesh(bad)
    assert e.value.code == 2
    assert "out of range" in str(e.value)


def test_host_tables_from_concurrent_threads(ald_lib, workdir):
    """Several host threads reading input directories at once (as contexts
    created on different threads do): every thread shares the library's one
    worker pool, and each gets the tables a lone call gives."""
    import threading
    dirs = [make_case(workdir, 1, (6, 6, 6)), make_case(workdir, 0, (10, 10, 10)),
            make_case(workdir, 3, (6, 12, 12), p=2), make_case(workdir, 1, (16, 16, 16))]
    want = [ald_lib.read_mesh(d)[1] for d in dirs]
    got, errs = {}, []

    def work(i, d):
        try:
            for _ in range(3):
                got[(i, _)] = ald_lib.read_mesh(d)[1]
        except Exception as e:  # reported below
            errs.append(e)
    th = [threading.Thread(target=work, args=(i, d)) for i, d in enumerate(dirs * 2)]
    for t in th:
        t.start()
    for t in th:
        t.join()
    assert not errs, errs
    for (i, _), M in got.items():
        for k in ("mapibz", "mapinv", "kpc", "wibz"):
            assert np.array_equal(M[k], want[i % len(dirs)][k])


@pytest.fixture(scope="module")
def fc_reader(tmp_path_factory):
    """The library's reader (ald_host.cpp) built into a small program that
    prints the FC values it read."""
    import subprocess
    exe = str(tmp_path_factory.mktemp("fcread") / "fc_read")
    src = os.path.join(ROOT, "anharmonic-lattice-dynamics_b200", "csrc")
    subprocess.check_call(["g++", "-std=c++17", "-O2", "-I/usr/local/cuda/include", "-o", exe,
                           os.path.join(ROOT, "tests", "fc_read_harness.cpp"), os.path.join(src, "ald_host.cpp"),
                           os.path.join(src, "ald_pool.cpp"), "-L/usr/local/cuda/lib64", "-lcudart", "-lpthread",
                           "-Wl,-rpath,/usr/local/cuda/lib64"])
    return exe


def test_fc_values_read_as_strtod_reads_them(fc_reader, workdir):
    """Every FC3 value written in another Fortran-readable form -- a D
    exponent, a leading '+', no leading digit, a subnormal, a long token --
    reads to the double that strtod gives for it (Python's float is the same
    correctly rounded conversion), in the records the worker pool parses."""
    import subprocess
    rng = np.random.default_rng(17)
    forms = [lambda v: "%.17E" % v, lambda v: ("%.15E" % v).replace("E", "D"), lambda v: "%+.12e" % v,
             lambda v: ("%.9f" % v).replace("0.", ".", 1) if abs(v) < 1 else "%.9f" % v,
             lambda v: "%.40e" % v, lambda v: "%.6g" % (v * 1e-310), lambda v: "%.17g" % v]
    expect = []

    def edit(lines):
        out = lines[:1]
        for j, l in enumerate(lines[1:]):
            t = l.split()
            v = rng.standard_normal() * 10.0 ** rng.integers(-6, 4)
            tok = forms[j % len(forms)](v)
            expect.append(float(tok.replace("D", "e")))
            out.append(" ".join(t[:-1] + [tok]))
        return out
    d = _fc3_variant(workdir, "fc3_forms", edit)
    txt = subprocess.run([fc_reader, d], capture_output=True, text=True, check=True).stdout.split("\n")
    f3 = [float.fromhex(l.split()[1]) for l in txt if l.startswith("f3 ")]
    assert len(f3) == len(expect) > 256
    assert all(a == b for a, b in zip(f3, expect)), next((i, a, b) for i, (a, b) in enumerate(zip(f3, expect))
                                                         if a != b)
    # the index tuples are those of the file
    lines = open(os.path.join(d, "fc3.dat")).read().split("\n")[1:]
    t3 = [tuple(int(x) for x in l.split()[2:8]) for l in txt if l.startswith("f3 ")]
    assert t3 == [tuple(int(x) for x in l.split()[2:8]) for l in lines if l.strip()]
