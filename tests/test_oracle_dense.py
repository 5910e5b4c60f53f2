"""The factorised CPU |V3|^2 (tests/oracle_dense.py) against the literal
oracle's term-by-term matrix_elt_simplified (CPU).

oracle_dense stands in for the literal oracle where that one is out of
reach (the 192-band cell); this pins it on cells where both run: the
rock-salt crystal (6 bands) and the 8-atom LJ superlattice (24 bands,
nearest-neighbour cutoff).  Bars: 1e-12 relative normwise, and per element
|fac - lit| <= 1e-10 |lit| + 1e-12 max|lit|, the FP64 bar of the GPU tests
(the sums are reordered, so entries that cancel to near zero differ most).
"""
import numpy as np
import pytest

import oracle_dense
from conftest import make_case


@pytest.mark.parametrize("cfg,mesh,kw,rows", [(1, (4, 4, 4), {}, (1, 3)),
                                             (3, (2, 4, 4), {"p": 2, "rc_sigma": 1.2}, (2, 2))],
                         ids=["rocksalt6", "superlattice24"])
def test_factorised_v3_matches_literal(oracle_lib, workdir, cfg, mesh, kw, rows):
    d = make_case(workdir, cfg, mesh, **kw)
    O = oracle_lib.Oracle(d)
    O.mesh()
    O.phonons()
    lit = O.v3(*rows)
    fac = oracle_dense.v3_factorised(O, *rows)
    scale = np.abs(lit).max()
    assert np.linalg.norm(fac - lit) <= 1e-12 * np.linalg.norm(lit)
    assert np.all(np.abs(fac - lit) <= 1e-10 * np.abs(lit) + 1e-12 * scale)
