"""ald_cg_quadratic_static against ald_cg_quadratic (GPU).

ald_cg_quadratic_static serves callers whose device memory all comes from
their own pool (a host code that sets up its device arrays once, a solver
inside another framework's allocator): they pass device buffers and the
library allocates nothing, keeping its CG work vectors in a fixed __device__
array.  Its results must equal those of the allocating entry point
ald_cg_quadratic on the same system, within the CG tolerance of the other
parity tests (rtol 1e-10, atol 1e-10 of the largest entry), on two calls in
a row -- the second of a different size, so that a call never depends on
what the previous one left in the shared array -- and the second call must
leave the device's free memory exactly as it found it.

This file is collected last so that a run stopping at its first failure has
already run every other test.
"""
import numpy as np
import pytest

pytestmark = pytest.mark.gpu


def _spd_system(n, seed):
    """A seeded symmetric positive-definite system with a spread spectrum,
    plus an initial guess, in the reference's column-major layout."""
    rng = np.random.default_rng(seed)
    Q, _ = np.linalg.qr(rng.standard_normal((n, n)))
    lam = np.geomspace(1.0, 50.0, n)
    A = np.asfortranarray((Q * lam) @ Q.T)
    A = np.asfortranarray(0.5 * (A + A.T))
    b = rng.standard_normal(n)
    x0 = 0.1 * rng.standard_normal(n)
    return A, b, x0


def _close(g, r, rtol=1e-10, atol=1e-10):
    scale = np.abs(r).max()
    return bool(np.all(np.abs(g - r) <= rtol * np.abs(r) + atol * scale))


def test_cg_static_matches_allocating_entry_point(ald_lib):
    import torch
    dev = torch.device("cuda:0")
    torch.cuda.set_device(dev)
    stream = torch.cuda.current_stream(dev)
    for call, (n, seed, ndig) in enumerate([(600, 11, 4), (257, 12, 2)]):
        A, b, x0 = _spd_system(n, seed)
        x_ref, fm_ref, it_ref, st_ref = ald_lib.cg_quadratic(A, b, x0, max_iter=100, n_dig_accur=ndig)
        # column-major a(n,n) on the device: the transpose's C-order buffer
        dA = torch.from_numpy(np.ascontiguousarray(A.T)).to(dev)
        db = torch.from_numpy(b.copy()).to(dev)
        dx = torch.from_numpy(x0.copy()).to(dev)
        torch.cuda.synchronize()
        free0 = torch.cuda.mem_get_info(dev)[0]
        fm, it, st = ald_lib.cg_quadratic_static(n, dA.data_ptr(), db.data_ptr(), dx.data_ptr(), max_iter=100,
                                                 n_dig_accur=ndig, stream=stream.cuda_stream)
        if call == 1:  # the first call may load the library's module; later calls allocate nothing
            assert torch.cuda.mem_get_info(dev)[0] == free0
        x = dx.cpu().numpy()
        assert st == st_ref, (call, st, st_ref)
        assert it == it_ref, (call, it, it_ref)
        assert _close(x, x_ref), (call, float(np.abs(x - x_ref).max() / np.abs(x_ref).max()))
        assert abs(fm - fm_ref) <= 1e-8 * abs(fm_ref) + 1e-12, (call, fm, fm_ref)


def test_cg_static_rejects_sizes_above_its_maximum(ald_lib):
    import torch
    dev = torch.device("cuda:0")
    n = ald_lib.CG_STATIC_MAX_N + 1
    small = torch.zeros(4, dtype=torch.float64, device=dev)
    # the size check comes before any pointer is touched
    with pytest.raises(ald_lib.AldError) as e:
        ald_lib.cg_quadratic_static(n, small.data_ptr(), small.data_ptr(), small.data_ptr())
    assert "ALD_CG_STATIC_MAX_N" in str(e.value)
    # host memory is refused instead of being handed to a kernel
    h = np.zeros(16)
    with pytest.raises(ald_lib.AldError):
        ald_lib.cg_quadratic_static(4, h.ctypes.data, h.ctypes.data, h.ctypes.data)
