"""Python binding of libald (the C ABI declared in include/ald.h).

Names follow the THERMACOND subroutines each call replaces
(calculate_w3_ibz_split_sq, calculate_FGR_mpi2, calculate_tauRTA_mpi2,
CollisionMatrix_mpi, cal_RHS_IBZ, cg_quadratic, mode_kappa_d ...).
Arrays come back as numpy arrays in the reference's Fortran layout
(order='F', 1-based index values), so indexing reads like the Fortran.

All compute runs in the CUDA library; if libald.so is missing the import
fails -- there is no CPU fallback.
"""
from __future__ import annotations

import ctypes as C
import os
from typing import Optional, Sequence, Tuple

import numpy as np

_PKG = os.path.dirname(os.path.dirname(os.path.dirname(os.path.abspath(__file__))))
LIB_PATH = os.path.join(_PKG, "lib", "libald.so")

ALD_OK = 0
ALD_WARN_CG_MAXITER = 100
STATUS = {1: "ALD_ERR_ARG", 2: "ALD_ERR_IO", 3: "ALD_ERR_NOT_KPOINT", 4: "ALD_ERR_DEN_ZERO", 5: "ALD_ERR_NBE",
          6: "ALD_ERR_INDEX", 7: "ALD_ERR_CUDA", 8: "ALD_ERR_UNSUPPORTED", 9: "ALD_ERR_NOMEM",
          100: "ALD_WARN_CG_MAXITER"}
DELTA_TETRA, DELTA_GAUSS = 0, 1
FP64, MIXED, MIXED_FP32 = 0, 1, 2
CG_REFERENCE, CG_RESIDUAL = 0, 1
DET_AUTO = -1  # Options.deterministic: FP64 deterministic, mixed with FP64 atomics


class AldError(RuntimeError):
    def __init__(self, code: int, msg: str):
        super().__init__("%s (%d): %s" % (STATUS.get(code, "?"), code, msg))
        self.code = code


class Options(C.Structure):
    _fields_ = [("delta", C.c_int), ("precision", C.c_int), ("cg_stop", C.c_int), ("cg_max_iter", C.c_int),
                ("cg_ndig", C.c_int), ("cg_tol", C.c_double), ("width_cm", C.c_double), ("device", C.c_int),
                ("chunk_bytes", C.c_size_t), ("deterministic", C.c_int)]


class Info(C.Structure):
    _fields_ = [("ndyn", C.c_int), ("natoms0", C.c_int), ("nc", C.c_int * 3), ("nkc", C.c_int), ("nibz", C.c_int),
                ("nterms2", C.c_int), ("nterms3", C.c_int), ("natoms", C.c_int), ("lattpgcount", C.c_int),
                ("born_flag", C.c_int), ("tempk", C.c_double), ("width_cm", C.c_double), ("volume_r", C.c_double)]


class KappaResult(C.Structure):
    _fields_ = [("kappa_rta", C.c_double * 9), ("kappa_cg", C.c_double * 9), ("cg_iters", C.c_int),
                ("status_cg", C.c_int), ("cg_err", C.c_double), ("stage_ms", C.c_double * 10),
                ("launches", C.c_int * 10), ("triplet_bands", C.c_double), ("d2h_bytes", C.c_double)]


class Tuning(C.Structure):
    _fields_ = [("chunk_bytes", C.c_size_t), ("v3_rows_per_cta", C.c_int), ("v3_epilogue_wg", C.c_int),
                ("v3_gemm_bytes", C.c_size_t), ("ms", C.c_double), ("from_cache", C.c_int), ("candidates", C.c_int)]


STAGES = ["phonons", "v3", "delta", "q_reduce", "rta", "collision", "rhs", "cg", "kappa_cg", "total"]


_lib = None
dp = C.POINTER(C.c_double)
ip = C.POINTER(C.c_int)
EXPORTS = ["ald_default_options", "ald_last_error", "ald_create_from_dir", "ald_destroy", "ald_get_info",
           "ald_read_mesh", "ald_get_mesh", "ald_get_frequencies", "ald_set_phonons",
           "ald_calculate_w3_ibz_split_sq", "ald_calculate_fgr", "ald_distribution", "ald_calculate_tau_rta",
           "ald_rta_kappa", "ald_collision_matrix", "ald_rhs", "ald_cg_quadratic", "ald_mode_kappa_d",
           "ald_kappa_pipeline", "ald_set_stream", "ald_h2d_bytes", "ald_cg_quadratic_static", "ald_update_mpi",
           "ald_kappa_iterative", "ald_collision_matrix_iso", "ald_p_iso_split", "ald_set_isotope_g",
           "ald_get_isotope_g", "ald_shard_rows", "ald_kappa_pipeline_sharded", "ald_kappa_pipeline_sharded_dev", "ald_tau_eff", "ald_qandtau",
           "ald_write_kappa", "ald_write_job1_files", "ald_format_value", "ald_make_kp_bs",
           "ald_function_self_w", "ald_self_energy_bs", "ald_release_cached_memory", "ald_kappa_batched", "ald_release_workspaces",
           "ald_autotune", "ald_set_tuning", "ald_weight_tet"]
CG_STATIC_MAX_N = 32768  # ALD_CG_STATIC_MAX_N of include/ald.h


def lib():
    global _lib
    if _lib is None:
        if not os.path.exists(LIB_PATH):
            raise ImportError("libald.so not built (%s); run anharmonic-lattice-dynamics_b200/python/ald/build.py"
                              % LIB_PATH)
        L = C.CDLL(LIB_PATH)
        L.ald_last_error.restype = C.c_char_p
        L.ald_default_options.argtypes = [C.POINTER(Options)]
        L.ald_create_from_dir.argtypes = [C.c_char_p, C.POINTER(Options), C.POINTER(C.c_void_p)]
        L.ald_destroy.argtypes = [C.c_void_p]
        L.ald_destroy.restype = None
        L.ald_h2d_bytes.restype = C.c_double
        L.ald_h2d_bytes.argtypes = [C.c_void_p]
        L.ald_set_stream.argtypes = [C.c_void_p, C.c_void_p]
        L.ald_cg_quadratic_static.argtypes = [C.c_int, C.c_void_p, C.c_void_p, C.c_void_p, C.POINTER(C.c_double),
                                              C.c_int, C.c_int, C.POINTER(C.c_int), C.c_void_p]
        L.ald_format_value.argtypes = [C.c_char_p, C.c_double, C.c_char_p, C.c_int]
        L.ald_release_cached_memory.restype = None
        L.ald_autotune.argtypes = [C.c_void_p, C.c_char_p, C.c_double, C.POINTER(Tuning)]
        L.ald_set_tuning.argtypes = [C.c_void_p, C.POINTER(Tuning)]
        L.ald_weight_tet.argtypes = [C.c_int, dp, C.c_double, C.c_int, dp]
        for n in EXPORTS[2:]:
            if n not in ("ald_destroy", "ald_h2d_bytes", "ald_release_cached_memory"):
                getattr(L, n).restype = C.c_int
        _lib = L
    return _lib


def kappa_batched(contexts, tempk):
    """ald_kappa_batched: the job=1 pipeline on several contexts at once.
    Returns one dict per context (kappa_rta, kappa_cg, cg_iters, status_cg,
    stage_ms, triplet_bands) and the per-context status codes."""
    n = len(contexts)
    hs = (C.c_void_p * n)(*[c.h.value for c in contexts])
    tk = (C.c_double * n)(*([float(tempk)] * n if np.isscalar(tempk) else [float(t) for t in tempk]))
    res = (KappaResult * n)()
    st = (C.c_int * n)()
    r = lib().ald_kappa_batched(n, hs, tk, res, st)
    _check(r)
    out = [{"kappa_rta": np.array(x.kappa_rta).reshape(3, 3, order="F"),
            "kappa_cg": np.array(x.kappa_cg).reshape(3, 3, order="F"), "cg_iters": x.cg_iters,
            "status_cg": x.status_cg, "stage_ms": dict(zip(STAGES, list(x.stage_ms))),
            "triplet_bands": x.triplet_bands} for x in res]
    return out, list(st)


def release_cached_memory() -> None:
    """Return the device blocks the library keeps for reuse to the driver."""
    lib().ald_release_cached_memory()


def format_value(edit: str, value) -> str:
    """One value formatted as the output writers format it (host only):
    edit "Iw", "Fw.d", "Ew.d", "Gw.d", "*" (list-directed REAL(8)) or "*I"
    (list-directed INTEGER)."""
    buf = C.create_string_buffer(512)
    n = lib().ald_format_value(edit.encode(), C.c_double(value), buf, 512)
    if n < 0:
        raise ValueError("bad edit descriptor %r" % edit)
    return buf.value.decode()


def _p(a):
    return None if a is None else a.ctypes.data_as(dp)


def _check(r: int, allow=(ALD_OK,)) -> int:
    if r not in allow:
        raise AldError(r, lib().ald_last_error().decode())
    return r


def default_options(**kw) -> Options:
    o = Options()
    lib().ald_default_options(C.byref(o))
    for k, v in kw.items():
        setattr(o, k, v)
    return o


def read_mesh(d: str):
    """Host-only mesh/IBZ tables of an input directory (no GPU needed)."""
    info = Info()
    _check(lib().ald_read_mesh(d.encode(), C.byref(info), None, None, None, None, None))
    kpc = np.zeros((3, info.nkc), order="F")
    mapibz = np.zeros(info.nkc, dtype=np.int32)
    mapinv = np.zeros(info.nibz, dtype=np.int32)
    kibz = np.zeros((3, info.nibz), order="F")
    wibz = np.zeros(info.nibz)
    _check(lib().ald_read_mesh(d.encode(), C.byref(info), _p(kpc), mapibz.ctypes.data_as(ip),
                               mapinv.ctypes.data_as(ip), _p(kibz), _p(wibz)))
    return info, {"kpc": kpc, "mapibz": mapibz, "mapinv": mapinv, "kibz": kibz, "wibz": wibz}


class Context:
    """One loaded system (lat_fc/fc2/fc3/params of a directory) on one GPU."""

    def __init__(self, d: str, options: Optional[Options] = None):
        h = C.c_void_p()
        _check(lib().ald_create_from_dir(d.encode(), C.byref(options) if options is not None else None, C.byref(h)))
        self.h = h
        info = Info()
        _check(lib().ald_get_info(h, C.byref(info)))
        self.info = info
        self.ndyn, self.nkc, self.nibz = info.ndyn, info.nkc, info.nibz
        self.nc = tuple(info.nc)

    def close(self):
        if getattr(self, "h", None):
            lib().ald_destroy(self.h)
            self.h = None

    def __del__(self):
        self.close()

    def __enter__(self):
        return self

    def __exit__(self, *a):
        self.close()

    def set_stream(self, stream_handle: Optional[int]):
        """Issue work on a caller's cudaStream_t (an int handle, e.g.
        torch.cuda.current_stream().cuda_stream); None restores the own stream."""
        _check(lib().ald_set_stream(self.h, C.c_void_p(stream_handle) if stream_handle else None))

    def h2d_bytes(self) -> float:
        return lib().ald_h2d_bytes(self.h)

    def autotune(self, cache_path=None, budget_s=0.0):
        """ald_autotune: time candidate launch shapes of the pipeline (or read
        them from the cache file), keep the fastest on this context; returns
        the choice as a dict."""
        t = Tuning()
        _check(lib().ald_autotune(self.h, cache_path.encode() if cache_path else None, float(budget_s), C.byref(t)))
        return {k: getattr(t, k) for k, _ in Tuning._fields_}

    def set_tuning(self, **kw):
        """ald_set_tuning: apply a choice (chunk_bytes, v3_rows_per_cta,
        v3_epilogue_wg, v3_gemm_bytes; missing fields = the built-in choice)."""
        t = Tuning()
        for k, v in kw.items():
            setattr(t, k, v)
        _check(lib().ald_set_tuning(self.h, C.byref(t)))

    def invalidate_phonons(self):
        """Make the next pipeline call recompute eigenpairs (get_frequencies)."""
        _check(lib().ald_get_frequencies(self.h, None, None, None))

    # ---------------------------------------------------------- tables
    def get_mesh(self):
        kpc = np.zeros((3, self.nkc), order="F")
        mapibz = np.zeros(self.nkc, dtype=np.int32)
        mapinv = np.zeros(self.nibz, dtype=np.int32)
        kibz = np.zeros((3, self.nibz), order="F")
        wibz = np.zeros(self.nibz)
        _check(lib().ald_get_mesh(self.h, _p(kpc), mapibz.ctypes.data_as(ip), mapinv.ctypes.data_as(ip), _p(kibz),
                                  _p(wibz)))
        return {"kpc": kpc, "mapibz": mapibz, "mapinv": mapinv, "kibz": kibz, "wibz": wibz}

    # ---------------------------------------------------------- stage 1
    def get_frequencies(self):
        """get_frequencies + subst_eivecs: eigenval(ndyn,nkc), eigenvec(ndyn,ndyn,nkc), veloc(3,ndyn,nkc)."""
        n, nk = self.ndyn, self.nkc
        ev = np.zeros((n, nk), order="F")
        vec = np.zeros((n, n, nk), dtype=complex, order="F")
        vel = np.zeros((3, n, nk), order="F")
        _check(lib().ald_get_frequencies(self.h, _p(ev), vec.ctypes.data_as(dp), _p(vel)))
        return ev, vec, vel

    def set_phonons(self, eigenval, eigenvec, veloc):
        ev = np.asfortranarray(eigenval, dtype=float)
        vec = np.asfortranarray(eigenvec, dtype=complex)
        vel = np.asfortranarray(veloc, dtype=float)
        _check(lib().ald_set_phonons(self.h, _p(ev), vec.ctypes.data_as(dp), _p(vel)))

    # ---------------------------------------------------------- stage 2-4
    def calculate_w3_ibz_split_sq(self, ksubset: Sequence[int]):
        k = (C.c_int * 2)(*ksubset)
        n, nk = self.ndyn, self.nkc
        out = np.zeros((ksubset[1] - ksubset[0] + 1, nk, n, n, n), order="F")
        _check(lib().ald_calculate_w3_ibz_split_sq(self.h, k, _p(out)))
        return out

    def calculate_fgr(self, ksubset, v33s8):
        k = (C.c_int * 2)(*ksubset)
        v = np.asfortranarray(v33s8, dtype=float)
        P1 = np.zeros_like(v, order="F")
        P2 = np.zeros_like(v, order="F")
        _check(lib().ald_calculate_fgr(self.h, k, _p(v), _p(P1), _p(P2)))
        return P1, P2

    def distribution(self, tempk: float):
        f = np.zeros((self.nkc, self.ndyn), order="F")
        d = np.zeros((self.nkc, self.ndyn), order="F")
        _check(lib().ald_distribution(self.h, C.c_double(tempk), _p(f), _p(d)))
        return f, d

    def calculate_tau_rta(self, ksubset, tempk, P1smpi, P2smpi, want_p=True):
        k = (C.c_int * 2)(*ksubset)
        nr = ksubset[1] - ksubset[0] + 1
        s1 = np.asfortranarray(P1smpi, dtype=float)
        s2 = np.asfortranarray(P2smpi, dtype=float)
        Q = np.zeros((nr, self.ndyn), order="F")
        QN, QU = np.zeros_like(Q), np.zeros_like(Q)
        P1 = np.zeros_like(s1, order="F") if want_p else None
        P2 = np.zeros_like(s1, order="F") if want_p else None
        _check(lib().ald_calculate_tau_rta(self.h, k, C.c_double(tempk), _p(s1), _p(s2), _p(Q), _p(QN), _p(QU),
                                           _p(P1), _p(P2)))
        return Q, QN, QU, P1, P2

    def rta_kappa(self, tempk, Q):
        q = np.asfortranarray(Q, dtype=float)
        FFF = np.zeros((self.nibz, self.ndyn, 3), order="F")
        kap = np.zeros((self.ndyn, 3, 3), order="F")
        _check(lib().ald_rta_kappa(self.h, C.c_double(tempk), _p(q), _p(FFF), _p(kap)))
        return FFF, kap

    def collision_matrix(self, ksubset, P1, P2):
        k = (C.c_int * 2)(*ksubset)
        nr = ksubset[1] - ksubset[0] + 1
        CM = np.zeros((nr * self.ndyn * 3, self.nibz * self.ndyn * 3), order="F")
        _check(lib().ald_collision_matrix(self.h, k, _p(np.asfortranarray(P1, dtype=float)),
                                          _p(np.asfortranarray(P2, dtype=float)), _p(CM)))
        return CM

    def collision_matrix_iso(self, P1, P2, Piso):
        """CollisionMatrix_iso (sub.f90:3387) over all IBZ rows."""
        n = self.nibz * self.ndyn * 3
        CM = np.zeros((n, n), order="F")
        f = lambda a: _p(np.asfortranarray(a, dtype=float))
        _check(lib().ald_collision_matrix_iso(self.h, f(P1), f(P2), f(Piso), _p(CM)))
        return CM

    def p_iso_split(self, ksubset):
        """P_iso_split (sub.f90:4825): Piso(nk1, ndyn) of IBZ rows ksubset."""
        k = (C.c_int * 2)(*ksubset)
        Piso = np.zeros((ksubset[1] - ksubset[0] + 1, self.ndyn), order="F")
        _check(lib().ald_p_iso_split(self.h, k, _p(Piso)))
        return Piso

    def set_isotope_g(self, g):
        """g (mass variance) per primitive atom, in place of the element table."""
        _check(lib().ald_set_isotope_g(self.h, _p(np.ascontiguousarray(g, dtype=float))))

    def isotope_g(self):
        g = np.zeros(self.info.natoms0)
        _check(lib().ald_get_isotope_g(self.h, _p(g)))
        return g

    def rhs(self, tempk):
        r = np.zeros(self.nibz * self.ndyn * 3)
        _check(lib().ald_rhs(self.h, C.c_double(tempk), _p(r)))
        return r

    def update_mpi(self, ksubset, P1, P2, Q, F_RTA, FFF):
        """update_mpi (sub.f90:2295): F2mpi(nk1, ndyn, 3) for IBZ rows ksubset."""
        k = (C.c_int * 2)(*ksubset)
        nr = ksubset[1] - ksubset[0] + 1
        F2 = np.zeros((nr, self.ndyn, 3), order="F")
        f = lambda a: _p(np.asfortranarray(a, dtype=float))
        _check(lib().ald_update_mpi(self.h, k, f(P1), f(P2), f(Q), f(F_RTA), f(FFF), _p(F2)))
        return F2

    def kappa_iterative(self, tempk=None, max_iter=150, update_mix=0.4):
        """The job=3 sequence (kappa.f90:1046-1487) on the device."""
        if tempk is None:
            tempk = self.info.tempk
        res = KappaResult()
        n, ni = self.ndyn, self.nibz
        Q = np.zeros((ni, n), order="F")
        kr = np.zeros((n, 3, 3), order="F")
        ki = np.zeros((n, 3, 3), order="F")
        F = np.zeros((ni, n, 3), order="F")
        r = _check(lib().ald_kappa_iterative(self.h, C.c_double(tempk), max_iter, C.c_double(update_mix),
                                             C.byref(res), _p(Q), _p(kr), _p(ki), _p(F)),
                   allow=(ALD_OK,))
        return {"kappa_rta": np.array(res.kappa_rta).reshape(3, 3, order="F"),
                "kappa_iter": np.array(res.kappa_cg).reshape(3, 3, order="F"), "iters": res.cg_iters,
                "normk": res.cg_err, "status": res.status_cg, "Q": Q, "kappa_rta_modes": kr,
                "kappa_iter_modes": ki, "F": F, "stage_ms": dict(zip(STAGES, res.stage_ms)),
                "launches": dict(zip(STAGES, res.launches)), "triplet_bands": res.triplet_bands}

    def mode_kappa_d(self, tempk, x):
        kap = np.zeros((self.ndyn, 3, 3), order="F")
        _check(lib().ald_mode_kappa_d(self.h, C.c_double(tempk), _p(np.ascontiguousarray(x, dtype=float)), _p(kap)))
        return kap

    def tau_eff(self, tempk, F, solution: int):
        """tauinv_eff(nibz, ndyn) per mode: mode_kappa's sum (solution 0, F =
        FFF(nibz,ndyn,3)) or mode_kappa_d's (solution 1, F = the CG solution)."""
        t = np.zeros((self.nibz, self.ndyn), order="F")
        f = np.asfortranarray(F, dtype=float) if solution == 0 else np.ascontiguousarray(F, dtype=float)
        _check(lib().ald_tau_eff(self.h, C.c_double(tempk), _p(f), int(solution), _p(t)))
        return t

    def qandtau(self, tempk, Q, QN, QU, qvalue_path: Optional[str] = None):
        """Qandtau (sub.f90:8198): tauinv_N, tauinv_U, tauinv_tot(nibz, ndyn) in
        1/s; writes Qvalue.dat to qvalue_path when given."""
        tN, tU, tT = (np.zeros((self.nibz, self.ndyn), order="F") for _ in range(3))
        f = lambda a: _p(np.asfortranarray(a, dtype=float))
        _check(lib().ald_qandtau(self.h, C.c_double(tempk), f(Q), f(QN), f(QU),
                                 qvalue_path.encode() if qvalue_path else None, _p(tN), _p(tU), _p(tT)))
        return tN, tU, tT

    def write_kappa(self, tempk, kappa_modes, tauinv_N, tauinv_U, tauinv_tot, tauinv_eff,
                    kappa_path: Optional[str] = None, tau_path: Optional[str] = None):
        """write_kappa (sub.f90:1818).  tauinv_N and tauinv_U must be float64
        Fortran-ordered arrays: zero entries become 1e10 in place, as in the
        reference."""
        for a in (tauinv_N, tauinv_U):
            if not (isinstance(a, np.ndarray) and a.dtype == np.float64 and a.flags.f_contiguous):
                raise TypeError("tauinv_N and tauinv_U must be float64 arrays in Fortran order")
        f = lambda a: _p(np.asfortranarray(a, dtype=float))
        _check(lib().ald_write_kappa(self.h, C.c_double(tempk), f(kappa_modes), _p(tauinv_N), _p(tauinv_U),
                                     f(tauinv_tot), f(tauinv_eff), kappa_path.encode() if kappa_path else None,
                                     tau_path.encode() if tau_path else None))

    def write_job1_files(self, out_dir: str, tempk, res: dict):
        """The five output files of kappa_full's job=1 block, from the dict
        kappa_pipeline() returns (it needs the per-mode arrays)."""
        f = lambda a: _p(np.asfortranarray(a, dtype=float))
        _check(lib().ald_write_job1_files(self.h, out_dir.encode(), C.c_double(tempk), f(res["Q"]), f(res["QN"]),
                                          f(res["QU"]), f(res["kappa_rta_modes"]), f(res["kappa_cg_modes"]),
                                          _p(np.ascontiguousarray(res["x"], dtype=float))))

    def make_kp_bs(self, d: str):
        """make_kp_bs (modules.f90:1507): kp_bs (3, nkp), dk_bs (nkp) of d/kpbs.params."""
        n = C.c_int(0)
        _check(lib().ald_make_kp_bs(self.h, d.encode(), C.byref(n), None, None, 0))
        kp = np.zeros((3, n.value), order="F")
        dk = np.zeros(n.value)
        _check(lib().ald_make_kp_bs(self.h, d.encode(), C.byref(n), _p(kp), _p(dk), n.value))
        return kp, dk

    def function_self_w(self, q, la, omega, temp, gauss=False):
        """function_self_w3 (gauss False) / function_self_w4 (True) for jobs
        q (3,n), la (n, 1-based), omega (n) and temp in cm^-1: nself, uself
        (n,) complex."""
        q = np.asfortranarray(q, dtype=float)
        n = q.shape[1]
        la = np.ascontiguousarray(la, dtype=np.int32)
        om = np.ascontiguousarray(omega, dtype=float)
        ns = np.zeros(2 * n)
        us = np.zeros(2 * n)
        _check(lib().ald_function_self_w(self.h, n, _p(q), la.ctypes.data_as(C.POINTER(C.c_int)), _p(om),
                                         C.c_double(temp), int(gauss), _p(ns), _p(us)))
        return ns[0::2] + 1j * ns[1::2], us[0::2] + 1j * us[1::2]

    def self_energy_bs(self, d: str, tempk, gauss=False, out_dir: Optional[str] = None):
        """The job=2 block: omega0 (ndyn, nkp), nself, uself (ndyn, nkp) complex
        along the path of d/kpbs.params; writes the lw-selfenergy files to
        out_dir when given."""
        kp, dk = self.make_kp_bs(d)
        n = kp.shape[1]
        om = np.zeros((self.ndyn, n), order="F")
        ns = np.zeros(2 * self.ndyn * n)
        us = np.zeros(2 * self.ndyn * n)
        _check(lib().ald_self_energy_bs(self.h, d.encode(), C.c_double(tempk), int(gauss), n, _p(om), _p(ns),
                                        _p(us), out_dir.encode() if out_dir else None))
        f = lambda a: (a[0::2] + 1j * a[1::2]).reshape(n, self.ndyn).T
        return {"kp_bs": kp, "dk_bs": dk, "omega0": om, "nself": f(ns), "uself": f(us)}

    def release_workspaces(self):
        """ald_release_workspaces: this context's pipeline workspaces back to the device-memory cache."""
        _check(lib().ald_release_workspaces(self.h))

    def kappa_pipeline(self, tempk: Optional[float] = None, want_modes=True):
        if tempk is None:
            tempk = self.info.tempk
        res = KappaResult()
        n, ni = self.ndyn, self.nibz
        Q = np.zeros((ni, n), order="F") if want_modes else None
        QN = np.zeros((ni, n), order="F") if want_modes else None
        QU = np.zeros((ni, n), order="F") if want_modes else None
        kr = np.zeros((n, 3, 3), order="F") if want_modes else None
        kc = np.zeros((n, 3, 3), order="F") if want_modes else None
        x = np.zeros(ni * n * 3) if want_modes else None
        _check(lib().ald_kappa_pipeline(self.h, C.c_double(tempk), C.byref(res), _p(Q), _p(QN), _p(QU), _p(kr),
                                        _p(kc), _p(x)))
        out = {"kappa_rta": np.array(res.kappa_rta).reshape(3, 3, order="F"),
               "kappa_cg": np.array(res.kappa_cg).reshape(3, 3, order="F"), "cg_iters": res.cg_iters,
               "status_cg": res.status_cg, "cg_err": res.cg_err,
               "stage_ms": dict(zip(STAGES, list(res.stage_ms))),
               "launches": dict(zip(STAGES, list(res.launches))),
               "triplet_bands": res.triplet_bands, "d2h_bytes": res.d2h_bytes}
        if want_modes:
            out.update({"Q": Q, "QN": QN, "QU": QU, "kappa_rta_modes": kr, "kappa_cg_modes": kc, "x": x})
        return out

    def shard_rows(self, rank: int, nranks: int) -> Tuple[int, int]:
        k = (C.c_int * 2)()
        _check(lib().ald_shard_rows(self.h, rank, nranks, k))
        return k[0], k[1]

    def kappa_pipeline_sharded(self, rank: int, nranks: int, gather, tempk: Optional[float] = None,
                               device: bool = False):
        """One rank of the row-sharded job=1 (ald_kappa_pipeline_sharded).
        `gather(mine, counts)` is the all-gather: it receives this rank's
        values (numpy) and the per-rank counts and returns every rank's values
        concatenated in rank order (e.g. torch_allgather()).  With device=True
        the exchange stays on the GPU (ald_kappa_pipeline_sharded_dev):
        `gather(mine_ptr, count, all_ptr, counts, stream)` gets device pointers
        and the context's stream (e.g. torch_allgather_device())."""
        if tempk is None:
            tempk = self.info.tempk
        err = []

        def cbd(user, mine, count, out, counts, nranks_, stream):
            try:
                gather(mine or 0, count, out or 0, [counts[k] for k in range(nranks_)], stream or 0)
                return 0
            except Exception as ex:  # reported after the call returns
                err.append(ex)
                return 1

        def cb(user, mine, count, out, counts, nranks_):
            try:
                cn = [counts[k] for k in range(nranks_)]
                a = np.ctypeslib.as_array(mine, shape=(count,)) if count > 0 else np.zeros(0)
                allv = np.asarray(gather(a.copy(), cn), dtype=float)
                if allv.shape != (sum(cn),):
                    raise ValueError("all-gather returned %s values, expected %d" % (allv.shape, sum(cn)))
                np.ctypeslib.as_array(out, shape=(sum(cn),))[:] = allv
                return 0
            except Exception as ex:  # reported after the call returns
                err.append(ex)
                return 1

        fn = ALLGATHER_DEV_FN(cbd) if device else ALLGATHER_FN(cb)
        entry = lib().ald_kappa_pipeline_sharded_dev if device else lib().ald_kappa_pipeline_sharded
        res = KappaResult()
        n, ni = self.ndyn, self.nibz
        Q, QN, QU = (np.zeros((ni, n), order="F") for _ in range(3))
        kr, kc = np.zeros((n, 3, 3), order="F"), np.zeros((n, 3, 3), order="F")
        x = np.zeros(ni * n * 3)
        r = entry(self.h, C.c_double(tempk), rank, nranks, fn, None, C.byref(res), _p(Q), _p(QN), _p(QU), _p(kr),
                  _p(kc), _p(x))
        if err:
            raise err[0]
        _check(r)
        return {"kappa_rta": np.array(res.kappa_rta).reshape(3, 3, order="F"),
                "kappa_cg": np.array(res.kappa_cg).reshape(3, 3, order="F"), "cg_iters": res.cg_iters,
                "status_cg": res.status_cg, "stage_ms": dict(zip(STAGES, list(res.stage_ms))),
                "launches": dict(zip(STAGES, list(res.launches))), "triplet_bands": res.triplet_bands,
                "d2h_bytes": res.d2h_bytes, "Q": Q, "QN": QN, "QU": QU, "kappa_rta_modes": kr,
                "kappa_cg_modes": kc, "x": x}


# int (*)(void* user, const double* mine, long long count, double* all, const long long* counts, int nranks)
ALLGATHER_FN = C.CFUNCTYPE(C.c_int, C.c_void_p, C.POINTER(C.c_double), C.c_longlong, C.POINTER(C.c_double),
                           C.POINTER(C.c_longlong), C.c_int)


# int (*)(void* user, const double* mine, long long count, double* all, const long long* counts, int nranks,
#        void* stream), device pointers
ALLGATHER_DEV_FN = C.CFUNCTYPE(C.c_int, C.c_void_p, C.c_void_p, C.c_longlong, C.c_void_p, C.POINTER(C.c_longlong),
                               C.c_int, C.c_void_p)


def shard_rows(nibz: int, rank: int, nranks: int) -> Tuple[int, int]:
    """The 1-based IBZ row range of a rank in the reference's MPI split
    (kappa.f90:418-428): nibz // nranks rows each, the last rank also takes
    the remainder (ald_shard_rows computes the same on the library side)."""
    local = nibz // nranks
    lo = rank * local + 1
    hi = nibz if rank == nranks - 1 else rank * local + local
    return lo, hi


def torch_allgather(group=None):
    """An all-gather for kappa_pipeline_sharded over torch.distributed: the
    ranks' arrays (different lengths allowed) padded to the longest, gathered
    with all_gather (on the current CUDA device for NCCL, on the CPU for
    gloo) and concatenated in rank order."""
    import torch
    import torch.distributed as dist

    def gather(mine: np.ndarray, counts: Sequence[int]) -> np.ndarray:
        dev = torch.device("cuda", torch.cuda.current_device()) if dist.get_backend(group) == "nccl" else "cpu"
        m = max(counts)
        buf = torch.zeros(m, dtype=torch.float64, device=dev)
        buf[:len(mine)] = torch.from_numpy(np.ascontiguousarray(mine)).to(dev)
        parts = [torch.empty_like(buf) for _ in counts]
        dist.all_gather(parts, buf, group=group)
        return np.concatenate([p[:c].cpu().numpy() for p, c in zip(parts, counts)])

    return gather


class _DeviceBuffer:
    """A raw device pointer of float64 values seen by torch through the CUDA
    array interface (no copy)."""

    def __init__(self, ptr: int, n: int):
        self.__cuda_array_interface__ = {"shape": (n,), "typestr": "<f8", "data": (ptr, False), "version": 2,
                                         "strides": None}


def torch_allgather_device(group=None):
    """A device all-gather for kappa_pipeline_sharded(device=True) over
    torch.distributed: the ranks' device values padded to the longest,
    gathered with all_gather on the context's stream and copied into the
    output in rank order -- on the GPU with NCCL; gloo (one GPU, tests) runs
    its collective on host copies inside this adapter."""
    import torch
    import torch.distributed as dist

    def gather(mine: int, count: int, out: int, counts: Sequence[int], stream: int) -> None:
        dev = torch.device("cuda", torch.cuda.current_device())
        m = max(counts)
        st = torch.cuda.ExternalStream(stream, device=dev) if stream else torch.cuda.current_stream(dev)
        with torch.cuda.stream(st):
            buf = torch.zeros(m, dtype=torch.float64, device=dev)
            if count > 0:
                buf[:count] = torch.as_tensor(_DeviceBuffer(mine, count), device=dev)
            if dist.get_backend(group) == "gloo":  # gloo collectives on host copies
                cpu = buf.cpu()
                parts = [torch.empty_like(cpu) for _ in counts]
                dist.all_gather(parts, cpu, group=group)
                parts = [p_.to(dev) for p_ in parts]
            else:
                parts = [torch.empty_like(buf) for _ in counts]
                dist.all_gather(parts, buf, group=group)
            dst = torch.as_tensor(_DeviceBuffer(out, sum(counts)), device=dev)
            off = 0
            for p_, c in zip(parts, counts):
                dst[off:off + c] = p_[:c]
                off += c

    return gather


def weight_tet(w, e: float, fp32: bool = False):
    """weight_tet (tetrahedron.f90:188) on the GPU: w(ntet, 4) corner
    energies of each tetrahedron -> c(ntet, 4) corner weights at energy e.
    fp32: the mixed pipeline's FP32 weights instead of the FP64 pipeline's."""
    W = np.ascontiguousarray(w, dtype=float).reshape(-1, 4)
    c = np.zeros_like(W)
    _check(lib().ald_weight_tet(W.shape[0], _p(W), float(e), 1 if fp32 else 0, _p(c)))
    return c


def cg_quadratic(a, b, vmin, max_iter=100, n_dig_accur=2):
    """cg_quadratic (cg.f90:19) on the GPU; returns (vmin, funcmin, iters, status)."""
    A = np.asfortranarray(a, dtype=float)
    n = A.shape[0]
    x = np.array(vmin, dtype=float)
    fm = C.c_double(0)
    it = C.c_int(0)
    r = _check(lib().ald_cg_quadratic(n, _p(A), _p(np.ascontiguousarray(b, dtype=float)), _p(x), C.byref(fm),
                                      max_iter, n_dig_accur, C.byref(it)), allow=(ALD_OK, ALD_WARN_CG_MAXITER))
    return x, fm.value, it.value, r


def cg_quadratic_static(n: int, a_ptr: int, b_ptr: int, x_ptr: int, max_iter=100, n_dig_accur=2, stream: int = 0):
    """cg_quadratic on caller-owned DEVICE buffers without any device
    allocation (ald_cg_quadratic_static).  a_ptr, b_ptr, x_ptr are device
    addresses of a(n,n) column-major, b(n) and the initial guess, which is
    overwritten by the solution; `stream` is a cudaStream_t handle (0 = the
    default stream).  Returns (funcmin, iters, status)."""
    fm = C.c_double(0)
    it = C.c_int(0)
    r = _check(lib().ald_cg_quadratic_static(n, C.c_void_p(a_ptr), C.c_void_p(b_ptr), C.c_void_p(x_ptr),
                                             C.byref(fm), max_iter, n_dig_accur, C.byref(it),
                                             C.c_void_p(stream) if stream else None),
               allow=(ALD_OK, ALD_WARN_CG_MAXITER))
    return fm.value, it.value, r
