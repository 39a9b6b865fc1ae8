"""ORACLE -- test infrastructure only.

ctypes wrapper of oracle/liboracle.so (the FP64 CPU restatement in
dg_oracle.c) and of oracle/_ref/libbfam_ref_ops.so (the reference's own
setup numerics compiled from its source).  Only tests/, the smoke check and
bench.py's CPU-baseline leg import this module, as the checker or the timed
CPU baseline; the product never does.
"""
from __future__ import annotations

import ctypes as C
from pathlib import Path

import numpy as np

HERE = Path(__file__).resolve().parent
ORACLE_LIB = HERE / "liboracle.so"
REF_LIB = HERE / "_ref" / "libbfam_ref_ops.so"

dp = C.POINTER(C.c_double)
i32p = C.POINTER(C.c_int32)

_lib = None


def lib() -> C.CDLL:
    global _lib
    if _lib is None:
        if not ORACLE_LIB.exists():
            raise ImportError(f"{ORACLE_LIB} missing; run `python -m bfam_b200.build`")
        L = C.CDLL(str(ORACLE_LIB))
        L.oracle_new.restype = C.c_void_p
        L.oracle_new.argtypes = [C.c_int, C.c_int, C.c_int32, i32p, C.POINTER(C.c_int),
                                 dp, dp, dp, dp, C.c_int]
        L.oracle_free.argtypes = [C.c_void_p]
        L.oracle_rhs.argtypes = [C.c_void_p, dp, dp, C.c_int]
        L.oracle_lsrk.argtypes = [C.c_void_p, dp, C.c_double, C.c_int, C.c_int, C.c_int]
        L.oracle_lsrk_from.argtypes = [C.c_void_p, dp, C.c_double, C.c_double, C.c_int,
                                       C.c_int, C.c_int]
        L.oracle_set_source.argtypes = [C.c_void_p, dp, dp, C.c_double, C.c_double]
        L.oracle_set_boundary.argtypes = [C.c_void_p, C.POINTER(C.c_int), C.POINTER(C.c_int)]
        L.oracle_sample.argtypes = [C.c_void_p, dp, C.c_int, dp, dp]
        L.oracle_energy.restype = C.c_double
        L.oracle_energy.argtypes = [C.c_void_p, dp]
        L.oracle_lgl_nodes.argtypes = [C.c_int, dp, dp]
        L.oracle_diff_matrix.argtypes = [C.c_int, dp, dp]
        L.oracle_mortar_ops.argtypes = [C.c_int, dp, dp, dp, dp]
        L.oracle_max_threads.restype = C.c_int
        _lib = L
    return _lib


def _dp(a):
    return a.ctypes.data_as(dp)


def max_threads() -> int:
    return int(lib().oracle_max_threads())


def lgl(N: int):
    n = N + 1
    r, w, D = np.zeros(n), np.zeros(n), np.zeros(n * n)
    lib().oracle_lgl_nodes(N, _dp(r), _dp(w))
    lib().oracle_diff_matrix(N, _dp(r), _dp(D))
    return r, w, D


def mortar(N: int):
    """I_bottom, I_top, P_bottom, P_top (column-major flat)."""
    n = (N + 1) ** 2
    Ib, It, Pb, Pt = (np.zeros(n) for _ in range(4))
    lib().oracle_mortar_ops(N, _dp(Ib), _dp(It), _dp(Pb), _dp(Pt))
    return Ib, It, Pb, Pt


class Oracle:
    """FP64 CPU DG RHS / LSRK on a brick given by element boxes."""

    def __init__(self, dim, N, ecoord, nbase, L, rho, lam, mu, flux=0):
        self.ecoord = np.ascontiguousarray(ecoord, dtype=np.int32).reshape(-1)
        K = self.ecoord.size // 4
        nb = (C.c_int * 3)(*[int(x) for x in list(nbase) + [1] * (3 - len(nbase))])
        LL = np.array(list(L) + [1.0] * (3 - len(L)), dtype=np.float64)
        self._arrs = [np.ascontiguousarray(np.broadcast_to(a, (K,)), dtype=np.float64)
                      for a in (rho, lam, mu)]
        self.K, self.dim, self.N = K, dim, N
        h = lib().oracle_new(dim, N, K, self.ecoord.ctypes.data_as(i32p), nb, _dp(LL),
                             *[_dp(a) for a in self._arrs], flux)
        if not h:
            raise ValueError("oracle_new rejected the mesh")
        self._h = h

    @classmethod
    def from_mesh(cls, mesh, rho, lam, mu, flux=0, bc=0):
        """bc: condition on the sides of a mesh's non-periodic axes, one value
        for all or one per side (-x, +x, -y, +y[, -z, +z]); 0 free surface,
        1 absorbing"""
        o = cls(mesh.dim, mesh.N, mesh.ecoord, mesh.nbase, mesh.L, rho, lam, mu, flux)
        periodic = getattr(mesh, "periodic", (True, True, True))
        if not all(periodic):
            o.set_boundary(periodic, bc)
        return o

    def set_boundary(self, periodic, bc) -> None:
        sides = np.broadcast_to(np.asarray(bc, dtype=np.int64), (2 * self.dim,))
        pv = (C.c_int * 3)(*[int(bool(periodic[a])) if a < self.dim else 1
                             for a in range(3)])
        bv = (C.c_int * 6)(*([int(x) for x in sides] + [0] * (6 - len(sides))))
        lib().oracle_set_boundary(self._h, pv, bv)

    def __del__(self):
        if getattr(self, "_h", None):
            try:
                lib().oracle_free(self._h)
            except (TypeError, AttributeError):  # interpreter shutdown
                pass
            self._h = None

    def rhs(self, q: np.ndarray, nthreads: int = 0) -> np.ndarray:
        q = np.ascontiguousarray(q, dtype=np.float64)
        out = np.empty_like(q)
        lib().oracle_rhs(self._h, _dp(q), _dp(out), nthreads)
        return out

    def lsrk(self, q: np.ndarray, dt: float, nsteps: int, nthreads: int = 0,
             method: int = 0) -> np.ndarray:
        q = np.array(q, dtype=np.float64, order="C", copy=True)
        rc = lib().oracle_lsrk(self._h, _dp(q), dt, nsteps, method, nthreads)
        if rc:
            raise ValueError("unsupported LSRK method for the oracle")
        return q

    def lsrk_from(self, q: np.ndarray, t: float, dt: float, nsteps: int,
                  nthreads: int = 0, method: int = 0) -> np.ndarray:
        """nsteps from time t (the point source is time dependent)"""
        q = np.array(q, dtype=np.float64, order="C", copy=True)
        rc = lib().oracle_lsrk_from(self._h, _dp(q), t, dt, nsteps, method, nthreads)
        if rc:
            raise ValueError("unsupported LSRK method for the oracle")
        return q

    def set_source(self, x, force, f0: float, t0: float) -> None:
        xv = np.zeros(3)
        fv = np.zeros(3)
        xv[:len(x)] = x
        fv[:len(force)] = force
        if lib().oracle_set_source(self._h, _dp(xv), _dp(fv), f0, t0):
            raise ValueError("source point outside the brick")

    def sample(self, q: np.ndarray, x: np.ndarray) -> np.ndarray:
        """fields at points x [nrecv][3] -> [nrecv][nfields]"""
        q = np.ascontiguousarray(q, dtype=np.float64)
        x = np.ascontiguousarray(np.asarray(x, dtype=np.float64).reshape(-1, 3))
        out = np.empty((len(x), q.shape[0]))
        if lib().oracle_sample(self._h, _dp(q), len(x), _dp(x), _dp(out)):
            raise ValueError("receiver outside the brick")
        return out

    def seismograms(self, q: np.ndarray, t: float, dt: float, nsteps: int,
                    x: np.ndarray, nthreads: int = 0):
        """step nsteps from time t, sampling x after every step: returns the
        final state and samples [nsteps][nrecv][nfields]"""
        out = []
        for _ in range(nsteps):
            q = self.lsrk_from(q, t, dt, 1, nthreads)
            t += dt
            out.append(self.sample(q, x))
        return q, np.array(out)

    def energy(self, q: np.ndarray) -> float:
        q = np.ascontiguousarray(q, dtype=np.float64)
        return float(lib().oracle_energy(self._h, _dp(q)))


# --------------------------------------------------- reference-compiled ops

def ref_available() -> bool:
    return REF_LIB.exists()


_ref = None


def ref_lib() -> C.CDLL:
    global _ref
    if _ref is None:
        L = C.CDLL(str(REF_LIB))
        L.bfam_ref_lgl.argtypes = [C.c_int, dp, dp, dp, dp, dp]
        L.bfam_ref_mass.argtypes = [C.c_int, dp]
        L.bfam_ref_interpolator.argtypes = [C.c_int, C.c_int, dp, dp, dp]
        L.bfam_ref_pcg32.argtypes = [C.c_uint64, C.c_uint64, C.c_int, C.POINTER(C.c_uint32)]
        L.bfam_ref_pcg32_bounded.argtypes = [C.c_uint64, C.c_uint64, C.c_uint32, C.c_int,
                                             C.POINTER(C.c_uint32)]
        _ref = L
    return _ref


def ref_lgl(N: int):
    n = N + 1
    r, w, wi, D, V = np.zeros(n), np.zeros(n), np.zeros(n), np.zeros(n * n), np.zeros(n * n)
    ref_lib().bfam_ref_lgl(N, _dp(r), _dp(w), _dp(wi), _dp(D), _dp(V))
    return r, w, wi, D


def ref_interpolator(N_src: int, N_dst: int):
    n = (N_src + 1) * (N_dst + 1)
    prj, mp, wmp = np.zeros(5 * n), np.zeros(5 * n), np.zeros(5 * n)
    ref_lib().bfam_ref_interpolator(N_src, N_dst, _dp(prj), _dp(mp), _dp(wmp))
    return prj.reshape(5, n), mp.reshape(5, n), wmp.reshape(5, n)


def ref_pcg32(seed: int, seq: int, n: int) -> np.ndarray:
    out = (C.c_uint32 * n)()
    ref_lib().bfam_ref_pcg32(seed, seq, n, out)
    return np.array(out, dtype=np.uint64)
