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
        L.oracle_new_ext.restype = C.c_void_p
        L.oracle_new_ext.argtypes = L.oracle_new.argtypes
        L.oracle_free.argtypes = [C.c_void_p]
        L.oracle_rhs.argtypes = [C.c_void_p, dp, dp, C.c_int]
        L.oracle_lsrk.argtypes = [C.c_void_p, dp, C.c_double, C.c_int, C.c_int, C.c_int]
        L.oracle_lsrk_from.argtypes = [C.c_void_p, dp, C.c_double, C.c_double, C.c_int,
                                       C.c_int, C.c_int]
        L.oracle_set_source.argtypes = [C.c_void_p, dp, dp, C.c_double, C.c_double]
        L.oracle_set_boundary.argtypes = [C.c_void_p, C.POINTER(C.c_int), C.POINTER(C.c_int)]
        L.oracle_set_glued.argtypes = [C.c_void_p, C.c_int, i32p, C.POINTER(C.c_int)]
        L.oracle_set_glued_jumps.argtypes = [C.c_void_p, dp]
        L.oracle_face_trace.argtypes = [C.c_void_p, dp, C.c_int32, C.c_int, dp]
        L.oracle_point_jumps.argtypes = [C.c_void_p, C.c_int, dp, dp, dp, dp, dp, dp]
        L.oracle_lsrk_coeffs.argtypes = [C.c_int, dp, dp, dp]
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

    def __init__(self, dim, N, ecoord, nbase, L, rho, lam, mu, flux=0, fine=None):
        """ecoord[e] = (x, y, z, size) of element e in finest-level cells;
        the brick has nbase base cells per axis, each halved once (fine=None),
        or `fine` finest cells per axis (multi-level forests)."""
        self.ecoord = np.ascontiguousarray(ecoord, dtype=np.int32).reshape(-1)
        K = self.ecoord.size // 4
        cells = [2 * int(x) for x in nbase] if fine is None else [int(x) for x in fine]
        nb = (C.c_int * 3)(*(cells + [1] * (3 - len(cells))))
        LL = np.array(list(L) + [1.0] * (3 - len(L)), dtype=np.float64)
        self._arrs = [np.ascontiguousarray(np.broadcast_to(a, (K,)), dtype=np.float64)
                      for a in (rho, lam, mu)]
        self.K, self.dim, self.N = K, dim, N
        h = lib().oracle_new_ext(dim, N, K, self.ecoord.ctypes.data_as(i32p), nb, _dp(LL),
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

    # faces glued to a subdomain of another order (see PGlueOracle)
    def set_glued(self, elem, face) -> None:
        e = np.ascontiguousarray(elem, dtype=np.int32)
        f = (C.c_int * len(e))(*[int(x) for x in face])
        if lib().oracle_set_glued(self._h, len(e), e.ctypes.data_as(i32p), f):
            raise ValueError("bad glued face")
        self._nglued = len(e)

    def set_glued_jumps(self, J: np.ndarray) -> None:
        J = np.ascontiguousarray(J, dtype=np.float64)
        assert J.size == self._nglued * 6 * self.Nfp
        lib().oracle_set_glued_jumps(self._h, _dp(J))

    @property
    def Nfp(self) -> int:
        return (self.N + 1) ** (self.dim - 1)

    @property
    def nfields(self) -> int:
        return 9 if self.dim == 3 else 5

    def face_trace(self, q: np.ndarray, e: int, f: int) -> np.ndarray:
        q = np.ascontiguousarray(q, dtype=np.float64)
        out = np.empty((self.nfields, self.Nfp))
        lib().oracle_face_trace(self._h, _dp(q), e, f, _dp(out))
        return out

    def point_jumps(self, qm, qp, nrm, matm, matp) -> np.ndarray:
        """(T* - T-, v* - v-) at points qm, qp [n][nfields] -> [n][6]"""
        qm = np.ascontiguousarray(qm, dtype=np.float64)
        qp = np.ascontiguousarray(qp, dtype=np.float64)
        out = np.empty((len(qm), 6))
        lib().oracle_point_jumps(self._h, len(qm), _dp(qm), _dp(qp),
                                 _dp(np.asarray(nrm, dtype=np.float64)),
                                 _dp(np.asarray(matm, dtype=np.float64)),
                                 _dp(np.asarray(matp, dtype=np.float64)), _dp(out))
        return out

    def material(self, e: int):
        return [float(a[e]) for a in self._arrs]


def lsrk_coeffs(method: int = 0):
    A, B, Cc = np.zeros(6), np.zeros(6), np.zeros(7)
    ns = lib().oracle_lsrk_coeffs(method, _dp(A), _dp(B), _dp(Cc))
    if ns < 0:
        raise ValueError("unsupported LSRK method for the oracle")
    return A[:ns], B[:ns], Cc[:ns + 1]


def _lgl_np(N: int):
    r, w, _ = lgl(N)
    return r, w


def glue_ops(N: int, Ng: int):
    """The oracle's own operators between order N and the glue order Ng >= N:
    I (Ng+1 x N+1) Lagrange interpolation at the glue's LGL nodes, and the L2
    projection P = M_N^{-1} I^T M_g (N+1 x Ng+1) with exact mass matrices
    (Gauss-Legendre quadrature of N + Ng + 2 points), the glue_m operators
    of src/bfam.c:5471-5514 restated."""
    r, _ = _lgl_np(N)
    rg, _ = _lgl_np(Ng)

    def lagrange(x, nodes):
        L = np.ones((len(x), len(nodes)))
        for j, xj in enumerate(nodes):
            for m, xm in enumerate(nodes):
                if m != j:
                    L[:, j] *= (x - xm) / (xj - xm)
        return L

    I = lagrange(rg, r)
    xq, wq = np.polynomial.legendre.leggauss(N + Ng + 2)
    Ln, Lg = lagrange(xq, r), lagrange(xq, rg)
    Mn = Ln.T @ (wq[:, None] * Ln)
    Mgn = Ln.T @ (wq[:, None] * Lg)  # int l_N l_g = I^T M_g exactly
    P = np.linalg.solve(Mn, Mgn)
    return I, P


class PGlueOracle:
    """Two oracles (subdomains of orders Na, Nb) joined at glued face pairs
    (ea, fa) <-> (eb, fb), opposite faces of one axis with the same extent:
    bfam's glue grid between two volume subdomains (src/bfam.c:7340-7414).
    Each stage both traces are interpolated to the order-Ng glue grid, the
    upwind jumps of each side are formed there with its own outward normal
    and material, projected back to its order and lifted by its element."""

    def __init__(self, oa: Oracle, ob: Oracle, pairs, Ng: int | None = None):
        self.o = (oa, ob)
        self.pairs = [tuple(int(x) for x in p) for p in pairs]
        self.Ng = Ng or max(oa.N, ob.N)
        self.ops = (glue_ops(oa.N, self.Ng), glue_ops(ob.N, self.Ng))
        oa.set_glued([p[0] for p in self.pairs], [p[1] for p in self.pairs])
        ob.set_glued([p[2] for p in self.pairs], [p[3] for p in self.pairs])
        self.dim = oa.dim

    def _to_glue(self, tr, I):
        n = I.shape[1]
        if self.dim == 2:
            return tr @ I.T
        t = tr.reshape(tr.shape[0], n, n)  # [c][b][a]
        return np.einsum("jb,ia,cba->cji", I, I, t).reshape(tr.shape[0], -1)

    def _from_glue(self, J, P):
        m = P.shape[1]
        if self.dim == 2:
            return J @ P.T
        t = J.reshape(J.shape[0], m, m)
        return np.einsum("bj,ai,cji->cba", P, P, t).reshape(J.shape[0], -1)

    def rhs(self, qa, qb, nthreads: int = 0):
        oa, ob = self.o
        (Ia, Pa), (Ib, Pb) = self.ops
        Ja, Jb = [], []
        for ea, fa, eb, fb in self.pairs:
            ga = self._to_glue(oa.face_trace(qa, ea, fa), Ia)
            gb = self._to_glue(ob.face_trace(qb, eb, fb), Ib)
            nrm = np.zeros(3)
            nrm[fa // 2] = 1.0 if fa % 2 else -1.0
            ma, mb = oa.material(ea), ob.material(eb)
            ja = oa.point_jumps(ga.T, gb.T, nrm, ma, mb).T  # [6][glue nodes]
            jb = ob.point_jumps(gb.T, ga.T, -nrm, mb, ma).T
            Ja.append(self._from_glue(ja, Pa))
            Jb.append(self._from_glue(jb, Pb))
        oa.set_glued_jumps(np.array(Ja))
        ob.set_glued_jumps(np.array(Jb))
        return oa.rhs(qa, nthreads), ob.rhs(qb, nthreads)

    def lsrk(self, qa, qb, dt: float, nsteps: int, nthreads: int = 0):
        A, B, _ = lsrk_coeffs(0)
        qa = np.array(qa, dtype=np.float64, copy=True)
        qb = np.array(qb, dtype=np.float64, copy=True)
        da, db = np.zeros_like(qa), np.zeros_like(qb)
        for _ in range(nsteps):
            for s in range(len(A)):
                ra, rb = self.rhs(qa, qb, nthreads)
                da = A[s] * da + dt * ra
                db = A[s] * db + dt * rb
                qa = qa + B[s] * da
                qb = qb + B[s] * db
        return qa, qb


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
