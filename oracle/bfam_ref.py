"""ORACLE -- test infrastructure only.

ctypes wrapper of oracle/_ref/libbfam_ref{2,3}d.so: the reference's own mesh
front end (src/bfam.c compiled from source with its vendored p4est-1.1, see
oracle/build_ref.sh) run on a seeded, adapted brick, and the arrays bfam holds
after bfam_domain_pxest_split_dgx_subdomains (src/bfam.c:7565-8054).  Only
tests/ import this module; the product never does.
"""
from __future__ import annotations

import ctypes as C
from pathlib import Path

import numpy as np

HERE = Path(__file__).resolve().parent
REF = HERE / "_ref"

i32p = C.POINTER(C.c_int32)
i8p = C.POINTER(C.c_int8)
dp = C.POINTER(C.c_double)


class Spec(C.Structure):
    _fields_ = [("n", C.c_int * 3), ("periodic", C.c_int * 3), ("L", C.c_double * 3),
                ("N", C.c_int), ("seed", C.c_uint64), ("levels", C.c_int),
                ("prob", C.c_double)]


class _Mesh(C.Structure):
    _fields_ = [("dim", C.c_int), ("N", C.c_int), ("Nq", C.c_int), ("Np", C.c_int),
                ("Nfp", C.c_int), ("NF", C.c_int), ("K", C.c_int32),
                ("r", dp), ("w", dp), ("Dr", dp), ("vmapM", i32p), ("vmapP", i32p),
                ("quads", i32p), ("x0", dp), ("h", dp), ("max_level", C.c_int),
                ("root_len", C.c_int32), ("num_trees", C.c_int32),
                ("tree_x0", dp), ("tree_h", dp),
                ("Kg", C.c_int32), ("EToEm", i32p), ("EToEp", i32p),
                ("EToFm", i8p), ("EToHm", i8p), ("EToHp", i8p), ("EToOp", i8p),
                ("interp", dp * 3), ("proj", dp * 3),
                ("Kb", C.c_int32), ("EToEb", i32p), ("EToFb", i8p),
                ("num_local_glue", C.c_int), ("num_boundary_glue", C.c_int)]


_libs: dict[int, C.CDLL] = {}


def lib_path(dim: int) -> Path:
    return REF / f"libbfam_ref{dim}d.so"


def available(dim: int = 3) -> bool:
    return lib_path(dim).exists()


def lib(dim: int) -> C.CDLL:
    if dim not in _libs:
        L = C.CDLL(str(lib_path(dim)), mode=C.RTLD_LOCAL)
        L.bfref_domain_new.restype = C.c_void_p
        L.bfref_domain_new.argtypes = [C.POINTER(Spec)]
        L.bfref_domain_free.argtypes = [C.c_void_p]
        L.bfref_mesh_new.argtypes = [C.c_void_p, C.POINTER(C.POINTER(_Mesh))]
        L.bfref_mesh_free.argtypes = [C.POINTER(_Mesh)]
        assert L.bfref_dim() == dim
        _libs[dim] = L
    return _libs[dim]


def make_spec(dim, n, N, seed=0, levels=1, prob=0.3, periodic=(1, 1, 1),
              L=(1.0, 1.0, 1.0)) -> Spec:
    s = Spec()
    nn = list(n) + [1] * (3 - len(n))
    for a in range(3):
        s.n[a] = int(nn[a])
        s.periodic[a] = int(bool(periodic[a])) if a < dim else 1
        s.L[a] = float(L[a]) if a < len(L) else 1.0
    s.N, s.seed, s.levels, s.prob = int(N), int(seed), int(levels), float(prob)
    return s


def _arr(ptr, n, dtype):
    if not ptr or n == 0:
        return np.zeros(0, dtype=dtype)
    return np.ctypeslib.as_array(ptr, shape=(n,)).astype(dtype, copy=True)


class BfamMesh:
    """The arrays of bfam's split of a seeded adapted brick (one volume
    subdomain of order N, its local glue grid and its boundary glue grids),
    and each element's p4est quadrant and box."""

    def __init__(self, dim, n, N, seed=0, levels=1, prob=0.3, periodic=(1, 1, 1),
                 L=(1.0, 1.0, 1.0)):
        Lb = lib(dim)
        spec = make_spec(dim, n, N, seed, levels, prob, periodic, L)
        d = Lb.bfref_domain_new(C.byref(spec))
        if not d:
            raise ValueError("bfref_domain_new rejected the spec")
        mp = C.POINTER(_Mesh)()
        try:
            rc = Lb.bfref_mesh_new(d, C.byref(mp))
            if rc:
                raise ValueError(f"bfref_mesh_new failed ({rc})")
            m = mp.contents
            self.dim, self.N, self.K = m.dim, m.N, m.K
            self.Nq, self.Np, self.Nfp, self.NF = m.Nq, m.Np, m.Nfp, m.NF
            nq = m.Nq
            self.r = _arr(m.r, nq, np.float64)
            self.w = _arr(m.w, nq, np.float64)
            self.Dr = _arr(m.Dr, nq * nq, np.float64)
            nmap = m.K * m.NF * m.Nfp
            self.vmapM = _arr(m.vmapM, nmap, np.int32)
            self.vmapP = _arr(m.vmapP, nmap, np.int32)
            self.quads = _arr(m.quads, 5 * m.K, np.int32).reshape(m.K, 5)
            self.x0 = _arr(m.x0, 3 * m.K, np.float64).reshape(m.K, 3)
            self.h = _arr(m.h, 3 * m.K, np.float64).reshape(m.K, 3)
            self.max_level, self.root_len = m.max_level, m.root_len
            self.tree_x0 = _arr(m.tree_x0, 3 * m.num_trees, np.float64).reshape(-1, 3)
            self.tree_h = _arr(m.tree_h, 3 * m.num_trees, np.float64).reshape(-1, 3)
            self.Kg = m.Kg
            self.EToEm = _arr(m.EToEm, m.Kg, np.int32)
            self.EToEp = _arr(m.EToEp, m.Kg, np.int32)
            self.EToFm = _arr(m.EToFm, m.Kg, np.int8)
            self.EToHm = _arr(m.EToHm, m.Kg, np.int8)
            self.EToHp = _arr(m.EToHp, m.Kg, np.int8)
            self.EToOp = _arr(m.EToOp, m.Kg, np.int8)
            self.interp = [_arr(m.interp[i], nq * nq, np.float64) if m.interp[i] else None
                           for i in range(3)]
            self.proj = [_arr(m.proj[i], nq * nq, np.float64) if m.proj[i] else None
                         for i in range(3)]
            self.Kb = m.Kb
            self.EToEb = _arr(m.EToEb, m.Kb, np.int32)
            self.EToFb = _arr(m.EToFb, m.Kb, np.int8)
            self.num_local_glue = m.num_local_glue
            self.num_boundary_glue = m.num_boundary_glue
        finally:
            if mp:
                Lb.bfref_mesh_free(mp)
            Lb.bfref_domain_free(d)
        self.nbase = tuple(int(x) for x in list(n)[:dim])
        self.periodic = tuple(bool(periodic[a]) for a in range(dim))
        self.L = tuple(float(L[a]) for a in range(dim))
        # element boxes in finest-level cells, for the oracle's owner map
        lv = self.max_level
        self.fine = tuple(self.nbase[a] << lv for a in range(dim))
        ec = np.zeros((self.K, 4), dtype=np.int32)
        shift = int(np.log2(self.root_len)) - lv
        tree_lo = np.rint(self.tree_x0[:, :dim] / self.tree_h[:, :dim]).astype(np.int64)
        for a in range(dim):
            ec[:, a] = ((tree_lo[self.quads[:, 0], a] << lv)
                        + (self.quads[:, 2 + a].astype(np.int64) >> shift))
        ec[:, 3] = 1 << (lv - self.quads[:, 1])
        self.ecoord = ec
        # element levels, for tests
        self.level = self.quads[:, 1].copy()

    @property
    def nfields(self) -> int:
        return 9 if self.dim == 3 else 5

    def quadrants(self):
        """(tree_x0, tree_h, quads, root_len) as bfam_gpu_quadrants_t takes
        them"""
        return (np.ascontiguousarray(self.tree_x0), np.ascontiguousarray(self.tree_h),
                np.ascontiguousarray(self.quads, dtype=np.int32), int(self.root_len))

    def node_coordinates(self, r=None):
        """node coordinates [3][K Np] (node i + Nq (j + Nq k), x fastest)"""
        r = self.r if r is None else np.asarray(r)
        Nq, dim = self.Nq, self.dim
        idx = np.arange(self.Np)
        ijk = [idx % Nq, (idx // Nq) % Nq, idx // (Nq * Nq)]
        out = []
        for a in range(3):
            if a < dim:
                x = self.x0[:, a:a + 1] + 0.5 * self.h[:, a:a + 1] * (r[ijk[a]][None, :] + 1)
            else:
                x = np.zeros((self.K, self.Np))
            out.append(x.reshape(-1))
        return out
