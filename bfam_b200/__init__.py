"""bfam_b200: B200 device layer for bfam's DG elastic right-hand side and LSRK
step, with a host front end that produces bfam's volume/glue data model.

Python here is a thin mirror over the C-ABI in ``include/bfam_gpu.h`` and
``include/bfam_b200_host.h`` (ctypes, no torch).  The compute path is the
CUDA library ``libbfam_b200.so``; if it is missing, importing this module
raises -- there is no fallback.
"""
from __future__ import annotations

import ctypes as C
from pathlib import Path

import numpy as np

_HERE = Path(__file__).resolve().parent
LIB_PATH = _HERE / "libbfam_b200.so"

FIELDS_2D = ("vx", "vy", "sxx", "syy", "sxy")
FIELDS_3D = ("vx", "vy", "vz", "sxx", "syy", "szz", "sxy", "sxz", "syz")

FLUX_UPWIND, FLUX_CENTRAL = 0, 1
BC_FREE_SURFACE, BC_ABSORBING, BC_GLUED = 0, 1, 2
NQUAD = 5  # tree, level, x, y, z per element (BFAM_GPU_NQUAD)
# status codes of the C-ABI
(BFAM_GPU_EINVAL, BFAM_GPU_ENOMEM, BFAM_GPU_ECUDA, BFAM_GPU_ETIMEOUT,
 BFAM_GPU_EUNSUPPORTED) = (-1, -2, -3, -4, -5)
PRECISION_FP64, PRECISION_FP32 = 0, 1
LSRK_KC54, LSRK_FE, LSRK_HEUN, LSRK_W33 = 0, 1, 2, 3


class BfamGpuError(RuntimeError):
    """Raised when a bfam_gpu_* call returns a nonzero status."""

    def __init__(self, code: int, msg: str):
        super().__init__(f"bfam_gpu error {code}: {msg}")
        self.code = code


_lib = None


def lib() -> C.CDLL:
    global _lib
    if _lib is None:
        if not LIB_PATH.exists():
            raise ImportError(
                f"{LIB_PATH} is missing: build it with `python -m bfam_b200.build` "
                "(the CUDA library is required; there is no CPU fallback)")
        _lib = C.CDLL(str(LIB_PATH))
        _declare(_lib)
    return _lib


P = C.POINTER
i8p, i32p, dp = P(C.c_int8), P(C.c_int32), P(C.c_double)


class BrickSpec(C.Structure):
    _fields_ = [("dim", C.c_int), ("N", C.c_int), ("n", C.c_int * 3),
                ("L", C.c_double * 3), ("periodic", C.c_int * 3),
                ("refine_prob", C.c_double), ("seed", C.c_uint64),
                ("refine_flags", P(C.c_uint8))]


class MeshStruct(C.Structure):
    _fields_ = [("dim", C.c_int), ("N", C.c_int), ("Nq", C.c_int), ("Np", C.c_int),
                ("Nfp", C.c_int), ("Nfaces", C.c_int), ("K", C.c_int32),
                ("ecoord", i32p), ("x0", dp), ("h", dp),
                ("EToE", i32p), ("EToF", i8p), ("vmapM", i32p), ("vmapP", i32p),
                ("Kg", C.c_int32), ("EToEm", i32p), ("EToFm", i8p), ("EToHm", i8p),
                ("EToEp", i32p), ("EToHp", i8p), ("EToOp", i8p),
                ("num_refined", C.c_int32),
                ("Kb", C.c_int32), ("EToEb", i32p), ("EToFb", i8p)]


class VolumeDesc(C.Structure):
    _fields_ = [("dim", C.c_int), ("N", C.c_int), ("K", C.c_int32),
                ("r", dp), ("w", dp), ("Dr", dp), ("vmapM", i32p), ("vmapP", i32p),
                ("x0", dp), ("h", dp), ("rho", dp), ("lambda_", dp), ("mu", dp)]


class GlueDesc(C.Structure):
    _fields_ = [("K", C.c_int32), ("EToEp", i32p), ("EToHp", i8p), ("EToOp", i8p),
                ("EToEm", i32p), ("EToFm", i8p), ("EToHm", i8p),
                ("interpolation", dp * 3), ("projection", dp * 3)]


class BoundaryDesc(C.Structure):
    _fields_ = [("K", C.c_int32), ("EToE", i32p), ("EToF", i8p), ("type", i8p)]


class QuadrantsDesc(C.Structure):
    _fields_ = [("num_trees", C.c_int32), ("tree_x0", dp), ("tree_h", dp),
                ("quads", i32p), ("root_len", C.c_int32)]


class PGlueDesc(C.Structure):
    _fields_ = [("K", C.c_int32), ("bm", i32p), ("bp", i32p), ("N_g", C.c_int),
                ("I_m2g", dp), ("P_g2m", dp), ("I_p2g", dp), ("P_g2p", dp)]


class SourceDesc(C.Structure):
    _fields_ = [("x", C.c_double * 3), ("force", C.c_double * 3),
                ("f0", C.c_double), ("t0", C.c_double)]


class KernelStat(C.Structure):
    _fields_ = [("level", C.c_int), ("launches", C.c_int64), ("elements", C.c_int64),
                ("ms", C.c_double), ("alg_bytes", C.c_double), ("gbs", C.c_double)]


class Options(C.Structure):
    _fields_ = [("flux", C.c_int), ("precision", C.c_int),
                ("mem_budget_bytes", C.c_size_t), ("device", C.c_int)]


def _declare(L: C.CDLL) -> None:
    vp = C.c_void_p
    sig = {
        "bfam_b200_brick_mesh_new": (C.c_int, [P(BrickSpec), P(P(MeshStruct))]),
        "bfam_b200_brick_mesh_free": (None, [P(MeshStruct)]),
        "bfam_b200_lgl_operators": (C.c_int, [C.c_int, dp, dp, dp, dp]),
        "bfam_b200_mortar_operators": (C.c_int, [C.c_int, C.c_int, dp]),
        "bfam_b200_lsrk_coefficients": (C.c_int, [C.c_int, dp, dp, dp]),
        "bfam_b200_material_random": (None, [C.c_int32, C.c_uint64, C.c_double, C.c_double,
                                              C.c_double, C.c_double, C.c_double,
                                              C.c_double, dp, dp, dp]),
        "bfam_b200_node_coordinates": (None, [P(MeshStruct), dp, dp, dp, dp]),
        "bfam_b200_init_plane_wave": (None, [P(MeshStruct), dp, dp, C.c_double, C.c_double,
                                              C.c_double, C.c_double, C.c_double, P(dp)]),
        "bfam_b200_init_gaussian_pulse": (None, [P(MeshStruct), dp, dp, C.c_double, P(dp)]),
        "bfam_b200_pcg32_seed": (None, [vp, C.c_uint64, C.c_uint64]),
        "bfam_b200_pcg32_next": (C.c_uint32, [vp]),
        "bfam_b200_pcg32_bounded": (C.c_uint32, [vp, C.c_uint32]),
        "bfam_b200_pcg32_uniform": (C.c_double, [vp]),
        "bfam_gpu_domain_create": (C.c_int, [P(VolumeDesc), P(GlueDesc), P(Options), P(vp)]),
        "bfam_gpu_domain_create_with_boundary": (C.c_int, [P(VolumeDesc), P(GlueDesc),
                                                           P(BoundaryDesc), P(Options),
                                                           P(vp)]),
        "bfam_gpu_domain_create_from_quadrants": (C.c_int, [P(VolumeDesc), P(GlueDesc),
                                                            P(BoundaryDesc), P(QuadrantsDesc),
                                                            P(Options), P(vp)]),
        "bfam_gpu_domain_get_geometry": (C.c_int, [vp, dp, dp]),
        "bfam_gpu_domain_free": (C.c_int, [vp]),
        "bfam_gpu_domain_num_fields": (C.c_int, [vp]),
        "bfam_gpu_domain_field_length": (C.c_size_t, [vp]),
        "bfam_gpu_domain_device_bytes": (C.c_size_t, [vp]),
        "bfam_gpu_domain_set_fields": (C.c_int, [vp, P(dp)]),
        "bfam_gpu_domain_get_fields": (C.c_int, [vp, P(dp)]),
        "bfam_gpu_domain_rhs": (C.c_int, [vp, P(dp)]),
        "bfam_gpu_domain_energy": (C.c_int, [vp, dp]),
        "bfam_gpu_domain_energy_noalloc": (C.c_int, [vp, dp]),
        "bfam_gpu_domain_field_device_ptr": (vp, [vp, C.c_int]),
        "bfam_gpu_domain_set_stream": (C.c_int, [vp, vp]),
        "bfam_gpu_domain_sync": (C.c_int, [vp]),
        "bfam_ts_lsrk_init": (C.c_int, [P(vp), vp, C.c_int, C.c_double]),
        "bfam_ts_lsrk_step": (C.c_int, [vp, C.c_double, C.c_int, C.c_int]),
        "bfam_ts_lsrk_time": (C.c_int, [vp, dp]),
        "bfam_ts_lsrk_free": (C.c_int, [vp]),
        "bfam_gpu_domain_set_source": (C.c_int, [vp, P(SourceDesc)]),
        "bfam_gpu_domain_set_receivers": (C.c_int, [vp, C.c_int, dp, C.c_int]),
        "bfam_gpu_domain_get_seismograms": (C.c_int, [vp, dp, P(C.c_int)]),
        "bfam_gpu_batch_create": (C.c_int, [P(vp), C.c_int, C.c_int, dp, P(vp)]),
        "bfam_gpu_batch_set_stream": (C.c_int, [vp, vp]),
        "bfam_gpu_batch_step": (C.c_int, [vp, dp, C.c_int, C.c_int]),
        "bfam_gpu_batch_time": (C.c_int, [vp, C.c_int, dp]),
        "bfam_gpu_batch_sync": (C.c_int, [vp]),
        "bfam_gpu_batch_free": (C.c_int, [vp]),
        "bfam_gpu_pglue_create": (C.c_int, [vp, vp, P(PGlueDesc), P(vp)]),
        "bfam_gpu_pglue_free": (C.c_int, [vp]),
        "bfam_gpu_batch_add_pglue": (C.c_int, [vp, vp]),
        "bfam_gpu_batch_launches_per_step": (C.c_int, [vp]),
        "bfam_gpu_domain_launch_levels": (C.c_int, [vp]),
        "bfam_gpu_batch_num_groups": (C.c_int, [vp]),
        "bfam_gpu_batch_group_info": (C.c_int, [vp, C.c_int, P(C.c_int), P(C.c_int),
                                                P(C.c_int), P(C.c_int64)]),
        "bfam_gpu_tile_count": (C.c_int, [C.c_int, C.c_int]),
        "bfam_gpu_tile_elements": (C.c_int, [C.c_int, C.c_int, C.c_int]),
        "bfam_gpu_tile_shape": (C.c_int, [C.c_int, C.c_int, C.c_int, P(C.c_int),
                                          P(C.c_int)]),
        "bfam_gpu_batch_set_tile": (C.c_int, [vp, C.c_int, C.c_int, C.c_int]),
        "bfam_gpu_launch_count": (C.c_uint64, []),
        "bfam_gpu_last_error": (C.c_int, [C.c_char_p, C.c_size_t]),
        "bfam_gpu_record_error": (C.c_int, [C.c_int, C.c_char_p]),
        "bfam_gpu_trim_pool": (C.c_int, [C.c_int, C.c_size_t]),
        "bfam_gpu_domain_profile": (C.c_int, [vp, C.c_int]),
        "bfam_gpu_domain_kernel_stats": (C.c_int, [vp, C.c_void_p, C.c_int,
                                                   P(C.c_int)]),
    }
    for name, (res, args) in sig.items():
        fn = getattr(L, name)
        fn.restype = res
        fn.argtypes = args


def last_error() -> str:
    buf = C.create_string_buffer(1024)
    lib().bfam_gpu_last_error(buf, 1024)
    return buf.value.decode()


def _check(rc: int) -> None:
    if rc != 0:
        raise BfamGpuError(rc, last_error())


def _dp(a: np.ndarray):
    return a.ctypes.data_as(dp)


def _ptrs(arrs) -> C.Array:
    return (dp * len(arrs))(*[_dp(a) for a in arrs])


def launch_count() -> int:
    return int(lib().bfam_gpu_launch_count())


# ----------------------------------------------------------------- operators

def lgl_operators(N: int):
    """r, w, wi, Dr (column-major flat) for order N."""
    n = N + 1
    r, w, wi, D = np.zeros(n), np.zeros(n), np.zeros(n), np.zeros(n * n)
    if lib().bfam_b200_lgl_operators(N, _dp(r), _dp(w), _dp(wi), _dp(D)):
        raise ValueError(f"bad order {N}")
    return r, w, wi, D


def mortar_operators(N_src: int, N_dst: int) -> np.ndarray:
    """(5, (N_dst+1)*(N_src+1)) column-major: same, cfb, cft, r2b, r2t."""
    n = (N_src + 1) * (N_dst + 1)
    out = np.zeros(5 * n)
    if lib().bfam_b200_mortar_operators(N_src, N_dst, _dp(out)):
        raise ValueError("bad orders")
    return out.reshape(5, n)


def lsrk_coefficients(method: int = LSRK_KC54):
    A, B, Cc = np.zeros(6), np.zeros(6), np.zeros(7)
    ns = lib().bfam_b200_lsrk_coefficients(method, _dp(A), _dp(B), _dp(Cc))
    if ns < 0:
        raise ValueError(f"unknown LSRK method {method}")
    return A[:ns].copy(), B[:ns].copy(), Cc[:ns + 1].copy()


class PCG32:
    """The PCG32 stream used for every seeded draw."""

    def __init__(self, seed: int, seq: int):
        self._st = (C.c_uint64 * 2)()
        lib().bfam_b200_pcg32_seed(C.cast(self._st, C.c_void_p), seed, seq)

    def next(self) -> int:
        return int(lib().bfam_b200_pcg32_next(C.cast(self._st, C.c_void_p)))

    def bounded(self, bound: int) -> int:
        return int(lib().bfam_b200_pcg32_bounded(C.cast(self._st, C.c_void_p), bound))

    def uniform(self) -> float:
        return float(lib().bfam_b200_pcg32_uniform(C.cast(self._st, C.c_void_p)))


# ---------------------------------------------------------------------- mesh

class Mesh:
    """Brick mesh in bfam's data model (see bfam_b200_brick_mesh_new)."""

    def __init__(self, dim: int, N: int, n, L=(1.0, 1.0, 1.0), refine_prob: float = 0.0,
                 seed: int = 0, refine_flags=None, periodic=(True, True, True)):
        spec = BrickSpec()
        spec.dim, spec.N = dim, N
        nn = list(n) + [1] * (3 - len(n))
        LL = list(L) + [1.0] * (3 - len(L))
        for a in range(3):
            spec.n[a] = int(nn[a])
            spec.L[a] = float(LL[a])
            spec.periodic[a] = 1 if (a >= dim or periodic[a]) else 0
        spec.refine_prob = float(refine_prob)
        spec.seed = int(seed)
        self._flags = None
        if refine_flags is not None:
            self._flags = np.ascontiguousarray(refine_flags, dtype=np.uint8)
            spec.refine_flags = self._flags.ctypes.data_as(P(C.c_uint8))
        ptr = P(MeshStruct)()
        rc = lib().bfam_b200_brick_mesh_new(C.byref(spec), C.byref(ptr))
        if rc:
            raise ValueError(f"bfam_b200_brick_mesh_new failed ({rc})")
        self._ptr = ptr
        m = ptr.contents
        self.dim, self.N, self.Nq, self.Np = m.dim, m.N, m.Nq, m.Np
        self.Nfp, self.Nfaces, self.K, self.Kg = m.Nfp, m.Nfaces, m.K, m.Kg
        self.nbase = tuple(nn[:3])
        self.periodic = tuple(bool(spec.periodic[a]) for a in range(3))
        self.L = tuple(LL[:3])
        self.num_refined = m.num_refined
        K, NF, Nfp, Kg = self.K, self.Nfaces, self.Nfp, self.Kg

        def arr(p, n, dt):
            return np.ctypeslib.as_array(p, shape=(n,)).astype(dt, copy=True) if n else np.zeros(0, dt)

        self.ecoord = arr(m.ecoord, 4 * K, np.int32).reshape(K, 4)
        self.x0 = arr(m.x0, 3 * K, np.float64).reshape(K, 3)
        self.h = arr(m.h, 3 * K, np.float64).reshape(K, 3)
        self.EToE = arr(m.EToE, NF * K, np.int32).reshape(K, NF)
        self.EToF = arr(m.EToF, NF * K, np.int8).reshape(K, NF)
        self.vmapM = arr(m.vmapM, K * NF * Nfp, np.int32)
        self.vmapP = arr(m.vmapP, K * NF * Nfp, np.int32)
        self.EToEm = arr(m.EToEm, Kg, np.int32)
        self.EToFm = arr(m.EToFm, Kg, np.int8)
        self.EToHm = arr(m.EToHm, Kg, np.int8)
        self.EToEp = arr(m.EToEp, Kg, np.int32)
        self.EToHp = arr(m.EToHp, Kg, np.int8)
        self.EToOp = arr(m.EToOp, Kg, np.int8)
        # boundary faces of non-periodic axes (element, face)
        self.Kb = m.Kb
        self.EToEb = arr(m.EToEb, m.Kb, np.int32)
        self.EToFb = arr(m.EToFb, m.Kb, np.int8)

    def __del__(self):
        try:
            if getattr(self, "_ptr", None):
                lib().bfam_b200_brick_mesh_free(self._ptr)
                self._ptr = None
        except Exception:
            pass

    @property
    def nfields(self) -> int:
        return 9 if self.dim == 3 else 5

    @property
    def ndof(self) -> int:
        return self.K * self.Np * self.nfields

    def node_coordinates(self, r):
        n = self.K * self.Np
        x, y, z = np.zeros(n), np.zeros(n), np.zeros(n)
        lib().bfam_b200_node_coordinates(self._ptr, _dp(np.ascontiguousarray(r)),
                                         _dp(x), _dp(y), _dp(z))
        return x, y, z

    def empty_fields(self) -> np.ndarray:
        return np.zeros((self.nfields, self.K * self.Np))

    def quadrants(self, root_len: int | None = None):
        """p4est's view of the mesh: one tree per base cell (numbered x
        fastest), tree boxes [T][3] (lower corner, edge lengths), and per
        element (tree, level, x, y, z) in integer coordinates of [0,
        root_len) (P4EST_ROOT_LEN: 2^30 in 2D, 2^19 in 3D)."""
        root = root_len or (1 << (19 if self.dim == 3 else 30))
        n = np.array(self.nbase[:3])
        unit = np.array(self.L[:3]) / n
        T = int(np.prod(n))
        t = np.arange(T)
        b = np.stack([t % n[0], (t // n[0]) % n[1], t // (n[0] * n[1])], axis=1)
        tree_x0 = np.ascontiguousarray(b * unit, dtype=np.float64)
        tree_h = np.ascontiguousarray(np.broadcast_to(unit, (T, 3)), dtype=np.float64)
        ec = self.ecoord.astype(np.int64)
        base = ec[:, :3] // 2
        tree = base[:, 0] + n[0] * (base[:, 1] + n[1] * base[:, 2])
        level = np.where(ec[:, 3] == 2, 0, 1)
        xyz = (ec[:, :3] - 2 * base) * (root // 2)
        if self.dim == 2:
            xyz[:, 2] = 0
        quads = np.ascontiguousarray(
            np.column_stack([tree, level, xyz]).astype(np.int32))
        return tree_x0, tree_h, quads, root

    def plane_wave(self, r, k, amplitude, rho, lam, mu, time=0.0) -> np.ndarray:
        q = self.empty_fields()
        kv = np.zeros(3)
        kv[:len(k)] = k
        lib().bfam_b200_init_plane_wave(self._ptr, _dp(np.ascontiguousarray(r)), _dp(kv),
                                        amplitude, rho, lam, mu, time, _ptrs(list(q)))
        return q

    def gaussian_pulse(self, r, center, width) -> np.ndarray:
        q = self.empty_fields()
        c = np.zeros(3)
        c[:len(center)] = center
        lib().bfam_b200_init_gaussian_pulse(self._ptr, _dp(np.ascontiguousarray(r)), _dp(c),
                                            width, _ptrs(list(q)))
        return q


def material_random(K: int, seed: int, rho=(1.0, 3.0), cp=(4.0, 6.0), ratio=(1.6, 2.0)):
    """rho ~ U[rho], cp ~ U[cp], cs = cp / U[ratio] per element -> rho, lambda, mu."""
    r, la, mu = np.zeros(K), np.zeros(K), np.zeros(K)
    lib().bfam_b200_material_random(K, seed, rho[0], rho[1], cp[0], cp[1], ratio[0],
                                    ratio[1], _dp(r), _dp(la), _dp(mu))
    return r, la, mu


# --------------------------------------------------------------- device layer

class GpuDomain:
    """A bfam_gpu_domain_t built from a Mesh's arrays (what an application
    would pass from its bfam_subdomain_dgx_t and glue grid)."""

    def __init__(self, mesh: Mesh, rho, lam, mu, flux: int = FLUX_UPWIND,
                 precision: int = PRECISION_FP64, mem_budget_bytes: int = 0,
                 device: int = 0, bc=BC_FREE_SURFACE, geometry: str = "host"):
        """bc: the condition on the boundary faces of a non-periodic mesh,
        one value for every side or one per side (-x, +x, -y, +y, -z, +z);
        geometry "host": element boxes uploaded (x0, h); "device": computed
        on the GPU from the mesh's quadrant data"""
        L = lib()
        self.mesh = mesh
        N = mesh.N
        self.r, self.w, self.wi, self.Dr = lgl_operators(N)
        ops = mortar_operators(N, N)
        self._keep = []
        # a mesh that carries its own operators (bfam's split: its
        # subdomain's r, w, Dr and its glue grid's interpolation/projection)
        # passes those instead
        own = getattr(mesh, "interp", None) is not None
        if own:
            self.r = np.ascontiguousarray(mesh.r, dtype=np.float64)
            self.w = np.ascontiguousarray(mesh.w, dtype=np.float64)
            self.Dr = np.ascontiguousarray(mesh.Dr, dtype=np.float64)
        self.rho = np.ascontiguousarray(np.broadcast_to(rho, (mesh.K,)), dtype=np.float64)
        self.lam = np.ascontiguousarray(np.broadcast_to(lam, (mesh.K,)), dtype=np.float64)
        self.mu = np.ascontiguousarray(np.broadcast_to(mu, (mesh.K,)), dtype=np.float64)
        vol = VolumeDesc()
        vol.dim, vol.N, vol.K = mesh.dim, N, mesh.K
        vol.r, vol.w, vol.Dr = _dp(self.r), _dp(self.w), _dp(self.Dr)
        vol.vmapM = mesh.vmapM.ctypes.data_as(i32p)
        vol.vmapP = mesh.vmapP.ctypes.data_as(i32p)
        x0 = np.ascontiguousarray(mesh.x0)
        hh = np.ascontiguousarray(mesh.h)
        self._keep += [x0, hh, ops]
        vol.x0, vol.h = _dp(x0), _dp(hh)
        vol.rho, vol.lambda_, vol.mu = _dp(self.rho), _dp(self.lam), _dp(self.mu)
        glue = GlueDesc()
        glue.K = mesh.Kg
        if mesh.Kg:
            glue.EToEp = mesh.EToEp.ctypes.data_as(i32p)
            glue.EToHp = mesh.EToHp.ctypes.data_as(i8p)
            glue.EToOp = mesh.EToOp.ctypes.data_as(i8p)
            glue.EToEm = mesh.EToEm.ctypes.data_as(i32p)
            glue.EToFm = mesh.EToFm.ctypes.data_as(i8p)
            glue.EToHm = mesh.EToHm.ctypes.data_as(i8p)
            # interpolation = {same, r2b, r2t}; projection = {same, cfb, cft}
            if own:
                for slot in range(3):
                    a, b = mesh.interp[slot], mesh.proj[slot]
                    glue.interpolation[slot] = _dp(a) if a is not None else dp()
                    glue.projection[slot] = _dp(b) if b is not None else dp()
            else:
                for slot, k in enumerate((0, 3, 4)):
                    glue.interpolation[slot] = _dp(ops[k]) if k else dp()
                for slot, k in enumerate((0, 1, 2)):
                    glue.projection[slot] = _dp(ops[k]) if k else dp()
        opt = Options()
        opt.flux, opt.precision = flux, precision
        opt.mem_budget_bytes, opt.device = mem_budget_bytes, device
        h = C.c_void_p()
        self.bc = None
        bnd = None
        if getattr(mesh, "Kb", 0):
            sides = np.broadcast_to(np.asarray(bc, dtype=np.int8), (2 * mesh.dim,))
            btype = np.ascontiguousarray(sides[mesh.EToFb], dtype=np.int8)
            self._keep += [btype]
            bnd = BoundaryDesc()
            bnd.K = mesh.Kb
            bnd.EToE = mesh.EToEb.ctypes.data_as(i32p)
            bnd.EToF = mesh.EToFb.ctypes.data_as(i8p)
            bnd.type = btype.ctypes.data_as(i8p)
            self.bc = tuple(int(x) for x in sides)
        if geometry == "device":
            tx0, th, quads, root = mesh.quadrants()
            self._keep += [tx0, th, quads]
            qd = QuadrantsDesc()
            qd.num_trees, qd.root_len = len(tx0), root
            qd.tree_x0, qd.tree_h = _dp(tx0), _dp(th)
            qd.quads = quads.ctypes.data_as(i32p)
            vol.x0, vol.h = dp(), dp()
            _check(L.bfam_gpu_domain_create_from_quadrants(
                C.byref(vol), C.byref(glue), C.byref(bnd) if bnd else None, C.byref(qd),
                C.byref(opt), C.byref(h)))
        elif geometry != "host":
            raise ValueError(f"geometry must be 'host' or 'device' (got {geometry!r})")
        elif bnd is not None:
            _check(L.bfam_gpu_domain_create_with_boundary(
                C.byref(vol), C.byref(glue), C.byref(bnd), C.byref(opt), C.byref(h)))
        else:
            _check(L.bfam_gpu_domain_create(C.byref(vol), C.byref(glue), C.byref(opt),
                                            C.byref(h)))
        self._h = h
        self.nfields = L.bfam_gpu_domain_num_fields(h)
        self.field_length = L.bfam_gpu_domain_field_length(h)

    @property
    def handle(self):
        return self._h

    def geometry(self):
        """element boxes the domain computes with: x0, h, [K][3] each"""
        K = self.mesh.K
        x0, h = np.zeros((K, 3)), np.zeros((K, 3))
        _check(lib().bfam_gpu_domain_get_geometry(self._h, _dp(x0), _dp(h)))
        return x0, h

    def free(self):
        if getattr(self, "_h", None) and self._h.value:
            lib().bfam_gpu_domain_free(self._h)
            self._h = C.c_void_p()

    def __del__(self):
        try:
            self.free()
        except Exception:
            pass

    def device_bytes(self) -> int:
        return int(lib().bfam_gpu_domain_device_bytes(self._h))

    def write_vtu(self, path, time: float | None = None, binary: bool = True):
        """download the fields and write them as a .vtu file (bfam_b200.vtk)"""
        from .vtk import write_vtu
        if self.mesh is None:
            raise ValueError("the domain no longer holds its mesh")
        return write_vtu(path, self.mesh, self.get_fields(), time=time, binary=binary)

    def launch_levels(self) -> int:
        """launches per LSRK stage (one per refinement level)"""
        return int(lib().bfam_gpu_domain_launch_levels(self._h))

    def set_fields(self, q: np.ndarray) -> None:
        q = np.ascontiguousarray(q, dtype=np.float64)
        assert q.shape == (self.nfields, self.field_length)
        _check(lib().bfam_gpu_domain_set_fields(self._h, _ptrs(list(q))))

    def get_fields(self, out: np.ndarray | None = None) -> np.ndarray:
        if out is None:
            out = np.empty((self.nfields, self.field_length))
        _check(lib().bfam_gpu_domain_get_fields(self._h, _ptrs(list(out))))
        return out

    def rhs(self) -> np.ndarray:
        out = np.empty((self.nfields, self.field_length))
        _check(lib().bfam_gpu_domain_rhs(self._h, _ptrs(list(out))))
        return out

    def energy(self) -> float:
        e = C.c_double()
        _check(lib().bfam_gpu_domain_energy(self._h, C.byref(e)))
        return e.value

    def energy_noalloc(self) -> float:
        """The energy through the entry point that allocates no device memory
        (fixed scratch compiled into the library; see bfam_gpu.h)."""
        e = C.c_double()
        _check(lib().bfam_gpu_domain_energy_noalloc(self._h, C.byref(e)))
        return e.value

    def sync(self) -> None:
        _check(lib().bfam_gpu_domain_sync(self._h))

    def field_device_ptr(self, f: int) -> int:
        return int(lib().bfam_gpu_domain_field_device_ptr(self._h, f) or 0)

    def set_stream(self, stream_ptr: int) -> None:
        _check(lib().bfam_gpu_domain_set_stream(self._h, C.c_void_p(stream_ptr)))

    def profile(self, enable: bool = True) -> None:
        """per-launch event timing of the stage kernels (steps run eagerly
        while it is on); enabling or disabling clears the totals"""
        _check(lib().bfam_gpu_domain_profile(self._h, int(bool(enable))))

    def kernel_stats(self) -> list[dict]:
        """per launch level: launches, elements, device ms, algorithmic
        bytes and GB/s since profiling was enabled"""
        buf = (KernelStat * 16)()
        n = C.c_int()
        _check(lib().bfam_gpu_domain_kernel_stats(self._h, C.cast(buf, C.c_void_p), 16,
                                                  C.byref(n)))
        return [{"level": s.level, "launches": int(s.launches), "elements": int(s.elements),
                 "ms": s.ms, "alg_bytes": s.alg_bytes, "gbs": s.gbs}
                for s in buf[:min(n.value, 16)]]

    def set_source(self, x, force, f0: float, t0: float) -> None:
        """Ricker point force f(t) F at x (bfam_gpu_domain_set_source)."""
        s = SourceDesc()
        for a in range(3):
            s.x[a] = x[a] if a < len(x) else 0.0
            s.force[a] = force[a] if a < len(force) else 0.0
        s.f0, s.t0 = f0, t0
        _check(lib().bfam_gpu_domain_set_source(self._h, C.byref(s)))

    def clear_source(self) -> None:
        _check(lib().bfam_gpu_domain_set_source(self._h, None))

    def set_receivers(self, x: np.ndarray, max_samples: int) -> None:
        x = np.ascontiguousarray(np.asarray(x, dtype=np.float64).reshape(-1, 3))
        self._nrecv = len(x)
        _check(lib().bfam_gpu_domain_set_receivers(self._h, len(x), _dp(x), max_samples))
        self._max_samples = max_samples

    def seismograms(self) -> np.ndarray:
        """samples [nsamples][nrecv][nfields]"""
        nr = getattr(self, "_nrecv", 0)
        out = np.empty((max(getattr(self, "_max_samples", 0), 1), max(nr, 1), self.nfields))
        n = C.c_int()
        _check(lib().bfam_gpu_domain_get_seismograms(self._h, _dp(out), C.byref(n)))
        return out[:n.value, :nr].copy()


def tile_shapes(dim: int, N: int) -> list[tuple[int, int]]:
    """(threads per element, resident CTAs per SM) of each compiled tile."""
    L = lib()
    out = []
    for t in range(L.bfam_gpu_tile_count(dim, N)):
        a, b = C.c_int(), C.c_int()
        _check(L.bfam_gpu_tile_shape(dim, N, t, C.byref(a), C.byref(b)))
        out.append((a.value, b.value))
    return out


def tile_elements(dim: int, N: int) -> list[int]:
    """elements per CTA of each compiled tile"""
    L = lib()
    out = []
    for t in range(L.bfam_gpu_tile_count(dim, N)):
        e = L.bfam_gpu_tile_elements(dim, N, t)
        _check(min(e, 0))
        out.append(int(e))
    return out


class Batch:
    """bfam_gpu_batch_t: domains stepped together, one persistent launch per
    order group and stage."""

    def __init__(self, domains, method: int = LSRK_KC54, t0=None):
        self.domains = list(domains)
        hs = (C.c_void_p * len(self.domains))(*[d.handle.value for d in self.domains])
        t = None if t0 is None else np.ascontiguousarray(
            np.broadcast_to(t0, (len(self.domains),)), dtype=np.float64)
        h = C.c_void_p()
        _check(lib().bfam_gpu_batch_create(hs, len(self.domains), method,
                                           _dp(t) if t is not None else None, C.byref(h)))
        self._h = h

    @property
    def handle(self):
        return self._h

    def step(self, dt, nsteps: int = 1, use_graph: bool = True) -> None:
        dts = np.ascontiguousarray(np.broadcast_to(dt, (len(self.domains),)),
                                   dtype=np.float64)
        _check(lib().bfam_gpu_batch_step(self._h, _dp(dts), nsteps, 1 if use_graph else 0))

    def add_pglue(self, g: "PGlue") -> None:
        """step the glue with the batch (bfam_gpu_batch_add_pglue)"""
        _check(lib().bfam_gpu_batch_add_pglue(self._h, g.handle))
        self._glues = getattr(self, "_glues", []) + [g]

    def time(self, i: int) -> float:
        t = C.c_double()
        _check(lib().bfam_gpu_batch_time(self._h, i, C.byref(t)))
        return t.value

    def set_stream(self, stream_ptr: int) -> None:
        _check(lib().bfam_gpu_batch_set_stream(self._h, C.c_void_p(stream_ptr)))

    def sync(self) -> None:
        _check(lib().bfam_gpu_batch_sync(self._h))

    def groups(self) -> list[dict]:
        L = lib()
        out = []
        for g in range(L.bfam_gpu_batch_num_groups(self._h)):
            d, n, p, k = C.c_int(), C.c_int(), C.c_int(), C.c_int64()
            _check(L.bfam_gpu_batch_group_info(self._h, g, C.byref(d), C.byref(n),
                                               C.byref(p), C.byref(k)))
            out.append({"dim": d.value, "N": n.value, "precision": p.value,
                        "elements": k.value})
        return out

    def launches_per_step(self) -> int:
        return int(lib().bfam_gpu_batch_launches_per_step(self._h))

    def set_tile(self, group: int, tile: int, ctas_per_sm: int = 0) -> None:
        _check(lib().bfam_gpu_batch_set_tile(self._h, group, tile, ctas_per_sm))

    def free(self):
        if getattr(self, "_h", None) and self._h.value:
            lib().bfam_gpu_batch_free(self._h)
            self._h = C.c_void_p()

    def __del__(self):
        try:
            self.free()
        except Exception:
            pass


class LSRK:
    """bfam_ts_lsrk_t over a GpuDomain."""

    def __init__(self, dom: GpuDomain, method: int = LSRK_KC54, t0: float = 0.0):
        self.dom = dom
        h = C.c_void_p()
        _check(lib().bfam_ts_lsrk_init(C.byref(h), dom.handle, method, t0))
        self._h = h

    def step(self, dt: float, nsteps: int = 1, use_graph: bool = False) -> None:
        _check(lib().bfam_ts_lsrk_step(self._h, dt, nsteps, 1 if use_graph else 0))

    @property
    def time(self) -> float:
        t = C.c_double()
        _check(lib().bfam_ts_lsrk_time(self._h, C.byref(t)))
        return t.value

    def free(self):
        if getattr(self, "_h", None) and self._h.value:
            lib().bfam_ts_lsrk_free(self._h)
            self._h = C.c_void_p()

    def __del__(self):
        try:
            self.free()
        except Exception:
            pass


# ------------------------------------------------ glue between two domains

def glued_x_pairs(ma: Mesh, mb: Mesh):
    """Boundary-list entries pairing two bricks that share their y/z extent
    and are glued along x into one periodic domain: a's +x side to b's -x
    side and b's +x side to a's -x side (elements meeting with the same
    box on the face).  Returns (entries of a, entries of b)."""
    def side(m, f):
        out = {}
        for k in np.flatnonzero(m.EToFb == f):
            e = int(m.EToEb[k])
            key = tuple(np.round(np.r_[m.x0[e, 1:m.dim], m.h[e, 1:m.dim]], 12))
            out[key] = int(k)
        return out

    am, ap, bm, bp = side(ma, 0), side(ma, 1), side(mb, 0), side(mb, 1)
    ea, eb = [], []
    for s, t in ((ap, bm), (am, bp)):
        if set(s) != set(t):
            raise ValueError("the glued sides do not match face by face")
        for key in sorted(s):
            ea.append(s[key])
            eb.append(t[key])
    return np.array(ea, dtype=np.int32), np.array(eb, dtype=np.int32)


class PGlue:
    """bfam_gpu_pglue_t: glue between domain dom_m (entries bm of its
    boundary list) and domain dom_p (entries bp), glue order Ng (default max of the two
    orders), with bfam's operators interpolation[0] / projection[0] of each
    side (mortar_operators(N, Ng)[0], mortar_operators(Ng, N)[0])."""

    def __init__(self, dom_m: GpuDomain, dom_p: GpuDomain, bm, bp, Ng: int | None = None):
        Nm, Np_ = dom_m.mesh.N, dom_p.mesh.N
        Ng = Ng or max(Nm, Np_)
        self._bm = np.ascontiguousarray(bm, dtype=np.int32)
        self._bp = np.ascontiguousarray(bp, dtype=np.int32)
        desc = PGlueDesc()
        desc.K = len(self._bm)
        desc.bm = self._bm.ctypes.data_as(i32p)
        desc.bp = self._bp.ctypes.data_as(i32p)
        desc.N_g = Ng
        self._ops = []
        for name_i, name_p, N in (("I_m2g", "P_g2m", Nm), ("I_p2g", "P_g2p", Np_)):
            if N == Ng:
                setattr(desc, name_i, dp())
                setattr(desc, name_p, dp())
                continue
            I = np.ascontiguousarray(mortar_operators(N, Ng)[0])
            P = np.ascontiguousarray(mortar_operators(Ng, N)[0])
            self._ops += [I, P]
            setattr(desc, name_i, _dp(I))
            setattr(desc, name_p, _dp(P))
        h = C.c_void_p()
        _check(lib().bfam_gpu_pglue_create(dom_m.handle, dom_p.handle, C.byref(desc),
                                           C.byref(h)))
        self._h = h
        self.Ng = Ng
        self.domains = (dom_m, dom_p)

    @property
    def handle(self):
        return self._h

    def free(self):
        if getattr(self, "_h", None) and self._h.value:
            lib().bfam_gpu_pglue_free(self._h)
            self._h = C.c_void_p()

    def __del__(self):
        try:
            self.free()
        except Exception:
            pass
