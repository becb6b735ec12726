"""ctypes bindings of include/chuanflow_b200.h."""
from __future__ import annotations

import ctypes as C
import os
from dataclasses import dataclass, field

import numpy as np

_HERE = os.path.dirname(os.path.abspath(__file__))
_SO = os.path.join(_HERE, "libchuanflow_b200.so")

BC = {"fixedValue": 0, "zeroGradient": 1, "fixedGradient": 2, "symmetry": 3, "outlet": 4, "wall": 5,
      "empty": 6}
GRAD = {"linear": 0, "corrected": 1, "leastSquares": 2}
DIV = {"upwind": 0, "linear": 1, "blend": 2, "linearUpwind": 3}
PRECOND = {"Jacobi": 0, "DIC": 1, "MPNN": 2, "AMG": 3, "IR32": 4, "AMG_MPNN": 5}

_f64p = C.POINTER(C.c_double)
_i64p = C.POINTER(C.c_int64)


class CfgError(RuntimeError):
    """A non-zero status from the library, with its message."""

    def __init__(self, code, msg):
        super().__init__(f"[{code}] {msg}")
        self.code = code


class _Schemes(C.Structure):
    _fields_ = [("div", C.c_int32), ("laplacian_corrected", C.c_int32), ("grad", C.c_int32),
                ("blend_coeff", C.c_double)]


class _Controls(C.Structure):
    _fields_ = [("max_iterations", C.c_int32), ("continuity_tol", C.c_double), ("pcorr_tol", C.c_double),
                ("momentum_tol", C.c_double), ("linear_tol", C.c_double), ("linear_max_iter", C.c_int32),
                ("non_orth_correctors", C.c_int32), ("relax_u", C.c_double), ("relax_p", C.c_double),
                ("p_relax_start", C.c_double), ("body_force", C.c_double * 3), ("nu", C.c_double),
                ("p_precond", C.c_int32), ("verbose", C.c_int32), ("p_ref_cell", C.c_int64),
                ("p_ref_value", C.c_double), ("dt", C.c_double), ("u_time_old", C.c_int32),
                ("u_precond", C.c_int32)]


class _Result(C.Structure):
    _fields_ = [("iterations", C.c_int32), ("converged", C.c_int32), ("final_continuity_error", C.c_double),
                ("final_momentum_residual", C.c_double), ("last_dp", C.c_double),
                ("last_continuity_corrected", C.c_double), ("u_inner_iterations", C.c_int64),
                ("p_inner_iterations", C.c_int64), ("diverged", C.c_int32)]


class _PoissonReport(C.Structure):
    _fields_ = [("inner_iterations", C.c_int64), ("outer_iterations", C.c_int32), ("converged", C.c_int32),
                ("true_rel_residual", C.c_double), ("device_ms", C.c_double), ("initial_rel_residual", C.c_double)]


POISSON = {"jacobi64": 0, "dic64": 1, "ir32": 2, "fcg_mpnn": 3, "fcg_amg": 4, "fcg_amg_mpnn": 5}


class _Report(C.Structure):
    _fields_ = [("iterations", C.c_int32), ("converged", C.c_int32), ("initial_residual", C.c_double),
                ("final_residual", C.c_double)]


_lib = None


def lib_path():
    return _SO


def lib():
    """The loaded library; raises if it has not been built."""
    global _lib
    if _lib is None:
        if not os.path.exists(_SO):
            raise ImportError(f"chuanflow_b200: {_SO} is missing; build it with `make -C chuanflow_b200/csrc`")
        _lib = C.CDLL(_SO)
        _lib.cfg_version.restype = C.c_char_p
        _lib.cfg_last_error.restype = C.c_size_t
        _lib.cfg_mesh_jitter_interior.argtypes = [C.c_void_p, C.c_double, C.c_uint64]
        _lib.cfg_amg_strength.argtypes = [C.c_void_p, C.c_double]
        _lib.cfg_mesh_destroy.argtypes = [C.c_void_p]
        _lib.cfg_ctx_destroy.argtypes = [C.c_void_p]
        _lib.cfg_set_patch_bc.argtypes = [C.c_void_p, C.c_char, C.c_int32, C.c_int32, _f64p]
    return _lib


def _err():
    buf = C.create_string_buffer(1024)
    lib().cfg_last_error(buf, 1024)
    return buf.value.decode()


def _check(rc):
    if rc != 0:
        raise CfgError(rc, _err())


def _dp(a):
    return a.ctypes.data_as(_f64p)


def _ip(a):
    return a.ctypes.data_as(_i64p)


def _f64(a, shape=None):
    a = np.ascontiguousarray(a, dtype=np.float64)
    return a.reshape(shape) if shape is not None else a


# --------------------------------------------------------------------------
# mesh
# --------------------------------------------------------------------------

class PolyMesh:
    """polyMesh held by the library (host addressing + geometry)."""

    def __init__(self, points, face_offsets, face_verts, owner, neighbour, patches):
        """patches: list of (name, type, start, size)."""
        pts = _f64(points).reshape(-1, 3)
        fo = np.ascontiguousarray(face_offsets, np.int64)
        fv = np.ascontiguousarray(face_verts, np.int64)
        own = np.ascontiguousarray(owner, np.int64)
        nbr = np.ascontiguousarray(neighbour, np.int64)
        names = (C.c_char_p * len(patches))(*[p[0].encode() for p in patches])
        types = (C.c_char_p * len(patches))(*[p[1].encode() for p in patches])
        ps = np.array([p[2] for p in patches], np.int64)
        pz = np.array([p[3] for p in patches], np.int64)
        h = C.c_void_p()
        _check(lib().cfg_mesh_create(_dp(pts), C.c_int64(pts.shape[0]), _ip(fo), _ip(fv), C.c_int64(own.size),
                                     _ip(own), _ip(nbr) if nbr.size else None, C.c_int64(nbr.size),
                                     C.c_int32(len(patches)), names, types, _ip(ps), _ip(pz), C.byref(h)))
        self._h = h
        self._counts()

    @classmethod
    def block(cls, mn, mx, cells, sides=None):
        """BlockMesh::create; sides maps xmin..zmax to (name, type)."""
        order = ["xmin", "xmax", "ymin", "ymax", "zmin", "zmax"]
        sides = sides or {}
        names = (C.c_char_p * 6)(*[(sides[k][0].encode() if k in sides else None) for k in order])
        types = (C.c_char_p * 6)(*[(sides[k][1].encode() if k in sides else None) for k in order])
        mn = _f64(mn)
        mx = _f64(mx)
        h = C.c_void_p()
        _check(lib().cfg_mesh_block(_dp(mn), _dp(mx), C.c_int64(cells[0]), C.c_int64(cells[1]),
                                    C.c_int64(cells[2]), names, types, C.byref(h)))
        self = cls.__new__(cls)
        self._h = h
        self._counts()
        return self

    @classmethod
    def from_cells(cls, points, cell_types, cell_offsets, cell_verts):
        """The polyMesh the reference's gmsh reader builds from these volume
        cells (4 tet, 5 hex, 6 prism; patches named after bounding-box planes)."""
        pts = _f64(points).reshape(-1, 3)
        ty = np.ascontiguousarray(cell_types, np.int32)
        off = np.ascontiguousarray(cell_offsets, np.int64)
        cv = np.ascontiguousarray(cell_verts, np.int64)
        h = C.c_void_p()
        _check(lib().cfg_mesh_from_cells(_dp(pts), C.c_int64(pts.shape[0]), ty.ctypes.data_as(C.POINTER(C.c_int32)),
                                         _ip(off), _ip(cv), C.c_int64(ty.size), C.byref(h)))
        self = cls.__new__(cls)
        self._h = h
        self._counts()
        return self

    @classmethod
    def read_gmsh(cls, path, patch_types=None):
        """GmshMesh::fromFile: an ASCII .msh 2.2 / 4.x file; patch_types maps
        physical-group names to boundary types (others "wall")."""
        pt = patch_types or {}
        names = (C.c_char_p * max(1, len(pt)))(*[k.encode() for k in pt])
        types = (C.c_char_p * max(1, len(pt)))(*[v.encode() for v in pt.values()])
        h = C.c_void_p()
        _check(lib().cfg_mesh_read_gmsh(str(path).encode(), C.c_int32(len(pt)), names, types, C.byref(h)))
        self = cls.__new__(cls)
        self._h = h
        self._counts()
        return self

    def write_vtu(self, path, fields=None, binary=True):
        """VtkWriter: cell fields {name: array (n) or (n, 3)}; binary=False
        writes the reference's ASCII file."""
        fields = fields or {}
        arrs = [np.ascontiguousarray(v, np.float64) for v in fields.values()]
        n = len(arrs)
        names = (C.c_char_p * max(1, n))(*[k.encode() for k in fields])
        comps = (C.c_int32 * max(1, n))(*[1 if a.ndim == 1 else 3 for a in arrs])
        ptrs = (C.POINTER(C.c_double) * max(1, n))(*[_dp(a) for a in arrs])
        _check(lib().cfg_mesh_write_vtu(self._h, str(path).encode(), C.c_int32(n), names, comps, ptrs,
                                        C.c_int32(int(binary))))

    def write_hdf5(self, path, fields=None):
        """writeFieldsHdf5: /points, /owner, /neighbour and /fields/<name>
        for cell fields {name: array (n_cells,)}."""
        fields = fields or {}
        arrs = [np.ascontiguousarray(v, np.float64) for v in fields.values()]
        for k, a in zip(fields, arrs):
            if a.shape != (self.n_cells,):
                raise CfgError(1, "hdf5: field '%s' size mismatch (expected %d cells)" % (k, self.n_cells))
        n = len(arrs)
        names = (C.c_char_p * max(1, n))(*[k.encode() for k in fields])
        ptrs = (C.POINTER(C.c_double) * max(1, n))(*[_dp(a) for a in arrs])
        _check(lib().cfg_mesh_write_hdf5(self._h, str(path).encode(), C.c_int32(n), names, ptrs))

    def _counts(self):
        c = np.zeros(5, np.int64)
        _check(lib().cfg_mesh_counts(self._h, _ip(c)))
        self.n_points, self.n_cells, self.n_faces, self.n_internal_faces, self.n_patches = (int(x) for x in c)
        self.patches = []
        for i in range(self.n_patches):
            nb = C.create_string_buffer(256)
            tb = C.create_string_buffer(256)
            s = C.c_int64()
            z = C.c_int64()
            _check(lib().cfg_mesh_patch(self._h, C.c_int32(i), nb, 256, tb, 256, C.byref(s), C.byref(z)))
            self.patches.append((nb.value.decode(), tb.value.decode(), s.value, z.value))

    def __del__(self):
        h = getattr(self, "_h", None)
        if h is not None and h.value and _lib is not None:
            _lib.cfg_mesh_destroy(h)
            self._h = None

    @property
    def n_boundary_faces(self):
        return self.n_faces - self.n_internal_faces

    def patch_id(self, name):
        for i, p in enumerate(self.patches):
            if p[0] == name:
                return i
        raise CfgError(4, f"polyMesh: no patch named '{name}'")

    def move_points(self, points):
        pts = _f64(points).reshape(-1, 3)
        _check(lib().cfg_mesh_move_points(self._h, _dp(pts), C.c_int64(pts.shape[0])))

    def jitter_interior(self, fraction, seed):
        _check(lib().cfg_mesh_jitter_interior(self._h, C.c_double(fraction), C.c_uint64(seed)))

    def device_order(self, order=None):
        """The device numbering a context of this order uses, new -> original."""
        out = np.zeros(self.n_cells, np.int64)
        _check(lib().cfg_mesh_device_order(self._h, C.c_int32(CELL_ORDER[order]), _ip(out)))
        return out

    def addressing(self):
        pts = np.zeros((self.n_points, 3))
        fo = np.zeros(self.n_faces + 1, np.int64)
        _check(lib().cfg_mesh_addressing(self._h, None, _ip(fo), None, None, None))
        fv = np.zeros(int(fo[-1]), np.int64)
        own = np.zeros(self.n_faces, np.int64)
        nbr = np.zeros(max(self.n_internal_faces, 1), np.int64)
        _check(lib().cfg_mesh_addressing(self._h, _dp(pts), _ip(fo), _ip(fv), _ip(own), _ip(nbr)))
        return {"points": pts, "face_offsets": fo, "face_verts": fv, "owner": own,
                "neighbour": nbr[:self.n_internal_faces]}

    def geometry(self):
        N, F = self.n_cells, self.n_faces
        g = {"V": np.zeros(N), "C": np.zeros((N, 3)), "Cf": np.zeros((F, 3)), "Sf": np.zeros((F, 3)),
             "magSf": np.zeros(F), "d": np.zeros((F, 3)), "invDist": np.zeros(F)}
        _check(lib().cfg_mesh_geometry(self._h, *[_dp(g[k]) for k in ("V", "C", "Cf", "Sf", "magSf", "d",
                                                                        "invDist")]))
        return g

    def weights(self):
        ow = np.zeros(max(1, self.n_internal_faces))
        sk = np.zeros((self.n_faces, 3))
        _check(lib().cfg_mesh_weights(self._h, _dp(ow), _dp(sk)))
        return ow, sk


# --------------------------------------------------------------------------
# case
# --------------------------------------------------------------------------

@dataclass
class Schemes:
    """Schemes (src/3d/include/cf/fvm/FvMatrix.h:30-38)."""
    div: str = "upwind"
    laplacian: str = "corrected"
    grad: str = "corrected"
    blend_coeff: float = 0.9

    def _c(self):
        return _Schemes(DIV[self.div], int(self.laplacian == "corrected"), GRAD.get(self.grad, 0),
                        self.blend_coeff)


@dataclass
class SimpleControls:
    """SimpleControls (src/3d/include/cf/fvm/SimpleSolver.h:13-64) with the
    reference's defaults, plus the gpu{} settings."""
    max_iterations: int = 200
    continuity_tol: float = 1e-6
    pcorr_tol: float = 0.0
    momentum_tol: float = 0.0
    linear_tol: float = 1e-7
    linear_max_iter: int = 2000
    non_orth_correctors: int = 2
    relax_u: float = 0.7
    relax_p: float = 0.3
    p_relax_start: float = 0.0
    body_force: tuple = (0.0, 0.0, 0.0)
    nu: float = 1e-4
    p_preconditioner: str = "Jacobi"
    verbose: bool = False
    p_ref_cell: int = -1
    p_ref_value: float = 0.0
    dt: float = 0.0          # SimpleControls::dt (pseudo-) time step; 0: steady
    u_time_old: int = 0      # 1: the velocity at the start of the call is the old level
    u_preconditioner: str = "Jacobi"  # the momentum BiCGStab's: "Jacobi" (the reference's) or "AMG"

    def _c(self):
        c = _Controls()
        c.max_iterations = self.max_iterations
        c.continuity_tol = self.continuity_tol
        c.pcorr_tol = self.pcorr_tol
        c.momentum_tol = self.momentum_tol
        c.linear_tol = self.linear_tol
        c.linear_max_iter = self.linear_max_iter
        c.non_orth_correctors = self.non_orth_correctors
        c.relax_u = self.relax_u
        c.relax_p = self.relax_p
        c.p_relax_start = self.p_relax_start
        for i in range(3):
            c.body_force[i] = self.body_force[i]
        c.nu = self.nu
        c.p_precond = PRECOND[self.p_preconditioner]
        c.verbose = int(self.verbose)
        c.p_ref_cell = self.p_ref_cell
        c.p_ref_value = self.p_ref_value
        c.dt = self.dt
        c.u_time_old = int(self.u_time_old)
        c.u_precond = U_PRECOND[self.u_preconditioner]
        return c


@dataclass
class SimpleResult:
    iterations: int
    converged: bool
    final_continuity_error: float
    final_momentum_residual: float
    last_dp: float
    last_continuity_corrected: float
    u_inner_iterations: int
    p_inner_iterations: int
    diverged: bool


@dataclass
class SolverReport:
    iterations: int
    converged: bool
    initial_residual: float
    final_residual: float


CELL_ORDER = {None: -1, "identity": 0, "colour": 1, "rcm": 2, "rcm-colour": 3}


U_PRECOND = {"Jacobi": 0, "AMG": 3}
KERNEL_SLOTS = ("cg_spmv", "cg_update", "cg_p", "bi_p", "bi_spmv1", "bi_spmv2", "bi_x", "dic_apply",
                "bia_p", "amgv_pre0", "amgv_coarse", "amgv_post0", "bia_spmv1", "bia_s", "bia_spmv2", "bia_x")


class SimpleCase:
    """U, p, phi and their boundary conditions on one device."""

    def __init__(self, mesh: PolyMesh, device: int = 0, schemes: Schemes | None = None, order: str | None = None):
        """order: the device cell numbering ("identity", "colour", "rcm",
        "rcm-colour"); None takes CHUANFLOW_CELL_ORDER, else "identity"."""
        self.mesh = mesh
        h = C.c_void_p()
        _check(lib().cfg_ctx_create_ordered(mesh._h, C.c_int32(device), None, C.c_int32(CELL_ORDER[order]),
                                            C.byref(h)))
        self._h = h
        self.set_schemes(schemes or Schemes())

    def __del__(self):
        h = getattr(self, "_h", None)
        if h is not None and h.value and _lib is not None:
            _lib.cfg_ctx_destroy(h)
            self._h = None

    def _patch(self, patch):
        return patch if isinstance(patch, int) else self.mesh.patch_id(patch)

    def set_patch_bc(self, field_name, patch, bc_type, value=0.0):
        """volVectorField / volScalarField ::setPatchValue."""
        v = _f64(np.atleast_1d(value))
        if field_name == "U" and v.size != 3:
            v = _f64(np.zeros(3) + v[0])
        _check(lib().cfg_set_patch_bc(self._h, field_name.encode(), self._patch(patch), BC[bc_type], _dp(v)))

    def set_face_values_U(self, faces, values):
        f = np.ascontiguousarray(faces, np.int64)
        v = _f64(values).reshape(-1, 3)
        _check(lib().cfg_set_face_values_U(self._h, C.c_int64(f.size), _ip(f), _dp(v)))

    def set_schemes(self, schemes: Schemes):
        self.schemes = schemes
        s = schemes._c()
        _check(lib().cfg_set_schemes(self._h, C.byref(s)))

    def upload(self, U=None, p=None, phi=None):
        _check(lib().cfg_fields_upload(self._h, _dp(_f64(U)) if U is not None else None,
                                       _dp(_f64(p)) if p is not None else None,
                                       _dp(_f64(phi)) if phi is not None else None))

    def download(self, U=None, p=None, phi=None):
        """U (n_cells x 3), p and phi; given arrays (C-contiguous float64 of
        those shapes, e.g. pinned buffers) are filled in place."""
        def out(a, shape):
            if a is None:
                return np.empty(shape)
            if a.dtype != np.float64 or a.shape != shape or not a.flags.c_contiguous or not a.flags.writeable:
                raise ValueError(f"download: expected a writeable C-contiguous float64 array of shape {shape}")
            return a
        U = out(U, (self.mesh.n_cells, 3))
        p = out(p, (self.mesh.n_cells,))
        phi = out(phi, (self.mesh.n_faces,))
        _check(lib().cfg_fields_download(self._h, _dp(U), _dp(p), _dp(phi)))
        return U, p, phi

    def init_flux(self, u0=None):
        _check(lib().cfg_fields_init_flux(self._h, _dp(_f64(u0)) if u0 is not None else None))

    def solve(self, controls: SimpleControls) -> SimpleResult:
        """solveIncompressibleSimple on the device fields."""
        r = _Result()
        c = controls._c()
        _check(lib().cfg_simple_iterate(self._h, C.byref(c), C.byref(r)))
        return SimpleResult(r.iterations, bool(r.converged), r.final_continuity_error,
                            r.final_momentum_residual, r.last_dp, r.last_continuity_corrected,
                            r.u_inner_iterations, r.p_inner_iterations, bool(r.diverged))

    def last_timing(self):
        ms = np.zeros(8)
        n = C.c_int64()
        _check(lib().cfg_last_timing(self._h, _dp(ms), C.byref(n)))
        return ms, n.value

    def kernel_timing(self, enable=True):
        _check(lib().cfg_kernel_timing(self._h, C.c_int32(int(enable))))

    def kernel_stats(self):
        out = np.zeros(2 * len(KERNEL_SLOTS))
        _check(lib().cfg_kernel_stats(self._h, _dp(out), C.c_int32(len(KERNEL_SLOTS))))
        return {n: (int(out[2 * i]), float(out[2 * i + 1])) for i, n in enumerate(KERNEL_SLOTS)}

    def kernel_components(self):
        """Per solver kernel, its timed launches weighted by the vector
        components each still iterated on."""
        out = np.zeros(len(KERNEL_SLOTS))
        _check(lib().cfg_kernel_components(self._h, _dp(out), C.c_int32(len(KERNEL_SLOTS))))
        return {n: float(out[i]) for i, n in enumerate(KERNEL_SLOTS)}

    # ---- the pressure-Poisson system on its own ----
    def poisson_setup(self, ref_cell=-1):
        """A = orthogonal laplacianFace(1) under the p conditions, pinned at ref_cell."""
        _check(lib().cfg_poisson_setup(self._h, C.c_int64(ref_cell)))

    def poisson_solve(self, b, method="dic64", tol=1e-8, x0=None, max_iter=20000, inner_max_iter=5000,
                      inner_tol=1e-4):
        """Returns (x, report dict); the residual test is |b - Ax|2/|b|2 in FP64."""
        x = np.zeros(self.mesh.n_cells) if x0 is None else np.array(x0, np.float64, copy=True)
        r = _PoissonReport()
        _check(lib().cfg_poisson_solve(self._h, _dp(_f64(b)), _dp(x), C.c_int32(POISSON[method]), C.c_double(tol),
                                       C.c_int32(max_iter), C.c_int32(inner_max_iter), C.c_double(inner_tol),
                                       C.byref(r)))
        return x, {"inner_iterations": r.inner_iterations, "outer_iterations": r.outer_iterations,
                   "converged": bool(r.converged), "true_rel_residual": r.true_rel_residual,
                   "device_ms": r.device_ms, "initial_rel_residual": r.initial_rel_residual}

    def poisson_amg_setup(self):
        """The FP32 aggregation-AMG hierarchy of the Poisson system: levels,
        rows per level, host structure and device value set-up times."""
        out = np.zeros(11)
        _check(lib().cfg_poisson_amg_setup(self._h, _dp(out)))
        nl = int(out[0])
        return {"levels": nl, "rows": [int(v) for v in out[1:1 + min(nl, 8)]], "structure_ms": float(out[9]),
                "values_ms": float(out[10])}

    def amg_strength(self, theta):
        """Strength-of-connection threshold of the pressure AMG hierarchy's
        aggregation (0: plain); set before the first AMG pressure solve."""
        _check(lib().cfg_amg_strength(self._h, float(theta)))

    def poisson_amg_apply(self, r):
        """One V-cycle z = V(r) of that hierarchy (FP32 inside, FP64 in and out)."""
        z = np.zeros(self.mesh.n_cells)
        _check(lib().cfg_poisson_amg_apply(self._h, _dp(_f64(r)), _dp(z)))
        return z

    def poisson_amg_apply3(self, r3, z3=None, done=(0, 0, 0)):
        """The three-component V-cycle on r3 (3 x n); component q is left as
        z3[q] (zeros by default) when done[q]."""
        n = self.mesh.n_cells
        z = np.zeros(3 * n) if z3 is None else np.array(z3, np.float64, copy=True).reshape(-1)
        d = (C.c_int32 * 3)(*[int(v) for v in done])
        _check(lib().cfg_poisson_amg_apply3(self._h, _dp(_f64(np.asarray(r3).reshape(-1))), _dp(z), d))
        return z.reshape(3, n)

    # ---- diagnostics ----
    def probe_equations(self, controls: SimpleControls, xprobe):
        N, F = self.mesh.n_cells, self.mesh.n_faces
        sizes = [("gradPn", 3 * N), ("U_diag", 3 * N), ("U_h0", 3 * N), ("U_h1", 3 * N), ("rAUf", F),
                 ("divPhi", N), ("contErr", 1), ("p_diag", N), ("p_h0", N), ("p_h1", N), ("gradPFull", 3 * N),
                 ("phiCorrected", F)]
        out = np.zeros(sum(s for _, s in sizes))
        c = controls._c()
        _check(lib().cfg_probe_equations(self._h, C.byref(c), _dp(_f64(xprobe)), _dp(out)))
        res, o = {}, 0
        for k, s in sizes:
            res[k] = out[o:o + s].copy()
            o += s
        for k in ("gradPn", "gradPFull"):
            res[k] = res[k].reshape(3, N).T.copy()
        for k in ("U_diag", "U_h0", "U_h1"):
            res[k] = res[k].reshape(3, N)
        return res

    def probe_dic(self, r):
        n = self.mesh.n_cells
        z = np.zeros(n)
        rd = np.zeros(n)
        nc = C.c_int32()
        _check(lib().cfg_probe_dic(self._h, _dp(_f64(r)), _dp(z), _dp(rd), C.byref(nc)))
        return z, rd, nc.value

    def gradient(self, data, bvals, scheme, vol_quirk=False):
        out = np.zeros((self.mesh.n_cells, 3))
        _check(lib().cfg_gradient(self._h, _dp(_f64(data)), _dp(_f64(bvals)), C.c_int32(GRAD.get(scheme, 0)),
                                  C.c_int32(int(vol_quirk)), _dp(out)))
        return out


# --------------------------------------------------------------------------
# linear solvers and the case-file runner
# --------------------------------------------------------------------------

def _sparse(method, row_start, cols, vals, b, x0, tol, max_iter, device):
    rs = np.ascontiguousarray(row_start, np.int64)
    cl = np.ascontiguousarray(cols, np.int64)
    vl = _f64(vals)
    x = np.array(x0, dtype=np.float64, copy=True)
    r = _Report()
    _check(lib().cfg_sparse_solve(None, C.c_int32(device), C.c_int64(rs.size - 1), _ip(rs), _ip(cl), _dp(vl),
                                  _dp(_f64(b)), _dp(x), C.c_double(tol), C.c_int32(max_iter), C.c_int32(method),
                                  C.byref(r)))
    return x, SolverReport(r.iterations, bool(r.converged), r.initial_residual, r.final_residual)


def solve_cg(row_start, cols, vals, b, x0, tol, max_iter, device=0):
    """solveCG on a CSR matrix (Matrix.cpp:153-222)."""
    return _sparse(0, row_start, cols, vals, b, x0, tol, max_iter, device)


def solve_bicgstab(row_start, cols, vals, b, x0, tol, max_iter, device=0):
    """solveBiCGStab on a CSR matrix (Matrix.cpp:224-319)."""
    return _sparse(1, row_start, cols, vals, b, x0, tol, max_iter, device)


def _number_or_word(x):
    try:
        return float(x)
    except ValueError:
        return x


def inspect_case_file(path):
    """Host-only parse of a case file: a dict of what the runner would use."""
    buf = C.create_string_buffer(1 << 16)
    _check(lib().cfg_case_inspect(str(path).encode(), buf, C.c_size_t(1 << 16)))
    out = {"patches": {}}
    for ln in buf.value.decode().splitlines():
        k, *v = ln.split()
        if k == "patch":
            out["patches"][v[0]] = {"type": v[1], "start": int(v[2]), "size": int(v[3]), "U_type": int(v[5]),
                                    "U": tuple(float(x) for x in v[6:9]), "p_type": int(v[10]), "p": float(v[11])}
        else:
            out[k] = [_number_or_word(x) for x in v]
    return out


def run_case_file(path, device=0, fields=False):
    """A chflow-simple-foam case file end to end; returns (result, counts),
    or with fields=True (result, counts, (U, p, phi)): the case is then run
    a second time into buffers sized by the first run's counts."""
    counts = np.zeros(5, np.int64)
    r = _Result()
    _check(lib().cfg_run_case_file(str(path).encode(), C.c_int32(device), C.byref(r), _ip(counts), None, None,
                                   None))
    res = lambda: SimpleResult(r.iterations, bool(r.converged), r.final_continuity_error, r.final_momentum_residual,
                               r.last_dp, r.last_continuity_corrected, r.u_inner_iterations, r.p_inner_iterations,
                               bool(r.diverged))
    if not fields:
        return res(), counts
    U, p, phi = np.zeros((int(counts[1]), 3)), np.zeros(int(counts[1])), np.zeros(int(counts[2]))
    _check(lib().cfg_run_case_file(str(path).encode(), C.c_int32(device), C.byref(r), _ip(counts), _dp(U), _dp(p),
                                   _dp(phi)))
    return res(), counts, (U, p, phi)


# ---- detail blocks and batches --------------------------------------------

class DetailMeasure(C.Structure):
    _fields_ = [("cells", C.c_int64), ("sweeps", C.c_int32), ("converged", C.c_int32), ("diverged", C.c_int32),
                ("dp_pa", C.c_double), ("imposed_q", C.c_double), ("flux_in", C.c_double),
                ("flux_out", C.c_double), ("inlet_area", C.c_double), ("plug_speed", C.c_double),
                ("device_ms", C.c_double), ("u_inner_iterations", C.c_int64), ("p_inner_iterations", C.c_int64),
                ("status", C.c_int32)]

    def as_dict(self):
        return {k: getattr(self, k) for k, _ in self._fields_}


def _detail_setup(self, inlet_shape="flat", rho=1.0):
    """DetailBlock's constructor on this case's mesh (inlet/outlet patches by
    type, cross-sections, inlet profile flat | parabolic | power1over7)."""
    _check(lib().cfg_detail_setup(self._h, inlet_shape.encode(), C.c_double(rho)))


def _detail_loss(self, q, controls):
    """DetailBlock::lossAt(q): boundary conditions of rate q, SIMPLE from the
    current fields, the measured drop (dict of BlockMeasure's fields)."""
    c = controls._c()
    m = DetailMeasure()
    _check(lib().cfg_detail_loss(self._h, C.c_double(q), C.byref(c), C.byref(m)))
    return m.as_dict()


def _turbulence_setup(self, model="kEpsilon", intensity=0.05, length_scale=-1.0, relaxation=0.7, nu=1e-4,
                      c_des=0.61, re_onset=0.0, onset_width=-1.0, gamma_rate=4.0):
    """RansModel::create for this case (model kEpsilon | kOmegaSST | des |
    gammaTransition | laminar): call after the velocity conditions are set;
    advanced once per SIMPLE iteration.  c_des (des) and re_onset,
    onset_width, gamma_rate (gammaTransition) are TurbulenceConfig's."""
    _check(lib().cfg_turbulence_params(self._h, C.c_double(c_des), C.c_double(re_onset), C.c_double(onset_width),
                                       C.c_double(gamma_rate)))
    _check(lib().cfg_turbulence_setup(self._h, model.encode(), C.c_double(intensity), C.c_double(length_scale),
                                      C.c_double(relaxation), C.c_double(nu)))


def _turbulence_fields(self):
    """k, the dissipation variable (key "eps": epsilon, or omega for
    kOmegaSST), nut (cells) and nu + nut on faces."""
    n, f = self.mesh.n_cells, self.mesh.n_faces
    k, e, nut, nuf = np.zeros(n), np.zeros(n), np.zeros(n), np.zeros(f)
    _check(lib().cfg_turbulence_fields(self._h, _dp(k), _dp(e), _dp(nut), _dp(nuf)))
    return {"k": k, "eps": e, "nut": nut, "nuEffFace": nuf}


def _detail_turbulence(self, model="kEpsilon", intensity=0.05, length_scale=-1.0, relaxation=0.7, nu=1e-4):
    """The detail block's RANS model, created at its first lossAt."""
    _check(lib().cfg_detail_turbulence(self._h, model.encode(), C.c_double(intensity), C.c_double(length_scale),
                                       C.c_double(relaxation), C.c_double(nu)))


def _mpnn_create(self, layers=4, seed=1):
    """The learned pressure preconditioner on this case's pressure matrix."""
    _check(lib().cfg_mpnn_create(self._h, C.c_int32(layers), C.c_uint64(seed)))


def _mpnn_weights(self, set=None):
    """The FP32 master weights (after setting `set`, when given)."""
    n = C.c_int64()
    _check(lib().cfg_mpnn_params(self._h, C.byref(n)))
    out = np.zeros(n.value, np.float32)
    src = None if set is None else np.ascontiguousarray(set, np.float32)
    _check(lib().cfg_mpnn_weights(self._h, out.ctypes.data_as(C.POINTER(C.c_float)),
                                  None if src is None else src.ctypes.data_as(C.POINTER(C.c_float)), n))
    return out


def _mpnn_loss_grad(self, r):
    n = C.c_int64()
    _check(lib().cfg_mpnn_params(self._h, C.byref(n)))
    g = np.zeros(n.value, np.float32)
    loss = C.c_double()
    _check(lib().cfg_mpnn_loss_grad(self._h, _dp(_f64(r)), C.byref(loss), g.ctypes.data_as(C.POINTER(C.c_float))))
    return loss.value, g


def _mpnn_loss_grad_pair(self, r, t):
    """One (residual, converged correction) pair's energy-norm loss and
    its gradient."""
    n = C.c_int64()
    _check(lib().cfg_mpnn_params(self._h, C.byref(n)))
    g = np.zeros(n.value, np.float32)
    loss = C.c_double()
    _check(lib().cfg_mpnn_loss_grad_pair(self._h, _dp(_f64(r)), _dp(_f64(t)), C.byref(loss),
                                         g.ctypes.data_as(C.POINTER(C.c_float))))
    return loss.value, g


def _mpnn_train_pairs(self, samples, targets, epochs=1, lr=1e-3):
    """Adam over (residual, converged correction) pairs (rows); returns the
    per-epoch mean losses."""
    s = np.ascontiguousarray(samples, np.float64)
    t = np.ascontiguousarray(targets, np.float64)
    if s.shape != t.shape:
        raise ValueError("mpnn_train_pairs: samples and targets differ in shape")
    losses = np.zeros(epochs)
    _check(lib().cfg_mpnn_train_pairs(self._h, _dp(s), _dp(t), C.c_int32(s.shape[0]), C.c_int32(epochs),
                                      C.c_float(lr), _dp(losses)))
    return losses


def _mpnn_time(self, reps):
    """(ms per application, ms per message-passing layer launch), CUDA
    events, on the current pressure matrix."""
    out = np.zeros(2)
    _check(lib().cfg_mpnn_time(self._h, C.c_int32(reps), _dp(out)))
    return float(out[0]), float(out[1])


def _mpnn_apply(self, r):
    z = np.zeros(self.mesh.n_cells)
    _check(lib().cfg_mpnn_apply(self._h, _dp(_f64(r)), _dp(z)))
    return z


def _mpnn_train(self, samples, epochs=1, lr=1e-3):
    """Adam over residual samples (rows); returns the per-epoch mean losses."""
    s = np.ascontiguousarray(samples, np.float64)
    losses = np.zeros(epochs)
    _check(lib().cfg_mpnn_train(self._h, _dp(s), C.c_int32(s.shape[0]), C.c_int32(epochs), C.c_float(lr),
                                _dp(losses)))
    return losses


def _poisson_residual(self, b, x):
    r = np.zeros(self.mesh.n_cells)
    _check(lib().cfg_poisson_residual(self._h, _dp(_f64(b)), _dp(_f64(x)), _dp(r)))
    return r


class _PisoControls(C.Structure):
    _fields_ = [("dt", C.c_double), ("correctors", C.c_int32), ("continuity_tol", C.c_double),
                ("linear_tol", C.c_double), ("linear_max_iter", C.c_int32), ("non_orth_correctors", C.c_int32),
                ("body_force", C.c_double * 3), ("nu", C.c_double), ("p_precond", C.c_int32)]


class _PisoResult(C.Structure):
    _fields_ = [("correctors_used", C.c_int32), ("converged", C.c_int32), ("diverged", C.c_int32),
                ("predicted_continuity_error", C.c_double), ("continuity_error", C.c_double),
                ("pressure_correction_max", C.c_double), ("u_inner_iterations", C.c_int64),
                ("p_inner_iterations", C.c_int64), ("device_ms", C.c_double)]


@dataclass
class PisoControls:
    """PisoControls (src/3d/include/cf/fvm/PisoSolver.h) + nu and the GPU
    pressure preconditioner."""
    dt: float = 0.01
    correctors: int = 2
    continuity_tol: float = 1e-10
    linear_tol: float = 1e-8
    linear_max_iter: int = 2000
    non_orth_correctors: int = 2
    body_force: tuple = (0.0, 0.0, 0.0)
    nu: float = 1e-4
    p_preconditioner: str = "Jacobi"

    def _c(self):
        c = _PisoControls()
        c.dt = self.dt
        c.correctors = self.correctors
        c.continuity_tol = self.continuity_tol
        c.linear_tol = self.linear_tol
        c.linear_max_iter = self.linear_max_iter
        c.non_orth_correctors = self.non_orth_correctors
        for i in range(3):
            c.body_force[i] = self.body_force[i]
        c.nu = self.nu
        c.p_precond = PRECOND[self.p_preconditioner]
        return c


def _piso_step(self, controls):
    """One transient PISO step of the device fields (dict of PisoStepResult)."""
    c = controls._c()
    r = _PisoResult()
    _check(lib().cfg_piso_step(self._h, C.byref(c), C.byref(r)))
    return {k: getattr(r, k) for k, _ in r._fields_}


def _write_vtu(self, path, binary=True):
    """The case's fields (p, k/epsilon/nut with a RANS model, U) as .vtu."""
    _check(lib().cfg_write_vtu(self._h, str(path).encode(), C.c_int32(int(binary))))


def _write_hdf5(self, path):
    """The case's cell fields as HDF5: /fields/p, k/epsilon (omega)/nut with
    a RANS model, Ux, Uy, Uz, beside the mesh's points, owner, neighbour."""
    _check(lib().cfg_write_hdf5(self._h, str(path).encode()))


SimpleCase.write_vtu = _write_vtu
SimpleCase.write_hdf5 = _write_hdf5
SimpleCase.piso_step = _piso_step
def _mpnn_collect(self, on=1, max_samples=64):
    """Keep (1) / stop keeping (0) / drop and keep (2) training pairs of
    later pressure solves (the residual each starts from and the correction
    it converges to); returns the count kept."""
    n = C.c_int32()
    _check(lib().cfg_mpnn_collect(self._h, C.c_int32(int(on)), C.c_int32(max_samples), C.byref(n)))
    return n.value


def _mpnn_train_collected(self, epochs=10, lr=1e-3):
    losses = np.zeros(epochs)
    _check(lib().cfg_mpnn_train_collected(self._h, C.c_int32(epochs), C.c_float(lr), _dp(losses)))
    return losses


SimpleCase.mpnn_collect = _mpnn_collect
SimpleCase.mpnn_train_collected = _mpnn_train_collected
SimpleCase.mpnn_create = _mpnn_create
SimpleCase.mpnn_weights = _mpnn_weights
SimpleCase.mpnn_loss_grad = _mpnn_loss_grad
SimpleCase.mpnn_apply = _mpnn_apply
SimpleCase.mpnn_train = _mpnn_train
SimpleCase.mpnn_loss_grad_pair = _mpnn_loss_grad_pair
SimpleCase.mpnn_train_pairs = _mpnn_train_pairs
SimpleCase.mpnn_time = lambda self, reps=20: _mpnn_time(self, reps)
SimpleCase.poisson_residual = _poisson_residual
SimpleCase.detail_turbulence = _detail_turbulence
SimpleCase.turbulence_setup = _turbulence_setup
SimpleCase.turbulence_fields = _turbulence_fields
SimpleCase.detail_setup = _detail_setup
SimpleCase.detail_loss = _detail_loss


class Batch:
    """Detail-block cases evaluated together, one stream each."""

    CANDIDATES = [(1, 0), (8, 1), (16, 1), (16, -1), (32, -1), (64, -1), (0, 1), (0, 2), (0, -1)]

    def __init__(self, cases):
        self.cases = list(cases)
        arr = (C.c_void_p * len(self.cases))(*[c._h.value for c in self.cases])
        h = C.c_void_p()
        _check(lib().cfg_batch_create(C.c_int32(len(self.cases)), arr, C.byref(h)))
        self._h = h

    def __del__(self):
        h = getattr(self, "_h", None)
        if h is not None and h.value and _lib is not None:
            _lib.cfg_batch_destroy(h)
            self._h = None

    def set_schedule(self, workers, row_blocks_per_sm=0):
        _check(lib().cfg_batch_set_schedule(self._h, C.c_int32(workers), C.c_int32(row_blocks_per_sm)))

    def _args(self, q, controls):
        n = len(self.cases)
        qa = _f64(q)
        if isinstance(controls, SimpleControls):
            controls = [controls] * n
        ca = (_Controls * n)(*[c._c() for c in controls])
        return qa, ca

    def loss(self, q, controls):
        """One coupling pass; returns (list of measure dicts, wall ms)."""
        qa, ca = self._args(q, controls)
        out = (DetailMeasure * len(self.cases))()
        ms = C.c_double()
        _check(lib().cfg_batch_loss(self._h, _dp(qa), ca, out, C.byref(ms)))
        return [m.as_dict() for m in out], ms.value

    def save(self):
        _check(lib().cfg_batch_save(self._h))

    def restore(self):
        _check(lib().cfg_batch_restore(self._h))

    def autotune(self, q, controls):
        """Runs one pass per candidate schedule and keeps the fastest;
        returns ((workers, row_blocks_per_sm), {candidate: ms})."""
        qa, ca = self._args(q, controls)
        w, r = C.c_int32(), C.c_int32()
        t = np.zeros(len(self.CANDIDATES))
        _check(lib().cfg_batch_autotune(self._h, _dp(qa), ca, C.byref(w), C.byref(r), _dp(t)))
        return (w.value, r.value), dict(zip(self.CANDIDATES, t.tolist()))
