"""ctypes view of the oracle (oracle/libcfo.so, the C restatement) and a thin
runner for the reference driver (oracle/_ref/cf_ref_driver).

Test infrastructure only: these are the checkers the CUDA path is compared
against.  Nothing in chuanflow_b200/ imports this module.
"""
from __future__ import annotations

import ctypes as C
import os
import subprocess
import tempfile
from dataclasses import dataclass

import numpy as np

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
ORACLE_DIR = os.path.join(ROOT, "oracle")
CFO_SO = os.path.join(ORACLE_DIR, "_build", "libcfo.so")
REF_DRIVER = os.path.join(ORACLE_DIR, "_ref", "cf_ref_driver")

BC = {"fixedValue": 0, "zeroGradient": 1, "fixedGradient": 2, "symmetry": 3, "outlet": 4,
      "wall": 5, "empty": 6}
GRAD = {"linear": 0, "corrected": 1, "leastSquares": 2}
DIV = {"upwind": 0, "linear": 1, "blend": 2, "linearUpwind": 3}

_f64p = C.POINTER(C.c_double)
_i64p = C.POINTER(C.c_int64)


def _p(a, ct=_f64p):
    return a.ctypes.data_as(ct) if a is not None else None


class Mesh(C.Structure):
    _fields_ = [("nP", C.c_int64), ("nC", C.c_int64), ("nF", C.c_int64), ("nInt", C.c_int64),
                ("nPatch", C.c_int64), ("pts", _f64p), ("fOff", _i64p), ("fV", _i64p),
                ("own", _i64p), ("nbr", _i64p), ("pStart", _i64p), ("pSize", _i64p),
                ("V", _f64p), ("C", _f64p), ("Cf", _f64p), ("Sf", _f64p), ("magSf", _f64p),
                ("d", _f64p), ("invDist", _f64p)]


class Bcs(C.Structure):
    _fields_ = [("uType", C.POINTER(C.c_int32)), ("uValue", _f64p), ("pType", C.POINTER(C.c_int32)),
                ("pValue", _f64p), ("uFaceSet", C.POINTER(C.c_uint8)), ("uFaceValue", _f64p)]


class Controls(C.Structure):
    _fields_ = [("maxIterations", C.c_int32), ("continuityTol", C.c_double), ("pcorrTol", C.c_double),
                ("momentumTol", C.c_double), ("linearTol", C.c_double), ("linearMaxIter", C.c_int32),
                ("nonOrthCorrectors", C.c_int32), ("relaxU", C.c_double), ("relaxP", C.c_double),
                ("pRelaxStart", C.c_double), ("bodyForce", C.c_double * 3), ("nu", C.c_double),
                ("div", C.c_int32), ("laplacianCorrected", C.c_int32), ("grad", C.c_int32),
                ("blendCoeff", C.c_double), ("verbose", C.c_int32), ("pRefCell", C.c_int64),
                ("pRefValue", C.c_double), ("pPrecond", C.c_int32)]


class Result(C.Structure):
    _fields_ = [("iterations", C.c_int32), ("converged", C.c_int32), ("finalContinuityError", C.c_double),
                ("finalMomentumResidual", C.c_double), ("lastUIters", C.c_int32), ("lastPIters", C.c_int32),
                ("error", C.c_int32), ("uItersTotal", C.c_int64), ("pItersTotal", C.c_int64)]


class Report(C.Structure):
    _fields_ = [("iterations", C.c_int32), ("converged", C.c_int32), ("initialResidual", C.c_double),
                ("finalResidual", C.c_double)]


_lib = None


def lib():
    global _lib
    if _lib is None:
        if not os.path.exists(CFO_SO):
            raise RuntimeError(f"oracle library missing: {CFO_SO} (run `make -C oracle`)")
        _lib = C.CDLL(CFO_SO)
        _lib.cfo_last_error.restype = C.c_char_p
        _lib.cfo_csr_build.restype = C.c_int64
    return _lib


def _check(rc):
    if rc != 0:
        raise RuntimeError(lib().cfo_last_error().decode())


@dataclass
class OMesh:
    """A polyMesh held as numpy arrays, with the oracle's geometry."""
    points: np.ndarray
    face_offsets: np.ndarray
    face_verts: np.ndarray
    owner: np.ndarray
    neighbour: np.ndarray
    patch_names: list
    patch_types: list
    patch_start: np.ndarray
    patch_size: np.ndarray

    def __post_init__(self):
        self.points = np.ascontiguousarray(self.points, dtype=np.float64).reshape(-1, 3)
        for k in ("face_offsets", "face_verts", "owner", "neighbour", "patch_start", "patch_size"):
            setattr(self, k, np.ascontiguousarray(getattr(self, k), dtype=np.int64))
        # the reference counts cells from owners alone (polyMesh.cpp:23), which
        # overruns its cell arrays when the last cell owns no face; count the
        # neighbours too, as chuanflow_b200 does
        self.nC = max(int(self.owner.max()) + 1 if self.owner.size else 0,
                      int(self.neighbour.max()) + 1 if self.neighbour.size else 0)
        self.nF = self.owner.size
        self.nInt = self.neighbour.size
        self.V = np.zeros(self.nC)
        self.C = np.zeros((self.nC, 3))
        self.Cf = np.zeros((self.nF, 3))
        self.Sf = np.zeros((self.nF, 3))
        self.magSf = np.zeros(self.nF)
        self.d = np.zeros((self.nF, 3))
        self.invDist = np.zeros(self.nF)
        self._c = self.cstruct()
        _check(lib().cfo_geometry(C.byref(self._c)))

    def cstruct(self):
        return Mesh(self.points.shape[0], self.nC, self.nF, self.nInt, len(self.patch_names),
                    _p(self.points), _p(self.face_offsets, _i64p), _p(self.face_verts, _i64p),
                    _p(self.owner, _i64p), _p(self.neighbour, _i64p), _p(self.patch_start, _i64p),
                    _p(self.patch_size, _i64p), _p(self.V), _p(self.C), _p(self.Cf), _p(self.Sf),
                    _p(self.magSf), _p(self.d), _p(self.invDist))

    def with_points(self, pts):
        return OMesh(pts, self.face_offsets, self.face_verts, self.owner, self.neighbour,
                     self.patch_names, self.patch_types, self.patch_start, self.patch_size)

    def owner_weights(self):
        ow = np.zeros(max(1, self.nInt))
        lib().cfo_owner_weights(C.byref(self._c), _p(ow))
        return ow

    def skew(self, ow=None):
        ow = self.owner_weights() if ow is None else ow
        s = np.zeros((self.nF, 3))
        lib().cfo_skew(C.byref(self._c), _p(ow), _p(s))
        return s

    def harmonic_gamma(self, gamma):
        g = np.zeros(self.nF)
        lib().cfo_harmonic_gamma(C.byref(self._c), C.c_double(gamma), _p(g))
        return g

    def grad(self, data, bvals, scheme, vol_quirk=False):
        data = np.ascontiguousarray(data, dtype=np.float64)
        bvals = np.ascontiguousarray(bvals, dtype=np.float64)
        out = np.zeros((self.nC, 3))
        _check(lib().cfo_grad(C.byref(self._c), _p(data), _p(bvals), GRAD.get(scheme, 0),
                              int(vol_quirk), _p(out)))
        return out


def block_mesh(mn, mx, cells, names=None, types=None):
    """The oracle's restatement of BlockMesh::create."""
    names = names or ["xmin", "xmax", "ymin", "ymax", "zmin", "zmax"]
    types = types or ["wall", "wall", "wall", "wall", "symmetry", "symmetry"]
    nx, ny, nz = cells
    cnt = np.zeros(4, np.int64)
    _check(lib().cfo_block_counts(C.c_int64(nx), C.c_int64(ny), C.c_int64(nz), _p(cnt, _i64p)))
    nP, nC, nF, nInt = (int(x) for x in cnt)
    pts = np.zeros((nP, 3))
    fOff = np.zeros(nF + 1, np.int64)
    fV = np.zeros(4 * nF, np.int64)
    own = np.zeros(nF, np.int64)
    nbr = np.zeros(nInt, np.int64)
    ps = np.zeros(6, np.int64)
    pz = np.zeros(6, np.int64)
    mn = np.asarray(mn, np.float64)
    mx = np.asarray(mx, np.float64)
    _check(lib().cfo_block_mesh(_p(mn), _p(mx), C.c_int64(nx), C.c_int64(ny), C.c_int64(nz), _p(pts),
                                _p(fOff, _i64p), _p(fV, _i64p), _p(own, _i64p), _p(nbr, _i64p),
                                _p(ps, _i64p), _p(pz, _i64p)))
    keep = pz > 0
    return OMesh(pts, fOff, fV, own, nbr, [n for n, k in zip(names, keep) if k],
                 [t for t, k in zip(types, keep) if k], ps[keep], pz[keep])


@dataclass
class Case:
    """A SIMPLE case in the reference's terms: per patch U/p conditions,
    schemes and SimpleControls."""
    mesh: OMesh
    u_type: list
    u_value: list
    p_type: list
    p_value: list
    nu: float
    div: str = "upwind"
    laplacian: str = "corrected"
    grad: str = "corrected"
    blend: float = 0.9
    max_iterations: int = 200
    continuity_tol: float = 1e-6
    pcorr_tol: float = 0.0
    momentum_tol: float = 0.0
    linear_tol: float = 1e-7
    linear_max_iter: int = 2000
    non_orth: int = 2
    relax_u: float = 0.7
    relax_p: float = 0.3
    p_relax_start: float = 0.0
    body_force: tuple = (0.0, 0.0, 0.0)
    u_face_values: dict = None
    p_ref_cell: int = -1
    p_ref_value: float = 0.0
    p_precond: int = 0

    def controls(self, verbose=False):
        c = Controls()
        c.maxIterations = self.max_iterations
        c.continuityTol = self.continuity_tol
        c.pcorrTol = self.pcorr_tol
        c.momentumTol = self.momentum_tol
        c.linearTol = self.linear_tol
        c.linearMaxIter = self.linear_max_iter
        c.nonOrthCorrectors = self.non_orth
        c.relaxU = self.relax_u
        c.relaxP = self.relax_p
        c.pRelaxStart = self.p_relax_start
        for i in range(3):
            c.bodyForce[i] = self.body_force[i]
        c.nu = self.nu
        c.div = DIV[self.div]
        c.laplacianCorrected = int(self.laplacian == "corrected")
        c.grad = GRAD.get(self.grad, 0)
        c.blendCoeff = self.blend
        c.verbose = int(verbose)
        c.pRefCell = self.p_ref_cell
        c.pRefValue = self.p_ref_value
        c.pPrecond = self.p_precond
        return c

    def bcs(self):
        m = self.mesh
        self._ut = np.array([BC[t] for t in self.u_type], np.int32)
        self._uv = np.ascontiguousarray(np.array(self.u_value, np.float64).reshape(-1, 3))
        self._pt = np.array([BC[t] for t in self.p_type], np.int32)
        self._pv = np.array(self.p_value, np.float64)
        b = Bcs(self._ut.ctypes.data_as(C.POINTER(C.c_int32)), _p(self._uv),
                self._pt.ctypes.data_as(C.POINTER(C.c_int32)), _p(self._pv), None, None)
        if self.u_face_values:
            self._fs = np.zeros(m.nF, np.uint8)
            self._fv = np.zeros((m.nF, 3))
            for f, v in self.u_face_values.items():
                self._fs[f] = 1
                self._fv[f] = v
            b.uFaceSet = self._fs.ctypes.data_as(C.POINTER(C.c_uint8))
            b.uFaceValue = _p(self._fv)
        return b

    def initial_flux(self, U):
        phi = np.zeros(self.mesh.nF)
        b = self.bcs()
        _check(lib().cfo_flux_from_U(C.byref(self.mesh._c), C.byref(b), _p(np.ascontiguousarray(U)), _p(phi)))
        return phi

    def run(self, U=None, p=None, phi=None, verbose=False):
        m = self.mesh
        U = np.zeros((m.nC, 3)) if U is None else np.array(U, np.float64, copy=True)
        p = np.zeros(m.nC) if p is None else np.array(p, np.float64, copy=True)
        phi = self.initial_flux(U) if phi is None else np.array(phi, np.float64, copy=True)
        res = Result()
        b = self.bcs()
        ctl = self.controls(verbose)
        _check(lib().cfo_simple(C.byref(m._c), C.byref(b), C.byref(ctl), _p(U), _p(p), _p(phi), C.byref(res)))
        return U, p, phi, res

    def pressure_csr(self, rAUf):
        m = self.mesh
        rs = np.zeros(m.nC + 1, np.int64)
        cols = np.zeros(m.nC + 2 * m.nInt, np.int64)
        vals = np.zeros(m.nC + 2 * m.nInt)
        b = self.bcs()
        ctl = self.controls()
        lib().cfo_pressure_csr.restype = C.c_int64
        nnz = lib().cfo_pressure_csr(C.byref(m._c), C.byref(b), C.byref(ctl),
                                     _p(np.ascontiguousarray(rAUf, np.float64)), _p(rs, _i64p), _p(cols, _i64p),
                                     _p(vals))
        if nnz < 0:
            raise RuntimeError(lib().cfo_last_error().decode())
        return rs, cols[:nnz].copy(), vals[:nnz].copy()

    def eqns(self, U, p, phi, xprobe):
        m = self.mesh
        nC, nF = m.nC, m.nF
        out = {k: np.zeros(s) for k, s in [("gradPn", (nC, 3)), ("U_diag", (3, nC)), ("U_h0", (3, nC)),
                                             ("U_h1", (3, nC)), ("rAUf", nF), ("divPhi", nC), ("contErr", 1),
                                             ("p_diag", nC), ("p_h0", nC), ("p_h1", nC),
                                             ("gradPFull", (nC, 3)), ("phiCorrected", nF)]}
        b = self.bcs()
        ctl = self.controls()
        arr = lambda a: _p(np.ascontiguousarray(a, dtype=np.float64))
        _check(lib().cfo_eqns(C.byref(m._c), C.byref(b), C.byref(ctl), arr(U), arr(p), arr(phi), arr(xprobe),
                              *[_p(out[k]) for k in ("gradPn", "U_diag", "U_h0", "U_h1", "rAUf", "divPhi",
                                                     "contErr", "p_diag", "p_h0", "p_h1", "gradPFull",
                                                     "phiCorrected")]))
        return out


def csr_from_triplets(n, rows, cols, vals, diag):
    rows = np.ascontiguousarray(rows, np.int64)
    cols = np.ascontiguousarray(cols, np.int64)
    vals = np.ascontiguousarray(vals, np.float64)
    diag = np.ascontiguousarray(diag, np.float64)
    rs = np.zeros(n + 1, np.int64)
    oc = np.zeros(rows.size + n, np.int64)
    ov = np.zeros(rows.size + n, np.float64)
    nnz = lib().cfo_csr_build(C.c_int64(n), C.c_int64(rows.size), _p(rows, _i64p), _p(cols, _i64p), _p(vals),
                              _p(diag), _p(rs, _i64p), _p(oc, _i64p), _p(ov))
    return rs, oc[:nnz].copy(), ov[:nnz].copy()


def solve(method, rs, cols, vals, b, x0, tol, max_iter):
    x = np.array(x0, np.float64, copy=True)
    rep = Report()
    fn = {"cg": lib().cfo_solve_cg, "bicgstab": lib().cfo_solve_bicgstab, "dic": lib().cfo_solve_dic_cg}[method]
    _check(fn(C.c_int64(rs.size - 1), _p(rs, _i64p), _p(cols, _i64p), _p(vals),
              _p(np.ascontiguousarray(b, np.float64)), _p(x), C.c_double(tol), C.c_int32(max_iter), C.byref(rep)))
    return x, rep


def dic(rs, cols, vals):
    """Colouring and DIC factor of a CSR matrix; returns (colour, nColours, rDinv, apply)."""
    rs = np.ascontiguousarray(rs, np.int64)
    cols = np.ascontiguousarray(cols, np.int64)
    vals = np.ascontiguousarray(vals, np.float64)
    n = rs.size - 1
    colour = np.zeros(n, np.int32)
    nc = lib().cfo_colour_cells(C.c_int64(n), _p(rs, _i64p), _p(cols, _i64p), colour.ctypes.data_as(C.POINTER(C.c_int32)))
    rDinv = np.zeros(n)
    lib().cfo_dic_factor(C.c_int64(n), _p(rs, _i64p), _p(cols, _i64p), _p(vals),
                         colour.ctypes.data_as(C.POINTER(C.c_int32)), C.c_int32(nc), _p(rDinv))

    def apply(r):
        r = np.ascontiguousarray(r, np.float64)
        z = np.zeros(n)
        lib().cfo_dic_apply(C.c_int64(n), _p(rs, _i64p), _p(cols, _i64p), _p(vals),
                            colour.ctypes.data_as(C.POINTER(C.c_int32)), C.c_int32(nc), _p(rDinv), _p(r), _p(z))
        return z
    return colour, nc, rDinv, apply


# --------------------------------------------------------------------------
# reference driver (oracle/_ref/cf_ref_driver, built from the reference's own
# sources by oracle/Makefile)
# --------------------------------------------------------------------------

def cell_order(n_cells, owner, neighbour, mode):
    """The restated device cell numbering (new -> old); mode 0..3 =
    identity, colour, rcm, rcm-colour."""
    own = np.ascontiguousarray(owner, np.int64)
    nbr = np.ascontiguousarray(neighbour, np.int64)
    out = np.zeros(n_cells, np.int64)
    _check(lib().cfo_cell_order(C.c_int64(n_cells), C.c_int64(nbr.size), _p(own, _i64p), _p(nbr, _i64p),
                                C.c_int32(mode), _p(out, _i64p)))
    return out


def have_ref():
    return os.path.exists(REF_DRIVER)


def ref_run(args, cwd=None, timeout=3600):
    r = subprocess.run([REF_DRIVER] + [str(a) for a in args], capture_output=True, text=True, cwd=cwd,
                       timeout=timeout)
    if r.returncode != 0:
        raise RuntimeError(f"cf_ref_driver {args[0]} failed: {r.stderr.strip()}")
    return r.stdout


def read(path, dtype=np.float64, shape=None):
    a = np.fromfile(path, dtype=dtype)
    return a.reshape(shape) if shape is not None else a


def ref_mesh(case_dict_path, points=None):
    """Addressing and geometry as the reference computes them."""
    with tempfile.TemporaryDirectory() as td:
        args = ["mesh", case_dict_path, td]
        if points is not None:
            pp = os.path.join(td, "points_in.f64")
            np.ascontiguousarray(points, np.float64).tofile(pp)
            args.append(pp)
        ref_run(args)
        counts = [int(x) for x in open(os.path.join(td, "counts.txt")).read().split()]
        out = {"counts": counts}
        out["patches"] = [ln.split() for ln in open(os.path.join(td, "patches.txt")).read().splitlines()]
        for k in ("points", "C", "Cf", "Sf", "d", "skew"):
            out[k] = read(os.path.join(td, k + ".f64"), shape=(-1, 3))
        for k in ("V", "magSf", "invDist", "ow", "gammaHarm"):
            out[k] = read(os.path.join(td, k + ".f64"))
        for k in ("face_offsets", "face_verts", "owner", "neighbour"):
            out[k] = read(os.path.join(td, k + ".i64"), np.int64)
        return out
