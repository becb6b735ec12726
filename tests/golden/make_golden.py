"""Generates the golden fixtures in this directory by running the reference
itself: oracle/_ref/cf_ref_driver, which oracle/Makefile compiles from the
reference's own sources.  Run here, where the reference tree is present:

    make -C oracle && python tests/golden/make_golden.py

Fixtures (small .npz files):
  mesh_block_2x2x2.npz     BlockMesh 2x2x2 unit cube: addressing + geometry
  mesh_tets22.npz          the reference's skewed tet cube (tests/meshes/cubeTets_22.msh)
                           through its gmsh reader: addressing, geometry, weights,
                           and fvc::grad of its two test fields under all schemes
  mesh_hex41.npz           the orthogonal hex cube (tests/meshes/cubeHex_41.msh), same
  mesh_groups.npz          a 3^3 hex box with physical surface groups (one written as triangles),
                           read by the reference's gmsh reader with patch types from the case
  mesh_delaunay.npz        a seeded Delaunay tetrahedralisation (chuanflow_b200.meshgen) written
                           as gmsh 2.2 and read by the reference's gmsh reader
  simple_cavity.npz        jittered 6x5x4 lid-driven cavity: 3 SIMPLE iterations
  simple_channel.npz       10x6x5 inlet/outlet channel: 4 SIMPLE iterations
  eqns_cavity.npz          the assembly probes of one outer iteration (eqns mode)
  solve_cg.npz, solve_bicgstab.npz   one CSR solve each
  piso_channel.npz         16x6x6 jittered channel: 4 transient PISO steps (dt 0.05, 2 correctors)
  simple_channel40.npz     the 16,000-cell channel: all 300 reference iterations, and 20 with
                           linear-upwind, Gauss linear and DIC-PCG by the C restatement (checksums, samples)
  simple_channel_dt.npz    the 10x6x5 channel by the reference's SIMPLE with its time term (dt 0.05,
                           uTimeOld the velocity each call starts from): six one-sweep calls
  poiseuille.npz           the reference's verification channel (100x20x1, K.poiseuille_dict) run by the
                           reference to its own outer stop: iterations and the whole U, p, phi
  simple_cavity128.npz     the 2M-cell bench cavity (pinned, so by the C restatement): checksums and
                           4096 seeded cell/face samples after one outer iteration
  vtk_cavity.npz           the reference's VtkWriter output (ASCII .vtu) of a jittered 3x3x2 cavity
                           with random p and U
  rans_channel.npz         12x5x5 orthogonal channel at Re_H 2e4 with the reference's k-epsilon:
                           5 SIMPLE iterations (U, p, phi, k, epsilon, nut, nu + nut on faces)
  coupled_laminar.npz      the reference's solveCoupled1d3d over three laminar DetailBlocks in
                           parallel (oracle/_ref/cf_coupled_driver): per pass and edge q, drop,
                           coefficient, sweeps
  coupled_kepsilon.npz     the same with the third block a k-epsilon duct
  rans_sst.npz, rans_des.npz, rans_transition.npz   the rans_channel case with the reference's
                           k-omega SST, DES and gamma-transition models
  piso_rans_keps.npz, piso_rans_sst.npz   the same channel stepped by the reference's PISO
                           (4 steps, dt 0.05) with k-epsilon and with k-omega SST

`python tests/golden/make_golden.py coupled` (or `rans`, `channel40`, `poiseuille`) rebuilds
only the coupled (or the three extra RANS, the 16,000-cell channel, the verification channel)
fixtures.
"""
import os
import subprocess
import sys
import tempfile

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(os.path.dirname(HERE))
sys.path.insert(0, os.path.join(ROOT, "tests"))
import _oracle as O  # noqa: E402
import _cases as K  # noqa: E402

# the reference source tree this script reads the reference's test meshes from
REF_MESHES = os.path.join(os.environ.get("CHUANFLOW_REFERENCE", "/root/reference"), "tests", "meshes")


def mesh_npz(name, case_text, points=None, grad_fields=False):
    with tempfile.TemporaryDirectory() as td:
        cp = os.path.join(td, "case.dict")
        open(cp, "w").write(case_text)
        r = O.ref_mesh(cp, points)
        out = {k: v for k, v in r.items() if k not in ("counts", "patches")}
        out["counts"] = np.array(r["counts"], np.int64)
        out["patch_names"] = np.array([p[0] for p in r["patches"]])
        out["patch_types"] = np.array([p[1] for p in r["patches"]])
        out["patch_start"] = np.array([int(p[2]) for p in r["patches"]], np.int64)
        out["patch_size"] = np.array([int(p[3]) for p in r["patches"]], np.int64)
        if grad_fields:
            C, Cf = r["C"], r["Cf"]
            nInt = r["neighbour"].size
            for fname, coef in K.POLY_FIELDS.items():
                t = K.poly(coef, C)
                b = K.poly(coef, Cf[nInt:])
                tp = os.path.join(td, "t.f64")
                bp = os.path.join(td, "b.f64")
                t.tofile(tp)
                b.tofile(bp)
                O.ref_run(["grad", cp, td, "-", tp, bp])
                out[f"T_{fname}"] = t
                out[f"B_{fname}"] = b
                for s in ("linear", "corrected", "leastSquares"):
                    out[f"grad_fn_{s}_{fname}"] = O.read(os.path.join(td, f"grad_fn_{s}.f64"), shape=(-1, 3))
                    out[f"grad_vol_{s}_{fname}"] = O.read(os.path.join(td, f"grad_vol_{s}.f64"), shape=(-1, 3))
        np.savez_compressed(os.path.join(HERE, name), **out)
        print("wrote", name)


def simple_npz(name, case, iters_dict_text, points, state=None):
    with tempfile.TemporaryDirectory() as td:
        cp = os.path.join(td, "case.dict")
        open(cp, "w").write(iters_dict_text)
        pp = os.path.join(td, "points.f64")
        np.ascontiguousarray(points).tofile(pp)
        args = ["simple", cp, td, pp]
        if state is not None:
            sd = os.path.join(td, "state")
            os.makedirs(sd)
            for k, v in state.items():
                np.ascontiguousarray(v).tofile(os.path.join(sd, k + ".f64"))
            args.append(sd)
        O.ref_run(args)
        res = open(os.path.join(td, "result.txt")).read().split()
        out = {"points": points, "U": O.read(os.path.join(td, "U.f64"), shape=(-1, 3)),
               "p": O.read(os.path.join(td, "p.f64")), "phi": O.read(os.path.join(td, "phi.f64")),
               "iterations": int(res[0]), "continuity": float(res[1]), "momentum": float(res[2]),
               "converged": int(res[3]), "dict": np.array(iters_dict_text)}
        if state is not None:
            for k, v in state.items():
                out["init_" + k] = v
        np.savez_compressed(os.path.join(HERE, name), **out)
        print("wrote", name, res[:4])


def eqns_npz(name, dict_text, points, state):
    with tempfile.TemporaryDirectory() as td:
        cp = os.path.join(td, "case.dict")
        open(cp, "w").write(dict_text)
        pp = os.path.join(td, "points.f64")
        np.ascontiguousarray(points).tofile(pp)
        sd = os.path.join(td, "state")
        os.makedirs(sd)
        for k, v in state.items():
            np.ascontiguousarray(v).tofile(os.path.join(sd, k + ".f64"))
        O.ref_run(["eqns", cp, td, pp, sd])
        out = {"points": points, "dict": np.array(dict_text)}
        out.update({"in_" + k: v for k, v in state.items()})
        for k in ("gradPn", "gradPFull"):
            out[k] = O.read(os.path.join(td, k + ".f64"), shape=(-1, 3))
        for q in range(3):
            out[f"U_diag{q}"] = O.read(os.path.join(td, f"U_diag{q}.f64"))
            out[f"U_h0_{q}"] = O.read(os.path.join(td, f"U_h0_{q}.f64"))
            out[f"U_h1_{q}"] = O.read(os.path.join(td, f"U_h1_{q}.f64"))
        for k in ("rAUf", "divPhi", "contErr", "p_diag", "p_h0", "p_h1", "phiCorrected"):
            out[k] = O.read(os.path.join(td, k + ".f64"))
        np.savez_compressed(os.path.join(HERE, name), **out)
        print("wrote", name)


def rans_npz(name, text, points):
    with tempfile.TemporaryDirectory() as td:
        cp = os.path.join(td, "case.dict")
        open(cp, "w").write(text)
        pp = os.path.join(td, "points.f64")
        np.ascontiguousarray(points).tofile(pp)
        O.ref_run(["rans", cp, td, pp])
        res = open(os.path.join(td, "result.txt")).read().split()
        out = {"points": points, "dict": np.array(text), "iterations": int(res[0]),
               "U": O.read(os.path.join(td, "U.f64"), shape=(-1, 3))}
        for k in ("p", "phi", "k", "eps", "nut", "nuEffFace", "wallUTau", "wallYPlus"):
            out[k] = O.read(os.path.join(td, k + ".f64"))
        np.savez_compressed(os.path.join(HERE, name), **out)
        print("wrote", name, res[:4])


def piso_npz(name, text, points):
    with tempfile.TemporaryDirectory() as td:
        cp = os.path.join(td, "case.dict")
        open(cp, "w").write(text)
        pp = os.path.join(td, "points.f64")
        np.ascontiguousarray(points).tofile(pp)
        O.ref_run(["piso", cp, td, pp])
        steps = np.loadtxt(os.path.join(td, "result.txt"), ndmin=2)
        out = {"points": points, "dict": np.array(text), "steps": steps,
               "U": O.read(os.path.join(td, "U.f64"), shape=(-1, 3)), "p": O.read(os.path.join(td, "p.f64")),
               "phi": O.read(os.path.join(td, "phi.f64"))}
        for k in ("k", "eps", "nut", "nuEffFace"):  # a case with a RANS model
            if os.path.exists(os.path.join(td, k + ".f64")):
                out[k] = O.read(os.path.join(td, k + ".f64"))
        np.savez_compressed(os.path.join(HERE, name), **out)
        print("wrote", name, steps[-1])


def vtk_npz(name, case_text, points, p, U):
    with tempfile.TemporaryDirectory() as td:
        cp = os.path.join(td, "case.dict")
        open(cp, "w").write(case_text)
        pp = os.path.join(td, "points.f64")
        if points is None:
            pp = "-"
        else:
            np.ascontiguousarray(points).tofile(pp)
        np.ascontiguousarray(p).tofile(os.path.join(td, "p.f64"))
        np.ascontiguousarray(U).tofile(os.path.join(td, "U.f64"))
        out = os.path.join(td, "out.vtu")
        O.ref_run(["vtk", cp, out, pp, os.path.join(td, "p.f64"), os.path.join(td, "U.f64")])
        data = np.frombuffer(open(out, "rb").read(), np.uint8)
        np.savez_compressed(os.path.join(HERE, name), text=data, p=p, U=U,
                            points=np.zeros((0, 3)) if points is None else points, dict=np.array(case_text))
        print("wrote", name, data.size, "bytes")


def cavity128_npz(name, n=128, iters=1, linear_tol=1e-11):
    """The 2M-cell jittered cavity of bench.py (pressure reference cell 0,
    which the reference lacks, so the oracle's C restatement runs it), its
    linear solves tightened to 1e-11 so that where the two codes' solves stop
    (a 2M-term reduction crossing the tolerance) moves the fields far less
    than the 1e-6 bar: the scalar results, field checksums and 4096 seeded
    cell and face samples after `iters` outer iterations from rest."""
    m = K._block((0, 0, 0), (1, 1, 1), (n, n, n), K.CAVITY_NAMES, ["wall"] * 6, 0.1, 7)
    case = O.Case(m, u_type=["fixedValue"] * 6,
                  u_value=[(1.0, 0, 0) if nm == "lid" else (0, 0, 0) for nm in m.patch_names],
                  p_type=["zeroGradient"] * 6, p_value=[0] * 6, nu=1.0 / 400.0, max_iterations=iters,
                  linear_tol=linear_tol, non_orth=1, relax_u=0.7, relax_p=0.3, p_relax_start=0.02)
    case.p_ref_cell = 0
    U, p, phi, r = case.run()
    rng = np.random.default_rng(2024)
    cells = np.sort(rng.choice(m.nC, 4096, replace=False))
    faces = np.sort(rng.choice(m.nF, 4096, replace=False))
    np.savez_compressed(os.path.join(HERE, name), n=n, iters=iters, linear_tol=linear_tol, iterations=r.iterations,
                        continuity=r.finalContinuityError, momentum=r.finalMomentumResidual,
                        u_inner=r.uItersTotal, p_inner=r.pItersTotal, U_sum=U.sum(0), p_sum=p.sum(),
                        phi_abs_sum=np.abs(phi).sum(), cells=cells, faces=faces, U_cells=U[cells],
                        p_cells=p[cells], phi_faces=phi[faces], points_sum=m.points.sum(0))
    print("wrote", name, r.iterations, r.uItersTotal, r.pItersTotal)


def channel40_npz(name, iters=300, lu_iters=20):
    """The 40x20x20 channel (2 x 0.1 x 0.1 m, inlet 0.1 m/s, nu 1e-4, the
    reference's stable relaxation 0.9 / 0.03 / pRelaxStart 0.02, nonOrth 2):
    the reference's own run of all 300 outer iterations, checksums and seeded
    samples; and lu_iters iterations of the same case with linear-upwind
    convection, Gauss linear gradients and DIC-PCG by the C restatement (no
    reference counterpart)."""
    text = K.channel_dict(40, 20, 20, nu=1e-4, iters=iters, L=(2.0, 0.1, 0.1))
    m = K._block((0, 0, 0), (2.0, 0.1, 0.1), (40, 20, 20), K.CHANNEL_NAMES, K.CHANNEL_TYPES, 0.0, 0)
    rng = np.random.default_rng(40)
    cells = np.sort(rng.choice(m.nC, 2048, replace=False))
    faces = np.sort(rng.choice(m.nF, 2048, replace=False))
    out = {"cells": cells, "faces": faces, "iters": iters, "lu_iters": lu_iters}
    with tempfile.TemporaryDirectory() as td:
        cp = os.path.join(td, "case.dict")
        open(cp, "w").write(text)
        O.ref_run(["simple", cp, td])
        res = open(os.path.join(td, "result.txt")).read().split()
        U = O.read(os.path.join(td, "U.f64"), shape=(-1, 3))
        p = O.read(os.path.join(td, "p.f64"))
        phi = O.read(os.path.join(td, "phi.f64"))
    out.update(ref_iterations=int(res[0]), ref_continuity=float(res[1]), ref_U_sum=U.sum(0), ref_p_sum=p.sum(),
               ref_U_cells=U[cells], ref_p_cells=p[cells], ref_phi_faces=phi[faces])
    c = O.Case(m, u_type=["fixedValue", "zeroGradient"] + ["fixedValue"] * 4,
               u_value=[(0.1, 0, 0)] + [(0, 0, 0)] * 5, p_type=["zeroGradient", "fixedValue"] + ["zeroGradient"] * 4,
               p_value=[0] * 6, nu=1e-4, max_iterations=lu_iters, linear_tol=1e-8, non_orth=2, relax_u=0.7,
               relax_p=0.3, p_relax_start=0.02, div="linearUpwind", grad="linear")
    c.p_precond = 1
    U, p, phi, r = c.run()
    out.update(lu_iterations=r.iterations, lu_continuity=r.finalContinuityError, lu_U_sum=U.sum(0),
               lu_p_sum=p.sum(), lu_U_cells=U[cells], lu_p_cells=p[cells], lu_phi_faces=phi[faces])
    np.savez_compressed(os.path.join(HERE, name), **out)
    print("wrote", name, res[:2], r.iterations)


def poiseuille_npz(name):
    """The reference's verification channel (K.poiseuille_dict) run by the
    reference to its own outer stop: iterations, convergence and the whole
    U, p, phi."""
    with tempfile.TemporaryDirectory() as td:
        cp = os.path.join(td, "case.dict")
        open(cp, "w").write(K.poiseuille_dict())
        O.ref_run(["simple", cp, td])
        res = open(os.path.join(td, "result.txt")).read().split()
        U = O.read(os.path.join(td, "U.f64"), shape=(-1, 3))
        p = O.read(os.path.join(td, "p.f64"))
        phi = O.read(os.path.join(td, "phi.f64"))
    np.savez_compressed(os.path.join(HERE, name), iterations=int(res[0]), continuity=float(res[1]),
                        momentum=float(res[2]), converged=int(res[3]), U=U, p=p, phi=phi)
    print("wrote", name, res[:4])


def pseudo_npz():
    """The reference's SIMPLE with its time term (SimpleControls::dt and
    uTimeOld, simpleSolver.cpp:75-97) on the 10x6x5 jittered channel: six
    calls of one sweep each, every call's old velocity the one it starts
    from (the driver's simple { dt } mode)."""
    ch = K.channel_case(10, 6, 5)
    text = K.channel_dict(10, 6, 5, iters=6).replace("maxIterations 6;", "maxIterations 6;\n    dt 0.05;")
    simple_npz("simple_channel_dt.npz", ch, text, ch.mesh.points)


def solve_npz(name, method, rs, cols, vals, b, x0, tol, max_iter):
    n = rs.size - 1
    rows = np.repeat(np.arange(n), np.diff(rs))
    off = rows != cols
    diag = np.zeros(n)
    diag[rows[~off]] = vals[~off]
    with tempfile.TemporaryDirectory() as td:
        trip = np.stack([rows[off], cols[off]], 1).astype(np.int64)
        trip.tofile(os.path.join(td, "t.i64"))
        vals[off].astype(np.float64).tofile(os.path.join(td, "v.f64"))
        diag.tofile(os.path.join(td, "d.f64"))
        b.tofile(os.path.join(td, "b.f64"))
        x0.tofile(os.path.join(td, "x0.f64"))
        O.ref_run(["solve", td, n, os.path.join(td, "t.i64"), os.path.join(td, "v.f64"), os.path.join(td, "d.f64"),
                   os.path.join(td, "b.f64"), os.path.join(td, "x0.f64"), method, repr(tol), max_iter])
        rep = open(os.path.join(td, "report.txt")).read().split()
        np.savez_compressed(os.path.join(HERE, name), row_start=rs, cols=cols, vals=vals, b=b, x0=x0,
                            x=O.read(os.path.join(td, "x.f64")), tol=tol, max_iter=max_iter,
                            iterations=int(rep[0]), initial=float(rep[1]), final=float(rep[2]),
                            converged=int(rep[3]))
        print("wrote", name, rep[:4])


def coupled_npz(name, text):
    """solveCoupled1d3d with the reference's DetailBlock partners."""
    drv = os.path.join(ROOT, "oracle", "_ref", "cf_coupled_driver")
    with tempfile.TemporaryDirectory() as td:
        cp = os.path.join(td, "case.dict")
        open(cp, "w").write(text)
        subprocess.run([drv, cp, td], check=True, stdout=subprocess.DEVNULL)
        lines = open(os.path.join(td, "history.txt")).read().split("\n")
    rows = [list(map(float, ln.split())) for ln in lines if ln and not ln.startswith("result")]
    res = [ln for ln in lines if ln.startswith("result")][0].split()[1:]
    np.savez_compressed(os.path.join(HERE, name), dict=np.array(text), history=np.array(rows),
                        iterations=int(res[0]), converged=int(res[1]), residual=float(res[2]))


def rans_fixtures():
    rc = K.channel_case(12, 5, 5, L=(1.0, 0.1, 0.1), jitter=0.0)
    for model, name in (("kOmegaSST", "rans_sst"), ("des", "rans_des"), ("gammaTransition", "rans_transition")):
        rans_npz(name + ".npz", K.rans_channel_dict(model=model), rc.mesh.points)
    for model, name in (("kEpsilon", "piso_rans_keps"), ("kOmegaSST", "piso_rans_sst")):
        piso_npz(name + ".npz", K.piso_rans_dict(model), rc.mesh.points)


def coupled_fixtures():
    coupled_npz("coupled_laminar.npz", K.coupled_network_dict())
    coupled_npz("coupled_kepsilon.npz", K.coupled_network_dict(turbulent=True))


def main():
    if not O.have_ref():
        sys.exit("oracle/_ref/cf_ref_driver missing: run `make -C oracle` where the reference is present")
    if sys.argv[1:] == ["coupled"]:
        coupled_fixtures()
        return
    if sys.argv[1:] == ["rans"]:
        rans_fixtures()
        return
    if sys.argv[1:] == ["channel40"]:
        channel40_npz("simple_channel40.npz")
        return
    if sys.argv[1:] == ["poiseuille"]:
        poiseuille_npz("poiseuille.npz")
        return
    if sys.argv[1:] == ["pseudo"]:
        pseudo_npz()
        return
    mesh_npz("mesh_block_2x2x2.npz", "block { min (0 0 0); max (1 1 1); cells (2 2 2); }\n")
    mesh_npz("mesh_tets22.npz", f'mesh {{ format gmsh; file "{REF_MESHES}/cubeTets_22.msh"; }}\n', grad_fields=True)
    mesh_npz("mesh_hex41.npz", f'mesh {{ format gmsh; file "{REF_MESHES}/cubeHex_41.msh"; }}\n', grad_fields=True)

    sys.path.insert(0, ROOT)
    from chuanflow_b200 import meshgen
    pts = meshgen.jittered_lattice(6, 0.1, 5)
    tets = meshgen.delaunay_tets(pts)
    with tempfile.TemporaryDirectory() as td:
        mp = os.path.join(td, "m.msh")
        K.write_msh22(mp, pts, tets)
        mesh_npz("mesh_delaunay.npz", f'mesh {{ format gmsh; file "{mp}"; }}\n')
    d = dict(np.load(os.path.join(HERE, "mesh_delaunay.npz")))
    d["tets"] = tets
    d["lattice_points"] = pts
    np.savez_compressed(os.path.join(HERE, "mesh_delaunay.npz"), **d)

    with tempfile.TemporaryDirectory() as td:
        mp = os.path.join(td, "box.msh")
        K.grouped_box_file(mp)
        mesh_npz("mesh_groups.npz", f'mesh {{ format gmsh; file "{mp}"; patches {{ inlet {{ type inlet; }} '
                                    f'outlet {{ type outlet; }} }} }}\n')

    channel40_npz("simple_channel40.npz")
    poiseuille_npz("poiseuille.npz")
    cavity128_npz("simple_cavity128.npz")

    vc = K.cavity_case(3, 3, 2)
    rv = np.random.default_rng(4)
    vtk_npz("vtk_cavity.npz", K.cavity_dict(3, 3, 2), vc.mesh.points, rv.normal(size=vc.mesh.nC),
            rv.normal(size=(vc.mesh.nC, 3)))

    cav = K.cavity_case(6, 5, 4)
    simple_npz("simple_cavity.npz", cav, K.cavity_dict(6, 5, 4, iters=3), cav.mesh.points)
    ch = K.channel_case(10, 6, 5)
    simple_npz("simple_channel.npz", ch, K.channel_dict(10, 6, 5, iters=4), ch.mesh.points)
    pseudo_npz()

    pc = K.channel_case(16, 6, 6)
    piso_npz("piso_channel.npz", K.piso_channel_dict(), pc.mesh.points)
    rc = K.channel_case(12, 5, 5, L=(1.0, 0.1, 0.1), jitter=0.0)
    rans_npz("rans_channel.npz", K.rans_channel_dict(), rc.mesh.points)
    rans_fixtures()

    rng = np.random.default_rng(11)
    m = cav.mesh
    U = rng.normal(size=(m.nC, 3)) * 0.3
    p = rng.normal(size=m.nC)
    phi = cav.initial_flux(U) + rng.normal(size=m.nF) * 1e-3 * (np.arange(m.nF) < m.nInt)
    xprobe = rng.normal(size=m.nC)
    eqns_npz("eqns_cavity.npz", K.cavity_dict(6, 5, 4, iters=1), m.points, {"U": U, "p": p, "phi": phi,
                                                                           "xprobe": xprobe})

    # one pressure-like SPD system and one convection-diffusion system
    n = 60
    rs, cols, vals = K.test_matrix(n, rng, symmetric=True)
    b = rng.normal(size=n)
    solve_npz("solve_cg.npz", "cg", rs, cols, vals, b, np.zeros(n), 1e-10, 500)
    rs, cols, vals = K.test_matrix(n, rng, symmetric=False)
    solve_npz("solve_bicgstab.npz", "bicgstab", rs, cols, vals, b, np.zeros(n), 1e-10, 500)
    coupled_fixtures()


if __name__ == "__main__":
    main()
