"""Pins the C restatement in oracle/ (the checker of the GPU tests) to the
reference: bit-for-bit against the golden fixtures the reference produced,
and, where the reference driver is built (oracle/_ref), against fresh runs
of the reference on cases the fixtures do not cover.  CPU only."""
import os
import re
import subprocess
import tempfile

import numpy as np
import pytest

import _cases as K
import _oracle as O


def omesh_from_fixture(g):
    return O.OMesh(g["points"], g["face_offsets"], g["face_verts"], g["owner"], g["neighbour"],
                   [str(x) for x in g["patch_names"]], [str(x) for x in g["patch_types"]], g["patch_start"],
                   g["patch_size"])


@pytest.mark.parametrize("fixture", ["mesh_block_2x2x2.npz", "mesh_tets22.npz", "mesh_hex41.npz"])
def test_geometry_matches_reference(golden, fixture):
    g = golden(fixture)
    m = omesh_from_fixture(g)
    for k in ("V", "C", "Cf", "Sf", "magSf", "d", "invDist"):
        assert np.array_equal(getattr(m, k), g[k]), k
    ow = m.owner_weights()
    assert np.array_equal(ow, g["ow"])
    assert np.array_equal(m.skew(ow), g["skew"])
    assert np.array_equal(m.harmonic_gamma(1e-4), g["gammaHarm"])


def test_block_addressing_matches_reference(golden):
    g = golden("mesh_block_2x2x2.npz")
    m = O.block_mesh((0, 0, 0), (1, 1, 1), (2, 2, 2))
    for k in ("face_offsets", "face_verts", "owner", "neighbour", "points"):
        assert np.array_equal(getattr(m, k), g[k]), k
    assert list(m.patch_start) == list(g["patch_start"])


def test_reference_kernel_unit_facts(golden):
    """tests/unit/kernelTests.cpp:58-83 on the 2x2x2 block."""
    g = golden("mesh_block_2x2x2.npz")
    nP, nC, nF, nInt, nPatch = g["counts"]
    assert nC == 8 and nInt == 12 and nF - nInt == 24
    assert abs(g["V"].sum() - 1.0) < 1e-10 and abs(g["V"][0] - 0.125) < 1e-10
    sums = np.zeros((nC, 3))
    np.add.at(sums, g["owner"], g["Sf"])
    np.add.at(sums, g["neighbour"], -g["Sf"][:nInt])
    assert np.abs(sums).max() < 1e-12


@pytest.mark.parametrize("fixture", ["mesh_tets22.npz", "mesh_hex41.npz"])
def test_gradients_match_reference(golden, fixture):
    g = golden(fixture)
    m = omesh_from_fixture(g)
    for fname in K.POLY_FIELDS:
        for s in ("linear", "corrected", "leastSquares"):
            assert np.array_equal(m.grad(g[f"T_{fname}"], g[f"B_{fname}"], s), g[f"grad_fn_{s}_{fname}"])
            assert np.array_equal(m.grad(g[f"T_{fname}"], g[f"B_{fname}"], s, vol_quirk=True),
                                  g[f"grad_vol_{s}_{fname}"])


def test_reference_gradient_unit_facts(golden):
    """tests/unit/gradientTests.cpp:92-154 on the oracle's gradients."""
    g = golden("mesh_tets22.npz")
    assert int(g["counts"][1]) == 95
    m = omesh_from_fixture(g)
    ow = m.owner_weights()
    nInt = m.nInt
    co = m.C[m.owner[:nInt]]
    d = m.d[:nInt]
    expected = 1.0 - np.clip(np.einsum("ij,ij->i", m.Cf[:nInt] - co, d) / np.einsum("ij,ij->i", d, d), 0, 1)
    assert np.abs(ow[:nInt] - expected).max() < 1e-15
    assert np.abs(ow[:nInt] - 0.5).max() > 0.05

    def err(mesh, c, s):
        t = K.poly(c, mesh.C)
        b = K.poly(c, mesh.Cf[mesh.nInt:])
        e = mesh.grad(t, b, s) - K.poly_grad(c, mesh.C)
        return np.sqrt((e ** 2).sum(1)).max()

    lin, quad = K.POLY_FIELDS["lin"], K.POLY_FIELDS["quad"]
    assert err(m, lin, "corrected") < 0.5 * err(m, lin, "linear")
    assert err(m, lin, "leastSquares") < 1e-9
    assert err(m, quad, "corrected") < 0.5 * err(m, quad, "linear")
    assert err(m, quad, "leastSquares") < err(m, quad, "corrected")
    assert err(m, lin, "unheard-of") == err(m, lin, "linear")
    h = omesh_from_fixture(golden("mesh_hex41.npz"))
    assert err(h, lin, "linear") < 1e-9 and err(h, lin, "corrected") < 1e-9 and err(h, lin, "leastSquares") < 1e-9
    assert abs(err(h, quad, "corrected") - err(h, quad, "linear")) < 1e-12
    assert err(h, quad, "leastSquares") < 1e-9


@pytest.mark.parametrize("fixture,builder", [("simple_cavity.npz", "cavity"), ("simple_channel.npz", "channel")])
def test_simple_matches_reference(golden, fixture, builder):
    g = golden(fixture)
    case = K.cavity_case(6, 5, 4) if builder == "cavity" else K.channel_case(10, 6, 5)
    assert np.array_equal(case.mesh.points, g["points"])
    U, p, phi, res = case.run()
    assert res.iterations == int(g["iterations"])
    for a, k in ((U, "U"), (p, "p"), (phi, "phi")):
        assert np.array_equal(a, g[k]), k


def test_equations_match_reference(golden):
    g = golden("eqns_cavity.npz")
    case = K.cavity_case(6, 5, 4)
    out = case.eqns(g["in_U"], g["in_p"], g["in_phi"], g["in_xprobe"])
    assert np.array_equal(out["gradPn"], g["gradPn"])
    for q in range(3):
        assert np.array_equal(out["U_diag"][q], g[f"U_diag{q}"])
        assert np.array_equal(out["U_h0"][q], g[f"U_h0_{q}"])
        assert np.array_equal(out["U_h1"][q], g[f"U_h1_{q}"])
    for k in ("rAUf", "divPhi", "p_diag", "p_h0", "p_h1", "phiCorrected", "gradPFull"):
        assert np.array_equal(out[k], g[k]), k
    assert out["contErr"][0] == g["contErr"][0]


@pytest.mark.parametrize("fixture,method", [("solve_cg.npz", "cg"), ("solve_bicgstab.npz", "bicgstab")])
def test_solvers_match_reference(golden, fixture, method):
    g = golden(fixture)
    x, rep = O.solve(method, g["row_start"], g["cols"], g["vals"], g["b"], g["x0"], float(g["tol"]),
                     int(g["max_iter"]))
    assert np.array_equal(x, g["x"])
    assert rep.iterations == int(g["iterations"]) and rep.converged == int(g["converged"])


def test_csr_build_merges_duplicates():
    """finishWithDiagonal: sorted rows and columns, duplicates summed, the
    diagonal in its column slot (Matrix.cpp:56-117)."""
    rs, cols, vals = O.csr_from_triplets(3, [2, 0, 0, 1, 0], [0, 2, 2, 2, 1], [1.0, 2.0, 3.0, 4.0, 5.0],
                                         [10.0, 20.0, 30.0])
    assert list(rs) == [0, 3, 5, 7]
    assert list(cols) == [0, 1, 2, 1, 2, 0, 2]
    assert list(vals) == [10.0, 5.0, 5.0, 20.0, 4.0, 1.0, 30.0]


# ---- fresh reference runs on cases the fixtures do not cover -------------

ref = pytest.mark.skipif(not O.have_ref(), reason="reference driver not built (oracle/_ref)")


def _variant_dict(text, **repl):
    for k, v in repl.items():
        text = text.replace(k, v)
    return text


@ref
@pytest.mark.parametrize("schemes", [
    ("upwind", "corrected", "linear"),
    ("blend", "corrected", "leastSquares"),
    ("linear", "none", "corrected"),
])
def test_simple_variants_match_fresh_reference(schemes):
    div, lap, grad = schemes
    case = K.channel_case(9, 5, 4, iters=3, seed=11)
    case.div, case.laplacian, case.grad = div, lap, grad
    text = _variant_dict(K.channel_dict(9, 5, 4, iters=3),
                         **{"div upwind; laplacian corrected; grad corrected;":
                            f"div {div}; laplacian {lap}; grad {grad}; blendCoeff 0.9;"})
    with tempfile.TemporaryDirectory() as td:
        cp = os.path.join(td, "case.dict")
        open(cp, "w").write(text)
        pp = os.path.join(td, "points.f64")
        case.mesh.points.tofile(pp)
        O.ref_run(["simple", cp, td, pp])
        rU = O.read(os.path.join(td, "U.f64"), shape=(-1, 3))
        rp = O.read(os.path.join(td, "p.f64"))
    U, p, phi, res = case.run()
    assert np.array_equal(U, rU) and np.array_equal(p, rp)


@ref
def test_jitter_and_blockmesh_match_fresh_reference():
    case = K.cavity_case(7, 6, 5, seed=3)
    with tempfile.TemporaryDirectory() as td:
        cp = os.path.join(td, "case.dict")
        open(cp, "w").write(K.cavity_dict(7, 6, 5))
        r = O.ref_mesh(cp, case.mesh.points)
    for k in ("face_offsets", "face_verts", "owner", "neighbour"):
        assert np.array_equal(getattr(case.mesh, k), r[k])
    for k in ("V", "C", "Cf", "Sf", "magSf", "d", "invDist"):
        assert np.array_equal(getattr(case.mesh, k), r[k]), k


COUPLED = os.path.join(os.path.dirname(os.path.dirname(os.path.abspath(__file__))), "oracle", "_ref",
                       "cf_coupled_driver")


@pytest.mark.skipif(not os.path.exists(COUPLED), reason="oracle/_ref/cf_coupled_driver not built")
def test_coupled_fixture_matches_fresh_reference(golden):
    """The reference's coupled interface over its own DetailBlocks, rerun
    here, gives the laminar fixture's history to the last bit."""
    g = golden("coupled_laminar.npz")
    with tempfile.TemporaryDirectory() as td:
        cp = os.path.join(td, "case.dict")
        open(cp, "w").write(str(g["dict"]))
        subprocess.run([COUPLED, cp, td], check=True, stdout=subprocess.DEVNULL, timeout=300)
        lines = open(os.path.join(td, "history.txt")).read().split("\n")
    rows = np.array([list(map(float, ln.split())) for ln in lines if ln and not ln.startswith("result")])
    assert np.array_equal(rows, g["history"])


@ref
def test_large_grouped_gmsh_file_matches_fresh_reference(tmp_path):
    """A 26^3 hex box with physical groups (the outlet as triangles over its
    quad faces), large enough that the product's reader splits its rows over
    threads, read by the reference's own gmsh reader and by the product's:
    addressing, patches and geometry bit for bit."""
    cf = pytest.importorskip("chuanflow_b200")
    mp = tmp_path / "box.msh"
    K.grouped_box_file(str(mp), n=26)
    cp = tmp_path / "case.dict"
    cp.write_text(f'mesh {{ format gmsh; file "{mp}"; patches {{ inlet {{ type inlet; }} '
                  f'outlet {{ type outlet; }} }} }}\n')
    r = O.ref_mesh(str(cp))
    m = cf.PolyMesh.read_gmsh(mp, {"inlet": "inlet", "outlet": "outlet"})
    assert m.n_cells == 26 ** 3
    a, g = m.addressing(), m.geometry()
    for k in ("face_offsets", "face_verts", "owner", "points"):
        assert np.array_equal(a[k], r[k]), k
    assert np.array_equal(a["neighbour"][:m.n_internal_faces], r["neighbour"])
    for k in ("V", "C", "Cf", "Sf", "magSf", "d", "invDist"):
        assert np.array_equal(g[k], r[k]), k
    assert [(n, t, s, z) for n, t, s, z in m.patches] == [(p[0], p[1], int(p[2]), int(p[3])) for p in r["patches"]]


@ref
@pytest.mark.parametrize("fmt", ["2.2", "4.1"])
def test_large_plane_named_gmsh_file_matches_fresh_reference(tmp_path, fmt):
    """A 30^3 hex box without surface groups, node tags sparse and shuffled,
    in both formats: boundary faces named after the bounding-box planes by
    both readers alike."""
    cf = pytest.importorskip("chuanflow_b200")
    pts, hexes, _ = K.hex_box_cells(30)
    tags = np.random.default_rng(5).permutation(len(pts)) * 2 + 3
    mp = tmp_path / "box.msh"
    K.write_msh_box(str(mp), pts, hexes, tags, fmt)
    cp = tmp_path / "case.dict"
    cp.write_text(f'mesh {{ format gmsh; file "{mp}"; }}\n')
    r = O.ref_mesh(str(cp))
    m = cf.PolyMesh.read_gmsh(mp)
    a, g = m.addressing(), m.geometry()
    for k in ("face_offsets", "face_verts", "owner", "points"):
        assert np.array_equal(a[k], r[k]), k
    assert np.array_equal(a["neighbour"][:m.n_internal_faces], r["neighbour"])
    for k in ("V", "C", "Cf", "Sf", "magSf", "d", "invDist"):
        assert np.array_equal(g[k], r[k]), k
    assert [(n, t, s, z) for n, t, s, z in m.patches] == [(p[0], p[1], int(p[2]), int(p[3])) for p in r["patches"]]


@ref
def test_large_ascii_vtu_is_the_reference_writers_file(tmp_path):
    """VtkWriter's ASCII .vtu of a jittered 28^3 cavity (its polyhedra built
    on the product writer's threads), byte for byte against the reference's
    writer run here."""
    cf = pytest.importorskip("chuanflow_b200")
    n = (28, 28, 28)
    m = cf.PolyMesh.block((0, 0, 0), (1, 1, 1), n, {s: (nm, "wall") for s, nm in zip(K.SIDES, K.CAVITY_NAMES)})
    m.jitter_interior(0.1, 11)
    rng = np.random.default_rng(8)
    p, U = rng.normal(size=m.n_cells), rng.normal(size=(m.n_cells, 3))
    cp = tmp_path / "case.dict"
    cp.write_text(K.cavity_dict(*n))
    pts = tmp_path / "points.f64"
    m.addressing()["points"].tofile(pts)
    p.tofile(tmp_path / "p.f64")
    U.tofile(tmp_path / "U.f64")
    ref_out = tmp_path / "ref.vtu"
    O.ref_run(["vtk", str(cp), str(ref_out), str(pts), str(tmp_path / "p.f64"), str(tmp_path / "U.f64")])
    out = tmp_path / "a.vtu"
    m.write_vtu(out, {"p": p, "U": U}, binary=False)
    assert out.read_bytes() == ref_out.read_bytes()


_MSH_HEAD = "$MeshFormat\n2.2 0 8\n$EndMeshFormat\n"
_NODES5 = "$Nodes\n5\n1 0 0 0\n2 1 0 0\n3 0 1 0\n4 0 0 1\n5 1 1 1\n$EndNodes\n"
_TET = "1 4 2 1 1 1 2 3 4"
_MSH41_HEAD = "$MeshFormat\n4.1 0 8\n$EndMeshFormat\n"
_NODES41 = ("$Nodes\n1 4 1 4\n3 1 0 4\n1\n2\n3\n4\n0 0 0\n1 0 0\n0 1 0\n0 0 1\n$EndNodes\n")

# malformed (and a few unusual but valid) files: both readers must agree on
# the outcome, and on the message when they refuse the file
GMSH_CASES = {
    "binary": "$MeshFormat\n2.2 1 8\n$EndMeshFormat\n",
    "version": "$MeshFormat\n3.0 0 8\n$EndMeshFormat\n",
    "no_format_fields": "$MeshFormat\n2.2\n$EndMeshFormat\n",
    "no_nodes": _MSH_HEAD + "$Elements\n1\n" + _TET + "\n$EndElements\n",
    "unterminated": _MSH_HEAD + "$Nodes\n1\n1 0 0 0\n",
    "empty_nodes": _MSH_HEAD + "$Nodes\n$EndNodes\n$Elements\n1\n" + _TET + "\n$EndElements\n",
    "nodes_ran_out": _MSH_HEAD + "$Nodes\n6\n1 0 0 0\n2 1 0 0\n$EndNodes\n",
    "short_node_row": _MSH_HEAD + "$Nodes\n2\n1 0 0 0\n2 1 0\n$EndNodes\n",
    "bad_tag": _MSH_HEAD + "$Nodes\n1\nx1 0 0 0\n$EndNodes\n",
    "bad_coordinate": _MSH_HEAD + "$Nodes\n1\n1 0 abc 0\n$EndNodes\n",
    "duplicate_tag": _MSH_HEAD + "$Nodes\n3\n1 0 0 0\n2 1 0 0\n2 0 1 0\n$EndNodes\n",
    "unknown_node": _MSH_HEAD + _NODES5 + "$Elements\n1\n1 4 2 1 1 1 2 3 9\n$EndElements\n",
    "second_order": _MSH_HEAD + _NODES5 + "$Elements\n1\n1 11 2 1 1 1 2 3 4 5 1 2 3 4 5\n$EndElements\n",
    "short_element": _MSH_HEAD + _NODES5 + "$Elements\n1\n1 4 2 1 1 1 2 3\n$EndElements\n",
    "element_row": _MSH_HEAD + _NODES5 + "$Elements\n1\n1 4\n$EndElements\n",
    "pyramid": _MSH_HEAD + _NODES5 + "$Elements\n1\n1 7 2 1 1 1 2 3 4 5\n$EndElements\n",
    "repeated_node": _MSH_HEAD + _NODES5 + "$Elements\n1\n1 4 2 1 1 1 2 2 4\n$EndElements\n",
    "no_volumes": _MSH_HEAD + _NODES5 + "$Elements\n1\n1 2 2 1 1 1 2 3\n$EndElements\n",
    # a node error in row 1 and a layout error in row 2: layout comes first
    "layout_before_nodes": _MSH_HEAD + _NODES5 + "$Elements\n2\n1 4 2 1 1 1 2 3 9\n2 4 2 1 1 1 2\n$EndElements\n",
    "elements_ran_out": _MSH_HEAD + _NODES5 + "$Elements\n3\n" + _TET + "\n$EndElements\n",
    "unnamed_group": _MSH_HEAD + '$PhysicalNames\n1\n2 1 ""\n$EndPhysicalNames\n' + _NODES5,
    "group_row": _MSH_HEAD + "$PhysicalNames\n1\n2 1\n$EndPhysicalNames\n" + _NODES5,
    "one_tet": _MSH_HEAD + _NODES5 + "$Elements\n1\n" + _TET + "\n$EndElements\n",
    "two_tets_shuffled_tags": _MSH_HEAD + "$Nodes\n5\n50 0 0 0\n7 1 0 0\n30 0 1 0\n4 0 0 1\n9 1 1 1\n$EndNodes\n"
                              "$Elements\n2\n1 4 0 50 7 30 4\n2 4 0 7 30 4 9\n$EndElements\n",
    "v41_tet": _MSH41_HEAD + _NODES41 + "$Elements\n1 1 1 1\n3 1 4 1\n1 1 2 3 4\n$EndElements\n",
    "v41_untagged_width": _MSH41_HEAD + _NODES41 + "$Elements\n1 1 1 1\n3 1 4 1\n1 2 3 4\n$EndElements\n",
    "v41_width": _MSH41_HEAD + _NODES41 + "$Elements\n1 1 1 1\n3 1 4 1\n1 2 3\n$EndElements\n",
    "v41_width_changed": _MSH41_HEAD + _NODES41 + "$Elements\n1 2 1 2\n3 1 4 2\n1 1 2 3 4\n1 2 3 4\n$EndElements\n",
    "v41_count": _MSH41_HEAD + _NODES41 + "$Elements\n1 2 1 1\n3 1 4 1\n1 1 2 3 4\n$EndElements\n",
    "v41_nodes_header": _MSH41_HEAD + "$Nodes\n1 4\n$EndNodes\n",
    "v41_node_block": _MSH41_HEAD + "$Nodes\n1 4 1 4\n3 1\n$EndNodes\n",
    "v41_node_count": _MSH41_HEAD + "$Nodes\n1 5 1 5\n3 1 0 4\n1\n2\n3\n4\n0 0 0\n1 0 0\n0 1 0\n0 0 1\n$EndNodes\n",
    # a block whose tag rows are missing: its nodes take the free tags
    "v41_untagged_nodes": _MSH41_HEAD + "$Nodes\n1 4 1 4\n3 1 0 4\n0 0 0\n1 0 0\n0 1 0\n0 0 1\n$EndNodes\n"
                          "$Elements\n1 1 1 1\n3 1 4 1\n1 1 2 3 4\n$EndElements\n",
    "v41_entities": _MSH41_HEAD + "$Entities\n0 0 1 0\n1 0 0 0 1 1\n$EndEntities\n" + _NODES41,
    "v41_elements_header": _MSH41_HEAD + _NODES41 + "$Elements\n1 1\n$EndElements\n",
}


@ref
@pytest.mark.parametrize("case", sorted(GMSH_CASES))
def test_gmsh_reader_outcomes_match_reference(tmp_path, case):
    """The product's gmsh reader and the reference's own, on small malformed
    or unusual files: the same refusal message, or the same mesh."""
    cf = pytest.importorskip("chuanflow_b200")
    mp = tmp_path / "m.msh"
    mp.write_text(GMSH_CASES[case])
    cp = tmp_path / "case.dict"
    cp.write_text(f'mesh {{ format gmsh; file "{mp}"; }}\n')
    try:
        r = O.ref_mesh(str(cp))
        ref_err = None
    except RuntimeError as e:
        # cfFatal prefixes the reference's source file:line
        r, ref_err = None, re.sub(r"^\S+:\d+ ", "", str(e).split("cf_ref_driver: ", 1)[-1])
    try:
        m = cf.PolyMesh.read_gmsh(mp)
        err = None
    except cf.CfgError as e:
        m, err = None, str(e).split("] ", 1)[-1]
    assert (ref_err is None) == (err is None), (ref_err, err)
    if err is not None:
        assert err == ref_err
        return
    a = m.addressing()
    for k in ("face_offsets", "face_verts", "owner", "points"):
        assert np.array_equal(a[k], r[k]), k
    assert [(n, t, s, z) for n, t, s, z in m.patches] == [(p[0], p[1], int(p[2]), int(p[3])) for p in r["patches"]]


def test_poiseuille_fixture_passes_the_reference_check(golden):
    """The reference's run of its verification channel (poiseuille.npz)
    passes tests/check_poiseuille.py's bands as restated in
    _cases.poiseuille_bands, so the GPU test's bands check the same thing."""
    g = golden("poiseuille.npz")
    assert int(g["converged"]) == 1
    m = O.block_mesh((0, 0, 0), (4.0, 0.2, 0.1), (100, 20, 1))
    b = K.poiseuille_bands(m.C, g["U"])
    assert b["column"] == 20
    assert b["v_max"] < 5e-3 and b["profile_err"] < 0.012
    assert abs(b["centreline"] / 0.15 - 1.0) < 0.08 and b["flux_err"] < 0.02
