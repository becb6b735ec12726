"""The product's host-side mesh (libchuanflow_b200.so, no device needed):
blockMesh addressing, geometry, weights and the interior jitter, bit-for-bit
against the reference (fixtures) and the oracle, plus the reference's mesh
errors.  CPU only."""
import os

import numpy as np
import pytest

import _cases as K
import _oracle as O

cf = pytest.importorskip("chuanflow_b200")


def check_same(mesh, om):
    a = mesh.addressing()
    g = mesh.geometry()
    for k in ("face_offsets", "face_verts", "owner", "neighbour", "points"):
        assert np.array_equal(a[k], getattr(om, k)), k
    for k in ("V", "C", "Cf", "Sf", "magSf", "d", "invDist"):
        assert np.array_equal(g[k], getattr(om, k)), k
    ow, sk = mesh.weights()
    assert np.array_equal(ow, om.owner_weights())
    assert np.array_equal(sk, om.skew())


def test_block_matches_fixture(golden):
    g = golden("mesh_block_2x2x2.npz")
    m = cf.PolyMesh.block((0, 0, 0), (1, 1, 1), (2, 2, 2))
    assert (m.n_cells, m.n_internal_faces, m.n_boundary_faces) == (8, 12, 24)
    a = m.addressing()
    for k in ("face_offsets", "face_verts", "owner", "neighbour", "points"):
        assert np.array_equal(a[k], g[k]), k
    geo = m.geometry()
    for k in ("V", "C", "Cf", "Sf", "magSf", "d", "invDist"):
        assert np.array_equal(geo[k], g[k]), k
    assert [p[0] for p in m.patches] == ["xmin", "xmax", "ymin", "ymax", "zmin", "zmax"]
    assert [p[1] for p in m.patches] == ["wall", "wall", "wall", "wall", "symmetry", "symmetry"]


@pytest.mark.parametrize("cells,jitter", [((6, 5, 4), 0.1), ((9, 3, 7), 0.2), ((1, 1, 1), 0.0), ((12, 1, 3), 0.1)])
def test_block_and_jitter_match_oracle(cells, jitter):
    mn, mx = (0.0, -1.0, 0.5), (2.0, 0.5, 1.25)
    mesh = cf.PolyMesh.block(mn, mx, cells, {s: (n, "wall") for s, n in zip(K.SIDES, K.CAVITY_NAMES)})
    om = O.block_mesh(mn, mx, cells, K.CAVITY_NAMES, ["wall"] * 6)
    if jitter:
        mesh.jitter_interior(jitter, 99)
        om = om.with_points(K.jitter_points(om.points, cells, mn, mx, jitter, 99))
    check_same(mesh, om)


@pytest.mark.parametrize("fixture", ["mesh_tets22.npz", "mesh_hex41.npz"])
def test_general_mesh_geometry_matches_reference(golden, fixture):
    g = golden(fixture)
    pats = [(str(n), str(t), int(s), int(z)) for n, t, s, z in
            zip(g["patch_names"], g["patch_types"], g["patch_start"], g["patch_size"])]
    m = cf.PolyMesh(g["points"], g["face_offsets"], g["face_verts"], g["owner"], g["neighbour"], pats)
    geo = m.geometry()
    for k in ("V", "C", "Cf", "Sf", "magSf", "d", "invDist"):
        assert np.array_equal(geo[k], g[k]), k
    ow, sk = m.weights()
    assert np.array_equal(ow, g["ow"]) and np.array_equal(sk, g["skew"])


def test_move_points_recomputes_geometry():
    m = cf.PolyMesh.block((0, 0, 0), (1, 1, 1), (3, 3, 3))
    pts = m.addressing()["points"] * 2.0
    m.move_points(pts)
    assert abs(m.geometry()["V"].sum() - 8.0) < 1e-12
    with pytest.raises(cf.CfgError, match="point count changed"):
        m.move_points(pts[:-1])


def test_mesh_errors_follow_reference():
    g = cf.PolyMesh.block((0, 0, 0), (1, 1, 1), (2, 1, 1))
    a = g.addressing()
    nI = g.n_internal_faces
    ok = [(p[0], p[1], p[2], p[3]) for p in g.patches]
    bad_internal = [("a", "wall", 0, 1)] + ok
    with pytest.raises(cf.CfgError, match="covers internal face"):
        cf.PolyMesh(a["points"], a["face_offsets"], a["face_verts"], a["owner"], a["neighbour"], bad_internal)
    with pytest.raises(cf.CfgError, match="is not in any patch"):
        cf.PolyMesh(a["points"], a["face_offsets"], a["face_verts"], a["owner"], a["neighbour"], ok[1:])
    twice = ok + [("dup", "wall", ok[0][2], 1)]
    with pytest.raises(cf.CfgError, match="in two patches"):
        cf.PolyMesh(a["points"], a["face_offsets"], a["face_verts"], a["owner"], a["neighbour"], twice)
    with pytest.raises(cf.CfgError, match="cell counts must be positive"):
        cf.PolyMesh.block((0, 0, 0), (1, 1, 1), (0, 1, 1))
    assert nI == 1


def test_mesh_from_cells_matches_reference_gmsh_reader(golden):
    """The reference's gmsh reader on a Delaunay tetrahedralisation and
    cfg_mesh_from_cells on the same elements give the same polyMesh."""
    g = golden("mesh_delaunay.npz")
    tets = g["tets"]
    off = np.arange(0, 4 * tets.shape[0] + 1, 4)
    m = cf.PolyMesh.from_cells(g["lattice_points"], np.full(tets.shape[0], 4, np.int32), off, tets.ravel())
    a = m.addressing()
    for k in ("face_offsets", "face_verts", "owner", "neighbour", "points"):
        assert np.array_equal(a[k], g[k]), k
    geo = m.geometry()
    for k in ("V", "C", "Cf", "Sf", "magSf", "d", "invDist"):
        assert np.array_equal(geo[k], g[k]), k
    assert [p[0] for p in m.patches] == [str(x) for x in g["patch_names"]]


def test_mesh_from_cells_hex_and_prism():
    """A 2x1x1 hex pair and its prism split: face counts and volumes."""
    pts = np.array([[x, y, z] for z in (0, 1) for y in (0, 1) for x in (0, 1, 2)], float)
    P = lambda x, y, z: x + 3 * (y + 2 * z)
    hexes = [[P(0, 0, 0), P(1, 0, 0), P(1, 1, 0), P(0, 1, 0), P(0, 0, 1), P(1, 0, 1), P(1, 1, 1), P(0, 1, 1)],
             [P(1, 0, 0), P(2, 0, 0), P(2, 1, 0), P(1, 1, 0), P(1, 0, 1), P(2, 0, 1), P(2, 1, 1), P(1, 1, 1)]]
    m = cf.PolyMesh.from_cells(pts, [5, 5], [0, 8, 16], np.ravel(hexes))
    assert (m.n_cells, m.n_internal_faces, m.n_boundary_faces) == (2, 1, 10)
    assert np.allclose(m.geometry()["V"], 1.0)
    cube = np.array([[x, y, z] for z in (0, 1) for y in (0, 1) for x in (0, 1)], float)
    Q = lambda x, y, z: x + 2 * (y + 2 * z)
    prisms = [[Q(0, 0, 0), Q(1, 0, 0), Q(0, 1, 0), Q(0, 0, 1), Q(1, 0, 1), Q(0, 1, 1)],
              [Q(1, 0, 0), Q(1, 1, 0), Q(0, 1, 0), Q(1, 0, 1), Q(1, 1, 1), Q(0, 1, 1)]]
    m = cf.PolyMesh.from_cells(cube, [6, 6], [0, 6, 12], np.ravel(prisms))
    assert (m.n_cells, m.n_internal_faces) == (2, 1)
    assert np.allclose(m.geometry()["V"], 0.5)
    with pytest.raises(cf.CfgError, match="not tet"):
        cf.PolyMesh.from_cells(pts, [7], [0, 5], [0, 1, 2, 3, 4])


ORDERS = ("identity", "colour", "rcm", "rcm-colour")


@pytest.mark.parametrize("source", ["block", "mesh_tets22.npz", "mesh_hex41.npz", "mesh_delaunay.npz"])
def test_device_cell_order_matches_restatement(golden, source):
    """The device numbering (colour blocks, reverse Cuthill-McKee and both)
    is a permutation equal element for element to the oracle's restatement;
    colour blocks are contiguous and no two neighbours share a colour."""
    if source == "block":
        m = cf.PolyMesh.block((0, 0, 0), (1, 1, 1), (7, 5, 4))
    else:
        g = golden(source)
        pats = [(str(n), str(t), int(s), int(z)) for n, t, s, z in
                zip(g["patch_names"], g["patch_types"], g["patch_start"], g["patch_size"])]
        m = cf.PolyMesh(g["points"], g["face_offsets"], g["face_verts"], g["owner"], g["neighbour"], pats)
    a = m.addressing()
    for mode, name in enumerate(ORDERS):
        got = m.device_order(name)
        assert np.array_equal(np.sort(got), np.arange(m.n_cells)), name
        assert np.array_equal(got, O.cell_order(m.n_cells, a["owner"], a["neighbour"], mode)), name
    # colours along the colour-block order: non-decreasing, proper
    own, nbr = a["owner"][:m.n_internal_faces], a["neighbour"]
    col = np.full(m.n_cells, -1)
    for c in range(m.n_cells):
        used = {col[x] for x in np.concatenate([nbr[own == c], own[nbr == c]]) if col[x] >= 0}
        k = 0
        while k in used:
            k += 1
        col[c] = k
    assert np.all(col[own] != col[nbr])
    blocks = col[m.device_order("colour")]
    assert np.all(np.diff(blocks) >= 0)


def test_rcm_reduces_bandwidth_of_shuffled_mesh(golden):
    """Reverse Cuthill-McKee on the Delaunay mesh (cells in qhull's order)
    shrinks the matrix bandwidth max|i - j| over neighbour pairs."""
    g = golden("mesh_delaunay.npz")
    own, nbr = g["owner"][:g["neighbour"].size], g["neighbour"]
    n = int(max(own.max(), nbr.max())) + 1
    perm = O.cell_order(n, own, nbr, 2)
    inv = np.empty(n, np.int64)
    inv[perm] = np.arange(n)
    assert np.abs(inv[own] - inv[nbr]).max() < np.abs(own - nbr).max()


def _reference_tree():
    """The reference source tree: CHUANFLOW_REFERENCE, else the one
    oracle/Makefile built its driver from (oracle/_ref/REFERENCE_PATH);
    empty when neither is there, and the tests that need it skip."""
    env = os.environ.get("CHUANFLOW_REFERENCE")
    if env:
        return env
    rec = os.path.join(os.path.dirname(os.path.dirname(os.path.abspath(__file__))), "oracle", "_ref",
                       "REFERENCE_PATH")
    return open(rec).read().strip() if os.path.exists(rec) else ""


REF_MESHES = os.path.join(_reference_tree(), "tests", "meshes") if _reference_tree() else ""


def check_fixture(m, g):
    a = m.addressing()
    for k in ("face_offsets", "face_verts", "owner", "neighbour", "points"):
        assert np.array_equal(a[k], g[k]), k
    geo = m.geometry()
    for k in ("V", "C", "Cf", "Sf", "magSf", "d", "invDist"):
        assert np.array_equal(geo[k], g[k]), k
    pats = [(str(n), str(t), int(s), int(z)) for n, t, s, z in
            zip(g["patch_names"], g["patch_types"], g["patch_start"], g["patch_size"])]
    assert m.patches == pats


def test_read_gmsh_physical_groups_match_reference(golden, tmp_path):
    """Physical surface groups (one written as triangles over quad faces)
    and patch types, against the reference's GmshMesh::fromFile."""
    p = tmp_path / "box.msh"
    K.grouped_box_file(str(p))
    m = cf.PolyMesh.read_gmsh(p, {"inlet": "inlet", "outlet": "outlet"})
    check_fixture(m, golden("mesh_groups.npz"))


def test_read_gmsh_delaunay_matches_reference(golden, tmp_path):
    g = golden("mesh_delaunay.npz")
    p = tmp_path / "d.msh"
    K.write_msh22(str(p), g["lattice_points"], g["tets"])
    check_fixture(cf.PolyMesh.read_gmsh(p), g)


@pytest.mark.skipif(not os.path.isdir(REF_MESHES), reason="the reference's test meshes are not present")
@pytest.mark.parametrize("name,fixture", [("cubeTets_22.msh", "mesh_tets22.npz"), ("cubeHex_41.msh", "mesh_hex41.npz")])
def test_read_gmsh_reference_test_meshes(golden, name, fixture):
    """The reference's own .msh test files (formats 2.2 and 4.1), read here
    where they are present, against its reader's output."""
    check_fixture(cf.PolyMesh.read_gmsh(os.path.join(REF_MESHES, name)), golden(fixture))


def test_read_gmsh_errors(tmp_path):
    with pytest.raises(cf.CfgError, match="cannot open"):
        cf.PolyMesh.read_gmsh(tmp_path / "missing.msh")
    p = tmp_path / "bin.msh"
    p.write_text("$MeshFormat\n2.2 1 8\n$EndMeshFormat\n")
    with pytest.raises(cf.CfgError, match="binary"):
        cf.PolyMesh.read_gmsh(p)
    p.write_text("$MeshFormat\n2.2 0 8\n$EndMeshFormat\n$Nodes\n5\n1 0 0 0\n2 1 0 0\n3 0 1 0\n4 0 0 1\n5 1 1 1\n"
                 "$EndNodes\n$Elements\n1\n1 7 2 1 1 1 2 3 4 5\n$EndElements\n")
    with pytest.raises(cf.CfgError, match="pyramid"):
        cf.PolyMesh.read_gmsh(p)
    p.write_text("$MeshFormat\n2.2 0 8\n$EndMeshFormat\n$Nodes\n1\n1 0 0 0\n$EndNodes\n$Elements\n1\n"
                 "1 4 2 1 1 1 2 3 4\n$EndElements\n")
    with pytest.raises(cf.CfgError, match="node 2"):
        cf.PolyMesh.read_gmsh(p)


def test_vtu_ascii_is_the_reference_writers_file(golden, tmp_path):
    """VtkWriter's ASCII .vtu (polyhedra, face stream, p and U), byte for byte."""
    g = golden("vtk_cavity.npz")
    m = cf.PolyMesh.block((0, 0, 0), (1, 1, 1), (3, 3, 2), {s: (n, "wall") for s, n in zip(K.SIDES, K.CAVITY_NAMES)})
    m.jitter_interior(0.1, 7)
    assert np.array_equal(m.addressing()["points"], g["points"])
    out = tmp_path / "a.vtu"
    m.write_vtu(out, {"p": g["p"], "U": g["U"]}, binary=False)
    assert out.read_bytes() == g["text"].tobytes()


def test_vtu_binary_holds_the_same_arrays(golden, tmp_path):
    """The appended binary form: the same points, connectivity, offsets,
    face stream and fields, read back raw."""
    g = golden("vtk_cavity.npz")
    m = cf.PolyMesh.block((0, 0, 0), (1, 1, 1), (3, 3, 2), {s: (n, "wall") for s, n in zip(K.SIDES, K.CAVITY_NAMES)})
    m.jitter_interior(0.1, 7)
    out = tmp_path / "b.vtu"
    m.write_vtu(out, {"p": g["p"], "U": g["U"]}, binary=True)
    raw = out.read_bytes()
    head, data = raw.split(b'<AppendedData encoding="raw">\n_', 1)
    import re
    arrays = {}
    for mt in re.finditer(rb'<DataArray type="(\w+)"(?: Name="(\w+)")?[^>]*offset="(\d+)"', head):
        typ, name, off = mt.group(1).decode(), (mt.group(2) or b"points").decode(), int(mt.group(3))
        nbytes = int(np.frombuffer(data[off:off + 8], np.uint64)[0])
        dt = {"Float64": np.float64, "Int64": np.int64, "UInt8": np.uint8}[typ]
        arrays[name] = np.frombuffer(data[off + 8:off + 8 + nbytes], dt)
    assert np.array_equal(arrays["points"].reshape(-1, 3), g["points"])
    assert np.array_equal(arrays["p"], g["p"]) and np.array_equal(arrays["U"].reshape(-1, 3), g["U"])
    text = g["text"].tobytes().decode()
    conn = re.search(r'Name="connectivity" format="ascii">\n(.*?)</DataArray>', text, re.S).group(1).split()
    assert np.array_equal(arrays["connectivity"], np.array(conn, np.int64))
    faces = re.search(r'Name="faces" format="ascii">\n(.*?)</DataArray>', text, re.S).group(1).split()
    assert np.array_equal(arrays["faces"], np.array(faces, np.int64))
    assert np.all(arrays["types"] == 42) and arrays["types"].size == m.n_cells


def _hex_box_rows(n):
    """An n^3 hex box as (points, 0-based hexes) in node order."""
    pts, hexes, _ = K.hex_box_cells(n)
    return pts, hexes


@pytest.mark.parametrize("fmt", ["2.2", "4.1"])
@pytest.mark.parametrize("sparse_tags", [False, True])
def test_read_gmsh_large_file_is_its_cells(tmp_path, fmt, sparse_tags):
    """A file large enough for the reader's parallel row decoding (27k hexes):
    the mesh equals the one built from the same cells, with dense node tags
    and with sparse, shuffled ones."""
    pts, hexes = _hex_box_rows(30)
    tags = np.arange(1, len(pts) + 1)
    if sparse_tags:
        tags = np.random.default_rng(3).permutation(len(pts)) * 3 + 7
    p = tmp_path / "box.msh"
    K.write_msh_box(str(p), pts, hexes, tags, fmt)
    m = cf.PolyMesh.read_gmsh(p)
    # the reader renumbers nodes in ascending tag order
    order = np.argsort(tags, kind="stable")
    rank = np.empty_like(order)
    rank[order] = np.arange(len(order))
    ref = cf.PolyMesh.from_cells(pts[order], np.full(len(hexes), 5, np.int32),
                                 np.arange(len(hexes) + 1) * 8, rank[hexes].ravel())
    a, b = m.addressing(), ref.addressing()
    for k in ("face_offsets", "face_verts", "owner", "neighbour", "points"):
        assert np.array_equal(a[k], b[k]), k
    assert m.patches == ref.patches


def test_read_gmsh_reports_the_first_bad_row(tmp_path):
    """Rows decode in parallel chunks, yet the error reported is the one of
    the first bad row in file order, and a short section still reads as
    truncated."""
    pts, hexes = _hex_box_rows(30)
    tags = np.arange(1, len(pts) + 1)
    p = tmp_path / "bad.msh"

    def write(mutate, fmt="2.2"):
        h = hexes.copy()
        mutate(h)
        K.write_msh_box(str(p), pts, h, tags, fmt)

    def undefined_late(h):  # row 20000 names node len(pts) + 5 (undefined); row 26000 repeats one
        h[20000, 0] = len(pts) + 4
        h[26000, 1] = h[26000, 0]

    def repeat_early(h):
        h[3, 1] = h[3, 0]
        h[25000, 0] = len(pts) + 4

    for fmt in ("2.2", "4.1"):
        write(undefined_late, fmt)
        with pytest.raises(cf.CfgError, match="node %d," % (len(pts) + 5)):
            cf.PolyMesh.read_gmsh(p)
        write(repeat_early, fmt)
        with pytest.raises(cf.CfgError, match="repeats a node"):
            cf.PolyMesh.read_gmsh(p)
    # a declared count above the rows present
    K.write_msh_box(str(p), pts, hexes, tags, "2.2")
    text = p.read_text().replace("$Elements\n%d\n" % len(hexes), "$Elements\n%d\n" % (len(hexes) + 1))
    p.write_text(text)
    with pytest.raises(cf.CfgError, match="truncated"):
        cf.PolyMesh.read_gmsh(p)
    # a 4.1 element line of another width after the first
    K.write_msh_box(str(p), pts, hexes, tags, "4.1")
    lines = p.read_text().split("\n")
    k = lines.index("$Elements") + 3 + 17000
    lines[k] = lines[k] + " 1"
    p.write_text("\n".join(lines))
    with pytest.raises(cf.CfgError, match="inconsistent element line width"):
        cf.PolyMesh.read_gmsh(p)


def _vtu_arrays(raw):
    import re
    head, data = raw.split(b'<AppendedData encoding="raw">\n_', 1)
    arrays = {}
    for mt in re.finditer(rb'<DataArray type="(\w+)"(?: Name="(\w+)")?[^>]*offset="(\d+)"', head):
        typ, name, off = mt.group(1).decode(), (mt.group(2) or b"points").decode(), int(mt.group(3))
        nbytes = int(np.frombuffer(data[off:off + 8], np.uint64)[0])
        dt = {"Float64": np.float64, "Int64": np.int64, "UInt8": np.uint8}[typ]
        arrays[name] = np.frombuffer(data[off + 8:off + 8 + nbytes], dt)
    return arrays


def test_vtu_polyhedra_of_a_large_mesh(tmp_path):
    """Cells split over the writer's threads (32^3 cells): connectivity in
    first-visit order over each cell's ascending faces, and the face
    stream, as polyMesh::cells gives them."""
    m = cf.PolyMesh.block((0, 0, 0), (1, 1, 1), (32, 32, 32))
    m.jitter_interior(0.1, 3)
    out = tmp_path / "big.vtu"
    m.write_vtu(out, {}, binary=True)
    arr = _vtu_arrays(out.read_bytes())
    a = m.addressing()
    fo, fv, own, nbr = a["face_offsets"], a["face_verts"], a["owner"], a["neighbour"][:m.n_internal_faces]
    cells = [[] for _ in range(m.n_cells)]
    for f in range(m.n_faces):
        cells[own[f]].append(f)
        if f < m.n_internal_faces:
            cells[nbr[f]].append(f)
    conn, offs, faces, foffs = [], [], [], []
    for cf_ in cells:
        seen = []
        for f in cf_:
            for v in fv[fo[f]:fo[f + 1]]:
                if v not in seen:
                    seen.append(v)
        conn += seen
        offs.append(len(conn))
        faces.append(len(cf_))
        for f in cf_:
            faces.append(fo[f + 1] - fo[f])
            faces += list(fv[fo[f]:fo[f + 1]])
        foffs.append(len(faces))
    assert np.array_equal(arr["connectivity"], conn) and np.array_equal(arr["offsets"], offs)
    assert np.array_equal(arr["faces"], faces) and np.array_equal(arr["faceoffsets"], foffs)
