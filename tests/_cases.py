"""Case definitions shared by the tests, the fixture generator and bench.py's
parity leg: the synthetic meshes, their boundary conditions and controls, and
the analytic fields of the reference's gradient test."""
from __future__ import annotations

import numpy as np

import _oracle as O

# the linear and quadratic fields of the reference's gradient test
# (tests/unit/gradientTests.cpp: linear anchor T = 1 + 2x - y + 0.5z and the
# quadratic of tests/cases/parallelDecomposition/caseTet.dict)
POLY_FIELDS = {
    "lin": [1, 2, -1, 0.5, 0, 0, 0, 0, 0, 0],
    "quad": [1, 2, -1, 0.5, 3, -0.25, 0, 1.5, -2, 0.75],
}


def poly(c, p):
    p = np.asarray(p, np.float64)
    x, y, z = p[..., 0], p[..., 1], p[..., 2]
    return (c[0] + c[1] * x + c[2] * y + c[3] * z + c[4] * x * x + c[5] * y * y + c[6] * z * z
            + c[7] * x * y + c[8] * y * z + c[9] * z * x)


def poly_grad(c, p):
    p = np.asarray(p, np.float64)
    x, y, z = p[..., 0], p[..., 1], p[..., 2]
    return np.stack([c[1] + 2.0 * c[4] * x + c[7] * y + c[9] * z,
                     c[2] + 2.0 * c[5] * y + c[7] * x + c[8] * z,
                     c[3] + 2.0 * c[6] * z + c[8] * y + c[9] * x], -1)


_M64 = (1 << 64) - 1


def _splitmix(x):
    x = (x + 0x9E3779B97F4A7C15) & _M64
    z = x
    z = ((z ^ (z >> 30)) * 0xBF58476D1CE4E5B9) & _M64
    z = ((z ^ (z >> 27)) * 0x94D049BB133111EB) & _M64
    return z ^ (z >> 31)


def jitter_points(points, cells, mn, mx, fraction, seed):
    """The interior-point jitter of cfg_mesh_jitter_interior, restated: every
    interior point of the block moves by (2u - 1) fraction h per axis, u from
    splitmix64(seed * 0x100000001B3 ^ (3 * point + axis)) >> 11 over 2^53."""
    nx, ny, nz = cells
    pts = np.array(points, np.float64, copy=True).reshape(-1, 3)
    h = [(mx[a] - mn[a]) / float(cells[a]) for a in range(3)]
    s0 = (seed * 0x100000001B3) & _M64
    for k in range(1, nz):
        for j in range(1, ny):
            for i in range(1, nx):
                pid = i + (nx + 1) * (j + (ny + 1) * k)
                for a in range(3):
                    r = _splitmix(s0 ^ ((pid * 3 + a) & _M64))
                    u = float(r >> 11) * (1.0 / 9007199254740992.0)
                    pts[pid, a] += (u * 2.0 - 1.0) * fraction * h[a]
    return pts


SIDES = ["xmin", "xmax", "ymin", "ymax", "zmin", "zmax"]


def _block(mn, mx, cells, names, types, jitter, seed):
    m = O.block_mesh(mn, mx, cells, names, types)
    if jitter:
        m = m.with_points(jitter_points(m.points, cells, mn, mx, jitter, seed))
    return m


# ---- the lid-driven cavity (the 128^3 benchmark's family) -----------------

CAVITY_NAMES = ["left", "right", "bottom", "lid", "front", "back"]


def cavity_case(nx, ny, nz, jitter=0.1, seed=7, nu=0.01, iters=3, linear_tol=1e-10, non_orth=1):
    m = _block((0, 0, 0), (1, 1, 1), (nx, ny, nz), CAVITY_NAMES, ["wall"] * 6, jitter, seed)
    u_val = [(1.0, 0, 0) if n == "lid" else (0, 0, 0) for n in m.patch_names]
    return O.Case(m, u_type=["fixedValue"] * 6, u_value=u_val, p_type=["zeroGradient"] * 6, p_value=[0] * 6,
                  nu=nu, max_iterations=iters, linear_tol=linear_tol, non_orth=non_orth, relax_u=0.7,
                  relax_p=0.3)


def cavity_dict(nx, ny, nz, nu=0.01, iters=3, linear_tol=1e-10, non_orth=1, max_iter=2000):
    sides = "\n".join(f"    {s} {{ name {n}; type wall; }}" for s, n in zip(SIDES, CAVITY_NAMES))
    pats = "\n".join(f"    {n} {{ U ({'1' if n == 'lid' else '0'} 0 0); }}" for n in CAVITY_NAMES)
    return f"""block
{{
    min (0 0 0);
    max (1 1 1);
    cells ({nx} {ny} {nz});
{sides}
}}
nu {nu!r};
patches
{{
{pats}
}}
schemes {{ ddt steady; div upwind; laplacian corrected; grad corrected; }}
simple
{{
    maxIterations {iters};
    relaxU 0.7;
    relaxP 0.3;
    nonOrthCorrectors {non_orth};
    linearTol {linear_tol!r};
    linearMaxIter {max_iter};
}}
"""


def cavity_product(nx, ny, nz, jitter=0.1, seed=7, device=0, schemes=None, order=None):
    """The same cavity through chuanflow_b200 (mesh, BCs, initial flux)."""
    import chuanflow_b200 as cf
    mesh = cf.PolyMesh.block((0, 0, 0), (1, 1, 1), (nx, ny, nz),
                             {s: (n, "wall") for s, n in zip(SIDES, CAVITY_NAMES)})
    if jitter:
        mesh.jitter_interior(jitter, seed)
    case = cf.SimpleCase(mesh, device, schemes, order=order)
    for n in CAVITY_NAMES:
        case.set_patch_bc("U", n, "fixedValue", (1.0, 0, 0) if n == "lid" else (0, 0, 0))
        case.set_patch_bc("p", n, "zeroGradient", 0.0)
    case.init_flux()
    return mesh, case


# ---- the inlet/outlet channel (the 16,000-cell benchmark's family) --------

CHANNEL_NAMES = ["inlet", "outlet", "bottom", "top", "front", "back"]
CHANNEL_TYPES = ["inlet", "outlet", "wall", "wall", "wall", "wall"]


def channel_case(nx, ny, nz, jitter=0.1, seed=5, nu=1e-3, iters=4, linear_tol=1e-10, non_orth=2,
                 L=(1.0, 0.2, 0.2)):
    m = _block((0, 0, 0), L, (nx, ny, nz), CHANNEL_NAMES, CHANNEL_TYPES, jitter, seed)
    ut = ["fixedValue", "zeroGradient", "fixedValue", "fixedValue", "fixedValue", "fixedValue"]
    uv = [(0.1, 0, 0)] + [(0, 0, 0)] * 5
    pt = ["zeroGradient", "fixedValue"] + ["zeroGradient"] * 4
    return O.Case(m, u_type=ut, u_value=uv, p_type=pt, p_value=[0] * 6, nu=nu, max_iterations=iters,
                  linear_tol=linear_tol, non_orth=non_orth, relax_u=0.9, relax_p=0.03, p_relax_start=0.02)


def poiseuille_dict(nx=100, ny=20, length=4.0, height=0.2, depth=0.1, u_mean=0.1, nu=0.01, iters=300):
    """The reference's verification channel (tests/cases/poiseuilleChannel,
    checked by tests/check_poiseuille.py): a planar nx x ny x 1 channel,
    uniform inlet, fixed-p outlet, no-slip top and bottom, symmetry front and
    back, run to the outer stop of its simple{} settings."""
    return f"""block
{{
    min (0 0 0);
    max ({length!r} {height!r} {depth!r});
    cells ({nx} {ny} 1);
    xmin {{ name inlet; type inlet; }}
    xmax {{ name outlet; type outlet; }}
    ymin {{ name bottom; type wall; }}
    ymax {{ name top; type wall; }}
    zmin {{ name front; type symmetry; }}
    zmax {{ name back; type symmetry; }}
}}
nu {nu!r};
patches
{{
    inlet  {{ U ({u_mean!r} 0 0); UType fixedValue; pType zeroGradient; }}
    outlet {{ UType zeroGradient; p 0; pType fixedValue; }}
    bottom {{ U (0 0 0); UType fixedValue; pType zeroGradient; }}
    top    {{ U (0 0 0); UType fixedValue; pType zeroGradient; }}
}}
schemes {{ ddt steady; div upwind; laplacian corrected; grad corrected; }}
simple
{{
    maxIterations {iters};
    continuityTol 1e-6;
    pcorrTol 1e-4;
    momentumTol 1e-4;
    relaxU 0.9;
    relaxP 0.03;
    pRelaxStart 0.02;
}}
"""


def poiseuille_bands(C, U, height=0.2, u_mean=0.1, x_dev=3.0, x_col=3.5, dx=0.04):
    """check_poiseuille.py's verdict on the developed region (cell centres
    past x_dev): max |v|, the largest deviation from the parabola
    1.5 u_mean (1 - ((y - h/2) / (h/2))^2), the centreline speed, and the
    flux of the one cell column at x_col against u_mean h."""
    dev = C[:, 0] > x_dev
    y = C[dev, 1]
    exact = 1.5 * u_mean * (1.0 - ((y - height / 2) / (height / 2)) ** 2)
    col = np.abs(C[:, 0] - x_col) < 0.125 * dx
    ny = int(col.sum())
    flux = float((U[col, 0] * (height / ny)).sum())
    return {"v_max": float(np.abs(U[dev, 1]).max()), "profile_err": float(np.abs(U[dev, 0] - exact).max()),
            "centreline": float(U[dev, 0].max()), "flux_err": abs(flux / (u_mean * height) - 1.0), "column": ny}


def channel_dict(nx, ny, nz, nu=1e-3, iters=4, linear_tol=1e-10, non_orth=2, L=(1.0, 0.2, 0.2)):
    sides = "\n".join(f"    {s} {{ name {n}; type {t}; }}" for s, n, t in zip(SIDES, CHANNEL_NAMES, CHANNEL_TYPES))
    return f"""block
{{
    min (0 0 0);
    max ({L[0]!r} {L[1]!r} {L[2]!r});
    cells ({nx} {ny} {nz});
{sides}
}}
nu {nu!r};
patches
{{
    inlet  {{ U (0.1 0 0); UType fixedValue;  pType zeroGradient; }}
    outlet {{ UType zeroGradient; p 0;        pType fixedValue;   }}
    bottom {{ U (0 0 0); }}
    top    {{ U (0 0 0); }}
    front  {{ U (0 0 0); }}
    back   {{ U (0 0 0); }}
}}
schemes {{ ddt steady; div upwind; laplacian corrected; grad corrected; }}
simple
{{
    maxIterations {iters};
    relaxU 0.9;
    relaxP 0.03;
    pRelaxStart 0.02;
    nonOrthCorrectors {non_orth};
    linearTol {linear_tol!r};
}}
"""


def channel_product(nx, ny, nz, jitter=0.1, seed=5, device=0, L=(1.0, 0.2, 0.2), schemes=None):
    import chuanflow_b200 as cf
    mesh = cf.PolyMesh.block((0, 0, 0), L, (nx, ny, nz),
                             {s: (n, t) for s, n, t in zip(SIDES, CHANNEL_NAMES, CHANNEL_TYPES)})
    if jitter:
        mesh.jitter_interior(jitter, seed)
    case = cf.SimpleCase(mesh, device, schemes)
    case.set_patch_bc("U", "inlet", "fixedValue", (0.1, 0, 0))
    case.set_patch_bc("p", "inlet", "zeroGradient", 0.0)
    case.set_patch_bc("U", "outlet", "zeroGradient", (0, 0, 0))
    case.set_patch_bc("p", "outlet", "fixedValue", 0.0)
    for n in ("bottom", "top", "front", "back"):
        case.set_patch_bc("U", n, "fixedValue", (0, 0, 0))
        case.set_patch_bc("p", n, "zeroGradient", 0.0)
    case.init_flux()
    return mesh, case


def controls_from(case: O.Case, **over):
    """The product's SimpleControls for an oracle Case."""
    import chuanflow_b200 as cf
    c = cf.SimpleControls(max_iterations=case.max_iterations, continuity_tol=case.continuity_tol,
                          pcorr_tol=case.pcorr_tol, momentum_tol=case.momentum_tol, linear_tol=case.linear_tol,
                          linear_max_iter=case.linear_max_iter, non_orth_correctors=case.non_orth,
                          relax_u=case.relax_u, relax_p=case.relax_p, p_relax_start=case.p_relax_start,
                          body_force=tuple(case.body_force), nu=case.nu)
    c.p_ref_cell = case.p_ref_cell
    c.p_ref_value = case.p_ref_value
    for k, v in over.items():
        setattr(c, k, v)
    return c


def test_matrix(n, rng, symmetric):
    """A random diagonally dominant sparse matrix, CSR with sorted columns."""
    rows = {i: {} for i in range(n)}
    for i in range(n):
        for j in rng.choice(n, size=4, replace=False):
            if j == i:
                continue
            v = -rng.uniform(0.1, 1.0)
            rows[i][j] = rows[i].get(j, 0) + v
            if symmetric:
                rows[j][i] = rows[j].get(i, 0) + v
            else:
                rows[j][i] = rows[j].get(i, 0) + v * rng.uniform(0.2, 1.8)
    rs, cols, vals = [0], [], []
    for i in range(n):
        off = sum(abs(v) for v in rows[i].values())
        rows[i][i] = off + rng.uniform(0.05, 0.5)
        for j in sorted(rows[i]):
            cols.append(j)
            vals.append(rows[i][j])
        rs.append(len(cols))
    return np.array(rs, np.int64), np.array(cols, np.int64), np.array(vals, np.float64)


def write_msh22(path, points, cells, cell_type=4):
    """A gmsh 2.2 ASCII file of volume elements only (no surface groups), the
    input of the reference's GmshMesh::fromFile."""
    with open(path, "w") as f:
        f.write("$MeshFormat\n2.2 0 8\n$EndMeshFormat\n$Nodes\n%d\n" % len(points))
        for i, p in enumerate(points):
            f.write("%d %.17g %.17g %.17g\n" % (i + 1, p[0], p[1], p[2]))
        f.write("$EndNodes\n$Elements\n%d\n" % len(cells))
        for e, c in enumerate(cells):
            f.write("%d %d 2 1 1 %s\n" % (e + 1, cell_type, " ".join(str(int(v) + 1) for v in c)))
        f.write("$EndElements\n")


RANS_OPTIONS = {"kEpsilon": "", "kOmegaSST": "", "des": "C_DES 0.61; ",
                "gammaTransition": "reOnset 20000; gammaRate 4; "}


def rans_channel_dict(nx=12, ny=5, nz=5, iters=5, model="kEpsilon"):
    """The orthogonal channel at Re_H = 0.5 * 0.1 / 2.5e-6 = 2e4 with one of
    the reference's RANS models (5% intensity, the automatic length scale);
    on the jittered 5x5 section the reference's own k-epsilon diverges."""
    t = channel_dict(nx, ny, nz, nu=2.5e-6, iters=iters, non_orth=1, L=(1.0, 0.1, 0.1))
    t = t.replace("inlet  { U (0.1 0 0);", "inlet  { U (0.5 0 0);")
    return t + f"turbulence {{ model {model}; {RANS_OPTIONS[model]}intensity 0.05; relaxation 0.7; }}\n"


def rans_channel_product(nx=12, ny=5, nz=5, model="kEpsilon"):
    mesh, case = channel_product(nx, ny, nz, jitter=0.0, L=(1.0, 0.1, 0.1))
    case.set_patch_bc("U", "inlet", "fixedValue", (0.5, 0, 0))
    case.init_flux()
    case.turbulence_setup(model, intensity=0.05, length_scale=-1.0, relaxation=0.7, nu=2.5e-6, c_des=0.61,
                          re_onset=20000.0, gamma_rate=4.0)
    return mesh, case


def piso_rans_dict(model, dt=0.05, steps=4):
    """The RANS channel stepped by PISO with its model (pisoSolver.cpp:29)."""
    return rans_channel_dict(model=model, iters=1) + (
        f"piso {{ dt {dt!r}; correctors 2; nonOrthCorrectors 1; linearTol 1e-10; steps {steps}; }}\n")


def piso_channel_dict(nx=16, ny=6, nz=6, dt=0.05, steps=4):
    """The jittered channel (nu 1e-3) stepped by the reference's PISO."""
    return channel_dict(nx, ny, nz, nu=1e-3, iters=1) + (
        f"piso {{ dt {dt!r}; correctors 2; nonOrthCorrectors 1; linearTol 1e-10; steps {steps}; }}\n")


def hex_box_cells(n):
    """An n^3 hex box in the unit cube as gmsh volume elements (0-based
    nodes) plus its boundary quads grouped by side: (points, hexes, sides)."""
    g = np.linspace(0.0, 1.0, n + 1)
    X, Y, Z = np.meshgrid(g, g, g, indexing="ij")
    pts = np.stack([X.ravel(), Y.ravel(), Z.ravel()], 1)
    idx = lambda i, j, k: (i * (n + 1) + j) * (n + 1) + k
    hexes = []
    for i in range(n):
        for j in range(n):
            for k in range(n):
                hexes.append([idx(i, j, k), idx(i + 1, j, k), idx(i + 1, j + 1, k), idx(i, j + 1, k),
                              idx(i, j, k + 1), idx(i + 1, j, k + 1), idx(i + 1, j + 1, k + 1), idx(i, j + 1, k + 1)])
    sides = {"xmin": [], "xmax": [], "ymin": [], "ymax": [], "zmin": [], "zmax": []}
    for a in range(n):
        for b in range(n):
            sides["xmin"].append([idx(0, a, b), idx(0, a + 1, b), idx(0, a + 1, b + 1), idx(0, a, b + 1)])
            sides["xmax"].append([idx(n, a, b), idx(n, a + 1, b), idx(n, a + 1, b + 1), idx(n, a, b + 1)])
            sides["ymin"].append([idx(a, 0, b), idx(a + 1, 0, b), idx(a + 1, 0, b + 1), idx(a, 0, b + 1)])
            sides["ymax"].append([idx(a, n, b), idx(a + 1, n, b), idx(a + 1, n, b + 1), idx(a, n, b + 1)])
            sides["zmin"].append([idx(a, b, 0), idx(a + 1, b, 0), idx(a + 1, b + 1, 0), idx(a, b + 1, 0)])
            sides["zmax"].append([idx(a, b, n), idx(a + 1, b, n), idx(a + 1, b + 1, n), idx(a, b + 1, n)])
    return pts, np.array(hexes), sides


def write_msh_box(path, pts, hexes, tags, fmt):
    """The box as gmsh 2.2 or 4.1 ASCII, nodes written under `tags`; a
    vertex index past the points becomes a tag past the last one."""
    def tag(v):
        return int(tags[v]) if v < len(tags) else int(max(tags)) + 1 + int(v) - len(tags)

    with open(path, "w") as f:
        if fmt == "2.2":
            f.write("$MeshFormat\n2.2 0 8\n$EndMeshFormat\n$Nodes\n%d\n" % len(pts))
            f.writelines("%d %.17g %.17g %.17g\n" % (t, *p) for t, p in zip(tags, pts))
            f.write("$EndNodes\n$Elements\n%d\n" % len(hexes))
            f.writelines("%d 5 2 1 1 %s\n" % (e + 1, " ".join(str(tag(v)) for v in c)) for e, c in enumerate(hexes))
        else:
            f.write("$MeshFormat\n4.1 0 8\n$EndMeshFormat\n$Nodes\n1 %d %d %d\n3 1 0 %d\n"
                    % (len(pts), min(tags), max(tags), len(pts)))
            f.writelines("%d\n" % t for t in tags)
            f.writelines("%.17g %.17g %.17g\n" % tuple(p) for p in pts)
            f.write("$EndNodes\n$Elements\n1 %d 1 %d\n3 1 5 %d\n" % (len(hexes), len(hexes), len(hexes)))
            f.writelines("%d %s\n" % (e + 1, " ".join(str(tag(v)) for v in c)) for e, c in enumerate(hexes))
        f.write("$EndElements\n")


def write_msh22_groups(path, points, hexes, groups):
    """gmsh 2.2 ASCII with physical surface groups: groups = [(name, quads,
    as_triangles)]; a group written as triangles splits each quad in two."""
    lines = []
    for g, (name, quads, tri) in enumerate(groups):
        for q in quads:
            if tri:
                lines.append((2, g + 1, [q[0], q[1], q[2]]))
                lines.append((2, g + 1, [q[0], q[2], q[3]]))
            else:
                lines.append((3, g + 1, list(q)))
    with open(path, "w") as f:
        f.write("$MeshFormat\n2.2 0 8\n$EndMeshFormat\n$PhysicalNames\n%d\n" % (len(groups) + 1))
        for g, (name, _, _) in enumerate(groups):
            f.write('2 %d "%s"\n' % (g + 1, name))
        f.write('3 %d "fluid"\n$EndPhysicalNames\n$Nodes\n%d\n' % (len(groups) + 1, len(points)))
        for i, p in enumerate(points):
            f.write("%d %.17g %.17g %.17g\n" % (i + 1, p[0], p[1], p[2]))
        f.write("$EndNodes\n$Elements\n%d\n" % (len(lines) + len(hexes)))
        e = 0
        for t, g, nodes in lines:
            e += 1
            f.write("%d %d 2 %d %d %s\n" % (e, t, g, g, " ".join(str(int(v) + 1) for v in nodes)))
        for c in hexes:
            e += 1
            f.write("%d 5 2 %d %d %s\n" % (e, len(groups) + 1, len(groups) + 1, " ".join(str(int(v) + 1) for v in c)))
        f.write("$EndElements\n")


def grouped_box_file(path, n=3):
    """The 3^3 box with physical groups: inlet (xmin, quads), outlet (xmax,
    triangles), walls (y and z sides, quads)."""
    pts, hexes, sides = hex_box_cells(n)
    groups = [("inlet", sides["xmin"], False), ("outlet", sides["xmax"], True),
              ("walls", sides["ymin"] + sides["ymax"] + sides["zmin"] + sides["zmax"], False)]
    write_msh22_groups(path, pts, hexes, groups)


def _duct_block(L, W, H, cells):
    walls = "\n".join(f"        {s} {{ name w{k}; type wall; }}" for k, s in enumerate(("ymin", "ymax", "zmin", "zmax")))
    return (f"block\n    {{\n        min (0 0 0);\n        max ({L!r} {W!r} {H!r});\n"
            f"        cells ({cells[0]} {cells[1]} {cells[2]});\n"
            f"        xmin {{ name inlet; type inlet; }}\n        xmax {{ name outlet; type outlet; }}\n{walls}\n    }}")


def coupled_network_dict(passes=6, sweeps=60, turbulent=False):
    """The coupled-network case of oracle/coupled_driver.cpp: a rate of 2e-3
    m3/s through Src -In- J1 -{X1 || X2 || X3}- J2 -Out- Snk, every X a
    detailed duct block (three sections, the three inlet profiles) warm
    started pass after pass, `sweeps` SIMPLE iterations per lossAt.  With
    `turbulent`, X3 is a k-epsilon block at a low viscosity."""
    blocks = [("X1", (1.0, 0.1, 0.1), (24, 6, 6), 1e-4, "parabolic", ""),
              ("X2", (0.8, 0.08, 0.1), (20, 5, 6), 1e-4, "flat", ""),
              ("X3", (0.6, 0.1, 0.12), (16, 6, 7), 1e-4, "power1over7", "")]
    if turbulent:
        blocks[2] = ("X3", (1.0, 0.1, 0.1), (12, 5, 5), 2.5e-6, "flat",
                     "turbulence { model kEpsilon; intensity 0.05; relaxation 0.7; }")
    body = "\n".join(f"    {n}\n    {{\n    {_duct_block(*g, c)}\n        nu {nu!r}; rho 800; shape {sh}; "
                     f"resistance 10000;\n        {tb}\n    }}" for n, g, c, nu, sh, tb in blocks)
    return f"""network {{ qIn 0.002; pOut 100000; rho 800; mu 0.08; rIn 10000; rOut 10000; }}
coupling {{ maxOuterIterations {passes}; relax 1; tolerance 1e-9; accelerate no; }}
schemes {{ ddt steady; div upwind; laplacian corrected; grad corrected; }}
simple {{ maxIterations {sweeps}; relaxU 0.7; relaxP 0.3; pRelaxStart 0.02; nonOrthCorrectors 1; linearTol 1e-10; continuityTol 1e-7; }}
blocks
{{
{body}
}}
"""
