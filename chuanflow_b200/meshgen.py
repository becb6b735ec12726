"""Synthetic meshes of the study cases that the reference has no generator
for: a seeded Delaunay tetrahedralisation of a jittered lattice.

The tetrahedra come from scipy.spatial.Delaunay (library code, on the host);
the polyMesh is then built by the library exactly as the reference's gmsh
reader would build it from the same elements (cfg_mesh_from_cells)."""
from __future__ import annotations

import numpy as np


def jittered_lattice(n, jitter=0.1, seed=0, lo=(0.0, 0.0, 0.0), hi=(1.0, 1.0, 1.0)):
    """(n+1)^3 lattice points of the box, each moved by a seeded uniform
    offset in [-jitter h, jitter h) along every axis it is free to move in:
    boundary points stay on their planes (and edge points on their edges),
    which also keeps Delaunay from leaving flat tetrahedra on the faces."""
    lo = np.asarray(lo, np.float64)
    hi = np.asarray(hi, np.float64)
    g = [lo[a] + (hi[a] - lo[a]) * np.arange(n + 1) / n for a in range(3)]
    z, y, x = np.meshgrid(g[2], g[1], g[0], indexing="ij")
    pts = np.stack([x.ravel(), y.ravel(), z.ravel()], 1)
    idx = np.stack(np.meshgrid(np.arange(n + 1), np.arange(n + 1), np.arange(n + 1), indexing="ij"), -1)
    k, j, i = idx[..., 0].ravel(), idx[..., 1].ravel(), idx[..., 2].ravel()
    free = np.stack([(i > 0) & (i < n), (j > 0) & (j < n), (k > 0) & (k < n)], 1)
    h = (hi - lo) / n
    rng = np.random.default_rng(seed)
    pts += np.where(free, (rng.random(pts.shape) * 2.0 - 1.0) * jitter * h, 0.0)
    return pts


def delaunay_tets(points, min_volume_fraction=1e-9):
    """Delaunay tetrahedra of the points, positively oriented, without the
    flat ones Qhull may leave on planar boundaries."""
    from scipy.spatial import Delaunay
    tri = Delaunay(points)
    t = np.ascontiguousarray(tri.simplices, np.int64)
    p = points[t]
    vol = np.einsum("ij,ij->i", np.cross(p[:, 1] - p[:, 0], p[:, 2] - p[:, 0]), p[:, 3] - p[:, 0]) / 6.0
    flip = vol < 0
    t[flip, 0], t[flip, 1] = t[flip, 1].copy(), t[flip, 0].copy()
    keep = np.abs(vol) > min_volume_fraction * np.abs(vol).mean()
    return t[keep]


def tet_mesh(n, jitter=0.1, seed=0):
    """PolyMesh of the Delaunay tetrahedralisation of an (n+1)^3 jittered
    lattice in the unit box (about 6 n^3 cells)."""
    from ._capi import PolyMesh
    pts = jittered_lattice(n, jitter, seed)
    tets = delaunay_tets(pts)
    off = np.arange(0, 4 * tets.shape[0] + 1, 4, dtype=np.int64)
    return PolyMesh.from_cells(pts, np.full(tets.shape[0], 4, np.int32), off, tets.ravel()), pts, tets


CHANNEL_SIDES = {"xmin": ("inlet", "inlet"), "xmax": ("outlet", "outlet"), "ymin": ("bottom", "wall"),
                 "ymax": ("top", "wall"), "zmin": ("front", "wall"), "zmax": ("back", "wall")}
SHAPES = ("flat", "parabolic", "power1over7")


def channel_block(cells, aspect, H=0.1):
    """A straight square duct L x H x H (L = aspect H) of about `cells`
    cubic hex cells along x: inlet at xmin, outlet at xmax, four walls."""
    from ._capi import PolyMesh
    ny = max(2, int(round((cells / aspect) ** (1.0 / 3.0))))
    nx = max(2, int(round(cells / (ny * ny))))
    return PolyMesh.block((0.0, 0.0, 0.0), (H * nx / ny, H, H), (nx, ny, ny), CHANNEL_SIDES)


def detail_block_set(n=64, seed=2024, cells_min=2_000, cells_max=200_000):
    """The batched detail-block workload: n ducts with cell counts drawn
    log-uniformly in [cells_min, cells_max], aspect ratios uniform in
    [5, 20], inlet profiles cycling flat / parabolic / power1over7, mean
    inlet speeds uniform in [0.05, 0.5] m/s; even-numbered blocks laminar
    (nu 1e-4), odd-numbered ones marked for k-epsilon (their viscosity is the caller's).
    Seeded numpy draws.  Returns a list of dicts."""
    rng = np.random.default_rng(seed)
    out = []
    for i in range(n):
        cells = float(np.exp(rng.uniform(np.log(cells_min), np.log(cells_max))))
        aspect = float(rng.uniform(5.0, 20.0))
        speed = float(rng.uniform(0.05, 0.5))
        out.append({"cells": cells, "aspect": aspect, "shape": SHAPES[i % 3], "speed": speed,
                    "laminar": i % 2 == 0})
    return out


def obstacle_channel_msh(path, nx=800, ny=200, nz=4, H=1.0, blockage=0.25, x_center=1.0):
    """A 2D-extruded channel of cubic hex cells (h = H/ny; L = nx h, depth
    nz h) with a square obstacle of side blockage*H centred at x_center on
    the axis, written as a gmsh 2.2 file with physical surfaces inlet
    (xmin), outlet (xmax), walls (y sides), obstacle, front and back (z
    sides).  Returns (n cells, cell size h)."""
    h = H / ny
    ns = int(round(blockage * ny))
    j0 = (ny - ns) // 2
    i0 = int(round(x_center / h)) - ns // 2
    inside = np.zeros((nx, ny), bool)
    inside[i0:i0 + ns, j0:j0 + ns] = True
    nid = lambda i, j, k: (k * (ny + 1) + j) * (nx + 1) + i + 1  # 1-based
    I, J, Kk = np.meshgrid(np.arange(nx + 1), np.arange(ny + 1), np.arange(nz + 1), indexing="ij")
    order = np.argsort(nid(I, J, Kk).ravel())
    pts = np.stack([I.ravel() * h, J.ravel() * h, Kk.ravel() * h], 1)[order]
    ci, cj, ck = np.nonzero(np.broadcast_to(~inside[:, :, None], (nx, ny, nz)))
    hexes = np.stack([nid(ci, cj, ck), nid(ci + 1, cj, ck), nid(ci + 1, cj + 1, ck), nid(ci, cj + 1, ck),
                      nid(ci, cj, ck + 1), nid(ci + 1, cj, ck + 1), nid(ci + 1, cj + 1, ck + 1),
                      nid(ci, cj + 1, ck + 1)], 1)
    quads = {name: [] for name in ("inlet", "outlet", "walls", "obstacle", "front", "back")}
    jj, kk = np.meshgrid(np.arange(ny), np.arange(nz), indexing="ij")
    jj, kk = jj.ravel(), kk.ravel()
    quads["inlet"] = np.stack([nid(0, jj, kk), nid(0, jj + 1, kk), nid(0, jj + 1, kk + 1), nid(0, jj, kk + 1)], 1)
    quads["outlet"] = np.stack([nid(nx, jj, kk), nid(nx, jj + 1, kk), nid(nx, jj + 1, kk + 1),
                                nid(nx, jj, kk + 1)], 1)
    ii, kk2 = np.meshgrid(np.arange(nx), np.arange(nz), indexing="ij")
    ii, kk2 = ii.ravel(), kk2.ravel()
    quads["walls"] = np.concatenate([
        np.stack([nid(ii, 0, kk2), nid(ii + 1, 0, kk2), nid(ii + 1, 0, kk2 + 1), nid(ii, 0, kk2 + 1)], 1),
        np.stack([nid(ii, ny, kk2), nid(ii + 1, ny, kk2), nid(ii + 1, ny, kk2 + 1), nid(ii, ny, kk2 + 1)], 1)])
    ob = []
    for k in range(nz):
        for j in range(j0, j0 + ns):
            ob.append([nid(i0, j, k), nid(i0, j + 1, k), nid(i0, j + 1, k + 1), nid(i0, j, k + 1)])
            ob.append([nid(i0 + ns, j, k), nid(i0 + ns, j + 1, k), nid(i0 + ns, j + 1, k + 1), nid(i0 + ns, j, k + 1)])
        for i in range(i0, i0 + ns):
            ob.append([nid(i, j0, k), nid(i + 1, j0, k), nid(i + 1, j0, k + 1), nid(i, j0, k + 1)])
            ob.append([nid(i, j0 + ns, k), nid(i + 1, j0 + ns, k), nid(i + 1, j0 + ns, k + 1), nid(i, j0 + ns, k + 1)])
    quads["obstacle"] = np.array(ob)
    fi, fj = np.nonzero(~inside)
    quads["front"] = np.stack([nid(fi, fj, 0), nid(fi + 1, fj, 0), nid(fi + 1, fj + 1, 0), nid(fi, fj + 1, 0)], 1)
    quads["back"] = np.stack([nid(fi, fj, nz), nid(fi + 1, fj, nz), nid(fi + 1, fj + 1, nz), nid(fi, fj + 1, nz)], 1)
    names = list(quads)
    with open(path, "w") as f:
        f.write("$MeshFormat\n2.2 0 8\n$EndMeshFormat\n$PhysicalNames\n%d\n" % (len(names) + 1))
        for g, name in enumerate(names):
            f.write('2 %d "%s"\n' % (g + 1, name))
        f.write('3 %d "fluid"\n$EndPhysicalNames\n$Nodes\n%d\n' % (len(names) + 1, len(pts)))
        np.savetxt(f, np.column_stack([np.arange(1, len(pts) + 1), pts]), fmt="%d %.17g %.17g %.17g")
        nq = sum(len(q) for q in quads.values())
        f.write("$EndNodes\n$Elements\n%d\n" % (nq + len(hexes)))
        e = 1
        for g, name in enumerate(names):
            q = np.asarray(quads[name])
            rows = np.column_stack([np.arange(e, e + len(q)), np.full(len(q), 3), np.full(len(q), 2),
                                    np.full(len(q), g + 1), np.full(len(q), g + 1), q])
            np.savetxt(f, rows, fmt="%d")
            e += len(q)
        rows = np.column_stack([np.arange(e, e + len(hexes)), np.full(len(hexes), 5), np.full(len(hexes), 2),
                                np.full(len(hexes), len(names) + 1), np.full(len(hexes), len(names) + 1), hexes])
        np.savetxt(f, rows, fmt="%d")
        f.write("$EndElements\n")
    return int(len(hexes)), h
