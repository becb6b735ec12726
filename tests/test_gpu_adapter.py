"""The C++ drop-in (chuanflow_b200/adapter): the reference's own driver,
built with its SIMPLE call switched to cf::gpu::solveIncompressibleSimple,
reproduces the reference's run of the same case.  The driver is built by
`make -C oracle` next to the reference driver; without it the test skips."""
import os
import subprocess
import tempfile

import numpy as np
import pytest

pytestmark = pytest.mark.gpu

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
DRIVER = os.path.join(ROOT, "oracle", "_ref", "cf_adapter_driver")
REL_TOL = 1e-6  # relative L2 of U, p and phi after the fixture's SIMPLE iterations (FP64)


def rel(a, b):
    nb = np.linalg.norm(b)
    return np.linalg.norm(a - b) / (nb if nb > 0 else 1.0)


@pytest.mark.skipif(not os.path.exists(DRIVER), reason="oracle/_ref/cf_adapter_driver not built")
def test_adapter_reproduces_reference_channel(golden):
    g = golden("simple_channel.npz")
    with tempfile.TemporaryDirectory() as td:
        cp = os.path.join(td, "case.dict")
        open(cp, "w").write(str(g["dict"]))
        pp = os.path.join(td, "points.f64")
        np.ascontiguousarray(g["points"]).tofile(pp)
        r = subprocess.run([DRIVER, "simple", cp, td, pp], capture_output=True, text=True, timeout=300)
        assert r.returncode == 0, r.stderr[-2000:]
        U = np.fromfile(os.path.join(td, "U.f64")).reshape(-1, 3)
        p = np.fromfile(os.path.join(td, "p.f64"))
        phi = np.fromfile(os.path.join(td, "phi.f64"))
        res = open(os.path.join(td, "result.txt")).read().split()
    assert int(res[0]) == int(g["iterations"])
    for a, b, name in ((U, g["U"], "U"), (p, g["p"], "p"), (phi, g["phi"], "phi")):
        assert rel(a, b) < REL_TOL, (name, rel(a, b))


REF_DRIVER = os.path.join(ROOT, "oracle", "_ref", "cf_ref_driver")


def run_driver(exe, text, points):
    with tempfile.TemporaryDirectory() as td:
        cp = os.path.join(td, "case.dict")
        open(cp, "w").write(text)
        pp = os.path.join(td, "points.f64")
        np.ascontiguousarray(points).tofile(pp)
        r = subprocess.run([exe, "simple", cp, td, pp], capture_output=True, text=True, timeout=600)
        assert r.returncode == 0, r.stderr[-2000:]
        return (np.fromfile(os.path.join(td, "U.f64")).reshape(-1, 3), np.fromfile(os.path.join(td, "p.f64")),
                np.fromfile(os.path.join(td, "phi.f64")), open(os.path.join(td, "result.txt")).read().split())


@pytest.mark.skipif(not (os.path.exists(DRIVER) and os.path.exists(REF_DRIVER)), reason="drivers not built")
def test_adapter_follows_reference_scheme_defaults():
    """Scheme names the reference does not know select its defaults (upwind
    convection, Gauss linear gradients, no laplacian correction); the adapter
    does the same, run live against the reference driver on one case."""
    import _cases as K
    g = K.channel_case(8, 5, 4)
    text = K.channel_dict(8, 5, 4, iters=4).replace(
        "schemes { ddt steady; div upwind; laplacian corrected; grad corrected; }",
        "schemes { ddt steady; div QUICK; laplacian uncorrected; grad fancy; }")
    assert "div QUICK" in text
    Ur, pr, phir, rr = run_driver(REF_DRIVER, text, g.mesh.points)
    Ua, pa, phia, ra = run_driver(DRIVER, text, g.mesh.points)
    assert int(ra[0]) == int(rr[0])
    for a, b, name in ((Ua, Ur, "U"), (pa, pr, "p"), (phia, phir, "phi")):
        assert rel(a, b) < REL_TOL, (name, rel(a, b))
