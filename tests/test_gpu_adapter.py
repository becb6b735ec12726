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


@pytest.mark.skipif(not os.path.exists(DRIVER), reason="oracle/_ref/cf_adapter_driver not built")
def test_adapter_rejects_what_the_gpu_path_lacks():
    """A scheme the GPU path does not carry is a cf::Error, as the
    reference's own unknown-scheme errors are; the driver exits non-zero."""
    text = ("block { min (0 0 0); max (1 1 1); cells (3 3 3); }\nnu 0.01;\n"
            "schemes { ddt steady; div QUICK; laplacian corrected; grad corrected; }\n"
            "simple { maxIterations 1; }\n")
    with tempfile.TemporaryDirectory() as td:
        cp = os.path.join(td, "case.dict")
        open(cp, "w").write(text)
        r = subprocess.run([DRIVER, "simple", cp, td], capture_output=True, text=True, timeout=300)
    assert r.returncode != 0
    assert "chuanflow_b200" in r.stderr, r.stderr[-2000:]
