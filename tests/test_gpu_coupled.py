"""GPU partners in the reference's coupled 1D-3D interface.

oracle/_ref/cf_coupled_gpu_driver runs the reference's own solveCoupled1d3d
(coupledNetwork.cpp:1401-) on a network with three parallel coupled edges,
its partners chuanflow_b200/adapter's GpuDetailBlock: asked one by one, and
through GpuDetailBlockBatch, which evaluates each pass's blocks concurrently
under the unchanged driver.  The fixtures hold the same run with the
reference's DetailBlock partners (tests/golden/make_golden.py).

Bars: the passes, sweeps and block-converged flags equal; the rate, drop and
coefficient of every edge in every pass within 1e-6 relative (FP64 SIMPLE,
parallel dot products); the batched run bit-identical to the one-by-one run,
with every pass evaluated as one batch.
"""
import os
import subprocess
import tempfile

import numpy as np
import pytest

pytestmark = pytest.mark.gpu

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
DRIVER = os.path.join(ROOT, "oracle", "_ref", "cf_coupled_gpu_driver")
REL_TOL = 1e-6


def run(text, mode):
    with tempfile.TemporaryDirectory() as td:
        cp = os.path.join(td, "case.dict")
        open(cp, "w").write(text)
        r = subprocess.run([DRIVER, cp, td, mode], capture_output=True, text=True, timeout=600)
        assert r.returncode == 0, r.stderr[-2000:]
        lines = open(os.path.join(td, "history.txt")).read().split("\n")
        batch = open(os.path.join(td, "batch.txt")).read().split() if mode == "batch" else None
    rows = np.array([list(map(float, ln.split())) for ln in lines if ln and not ln.startswith("result")])
    res = [ln for ln in lines if ln.startswith("result")][0].split()[1:]
    return rows, int(res[0]), int(res[1]), float(res[2]), batch


@pytest.mark.skipif(not os.path.exists(DRIVER), reason="oracle/_ref/cf_coupled_gpu_driver not built")
@pytest.mark.parametrize("fixture", ["coupled_laminar.npz", "coupled_kepsilon.npz"])
def test_gpu_partners_reproduce_reference_coupling(golden, fixture):
    g = golden(fixture)
    ref = g["history"]
    single, it_s, conv_s, _, _ = run(str(g["dict"]), "single")
    batch, it_b, conv_b, _, counts = run(str(g["dict"]), "batch")
    assert (it_s, conv_s) == (int(g["iterations"]), int(g["converged"]))
    assert (it_b, conv_b) == (it_s, conv_s)
    assert single.shape == ref.shape
    # pass, edge, sweeps, block converged
    for col in (0, 1, 5, 6):
        assert np.array_equal(single[:, col], ref[:, col]), col
    # rate, drop, coefficient
    for col, name in ((2, "q"), (3, "dp"), (4, "R")):
        err = np.max(np.abs(single[:, col] - ref[:, col]) / np.abs(ref[:, col]))
        assert err < REL_TOL, (name, err)
    assert np.array_equal(batch, single)
    assert counts == [str(it_s), "0"]
