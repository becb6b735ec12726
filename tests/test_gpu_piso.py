"""The device PISO step (solveTransientIncompressiblePiso) against the
reference's own run: 4 implicit-Euler steps of the jittered channel
(tests/golden/piso_channel.npz, made by the compiled reference)."""
import numpy as np
import pytest

import _cases as K

pytestmark = pytest.mark.gpu

REL_TOL = 1e-6  # relative L2 of U, p, phi after the steps (FP64)


def rel(a, b):
    nb = np.linalg.norm(b)
    return np.linalg.norm(a - b) / (nb if nb > 0 else 1.0)


@pytest.mark.parametrize("precond", ["Jacobi", "DIC"])
def test_piso_channel_matches_reference(golden, precond):
    import chuanflow_b200 as cf
    g = golden("piso_channel.npz")
    mesh, case = K.channel_product(16, 6, 6)
    assert np.array_equal(mesh.addressing()["points"], g["points"])
    ctl = cf.PisoControls(dt=0.05, correctors=2, continuity_tol=1e-10, linear_tol=1e-10, non_orth_correctors=1,
                          nu=1e-3, p_preconditioner=precond)
    for want in g["steps"]:
        r = case.piso_step(ctl)
        assert r["correctors_used"] == int(want[0])
        assert abs(r["continuity_error"] - want[2]) <= 1e-4 * abs(want[2]) + 1e-12
    U, p, phi = case.download()
    for a, b, name in ((U, g["U"], "U"), (p, g["p"], "p"), (phi, g["phi"], "phi")):
        assert rel(a, b) < REL_TOL, (name, rel(a, b))


def test_piso_rejects_bad_step():
    import chuanflow_b200 as cf
    mesh, case = K.channel_product(6, 3, 3)
    with pytest.raises(cf.CfgError, match="time step"):
        case.piso_step(cf.PisoControls(dt=0.0))
