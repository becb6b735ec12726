"""The device PISO step (solveTransientIncompressiblePiso) against the
reference's own runs: 4 implicit-Euler steps of the jittered channel
(tests/golden/piso_channel.npz) and of the RANS channel with k-epsilon and
k-omega SST (piso_rans_*.npz), all made by the compiled reference."""
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


@pytest.mark.parametrize("fixture,model", [("piso_rans_keps.npz", "kEpsilon"), ("piso_rans_sst.npz", "kOmegaSST")])
def test_piso_with_rans_model_matches_reference(golden, fixture, model):
    """The RANS model advances first in every step with the step's dt (ddt in
    k and the dissipation variable) and feeds nu + nut to the momentum."""
    import chuanflow_b200 as cf
    g = golden(fixture)
    mesh, case = K.rans_channel_product(model=model)
    assert np.array_equal(mesh.addressing()["points"], g["points"])
    ctl = cf.PisoControls(dt=0.05, correctors=2, continuity_tol=1e-10, linear_tol=1e-10, non_orth_correctors=1,
                          nu=2.5e-6)
    for want in g["steps"]:
        r = case.piso_step(ctl)
        assert r["correctors_used"] == int(want[0])
    U, p, phi = case.download()
    t = case.turbulence_fields()
    for a, b, name in ((U, g["U"], "U"), (p, g["p"], "p"), (phi, g["phi"], "phi"), (t["k"], g["k"], "k"),
                       (t["eps"], g["eps"], "eps"), (t["nut"], g["nut"], "nut"),
                       (t["nuEffFace"], g["nuEffFace"], "nuEffFace")):
        assert rel(a, b) < REL_TOL, (name, rel(a, b))


def test_piso_rejects_bad_step():
    import chuanflow_b200 as cf
    mesh, case = K.channel_product(6, 3, 3)
    with pytest.raises(cf.CfgError, match="time step"):
        case.piso_step(cf.PisoControls(dt=0.0))
