"""Linear-upwind convection, this library's extension (the reference's
fvm::div has upwind, linear and blend only, divScheme.cpp:18): CPU checks of
its C restatement in the oracle, and (gpu) the device assembly bit-identical
to that restatement and SIMPLE iterates within the FP64 bar."""
import dataclasses

import numpy as np
import pytest

import _cases as K
import _oracle as O

REL_TOL = 1e-6  # relative L2, U / p / phi after K SIMPLE iterations (FP64)


def rel(a, b):
    nb = np.linalg.norm(b)
    return np.linalg.norm(a - b) / (nb if nb > 0 else 1.0)


def eqns_inputs(case, seed=11):
    m = case.mesh
    rng = np.random.default_rng(seed)
    U = rng.normal(size=(m.nC, 3)) * 0.3
    p = rng.normal(size=m.nC)
    phi = case.initial_flux(U) + rng.normal(size=m.nF) * 1e-3 * (np.arange(m.nF) < m.nInt)
    return U, p, phi, rng.normal(size=m.nC)


def test_linear_upwind_is_exact_for_linear_fields():
    """With least-squares gradients (exact for linear fields), the deferred
    correction equals -sum(+-phi_f (U(Cf) - U(C_u))) for a linear U: the
    restated right-hand side minus the upwind one is that sum, per cell."""
    oc = K.cavity_case(5, 4, 3, jitter=0.15)
    oc.grad = "leastSquares"
    m = oc.mesh
    C, Cf = m.C, m.Cf
    A = np.array([[0.3, -0.2, 0.5], [0.1, 0.4, -0.3], [-0.2, 0.25, 0.15]])
    lin = lambda X: X @ A.T + np.array([0.05, -0.1, 0.2])
    U = lin(C)
    # boundary values consistent with the linear field: fixedValue per face
    nB = m.nF - m.nInt
    oc.u_face_values = {int(m.nInt + b): tuple(lin(Cf[m.nInt + b][None, :])[0]) for b in range(nB)}
    rng = np.random.default_rng(2)
    phi = rng.normal(size=m.nF)
    p = np.zeros(m.nC)
    x = np.zeros(m.nC)
    base = oc.eqns(U, p, phi, x)
    lu = dataclasses.replace(oc, div="linearUpwind").eqns(U, p, phi, x)
    own, nbr = m.owner[:m.nInt], m.neighbour
    up = np.where(phi[:m.nInt] >= 0, own, nbr)
    delta = phi[:m.nInt, None] * (lin(Cf[:m.nInt]) - U[up])
    want = np.zeros((m.nC, 3))
    np.add.at(want, own, -delta)
    np.add.at(want, nbr, delta)
    got = (lu["U_h0"] - base["U_h0"]).T
    assert np.allclose(got, want, rtol=1e-9, atol=1e-12 * np.abs(want).max())
    # the matrix is the upwind one
    assert np.array_equal(lu["U_diag"], base["U_diag"])


@pytest.mark.gpu
def test_linear_upwind_equations_bit_exact():
    """The device momentum assembly with linear-upwind convection equals the
    oracle's restatement bit for bit (diagonal, right-hand sides, operator)."""
    import chuanflow_b200 as cf
    oc = dataclasses.replace(K.cavity_case(6, 5, 4), div="linearUpwind")
    U, p, phi, x = eqns_inputs(oc)
    want = oc.eqns(U, p, phi, x)
    mesh, case = K.cavity_product(6, 5, 4, schemes=cf.Schemes(div="linearUpwind"))
    case.upload(U, p, phi)
    got = case.probe_equations(K.controls_from(oc), x)
    for q in range(3):
        assert np.array_equal(got["U_diag"][q], want["U_diag"][q]), q
        assert np.array_equal(got["U_h0"][q], want["U_h0"][q]), q
        assert np.array_equal(got["U_h1"][q], want["U_h1"][q]), q
    for k in ("rAUf", "p_diag", "p_h0", "p_h1", "phiCorrected"):
        assert np.array_equal(got[k], want[k]), k


@pytest.mark.gpu
@pytest.mark.parametrize("grad", ["linear", "corrected", "leastSquares"])
def test_linear_upwind_simple_matches_oracle(grad):
    """SIMPLE iterations of the jittered channel with linear-upwind
    convection against the oracle's run of the same case."""
    import chuanflow_b200 as cf
    oc = dataclasses.replace(K.channel_case(10, 6, 5), div="linearUpwind", grad=grad, max_iterations=5)
    U0, p0, phi0, r0 = oc.run()
    mesh, case = K.channel_product(10, 6, 5, schemes=cf.Schemes(div="linearUpwind", grad=grad))
    res = case.solve(K.controls_from(oc))
    U, p, phi = case.download()
    assert res.iterations == r0.iterations
    for a, b, name in ((U, U0, "U"), (p, p0, "p"), (phi, phi0, "phi")):
        assert rel(a, b) < REL_TOL, (name, rel(a, b))
