"""The learned pressure preconditioner: the device forward and backward
kernels against the FP64 PyTorch restatement (tests/_mpnn_ref.py) on the
same BF16 weights, training on the device from the plain solver's
residuals, and the gain of the trained network in flexible CG."""
import numpy as np
import pytest

import _cases as K
import _mpnn_ref as R
import _oracle as O

pytestmark = pytest.mark.gpu


def poisson_case(n=8):
    import chuanflow_b200 as cf
    mesh = cf.PolyMesh.block((0, 0, 0), (1, 1, 1), (n, n, n))
    mesh.jitter_interior(0.15, 3)
    case = cf.SimpleCase(mesh)
    for p in mesh.patches:
        case.set_patch_bc("U", p[0], "fixedValue", (0, 0, 0))
        case.set_patch_bc("p", p[0], "zeroGradient", 0.0)
    case.poisson_setup(ref_cell=0)
    return mesh, case


def oracle_csr(mesh):
    a = mesh.addressing()
    om = O.OMesh(a["points"], a["face_offsets"], a["face_verts"], a["owner"], a["neighbour"],
                 [p[0] for p in mesh.patches], [p[1] for p in mesh.patches], [p[2] for p in mesh.patches],
                 [p[3] for p in mesh.patches])
    oc = O.Case(om, u_type=["fixedValue"] * mesh.n_patches, u_value=[(0, 0, 0)] * mesh.n_patches,
                p_type=["zeroGradient"] * mesh.n_patches, p_value=[0] * mesh.n_patches, nu=1.0)
    oc.p_ref_cell = 0
    return oc.pressure_csr(np.ones(mesh.n_faces))


@pytest.mark.parametrize("layers", [1, 4])
def test_mpnn_gradient_matches_fp64_autograd(layers):
    """Loss and every weight's gradient against FP64 autograd on the same
    (BF16-exact) weights: FP32 activations and accumulation bound the gap."""
    mesh, case = poisson_case(8)
    case.mpnn_create(layers, seed=5)
    rng = np.random.default_rng(7)
    w = R.bf16_round(rng.normal(size=R.n_params(layers)).astype(np.float32) * 0.2)
    case.mpnn_weights(set=w)
    r = rng.normal(size=mesh.n_cells)
    loss, g = case.mpnn_loss_grad(r)
    rs, cols, vals = oracle_csr(mesh)
    loss0, g0, z0 = R.loss_and_grad(rs, cols, vals, r, w, layers)
    assert abs(loss - loss0) <= 1e-5 * abs(loss0), (loss, loss0)
    assert np.linalg.norm(g - g0) <= 2e-4 * np.linalg.norm(g0), np.linalg.norm(g - g0) / np.linalg.norm(g0)
    z = case.mpnn_apply(r)
    assert np.linalg.norm(z - z0) <= 1e-5 * np.linalg.norm(z0)


def test_untrained_network_is_jacobi():
    mesh, case = poisson_case(6)
    case.mpnn_create(4, seed=1)
    r = np.random.default_rng(2).normal(size=mesh.n_cells)
    rs, cols, vals = oracle_csr(mesh)
    n = mesh.n_cells
    rows = np.repeat(np.arange(n), np.diff(rs))
    d = np.zeros(n)
    np.add.at(d, rows[rows == cols], vals[rows == cols])
    assert np.array_equal(case.mpnn_apply(r), r / d)


def test_trained_network_gains_in_flexible_cg():
    """Trained on residuals of the plain Jacobi-PCG's iterates, the network
    lowers its training loss, and flexible CG with it needs fewer
    iterations to the same FP64 true residual than with the untrained
    (Jacobi) network; both reach the DIC-PCG solution."""
    mesh, case = poisson_case(16)
    rng = np.random.default_rng(11)
    samples = []
    for k in range(6):
        b = rng.normal(size=mesh.n_cells)
        b -= b.mean()
        for it in (0, 5, 20, 60):
            x, _ = case.poisson_solve(b, "jacobi64", tol=1e-14, max_iter=max(it, 1)) if it else (np.zeros_like(b), None)
            samples.append(case.poisson_residual(b, x))
    samples = np.array(samples)
    case.mpnn_create(4, seed=3)
    b = rng.normal(size=mesh.n_cells)
    b -= b.mean()
    x0, r0 = case.poisson_solve(b, "fcg_mpnn", tol=1e-8)
    losses = case.mpnn_train(samples, epochs=40, lr=2e-3)
    assert losses[-1] < 0.8 * losses[0], losses
    x1, r1 = case.poisson_solve(b, "fcg_mpnn", tol=1e-8)
    xd, rd = case.poisson_solve(b, "dic64", tol=1e-12)
    assert r0["converged"] and r1["converged"]
    assert r1["inner_iterations"] < r0["inner_iterations"], (r1, r0)
    for x in (x0, x1):
        assert np.linalg.norm(x - xd) <= 1e-6 * np.linalg.norm(xd)


def test_learned_pressure_in_piso_steps(tmp_path):
    """Residuals kept from the DIC-PCG pressure solves of PISO steps train
    the network; steps with the network's flexible CG (DIC fallback) from
    the same fields reach the same flow as DIC-PCG steps."""
    import chuanflow_b200 as cf
    from chuanflow_b200 import meshgen
    path = tmp_path / "o.msh"
    n, h = meshgen.obstacle_channel_msh(str(path), 80, 20, 2)
    mesh = cf.PolyMesh.read_gmsh(path, {"inlet": "inlet", "outlet": "outlet"})
    case = cf.SimpleCase(mesh)
    bcs = {"inlet": ("fixedValue", (1.0, 0, 0), "zeroGradient"), "outlet": ("zeroGradient", 0.0, "fixedValue"),
           "walls": ("fixedValue", (0, 0, 0), "zeroGradient"), "obstacle": ("fixedValue", (0, 0, 0), "zeroGradient"),
           "front": ("zeroGradient", 0.0, "zeroGradient"), "back": ("zeroGradient", 0.0, "zeroGradient")}
    for name, (ut, uv, pt) in bcs.items():
        case.set_patch_bc("U", name, ut, uv)
        case.set_patch_bc("p", name, pt, 0.0)
    case.init_flux()
    ctl = cf.PisoControls(dt=0.5 * h, correctors=2, linear_tol=1e-8, non_orth_correctors=0, nu=0.25 / 200,
                          p_preconditioner="DIC")
    case.mpnn_create(4, seed=3)
    for s in range(24):
        case.mpnn_collect(2 if s == 0 else 1, 48)
        case.piso_step(ctl)
    kept = case.mpnn_collect(0, 48)
    assert kept == 48
    losses = case.mpnn_train_collected(20, 2e-3)
    assert losses[-1] < losses[0]
    b = cf.Batch([case])
    b.save()
    for _ in range(6):
        case.piso_step(ctl)
    U0, p0, _ = case.download()
    b.restore()
    import dataclasses
    c2 = dataclasses.replace(ctl, p_preconditioner="MPNN")
    for _ in range(6):
        r = case.piso_step(c2)
        assert not r["diverged"]
    U1, p1, _ = case.download()
    assert np.linalg.norm(U1 - U0) <= 1e-6 * np.linalg.norm(U0)


@pytest.mark.parametrize("layers", [1, 4])
def test_mpnn_pair_gradient_matches_fp64_autograd(layers):
    """The energy-norm loss on a (residual, converged correction) pair --
    e.Ae / t.At with e = M(r) - t -- and every weight's gradient against FP64
    autograd of the same network on the same BF16 weights."""
    mesh, case = poisson_case(8)
    case.mpnn_create(layers, seed=6)
    rng = np.random.default_rng(9)
    w = R.bf16_round(rng.normal(size=R.n_params(layers)).astype(np.float32) * 0.2)
    case.mpnn_weights(set=w)
    rs, cols, vals = oracle_csr(mesh)
    n = mesh.n_cells
    rows = np.repeat(np.arange(n), np.diff(rs))
    A = np.zeros((n, n))
    np.add.at(A, (rows, cols), vals)
    t = rng.normal(size=n)
    r = A @ t
    loss, g = case.mpnn_loss_grad_pair(r, t)
    loss0, g0, _ = R.loss_and_grad(rs, cols, vals, r, w, layers, t=t)
    assert abs(loss - loss0) <= 1e-4 * abs(loss0), (loss, loss0)
    assert np.linalg.norm(g - g0) <= 1e-3 * np.linalg.norm(g0), np.linalg.norm(g - g0) / np.linalg.norm(g0)


def test_piso_pairs_train_the_initial_guess():
    """PISO on a small obstacle channel collects (residual, converged
    correction) pairs from its DIC-PCG pressure solves; trained on them, the
    network lowers its energy-norm loss, and as the initial guess of the
    pressure solves (with the FP32 AMG flexible CG after it) the same steps
    need fewer pressure iterations than the AMG flexible CG from the
    previous pressure, with the velocity within 1e-6 of the DIC run."""
    import dataclasses
    import chuanflow_b200 as cf
    from chuanflow_b200 import meshgen
    import tempfile, os
    nx, ny = 48, 12
    with tempfile.TemporaryDirectory() as td:
        path = os.path.join(td, "o.msh")
        ncell, h = meshgen.obstacle_channel_msh(path, nx, ny, 2)
        mesh = cf.PolyMesh.read_gmsh(path, {"inlet": "inlet", "outlet": "outlet"})
    case = cf.SimpleCase(mesh)
    for name, _, _, _ in mesh.patches:
        if name == "inlet":
            case.set_patch_bc("U", name, "fixedValue", (1.0, 0, 0))
            case.set_patch_bc("p", name, "zeroGradient", 0.0)
        elif name == "outlet":
            case.set_patch_bc("U", name, "zeroGradient", 0.0)
            case.set_patch_bc("p", name, "fixedValue", 0.0)
        elif name in ("walls", "obstacle"):
            case.set_patch_bc("U", name, "fixedValue", (0, 0, 0))
            case.set_patch_bc("p", name, "zeroGradient", 0.0)
        else:
            case.set_patch_bc("U", name, "zeroGradient", 0.0)
            case.set_patch_bc("p", name, "zeroGradient", 0.0)
    case.init_flux()
    ctl = cf.PisoControls(dt=0.5 * h, correctors=2, continuity_tol=1e-10, linear_tol=1e-8, non_orth_correctors=0,
                          nu=0.25 / 200.0, p_preconditioner="DIC")
    case.mpnn_create(4, seed=3)
    case.mpnn_collect(2, 64)
    for _ in range(40):
        case.piso_step(ctl)
    case.mpnn_collect(0, 64)
    losses = case.mpnn_train_collected(40, 2e-3)
    assert losses[-1] < 0.7 * losses[0], losses
    batch = cf.Batch([case])
    batch.save()
    legs = {}
    for name in ("DIC", "AMG", "AMG_MPNN"):
        batch.restore()
        c2 = dataclasses.replace(ctl, p_preconditioner=name)
        it = 0
        for _ in range(10):
            r = case.piso_step(c2)
            it += r["p_inner_iterations"]
        legs[name] = (it, case.download()[0])
    assert legs["AMG_MPNN"][0] < legs["AMG"][0], {k: v[0] for k, v in legs.items()}
    for k in ("AMG", "AMG_MPNN"):
        U, U0 = legs[k][1], legs["DIC"][1]
        assert np.linalg.norm(U - U0) <= 1e-6 * np.linalg.norm(U0), k
