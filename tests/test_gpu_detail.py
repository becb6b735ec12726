"""Detail blocks (DetailBlock, src/coupling/src/coupledNetwork.cpp) and their
batched evaluation.  The oracle side restates the block's set-up (inlet
profile, cross-sections), boundary conditions and measurement in numpy
around the oracle's SIMPLE; the device block must match it within the FP64
bar, and a batch must reproduce its blocks evaluated alone."""
import dataclasses

import numpy as np
import pytest

import _cases as K
import _oracle as O

pytestmark = pytest.mark.gpu

REL_TOL = 1e-6


def rel(a, b):
    nb = np.linalg.norm(b)
    return np.linalg.norm(a - b) / (nb if nb > 0 else 1.0)


def profile_weights(m, shape, inlet, axis=0):
    """buildInletProfile (coupledNetwork.cpp:768-877) on the oracle mesh."""
    start, size = m.patch_start[inlet], m.patch_size[inlet]
    faces = np.arange(start, start + size)
    if shape == "flat":
        return faces, None
    lo, hi = m.points.min(0), m.points.max(0)
    axes = []
    for k in range(3):
        if k == axis:
            continue
        b = [0, 0]
        for pi, t in enumerate(m.patch_types):
            if t != "wall":
                continue
            sf = m.Sf[m.patch_start[pi]:m.patch_start[pi] + m.patch_size[pi]].sum(0)
            kk = int(np.argmax(np.abs(sf)))
            if kk == k:
                b[0 if sf[k] < 0 else 1] = 1
        if b[0] and b[1]:
            axes.append(k)
    w = np.ones(size)
    for k in axes:
        mid, half = 0.5 * (hi[k] + lo[k]), 0.5 * (hi[k] - lo[k])
        eta = (m.Cf[faces, k] - mid) / half
        w *= (1.0 - eta * eta) if shape == "parabolic" else np.power(1.0 - np.abs(eta), 1.0 / 7.0)
    a = np.linalg.norm(m.Sf[faces], axis=1)
    return faces, w / ((w * a).sum() / a.sum())


def oracle_block(m, shape, q, rho, ctl_case, state=None):
    """lossAt(q) restated: applyBoundary, SIMPLE (oracle), measure."""
    names = list(m.patch_names)
    types = list(m.patch_types)
    inlet, outlet = types.index("inlet"), types.index("outlet")
    sf_in = m.Sf[m.patch_start[inlet]:m.patch_start[inlet] + m.patch_size[inlet]].sum(0)
    area = np.linalg.norm(sf_in)
    u_in = np.zeros(3)
    u_in[0] = q / area  # inlet at xmin: flow along +x
    ut, uv, pt = [], [], []
    for i, t in enumerate(types):
        if i == inlet:
            ut.append("fixedValue"); uv.append(tuple(u_in)); pt.append("zeroGradient")
        elif i == outlet:
            ut.append("zeroGradient"); uv.append((0, 0, 0)); pt.append("fixedValue")
        elif t == "wall":
            ut.append("fixedValue"); uv.append((0, 0, 0)); pt.append("zeroGradient")
        else:
            ut.append("zeroGradient"); uv.append((0, 0, 0)); pt.append("zeroGradient")
    faces, w = profile_weights(m, shape, inlet)
    fv = None if w is None else {int(f): tuple(u_in * wi) for f, wi in zip(faces, w)}
    c = O.Case(m, u_type=ut, u_value=uv, p_type=pt, p_value=[0.0] * len(types), nu=ctl_case.nu,
               max_iterations=ctl_case.max_iterations, linear_tol=ctl_case.linear_tol, non_orth=ctl_case.non_orth,
               relax_u=ctl_case.relax_u, relax_p=ctl_case.relax_p, p_relax_start=ctl_case.p_relax_start,
               u_face_values=fv)
    if state is None:
        U, p, phi = None, None, None
    else:
        U, p, phi = (np.array(a, copy=True) for a in state)
        phi[m.nInt:] = c.initial_flux(U)[m.nInt:]
    U, p, phi, r = c.run(U, p, phi)
    x = m.C[:, 0]
    band = 1e-9 * (m.points[:, 0].max() - m.points[:, 0].min())
    first = np.abs(x - x.min()) <= band
    last = np.abs(x - x.max()) <= band
    dp = rho * (p[first] * m.V[first]).sum() / m.V[first].sum() - rho * (p[last] * m.V[last]).sum() / m.V[last].sum()
    fin = -phi[m.patch_start[inlet]:m.patch_start[inlet] + m.patch_size[inlet]].sum()
    fout = phi[m.patch_start[outlet]:m.patch_start[outlet] + m.patch_size[outlet]].sum()
    return {"dp_pa": dp, "flux_in": fin, "flux_out": fout, "sweeps": r.iterations}, (U, p, phi)


@pytest.mark.parametrize("shape", ["flat", "parabolic", "power1over7"])
def test_detail_loss_matches_restatement(shape):
    """Two coupling passes (rate q, then a warm start at 1.3 q) of one block."""
    import chuanflow_b200 as cf
    cells, L = (14, 5, 4), (0.7, 0.1, 0.1)
    om = O.block_mesh((0, 0, 0), L, cells, K.CHANNEL_NAMES, K.CHANNEL_TYPES)
    oc = O.Case(om, u_type=["zeroGradient"] * 6, u_value=[(0, 0, 0)] * 6, p_type=["zeroGradient"] * 6,
                p_value=[0] * 6, nu=1e-3, max_iterations=3, linear_tol=1e-10, non_orth=1, relax_u=0.9,
                relax_p=0.3, p_relax_start=0.02)
    mesh = cf.PolyMesh.block((0, 0, 0), L, cells, dict(zip(K.SIDES, zip(K.CHANNEL_NAMES, K.CHANNEL_TYPES))))
    case = cf.SimpleCase(mesh)
    case.detail_setup(shape, rho=998.0)
    ctl = K.controls_from(oc)
    state = None
    for q in (2e-4, 2.6e-4):
        want, state = oracle_block(om, shape, q, 998.0, oc, state)
        got = case.detail_loss(q, ctl)
        assert got["sweeps"] == want["sweeps"]
        for k in ("dp_pa", "flux_in", "flux_out"):
            assert abs(got[k] - want[k]) <= REL_TOL * abs(want[k]), (k, got[k], want[k])
        assert abs(got["flux_in"] - q) <= 1e-12 * q
        U, p, phi = case.download()
        assert rel(U, state[0]) < REL_TOL and rel(phi, state[2]) < REL_TOL


def test_detail_setup_errors():
    import chuanflow_b200 as cf
    mesh = cf.PolyMesh.block((0, 0, 0), (1, 0.1, 0.1), (6, 3, 3))  # no inlet/outlet patch types
    case = cf.SimpleCase(mesh)
    with pytest.raises(cf.CfgError, match="inlet"):
        case.detail_setup("flat")
    mesh = cf.PolyMesh.block((0, 0, 0), (1, 0.1, 0.1), (6, 3, 3), dict(zip(K.SIDES, zip(K.CHANNEL_NAMES,
                                                                                          K.CHANNEL_TYPES))))
    case = cf.SimpleCase(mesh)
    with pytest.raises(cf.CfgError, match="profile"):
        case.detail_setup("cosine")
    case.detail_setup("flat")
    with pytest.raises(cf.CfgError, match="non-positive"):
        case.detail_loss(0.0, cf.SimpleControls(max_iterations=1, nu=1e-3))


def test_batch_matches_blocks_alone():
    """A concurrent pass over uneven blocks gives, block for block, the bits
    of the same blocks evaluated one after another with the same grid; the
    autotuner picks one of its candidates."""
    import chuanflow_b200 as cf
    from chuanflow_b200 import meshgen
    spec = meshgen.detail_block_set(6, seed=3, cells_min=500, cells_max=6000)
    ctl = cf.SimpleControls(max_iterations=3, relax_u=0.7, relax_p=0.3, p_relax_start=0.02, non_orth_correctors=1,
                            linear_tol=1e-8, nu=1e-4, p_preconditioner="DIC")

    def build():
        cases = []
        for s in spec:
            c = cf.SimpleCase(meshgen.channel_block(s["cells"], s["aspect"]))
            c.detail_setup(s["shape"])
            cases.append(c)
        return cases

    q = [s["speed"] * 0.01 for s in spec]
    a_cases, b_cases = build(), build()
    a, b = cf.Batch(a_cases), cf.Batch(b_cases)
    a.set_schedule(1, 1)
    b.set_schedule(4, 1)
    for _ in range(2):
        ra, _ = a.loss(q, ctl)
        rb, _ = b.loss(q, ctl)
        for x, y in zip(ra, rb):
            assert x["dp_pa"] == y["dp_pa"] and x["flux_out"] == y["flux_out"]
            assert (x["status"] == 0) == (x["dp_pa"] > 0)
    for ca, cb in zip(a_cases, b_cases):
        for u, v in zip(ca.download(), cb.download()):
            assert np.array_equal(u, v)
    sched, times = b.autotune(q, ctl)
    assert sched in cf.Batch.CANDIDATES and len(times) == len(cf.Batch.CANDIDATES)


def test_rans_blocks_batch_and_restore():
    """k-epsilon detail blocks in a batch: the model is created at the first
    lossAt, a pass repeated from restored fields (velocity, pressure, flux,
    k, epsilon, nut) gives the same bits, and the drop is finite."""
    import chuanflow_b200 as cf
    from chuanflow_b200 import meshgen
    cases = []
    for cells, aspect, shape in ((1500, 6.0, "flat"), (3000, 9.0, "power1over7")):
        c = cf.SimpleCase(meshgen.channel_block(cells, aspect))
        c.detail_setup(shape)
        c.detail_turbulence("kEpsilon", nu=0.3 * 0.1 / 2e4)
        cases.append(c)
    b = cf.Batch(cases)
    b.set_schedule(2, 1)
    ctl = cf.SimpleControls(max_iterations=2, relax_u=0.7, relax_p=0.3, p_relax_start=0.02, non_orth_correctors=1,
                            linear_tol=1e-8, nu=0.3 * 0.1 / 2e4, p_preconditioner="DIC")
    q = [0.3 * 0.01, 0.2 * 0.01]
    b.loss(q, ctl)
    b.save()
    r1, _ = b.loss(q, ctl)
    t1 = [c.turbulence_fields()["k"] for c in cases]
    b.restore()
    r2, _ = b.loss(q, ctl)
    t2 = [c.turbulence_fields()["k"] for c in cases]
    for x, y, a, bb in zip(r1, r2, t1, t2):
        assert x["dp_pa"] == y["dp_pa"] and np.isfinite(x["dp_pa"])
        assert np.array_equal(a, bb)


@pytest.mark.parametrize("pressure", ["DIC", "Jacobi"])
def test_graph_pass_matches_blocks_alone(pressure):
    """The whole coupling pass as one CUDA-graph launch (schedule workers 0:
    every block's outer iteration a branch of the graph, its solver loops
    device-side while-nodes) gives, pass after pass, the bits of the same
    blocks evaluated one after another with the same solver grid -- drops,
    fluxes, inner iteration counts and fields -- for laminar and k-epsilon
    blocks alike."""
    import chuanflow_b200 as cf
    from chuanflow_b200 import meshgen
    spec = meshgen.detail_block_set(6, seed=5, cells_min=500, cells_max=8000)

    def build():
        cases = []
        for k, s in enumerate(spec):
            c = cf.SimpleCase(meshgen.channel_block(s["cells"], s["aspect"]))
            c.detail_setup(s["shape"])
            if k % 2:
                c.detail_turbulence("kEpsilon", nu=s["speed"] * 0.1 / 2e4)
            cases.append(c)
        return cases

    ctls = [cf.SimpleControls(max_iterations=1, relax_u=0.7, relax_p=0.3, p_relax_start=0.02, non_orth_correctors=1,
                              linear_tol=1e-8, nu=(1e-4 if k % 2 == 0 else s["speed"] * 0.1 / 2e4),
                              p_preconditioner=pressure) for k, s in enumerate(spec)]
    q = [s["speed"] * 0.01 for s in spec]
    a_cases, b_cases = build(), build()
    a, b = cf.Batch(a_cases), cf.Batch(b_cases)
    a.set_schedule(1, 1)
    b.set_schedule(0, 1)
    for _ in range(3):
        ra, _ = a.loss(q, ctls)
        rb, _ = b.loss(q, ctls)
        for x, y in zip(ra, rb):
            assert x["dp_pa"] == y["dp_pa"] and x["flux_out"] == y["flux_out"] and x["flux_in"] == y["flux_in"]
            assert x["u_inner_iterations"] == y["u_inner_iterations"]
            assert x["p_inner_iterations"] == y["p_inner_iterations"]
            assert x["sweeps"] == y["sweeps"] == 1 and x["status"] == y["status"]
    for ca, cb in zip(a_cases, b_cases):
        for u, v in zip(ca.download(), cb.download()):
            assert np.array_equal(u, v)
    # the controls the single-graph pass cannot take are refused
    with pytest.raises(cf.CfgError, match="single-graph"):
        b.loss(q, [dataclasses.replace(c, max_iterations=2) for c in ctls])
