"""The device RANS models (RansModel with KEpsilon, KOmegaSST, DesModel and
TransitionModel, Spalding wall functions) inside SIMPLE against the
reference's own runs of the same channel at Re_H 2e4 (tests/golden/rans_*.npz,
made by the compiled reference).  The wall functions and the SST blend
evaluate exp, pow, tanh and cbrt on the device, so the bar is relative, not
bit-for-bit."""
import numpy as np
import pytest

import _cases as K

pytestmark = pytest.mark.gpu

REL_TOL = 1e-6  # relative L2 of every field after the fixture's iterations (FP64)


def rel(a, b):
    nb = np.linalg.norm(b)
    return np.linalg.norm(a - b) / (nb if nb > 0 else 1.0)


@pytest.mark.parametrize("fixture,model", [("rans_channel.npz", "kEpsilon"), ("rans_sst.npz", "kOmegaSST"),
                                           ("rans_des.npz", "des"), ("rans_transition.npz", "gammaTransition")])
def test_rans_channel_matches_reference(golden, fixture, model):
    import chuanflow_b200 as cf
    g = golden(fixture)
    mesh, case = K.rans_channel_product(model=model)
    assert np.array_equal(mesh.addressing()["points"], g["points"])
    oc = K.channel_case(12, 5, 5, L=(1.0, 0.1, 0.1), jitter=0.0, nu=2.5e-6, iters=int(g["iterations"]),
                         non_orth=1)
    res = case.solve(K.controls_from(oc))
    assert res.iterations == int(g["iterations"])
    U, p, phi = case.download()
    t = case.turbulence_fields()
    for a, b, name in ((U, g["U"], "U"), (p, g["p"], "p"), (phi, g["phi"], "phi"), (t["k"], g["k"], "k"),
                       (t["eps"], g["eps"], "eps"), (t["nut"], g["nut"], "nut"),
                       (t["nuEffFace"], g["nuEffFace"], "nuEffFace")):
        assert rel(a, b) < REL_TOL, (name, rel(a, b))


def test_turbulence_setup_errors():
    import chuanflow_b200 as cf
    mesh, case = K.channel_product(6, 3, 3)
    with pytest.raises(cf.CfgError, match="not on the GPU path"):
        case.turbulence_setup("spalartAllmaras")
    with pytest.raises(cf.CfgError, match="reOnset"):
        case.turbulence_setup("gammaTransition", re_onset=0.0)
    with pytest.raises(cf.CfgError, match="C_DES"):
        case.turbulence_setup("des", c_des=0.0)
    with pytest.raises(cf.CfgError, match="relaxation"):
        case.turbulence_setup("kEpsilon", relaxation=1.5)
    with pytest.raises(cf.CfgError, match="no turbulence"):
        case.turbulence_fields()
    case.turbulence_setup("kEpsilon", nu=1e-3)
    case.turbulence_setup("laminar")
    with pytest.raises(cf.CfgError, match="no turbulence"):
        case.turbulence_fields()


def test_case_vtu_carries_the_device_fields(tmp_path):
    """cfg_write_vtu of a k-epsilon case: p, k, epsilon, nut and U as the
    device holds them (binary arrays read back)."""
    import re
    mesh, case = K.rans_channel_product(8, 4, 4)
    import chuanflow_b200 as cf
    case.solve(cf.SimpleControls(max_iterations=2, relax_u=0.9, relax_p=0.03, p_relax_start=0.02,
                                 non_orth_correctors=1, linear_tol=1e-8, nu=2.5e-6))
    out = tmp_path / "c.vtu"
    case.write_vtu(out, binary=True)
    head, data = out.read_bytes().split(b'<AppendedData encoding="raw">\n_', 1)
    got = {}
    for mt in re.finditer(rb'<DataArray type="Float64" Name="(\w+)"[^>]*offset="(\d+)"', head):
        off = int(mt.group(2))
        n = int(np.frombuffer(data[off:off + 8], np.uint64)[0])
        got[mt.group(1).decode()] = np.frombuffer(data[off + 8:off + 8 + n], np.float64)
    U, p, _ = case.download()
    t = case.turbulence_fields()
    assert list(got) == ["p", "k", "epsilon", "nut", "U"]
    assert np.array_equal(got["p"], p) and np.array_equal(got["U"].reshape(-1, 3), U)
    assert np.array_equal(got["k"], t["k"]) and np.array_equal(got["nut"], t["nut"])


def test_case_hdf5_carries_the_device_fields(tmp_path):
    """cfg_write_hdf5 of a k-omega SST case: /fields/p, k, omega, nut and
    Ux, Uy, Uz as the device holds them, beside the mesh datasets."""
    from _hdf5_read import read
    mesh, case = K.rans_channel_product(8, 4, 4, model="kOmegaSST")
    import chuanflow_b200 as cf
    case.solve(cf.SimpleControls(max_iterations=2, relax_u=0.9, relax_p=0.03, p_relax_start=0.02,
                                 non_orth_correctors=1, linear_tol=1e-8, nu=2.5e-6))
    out = tmp_path / "c.h5"
    case.write_hdf5(out)
    data, listing = read(out)
    U, p, _ = case.download()
    t = case.turbulence_fields()
    assert listing["/fields/"] == ["Ux", "Uy", "Uz", "k", "nut", "omega", "p"]
    assert np.array_equal(data["/fields/p"], p)
    for q, c in enumerate("xyz"):
        assert np.array_equal(data["/fields/U" + c], U[:, q])
    assert np.array_equal(data["/fields/k"], t["k"]) and np.array_equal(data["/fields/nut"], t["nut"])
    assert np.array_equal(data["/fields/omega"], t["eps"])
    assert np.array_equal(data["/points"], mesh.addressing()["points"])


@pytest.mark.parametrize("fixture", ["rans_channel.npz", "rans_sst.npz", "rans_des.npz", "rans_transition.npz"])
def test_case_file_with_turbulence_matches_reference(golden, tmp_path, fixture):
    """cfg_run_case_file on the fixture's own case file, turbulence{} block
    included, as the reference's simpleFoam app reads it: the same fields."""
    import chuanflow_b200 as cf
    g = golden(fixture)
    path = tmp_path / "case.dict"
    path.write_text(str(g["dict"]))
    res, counts, (U, p, phi) = cf.run_case_file(path, fields=True)
    assert res.iterations == int(g["iterations"])
    for a, b, name in ((U, g["U"], "U"), (p, g["p"], "p"), (phi, g["phi"], "phi")):
        assert rel(a, b) < REL_TOL, (name, rel(a, b))
