"""writeFieldsHdf5 (src/3d/src/io/hdf5Write.cpp:38-95): the library's own
HDF5 encoder, read back by a reader written from the file format
specification (no HDF5 library is in the image).  CPU only."""
import numpy as np
import pytest

import _cases as K
from _hdf5_read import read

cf = pytest.importorskip("chuanflow_b200")


def _mesh():
    m = cf.PolyMesh.block((0, 0, 0), (1, 1, 1), (4, 3, 2), {s: (n, "wall") for s, n in zip(K.SIDES, K.CAVITY_NAMES)})
    m.jitter_interior(0.1, 7)
    return m


def test_layout_and_values_are_the_reference_writers(tmp_path):
    """/points (nP x 3), /owner, /neighbour and /fields/<name>, as the
    reference lays them out; every value bit-exact."""
    m = _mesh()
    rng = np.random.default_rng(0)
    fields = {"p": rng.standard_normal(m.n_cells), "Ux": rng.standard_normal(m.n_cells)}
    out = tmp_path / "a.h5"
    m.write_hdf5(out, fields)
    data, listing = read(out)
    a = m.addressing()
    assert listing["/"] == ["fields", "neighbour", "owner", "points"]
    assert listing["/fields/"] == ["Ux", "p"]
    assert data["/points"].shape == (m.n_points, 3) and np.array_equal(data["/points"], a["points"])
    assert data["/owner"].dtype == np.int64 and np.array_equal(data["/owner"], a["owner"])
    assert np.array_equal(data["/neighbour"], a["neighbour"][:m.n_internal_faces])
    for k, v in fields.items():
        assert np.array_equal(data["/fields/" + k], v), k


def test_many_fields_span_several_symbol_table_nodes(tmp_path):
    """Beyond eight links a group holds several symbol-table nodes under
    one B-tree node; names stay in strcmp order across them."""
    m = _mesh()
    names = ["f%02d" % i for i in range(37)] + ["Z", "_a", "a_b", "nut"]
    fields = {n: np.full(m.n_cells, float(i)) for i, n in enumerate(names)}
    out = tmp_path / "b.h5"
    m.write_hdf5(out, fields)
    data, listing = read(out)
    assert listing["/fields/"] == sorted(names, key=lambda s: s.encode())
    for i, n in enumerate(names):
        assert np.array_equal(data["/fields/" + n], np.full(m.n_cells, float(i)))


def test_no_fields_and_a_single_cell(tmp_path):
    m = cf.PolyMesh.block((0, 0, 0), (1, 1, 1), (1, 1, 1))
    out = tmp_path / "c.h5"
    m.write_hdf5(out)
    data, listing = read(out)
    assert listing["/fields/"] == [] and data["/neighbour"].shape == (0,)
    assert data["/owner"].shape == (6,)


def test_errors(tmp_path):
    m = _mesh()
    v = np.zeros(m.n_cells)
    with pytest.raises(cf.CfgError, match="size mismatch"):
        m.write_hdf5(tmp_path / "e.h5", {"p": np.zeros(m.n_cells + 1)})
    for bad in ("", "a/b", "."):
        with pytest.raises(cf.CfgError, match="cannot create dataset"):
            m.write_hdf5(tmp_path / "e.h5", {bad: v})
    with pytest.raises(cf.CfgError, match="at most 256"):
        m.write_hdf5(tmp_path / "e.h5", {"f%d" % i: v for i in range(257)})
    with pytest.raises(cf.CfgError, match="cannot open"):
        m.write_hdf5(tmp_path / "no" / "dir.h5", {"p": v})
