"""The C ABI: the library loads, exports every function include/*.h
declares, reports errors by status and message, and parses case files the
way the reference's simpleFoamApp reads them.  CPU only (no device calls)."""
import glob
import os
import re

import pytest

cf = pytest.importorskip("chuanflow_b200")
ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


def declared_functions():
    names = set()
    for h in glob.glob(os.path.join(ROOT, "include", "*.h")):
        text = re.sub(r"/\*.*?\*/", "", open(h).read(), flags=re.S)
        for m in re.finditer(r"^\s*(?:const\s+)?[A-Za-z_][A-Za-z0-9_]*\s*\**\s*(cfg_[A-Za-z0-9_]+)\s*\(", text, re.M):
            names.add(m.group(1))
    return sorted(names)


def test_every_declared_symbol_is_exported():
    lib = cf.lib()
    names = declared_functions()
    assert len(names) > 20
    missing = [n for n in names if not hasattr(lib, n)]
    assert not missing, missing


def test_version_and_error_channel():
    assert cf.lib().cfg_version().startswith(b"chuanflow_b200")
    with pytest.raises(cf.CfgError) as e:
        cf.PolyMesh.block((0, 0, 0), (1, 1, 1), (-1, 1, 1))
    assert e.value.code == 3


def write(tmp_path, text):
    p = tmp_path / "case.dict"
    p.write_text(text)
    return p


CASE = """// a case in the reference's grammar
block
{
    min   (0 0 0);
    max   (4 0.2 0.1);
    cells (10 4 2);
    xmin  { name inlet;   type inlet;    }
    xmax  { name outlet;  type outlet;   }
    ymin  { name bottom;  type wall;     }
    ymax  { name top;     type wall;     }
    zmin  { name front;   type symmetry; }
    zmax  { name back;    type symmetry; }
}
nu 0.01;   # kinematic viscosity
patches
{
    inlet  { U (0.1 0 0); UType fixedValue;  pType zeroGradient; }
    outlet { UType zeroGradient; p 0;        pType fixedValue;   }
    bottom { U (0 0 0);   UType fixedValue;  pType zeroGradient; }
    top    { }
}
schemes { ddt steady; div blend; blendCoeff 0.75; laplacian corrected; grad leastSquares; }
simple
{
    maxIterations 300;
    pcorrTol      1e-4;
    momentumTol   1e-4;
    relaxU        0.9;
    relaxP        0.03;
    pRelaxStart   0.02;
    linearTol     1e-8;
    force         (1 0 0);
}
initial { U (0.1 0 0); }
"""


def test_case_file_keys_follow_the_reference(tmp_path):
    s = cf.inspect_case_file(write(tmp_path, CASE))
    assert s["cells"] == [80.0]
    P = s["patches"]
    assert P["inlet"]["U_type"] == cf.BC["fixedValue"] and P["inlet"]["U"] == (0.1, 0.0, 0.0)
    assert P["outlet"]["U_type"] == cf.BC["zeroGradient"] and P["outlet"]["p_type"] == cf.BC["fixedValue"]
    # a listed wall without U is a no-slip wall (simpleFoamApp.cpp:69-80)
    assert P["top"]["U_type"] == cf.BC["fixedValue"] and P["top"]["p_type"] == cf.BC["zeroGradient"]
    # unlisted patches keep the fields' zeroGradient default
    assert P["front"]["U_type"] == cf.BC["zeroGradient"] and P["front"]["type"] == "symmetry"
    assert s["schemes"] == [2.0, 1.0, 2.0, 0.75]
    mi, ctol, pcorr, mtol, ltol, lmax, northo, ru, rp, rps = s["simple"]
    assert (mi, ctol, pcorr, mtol, ltol, lmax, northo) == (300, 1e-6, 1e-4, 1e-4, 1e-8, 2000, 2)
    assert (ru, rp, rps) == (0.9, 0.03, 0.02)
    assert s["force"] == [1.0, 0.0, 0.0] and s["nu"] == [0.01]
    assert s["gpu"] == [0.0, -1.0, 0.0, 0.0]
    assert s["initialU"] == [0.1, 0.0, 0.0]


def test_case_file_defaults_and_gpu_block(tmp_path):
    text = "block { min (0 0 0); max (1 1 1); cells (2 2 2); }\nnu 1;\ngpu { pRefCell 3; pRefValue 1.5; }\n"
    s = cf.inspect_case_file(write(tmp_path, text))
    assert s["simple"] == [200.0, 1e-6, 0.0, 0.0, 1e-7, 2000.0, 2.0, 0.7, 0.3, 0.0]
    assert s["schemes"] == [0.0, 1.0, 1.0, 0.9]
    assert s["gpu"] == [0.0, 3.0, 1.5, 0.0]
    for word, code in (("DIC", 1.0), ("AMG", 3.0)):
        s = cf.inspect_case_file(write(tmp_path, text.replace("gpu {", f"gpu {{ pPreconditioner {word};")))
        assert s["gpu"] == [code, 3.0, 1.5, 0.0]
    s = cf.inspect_case_file(write(tmp_path, text.replace("gpu {", "gpu { uPreconditioner AMG;")))
    assert s["gpu"] == [0.0, 3.0, 1.5, 3.0]
    with pytest.raises(cf.CfgError, match="unknown uPreconditioner 'DIC'"):
        cf.inspect_case_file(write(tmp_path, text.replace("gpu {", "gpu { uPreconditioner DIC;")))


@pytest.mark.parametrize("text,msg", [
    ("block { min (0 0 0); max (1 1 1); cells (2 2 2); }\n", "missing key 'nu'"),
    ("block { min (0 0 0); max (1 1 1); cells (2 2 2); }\nnu 1;\npatches { nowhere { U (0 0 0); } }\n",
     "no patch named 'nowhere'"),
    ("block { min (0 0 0); max (1 1 1); cells (2 2); }\nnu 1;\n", "need 3 values"),
    ("block { min (0 0 0); max (1 1 1); cells (2 2 2); }\nnu 1;\npatches { xmin { U (1 0 0); UType bogus; } }\n",
     "unknown patch bc type"),
    ("block { min (0 0 0) max (1 1 1); }\n", "missing ';'"),
])
def test_case_file_errors(tmp_path, text, msg):
    with pytest.raises(cf.CfgError, match=re.escape(msg)):
        cf.inspect_case_file(write(tmp_path, text))


def test_writers_refuse_null_arguments():
    """The output entry points report a null mesh, path or field as
    CFG_EINVAL through the status and the error channel, never a crash."""
    import ctypes as C
    lib = cf.lib()
    m = cf.PolyMesh.block((0, 0, 0), (1, 1, 1), (2, 2, 2))
    one = (C.c_char_p * 1)(b"p")
    assert lib.cfg_mesh_write_hdf5(None, b"x.h5", 0, None, None) == 1
    assert lib.cfg_mesh_write_hdf5(m._h, None, 0, None, None) == 1
    assert lib.cfg_mesh_write_hdf5(m._h, b"x.h5", 1, one, None) == 1
    assert lib.cfg_mesh_write_hdf5(m._h, b"x.h5", 1, one, (C.POINTER(C.c_double) * 1)()) == 1
    assert lib.cfg_mesh_write_hdf5(m._h, b"x.h5", -1, None, None) == 1
    buf = C.create_string_buffer(256)
    lib.cfg_last_error(buf, 256)
    assert b"cfg_mesh_write_hdf5" in buf.value
    assert lib.cfg_write_hdf5(None, b"x.h5") == 1
    assert lib.cfg_mesh_write_vtu(None, b"x.vtu", 0, None, None, None, 1) == 1


def test_case_file_turbulence_block(tmp_path):
    """turbulence{} as TurbulenceConfig::fromCase reads it (its defaults when
    keys are missing, laminar without the block) and its refusals."""
    base = "block { min (0 0 0); max (1 1 1); cells (2 2 2); }\nnu 1;\n"
    out = cf.inspect_case_file(write(tmp_path, base))
    assert out["turbulence"] == ["laminar", 0.05, -1.0, 0.7, 0.61, 0.0, -1.0, 4.0]
    out = cf.inspect_case_file(write(tmp_path, base + "turbulence { model des; intensity 0.02; lengthScale 0.01; "
                                                     "relaxation 0.5; C_DES 0.65; }\n"))
    assert out["turbulence"] == ["des", 0.02, 0.01, 0.5, 0.65, 0.0, -1.0, 4.0]
    for text, msg in (("turbulence { model kOmega; }", "unknown model 'kOmega'"),
                      ("turbulence { model kEpsilon; relaxation 0; }", "relaxation must be in (0, 1]"),
                      ("turbulence { model kEpsilon; intensity -1; }", "intensity must be non-negative")):
        with pytest.raises(cf.CfgError, match=re.escape(msg)):
            cf.inspect_case_file(write(tmp_path, base + text + "\n"))


def test_amg_strength_refuses_a_null_context():
    """cfg_amg_strength reports a null context as CFG_EINVAL with its name
    on the error channel (no device is touched)."""
    import ctypes as C
    lib = cf.lib()
    assert lib.cfg_amg_strength(None, C.c_double(0.25)) == 1
    buf = C.create_string_buffer(256)
    lib.cfg_last_error(buf, 256)
    assert b"cfg_amg_strength" in buf.value
