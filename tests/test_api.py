"""Host-side tests that need no GPU: the C ABI library loads and exports every
symbol include/glued_b200.h declares; GluedForce descriptor semantics and XML
round trips (tests/test_xml_serialization.py:55-210 of the reference); the
reference's unchanged python/glued.py driving this library's gluedplugin."""
import math
import os
import re
import subprocess
import sys
import types

import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


def test_library_exports_every_declared_symbol():
    from gluedmd_b200 import _native
    _native.lib()
    hdr = open(os.path.join(ROOT, "include", "glued_b200.h")).read()
    declared = set(re.findall(r"\b(glued_\w+)\s*\(", hdr))
    out = subprocess.run(["nm", "-D", "--defined-only", _native.LIB_PATH], capture_output=True, text=True).stdout
    exported = set(re.findall(r"\bT (glued_\w+)", out))
    missing = declared - exported
    assert not missing, missing
    assert set(_native.exported_symbols()) <= exported


def test_descriptor_semantics():
    from gluedmd_b200 import GluedForce, GluedError
    f = GluedForce()
    assert f.addCollectiveVariable(f.CV_DISTANCE, [0, 1]) == 0
    assert f.addCollectiveVariable(f.CV_PATH, [0], [1.0, 2, 0, 0, 0, 1, 1, 1]) == 1
    assert f.addCollectiveVariable(f.CV_ANGLE, [0, 1, 2]) == 3
    assert f.getNumCollectiveVariables() == 4
    assert f.getNumCollectiveVariableSpecs() == 3
    with pytest.raises(GluedError):
        f.addCollectiveVariable(-1, [0])
    with pytest.raises(GluedError, match="out of range"):
        f.addBias(f.BIAS_HARMONIC, [4], [1.0, 0.0])
    assert f.addBias(f.BIAS_HARMONIC, [3], [10.0, 1.0], [0]) == 0
    t, c, p, ip = f.getBiasParameters(0)
    assert (t, c, p, ip) == (1, [3], [10.0, 1.0], [0])
    g = GluedForce(f)  # copy does not share context binding
    assert g.getNumBiases() == 1 and g._context is None
    with pytest.raises(GluedError, match="no Context"):
        f.getBiasState()
    assert GluedForce.barrierToGamma(50.0, 2.5) == 20.0
    assert abs(GluedForce.kTFromTemperature(300.0) - 2.494338785) < 1e-9
    f.setTestBiasGradients([1.0, 2.0])
    assert f.getTestBiasGradients() == [1.0, 2.0]
    f.setTestForce(2, 0.5)
    assert f.getTestForceMode() == 2 and f.getTestForceScale() == 0.5
    with pytest.raises(GluedError):
        f.setForceGroup(40)


def _roundtrip(f):
    from gluedmd_b200 import GluedForce
    x = f.toXml()
    return GluedForce.fromXml(x), x


def test_xml_round_trips():
    from gluedmd_b200 import GluedForce
    f = GluedForce()
    f.setTemperature(300.0)
    f.setUsesPeriodicBoundaryConditions(True)
    f.setForceGroup(5)
    f.addCollectiveVariable(f.CV_DISTANCE, [3, 7])
    f.addCollectiveVariable(f.CV_COORDINATION, [1, 0, 2], [0.35, 6, 12])
    f.addCollectiveVariable(f.CV_RMSD, [0, 1], [0.1, 1e-17, math.pi, -2.5, 1 / 3, 7e5])
    f.addExpressionCV('cv0 * 2 + "x" < 3 & y', [0, 1])
    f.addPyTorchCV("/tmp/model.pt", [0, 1, 2], [0.5])
    f.addBias(f.BIAS_OPES, [0, 1], [2.49, 20.05, 0.1, 0.2, 0.005], [0, 500, 1000])
    f.addBias(f.BIAS_METAD, [0], [1.2, 0.35, 10, 2.49, -math.pi, math.pi], [500, 256, 1])
    rt, xml = _roundtrip(f)
    assert xml.startswith('<?xml version="1.0" ?>')
    assert '<Force forceGroup="5"' in xml and 'type="GluedForce"' in xml
    assert rt.getNumCollectiveVariableSpecs() == 5 and rt.getNumBiases() == 2
    assert rt.getTemperature() == 300.0 and rt.usesPeriodicBoundaryConditions() is True
    assert rt.getForceGroup() == 5
    for i in range(5):
        assert rt.getCollectiveVariableParameters(i) == f.getCollectiveVariableParameters(i)
    for i in range(2):
        assert rt.getBiasParameters(i) == f.getBiasParameters(i)
    assert rt.getExpressionCVInfo(3) == f.getExpressionCVInfo(3)
    assert rt.getPyTorchCVModelPath(4) == "/tmp/model.pt"
    assert rt.toXml() == xml


def test_xml_rejects_bad_input():
    from gluedmd_b200 import GluedForce, GluedError
    with pytest.raises(GluedError, match="unsupported format version"):
        GluedForce.fromXml('<Force type="GluedForce" version="2"><CollectiveVariables/><Biases/></Force>')
    with pytest.raises(GluedError):
        GluedForce.fromXml('<Force type="GluedForce" version="1"><CollectiveVariables>')
    f = GluedForce.fromXml('<?xml version="1.0" ?>\n<Force type="GluedForce" version="1" usesPBC="true">'
                           '<CollectiveVariables><CV type="1" numAtoms="2" atom0="0" atom1="1" numParams="0"/>'
                           '</CollectiveVariables><Biases></Biases></Force>')
    assert f.usesPeriodicBoundaryConditions() and f.getNumCollectiveVariables() == 1


# The reference tree's location comes from GLUED_REFERENCE only; the test is
# skipped when it is unset.
REF_GLUED = os.path.join(os.environ.get("GLUED_REFERENCE", ""), "python", "glued.py")


@pytest.mark.skipif(not (os.environ.get("GLUED_REFERENCE") and os.path.exists(REF_GLUED)),
                    reason="GLUED_REFERENCE not set to a reference tree")
def test_reference_glued_py_runs_unchanged_on_this_gluedplugin():
    """GLUED's own python/glued.py (imported from the reference tree, not copied)
    builds forces through this library's gluedplugin; its encoded parameter
    vectors are what the reference kernels consume."""
    import importlib.util
    from gluedmd_b200 import gluedplugin
    stub = types.ModuleType("openmm")
    stub.vectori = type("vectori", (list,), {})
    stub.vectord = type("vectord", (list,), {})
    saved = {k: sys.modules.get(k) for k in ("openmm", "gluedplugin")}
    sys.modules["openmm"] = stub
    sys.modules["gluedplugin"] = gluedplugin
    try:
        spec = importlib.util.spec_from_file_location("glued_ref_wrapper", REF_GLUED)
        glued = importlib.util.module_from_spec(spec)
        spec.loader.exec_module(glued)
        f = glued.Force(pbc=True, temperature=300.0)
        phi = f.add_dihedral([4, 6, 8, 14])
        psi = f.add_dihedral([6, 8, 14, 16])
        cn = f.add_coordination([0, 1], [2, 3, 4], r0=0.35)
        f.add_opes([phi, psi], sigma=0.05, gamma=10.0, pace=500)
        f.add_metad([phi, psi], sigma=0.35, height=1.2, pace=500, grid_min=-math.pi, grid_max=math.pi,
                    bins=256, periodic=True, gamma=10.0)
        f.add_harmonic(cn, kappa=100.0, at=1.5)
        assert (phi, psi, cn) == (0, 1, 2)
        assert f.getCollectiveVariableParameters(2) == (6, [2, 0, 1, 2, 3, 4], [0.35, 6.0, 12.0])
        kT = 8.314462618e-3 * 300.0
        t, c, p, ip = f.getBiasParameters(0)
        assert t == 5 and c == [0, 1] and ip == [0, 500, 100000]
        assert p[:2] == [kT, 10.0] and p[2:4] == [0.05, 0.05]
        t, c, p, ip = f.getBiasParameters(1)
        assert t == 3 and ip == [500, 256, 256, 1, 1]
        assert p[0] == 1.2 and p[1:3] == [0.35, 0.35] and p[3:5] == [10.0, kT]
        assert f.getBiasParameters(2) == (1, [2], [100.0, 1.5], [0])
        rt = gluedplugin.GluedForce.fromXml(f.toXml())
        assert rt.getBiasParameters(1) == f.getBiasParameters(1)
    finally:
        for k, v in saved.items():
            if v is None:
                sys.modules.pop(k, None)
            else:
                sys.modules[k] = v
