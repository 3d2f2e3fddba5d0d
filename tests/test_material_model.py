"""Material model layer (closim_b200.material) against the reference's
tests/material/material-params.test.ts, on the CPU: SI unit table, parameter
validation codes, calibration metadata, JSON round trips, legacy bridge and
immutable snapshots. The GPU numerics are in tests/test_gpu_material.py."""
import json
import math

import pytest

from closim_b200.material import (FRICTION_OWNERSHIP_NOTE, MaterialValidationError, OrthotropicStVKMaterial,
                                  describeParameters)
from closim_b200.solver import ClothMaterial


def valid_params():
    return {"inertia": {"arealDensityKgM2": 0.15}, "thicknessM": 0.001,
            "membrane": {"warpPa": 20000, "weftPa": 20000, "couplingPa": 0, "shearPa": 5000},
            "bending": {"warpNm": 1e-5, "weftNm": 1e-5}, "dampingRatio": 0.001}


def test_si_unit_table_and_friction_ownership():
    assert describeParameters() == [
        {"path": "inertia.arealDensityKgM2", "unit": "kg/m^2"}, {"path": "thicknessM", "unit": "m"},
        {"path": "membrane.warpPa", "unit": "Pa"}, {"path": "membrane.weftPa", "unit": "Pa"},
        {"path": "membrane.couplingPa", "unit": "Pa"}, {"path": "membrane.shearPa", "unit": "Pa"},
        {"path": "bending.warpNm", "unit": "N*m"}, {"path": "bending.weftNm", "unit": "N*m"},
        {"path": "dampingRatio", "unit": "dimensionless"}]
    assert "contact" in FRICTION_OWNERSHIP_NOTE


def _set(p, path, v):
    keys = path.split(".")
    for k in keys[:-1]:
        p = p[k]
    p[keys[-1]] = v


@pytest.mark.parametrize("name,changes,code", [
    ("zero thickness", {"thicknessM": 0}, "non-positive-thickness"),
    ("negative thickness", {"thicknessM": -1e-4}, "non-positive-thickness"),
    ("NaN thickness", {"thicknessM": math.nan}, "non-finite"),
    ("infinite stiffness", {"membrane.warpPa": math.inf}, "non-finite"),
    ("zero density", {"inertia.arealDensityKgM2": 0}, "non-positive-density"),
    ("negative density", {"inertia.arealDensityKgM2": -0.2}, "non-positive-density"),
    ("negative warp", {"membrane.warpPa": -1}, "negative-stiffness"),
    ("negative shear", {"membrane.shearPa": -50}, "negative-stiffness"),
    ("negative bending", {"bending.warpNm": -1e-9}, "negative-stiffness"),
    ("indefinite coupling", {"membrane.warpPa": 1e3, "membrane.weftPa": 1e3, "membrane.couplingPa": 5000},
     "indefinite-coupling"),
    ("negative damping", {"dampingRatio": -0.1}, "damping-range"),
    ("damping above 1", {"dampingRatio": 1.5}, "damping-range"),
    ("NaN damping", {"dampingRatio": math.nan}, "non-finite"),
])
def test_rejects_invalid_params(name, changes, code):
    p = valid_params()
    for k, v in changes.items():
        _set(p, k, v)
    with pytest.raises(MaterialValidationError) as e:
        OrthotropicStVKMaterial(p)
    assert e.value.code == code, name


def test_malformed_shapes_and_valid_edges():
    for bad in ({}, None):
        with pytest.raises(MaterialValidationError):
            OrthotropicStVKMaterial(bad)
    zero = valid_params()
    zero["membrane"] = {"warpPa": 0, "weftPa": 0, "couplingPa": 0, "shearPa": 0}
    OrthotropicStVKMaterial(zero)  # fully compliant membrane: degenerate but valid
    edge = valid_params()
    edge["membrane"].update(warpPa=4e4, weftPa=1e4, couplingPa=math.sqrt(4e4 * 1e4))
    OrthotropicStVKMaterial(edge)  # PSD boundary (equality) is allowed


def test_legacy_bridge_validates():
    OrthotropicStVKMaterial.fromLegacy(ClothMaterial())
    with pytest.raises(MaterialValidationError):
        OrthotropicStVKMaterial.fromLegacy(ClothMaterial(thickness=-0.5))
    m = OrthotropicStVKMaterial(valid_params())
    assert OrthotropicStVKMaterial.fromLegacy(m.toLegacy()).toLegacy() == m.toLegacy()


def test_calibration_metadata_round_trip_and_rejections():
    cal = {"elastic": {"dataset": "Fabric-101", "specimenId": "cotton-poplin-03",
                       "protocol": "uniaxial-warp/weft + 45deg-shear", "measuredAt": "2026-03-14",
                       "moduliPa": {"warp": 21000, "weft": 19000, "coupling": 500, "shear": 5200}},
           "hysteresis": {"model": "none", "notes": "recoverable loop area recorded off-model"},
           "plasticity": {"model": "none"}, "provenanceNotes": "lab-conditioned 20C/65%RH"}
    m = OrthotropicStVKMaterial(valid_params(), cal)
    assert m.calibration["elastic"]["dataset"] == "Fabric-101"
    assert m.calibration["plasticity"]["model"] == "none"
    back = OrthotropicStVKMaterial.fromJSON(json.dumps(m.toJSON()))
    assert back.toJSON()["calibration"] == m.toJSON()["calibration"]
    with pytest.raises(MaterialValidationError):
        OrthotropicStVKMaterial(valid_params(), {"elastic": {"dataset": ""}})
    for kind, model in (("plasticity", "j2-plastic"), ("hysteresis", "prandtl")):
        with pytest.raises(MaterialValidationError, match="not-implemented"):
            OrthotropicStVKMaterial(valid_params(), {"elastic": {"dataset": "Fabric-101"}, kind: {"model": model}})


def test_json_tags_are_load_bearing():
    m = OrthotropicStVKMaterial(valid_params(), {"elastic": {"dataset": "Fabric-101", "specimenId": "s-1"}})
    j = m.toJSON()
    assert j["kind"] == "orthotropic-stvk" and j["version"] == 1
    for restored in (OrthotropicStVKMaterial.fromJSON(json.dumps(j)), OrthotropicStVKMaterial.fromJSON(j)):
        assert restored.toLegacy() == m.toLegacy()
    with pytest.raises(MaterialValidationError, match="unknown-kind"):
        OrthotropicStVKMaterial.fromJSON(dict(j, kind="neo-hookean"))
    with pytest.raises(MaterialValidationError, match="version"):
        OrthotropicStVKMaterial.fromJSON(dict(j, version=999))
    with pytest.raises(ValueError):
        OrthotropicStVKMaterial.fromJSON("not json")
    plain = OrthotropicStVKMaterial(valid_params())
    assert plain.calibration is None
    assert OrthotropicStVKMaterial.fromJSON(json.dumps(plain.toJSON())).calibration is None


def test_clone_and_immutable_snapshot():
    src = valid_params()
    m = OrthotropicStVKMaterial(src, {"elastic": {"dataset": "d"}})
    src["thicknessM"] = 0.5  # the caller's dict is not shared
    assert m.toLegacy().thickness == 0.001
    c = m.clone()
    assert c is not m and c.params is not m.params and c.calibration is not m.calibration
    assert c.toLegacy() == m.toLegacy()
    with pytest.raises(TypeError):
        m.params["thicknessM"] = 0.002  # frozen against silent mutation
    with pytest.raises(TypeError):
        m.params["membrane"]["warpPa"] = 1.0
