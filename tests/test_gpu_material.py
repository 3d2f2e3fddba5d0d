"""Material model numerics on the GPU (closim_b200.material) against the
oracle's legacy path, as the reference's tests/material/material-model.test.ts
pins OrthotropicStVKMaterial to fem.ts / membrane-hvp.ts: energy, gradient and
max strain bitwise equal to evalInternal / internalEnergyOnly, the analytic HVP
bitwise equal to evalMembraneHvp, and within 1e-7 of the central-difference
membraneHvp; default and randomized valid materials on rest, stretched,
sheared and jittered states; Float32 inputs and caller-owned out buffers."""
import numpy as np
import pytest

import closim_b200 as cb
from closim_b200.material import OrthotropicStVKMaterial
from closim_b200.solver import ClothMaterial
from oracle import oracle as O

pytestmark = pytest.mark.gpu


def meshes():
    pos, uv, idx = cb.buildGrid(3, 2, 0.06, 0.04)
    return cb.preprocess(pos, uv, idx, 0.15), O.Mesh(pos, uv, idx, 0.15)


def states(mesh, rng):
    base = mesh.positions.astype(np.float64)
    n = mesh.count
    out = [base.copy()]
    s = base.copy()
    s[0::3] *= 1.2
    out.append(s)
    s = base.copy()
    s[0::3] += 0.3 * base[1::3]
    out.append(s)
    s = base.copy() + rng.uniform(-0.004, 0.004, 3 * n)
    out.append(s)
    return out


def rand_params(rng):
    c00, c11 = 1e3 + rng.random() * 9.9e4, 1e3 + rng.random() * 9.9e4
    rho = rng.random() * 2 - 1
    return {"inertia": {"arealDensityKgM2": 0.05 + rng.random() * 0.3}, "thicknessM": 1e-4 + rng.random() * 1.9e-3,
            "membrane": {"warpPa": c00, "weftPa": c11, "couplingPa": rho * 0.95 * np.sqrt(c00 * c11),
                         "shearPa": 0.0 if rng.random() < 0.1 else 1e3 + rng.random() * 1.9e4},
            "bending": {"warpNm": rng.random() * 2e-5, "weftNm": rng.random() * 2e-5},
            "dampingRatio": rng.random() * 0.1}


def oracle_mat(legacy: ClothMaterial):
    return dict(arealDensity=legacy.arealDensityKgM2, thickness=legacy.thickness, C00=legacy.stretchWarp,
                C11=legacy.stretchWeft, C01=legacy.stretchCoupling, G=legacy.shear, bendWarp=legacy.bendWarp,
                bendWeft=legacy.bendWeft, damping=legacy.damping)


def check_bitwise(model, mesh, omesh, x, direction):
    om = oracle_mat(model.toLegacy())
    assert model.energy(x, mesh) == O.internal_energy_only(omesh, om, x)
    e_old, g_old, s_old = O.eval_internal(omesh, om, x)
    r = model.gradient(x, mesh)
    assert r.energy == e_old and r.maxStrain == s_old
    assert np.array_equal(r.grad, g_old)
    assert np.array_equal(model.hessianVector(x, direction, mesh), O.eval_membrane_hvp(omesh, om, x, direction))


def test_default_material_bitwise_on_all_states():
    mesh, omesh = meshes()
    rng = np.random.default_rng(0x6A11)
    model = OrthotropicStVKMaterial.fromLegacy(ClothMaterial())
    direction = rng.uniform(-1, 1, 3 * mesh.count)
    for x in states(mesh, rng):
        check_bitwise(model, mesh, omesh, x, direction)


def test_randomized_materials_bitwise():
    mesh, omesh = meshes()
    rng = np.random.default_rng(0x7A1C)
    for _ in range(40):
        model = OrthotropicStVKMaterial(rand_params(rng))
        direction = rng.uniform(-1, 1, 3 * mesh.count)
        for x in states(mesh, rng):
            check_bitwise(model, mesh, omesh, x, direction)


def test_model_hvp_matches_fd_oracle():
    mesh, omesh = meshes()
    rng = np.random.default_rng(0xFD07)
    worst = 0.0
    for _ in range(20):
        model = OrthotropicStVKMaterial(rand_params(rng))
        x = states(mesh, rng)[3]
        direction = rng.uniform(-1, 1, 3 * mesh.count)
        a = model.hessianVector(x, direction, mesh)
        b = O.membrane_hvp(omesh, oracle_mat(model.toLegacy()), x, direction)
        e = np.sqrt(np.sum((a - b) ** 2) / max(np.sum(b * b), 1e-300))
        worst = max(worst, e)
        assert e < 1e-7
    print(f"worst model-vs-FD rel err {worst:.2e}")


def test_float32_inputs_and_out_buffers():
    mesh, omesh = meshes()
    rng = np.random.default_rng(5)
    model = OrthotropicStVKMaterial.fromLegacy(ClothMaterial())
    om = oracle_mat(model.toLegacy())
    x64 = states(mesh, rng)[2]
    x32 = x64.astype(np.float32)
    assert model.energy(x32, mesh) == O.internal_energy_only(omesh, om, x32.astype(np.float64))
    assert np.array_equal(model.gradient(x32, mesh).grad, O.eval_internal(omesh, om, x32.astype(np.float64))[1])
    out = np.full(3 * mesh.count, 123.456)
    r = model.gradient(x64, mesh, out)
    assert r.grad is out and np.array_equal(out, O.eval_internal(omesh, om, x64)[1])
    direction = np.full(3 * mesh.count, 0.25)
    hout = np.full(3 * mesh.count, -7.0)
    assert model.hessianVector(x64, direction, mesh, hout) is hout
    assert np.array_equal(hout, O.eval_membrane_hvp(omesh, om, x64, direction))


def test_json_round_trip_restores_bitwise_numerics():
    mesh, _ = meshes()
    x = mesh.positions.astype(np.float64) * 1.1
    m = OrthotropicStVKMaterial(rand_params(np.random.default_rng(3)), {"elastic": {"dataset": "Fabric-101"}})
    import json
    for back in (OrthotropicStVKMaterial.fromJSON(json.dumps(m.toJSON())), OrthotropicStVKMaterial.fromJSON(m.toJSON()),
                 m.clone()):
        assert back.energy(x, mesh) == m.energy(x, mesh)
        assert np.array_equal(back.gradient(x, mesh).grad, m.gradient(x, mesh).grad)
    thicker = OrthotropicStVKMaterial(dict(m.toJSON()["params"], thicknessM=0.002))
    assert thicker.energy(x, mesh) != m.energy(x, mesh)
