"""The model -> operator mapping (crates/rapidfem-td/src/build.rs:74-259) on
the CPU: materials by volume tag, PML regions as graded matched absorbers
(build.rs:36-68, :109-118), ports in the reference's order with its errors,
internal PEC plates severed from their neighbours (rhs.rs:862-880), and the
reference's absorbing-layer test (build.rs:278-326) on the oracle."""
import warnings

import numpy as np
import pytest

from oracle import oracle as R
from rapidfem_b200 import model as M
from rapidfem_b200 import operator as O


def _channel():
    """structured_box(1, 1, 10, 0.5, 0.5, 5) with volume tag 2 for z > 1.5."""
    tm = M.box_tagged(1, 1, 10, 0.5, 0.5, 5.0)
    cen = tm.mesh.nodes[tm.mesh.tets].mean(axis=1)
    tm.volume_tags = np.where(cen[:, 2] > 1.5, 2, 1).astype(np.int32)
    return tm


def test_materials_and_pml_rates():
    tm = _channel()
    model = M.Model(materials=[M.Material(1, er=2.0, ur_diag=(1.0, 1.5, 2.0), conductivity=0.3)],
                    pml=[M.Pml(2, direction=(0, 0, 1), inner_face=1.5, thickness=3.5)])
    mat = M.materials_of(tm, model)
    t1 = tm.tets_of(1)
    assert np.all(mat[t1, 0:3] == 2.0) and np.all(mat[t1, 3:6] == [1.0, 1.5, 2.0]) and np.all(mat[t1, 6] == 0.3)
    t2 = tm.tets_of(2)
    cz = tm.mesh.nodes[tm.mesh.tets[t2]][:, :, 2].mean(axis=1)
    nu = (M.ABSORBER_LOSS_BUDGET / 3.5) * np.clip((cz - 1.5) / 3.5, 0, 1) ** 2
    assert np.allclose(mat[t2, 6], nu * 1.0) and np.allclose(mat[t2, 7], nu * 1.0)  # sigma = nu eps, sigma* = nu mu
    assert np.all(mat[t2, 0:6] == 1.0)
    # a layer toward decreasing z: nothing in front of its inner plane is lossy
    model2 = M.Model(pml=[M.Pml(1, direction=(0, 0, -1), inner_face=1.0, thickness=1.0)])
    mat2 = M.materials_of(tm, model2)
    cz1 = tm.mesh.nodes[tm.mesh.tets[t1]][:, :, 2].mean(axis=1)
    assert np.all(mat2[t1[cz1 >= 1.0], 6] == 0.0) and np.all(mat2[t1[cz1 < 1.0], 6] > 0.0)


def test_port_order_codes_and_errors():
    tm = M.box_tagged(2, 2, 3)
    model = M.Model(faces=[M.AbcFace(6), M.RectangularPort(5, (1, 0))])
    code, tags, modes = M.face_codes_of(tm, model)
    # rectangular ports first, then ABC faces (build.rs:121-231)
    assert tags == [5, 6] and modes == [(1, 0), None]
    assert np.array_equal(code == 0, tm.faces_of(5)) and np.array_equal(code == 1, tm.faces_of(6))
    with pytest.raises(ValueError, match="mode \\(0, 0\\) carries no TE field"):
        M.face_codes_of(tm, M.Model(faces=[M.RectangularPort(5, (0, 0))]))
    with pytest.raises(ValueError, match="LumpedPort is not supported by the time-domain backend"):
        M.face_codes_of(tm, M.Model(faces=[M.OtherFace(5, "lumped")]))
    with pytest.raises(NotImplementedError):
        M.face_codes_of(tm, M.Model(faces=[M.OtherFace(5, "coax")]))
    with pytest.raises(ValueError, match="periodic pair \\(1, 99\\): a face tag has no triangles"):
        M.periodic_faces_of(tm, M.Model(periodic=[(1, 99)]))
    with pytest.raises(NotImplementedError):
        M.materials_of(tm, M.Model(materials=[M.Material(1, debye=(2.0, 4.0, 1e-3))]))
    with warnings.catch_warnings(record=True) as w:
        warnings.simplefilter("always")
        M.face_codes_of(tm, M.Model(faces=[M.OtherFace(3, "pmc")], far_field_tag=4))
    assert len(w) == 2
    with pytest.raises(ValueError, match="has no triangles"):
        M.face_codes_of(tm, M.Model(faces=[M.AbcFace(99)]))


def test_pec_plate_severs_faces_on_both_sides():
    tm = M.box_tagged(2, 2, 4)
    plate = M.plane_triangles(tm.mesh, 2, 0.5, lo=(0.0, 0.0, 0.0), hi=(0.5, 1.0, 1.0))
    tm.face_tags[10] = plate
    mo = M.operator_from_model(tm, M.Model(pec_tags=[10]), 2)
    on = tm.faces_of(10)
    assert on.sum() == 2 * len(plate)  # both sides of every plate triangle
    nbr = mo.op.get("nbr").reshape(-1, 4)
    port = mo.op.get("port").reshape(-1, 4)
    assert np.all(nbr[on] == -1) and np.all(port[on] == -1)
    free = O.MaxwellOperator(tm.mesh, 2, 1.0)
    assert np.all(free.get("nbr").reshape(-1, 4)[on] >= 0)
    # the oracle built with the same face codes agrees on the RHS
    orc = R.Operator(tm.mesh.nodes, tm.mesh.tets, 2, 1.0, face_port=mo.face_port, materials=mo.materials)
    assert np.array_equal(orc.get("nbr").reshape(-1, 4)[on], nbr[on])


def _energy_fraction(orc, y0, steps=900, h=0.06, m=24):
    e0 = orc.field_energy(y0)
    y = y0
    for _ in range(steps):
        y, _ = orc.expmv(y, h, m, 0.0)
    return orc.field_energy(y) / e0


def test_absorbing_layer_drains_field_energy_oracle():
    """build.rs:278-326: a disturbance in a closed PEC channel; with central
    flux vacuum conserves its energy, a matched absorbing layer (nu_max 6,
    3.5 deep at the far end) drains it."""
    lz, thickness = 5.0, 3.5
    mesh = O.structured_box(1, 1, 10, 0.5, 0.5, lz)
    K = mesh.n_tets
    nu = M.absorber_rate(mesh, np.arange(K), 2, False, lz - thickness, thickness, 6.0)
    mat = np.zeros((K, 8))
    mat[:, 0:6] = 1.0
    ok = ~np.isnan(nu)
    mat[ok, 6] = nu[ok]
    mat[ok, 7] = nu[ok]
    vac = R.Operator(mesh.nodes, mesh.tets, 2, 0.0)
    ab = R.Operator(mesh.nodes, mesh.tets, 2, 0.0, materials=mat)
    prod = O.MaxwellOperator(mesh, 2, 0.0)
    y0 = np.zeros(prod.n_dof)
    y0[prod.nearest_node_dof([0.25, 0.25, 0.6], 0, 0)] = 1.0
    frac_vac = _energy_fraction(vac, y0)
    frac_abs = _energy_fraction(ab, y0)
    assert frac_vac > 0.9
    assert frac_abs < 0.4
    assert frac_vac / frac_abs > 2.5
