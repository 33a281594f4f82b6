"""Operators built from a model (build.rs:74-259) on the device: the RHS of a
model with materials, a PML absorber, a rectangular port, an ABC face and an
internal PEC plate against the f64 oracle built from the same face codes and
material table, on both stage engines; the reference's absorbing-layer test
(build.rs:278-326) run with the device Krylov propagator; and a model port's
incident-field source against the oracle's."""
import numpy as np
import pytest

from oracle import oracle as R
from rapidfem_b200 import gpu as G
from rapidfem_b200 import model as M
from rapidfem_b200 import operator as O
from rapidfem_b200 import td as T
from rapidfem_b200._native import ENGINE_FP32, ENGINE_TF32X3

from .conftest import rel_l2

pytestmark = pytest.mark.gpu


@pytest.fixture(scope="module")
def ctx():
    return G.GpuContext(0)


def _model_problem():
    tm = M.box_tagged(3, 2, 6, 1.0, 0.5, 2.0)
    cen = tm.mesh.nodes[tm.mesh.tets].mean(axis=1)
    tm.volume_tags = np.where(cen[:, 2] > 1.4, 3, np.where(cen[:, 0] < 0.5, 2, 1)).astype(np.int32)
    tm.face_tags[20] = M.plane_triangles(tm.mesh, 2, 1.0, lo=(0.0, 0.0, 0.0), hi=(0.34, 0.5, 2.0))
    model = M.Model(materials=[M.Material(2, er=3.0, conductivity=0.5)],
                    pml=[M.Pml(3, direction=(0, 0, 1), inner_face=1.4, thickness=0.6)],
                    faces=[M.RectangularPort(5, (1, 0)), M.AbcFace(6)], pec_tags=[20])
    return tm, model


@pytest.mark.parametrize("engine", [ENGINE_FP32, ENGINE_TF32X3], ids=["fp32", "tf32x3"])
def test_model_operator_apply_matches_oracle(ctx, engine):
    tm, model = _model_problem()
    mo = M.operator_from_model(tm, model, 3)
    assert mo.port_tags == [5, 6]
    gop = G.GpuOperator(ctx, mo.op)
    gop.set_engine(engine)
    orc = R.Operator(tm.mesh.nodes, tm.mesh.tets, 3, 1.0, face_port=mo.face_port, materials=mo.materials)
    y = np.sin(0.3 + 0.017 * np.arange(mo.op.n_dof)).astype(np.float32)
    assert rel_l2(gop.apply(y), orc.apply(y.astype(np.float64))) < 1e-5
    # the plate and the absorber change the operator
    plain = R.Operator(tm.mesh.nodes, tm.mesh.tets, 3, 1.0)
    assert rel_l2(plain.apply(y.astype(np.float64)), orc.apply(y.astype(np.float64))) > 1e-2


def test_absorbing_layer_drains_field_energy_device(ctx):
    """build.rs:278-326 with the device Krylov propagator (m = 24 as two
    KRYLOV_CHUNK sub-steps), against the same run on the f64 oracle."""
    lz, thickness = 5.0, 3.5
    tm = M.box_tagged(1, 1, 10, 0.5, 0.5, lz)
    mesh = tm.mesh
    K = mesh.n_tets
    nu = M.absorber_rate(mesh, np.arange(K), 2, False, lz - thickness, thickness, 6.0)
    mat = np.zeros((K, 8))
    mat[:, 0:6] = 1.0
    ok = ~np.isnan(nu)
    mat[ok, 6] = nu[ok]
    mat[ok, 7] = nu[ok]
    fracs = {}
    for name, materials in (("vacuum", None), ("absorber", mat)):
        op = O.MaxwellOperator(mesh, 2, 0.0, materials=materials)
        gop = G.GpuOperator(ctx, op)
        gop.set_krylov_precision(64)
        sess = T.TdSession(op, 1.0)
        y = np.zeros(op.n_dof)
        y[op.nearest_node_dof([0.25, 0.25, 0.6], 0, 0)] = 1.0
        e0 = sess.field_energy(y)
        for _ in range(900):
            y, _ = gop.expmv(y, 0.06, 24)
        fracs[name] = sess.field_energy(y) / e0
    assert fracs["vacuum"] > 0.9
    assert fracs["absorber"] < 0.4
    assert fracs["vacuum"] / fracs["absorber"] > 2.5
    # the same run on the oracle, composed over the device's sub-steps
    orc = R.Operator(mesh.nodes, mesh.tets, 2, 0.0, materials=mat)
    y = np.zeros(orc.n_dof)
    y[O.MaxwellOperator(mesh, 2, 0.0).nearest_node_dof([0.25, 0.25, 0.6], 0, 0)] = 1.0
    e0 = orc.field_energy(y)
    for _ in range(900):
        for _ in range(2):
            y, _ = orc.expmv(y, 0.03, 12, 0.0)
    assert abs(fracs["absorber"] - orc.field_energy(y) / e0) < 1e-6


def test_model_port_source_matches_oracle(ctx):
    tm, model = _model_problem()
    sess = T.TdSession.from_model(tm, model, 3)
    mo = sess.model_operator
    k, spec = sess._ports[5]
    assert np.allclose(spec["inward_normal"], (0.0, 0.0, 1.0))
    prof = mo.op.rect_port_profiles(k, spec["inward_normal"], spec["mode"])
    orc = R.Operator(tm.mesh.nodes, tm.mesh.tets, 3, 1.0, face_port=mo.face_port, materials=mo.materials)
    b = sess.port_source(5)
    assert rel_l2(b, orc.port_source(k, prof)) < 1e-12 and np.linalg.norm(b) > 0
    assert np.all(sess.port_source(6) == 0.0)  # an ABC face injects nothing
