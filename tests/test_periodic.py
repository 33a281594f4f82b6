"""Periodic face pairs (PeriodicSpec / link_periodic_faces, rhs.rs:253-270,
546-770; build.rs:235-240): the native host build against the oracle's
restatement, the geometry of the links, the reference's error cases, and a
plane wave crossing a box that is periodic in x and z (a travelling wave
needs the links; PEC walls there would reflect it)."""
import numpy as np
import pytest

from oracle import oracle as R
from rapidfem_b200 import model as M
from rapidfem_b200 import operator as O

from .conftest import rel_l2


def _tagged(nx, ny, nz, lx, ly, lz, warp=0.0):
    """The tagged Kuhn box, its nodes optionally moved by a smooth
    displacement that is periodic in all three directions and keeps each
    boundary plane in place (the component normal to a wall vanishes there),
    so opposite walls still match under the period translation while the
    elements are distorted."""
    tm = M.box_tagged(nx, ny, nz, lx, ly, lz)
    if warp:
        x = tm.mesh.nodes.copy()
        L = np.array([lx, ly, lz])
        s = np.sin(2.0 * np.pi * x / L)
        c = np.cos(2.0 * np.pi * x / L + 0.4)
        h = (L / np.array([nx, ny, nz])).min()
        d = warp * h * np.stack([s[:, 0] * c[:, 1] * c[:, 2], s[:, 1] * c[:, 0] * c[:, 2],
                                 s[:, 2] * c[:, 0] * c[:, 1]], axis=1)
        tm.mesh = O.Mesh(x + d, tm.mesh.tets)
    return tm


def _linked(tm, order, pairs, alpha=1.0):
    mo = M.operator_from_model(tm, M.Model(periodic=pairs), order, alpha)
    orc = R.Operator(tm.mesh.nodes, tm.mesh.tets, order, alpha)
    for a, b in M.periodic_faces_of(tm, M.Model(periodic=pairs)):
        orc.link_periodic(a, b)
    return mo.op, orc


@pytest.mark.parametrize("order", [2, 3])
@pytest.mark.parametrize("warp", [0.0, 0.2], ids=["regular", "warped"])
def test_links_match_oracle(order, warp):
    tm = _tagged(3, 2, 4, 1.5, 1.0, 2.0, warp)
    op, orc = _linked(tm, order, [(1, 2), (3, 4), (5, 6)])
    for name in ("nbr", "nbr_lf", "perm"):
        assert np.array_equal(op.get(name), orc.get(name)), name
    nbr = op.get("nbr").astype(np.int64)
    assert np.all(nbr >= 0)  # every face of a fully periodic box has a neighbour


def test_link_geometry():
    """A linked face's nodes, shifted by the period, land on its partner's
    nodes in the permuted order, and the two permutations invert each other."""
    lx, ly, lz = 1.5, 1.0, 2.0
    tm = _tagged(3, 2, 4, lx, ly, lz, 0.2)
    base = M.operator_from_model(tm, M.Model(), 3).op
    op, _ = _linked(tm, 3, [(1, 2)])
    nbr0, nbr = base.get("nbr").astype(np.int64), op.get("nbr").astype(np.int64)
    lf = op.get("nbr_lf").astype(np.int64)
    perm = op.get("perm").astype(np.int64).reshape(-1, op.nfp)
    fn = op.get("face_nodes").astype(np.int64).reshape(4, op.nfp)
    x = op.node_coords().reshape(op.n_elem, op.np, 3)
    (fa, fb), = M.periodic_faces_of(tm, M.Model(periodic=[(1, 2)]))
    assert np.all(nbr0[fa] < 0) and np.all(nbr0[fb] < 0)
    changed = np.flatnonzero(nbr != nbr0)
    assert np.array_equal(np.sort(changed), np.sort(np.concatenate([fa, fb])))
    for f in fa:
        e, l = divmod(int(f), 4)
        g = int(nbr[f]) * 4 + int(lf[f])
        assert g in set(fb.tolist())
        here = x[e, fn[l]] + np.array([lx, 0.0, 0.0])
        there = x[g // 4, fn[g % 4]][perm[f]]
        assert np.max(np.abs(here - there)) < 1e-12
        assert nbr[g] == e and lf[g] == l
        assert np.array_equal(perm[g][perm[f]], np.arange(op.nfp))


def _two_duplicates(op, faces):
    """`faces` with faces p and r replaced by q and s, where the triangle
    centroids satisfy c_q - c_p = c_r - c_s: the side's mean centroid (and so
    the inferred translation) is unchanged, but q and s each appear twice."""
    x = op.node_coords().reshape(op.n_elem, op.np, 3)
    fn = op.get("face_nodes").astype(np.int64).reshape(4, op.nfp)
    c = np.array([x[f // 4, fn[f % 4]].mean(axis=0) for f in faces])
    n = len(faces)
    for p in range(n):
        for q in range(n):
            for r in range(n):
                for s in range(n):
                    if len({p, q, r, s}) == 4 and np.allclose(c[q] - c[p], c[r] - c[s], atol=1e-12):
                        out = np.array(faces).copy()
                        out[p], out[r] = faces[q], faces[s]
                        return out
    raise AssertionError("no parallelogram of face centroids")


def test_link_errors_leave_operator_unchanged():
    tm = _tagged(2, 2, 3, 1.0, 1.0, 1.5)
    (fa, fb), = M.periodic_faces_of(tm, M.Model(periodic=[(1, 2)]))
    op = M.operator_from_model(tm, M.Model(), 2).op
    orc = R.Operator(tm.mesh.nodes, tm.mesh.tets, 2)
    nbr0 = op.get("nbr")
    interior = int(np.flatnonzero(nbr0 >= 0)[0])
    cases = {
        "different triangle counts": (fa, fb[:-1]),
        "not on the domain boundary": (np.concatenate([fa[:-1], [interior]]), fb),
        "no partner": (fa, M.periodic_faces_of(tm, M.Model(periodic=[(3, 4)]))[0][1]),
        "bijection": (_two_duplicates(op, fa), fb),
    }
    for msg, (a, b) in cases.items():
        with pytest.raises(RuntimeError, match=msg):
            op.link_periodic(a, b)
        with pytest.raises(ValueError):
            orc.link_periodic(a, b)
        assert np.array_equal(op.get("nbr"), nbr0), msg
    # a port face cannot also be periodic
    code = -np.ones((tm.n_tets, 4), dtype=np.int32)
    code.ravel()[fa[0]] = 0
    pop = O.MaxwellOperator(tm.mesh, 2, face_port=code)
    with pytest.raises(RuntimeError, match="both port and periodic"):
        pop.link_periodic(fa, fb)
    porc = R.Operator(tm.mesh.nodes, tm.mesh.tets, 2, face_port=code)
    with pytest.raises(ValueError, match="a port face"):
        porc.link_periodic(fa, fb)


def _plane_wave(xyz, t, lx):
    """E_y = H_z = sin(2 pi (x - t) / lx): a wave travelling along +x at c = 1;
    E_y is normal and H_z tangential on the y walls, so it is PEC-compatible
    there."""
    k = 2.0 * np.pi / lx
    s = np.sin(k * (xyz[:, 0] - t))
    y = np.zeros((xyz.shape[0], 6))
    y[:, 1] = s
    y[:, 5] = s
    return y.ravel()


def test_plane_wave_crosses_periodic_box():
    lx, ly, lz = 1.0, 0.5, 0.5
    tm = _tagged(4, 2, 2, lx, ly, lz)
    op, orc = _linked(tm, 3, [(1, 2), (5, 6)])
    walls = R.Operator(tm.mesh.nodes, tm.mesh.tets, 3)
    xyz = orc.node_coords()
    t_end, steps = 0.5, 250
    y0 = _plane_wave(xyz, 0.0, lx)
    exact = _plane_wave(xyz, t_end, lx)
    got = orc.lserk(y0, t_end / steps, steps)
    assert rel_l2(got, exact) < 5e-3
    # without the links the x and z walls are PEC and the wave does not travel
    assert rel_l2(walls.lserk(y0, t_end / steps, steps), exact) > 0.2


def test_periodic_with_port_and_plate_matches_oracle():
    """Periodic pairs in x next to an ABC port on z = lz and an internal PEC
    plate: the host build and the oracle agree on every face array, and the
    oracle's RHS differs from the same model without the pairs."""
    tm = _tagged(4, 2, 4, 1.0, 0.5, 1.0)
    tm.face_tags[20] = M.plane_triangles(tm.mesh, 2, 0.5, lo=(0.0, 0.0, 0.0), hi=(0.5, 0.5, 1.0))
    model = M.Model(faces=[M.AbcFace(6)], pec_tags=[20], periodic=[(1, 2)])
    mo = M.operator_from_model(tm, model, 2)
    orc = R.Operator(tm.mesh.nodes, tm.mesh.tets, 2, 1.0, face_port=mo.face_port, materials=mo.materials)
    for a, b in M.periodic_faces_of(tm, model):
        orc.link_periodic(a, b)
    for name in ("nbr", "nbr_lf", "perm", "port"):
        assert np.array_equal(mo.op.get(name), orc.get(name)), name
    plain = R.Operator(tm.mesh.nodes, tm.mesh.tets, 2, 1.0, face_port=mo.face_port, materials=mo.materials)
    y = np.sin(0.3 + 0.017 * np.arange(orc.n_dof))
    assert rel_l2(plain.apply(y), orc.apply(y)) > 1e-2


# The reference's periodic-boundary tests (rhs.rs:3261-3436 and :3437-3620),
# run on the oracle here and on the device in tests/test_gpu_periodic.py.

def _column(nx, ny, nz, lx, ly, lz, pairs, order=2):
    """The Kuhn box with the given periodic pairs of its face groups 1..6,
    central flux, as (host operator, oracle with the same links)."""
    tm = M.box_tagged(nx, ny, nz, lx, ly, lz)
    return _linked(tm, order, pairs, alpha=0.0)


def _packet(xyz, lz):
    """E_x = f(z), H_y = -f(z): a Gaussian TEM packet along the column, so the
    forward coherence sum(E_x (-H_y)) / sum(E_x^2) starts at 1."""
    f = np.exp(-((xyz[:, 2] - 0.5 * lz) / 0.40) ** 2)
    y = np.zeros((xyz.shape[0], 6))
    y[:, 0] = f
    y[:, 4] = -f
    return y.ravel()


def coherence(y):
    y = y.reshape(-1, 6)
    return float(np.sum(y[:, 0] * -y[:, 4]) / np.sum(y[:, 0] ** 2))


def test_periodic_column_passes_plane_wave_oracle():
    """rhs.rs:3261-3436: the packet crosses the periodic z pair as a clean
    forward wave (energy within 5e-3, coherence > 0.85 after 2.5 box
    periods), while PEC z walls reflect it (coherence lower by > 0.3)."""
    lz = 4.0
    _, per = _column(1, 1, 16, 0.5, 0.5, lz, [(1, 2), (3, 4), (5, 6)])
    _, pec = _column(1, 1, 16, 0.5, 0.5, lz, [(1, 2), (3, 4)])
    y0 = _packet(per.node_coords(), lz)
    assert abs(coherence(y0) - 1.0) < 1e-9
    zero = np.zeros_like(y0)
    yp, yc = y0.copy(), y0.copy()
    for _ in range(250):
        yp, _ = per.etd_step(yp, zero, 0.04, 24)
        yc, _ = pec.etd_step(yc, zero, 0.04, 24)
    assert np.all(np.isfinite(yp)) and np.all(np.isfinite(yc))
    e0 = per.field_energy(y0)
    assert abs(per.field_energy(yp) - e0) / e0 < 5e-3
    assert coherence(yp) > 0.85
    assert coherence(yp) - coherence(yc) > 0.3


def test_periodic_box_is_translation_invariant_oracle():
    """rhs.rs:3437-3620: a uniform E_x in a fully periodic box stays uniform
    (std < 1e-9 after 80 ETD steps); with PEC z walls it develops structure
    (std > 100x that)."""
    _, per = _column(1, 1, 4, 0.5, 0.5, 1.5, [(1, 2), (3, 4), (5, 6)])
    _, zpec = _column(1, 1, 4, 0.5, 0.5, 1.5, [(1, 2), (3, 4)])
    y0 = np.zeros(per.n_dof)
    y0[0::6] = 1.0
    zero = np.zeros_like(y0)
    ya, yz = y0.copy(), y0.copy()
    for _ in range(80):
        ya, _ = per.etd_step(ya, zero, 0.05, 18)
        yz, _ = zpec.etd_step(yz, zero, 0.05, 18)
    s_all, s_z = float(np.std(ya[0::6])), float(np.std(yz[0::6]))
    assert s_all < 1e-9
    assert s_z > 100.0 * s_all
