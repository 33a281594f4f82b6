"""Batched instances (host side): the order groups are disjoint unions of the
instances (no face couples two instances; every element keeps its own
geometry, materials and step), checked against per-instance host builds."""
import numpy as np

from rapidfem_b200 import batch as B
from rapidfem_b200 import operator as O


def test_groups_are_disjoint_unions():
    inst = B.random_cavities(7, seed=5, cells=(2, 3), orders=(2, 3))
    groups = B.build_groups(inst)
    assert sorted(i for g in groups for i in g.members) == list(range(7))
    for g in groups:
        nbr = g.op.get("nbr").reshape(-1, 4)
        jinv = g.op.get("jinv").reshape(-1, 9)
        ieps = g.op.get("inv_eps").reshape(-1, 3)
        for j, i in enumerate(g.members):
            a, b = g.elem_off[j], g.elem_off[j + 1]
            own = nbr[a:b]
            assert np.all((own == -1) | ((own >= a) & (own < b)))  # no face leaves the instance
            solo = O.MaxwellOperator(O.structured_box(inst[i].cells, inst[i].cells, inst[i].cells), g.order, 1.0,
                                     materials=inst[i].materials)
            assert np.array_equal(jinv[a:b], solo.get("jinv").reshape(-1, 9))
            assert np.array_equal(ieps[a:b], solo.get("inv_eps").reshape(-1, 3))
            assert np.array_equal(np.where(own >= 0, own - a, -1), solo.get("nbr").reshape(-1, 4))
    B.initial_fields(groups, inst)
    for g in groups:
        assert g.y0.dtype == np.float32 and g.y0.size == g.n_dof and np.max(g.y0) > 0.5
