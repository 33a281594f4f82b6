"""Host side of the probed state-space assembly: the distance-2 element
colouring that lets one probe recover a column of every element of a colour
(no two elements of a colour are face neighbours or share one)."""
import numpy as np

from rapidfem_b200 import operator as O
from rapidfem_b200 import partition as PT
from rapidfem_b200.td import _distance2_colors


def test_distance2_colouring():
    mesh = O.structured_box_jittered(4, 3, 3, 1.0, 0.8, 0.9, 0.1, 7)
    nbr = PT.face_neighbours(mesh.tets)
    color = _distance2_colors(nbr)
    assert color.min() == 0 and color.max() < 17  # at most 1 + 4 + 4 * 3 conflicts
    for e in range(nbr.shape[0]):
        sten = [e] + [int(x) for x in nbr[e] if x >= 0]
        # every stencil holds each colour at most once
        assert len({int(color[x]) for x in sten}) == len(sten)
