"""Batched instances on the device: every instance of an autotuned, graph-
captured batch ends where its own solo run with its own dt ends (the same to
the bit on the FP32 engine, to f32 rounding on the tensor-core engine), and
graph replays equal direct launches."""
import numpy as np
import pytest

from rapidfem_b200 import batch as B
from rapidfem_b200 import gpu as G
from rapidfem_b200 import operator as O
from rapidfem_b200._native import ENGINE_FP32

from .conftest import rel_l2

pytestmark = pytest.mark.gpu


@pytest.fixture(scope="module")
def ctx():
    return G.GpuContext(0)


def test_batch_matches_solo_runs(ctx):
    inst = B.random_cavities(8, seed=11, cells=(2, 4), orders=(2, 5))
    groups = B.build_groups(inst)
    B.initial_fields(groups, inst)
    B.assign_steps(ctx, groups, inst, iters=20)
    runner = B.BatchRunner(ctx, groups)
    tuning = runner.autotune(trial_steps=1)
    assert [t["order"] for t in tuning] == [g.order for g in groups]
    runner.capture(steps_per_graph=2)
    runner.run(4)
    got = runner.states(inst)
    runner.graph = None  # direct launches from the initial state
    runner.load()
    runner.run(4)
    direct = runner.states(inst)
    for a, b in zip(got, direct):
        assert np.array_equal(a, b)
    for g, t in zip(groups, tuning):
        for j, i in enumerate(g.members):
            solo = G.GpuOperator(ctx, O.MaxwellOperator(O.structured_box(inst[i].cells, inst[i].cells,
                                                                         inst[i].cells), g.order, 1.0,
                                                        materials=inst[i].materials))
            solo.set_engine(ENGINE_FP32 if t["engine"] == "fp32" else 1)
            solo.upload(g.y0[g.dof_slice(j)])
            solo.run_lserk(np.float32(inst[i].dt), 4)
            want = solo.download()
            if t["engine"] == "fp32":
                assert np.array_equal(got[i], want)
            else:
                assert rel_l2(got[i], want) < 1e-6
            assert np.all(np.isfinite(got[i])) and np.max(np.abs(got[i])) > 0
