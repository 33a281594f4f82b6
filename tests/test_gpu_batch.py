"""Batched instances on the device: every instance of an autotuned, graph-
captured batch ends where its own solo run with its own dt on the engine the
autotuner chose ends (the same to the bit on both FP32 engines, to f32
rounding on the tensor-core engine), and graph replays equal direct launches."""
import numpy as np
import pytest

from rapidfem_b200 import batch as B
from rapidfem_b200 import gpu as G
from rapidfem_b200 import operator as O
from rapidfem_b200._native import ENGINE_FP32, ENGINE_FP32_SMALL_TILES, ENGINE_TF32X3

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
            engine = {"fp32": ENGINE_FP32, "fp32_small_tiles": ENGINE_FP32_SMALL_TILES,
                      "tf32x3": ENGINE_TF32X3}[t["engine"]]
            solo.set_engine(engine)
            solo.upload(g.y0[g.dof_slice(j)])
            solo.run_lserk(np.float32(inst[i].dt), 4)
            want = solo.download()
            if engine != ENGINE_TF32X3:
                assert np.array_equal(got[i], want)
            else:
                assert rel_l2(got[i], want) < 1e-6
            assert np.all(np.isfinite(got[i])) and np.max(np.abs(got[i])) > 0


def test_batch_instances_match_oracle():
    """One instance of every order (2..5) of an autotuned, graph-replayed batch
    of uneven cavities against the f64 oracle run alone with that instance's
    own dt and initial field: 500 LSERK4 steps (explicit.rs:100-135), relative
    L2 < 1e-4 at the final step."""
    from oracle import oracle as R

    inst = B.random_cavities(12, seed=5, cells=(2, 4), orders=(2, 5))
    assert {i.order for i in inst} == {2, 3, 4, 5}
    groups = B.build_groups(inst)
    B.initial_fields(groups, inst)
    B.assign_steps(ctx_holder := G.GpuContext(0), groups, inst, iters=20)
    runner = B.BatchRunner(ctx_holder, groups)
    runner.autotune(trial_steps=1)
    runner.capture(steps_per_graph=10)
    steps = 500
    runner.run(steps)
    got = runner.states(inst)
    for g in groups:
        j = len(g.members) - 1  # the last member: a nonzero element offset in the group
        i = g.members[j]
        n = inst[i].cells
        nodes, tets = R.box_mesh(n, n, n, 1.0, 1.0, 1.0)
        orc = R.Operator(nodes, tets, g.order, 1.0, materials=inst[i].materials)
        y0 = g.y0[g.dof_slice(j)].astype(np.float64)
        want = orc.lserk(y0, float(np.float32(inst[i].dt)), steps)
        assert rel_l2(got[i], want) < 1e-4, (g.order, rel_l2(got[i], want))
        assert np.max(np.abs(want)) > 1e-3 * np.max(np.abs(y0))
