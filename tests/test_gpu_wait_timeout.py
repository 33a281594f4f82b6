"""The tensor-core kernels' bounded waits, made to run out on purpose: one
thread waits, with the kernels' own wait helper, on an mbarrier that nothing
arrives on, gives up at its poll limit, and the host gets DGTD_ERR_TIMEOUT
through the same device flag a stage kernel raises.  Nothing faults, and the
context keeps working afterwards."""
import numpy as np
import pytest

from rapidfem_b200 import gpu as G
from rapidfem_b200 import operator as O
from rapidfem_b200._native import DgtdError

pytestmark = pytest.mark.gpu

TIMEOUT = 4  # DGTD_ERR_TIMEOUT
KERNEL_LIMIT = 2**19  # polls per wait in the stage kernels


@pytest.fixture(scope="module")
def ctx():
    return G.GpuContext(0)


def test_wait_gives_up_after_its_polls(ctx):
    with pytest.raises(DgtdError) as ei:
        ctx.wait_timeout_probe(max_polls=300)
    assert ei.value.code == TIMEOUT
    assert ei.value.waited_s < 0.5


def test_kernel_wait_limit_is_seconds_not_minutes(ctx):
    # a failed poll suspends the thread for a hardware time limit (~4 us), so
    # the kernels' poll limit is a wall-clock limit of about 2 s
    with pytest.raises(DgtdError) as ei:
        ctx.wait_timeout_probe(max_polls=KERNEL_LIMIT)
    assert ei.value.code == TIMEOUT
    assert 0.2 < ei.value.waited_s < 10.0


def test_context_usable_after_timeouts(ctx):
    with pytest.raises(DgtdError):
        ctx.wait_timeout_probe(max_polls=1000)
    prod = O.MaxwellOperator(O.structured_box(2, 2, 2), 3, 1.0)
    gop = G.GpuOperator(ctx, prod)
    y = np.sin(0.3 + 0.017 * np.arange(gop.n_dof()))
    for engine in (0, 1):
        gop.set_engine(engine)
        out = gop.apply(y)
        assert np.all(np.isfinite(out)) and np.linalg.norm(out) > 0


def test_probe_rejects_bad_limits(ctx):
    with pytest.raises(DgtdError):
        ctx.wait_timeout_probe(max_polls=0)
    with pytest.raises(DgtdError):
        ctx.wait_timeout_probe(max_polls=KERNEL_LIMIT + 1)
