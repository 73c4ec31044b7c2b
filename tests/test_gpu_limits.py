"""Bounded loops of the tree build: a bound that runs out ends the build with
TSR_ERR_TIMEOUT and leaves the device usable.

The sampling pass resolves each round's conflicts in waves inside one
cooperative launch; its wave loop stops at the bound set by
tsr_set_iteration_limits, records the fact and returns, and the host reports
it before anything of the round is applied.  The host-side round loops have
their own bound.  Both are made to run out here on purpose: the failure is a
bounded loop that ends, not a fault.
"""
import numpy as np
import pytest

pytestmark = pytest.mark.gpu

TSR_ERR_TIMEOUT = 6


def _build(scene):
    from tsr_b200 import core
    return core.Tree(core.Samples.from_scene(scene))


def test_wave_bound_runs_out_and_device_stays_usable(csg_small):
    from tsr_b200 import core
    ref = _build(csg_small)
    # some round needs more than one conflict wave, so a bound of one runs out
    assert ref.counts["sampling_waves"] > ref.counts["sampling_rounds"], ref.counts
    core.set_iteration_limits(max_sampling_waves=1)
    try:
        with pytest.raises(core.TsrError) as e:
            _build(csg_small)
    finally:
        core.set_iteration_limits()
    assert e.value.status == TSR_ERR_TIMEOUT
    assert "waves" in str(e.value)
    again = _build(csg_small)
    np.testing.assert_array_equal(again.getNodes().children, ref.getNodes().children)
    np.testing.assert_array_equal(again.getDualCells(), ref.getDualCells())


def test_round_bound_runs_out(csg_small):
    from tsr_b200 import core
    ref = _build(csg_small)
    assert ref.counts["sampling_rounds"] > 1
    core.set_iteration_limits(max_rounds=1)
    try:
        with pytest.raises(core.TsrError) as e:
            _build(csg_small)
    finally:
        core.set_iteration_limits()
    assert e.value.status == TSR_ERR_TIMEOUT
    again = _build(csg_small)
    np.testing.assert_array_equal(again.getNodes().children, ref.getNodes().children)
