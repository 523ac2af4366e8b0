"""GPU: a contraction uploaded as a caller-built task list
(ltg_plan_contract2_upload) runs the plain FP64 kernels on exactly the
products of the plan it was exported from, so both give identical bits;
subsets and rescaled tasks match a numpy evaluation of the same list; task
lists that would make C blocks overlap are rejected before any launch."""
import numpy as np
import pytest

from libtensor_b200.core import Context, MODE_OZAKI_CRT, contract2_task_plan
from libtensor_b200._capi import LtgError
from tests.cases import cases
from tests.test_task_lists import _setup, apply_tasks

pytestmark = pytest.mark.gpu
CASES = [c for c in cases() if not c.symmetry_error]


@pytest.fixture(scope="module")
def gctx():
    c = Context(0)
    yield c
    c.close()


@pytest.mark.parametrize("case", CASES, ids=[c.name for c in CASES])
def test_uploaded_tasks_match_the_plan_bitwise(gctx, case):
    A, B, _, _, _, _, op = _setup(gctx, case)
    op.set_grouping(False)
    C1 = op.make_result()
    op.perform(C1)
    C2 = op.make_result()
    plan = contract2_task_plan(A, B, op.export_tasks(C2), case.ka, case.kb, case.kc)
    plan.perform(C2)
    x1, x2 = C1.download(), C2.download()
    assert np.array_equal(x1.view(np.int64), x2.view(np.int64))
    # accumulate: C += 0.75 * contr(A, B) on both
    op.perform(C1, 0.75)
    plan.perform(C2, 0.75)
    assert np.array_equal(C1.download().view(np.int64), C2.download().view(np.int64))
    plan.close()


def test_subset_of_rescaled_tasks_matches_numpy(gctx):
    case = CASES[0]
    A, B, _, _, arena_a, arena_b, op = _setup(gctx, case)
    C_ = op.make_result()
    tasks = op.export_tasks(C_)
    # the tasks of the first three C blocks, coefficients times 2.5
    starts = np.flatnonzero(np.r_[True, tasks[1:, 0] != tasks[:-1, 0]])
    sub = tasks[:starts[3] if len(starts) > 3 else len(tasks)].copy()
    coeff = sub[:, 42].view(np.float64) * 2.5
    sub[:, 42] = coeff.view(np.int64)
    C_.upload(np.full(C_.nelems, 7.0))          # assign mode overwrites everything
    plan = contract2_task_plan(A, B, sub, 0.5, 1.0, -2.0)
    plan.perform(C_)
    want = apply_tasks(sub, arena_a, arena_b, C_.nelems, -1.0)
    got = C_.download()
    for off, size in zip(C_.offsets, C_.sizes):
        w, g = want[off:off + size], got[off:off + size]
        assert np.max(np.abs(g - w)) <= 1e-13 * max(1.0, np.max(np.abs(w)))
    plan.close()


def test_overlapping_or_misplaced_blocks_are_rejected(gctx):
    case = CASES[0]
    A, B, _, _, _, _, op = _setup(gctx, case)
    C_ = op.make_result()
    tasks = op.export_tasks(C_)
    starts = np.flatnonzero(np.r_[True, tasks[1:, 0] != tasks[:-1, 0]])
    assert len(starts) >= 2
    # the first C block's tasks again after the second block's
    again = np.concatenate([tasks[:starts[2] if len(starts) > 2 else len(tasks)], tasks[:1]])
    plan = contract2_task_plan(A, B, again)
    with pytest.raises(LtgError, match="consecutive"):
        plan.perform(C_)
    plan.close()
    # c_off inside a block
    shifted = tasks[:1].copy()
    shifted[0, 0] += 1
    plan = contract2_task_plan(A, B, shifted)
    with pytest.raises(LtgError):
        plan.perform(C_)
    with pytest.raises(LtgError, match="plain FP64"):
        plan.perform(C_, mode=MODE_OZAKI_CRT)
    plan.close()
