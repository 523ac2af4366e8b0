"""Edge cases of the GPU path against the reference: an operand with no
non-zero block (empty schedule: assign zeroes C, add leaves it), a dot
product of zero tensors, and the error codes of invalid calls."""
import numpy as np
import pytest

from libtensor_b200._capi import LtgError
from libtensor_b200.core import (MODE_OZAKI_CRT, MODE_PLAIN_FP64, Context, block_tensor, btod_contract2,
                                 btod_dotprod, contraction2)
from libtensor_b200 import spec as S
from oracle import refapi as R
from tests.cases import cases
from tests.helpers import seeded_pair

pytestmark = [pytest.mark.gpu, pytest.mark.skipif(not R.available(), reason="oracle/_ref not built")]

CASES = [c for c in cases() if not c.symmetry_error]


@pytest.fixture(scope="module")
def gctx():
    c = Context(0)
    yield c
    c.close()


def _op(gctx, case, zero_a):
    if zero_a:
        A = block_tensor(gctx, case.a)
        A.set_zero()
        ra = R.RefBT(case.a)                     # no blocks set: all zero
    else:
        A, ra, _ = seeded_pair(gctx, case.a, 41, case.a_scale, case.zero_a)
    B, rb, _ = seeded_pair(gctx, case.b, 42, case.b_scale)
    contr = contraction2(case.n, case.m, case.k, case.permc)
    for p in case.pairs:
        contr.contract(*p)
    op = btod_contract2(contr, A, B, case.ka, case.kb, case.kc)
    rop = R.RefContract2(case.n, case.m, case.k, case.permc, case.pairs, ra, rb, case.ka, case.kb, case.kc)
    return op, rop


@pytest.mark.parametrize("mode,S_", [(MODE_PLAIN_FP64, 0), (MODE_OZAKI_CRT, 13)], ids=["plain", "crt13"])
@pytest.mark.parametrize("case", CASES, ids=[c.name for c in CASES])
def test_zero_operand_gives_empty_schedule(gctx, case, mode, S_):
    op, rop = _op(gctx, case, zero_a=True)
    assert op.get_schedule() == [] == rop.schedule()
    C = op.make_result()
    C.upload(np.full(max(1, C.nelems), 3.0)[:C.nelems])
    op.perform(C, 1.0, mode=mode, nslices=S_)               # add: C unchanged
    assert all(np.all(blk == 3.0) for _, blk in C.blocks(C.download()))
    op.perform(C, mode=mode, nslices=S_)                    # assign: C = 0
    assert not any(np.any(blk) for _, blk in C.blocks(C.download()))
    assert C.nonzero() == []


def test_dot_of_zero_tensors_is_zero(gctx):
    spec = S.LADDER_SMALL.t_spec()
    A, B = block_tensor(gctx, spec), block_tensor(gctx, spec)
    A.set_zero()
    B.set_zero()
    assert btod_dotprod(A, None, B, (1, 0, 3, 2)).calculate() == 0.0


def test_invalid_calls_report_errors(gctx):
    case = CASES[0]
    op, _ = _op(gctx, case, zero_a=False)
    C = op.make_result()
    with pytest.raises(LtgError) as e:
        op.perform(C, mode=99)
    assert "BAD_ARG" in str(e.value)
    with pytest.raises(LtgError) as e:
        op.perform(C, mode=MODE_OZAKI_CRT, nslices=5)      # 8..16 moduli
    assert "BAD_ARG" in str(e.value)
    other = block_tensor(gctx, S.LADDER_SMALL.v_spec())     # a different block index space
    with pytest.raises(LtgError) as e:
        op.perform(other)
    assert "BAD_DIMS" in str(e.value)
    op.perform(C)                                           # the plan still works afterwards
