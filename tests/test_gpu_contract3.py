"""GPU parity of btod_contract3 and direct_block_tensor
(libtensor/block_tensor/btod_contract3.h:36, direct_block_tensor.h:22):

    D(i,j,k,l) = kd * sum_ab [ sum_cd t(i,j,c,d) V(a,b,c,d) ] t(k,l,a,b)

on the ladder o=10 v=40 tensors (antisymmetric pairs, spin blocks): the
three-tensor contraction with one batch and with the intermediate formed in
batches of V's blocks, against the reference's two btod_contract2 one after
the other (its btod_contract3 forms the same intermediate in batches), and a
direct block tensor of the first contraction used as an operand."""
import numpy as np
import pytest

from libtensor_b200 import spec as S
from libtensor_b200.core import (Context, block_tensor, btod_contract2, btod_contract3, contraction2,
                                 direct_block_tensor)
from oracle import refapi as R
from tests.helpers import block_errors, max_rel_block_error

pytestmark = [pytest.mark.gpu, pytest.mark.skipif(not R.available(), reason="oracle/_ref not built")]

TOL = 1e-13


@pytest.fixture(scope="module")
def setup():
    ctx = Context(0)
    cfg = S.LADDER_SMALL
    t, v = block_tensor(ctx, cfg.t_spec()), block_tensor(ctx, cfg.v_spec())
    t.fill_seeded(11, 0.1)
    v.fill_seeded(23, 1.0)
    rt, rv = R.RefBT(cfg.t_spec()), R.RefBT(cfg.v_spec())
    rt.fill_seeded(11, 0.1)
    rv.fill_seeded(23, 1.0)
    pairs = [(2, 2), (3, 3)]
    r1 = R.RefContract2(2, 2, 2, None, pairs, rt, rv)
    rab = r1.make_result()
    r1.perform(rab)
    r2 = R.RefContract2(2, 2, 2, None, pairs, rab, rt, 1.0, 1.0, 0.25)
    rd = r2.make_result()
    r2.perform(rd)
    yield ctx, t, v, rd
    ctx.close()


def _contr():
    return contraction2(2, 2, 2).contract(2, 2).contract(3, 3)


@pytest.mark.parametrize("batches", [1, 3])
def test_contract3_matches_reference(setup, batches):
    ctx, t, v, rd = setup
    op = btod_contract3(_contr(), _contr(), t, v, t, kd=0.25, batches=batches)
    d = op.make_result()
    op.perform(d)
    assert max_rel_block_error(block_errors(d, d.download(), rd, None)) <= TOL
    op.perform(d, 2.0)                              # D += 2 * (...): 3 x the result
    got = d.download()
    worst = 0.0
    for bidx, blk in d.blocks(got):
        r = rd.get_block(bidx, blk.shape)
        m = float(np.max(np.abs(r))) if r.size else 0.0
        if m > 0:
            worst = max(worst, float(np.max(np.abs(blk - 3.0 * r))) / (3.0 * m))
    assert worst <= TOL
    op.close()


def test_direct_block_tensor_as_operand(setup):
    ctx, t, v, rd = setup
    ab = direct_block_tensor(btod_contract2(_contr(), t, v))     # nothing computed yet
    op2 = btod_contract2(_contr(), ab, t, kc=0.25)                # reads ab: formed now
    d = op2.make_result()
    op2.perform(d)
    assert max_rel_block_error(block_errors(d, d.download(), rd, None)) <= TOL
