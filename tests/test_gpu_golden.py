"""GPU path against the committed golden fixtures (tests/golden, produced by
the reference compiled from its sources).  Needs no reference library at run
time: inputs are regenerated on the device by the seeded generator."""
import numpy as np
import pytest

from libtensor_b200.core import (Context, block_tensor, btod_add, btod_contract2, btod_copy,
                                 btod_dotprod, contraction2, MODE_PLAIN_FP64)
from libtensor_b200.spec import permuted_spec
from tests.golden.make_golden import SEED_A, SEED_B, transfer_specs
from tests.test_golden import CASES, T, TOL, _transfer_golden, golden_blocks, rel_err

pytestmark = pytest.mark.gpu


@pytest.fixture(scope="module")
def gctx():
    c = Context(0)
    yield c
    c.close()


def _device_tensor(ctx, spec, seed, scale, zero=()):
    t = block_tensor(ctx, spec)
    t.fill_seeded(seed, scale)
    for z in zero:
        t.zero_block(z)
    return t


@pytest.mark.parametrize("i", range(len(CASES)), ids=[c.name for c in CASES])
def test_contract2_matches_golden(gctx, i):
    case = CASES[i]
    A = _device_tensor(gctx, case.a, SEED_A, case.a_scale, case.zero_a)
    B = _device_tensor(gctx, case.b, SEED_B, case.b_scale)
    contr = contraction2(case.n, case.m, case.k, case.permc)
    for p in case.pairs:
        contr.contract(*p)
    op = btod_contract2(contr, A, B, case.ka, case.kb, case.kc)
    C = op.make_result()
    op.perform(C, mode=MODE_PLAIN_FP64)
    gold = golden_blocks(i)
    assert C.nonzero() == sorted(gold)
    arena = C.download()
    for bidx, blk in C.blocks(arena):
        a = C.abs_index(bidx)
        if a in gold:
            assert rel_err(blk, gold[a]) <= TOL, (case.name, a)
        else:
            assert not np.any(blk), (case.name, a)
    for t in (C, A, B):
        t.close()
    op.close()


def test_transfers_match_golden(gctx):
    t_spec, x_spec = transfer_specs()
    ta = _device_tensor(gctx, t_spec, 3, 0.01)
    tb = ta.permuted((0, 2, 1, 3))
    btod_copy(ta, (0, 2, 1, 3), -0.5).perform(tb)
    gold = _transfer_golden("copy", permuted_spec(t_spec, (0, 2, 1, 3)))
    arena = tb.download()
    got = {tuple(b): blk for b, blk in tb.blocks(arena)}
    for bidx, blk in gold.items():
        assert np.array_equal(got[bidx], blk), bidx          # bit-exact copy

    xa = _device_tensor(gctx, x_spec, 4, 1.0)
    xb = _device_tensor(gctx, x_spec, 5, 1.0)
    xc = block_tensor(gctx, x_spec)
    op = btod_add(xa, None, 1.0)
    op.add_op(xb, (1, 0, 3, 2), -0.5)
    op.add_op(xa, (1, 0, 3, 2), 0.25)
    op.perform(xc)
    arena = xc.download()
    got = {tuple(b): blk for b, blk in xc.blocks(arena)}
    for bidx, blk in _transfer_golden("add", x_spec).items():
        assert rel_err(got[bidx], blk) <= 1e-15, bidx

    d1 = btod_dotprod(ta, None, ta, None).calculate()
    assert abs(d1 - T["dot_t_t"][0]) <= 1e-13 * abs(T["dot_t_t"][0])
    d2 = btod_dotprod(xa, None, xb, (1, 0, 3, 2)).calculate()
    assert abs(d2 - T["dot_x_xp"][0]) <= 1e-13 * abs(T["dot_x_xp"][0])
    for t in (ta, tb, xa, xb, xc):
        t.close()
