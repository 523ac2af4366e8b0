"""Host-side planning of grouped modular products (no GPU): which C blocks
the modular mode computes as grouped products, and how much work the
grouped products do compared with the blocks' algorithmic flops."""
import pytest

from libtensor_b200 import spec as S
from libtensor_b200.core import Context, block_tensor, btod_contract2, contraction2


@pytest.fixture(scope="module")
def hctx():
    c = Context(-1)
    yield c
    c.close()


def _op(ctx, cfg, a_spec, b_spec):
    A, B = block_tensor(ctx, a_spec), block_tensor(ctx, b_spec)
    A.mark_nonzero()
    B.mark_nonzero()
    c = cfg.contraction
    contr = contraction2(c["n"], c["m"], c["k"], c["permc"])
    for p in c["pairs"]:
        contr.contract(*p)
    op = btod_contract2(contr, A, B, 1.0, 1.0, cfg.kc)
    return op, op.make_result(), (A, B)


def test_ring_d2h_is_grouped_per_irrep_and_spin_class(hctx):
    # one grouped product per irrep (8) and spin class (aa/bb rows with aa/bb
    # columns, ab rows with ba columns, ba rows with ab columns)
    cfg = S.RING_D2H
    op, C, _ = _op(hctx, cfg, cfg.t_spec(), cfg.w_spec())
    ng, nb, gflops, bflops = op.group_info(C)
    assert ng == 24
    assert nb == len(op.get_schedule()) == 3072
    assert bflops == pytest.approx(14779424320.0)
    assert bflops <= gflops <= 1.01 * bflops       # padding of contracted blocks to 4 only


def test_coalesced_ladder_is_not_grouped(hctx):
    # the ladder's pair lists are coalesced (c <-> d), so a grouped product
    # would repeat the merged pairs
    cfg = S.LADDER_SMALL
    op, C, _ = _op(hctx, cfg, cfg.t_spec(), cfg.v_spec())
    assert op.group_info(C) == (0, 0, 0.0, 0.0)


def test_grouping_switch(hctx):
    cfg = S.RING_D2H_SMALL
    op, C, _ = _op(hctx, cfg, cfg.t_spec(), cfg.w_spec())
    ng, nb, gflops, bflops = op.group_info(C)
    assert ng > 0 and 0 < nb <= len(op.get_schedule())
    assert gflops <= 1.5 * bflops                    # groups doing more work stay per block
    op.set_grouping(False)
    assert op.group_info(C)[0] == 0
    op.set_grouping(True)
    assert op.group_info(C)[0] == ng
