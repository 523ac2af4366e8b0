"""The flop count behind every TFLOP/s figure, pinned to the reference.

The product's `flops()` (ltg_plan_flops) must equal 2 x the schedule's work as
the reference's task cost counts it: for every scheduled C block and every
pair of its coalesced pair list, the product of A's block extents on the
indices contracted with B times the C block's size
(libtensor/gen_block_tensor/impl/gen_bto_contract2_block_impl.h:63-95, summed
before that function's per-pair division by 1000).  No GPU is needed: the
schedule is host work on both sides."""
import numpy as np
import pytest

from libtensor_b200 import spec as S
from libtensor_b200.core import Context, block_tensor, btod_contract2, contraction2
from oracle import refapi as R
from tests.cases import cases

pytestmark = pytest.mark.skipif(not R.available(), reason="oracle/_ref not built")

CASES = [c for c in cases() if not c.symmetry_error]


def _ref_with_blocks(spec, t, zero=()):
    """Reference tensor with every canonical allowed block non-zero (ones)."""
    r = R.RefBT(spec)
    zero = {tuple(z) for z in zero}
    for s in range(t.nblocks):
        bidx = tuple(t.block_index(t.abs_idx[s]))
        if bidx not in zero:
            r.set_block(bidx, np.ones(tuple(spec.block_extent(d, b) for d, b in enumerate(bidx))))
    return r


@pytest.fixture(scope="module")
def hctx():
    c = Context(-1)
    yield c
    c.close()


def _pair(hctx, a_spec, b_spec, n, m, k, permc, pairs, ka=1.0, kb=1.0, kc=1.0, zero_a=()):
    A, B = block_tensor(hctx, a_spec), block_tensor(hctx, b_spec)
    A.mark_nonzero(); B.mark_nonzero()
    for z in zero_a:
        A.zero_block(z)
    contr = contraction2(n, m, k, permc)
    for p in pairs:
        contr.contract(*p)
    op = btod_contract2(contr, A, B, ka, kb, kc)
    ra, rb = _ref_with_blocks(a_spec, A, zero_a), _ref_with_blocks(b_spec, B)
    rop = R.RefContract2(n, m, k, permc, pairs, ra, rb, ka, kb, kc)
    return op, rop


@pytest.mark.parametrize("case", CASES, ids=[c.name for c in CASES])
def test_flops_equal_reference_cost(hctx, case):
    op, rop = _pair(hctx, case.a, case.b, case.n, case.m, case.k, case.permc, case.pairs,
                    case.ka, case.kb, case.kc, case.zero_a)
    exact, ref_cost = rop.cost()
    assert op.get_schedule() == rop.schedule()
    assert op.flops() == 2 * exact
    # the reference's own summands (integer division per pair) never exceed it
    assert 1000 * ref_cost <= exact


def _cfg_pair(hctx, cfg):
    c = cfg.contraction
    b_spec = cfg.v_spec() if hasattr(cfg, "v_spec") else cfg.w_spec()
    return _pair(hctx, cfg.t_spec(), b_spec, c["n"], c["m"], c["k"], c["permc"], c["pairs"], kc=cfg.kc)


@pytest.mark.parametrize("cfg", [S.RING_D2H, S.RING_D2H_SMALL, S.LadderConfig("fine ladder", [2, 2], [3] * 5)],
                         ids=["ring D2h o=46 v=296", "ring D2h small", "fine ladder"])
def test_flops_equal_reference_cost_workloads(hctx, cfg):
    """The ring workload at its full size (3072 C blocks, uneven 1-40 blocks)
    and a finely blocked ladder whose pair lists are coalesced."""
    op, rop = _cfg_pair(hctx, cfg)
    exact, _ = rop.cost()
    assert op.flops() == 2 * exact
