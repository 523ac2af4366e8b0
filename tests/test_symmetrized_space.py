"""The result space of a symmetrizer fused into a contraction (no GPU):
ltg_contract2_make_symmetrized builds, from the plan alone, the same block
space and canonical blocks as ltg_bt_create_symmetrized over the
contraction's result tensor (btod_symmetrize2 over btod_contract2,
libtensor/block_tensor/btod_symmetrize2.h:19), for index pairs and a unitary
pair exchange, symmetric and antisymmetric, on the ring and the ladder."""
import numpy as np
import pytest

from libtensor_b200 import spec as S
from libtensor_b200.core import Context, block_tensor, btod_contract2, btod_symmetrize, contraction2

CASES = [dict(symm=False, idx=(0, 1)), dict(symm=True, idx=(2, 3)), dict(symm=False, perm=(1, 0, 3, 2)),
         dict(symm=True, perm=(1, 0, 3, 2))]
IDS = ["asymm(0,1)", "symm(2,3)", "asymm P(01)P(23)", "symm P(01)P(23)"]


@pytest.fixture(scope="module")
def hctx():
    c = Context(-1)
    yield c
    c.close()


def _op(ctx, cfg):
    c = cfg.contraction
    A = block_tensor(ctx, cfg.t_spec())
    B = block_tensor(ctx, cfg.v_spec() if hasattr(cfg, "v_spec") else cfg.w_spec())
    A.mark_nonzero()
    B.mark_nonzero()
    contr = contraction2(c["n"], c["m"], c["k"], c["permc"])
    for p in c["pairs"]:
        contr.contract(*p)
    return btod_contract2(contr, A, B, kc=cfg.kc), (A, B)


@pytest.mark.parametrize("kw", CASES, ids=IDS)
@pytest.mark.parametrize("cfg", [S.RING_D2H_SMALL, S.LADDER_SMALL], ids=["ring", "ladder"])
def test_fused_space_equals_symmetrizer_space(hctx, cfg, kw):
    op, keep = _op(hctx, cfg)
    fused = op.make_symmetrized(**kw)
    T = op.make_result()
    unfused = btod_symmetrize(T, **kw).make_result()
    assert fused.order == unfused.order
    assert np.array_equal(fused.abs_idx, unfused.abs_idx)
    assert np.array_equal(fused.sizes, unfused.sizes)
    for t in (fused, unfused, T, op, *keep):
        t.close()


def test_fused_symmetrizer_needs_a_device(hctx):
    """On a host-only context the fused symmetrizer reports an error instead
    of running (there is no CPU path)."""
    op, keep = _op(hctx, S.RING_D2H_SMALL)
    r = op.make_symmetrized(False, idx=(0, 1))
    with pytest.raises(Exception):
        op.perform_symmetrized(r, False, idx=(0, 1))
    for t in (r, op, *keep):
        t.close()
