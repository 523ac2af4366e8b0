"""Host-side symmetry of a sum's intermediate (ltg_bt_create_sum_space, no
GPU): the block index space of the terms and the symmetry they all have --
common permutational elements, and partition or label rules only when every
term carries the same ones."""
import ctypes as C

import numpy as np
import pytest

from libtensor_b200 import spec as S
from libtensor_b200._capi import LtgError, check, lib
from libtensor_b200.core import Context, block_tensor
from libtensor_b200.spec import BTSpec, permuted_spec


@pytest.fixture(scope="module")
def hctx():
    c = Context(-1)
    yield c
    c.close()


def _sum_space(ctx, terms):
    hs = (C.c_void_p * len(terms))(*[t.h for t, _ in terms])
    n = terms[0][0].order if hasattr(terms[0][0], "order") else len(terms[0][0].bidims)
    perms = []
    for _, p in terms:
        perms += list(p) if p is not None else list(range(n))
    pa = (C.c_int32 * len(perms))(*perms)
    h = C.c_void_p()
    check(lib().ltg_bt_create_sum_space(len(terms), hs, pa, C.byref(h)))
    return block_tensor(ctx, None, _handle=h)


def _orbits(t):
    return [t.orbit(a) for a in range(int(np.prod(t.bidims)))]


def test_sum_of_equal_symmetries_keeps_them(hctx):
    cfg = S.LADDER_SMALL
    t = block_tensor(hctx, cfg.t_spec())
    u = _sum_space(hctx, [(t, None), (t, (1, 0, 3, 2))])
    assert _orbits(u) == _orbits(t)
    assert list(u.abs_idx) == list(t.abs_idx)


def test_sum_with_spin_only_term_drops_permutations(hctx):
    cfg = S.LADDER_SMALL
    t = block_tensor(hctx, cfg.t_spec())
    x = block_tensor(hctx, cfg.x_spec())          # spin blocks only
    u = _sum_space(hctx, [(t, None), (x, None)])
    assert _orbits(u) == _orbits(x)


def test_sum_with_other_partitions_allows_every_block(hctx):
    cfg = S.LADDER_SMALL
    t = block_tensor(hctx, cfg.t_spec())
    plain = block_tensor(hctx, BTSpec(dims=t.spec.dims, splits=t.spec.splits,
                                      perms=S.antisym_pairs(4, [(0, 1), (2, 3)])))
    u = _sum_space(hctx, [(t, None), (plain, None)])
    assert _orbits(u) == _orbits(plain)
    assert all(o[3] for o in _orbits(u))          # every block allowed


def test_sum_of_permuted_terms(hctx):
    """P_0 sets the space: the sum of P(0,2,1,3) t and a tensor already in
    that order has the permuted space and the common symmetry."""
    cfg = S.LADDER_SMALL
    t = block_tensor(hctx, cfg.t_spec())
    tp = block_tensor(hctx, permuted_spec(cfg.t_spec(), (0, 2, 1, 3)))
    u = _sum_space(hctx, [(t, (0, 2, 1, 3)), (tp, None)])
    assert _orbits(u) == _orbits(tp)


def test_sum_of_different_spaces_is_rejected(hctx):
    t = block_tensor(hctx, S.LADDER_SMALL.t_spec())
    v = block_tensor(hctx, S.LADDER_SMALL.v_spec())
    with pytest.raises(LtgError) as ei:
        _sum_space(hctx, [(t, None), (v, None)])
    assert ei.value.code == 2                     # LTG_ERR_BAD_DIMS
