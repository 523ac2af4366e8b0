"""Bounded device waits of the tcgen05 products kernels.

Every mbarrier wait of the split-precision products kernels (crt.cu,
ozaki.cu) is bounded by the context's wait limit.  With a limit of 0 a wait
whose phase has not completed at its first test gives up: the kernel sets the
context's error word, lets its bulk copies and MMAs in flight finish, frees
its tensor memory and returns.  The host then reports LTG_ERR_TIMEOUT once
(at synchronisation), and the context stays usable: with the default limit
the next call gives the same bits as before."""
import numpy as np
import pytest

from libtensor_b200 import spec as S
from libtensor_b200._capi import LtgError
from libtensor_b200.core import (MODE_OZAKI_CRT, MODE_OZAKI_INT8, Context, block_tensor, btod_contract2,
                                 contraction2)

pytestmark = pytest.mark.gpu

LTG_ERR_TIMEOUT = 7
DEFAULT_NS = 2_000_000_000


@pytest.fixture(scope="module")
def gctx():
    c = Context(0)
    yield c
    c.close()


@pytest.mark.parametrize("mode,nslices", [(MODE_OZAKI_CRT, 13), (MODE_OZAKI_INT8, 7)], ids=["crt13", "int8x7"])
def test_zero_wait_limit_times_out_and_context_recovers(gctx, mode, nslices):
    cfg = S.LADDER_SMALL
    A, B = block_tensor(gctx, cfg.t_spec()), block_tensor(gctx, cfg.v_spec())
    A.fill_seeded(11, cfg.t_scale)
    B.fill_seeded(23, cfg.v_scale)
    c = cfg.contraction
    contr = contraction2(c["n"], c["m"], c["k"], c["permc"])
    for p in c["pairs"]:
        contr.contract(*p)
    op = btod_contract2(contr, A, B, kc=cfg.kc)
    C = op.make_result()
    assert gctx.wait_limit() == DEFAULT_NS
    op.perform(C, mode=mode, nslices=nslices)
    gctx.synchronize()
    good = C.download().copy()

    gctx.set_wait_limit(0)
    try:
        op.perform(C, mode=mode, nslices=nslices)
        with pytest.raises(LtgError) as ei:
            gctx.synchronize()
        assert ei.value.code == LTG_ERR_TIMEOUT
    finally:
        gctx.set_wait_limit(DEFAULT_NS)
    gctx.synchronize()                       # reported once, then cleared

    op.perform(C, mode=mode, nslices=nslices)
    gctx.synchronize()
    assert np.array_equal(C.download().view(np.uint64), good.view(np.uint64))
    for x in (C, A, B):
        x.close()
    op.close()
