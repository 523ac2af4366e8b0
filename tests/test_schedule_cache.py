"""The process-wide schedule cache (no GPU): a btod_contract2 built again from
operands of the same description (block index spaces, symmetry, non-zero
blocks) reuses the schedule -- identical to the reference's, and to the one
built from scratch -- at a small fraction of the construction time; a
different non-zero pattern or contraction builds its own."""
import ctypes as C
import time

import pytest

from libtensor_b200 import spec as S
from libtensor_b200._capi import check, lib
from libtensor_b200.core import Context, block_tensor, btod_contract2, contraction2
from oracle import refapi as R


@pytest.fixture(scope="module")
def hctx():
    c = Context(-1)
    yield c
    c.close()


def _stats():
    h, m, e = C.c_int64(), C.c_int64(), C.c_int64()
    check(lib().ltg_schedule_cache_stats(C.byref(h), C.byref(m), C.byref(e)))
    return h.value, m.value, e.value


def _op(ctx, cfg, zero_a=()):
    c = cfg.contraction
    a = cfg.t_spec()
    b = cfg.v_spec() if hasattr(cfg, "v_spec") else cfg.w_spec()
    A, B = block_tensor(ctx, a), block_tensor(ctx, b)
    A.mark_nonzero()
    B.mark_nonzero()
    for z in zero_a:
        A.zero_block(z)
    contr = contraction2(c["n"], c["m"], c["k"], c["permc"])
    for p in c["pairs"]:
        contr.contract(*p)
    t0 = time.perf_counter()
    op = btod_contract2(contr, A, B, kc=cfg.kc)
    return op, time.perf_counter() - t0, (A, B)


def _listing(op):
    sched = op.get_schedule()
    return sched, [op.pairs(i) for i in range(len(sched))], op.flops()


def test_second_construction_reuses_the_schedule(hctx):
    check(lib().ltg_schedule_cache_set_capacity(0))          # start empty
    check(lib().ltg_schedule_cache_set_capacity(64))
    cfg = S.RING_D2H                                          # 3072 C blocks, 40960 pairs
    h0, m0, _ = _stats()
    op1, t1, keep1 = _op(hctx, cfg)
    h1, m1, _ = _stats()
    assert (h1, m1) == (h0, m0 + 1)
    times = []
    for _ in range(5):
        op2, t2, keep2 = _op(hctx, cfg)
        times.append(t2)
    h2, m2, _ = _stats()
    assert (h2, m2) == (h1 + 5, m1)
    assert _listing(op2) == _listing(op1)
    assert sorted(times)[2] <= 0.01 * t1, (t1, times)


def test_cached_schedule_matches_reference(hctx):
    check(lib().ltg_schedule_cache_set_capacity(64))
    cfg = S.RING_D2H_SMALL
    op1, _, keep1 = _op(hctx, cfg)
    op2, _, keep2 = _op(hctx, cfg)                            # from the cache
    ra, rb = R.RefBT(cfg.t_spec()), R.RefBT(cfg.w_spec())
    ra.fill_seeded(1, 1.0)
    rb.fill_seeded(2, 1.0)
    c = cfg.contraction
    rop = R.RefContract2(c["n"], c["m"], c["k"], c["permc"], c["pairs"], ra, rb, 1.0, 1.0, cfg.kc)
    sched = op2.get_schedule()
    assert sched == rop.schedule()
    for i, cabs in enumerate(sched):
        assert op2.pairs(i) == rop.pairs(cabs)


def test_other_descriptions_build_their_own(hctx):
    check(lib().ltg_schedule_cache_set_capacity(64))
    cfg = S.LADDER_SMALL
    op1, _, k1 = _op(hctx, cfg)
    h, m, _ = _stats()
    op2, _, k2 = _op(hctx, cfg, zero_a=[(0, 1, 0, 2)])       # another non-zero pattern
    assert _stats()[:2] == (h, m + 1)
    assert _listing(op2) != _listing(op1)
    check(lib().ltg_schedule_cache_set_capacity(0))           # off: every construction builds
    h, m, e = _stats()
    assert e == 0
    _op(hctx, cfg)
    assert _stats()[:2] == (h, m + 1)
    check(lib().ltg_schedule_cache_set_capacity(64))
