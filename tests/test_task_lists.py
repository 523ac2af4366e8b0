"""Caller-built task lists (ltg_plan_export_tasks / ltg_plan_contract2_upload):
the exported block-pair products, evaluated here in numpy over the arenas,
give the reference's contraction; malformed task records are rejected at
upload; a task-list plan has no schedule of its own.  No GPU."""
import ctypes as C

import numpy as np
import pytest

from libtensor_b200 import _capi
from libtensor_b200._capi import lib
from libtensor_b200.core import Context, btod_contract2, contract2_task_plan, contraction2
from oracle import refapi as R
from tests.cases import cases
from tests.helpers import block_errors, max_rel_block_error, seeded_pair

W = _capi.LTG_TASK_WORDS
ERR_BAD_ARG, ERR_UNSUPPORTED = 1, 4          # LTG_ERR_BAD_ARG, LTG_ERR_UNSUPPORTED
CASES = [c for c in cases() if not c.symmetry_error]


@pytest.fixture(scope="module")
def hctx():
    c = Context(-1)
    yield c
    c.close()


def _sub(rec, base):
    """(extents, strides of the first tensor, strides of the second) of one
    sub-dimension group of a task record."""
    n = int(rec[base])
    ext = [int(rec[base + 1 + 3 * i]) for i in range(n)]
    s0 = [int(rec[base + 2 + 3 * i]) for i in range(n)]
    s1 = [int(rec[base + 3 + 3 * i]) for i in range(n)]
    return ext, s0, s1


def _offsets(ext, strides):
    off = np.zeros(1, np.int64)
    for e, s in zip(ext, strides):
        off = (off[:, None] + np.arange(e, dtype=np.int64)[None, :] * s).reshape(-1)
    return off


def apply_tasks(tasks, a, b, c_size, kabc):
    """C = kabc * sum over tasks of coeff * A[m,k] B[n,k], over flat arenas."""
    c = np.zeros(c_size)
    for rec in tasks:
        c_off, a_off, b_off = int(rec[0]), int(rec[1]), int(rec[2])
        me, ma, mc = _sub(rec, 3)
        ne, nb, nc = _sub(rec, 16)
        ke, ka, kb = _sub(rec, 29)
        coeff = np.frombuffer(np.int64(rec[42]).tobytes(), np.float64)[0]
        am = a[a_off + _offsets(me, ma)[:, None] + _offsets(ke, ka)[None, :]]
        bn = b[b_off + _offsets(ne, nb)[:, None] + _offsets(ke, kb)[None, :]]
        idx = c_off + _offsets(me, mc)[:, None] + _offsets(ne, nc)[None, :]
        c[idx] += coeff * kabc * (am @ bn.T)
    return c


def _setup(hctx, case):
    A, ra, arena_a = seeded_pair(hctx, case.a, 11, case.a_scale, case.zero_a)
    B, rb, arena_b = seeded_pair(hctx, case.b, 23, case.b_scale)
    for z in case.zero_a:
        for bidx, blk in A.blocks(arena_a):
            if tuple(bidx) == tuple(z):
                blk[...] = 0.0
    contr = contraction2(case.n, case.m, case.k, case.permc)
    for p in case.pairs:
        contr.contract(*p)
    op = btod_contract2(contr, A, B, case.ka, case.kb, case.kc)
    return A, B, ra, rb, arena_a, arena_b, op


@pytest.mark.skipif(not R.available(), reason="oracle/_ref not built")
@pytest.mark.parametrize("case", CASES, ids=[c.name for c in CASES])
def test_exported_tasks_give_the_reference_contraction(hctx, case):
    A, B, ra, rb, arena_a, arena_b, op = _setup(hctx, case)
    C_ = op.make_result()
    tasks = op.export_tasks(C_)
    flops = sum(2.0 * np.prod(_sub(t, 3)[0]) * np.prod(_sub(t, 16)[0]) * np.prod(_sub(t, 29)[0]) for t in tasks)
    assert flops == pytest.approx(op.flops())
    arena_c = apply_tasks(tasks, arena_a, arena_b, C_.nelems, case.ka * case.kb * case.kc)
    rop = R.RefContract2(case.n, case.m, case.k, case.permc, case.pairs, ra, rb, case.ka, case.kb, case.kc)
    RC = rop.make_result()
    rop.perform(RC)
    errs = block_errors(C_, arena_c, RC, None)
    assert max_rel_block_error(errs) <= 1e-13


def _plan_upload(hctx, A, B, tasks):
    h = C.c_void_p()
    t = np.ascontiguousarray(tasks, np.int64)
    st = lib().ltg_plan_contract2_upload(hctx.h, A.h, B.h, t.ctypes.data_as(_capi.c_i64p), len(t), C.byref(h))
    if st == 0:
        lib().ltg_plan_free(h)
    return st


def test_malformed_task_records_are_rejected(hctx):
    case = CASES[0]
    A, B, _, _, _, _, op = _setup(hctx, case)
    tasks = op.export_tasks(op.make_result())
    assert len(tasks) > 0
    assert _plan_upload(hctx, A, B, tasks) == 0
    bad = tasks[:1].copy()
    bad[0, 3] = 5                      # five m sub-dimensions
    assert _plan_upload(hctx, A, B, bad) == ERR_BAD_ARG
    bad = tasks[:1].copy()
    bad[0, 4] = 0                      # zero extent
    assert _plan_upload(hctx, A, B, bad) == ERR_BAD_ARG
    bad = tasks[:1].copy()
    bad[0, 5] = -1                     # negative stride
    assert _plan_upload(hctx, A, B, bad) == ERR_BAD_ARG
    assert "stride" in lib().ltg_last_error_string().decode()
    bad = tasks[:1].copy()
    bad[0, 5] = 1 << 31                # stride beyond int32
    assert _plan_upload(hctx, A, B, bad) == ERR_BAD_ARG
    bad = tasks[:1].copy()
    bad[0, 4] = 1 << 20                # 2^20 x 2^20 rows: dimension too large
    bad[0, 3] = 2
    bad[0, 7] = 1 << 20
    assert _plan_upload(hctx, A, B, bad) == ERR_BAD_ARG
    assert _plan_upload(hctx, A, B, tasks[:0]) == 0     # an empty list is a valid plan


def test_task_plan_has_no_schedule(hctx):
    case = CASES[0]
    A, B, _, _, _, _, op = _setup(hctx, case)
    C_ = op.make_result()
    plan = contract2_task_plan(A, B, op.export_tasks(C_))
    assert plan.flops() == pytest.approx(op.flops())
    h = C.c_void_p()
    assert lib().ltg_contract2_make_result(plan.h, C.byref(h)) == ERR_UNSUPPORTED
    n = C.c_int64()
    assert lib().ltg_plan_export_tasks(plan.h, C_.h, None, 0, C.byref(n)) == ERR_BAD_ARG
    plan.close()


def test_export_reports_the_full_count(hctx):
    case = CASES[0]
    A, B, _, _, _, _, op = _setup(hctx, case)
    C_ = op.make_result()
    tasks = op.export_tasks(C_)
    n = C.c_int64()
    buf = np.zeros((1, W), np.int64)
    assert lib().ltg_plan_export_tasks(op.h, C_.h, buf.ctypes.data_as(_capi.c_i64p), 1, C.byref(n)) == 0
    assert n.value == len(tasks)
    assert np.array_equal(buf[0], tasks[0])
