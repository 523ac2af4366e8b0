"""GPU parity of btod_contract2 (plain FP64 DMMA path) against the reference
compiled from its own sources: identical non-zero C block list and every C
block within 1e-13 relative (block max-norm) of the reference's CPU result."""
import numpy as np
import pytest

from libtensor_b200.core import Context, btod_contract2, contraction2, MODE_PLAIN_FP64
from oracle import refapi as R
from tests.cases import cases
from tests.helpers import block_errors, max_rel_block_error, seeded_pair

pytestmark = [pytest.mark.gpu, pytest.mark.skipif(not R.available(), reason="oracle/_ref not built")]

TOL = 1e-13
CASES = [c for c in cases() if not c.symmetry_error]


@pytest.fixture(scope="module")
def gctx():
    c = Context(0)
    yield c
    c.close()


def _run(gctx, case, seed_a=11, seed_b=23):
    A, ra, _ = seeded_pair(gctx, case.a, seed_a, case.a_scale, case.zero_a)
    B, rb, _ = seeded_pair(gctx, case.b, seed_b, case.b_scale)
    contr = contraction2(case.n, case.m, case.k, case.permc)
    for p in case.pairs:
        contr.contract(*p)
    op = btod_contract2(contr, A, B, case.ka, case.kb, case.kc)
    rop = R.RefContract2(case.n, case.m, case.k, case.permc, case.pairs, ra, rb, case.ka, case.kb, case.kc)
    return A, B, op, rop


@pytest.mark.parametrize("case", CASES, ids=[c.name for c in CASES])
def test_contract_assign_matches_reference(gctx, case):
    A, B, op, rop = _run(gctx, case)
    C = op.make_result()
    RC = rop.make_result()
    op.perform(C, mode=MODE_PLAIN_FP64)
    rop.perform(RC)
    assert op.get_schedule() == rop.schedule()
    assert C.nonzero() == RC.nonzero()
    arena = C.download()
    errs = block_errors(C, arena, RC, None)
    assert max_rel_block_error(errs) <= TOL, sorted(errs, key=lambda e: -e[1])[:3]


@pytest.mark.parametrize("case", CASES[:3], ids=[c.name for c in CASES[:3]])
def test_contract_add_matches_reference(gctx, case):
    A, B, op, rop = _run(gctx, case, 5, 7)
    C = op.make_result()
    RC = rop.make_result()
    op.perform(C)
    rop.perform(RC)
    op.perform(C, 0.75)          # C += 0.75 * contr(A, B)
    rop.perform(RC, 0.75)
    arena = C.download()
    errs = block_errors(C, arena, RC, None)
    assert max_rel_block_error(errs) <= TOL


@pytest.mark.parametrize("cfg", range(22))
@pytest.mark.parametrize("case", [CASES[0], CASES[1], CASES[5]], ids=["ladder", "ring", "K=1"])
def test_every_tile_shape_matches_reference(gctx, case, cfg):
    A, B, op, rop = _run(gctx, case)
    op.set_tile(cfg)
    C = op.make_result()
    RC = rop.make_result()
    op.perform(C)
    rop.perform(RC)
    errs = block_errors(C, C.download(), RC, None)
    assert max_rel_block_error(errs) <= TOL


def test_autotune_keeps_results(gctx):
    case = CASES[0]
    A, B, op, rop = _run(gctx, case)
    C = op.make_result()
    table = op.autotune(C, reps=1)
    assert table and all(0 <= v < 22 for v in table.values())
    RC = rop.make_result()
    op.perform(C)
    rop.perform(RC)
    assert max_rel_block_error(block_errors(C, C.download(), RC, None)) <= TOL


def test_contract_repeat_is_deterministic(gctx):
    case = CASES[0]
    A, B, op, rop = _run(gctx, case)
    C = op.make_result()
    op.perform(C)
    x1 = C.download().copy()
    op.perform(C)
    x2 = C.download()
    assert np.array_equal(x1, x2)


@pytest.mark.parametrize("case", CASES, ids=[c.name for c in CASES])
def test_grouped_products_match_per_block(gctx, case):
    """Small blocks computed as grouped dense products (gathered panels, one
    DMMA product per group, scattered into the C blocks) agree with one
    product per C block and pair, in assign and add mode."""
    A, B, op, _ = _run(gctx, case, 31, 32)
    out = []
    for grouped in (True, False):
        op.set_grouping(grouped)
        C = op.make_result()
        op.perform(C)
        op.perform(C, 0.5)
        gctx.synchronize()
        out.append(C.download())
    op.set_grouping(True)
    scale = float(np.max(np.abs(out[1]))) if out[1].size else 1.0
    assert float(np.max(np.abs(out[0] - out[1]))) <= TOL * max(scale, 1e-300)


@pytest.mark.parametrize("split", [2, 3, 4])
@pytest.mark.parametrize("case", [CASES[0], CASES[1], CASES[5]], ids=["ladder", "ring", "K=1"])
def test_k_split_tiles_match_reference(gctx, case, split):
    """Every tile's k range cut into chunks (partial tiles summed in chunk
    order by the split reduction), in assign and add mode, grouped products
    included (ring)."""
    A, B, op, rop = _run(gctx, case)
    op.set_split_k(split)
    C = op.make_result()
    RC = rop.make_result()
    op.perform(C)
    rop.perform(RC)
    assert max_rel_block_error(block_errors(C, C.download(), RC, None)) <= TOL
    op.perform(C, 0.5)
    rop.perform(RC, 0.5)
    assert max_rel_block_error(block_errors(C, C.download(), RC, None)) <= TOL
    # the chunked sum is fixed in order: repeated calls give the same bits
    x1 = C.download().copy()
    op.perform(C)
    op.perform(C, 0.5)
    assert np.array_equal(x1.view(np.uint64), C.download().view(np.uint64))
    op.set_split_k(0)
