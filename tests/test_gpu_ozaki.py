"""GPU checks of the split-precision (Ozaki) contraction on tcgen05 tensor
cores: same non-zero C blocks as the reference and every C block within the
stated relative error (block max-norm) of the reference's FP64 result."""
import numpy as np
import pytest

from libtensor_b200.core import (Context, MODE_OZAKI_BF16, MODE_OZAKI_CRT, MODE_OZAKI_FP8, MODE_OZAKI_INT8,
                                 btod_contract2, contraction2)
from oracle import refapi as R
from tests.cases import cases
from tests.helpers import block_errors, max_rel_block_error, seeded_pair

pytestmark = [pytest.mark.gpu, pytest.mark.skipif(not R.available(), reason="oracle/_ref not built")]

CASES = [c for c in cases() if not c.symmetry_error]

# (mode, slices, bound on the block-relative error).  INT8 slices carry 7
# bits (6 for the first), BF16 slices are given the same 7 bits (exact
# partial sums in FP32), FP8 E4M3 slices 5 bits (4 for the first); the bounds
# are a few units of the dropped tail 2^-(b0 + b(S-1)) times sqrt(K).  The
# modular mode with L moduli rounds each operand to P bits, P = floor((log2 M
# - 1 - log2(sum_p |c_p| K_p)) / 2) (M the product of the moduli, at most 45):
# P = 45 for 13 and 16 moduli on these cases, about 31 for 9.
MODES = [
    (MODE_OZAKI_INT8, 7, 1e-12),
    (MODE_OZAKI_INT8, 6, 1e-10),
    (MODE_OZAKI_INT8, 3, 1e-3),
    (MODE_OZAKI_BF16, 7, 1e-12),
    (MODE_OZAKI_FP8, 8, 1e-9),
    (MODE_OZAKI_CRT, 13, 1e-12),
    (MODE_OZAKI_CRT, 16, 1e-12),
    (MODE_OZAKI_CRT, 9, 1e-7),
]


@pytest.fixture(scope="module")
def gctx():
    c = Context(0)
    yield c
    c.close()


@pytest.mark.parametrize("mode,S,tol", MODES, ids=[f"mode{m}-S{s}" for m, s, _ in MODES])
@pytest.mark.parametrize("case", CASES, ids=[c.name for c in CASES])
def test_split_precision_matches_reference(gctx, case, mode, S, tol):
    A, ra, _ = seeded_pair(gctx, case.a, 11, case.a_scale, case.zero_a)
    B, rb, _ = seeded_pair(gctx, case.b, 23, case.b_scale)
    contr = contraction2(case.n, case.m, case.k, case.permc)
    for p in case.pairs:
        contr.contract(*p)
    op = btod_contract2(contr, A, B, case.ka, case.kb, case.kc)
    rop = R.RefContract2(case.n, case.m, case.k, case.permc, case.pairs, ra, rb, case.ka, case.kb, case.kc)
    C = op.make_result()
    RC = rop.make_result()
    op.perform(C, mode=mode, nslices=S)
    gctx.synchronize()
    rop.perform(RC)
    assert C.nonzero() == RC.nonzero()
    errs = block_errors(C, C.download(), RC, None)
    err = max_rel_block_error(errs)
    print(f"{case.name} mode={mode} S={S}: max block rel err {err:.3e}")
    assert err <= tol, sorted(errs, key=lambda e: -e[1])[:3]


@pytest.mark.parametrize("mode,S", [(MODE_OZAKI_INT8, 7), (MODE_OZAKI_CRT, 13)], ids=["int8-S7", "crt-L13"])
def test_split_precision_add_mode(gctx, mode, S):
    case = CASES[0]
    A, ra, _ = seeded_pair(gctx, case.a, 3, case.a_scale)
    B, rb, _ = seeded_pair(gctx, case.b, 4, case.b_scale)
    contr = contraction2(case.n, case.m, case.k, case.permc)
    for p in case.pairs:
        contr.contract(*p)
    op = btod_contract2(contr, A, B, case.ka, case.kb, case.kc)
    rop = R.RefContract2(case.n, case.m, case.k, case.permc, case.pairs, ra, rb, case.ka, case.kb, case.kc)
    C, RC = op.make_result(), rop.make_result()
    op.perform(C)
    rop.perform(RC)
    op.perform(C, 0.5, mode=mode, nslices=S)
    rop.perform(RC, 0.5)
    assert max_rel_block_error(block_errors(C, C.download(), RC, None)) <= 1e-12


@pytest.mark.parametrize("case", CASES, ids=[c.name for c in CASES])
def test_crt_grouped_products_are_bit_identical(gctx, case):
    """The modular products are exact integers, so computing small C blocks as
    grouped products gives the same bits as one product per block and pair."""
    A, _, _ = seeded_pair(gctx, case.a, 5, case.a_scale, case.zero_a)
    B, _, _ = seeded_pair(gctx, case.b, 6, case.b_scale)
    contr = contraction2(case.n, case.m, case.k, case.permc)
    for p in case.pairs:
        contr.contract(*p)
    op = btod_contract2(contr, A, B, case.ka, case.kb, case.kc)
    C1, C2 = op.make_result(), op.make_result()
    op.perform(C1, mode=MODE_OZAKI_CRT, nslices=13)
    op.set_grouping(False)
    op.perform(C2, mode=MODE_OZAKI_CRT, nslices=13)
    op.set_grouping(True)
    gctx.synchronize()
    assert np.array_equal(C1.download().view(np.uint64), C2.download().view(np.uint64))


def _crt_variants(gctx, case, seeds, setters):
    """Results of the modular mode (13 moduli) under each setting of a plan
    switch, as raw bits."""
    A, _, _ = seeded_pair(gctx, case.a, seeds[0], case.a_scale, case.zero_a)
    B, _, _ = seeded_pair(gctx, case.b, seeds[1], case.b_scale)
    contr = contraction2(case.n, case.m, case.k, case.permc)
    for p in case.pairs:
        contr.contract(*p)
    op = btod_contract2(contr, A, B, case.ka, case.kb, case.kc)
    out = []
    for setter in setters:
        C = op.make_result()
        setter(op)
        op.perform(C, mode=MODE_OZAKI_CRT, nslices=13)
        gctx.synchronize()
        out.append(C.download().view(np.uint64))
    return out


@pytest.mark.parametrize("case", CASES, ids=[c.name for c in CASES])
def test_crt_item_rows_are_bit_identical(gctx, case):
    """Work items of 128 rows (alternating accumulator slots) and of 256 rows
    (two MMA tiles per item) compute the same exact integers."""
    out = _crt_variants(gctx, case, (7, 8), [lambda op: op.set_crt_rows(128), lambda op: op.set_crt_rows(256)])
    assert np.array_equal(out[0], out[1])


def test_grouped_products_with_zero_operand_blocks(gctx):
    """Ring D2h with some t blocks zero: cells of the grouped products that no
    pair uses stay zero; grouped and per-block products agree (bit-identical
    in the modular mode, 1e-13 in FP64) and match the reference."""
    from libtensor_b200 import spec as S
    from libtensor_b200.core import MODE_PLAIN_FP64
    case = next(c for c in CASES if c.name == "ring D2h small")
    A, ra, _ = seeded_pair(gctx, case.a, 51, case.a_scale)
    nz = A.nonzero()
    zero = [tuple(A.block_index(a)) for a in nz[::3]]       # every third non-zero canonical block
    A, ra, _ = seeded_pair(gctx, case.a, 51, case.a_scale, zero)
    B, rb, _ = seeded_pair(gctx, case.b, 52, case.b_scale)
    contr = contraction2(case.n, case.m, case.k, case.permc)
    for p in case.pairs:
        contr.contract(*p)
    op = btod_contract2(contr, A, B, case.ka, case.kb, case.kc)
    C = op.make_result()
    assert op.group_info(C)[0] > 0
    rop = R.RefContract2(case.n, case.m, case.k, case.permc, case.pairs, ra, rb, case.ka, case.kb, case.kc)
    RC = rop.make_result()
    rop.perform(RC)
    for mode, S_, tol in ((MODE_PLAIN_FP64, 0, 1e-13), (MODE_OZAKI_CRT, 13, 1e-12)):
        out = []
        for grouped in (True, False):
            op.set_grouping(grouped)
            Cg = op.make_result()
            op.perform(Cg, mode=mode, nslices=S_)
            gctx.synchronize()
            out.append(Cg.download())
            assert max_rel_block_error(block_errors(Cg, out[-1], RC, None)) <= tol, (mode, grouped)
        op.set_grouping(True)
        if mode == MODE_OZAKI_CRT:
            assert np.array_equal(out[0].view(np.uint64), out[1].view(np.uint64))


@pytest.mark.parametrize("which", ["ladder", "ring", "ladder o=40 v=160"])
def test_fused_split_matches_two_pass(gctx, which):
    """Row families split in one read of the operand (exponents and residues
    in one kernel, the second read from L2) give the same bits as the
    exponent pass followed by the residue pass, in assign and add mode."""
    from libtensor_b200 import spec as S
    from libtensor_b200.core import block_tensor, btod_contract2, contraction2
    cfg = {"ladder": S.LADDER_SMALL, "ring": S.RING_D2H_SMALL, "ladder o=40 v=160": S.LADDER_PROF}[which]
    a_spec = cfg.t_spec()
    b_spec = cfg.v_spec() if hasattr(cfg, "v_spec") else cfg.w_spec()
    A, B = block_tensor(gctx, a_spec), block_tensor(gctx, b_spec)
    A.fill_seeded(11, cfg.t_scale)
    B.fill_seeded(23, cfg.v_scale)
    c = cfg.contraction
    contr = contraction2(c["n"], c["m"], c["k"], c["permc"])
    for p in c["pairs"]:
        contr.contract(*p)
    op = btod_contract2(contr, A, B, kc=cfg.kc)
    op.set_crt_bound(False)                  # exact exponents on both sides of the comparison
    out = []
    for fused in (1, 2, 0):
        op.set_fused_split(fused)
        C = op.make_result()
        op.perform(C, mode=MODE_OZAKI_CRT, nslices=13)
        op.perform(C, 0.5, mode=MODE_OZAKI_CRT, nslices=13)
        gctx.synchronize()
        out.append(C.download())
        C.close()
    for x in out[:-1]:
        assert np.array_equal(x.view(np.uint64), out[-1].view(np.uint64))
    op.close()
    A.close()
    B.close()


def _ladder_prof(gctx):
    from libtensor_b200 import spec as S
    from libtensor_b200.core import block_tensor
    cfg = S.LADDER_PROF
    A, B = block_tensor(gctx, cfg.t_spec()), block_tensor(gctx, cfg.v_spec())
    A.fill_seeded(11, cfg.t_scale)
    B.fill_seeded(23, cfg.v_scale)
    c = cfg.contraction
    contr = contraction2(c["n"], c["m"], c["k"], c["permc"])
    for p in c["pairs"]:
        contr.contract(*p)
    return cfg, A, B, btod_contract2(contr, A, B, kc=cfg.kc)


def _modes_against_plain(gctx, op):
    """Block-relative error of the modular result (sampled and exact row
    exponents) against the plain FP64 result of the same call."""
    P = op.make_result()
    op.perform(P)
    gctx.synchronize()
    want = P.download()
    errs = {}
    for sampled in (True, False):
        op.set_crt_bound(sampled)
        C = op.make_result()
        op.perform(C, mode=MODE_OZAKI_CRT, nslices=13)
        op.perform(C, 0.5, mode=MODE_OZAKI_CRT, nslices=13)           # C += 0.5 (...): 1.5 x
        gctx.synchronize()
        got = C.download()
        worst = 0.0
        for (bidx, g), (_, w) in zip(C.blocks(got), P.blocks(want)):
            m = float(np.max(np.abs(w))) if w.size else 0.0
            if m > 0:
                worst = max(worst, float(np.max(np.abs(g - 1.5 * w))) / (1.5 * m))
        errs[sampled] = worst
        C.close()
    op.set_crt_bound(True)
    P.close()
    return errs


def test_sampled_row_bounds_within_error():
    """Ladder o=40 v=160 (rows of 1024-2304 k words, so the long rows take
    sampled exponent bounds): both ways of finding the row exponents stay
    within 1e-12 of the plain FP64 result, assign and add."""
    ctx = Context(0)
    cfg, A, B, op = _ladder_prof(ctx)
    errs = _modes_against_plain(ctx, op)
    assert errs[True] <= 1e-12 and errs[False] <= 1e-12, errs
    op.close(); A.close(); B.close(); ctx.close()


def test_rows_whose_sample_misses_the_maximum_are_redone():
    """Large elements placed between the sampled groups of many operand rows
    (k = 40 and k = 300 of row 0 of every V block, outside the sampled runs
    k = 0..31, 512..543, ...; 1e4 times the block's magnitude) make the
    sampled bounds too small for those rows; the residue pass must find it
    and redo them.  Residues formed with a bound 2^13 too small would exceed
    the CRT range and give errors of order one; redone, the error against the
    plain FP64 result is that of exact exponents within the one binade of
    headroom the sampled bounds of the other side's rows may take (the large
    elements cost the other elements of their rows about 13 of their P bits,
    hence the looser bound)."""
    ctx = Context(0)
    cfg, A, B, op = _ladder_prof(ctx)
    arena = B.download().copy()
    for bidx, blk in B.blocks(arena):
        flat = blk.reshape(-1)
        if flat.size > 300:
            m = float(np.max(np.abs(flat))) or 1.0
            flat[40] = 1e4 * m
            flat[300] = -1e4 * m
    B.upload(arena)
    errs = _modes_against_plain(ctx, op)
    assert errs[True] <= 1e-10 and errs[False] <= 1e-10, errs
    assert errs[True] <= 4.0 * errs[False], errs
    op.close(); A.close(); B.close(); ctx.close()
