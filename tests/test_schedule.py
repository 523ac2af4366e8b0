"""Integer parity of the host engine against the reference (no GPU):
orbits, result symmetry, non-zero C block list (bit-identical) and the
coalesced pair lists (gen_bto_contract2_nzorb / clst_builder / clst_optimize)."""
import numpy as np
import pytest

from libtensor_b200._capi import LtgError
from libtensor_b200.core import Context, block_tensor, btod_contract2, contraction2
from oracle import refapi as R
from tests.cases import cases

pytestmark = pytest.mark.skipif(not R.available(), reason="oracle/_ref not built")

CASES = cases()


@pytest.fixture(scope="module")
def hctx():
    c = Context(-1)
    yield c
    c.close()


def _ref_with_blocks(spec, t, zero=()):
    r = R.RefBT(spec)
    zero = {tuple(z) for z in zero}
    for s in range(t.nblocks):
        bidx = tuple(t.block_index(t.abs_idx[s]))
        if bidx in zero:
            continue
        shape = tuple(spec.block_extent(d, b) for d, b in enumerate(bidx))
        r.set_block(bidx, np.ones(shape))
    return r


@pytest.mark.parametrize("case", CASES, ids=[c.name for c in CASES])
def test_orbits_match_reference(hctx, case):
    for spec in (case.a, case.b):
        t = block_tensor(hctx, spec)
        r = R.RefBT(spec)
        nb = int(np.prod(t.bidims))
        for a in range(nb):
            canon, perm, coeff, allowed = t.orbit(a)
            rc, rperm, rcoeff, rallowed, _ = r.orbit(a)
            assert (canon, allowed) == (rc, rallowed), (case.name, a)
            assert perm == rperm and coeff == rcoeff, (case.name, a)
        # canonical allowed blocks == reference orbit list
        ref_canon = sorted({r.orbit(a)[0] for a in range(nb) if r.orbit(a)[3]})
        assert list(t.abs_idx) == ref_canon
        t.close(); r.close()


@pytest.mark.parametrize("case", CASES, ids=[c.name for c in CASES])
def test_schedule_and_pairs_match_reference(hctx, case):
    A = block_tensor(hctx, case.a)
    B = block_tensor(hctx, case.b)
    A.mark_nonzero(); B.mark_nonzero()
    for z in case.zero_a:
        A.zero_block(z)
    contr = contraction2(case.n, case.m, case.k, case.permc)
    for p in case.pairs:
        contr.contract(*p)
    ra = _ref_with_blocks(case.a, A, case.zero_a)
    rb = _ref_with_blocks(case.b, B)
    if case.symmetry_error:
        with pytest.raises(LtgError) as ei:
            btod_contract2(contr, A, B, case.ka, case.kb, case.kc)
        assert ei.value.code == 3      # LTG_ERR_SYMMETRY
        with pytest.raises(RuntimeError, match="bad_symmetry"):
            R.RefContract2(case.n, case.m, case.k, case.permc, case.pairs, ra, rb, case.ka, case.kb, case.kc)
        return
    op = btod_contract2(contr, A, B, case.ka, case.kb, case.kc)
    rop = R.RefContract2(case.n, case.m, case.k, case.permc, case.pairs, ra, rb, case.ka, case.kb, case.kc)
    sched, rsched = op.get_schedule(), rop.schedule()
    assert sched == rsched
    for i, cabs in enumerate(sched):
        assert op.pairs(i) == rop.pairs(cabs), (case.name, cabs)
    # result block index space and symmetry: same canonical/allowed blocks
    C = op.make_result()
    RC = rop.make_result()
    assert C.bidims == RC.bidims
    nb = int(np.prod(C.bidims))
    for a in range(nb):
        canon, _, _, allowed = C.orbit(a)
        rc, _, _, rallowed, _ = RC.orbit(a)
        assert canon == rc, (case.name, a)
        if allowed != rallowed:
            # the derived rule may differ only on blocks no pair can reach
            assert a not in rsched
    for x in (C, A, B):
        x.close()
    op.close()


def _fine_ladder_op(ctx, occ, vir):
    from libtensor_b200 import spec as S
    cfg = S.LadderConfig("fine", occ, vir)
    A, B = block_tensor(ctx, cfg.t_spec()), block_tensor(ctx, cfg.v_spec())
    A.mark_nonzero(); B.mark_nonzero()
    c = cfg.contraction
    contr = contraction2(c["n"], c["m"], c["k"], c["permc"])
    for p in c["pairs"]:
        contr.contract(*p)
    return cfg, A, B, btod_contract2(contr, A, B, 1.0, 1.0, cfg.kc)


def test_schedule_does_not_depend_on_host_threads():
    """The schedule is built in chunks over host threads and joined in order."""
    out = []
    for nt in (1, 7):
        ctx = Context(-1)
        ctx.set_host_threads(nt)
        _, A, B, op = _fine_ladder_op(ctx, [3, 3], [4] * 6)
        sched = op.get_schedule()
        out.append((sched, [op.pairs(i) for i in range(len(sched))], op.flops()))
        ctx.close()
    assert len(out[0][0]) > 64                        # several chunks
    assert out[0] == out[1]


def test_fine_blocking_schedule_matches_reference(hctx):
    """Many blocks per index (long pair lists with coalescing): schedule and
    coalesced pair lists as the reference builds them."""
    cfg, A, B, op = _fine_ladder_op(hctx, [2, 2], [3] * 5)
    ra = _ref_with_blocks(cfg.t_spec(), A)
    rb = _ref_with_blocks(cfg.v_spec(), B)
    c = cfg.contraction
    rop = R.RefContract2(c["n"], c["m"], c["k"], c["permc"], c["pairs"], ra, rb, 1.0, 1.0, cfg.kc)
    sched = op.get_schedule()
    assert sched == rop.schedule()
    for i, cabs in enumerate(sched):
        assert op.pairs(i) == rop.pairs(cabs), cabs
