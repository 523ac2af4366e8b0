"""GPU parity of the symmetrizers (ltg_symmetrize; btod_symmetrize2 /
btod_symmetrize4 of libtensor/block_tensor/btod_symmetrize2.h:19,
btod_symmetrize4.h:27):

* the exchange of two indexes and a unitary pair exchange P(01)P(23), symmetric
  and antisymmetric, of a tensor and of a contraction's result (the ring
  term), against the reference's btod_symmetrize2 wrapping btod_copy or the
  btod_contract2 itself, assign and add;
* the 24-term sum over four indexes against the dense numpy restatement (the
  reference's btod_symmetrize4 leaves index i1 without a group in its
  make_symmetry, gen_bto_symmetrize4_impl.h:219-249, and fails).
The product's result space (ltg_bt_create_symmetrized) has the reference's
canonical blocks in these cases, so results compare block by block."""
from itertools import permutations

import numpy as np
import pytest

from libtensor_b200 import spec as S
from libtensor_b200.core import Context, block_tensor, btod_contract2, btod_symmetrize, contraction2
from libtensor_b200.spec import BTSpec
from oracle import refapi as R
from oracle import restate as X
from tests.helpers import block_errors, max_rel_block_error

pytestmark = [pytest.mark.gpu, pytest.mark.skipif(not R.available(), reason="oracle/_ref not built")]

TOL = 1e-15


@pytest.fixture(scope="module")
def gctx():
    c = Context(0)
    yield c
    c.close()


CASES = [dict(symm=False, idx=(0, 1)), dict(symm=True, idx=(2, 3)), dict(symm=False, perm=(1, 0, 3, 2)),
         dict(symm=True, perm=(1, 0, 3, 2))]
IDS = ["asymm(0,1)", "symm(2,3)", "asymm P(01)P(23)", "symm P(01)P(23)"]


@pytest.mark.parametrize("kw", CASES, ids=IDS)
def test_symmetrize_tensor_matches_reference(gctx, kw):
    spec = S.RING_D2H_SMALL.t_spec()
    x_spec = BTSpec(dims=spec.dims, splits=spec.splits, part_pdims=spec.part_pdims,
                    part_forbidden=spec.part_forbidden, labels=spec.labels, label_nirrep=spec.label_nirrep,
                    label_intr=spec.label_intr)              # spin and labels, no permutational symmetry
    a = block_tensor(gctx, x_spec)
    a.fill_seeded(41, 1.0)
    ra = R.RefBT(x_spec)
    ra.fill_seeded(41, 1.0)
    op = btod_symmetrize(a, c=0.5, **kw)
    b = op.make_result()
    op.perform(b)
    rb = R.RefBT(x_spec)
    R.ref_symmetrize(ra, 0.5, rb, **kw)
    errs = block_errors(b, b.download(), rb, None)
    assert max_rel_block_error(errs) <= TOL
    op.perform(b, 2.0)                                       # b += 2 * (sum)
    R.ref_symmetrize(ra, 0.5, rb, d=2.0, **kw)
    assert max_rel_block_error(block_errors(b, b.download(), rb, None)) <= TOL


@pytest.mark.parametrize("kw", [CASES[0], CASES[2]], ids=[IDS[0], IDS[2]])
def test_symmetrize_contraction_matches_reference(gctx, kw):
    """The ring term r(i,j,a,b) = sum_kc t(i,k,a,c) W(k,b,c,j) antisymmetrized
    (the result of the product's contraction, symmetrized) against the
    reference's btod_symmetrize2 wrapping its btod_contract2."""
    cfg = S.RING_D2H_SMALL
    c = cfg.contraction
    A, B = block_tensor(gctx, cfg.t_spec()), block_tensor(gctx, cfg.w_spec())
    A.fill_seeded(11, cfg.t_scale)
    B.fill_seeded(23, cfg.v_scale)
    contr = contraction2(c["n"], c["m"], c["k"], c["permc"])
    for p in c["pairs"]:
        contr.contract(*p)
    op = btod_contract2(contr, A, B)
    G = op.make_result()
    op.perform(G)
    sy = btod_symmetrize(G, **kw)
    out = sy.make_result()
    sy.perform(out)
    ra, rb = R.RefBT(cfg.t_spec()), R.RefBT(cfg.w_spec())
    ra.fill_seeded(11, cfg.t_scale)
    rb.fill_seeded(23, cfg.v_scale)
    rop = R.RefContract2(c["n"], c["m"], c["k"], c["permc"], c["pairs"], ra, rb)
    rout = rop.make_result()
    rop.symmetrize(rout, **kw)
    errs = block_errors(out, out.download(), rout, None)
    assert max_rel_block_error(errs) <= 1e-13


def _parity(p):
    p, s = list(p), 1
    for i in range(len(p)):
        while p[i] != i:
            j = p[i]
            p[i], p[j] = p[j], p[i]
            s = -s
    return s


@pytest.mark.parametrize("symm", [True, False], ids=["symm", "asymm"])
def test_symmetrize4_matches_dense(gctx, symm):
    spec = BTSpec(dims=[12] * 4, splits=[[5]] * 4)
    a = block_tensor(gctx, spec)
    a.fill_seeded(6, 1.0)
    d = X.seeded_dense(spec, 6, 1.0)
    want = sum((1 if symm else _parity(p)) * np.transpose(d, p) for p in permutations(range(4)))
    op = btod_symmetrize(a, symm, idx=(0, 1, 2, 3))
    b = op.make_result()
    op.perform(b)
    got = b.download()
    worst = 0.0
    for bidx, blk in b.blocks(got):
        w = X.block_view(spec, want, bidx)
        worst = max(worst, float(np.max(np.abs(blk - w))) / max(1e-300, float(np.max(np.abs(want)))))
    assert worst <= 1e-14
    # the result space has the symmetric group of the four indexes: with two
    # blocks per index, one canonical block per number of second blocks
    assert len(b.abs_idx) == 5


def _ring_op(gctx, cfg):
    c = cfg.contraction
    A, B = block_tensor(gctx, cfg.t_spec()), block_tensor(gctx, cfg.w_spec())
    A.fill_seeded(11, cfg.t_scale)
    B.fill_seeded(23, cfg.v_scale)
    contr = contraction2(c["n"], c["m"], c["k"], c["permc"])
    for p in c["pairs"]:
        contr.contract(*p)
    return A, B, btod_contract2(contr, A, B)


# (mode, bound on the block-relative error, bound relative to the result's
# largest element).  The antisymmetrized result cancels inside some blocks,
# whose norms then fall below the contraction's scale: the modular mode's
# rounding (about 1e-13 of the contraction's scale) is measured against the
# result's own magnitude, and the block-relative bound is looser.
@pytest.mark.parametrize("mode,tol,gtol", [(0, 1e-13, 1e-13), (4, 1e-11, 1e-12)], ids=["plain", "modular13"])
@pytest.mark.parametrize("kw", [CASES[0], CASES[2]], ids=[IDS[0], IDS[2]])
def test_fused_symmetrize_contraction_matches_reference(gctx, kw, mode, tol, gtol):
    """The ring term antisymmetrized with both terms written by the
    contraction's kernels (ltg_contract2_symmetrized, no temporary: the plain
    path's grouped-product scatter, or the modular recombination with 13
    moduli) against the reference's btod_symmetrize2 wrapping its
    btod_contract2: the same non-zero blocks, every block within the mode's
    bound; two calls give the same bits (two adds per element onto zero)."""
    cfg = S.RING_D2H_SMALL
    A, B, op = _ring_op(gctx, cfg)
    out = op.make_symmetrized(**kw)
    op.perform_symmetrized(out, mode=mode, **kw)
    gctx.synchronize()
    got = out.download().copy()
    op.perform_symmetrized(out, mode=mode, **kw)
    gctx.synchronize()
    assert np.array_equal(out.download(), got)
    c = cfg.contraction
    ra, rb = R.RefBT(cfg.t_spec()), R.RefBT(cfg.w_spec())
    ra.fill_seeded(11, cfg.t_scale)
    rb.fill_seeded(23, cfg.v_scale)
    rop = R.RefContract2(c["n"], c["m"], c["k"], c["permc"], c["pairs"], ra, rb)
    rout = rop.make_result()
    rop.symmetrize(rout, **kw)
    assert out.nonzero() == rout.nonzero()
    errs = block_errors(out, got, rout, None)
    assert max_rel_block_error(errs) <= tol
    assert max(d for _, d, _ in errs) <= gtol * max(m for _, _, m in errs)
    out.close(); op.close(); A.close(); B.close()


@pytest.mark.parametrize("mode", [0, 4, 1, 2], ids=["plain", "modular13", "bf16x7", "fp8x8"])
@pytest.mark.parametrize("kw", CASES, ids=IDS)
def test_fused_symmetrize_equals_symmetrizer_of_result(gctx, kw, mode):
    """Fused and unfused forms of the same symmetrizer over the ring term and
    over the ladder (whose result is antisymmetric already, so its orbit
    signs enter every term) agree to rounding; a scale c applies to both
    terms."""
    for cfg in (S.RING_D2H_SMALL, S.LADDER_SMALL):
        if cfg is S.RING_D2H_SMALL:
            A, B, op = _ring_op(gctx, cfg)
        else:
            c = cfg.contraction
            A, B = block_tensor(gctx, cfg.t_spec()), block_tensor(gctx, cfg.v_spec())
            A.fill_seeded(11, cfg.t_scale)
            B.fill_seeded(23, cfg.v_scale)
            contr = contraction2(c["n"], c["m"], c["k"], c["permc"])
            for p in c["pairs"]:
                contr.contract(*p)
            op = btod_contract2(contr, A, B, kc=cfg.kc)
        G = op.make_result()
        op.perform(G, mode=mode)
        sy = btod_symmetrize(G, c=0.5, **kw)
        want_t = sy.make_result()
        sy.perform(want_t)
        out = op.make_symmetrized(**kw)
        op.perform_symmetrized(out, c=0.5, mode=mode, **kw)
        gctx.synchronize()
        got, want = out.download(), want_t.download()
        assert np.array_equal(out.abs_idx, want_t.abs_idx)
        assert out.nonzero() == want_t.nonzero()
        # relative to the contraction's largest element: a symmetrizer whose
        # terms cancel (P(01)P(23) of the ladder's doubly antisymmetric
        # result) leaves a result of rounding size
        scale = max(1e-300, float(np.max(np.abs(G.download()))))
        assert float(np.max(np.abs(got - want))) <= 1e-14 * scale, cfg.name
        for t in (out, want_t, G, op, A, B):
            t.close()


def test_fused_symmetrize_rejects_four_indexes(gctx):
    cfg = S.RING_D2H_SMALL
    A, B, op = _ring_op(gctx, cfg)
    out = op.make_symmetrized(True, idx=(0, 1))
    with pytest.raises(Exception):
        op.perform_symmetrized(out, True, idx=(0, 1, 2, 3))
    out.close(); op.close(); A.close(); B.close()


def test_fused_symmetrize_in_captured_graph(gctx):
    """A fused symmetrizer call (zeroing the result, then the contraction's
    kernels adding into it) captured as a CUDA graph replays to the eager
    bits, plain and modular."""
    cfg = S.RING_D2H_SMALL
    A, B, op = _ring_op(gctx, cfg)
    for mode in (0, 4):
        out = op.make_symmetrized(False, idx=(0, 1))
        op.perform_symmetrized(out, False, idx=(0, 1), mode=mode)      # prepared outside the capture
        gctx.synchronize()
        want = out.download().copy()
        out.upload(np.zeros(out.nelems))
        gctx.graph_begin()
        op.perform_symmetrized(out, False, idx=(0, 1), mode=mode)
        g = gctx.graph_end()
        for _ in range(2):
            g.launch()
        gctx.synchronize()
        assert np.array_equal(out.download(), want), mode
        g.close()
        out.close()
    op.close(); A.close(); B.close()


def test_fused_modular_symmetrizer_after_plan_change(gctx):
    """Changing the plan's modular settings drops the prepared modular
    contractions and the fused symmetrizers built on them together: the next
    fused call prepares again and gives the same result within the mode's
    bound (exact instead of sampled row exponents)."""
    cfg = S.RING_D2H_SMALL
    A, B, op = _ring_op(gctx, cfg)
    out = op.make_symmetrized(False, idx=(0, 1))
    op.perform_symmetrized(out, False, idx=(0, 1), mode=4)
    gctx.synchronize()
    first = out.download().copy()
    op.set_crt_bound(False)
    op.perform_symmetrized(out, False, idx=(0, 1), mode=4)
    gctx.synchronize()
    second = out.download()
    scale = max(1e-300, float(np.max(np.abs(first))))
    assert float(np.max(np.abs(second - first))) <= 1e-12 * scale
    out.close(); op.close(); A.close(); B.close()


def test_fused_slice_symmetrizer_takes_default_slice_count(gctx):
    """The slice modes' fused symmetrizer runs at their default slice counts;
    another count is refused (LTG_ERR_UNSUPPORTED) before anything runs."""
    cfg = S.RING_D2H_SMALL
    A, B, op = _ring_op(gctx, cfg)
    out = op.make_symmetrized(False, idx=(0, 1))
    with pytest.raises(Exception):
        op.perform_symmetrized(out, False, idx=(0, 1), mode=1, nslices=4)
    op.perform_symmetrized(out, False, idx=(0, 1), mode=1)
    gctx.synchronize()
    out.close(); op.close(); A.close(); B.close()


def test_fused_symmetrizer_refuses_an_operand_as_result(gctx):
    """The fused form zeroes its result before the contraction reads the
    operands, so a result that is an operand is refused (the C++ class then
    goes through a temporary)."""
    cfg = S.RING_D2H_SMALL
    A, B, op = _ring_op(gctx, cfg)
    with pytest.raises(Exception):
        op.perform_symmetrized(A, False, idx=(0, 1))
    op.close(); A.close(); B.close()
