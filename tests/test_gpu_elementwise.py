"""GPU parity of btod_copy / btod_add / btod_dotprod / scale and of the
device input generator against the reference (copies bit-exact)."""
import numpy as np
import pytest

from libtensor_b200 import spec as S
from libtensor_b200.core import Context, block_tensor, btod_add, btod_copy, btod_dotprod
from libtensor_b200.spec import BTSpec, permuted_spec
from oracle import refapi as R
from tests.helpers import block_errors, max_rel_block_error, seeded_pair

pytestmark = [pytest.mark.gpu, pytest.mark.skipif(not R.available(), reason="oracle/_ref not built")]


@pytest.fixture(scope="module")
def gctx():
    c = Context(0)
    yield c
    c.close()


def _spin_x(o=(3,), v=(4, 3)):
    so, sv = S.spin_splits(list(o)), S.spin_splits(list(v))
    no, nv = 2 * sum(o), 2 * sum(v)
    return BTSpec(dims=[no, no, nv, nv], splits=[so, so, sv, sv], part_pdims=[2, 2, 2, 2],
                  part_forbidden=S.spin_forbidden([((0, 1), (2, 3))], 4))


def test_device_fill_matches_host_fill(gctx):
    spec = S.LADDER_SMALL.t_spec()
    t = block_tensor(gctx, spec)
    host = t.fill_seeded_host(99, 0.01)
    t.fill_seeded(99, 0.01)
    dev = t.download()
    assert np.array_equal(host.view(np.uint64), dev.view(np.uint64))


@pytest.mark.parametrize("perm", [(0, 2, 1, 3), (1, 0, 2, 3), (2, 3, 0, 1), (0, 1, 3, 2)])
def test_copy_is_bit_exact(gctx, perm):
    spec = S.LADDER_SMALL.t_spec()
    A, ra, _ = seeded_pair(gctx, spec, 3, 0.01)
    B = A.permuted(perm)
    btod_copy(A, perm, 1.0).perform(B)
    rb = R.RefBT(permuted_spec(spec, perm))
    R.ref_copy(ra, perm, 1.0, rb)
    assert B.nonzero() == rb.nonzero()
    arena = B.download()
    for bidx, blk in B.blocks(arena):
        assert np.array_equal(blk, rb.get_block(bidx, blk.shape)), bidx


def test_copy_scaled_add_mode(gctx):
    spec = _spin_x()
    A, ra, _ = seeded_pair(gctx, spec, 4, 1.0)
    B, rb, _ = seeded_pair(gctx, spec, 5, 1.0)
    btod_copy(A, (1, 0, 3, 2), -0.5).perform(B, 2.0)
    R.ref_copy(ra, (1, 0, 3, 2), -0.5, rb, 2.0)
    errs = block_errors(B, B.download(), rb, None)
    assert max_rel_block_error(errs) <= 1e-15


def test_add_four_permuted_terms(gctx):
    spec = _spin_x()
    X, rx, _ = seeded_pair(gctx, spec, 6, 1.0)
    terms = [((0, 1, 2, 3), 1.0), ((1, 0, 2, 3), -1.0), ((0, 1, 3, 2), -1.0), ((1, 0, 3, 2), 1.0)]
    Y = block_tensor(gctx, spec)
    op = btod_add(X, *terms[0])
    for p, c in terms[1:]:
        op.add_op(X, p, c)
    op.perform(Y)
    ry = R.RefBT(spec)
    R.ref_add([(rx, p, c) for p, c in terms], ry)
    assert Y.nonzero() == ry.nonzero()
    errs = block_errors(Y, Y.download(), ry, None)
    assert max_rel_block_error(errs) <= 1e-15


def test_add_eight_transposing_terms(gctx):
    # 8 terms that all move the innermost index: every term goes through the
    # shared-memory tiles (more than 48 KiB of them per CTA)
    spec = BTSpec(dims=[20, 70, 90], splits=[[7], [30], [40, 65]])
    X, rx, _ = seeded_pair(gctx, spec, 14, 1.0)
    perms = [(0, 2, 1)] * 4 + [(0, 2, 1)] * 4
    coeffs = [1.0, -0.5, 0.25, 2.0, -1.0, 0.125, 3.0, -0.75]
    src = [X] * 8
    out_spec = BTSpec(dims=[20, 90, 70], splits=[[7], [40, 65], [30]])
    Y = block_tensor(gctx, out_spec)
    op = btod_add(src[0], perms[0], coeffs[0])
    for t in range(1, 8):
        op.add_op(src[t], perms[t], coeffs[t])
    op.perform(Y)
    ry = R.RefBT(out_spec)
    R.ref_add([(rx, p, c) for p, c in zip(perms, coeffs)], ry)
    errs = block_errors(Y, Y.download(), ry, None)
    assert max_rel_block_error(errs) <= 1e-15


def test_dotprod_transposed_no_symmetry(gctx):
    spec = BTSpec(dims=[33, 70, 70], splits=[[16], [20, 45], [20, 45]])
    A, ra, _ = seeded_pair(gctx, spec, 15, 1.0)
    B, rb, _ = seeded_pair(gctx, spec, 16, 1.0)
    v = btod_dotprod(A, None, B, (0, 2, 1)).calculate()
    rv = R.ref_dotprod(ra, None, rb, (0, 2, 1))
    assert abs(v - rv) <= 1e-12 * abs(rv), (v, rv)


def test_add_into_existing_with_coefficients(gctx):
    spec = S.LADDER_SMALL.t_spec()
    A, ra, _ = seeded_pair(gctx, spec, 8, 1.0)
    B, rb, _ = seeded_pair(gctx, spec, 9, 1.0)
    Y, ry, _ = seeded_pair(gctx, spec, 10, 1.0)
    btod_add(A, None, 0.5).add_op(B, (1, 0, 3, 2), -0.5).perform(Y, 1.0)
    R.ref_add([(ra, None, 0.5), (rb, (1, 0, 3, 2), -0.5)], ry, 1.0)
    errs = block_errors(Y, Y.download(), ry, None)
    assert max_rel_block_error(errs) <= 1e-15


@pytest.mark.parametrize("pa,pb", [(None, None), ((1, 0, 2, 3), None), ((1, 0, 3, 2), (0, 1, 2, 3))])
def test_dotprod_matches_reference(gctx, pa, pb):
    spec = S.LADDER_SMALL.t_spec()
    A, ra, _ = seeded_pair(gctx, spec, 12, 1.0)
    B, rb, _ = seeded_pair(gctx, spec, 13, 1.0)
    v = btod_dotprod(A, pa, B, pb).calculate()
    rv = R.ref_dotprod(ra, pa, rb, pb)
    assert abs(v - rv) <= 1e-12 * max(1.0, abs(rv)), (v, rv)


def test_dotprod_d2h_labels(gctx):
    spec = S.RING_D2H_SMALL.t_spec()
    A, ra, _ = seeded_pair(gctx, spec, 14, 1.0)
    B, rb, _ = seeded_pair(gctx, spec, 15, 1.0)
    v = btod_dotprod(A, None, B, None).calculate()
    rv = R.ref_dotprod(ra, None, rb, None)
    assert abs(v - rv) <= 1e-12 * max(1.0, abs(rv))


def test_scale(gctx):
    spec = S.LADDER_SMALL.t_spec()
    A = block_tensor(gctx, spec)
    host = A.fill_seeded_host(1, 1.0)
    A.upload(host)
    A.scale(-0.25)
    assert np.array_equal(A.download(), host * -0.25)
