"""Pins the oracle (no GPU): the compiled reference against the numpy
restatement (dense tensors, the pattern of the reference's own tests
tests/block_tensor/btod_contract2_test.C:796-817), and the restated input
generator against the product's host generator, bit for bit."""
import numpy as np
import pytest

from libtensor_b200 import spec as S
from libtensor_b200.core import Context, block_tensor
from libtensor_b200.spec import permuted_spec
from oracle import refapi as R
from oracle import restate as X
from tests.cases import cases

pytestmark = pytest.mark.skipif(not R.available(), reason="oracle/_ref not built")

CASES = [c for c in cases() if not c.symmetry_error and not c.zero_a]


@pytest.fixture(scope="module")
def hctx():
    c = Context(-1)
    yield c
    c.close()


def _ref_from_dense(spec, dense, canon):
    r = R.RefBT(spec)
    bid = spec.bidims()
    for a in canon:
        bidx = X._unabs(a, bid)
        r.set_block(bidx, X.block_view(spec, dense, bidx))
    return r


@pytest.mark.parametrize("spec", [S.LADDER_SMALL.t_spec(), S.LADDER_SMALL.v_spec(),
                                  S.RING_D2H_SMALL.t_spec(), S.RING_D2H_SMALL.w_spec()],
                         ids=["t ladder", "V ladder", "t ring", "W ring"])
def test_restated_generator_is_bit_identical(hctx, spec):
    t = block_tensor(hctx, spec)
    host = t.fill_seeded_host(1234, 0.01)
    dense = X.seeded_dense(spec, 1234, 0.01)
    packed = X.pack_canonical(spec, dense, t.abs_idx, t.offsets, t.nelems)
    assert np.array_equal(host.view(np.uint64), packed.view(np.uint64))
    assert list(t.abs_idx) == X.canonical_blocks(spec)


@pytest.mark.parametrize("spec", [S.LADDER_SMALL.t_spec(), S.LADDER_SMALL.v_spec(),
                                  S.RING_D2H_SMALL.t_spec(), S.RING_D2H_SMALL.w_spec()],
                         ids=["t ladder", "V ladder", "t ring", "W ring"])
def test_reference_side_generator_is_bit_identical(spec):
    """The generator inside the reference library (seeded inputs for a
    CPU-only caller) writes the restatement's bits into every canonical
    allowed block, and only into those."""
    r = R.RefBT(spec)
    r.fill_seeded(99, 0.5, nthreads=3)
    dense = X.seeded_dense(spec, 99, 0.5)
    canon = X.canonical_blocks(spec)
    assert sorted(r.nonzero()) == canon
    bid = spec.bidims()
    for a in canon:
        bidx = X._unabs(a, bid)
        want = X.block_view(spec, dense, bidx)
        got = r.get_block(bidx, want.shape)
        assert np.array_equal(got.view(np.uint64), np.ascontiguousarray(want).view(np.uint64))
    r.close()


def test_generator_symmetry():
    spec = S.LADDER_SMALL.t_spec()
    d = X.seeded_dense(spec, 7, 1.0)
    assert np.array_equal(d, -d.transpose(1, 0, 2, 3))
    assert np.array_equal(d, -d.transpose(0, 1, 3, 2))
    assert abs(d.std() / np.sqrt(4) - 1.0) < 0.05 * 4 or d.std() > 0   # sum of 4 N(0,1)-like terms


@pytest.mark.parametrize("case", CASES, ids=[c.name for c in CASES])
def test_reference_contraction_matches_dense(case):
    da = X.seeded_dense(case.a, 31, case.a_scale)
    db = X.seeded_dense(case.b, 37, case.b_scale)
    ra = _ref_from_dense(case.a, da, X.canonical_blocks(case.a))
    rb = _ref_from_dense(case.b, db, X.canonical_blocks(case.b))
    op = R.RefContract2(case.n, case.m, case.k, case.permc, case.pairs, ra, rb, case.ka, case.kb, case.kc)
    rc = op.make_result()
    op.perform(rc)
    dc = X.dense_contract(da, db, case.n, case.m, case.k, case.permc, case.pairs,
                          case.ka * case.kb * case.kc)
    # result splits follow the connected argument dims
    na = case.n + case.k
    conn = _result_sources(case)
    splits = [(case.a if s < na else case.b).splits[s if s < na else s - na] for s in conn]
    worst = 0.0
    for a in op.schedule():
        bidx = rc.block_index(a)
        sl = []
        for d, b in enumerate(bidx):
            st = [0] + list(splits[d]) + [dc.shape[d]]
            sl.append(slice(st[b], st[b + 1]))
        ref_blk = dc[tuple(sl)]
        got = rc.get_block(bidx, ref_blk.shape)
        m = np.max(np.abs(ref_blk))
        if m > 0:
            worst = max(worst, np.max(np.abs(got - ref_blk)) / m)
    assert worst <= 1e-12


def _result_sources(case):
    """For every result dim, the argument dim it comes from (A dims 0..na-1,
    B dims na..): uncontracted A then B dims, permuted by permc."""
    na, nb = case.n + case.k, case.m + case.k
    ca = {p[0] for p in case.pairs}
    cb = {p[1] for p in case.pairs}
    natural = [i for i in range(na) if i not in ca] + [na + j for j in range(nb) if j not in cb]
    pc = case.permc if case.permc is not None else list(range(case.n + case.m))
    return [natural[pc[i]] for i in range(case.n + case.m)]


def test_reference_copy_add_dot_match_dense():
    spec = S.LADDER_SMALL.t_spec()
    d1 = X.seeded_dense(spec, 41, 1.0)
    d2 = X.seeded_dense(spec, 43, 1.0)
    canon = X.canonical_blocks(spec)
    r1, r2 = _ref_from_dense(spec, d1, canon), _ref_from_dense(spec, d2, canon)
    perm = (0, 2, 1, 3)
    pspec = permuted_spec(spec, perm)
    rb = R.RefBT(pspec)
    R.ref_copy(r1, perm, 2.0, rb)
    dp = 2.0 * X.dense_permute(d1, perm)
    for a in rb.nonzero():
        bidx = rb.block_index(a)
        v = X.block_view(pspec, dp, bidx)
        assert np.array_equal(rb.get_block(bidx, v.shape), v)
    ry = R.RefBT(spec)
    R.ref_add([(r1, None, 1.0), (r2, (1, 0, 3, 2), -0.5)], ry)
    dy = d1 - 0.5 * X.dense_permute(d2, (1, 0, 3, 2))
    for a in ry.nonzero():
        bidx = ry.block_index(a)
        v = X.block_view(spec, dy, bidx)
        assert np.allclose(ry.get_block(bidx, v.shape), v, rtol=0, atol=1e-14)
    dot = R.ref_dotprod(r1, None, r2, (1, 0, 2, 3))
    ddot = float(np.sum(d1 * X.dense_permute(d2, (1, 0, 2, 3))))
    assert abs(dot - ddot) <= 1e-12 * max(1.0, abs(ddot))


def test_reference_ccd_iteration_matches_dense_algebra():
    """The reference-side CCD iteration (oracle/ref_ccd.py: the reference's
    operations one after the other) against the dense numpy algebra."""
    from oracle.ref_ccd import RefCCDIteration
    it = RefCCDIteration([3], [4, 3])
    t0 = X.seeded_dense(it.t.spec, 7, 0.01)
    V = X.seeded_dense(it.V.spec, 8, 0.01)
    W = X.seeded_dense(it.W.spec, 9, 0.01)
    it.step()
    L = 0.5 * np.einsum("ijcd,abcd->ijab", t0, V)
    G = np.einsum("ikac,kbcj->ijab", t0, W)
    Rm = L + 0.5 * (G - G.transpose(1, 0, 2, 3) - G.transpose(0, 1, 3, 2) + G.transpose(1, 0, 3, 2))
    o, v, e = it.o, it.v, it.eps
    D = e[:o, None, None, None] + e[o:2 * o][None, :, None, None] - e[2 * o:2 * o + v][None, None, :, None] \
        - e[2 * o + v:][None, None, None, :]
    Rd = np.where(X.allowed_element_mask(it.R.spec if it.R.spec else it.t.spec), Rm / D, 0.0)
    for a in X.canonical_blocks(it.t.spec):
        bidx = X._unabs(a, it.t.spec.bidims())
        want = X.block_view(it.t.spec, Rd, bidx)
        got = it.t.get_block(bidx, want.shape)
        assert np.max(np.abs(got - want)) <= 1e-13 * max(1e-300, np.max(np.abs(want)))
    E = float(np.sum(Rd * t0))
    assert abs(it.energy - E) <= 1e-12 * abs(E)
    Xd = np.transpose(t0, (0, 2, 1, 3))
    from libtensor_b200.spec import permuted_spec
    xs = permuted_spec(it.t.spec, (0, 2, 1, 3))
    for a in X.canonical_blocks(xs):
        bidx = X._unabs(a, xs.bidims())
        want = X.block_view(xs, Xd, bidx)
        assert np.array_equal(it.X.get_block(bidx, want.shape), want)
    it.close()
