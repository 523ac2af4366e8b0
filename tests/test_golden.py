"""Golden fixtures (tests/golden, produced by the reference compiled from its
sources) against, without a GPU:
  - the numpy restatement of the path (oracle/restate.py): dense contraction,
    permuted copy, multi-term add and dot product of the seeded inputs;
  - the product's host schedule engine: non-zero C schedule and coalesced
    pair lists, bit for bit;
  - the reference library as built now (when oracle/_ref is present)."""
import hashlib
import json
import os

import numpy as np
import pytest

from libtensor_b200.core import Context, block_tensor, btod_contract2, contraction2
from libtensor_b200.spec import BTSpec, permuted_spec
from oracle import refapi as R
from oracle import restate as X
from tests.cases import cases
from tests.golden.make_golden import SEED_A, SEED_B, result_spec, transfer_specs

HERE = os.path.dirname(os.path.abspath(__file__))
G = np.load(os.path.join(HERE, "golden", "golden_contract2.npz"))
T = np.load(os.path.join(HERE, "golden", "golden_transfer.npz"))
META = json.loads(bytes(G["meta"]).decode())
CASES = [c for c in cases() if not c.symmetry_error]
assert [m["name"] for m in META["cases"]] == [c.name for c in CASES]

# Block max-norm relative bound between two FP64 evaluations of the same
# contraction in different summation orders.
TOL = 1e-13


def golden_blocks(i):
    """{abs index: flat data} of the reference's non-zero result blocks."""
    spec = result_spec(CASES[i])
    out, off = {}, 0
    data = G[f"c{i}_c_data"]
    for a in G[f"c{i}_c_abs"]:
        shape = tuple(spec.block_extent(d, b) for d, b in enumerate(X._unabs(int(a), spec.bidims())))
        n = int(np.prod(shape))
        out[int(a)] = data[off:off + n].reshape(shape)
        off += n
    assert off == data.size
    return out


def dense_input(spec, seed, scale, zero=()):
    """Seeded dense tensor with the orbits of the listed blocks zeroed."""
    d = X.seeded_dense(spec, seed, scale)
    if zero:
        orb = X.orbits(spec)
        bid = spec.bidims()
        zc = set()
        for z in zero:
            a = 0
            for k in range(len(bid)):
                a = a * bid[k] + z[k]
            zc.add(orb[a][0])
        for a, (c, _) in orb.items():
            if c in zc:
                X.block_view(spec, d, X._unabs(a, bid))[...] = 0.0
    return d


def rel_err(got, ref):
    m = float(np.max(np.abs(ref))) if ref.size else 0.0
    diff = float(np.max(np.abs(got - ref))) if ref.size else 0.0
    return diff / m if m > 0 else diff


@pytest.mark.parametrize("i", range(len(CASES)), ids=[c.name for c in CASES])
def test_restatement_matches_golden(i):
    case = CASES[i]
    da = dense_input(case.a, SEED_A, case.a_scale, case.zero_a) * case.ka
    db = dense_input(case.b, SEED_B, case.b_scale) * case.kb
    dc = X.dense_contract(da, db, case.n, case.m, case.k, case.permc, case.pairs, case.kc)
    spec = result_spec(case)
    gold = golden_blocks(i)
    assert gold, "the reference produced no non-zero blocks"
    for a, blk in gold.items():
        assert rel_err(X.block_view(spec, dc, X._unabs(a, spec.bidims())), blk) <= TOL, (case.name, a)


@pytest.mark.parametrize("i", range(len(CASES)), ids=[c.name for c in CASES])
def test_host_schedule_matches_golden(i):
    case = CASES[i]
    ctx = Context(-1)
    try:
        A, B = block_tensor(ctx, case.a), block_tensor(ctx, case.b)
        A.mark_nonzero(); B.mark_nonzero()
        for z in case.zero_a:
            A.zero_block(z)
        contr = contraction2(case.n, case.m, case.k, case.permc)
        for p in case.pairs:
            contr.contract(*p)
        op = btod_contract2(contr, A, B, case.ka, case.kb, case.kc)
        sched = op.get_schedule()
        assert sched == [int(x) for x in G[f"c{i}_schedule"]]
        counts, recs = [], []
        for s in range(len(sched)):
            p = op.pairs(s)
            counts.append(len(p))
            for aia, acia, pa, ca, aib, acib, pb, cb in p:
                recs += [aia, acia, *pa, int(np.float64(ca).view(np.int64)),
                         aib, acib, *pb, int(np.float64(cb).view(np.int64))]
        assert counts == [int(x) for x in G[f"c{i}_pair_count"]]
        recs = np.array(recs, np.int64)
        if f"c{i}_pairs" in G.files:
            assert np.array_equal(recs, G[f"c{i}_pairs"])
        else:
            assert hashlib.sha256(recs.tobytes()).digest() == bytes(G[f"c{i}_pairs_sha256"])
    finally:
        ctx.close()


@pytest.mark.skipif(not R.available(), reason="oracle/_ref not built")
@pytest.mark.parametrize("i", [0, 3, 4, 5], ids=[CASES[i].name for i in (0, 3, 4, 5)])
def test_reference_build_matches_golden(i):
    from tests.golden.make_golden import ref_tensor
    case = CASES[i]
    ra = ref_tensor(case.a, SEED_A, case.a_scale, case.zero_a)
    rb = ref_tensor(case.b, SEED_B, case.b_scale)
    op = R.RefContract2(case.n, case.m, case.k, case.permc, case.pairs, ra, rb, case.ka, case.kb, case.kc)
    assert op.schedule() == [int(x) for x in G[f"c{i}_schedule"]]
    rc = op.make_result()
    op.perform(rc)
    spec = result_spec(case)
    # OpenBLAS chooses its dgemm kernel by CPU model, so the reference's own
    # summation order (and its last bits) depends on the host it runs on
    for a, blk in golden_blocks(i).items():
        assert rel_err(rc.get_block(X._unabs(a, spec.bidims()), blk.shape), blk) <= TOL
    for t in (rc, ra, rb):
        t.close()
    op.close()


def _transfer_golden(prefix, spec):
    out, off = {}, 0
    data = T[f"{prefix}_data"]
    for a in T[f"{prefix}_abs"]:
        bidx = X._unabs(int(a), spec.bidims())
        shape = tuple(spec.block_extent(d, b) for d, b in enumerate(bidx))
        n = int(np.prod(shape))
        out[bidx] = data[off:off + n].reshape(shape)
        off += n
    return out


def test_restated_transfers_match_golden():
    t_spec, x_spec = transfer_specs()
    dt = X.seeded_dense(t_spec, 3, 0.01)
    # btod_copy: -0.5 * P(0,2,1,3) t, bit-exact (one exact scaling)
    pspec = permuted_spec(t_spec, (0, 2, 1, 3))
    dcopy = -0.5 * X.dense_permute(dt, (0, 2, 1, 3))
    for bidx, blk in _transfer_golden("copy", pspec).items():
        assert np.array_equal(X.block_view(pspec, dcopy, bidx), blk), bidx
    # btod_add of three terms
    xa, xb = X.seeded_dense(x_spec, 4, 1.0), X.seeded_dense(x_spec, 5, 1.0)
    dadd = xa - 0.5 * X.dense_permute(xb, (1, 0, 3, 2)) + 0.25 * X.dense_permute(xa, (1, 0, 3, 2))
    for bidx, blk in _transfer_golden("add", x_spec).items():
        assert rel_err(X.block_view(x_spec, dadd, bidx), blk) <= 1e-15, bidx
    # btod_dotprod over the full tensors
    assert abs(float(np.sum(dt * dt)) - T["dot_t_t"][0]) <= 1e-13 * abs(T["dot_t_t"][0])
    ref = T["dot_x_xp"][0]
    assert abs(float(np.sum(xa * X.dense_permute(xb, (1, 0, 3, 2)))) - ref) <= 1e-13 * abs(ref)
