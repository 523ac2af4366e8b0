"""Generate the golden fixtures of this directory from the reference itself.

Runs libtensor's own btod_contract2 / btod_copy / btod_add / btod_dotprod (the
library compiled from the reference sources by oracle/Makefile, loaded through
oracle/refapi.py) on the seeded inputs of tests/cases.py and stores what the
reference produced:

  golden_contract2.npz   per case: non-zero C schedule, coalesced pair lists
                         (int64 records as ltg_plan_pairs returns them, or
                         their SHA-256 when long), non-zero result blocks and
                         their data
  golden_transfer.npz    btod_copy / btod_add results and btod_dotprod values

Inputs are not stored: they are regenerated bit-identically from
(spec, seed, scale) by the seeded generator (oracle/restate.py on the host,
ltg_bt_fill_seeded on the device).

Usage (from the repository root, after `make -C oracle`):
    python tests/golden/make_golden.py
"""
import hashlib
import json
import os
import sys

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(os.path.dirname(HERE))
sys.path.insert(0, ROOT)

from libtensor_b200 import spec as S  # noqa: E402
from libtensor_b200.spec import BTSpec, permuted_spec  # noqa: E402
from oracle import refapi as R  # noqa: E402
from oracle import restate as RS  # noqa: E402
from tests.cases import cases  # noqa: E402

SEED_A, SEED_B = 11, 23


def result_spec(case):
    """Block index space of C: outer dims of A then of B, permuted by permc."""
    na = case.n + case.k
    ca = {p[0] for p in case.pairs}
    cb = {p[1] for p in case.pairs}
    dims, splits = [], []
    for d in range(na):
        if d not in ca:
            dims.append(case.a.dims[d]); splits.append(list(case.a.splits[d]))
    for d in range(case.m + case.k):
        if d not in cb:
            dims.append(case.b.dims[d]); splits.append(list(case.b.splits[d]))
    pc = case.permc if case.permc is not None else list(range(case.n + case.m))
    return BTSpec(dims=[dims[pc[i]] for i in range(len(pc))], splits=[splits[pc[i]] for i in range(len(pc))])


def ref_tensor(spec, seed, scale, zero=()):
    """Reference block tensor holding the seeded canonical blocks."""
    dense = RS.seeded_dense(spec, seed, scale)
    r = R.RefBT(spec)
    bid = spec.bidims()
    zero = {tuple(z) for z in zero}
    for a in RS.canonical_blocks(spec):
        bidx = RS._unabs(a, bid)
        if bidx in zero:
            continue
        r.set_block(bidx, np.ascontiguousarray(RS.block_view(spec, dense, bidx)))
    return r


def block_shape(spec, bidx):
    return tuple(spec.block_extent(d, b) for d, b in enumerate(bidx))


def dump_blocks(r, spec):
    abs_idx = r.nonzero()
    data = [r.get_block(r.block_index(a), block_shape(spec, r.block_index(a))).ravel() for a in abs_idx]
    return np.array(abs_idx, np.int64), (np.concatenate(data) if data else np.zeros(0))


def pair_records(pairs):
    rec = []
    for aia, acia, pa, ca, aib, acib, pb, cb in pairs:
        rec += [aia, acia, *pa, int(np.float64(ca).view(np.int64)),
                aib, acib, *pb, int(np.float64(cb).view(np.int64))]
    return rec


def transfer_specs():
    so, sv = S.spin_splits([3]), S.spin_splits([4, 3])
    x = BTSpec(dims=[6, 6, 14, 14], splits=[so, so, sv, sv], part_pdims=[2, 2, 2, 2],
               part_forbidden=S.spin_forbidden([((0, 1), (2, 3))], 4))
    return S.LADDER_SMALL.t_spec(), x


def main():
    if not R.available():
        raise SystemExit("oracle/_ref/libltref.so is not built (make -C oracle)")
    out, meta = {}, {"cases": []}
    for i, case in enumerate(c for c in cases() if not c.symmetry_error):
        ra = ref_tensor(case.a, SEED_A, case.a_scale, case.zero_a)
        rb = ref_tensor(case.b, SEED_B, case.b_scale)
        op = R.RefContract2(case.n, case.m, case.k, case.permc, case.pairs, ra, rb,
                            case.ka, case.kb, case.kc)
        sched = op.schedule()
        counts, recs = [], []
        for cabs in sched:
            p = op.pairs(cabs)
            counts.append(len(p))
            recs += pair_records(p)
        rc = op.make_result()
        op.perform(rc)
        c_abs, c_data = dump_blocks(rc, result_spec(case))
        out[f"c{i}_schedule"] = np.array(sched, np.int64)
        out[f"c{i}_pair_count"] = np.array(counts, np.int64)
        recs = np.array(recs, np.int64)
        if recs.size > 20000:     # long lists: a digest of the int64 records
            out[f"c{i}_pairs_sha256"] = np.frombuffer(hashlib.sha256(recs.tobytes()).digest(), np.uint8)
        else:
            out[f"c{i}_pairs"] = recs
        out[f"c{i}_c_abs"] = c_abs
        out[f"c{i}_c_data"] = c_data
        meta["cases"].append({"index": i, "name": case.name, "seed_a": SEED_A, "seed_b": SEED_B})
        for t in (rc, ra, rb):
            t.close()
        op.close()
    out["meta"] = np.frombuffer(json.dumps(meta).encode(), np.uint8)
    np.savez_compressed(os.path.join(HERE, "golden_contract2.npz"), **out)

    # btod_copy / btod_add / btod_dotprod
    t_spec, x_spec = transfer_specs()
    tr = {}
    ta = ref_tensor(t_spec, 3, 0.01)
    perm = (0, 2, 1, 3)
    tb = R.RefBT(permuted_spec(t_spec, perm))
    R.ref_copy(ta, perm, -0.5, tb)
    tr["copy_abs"], tr["copy_data"] = dump_blocks(tb, permuted_spec(t_spec, perm))
    xa = ref_tensor(x_spec, 4, 1.0)
    xb = ref_tensor(x_spec, 5, 1.0)
    xc = R.RefBT(x_spec)
    R.ref_add([(xa, None, 1.0), (xb, (1, 0, 3, 2), -0.5), (xa, (1, 0, 3, 2), 0.25)], xc)
    tr["add_abs"], tr["add_data"] = dump_blocks(xc, x_spec)
    tr["dot_t_t"] = np.array([R.ref_dotprod(ta, None, ta, None)])
    tr["dot_x_xp"] = np.array([R.ref_dotprod(xa, None, xb, (1, 0, 3, 2))])
    np.savez_compressed(os.path.join(HERE, "golden_transfer.npz"), **tr)
    for t in (ta, tb, xa, xb, xc):
        t.close()
    print("wrote", sorted(os.listdir(HERE)))


if __name__ == "__main__":
    main()
