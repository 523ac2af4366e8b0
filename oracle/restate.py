"""CPU restatement (numpy) of the reference's block-tensor contraction path.

TEST INFRASTRUCTURE ONLY (oracle).  It restates, in plain numpy:
  - the seeded, symmetrised test inputs (same bits as the product's
    generator: splitmix64 sum-of-12-uniforms, one final multiply);
  - orbits of blocks under a permutational symmetry group: canonical block =
    minimum absolute index in the orbit (libtensor/core/impl/orbit_impl.h:139-297),
    allowed = every orbit member allowed by se_part / se_label
    (libtensor/symmetry/inst/se_part_impl.h:291-296,
     libtensor/symmetry/inst/se_label_impl.h:74-112);
  - the dense contraction the reference's own tests compare against
    (tests/block_tensor/btod_contract2_test.C:796-817: tod_btconv unfolds the
    block tensors, tod_contract2 contracts the dense tensors), here with
    numpy.einsum;
  - dense copy/add/dot-product (tod_copy, tod_add, tod_dotprod).
"""
from __future__ import annotations

from itertools import product
from typing import List, Sequence, Tuple

import numpy as np

_G = np.uint64(0x9E3779B97F4A7C15)
_C1 = np.uint64(0xBF58476D1CE4E5B9)
_C2 = np.uint64(0x94D049BB133111EB)
_M32 = np.uint64(0xFFFFFFFF)


def sm64_mix(z):
    with np.errstate(over="ignore"):
        z = z + _G
        z = (z ^ (z >> np.uint64(30))) * _C1
        z = (z ^ (z >> np.uint64(27))) * _C2
        return z ^ (z >> np.uint64(31))


def seeded_int(seed: int, lin: np.ndarray) -> np.ndarray:
    key = sm64_mix(np.uint64(seed))
    s = np.zeros(lin.shape, np.uint64)
    with np.errstate(over="ignore"):
        for r in range(6):
            h = sm64_mix(key + lin * np.uint64(6) + np.uint64(r))
            s += (h & _M32) + (h >> np.uint64(32))
    return s.astype(np.int64) - np.int64(6 << 32)


def perm_group(n: int, gens: Sequence[Tuple[Tuple[int, ...], float]]):
    """All (perm, coeff) of the group generated by the se_perm generators."""
    ident = tuple(range(n))
    g = [(ident, 1.0)]
    i = 0
    while i < len(g):
        p, c = g[i]
        for q, cq in gens:
            r = tuple(p[q[k]] for k in range(n))     # "p then q"
            if all(r != x for x, _ in g):
                g.append((r, c * cq))
        i += 1
    return g


def seeded_dense(spec, seed: int, scale: float) -> np.ndarray:
    """Full dense tensor of the seeded symmetrised distribution, with the
    blocks forbidden by se_part / se_label set to zero."""
    dims = spec.dims
    n = len(dims)
    grids = np.indices(dims, dtype=np.uint64).reshape(n, -1)
    v = np.zeros(grids.shape[1], np.int64)
    for p, c in perm_group(n, spec.perms):
        lin = np.zeros(grids.shape[1], np.uint64)
        for d in range(n):
            lin = lin * np.uint64(dims[d]) + grids[p[d]]
        s = seeded_int(seed, lin)
        v = v + s if c > 0 else v - s
    out = v.astype(np.float64) * (scale * 2.0 ** -32)
    out = out.reshape(dims)
    mask = allowed_element_mask(spec)
    return np.where(mask, out, 0.0)


def block_of(spec, d: int) -> np.ndarray:
    """Block number of every index of dim d."""
    st = [0] + list(spec.splits[d]) + [spec.dims[d]]
    b = np.zeros(spec.dims[d], np.int64)
    for k in range(len(st) - 1):
        b[st[k]:st[k + 1]] = k
    return b


def block_allowed(spec, bidx: Sequence[int]) -> bool:
    n = spec.order
    if spec.part_pdims is not None:
        bid = spec.bidims()
        pidx = tuple(bidx[d] // (bid[d] // spec.part_pdims[d]) for d in range(n))
        if pidx in set(tuple(f) for f in spec.part_forbidden):
            return False
    if spec.labels is not None:
        ls = [spec.labels[d][bidx[d]] for d in range(n)]
        if all(x >= 0 for x in ls):
            prod = 0
            for x in ls:
                prod ^= x
            if prod not in spec.label_intr:
                return False
    return True


def allowed_element_mask(spec) -> np.ndarray:
    n = spec.order
    bid = spec.bidims()
    ab = np.zeros(bid, bool)
    for bidx in product(*[range(x) for x in bid]):
        ab[bidx] = block_allowed(spec, bidx)
    idx = np.ix_(*[block_of(spec, d) for d in range(n)])
    return ab[idx]


def orbits(spec):
    """{abs block index: (canonical abs index, allowed)} under the se_perm
    group; allowed when every member is allowed."""
    n = spec.order
    bid = spec.bidims()
    grp = perm_group(n, spec.perms)

    def absi(b):
        a = 0
        for d in range(n):
            a = a * bid[d] + b[d]
        return a

    out = {}
    for b in product(*[range(x) for x in bid]):
        a = absi(b)
        if a in out:
            continue
        mem = {absi(tuple(b[p[d]] for d in range(n))) for p, _ in grp}
        members = sorted(mem)
        allowed = all(block_allowed(spec, _unabs(m, bid)) for m in members)
        for m in members:
            out[m] = (members[0], allowed)
    return out


def _unabs(a, bid):
    out = []
    for d in reversed(bid):
        out.append(a % d)
        a //= d
    return tuple(out[::-1])


def canonical_blocks(spec) -> List[int]:
    return sorted({c for c, ok in orbits(spec).values() if ok})


def block_view(spec, dense: np.ndarray, bidx) -> np.ndarray:
    sl = []
    for d, b in enumerate(bidx):
        st = [0] + list(spec.splits[d]) + [spec.dims[d]]
        sl.append(slice(st[b], st[b + 1]))
    return dense[tuple(sl)]


def pack_canonical(spec, dense: np.ndarray, abs_idx, offsets, total) -> np.ndarray:
    """Arena layout of the product: canonical blocks at the given offsets."""
    arena = np.zeros(max(1, total), np.float64)
    bid = spec.bidims()
    for a, off in zip(abs_idx, offsets):
        blk = block_view(spec, dense, _unabs(int(a), bid))
        arena[off:off + blk.size] = blk.ravel()
    return arena[:total]


def dense_contract(a: np.ndarray, b: np.ndarray, n: int, m: int, k: int, permc, pairs, scale=1.0):
    """C = scale * contraction2<n,m,k>(permc) of dense a, b (tod_contract2)."""
    letters = "abcdefghijklmnopqrstuvwxyz"
    na, nb = n + k, m + k
    sa = [None] * na
    sb = [None] * nb
    li = 0
    for ia, ib in pairs:
        sa[ia] = sb[ib] = letters[li]
        li += 1
    outs = []
    for i in range(na):
        if sa[i] is None:
            sa[i] = letters[li]
            outs.append(letters[li])
            li += 1
    for j in range(nb):
        if sb[j] is None:
            sb[j] = letters[li]
            outs.append(letters[li])
            li += 1
    pc = list(permc) if permc is not None else list(range(n + m))
    out = "".join(outs[pc[i]] for i in range(n + m))
    return scale * np.einsum(f"{''.join(sa)},{''.join(sb)}->{out}", a, b, optimize=True)


def dense_permute(a: np.ndarray, perm) -> np.ndarray:
    """B = P(A) with B[y] = A[x], y[d] = x[perm[d]] (libtensor permutation)."""
    return a if perm is None else np.transpose(a, axes=list(perm))
