"""Block-tensor descriptions (block index space + symmetry) and the synthetic
workloads of the contraction path.

A `BTSpec` carries what libtensor's `block_index_space<N>` and
`symmetry<N,double>` carry for this path: per-dimension split points,
`se_perm` generators, one `se_part` element with forbidden partitions and one
`se_label` element for an abelian (XOR) point group.  The same description
feeds the product library (as an `ltg_bt_spec`) and the oracle (as its flat
int64 spec).
"""
from __future__ import annotations

import ctypes as C
from dataclasses import dataclass, field
from itertools import product
from typing import List, Optional, Sequence, Tuple

import numpy as np


@dataclass
class BTSpec:
    dims: List[int]
    splits: List[List[int]]
    perms: List[Tuple[Tuple[int, ...], float]] = field(default_factory=list)
    part_pdims: Optional[List[int]] = None
    part_forbidden: List[Tuple[int, ...]] = field(default_factory=list)
    labels: Optional[List[List[int]]] = None      # per dim, per block (-1: none)
    label_nirrep: int = 8
    label_intr: List[int] = field(default_factory=lambda: [0])

    @property
    def order(self) -> int:
        return len(self.dims)

    def bidims(self) -> List[int]:
        return [len(s) + 1 for s in self.splits]

    def block_starts(self, d: int) -> List[int]:
        return [0] + list(self.splits[d])

    def block_extent(self, d: int, b: int) -> int:
        st = self.block_starts(d) + [self.dims[d]]
        return st[b + 1] - st[b]

    # ------------------------------------------------------------ product ABI
    def to_ltg(self):
        from ._capi import ltg_bt_spec
        n = self.order
        keep = []

        def arr(ctype, vals):
            a = (ctype * max(1, len(vals)))(*vals)
            keep.append(a)
            return a

        s = ltg_bt_spec()
        s.order = n
        s.dims = arr(C.c_int64, self.dims)
        s.nsplit = arr(C.c_int32, [len(x) for x in self.splits])
        s.splits = arr(C.c_int64, [v for x in self.splits for v in x])
        s.nperm = len(self.perms)
        s.perm = arr(C.c_int32, [v for p, _ in self.perms for v in p])
        s.perm_coeff = arr(C.c_double, [c for _, c in self.perms])
        s.has_part = 1 if self.part_pdims is not None else 0
        s.part_pdims = arr(C.c_int64, self.part_pdims or [1] * n)
        s.npart_forbidden = len(self.part_forbidden)
        s.part_forbidden = arr(C.c_int64, [v for f in self.part_forbidden for v in f])
        s.has_label = 1 if self.labels is not None else 0
        s.label_nirrep = self.label_nirrep
        s.labels = arr(C.c_int32, [v for x in (self.labels or []) for v in x])
        s.label_nintr = len(self.label_intr)
        s.label_intr = arr(C.c_int32, self.label_intr)
        s._keep = keep
        return s

    # ------------------------------------------------------------ oracle spec
    def to_ref_blob(self) -> np.ndarray:
        n = self.order
        types, seen = [], []
        for d in range(n):
            key = (self.dims[d], tuple(self.splits[d]))
            if key not in seen:
                seen.append(key)
            types.append(seen.index(key))
        v = [n, *self.dims, *types]
        for t, (_, sp) in enumerate(seen):
            v += [len(sp), *sp]
        v.append(len(self.perms))
        for p, c in self.perms:
            v += [*p, int(c)]
        if self.part_pdims is not None:
            v += [1, *self.part_pdims, len(self.part_forbidden)]
            for f in self.part_forbidden:
                v += list(f)
            v.append(0)     # no partition maps
        else:
            v.append(0)
        if self.labels is not None:
            v += [1, self.label_nirrep]
            for d in range(n):
                v += [len(self.labels[d]), *self.labels[d]]
            v += [len(self.label_intr), *self.label_intr]
        else:
            v.append(0)
        return np.asarray(v, dtype=np.int64)


def permuted_spec(s: BTSpec, perm: Sequence[int]) -> BTSpec:
    """Description of P(A) for B[y] = A[x], y[d] = x[perm[d]] (so_permute)."""
    n = s.order
    p = list(perm)
    pinv = [0] * n
    for i, v in enumerate(p):
        pinv[v] = i
    perms = [(tuple(pinv[q[p[i]]] for i in range(n)), c) for q, c in s.perms]
    forb = [tuple(f[p[d]] for d in range(n)) for f in s.part_forbidden]
    return BTSpec(dims=[s.dims[p[d]] for d in range(n)], splits=[list(s.splits[p[d]]) for d in range(n)],
                  perms=perms, part_pdims=None if s.part_pdims is None else [s.part_pdims[p[d]] for d in range(n)],
                  part_forbidden=forb, labels=None if s.labels is None else [list(s.labels[p[d]]) for d in range(n)],
                  label_nirrep=s.label_nirrep, label_intr=list(s.label_intr))


# ---------------------------------------------------------------- helpers

def spin_splits(per_spin_blocks: Sequence[int]) -> List[int]:
    """Split points of a dimension holding alpha blocks then beta blocks."""
    sizes = list(per_spin_blocks) * 2
    pos, out = 0, []
    for s in sizes[:-1]:
        pos += s
        out.append(pos)
    return out


def spin_forbidden(pairs: Sequence[Tuple[Sequence[int], Sequence[int]]], n: int):
    """Forbidden spin partitions of an n-index tensor: a partition index p
    (0 = alpha, 1 = beta per dim) is allowed when, for each (bra, ket) group,
    the number of beta indices in bra equals that in ket."""
    forb = []
    for p in product(range(2), repeat=n):
        ok = all(sum(p[i] for i in bra) == sum(p[i] for i in ket) for bra, ket in pairs)
        if not ok:
            forb.append(tuple(p))
    return forb


def antisym_pairs(n, pairs):
    """se_perm generators swapping each (i, j) with coefficient -1."""
    gens = []
    for i, j in pairs:
        p = list(range(n))
        p[i], p[j] = p[j], p[i]
        gens.append((tuple(p), -1.0))
    return gens


# ---------------------------------------------------------------- workloads

@dataclass
class LadderConfig:
    """r(i,j,a,b) = 0.5 * sum_cd t(i,j,c,d) V(a,b,c,d), spin-orbital,
    antisymmetric in i<->j, a<->b, c<->d, spin-nonconserving blocks zero."""
    name: str
    occ_blocks: List[int]      # per spin
    vir_blocks: List[int]      # per spin

    @property
    def o(self):
        return 2 * sum(self.occ_blocks)

    @property
    def v(self):
        return 2 * sum(self.vir_blocks)

    def t_spec(self) -> BTSpec:
        so, sv = spin_splits(self.occ_blocks), spin_splits(self.vir_blocks)
        return BTSpec(dims=[self.o, self.o, self.v, self.v], splits=[so, so, sv, sv],
                      perms=antisym_pairs(4, [(0, 1), (2, 3)]), part_pdims=[2, 2, 2, 2],
                      part_forbidden=spin_forbidden([((0, 1), (2, 3))], 4))

    def v_spec(self) -> BTSpec:
        sv = spin_splits(self.vir_blocks)
        return BTSpec(dims=[self.v] * 4, splits=[sv] * 4,
                      perms=antisym_pairs(4, [(0, 1), (2, 3)]), part_pdims=[2, 2, 2, 2],
                      part_forbidden=spin_forbidden([((0, 1), (2, 3))], 4))

    def x_spec(self) -> BTSpec:
        """An (o,o,v,v) intermediate before antisymmetrisation: spin blocks
        only, no permutational symmetry (the input of P(ij)P(ab) in a CC
        residual)."""
        so, sv = spin_splits(self.occ_blocks), spin_splits(self.vir_blocks)
        return BTSpec(dims=[self.o, self.o, self.v, self.v], splits=[so, so, sv, sv],
                      part_pdims=[2, 2, 2, 2],
                      part_forbidden=spin_forbidden([((0, 1), (2, 3))], 4))

    # contraction2<2,2,2>: contract t.2 with V.2 and t.3 with V.3
    contraction = dict(n=2, m=2, k=2, permc=None, pairs=[(2, 2), (3, 3)])
    kc = 0.5
    t_scale = 0.01
    v_scale = 1.0


LADDER_SMALL = LadderConfig("ladder o=10 v=40", [5], [16, 4])
LADDER_LARGE = LadderConfig("ladder o=40 v=240", [20], [48, 40, 32])
LADDER_SPLIT = LadderConfig("ladder o=40 v=240 (64,56)", [20], [64, 56])
LADDER_CCD = LadderConfig("ladder o=30 v=300", [15], [50, 50, 50])
LADDER_PROF = LadderConfig("ladder o=40 v=160", [20], [48, 32])   # profiling size (< 1 GB)

D2H_OCC = [6, 2, 3, 1, 5, 2, 3, 1]
D2H_VIR = [40, 12, 18, 8, 36, 10, 16, 8]


@dataclass
class RingConfig:
    """r(i,j,a,b) += sum_kc t(i,k,a,c) W(k,b,c,j) with D2h labels (one block per
    irrep and spin) and spin partitions."""
    name: str
    occ_irrep: List[int]
    vir_irrep: List[int]
    nirrep: int = 8

    @property
    def o(self):
        return 2 * sum(self.occ_irrep)

    @property
    def v(self):
        return 2 * sum(self.vir_irrep)

    def _labels(self, nblk):
        return [b % self.nirrep for b in range(nblk)]

    def t_spec(self) -> BTSpec:
        so, sv = spin_splits(self.occ_irrep), spin_splits(self.vir_irrep)
        lo, lv = self._labels(len(so) + 1), self._labels(len(sv) + 1)
        return BTSpec(dims=[self.o, self.o, self.v, self.v], splits=[so, so, sv, sv],
                      perms=antisym_pairs(4, [(0, 1), (2, 3)]), part_pdims=[2, 2, 2, 2],
                      part_forbidden=spin_forbidden([((0, 1), (2, 3))], 4),
                      labels=[lo, lo, lv, lv], label_nirrep=self.nirrep, label_intr=[0])

    def w_spec(self) -> BTSpec:
        so, sv = spin_splits(self.occ_irrep), spin_splits(self.vir_irrep)
        lo, lv = self._labels(len(so) + 1), self._labels(len(sv) + 1)
        return BTSpec(dims=[self.o, self.v, self.v, self.o], splits=[so, sv, sv, so],
                      perms=[], part_pdims=[2, 2, 2, 2],
                      part_forbidden=spin_forbidden([((0, 1), (2, 3))], 4),
                      labels=[lo, lv, lv, lo], label_nirrep=self.nirrep, label_intr=[0])

    # t(i,k,a,c) W(k,b,c,j): contract t.1-W.0 (k), t.3-W.2 (c); the natural
    # result order (i,a,b,j) is permuted to (i,j,a,b).
    contraction = dict(n=2, m=2, k=2, permc=[0, 3, 1, 2], pairs=[(1, 0), (3, 2)])
    kc = 1.0
    t_scale = 0.01
    v_scale = 1.0


RING_D2H = RingConfig("ring D2h o=46 v=296", D2H_OCC, D2H_VIR)
RING_D2H_SMALL = RingConfig("ring D2h small", [2, 1, 1, 1, 2, 1, 1, 1], [5, 2, 3, 1, 4, 2, 3, 1])


@dataclass
class DenseConfig:
    """C(i,j) = sum_k A(i,k) B(j,k) with one block per tensor and no symmetry:
    the DMMA kernel on one long product, without a schedule's uneven end."""
    name: str
    n: int

    @property
    def o(self):
        return self.n

    @property
    def v(self):
        return self.n

    def t_spec(self) -> BTSpec:
        return BTSpec(dims=[self.n, self.n], splits=[[], []])

    def v_spec(self) -> BTSpec:
        return BTSpec(dims=[self.n, self.n], splits=[[], []])

    contraction = dict(n=1, m=1, k=1, permc=None, pairs=[(1, 1)])
    kc = 1.0
    t_scale = 1.0
    v_scale = 1.0


DENSE_6144 = DenseConfig("dense 6144^3", 6144)

