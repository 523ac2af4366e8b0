"""Small contraction cases shared by the schedule (CPU) and parity (GPU) tests.
Each mirrors a symmetry situation the reference's btod_contract2 tests cover
(tests/block_tensor/btod_contract2_test.C): antisymmetric pairs (test_contr_4..6),
spin-like partitions (test_contr_20a/b, 21), D2h labels plus spin
(test_contr_24..26), sign cancellation, zero blocks, K = 1 contractions and
permuted results."""
from dataclasses import dataclass, field
from typing import List, Optional, Tuple

from libtensor_b200 import spec as S
from libtensor_b200.spec import BTSpec


@dataclass
class Case:
    name: str
    a: BTSpec
    b: BTSpec
    n: int
    m: int
    k: int
    permc: Optional[List[int]]
    pairs: List[Tuple[int, int]]
    ka: float = 1.0
    kb: float = 1.0
    kc: float = 1.0
    zero_a: List[Tuple[int, ...]] = field(default_factory=list)
    symmetry_error: bool = False          # both sides must reject the contraction
    a_scale: float = 1.0
    b_scale: float = 1.0


def _ladder(cfg, **kw):
    c = cfg.contraction
    return Case(cfg.name, cfg.t_spec(), cfg.v_spec(), c["n"], c["m"], c["k"], c["permc"], c["pairs"],
                kc=cfg.kc, a_scale=cfg.t_scale, b_scale=cfg.v_scale, **kw)


def _ring(cfg, **kw):
    c = cfg.contraction
    return Case(cfg.name, cfg.t_spec(), cfg.w_spec(), c["n"], c["m"], c["k"], c["permc"], c["pairs"],
                kc=cfg.kc, a_scale=cfg.t_scale, b_scale=cfg.v_scale, **kw)


def cases():
    out = []
    out.append(_ladder(S.LADDER_SMALL))
    out.append(_ring(S.RING_D2H_SMALL))
    # ladder with zero blocks in t
    z = _ladder(S.LADDER_SMALL, zero_a=[(0, 1, 0, 2), (1, 1, 2, 3)])
    z.name = "ladder small, zero t blocks"
    out.append(z)
    # matrix product with symmetric A (i <-> p), uneven splits
    a = BTSpec(dims=[13, 13], splits=[[4, 9], [4, 9]], perms=[((1, 0), 1.0)])
    b = BTSpec(dims=[7, 13], splits=[[3], [4, 9]])
    out.append(Case("matrix sym A", a, b, 1, 1, 1, None, [(1, 1)], ka=0.7, kc=-1.5))
    # antisymmetric(cd) x symmetric(cd): the contraction vanishes identically;
    # the reference rejects the derived symmetry (anti-symmetric identity
    # permutation, so_reduce_se_perm_impl.h:86) and so must the product.
    an = BTSpec(dims=[6, 6, 9, 9], splits=[[3], [3], [4], [4]], perms=S.antisym_pairs(4, [(2, 3)]))
    sy = BTSpec(dims=[5, 9, 9], splits=[[2], [4], [4]], perms=[((0, 2, 1), 1.0)])
    out.append(Case("antisym x sym rejected", an, sy, 2, 1, 2, None, [(2, 1), (3, 2)],
                    symmetry_error=True))
    # K = 1, 3-index operands, permuted result C(i,a,j,b) <- A(i,j,k) B(a,b,k)
    a3 = BTSpec(dims=[8, 8, 10], splits=[[3], [3], [4, 7]], perms=[((1, 0, 2), -1.0)])
    b3 = BTSpec(dims=[9, 9, 10], splits=[[5], [5], [4, 7]], perms=[((1, 0, 2), 1.0)])
    out.append(Case("K=1 permuted result", a3, b3, 2, 2, 1, [0, 2, 1, 3], [(2, 2)], kb=2.0))
    # spin partitions with a contraction over one occupied and one virtual index
    o, v = [3], [4, 2]
    so, sv = S.spin_splits(o), S.spin_splits(v)
    t = BTSpec(dims=[6, 6, 12, 12], splits=[so, so, sv, sv], perms=S.antisym_pairs(4, [(0, 1), (2, 3)]),
               part_pdims=[2, 2, 2, 2], part_forbidden=S.spin_forbidden([((0, 1), (2, 3))], 4))
    w = BTSpec(dims=[6, 12, 12, 6], splits=[so, sv, sv, so], part_pdims=[2, 2, 2, 2],
               part_forbidden=S.spin_forbidden([((0, 1), (2, 3))], 4))
    out.append(Case("spin ring no labels", t, w, 2, 2, 2, [0, 3, 1, 2], [(1, 0), (3, 2)], a_scale=0.01))
    return out
