"""One CCD amplitude iteration on the reference (oracle/_ref), operation by
operation, on the same seeded inputs as the product's CCD iteration:

    X  = P(0,2,1,3) t                                      (btod_copy)
    L  = 1/2 sum_cd t(i,j,c,d) V(a,b,c,d)                  (btod_contract2, ladder)
    G  = sum_kc t(i,k,a,c) W(k,b,c,j)                      (btod_contract2, ring)
    R  = L + 1/2 (G - P(ij) G - P(ab) G + P(ij)P(ab) G)    (btod_add)
    R /= e_i + e_j - e_a - e_b                             (caller loop over blocks)
    E  = <R, t>                                            (btod_dotprod)
    t  = R                                                 (btod_copy)

TEST INFRASTRUCTURE ONLY: the parity check of the product's iteration (energy,
amplitudes, the permuted copy) and the CPU baseline of the CCD workload.
"""
from __future__ import annotations

from typing import List

import numpy as np

from libtensor_b200.spec import BTSpec, LadderConfig, permuted_spec, spin_forbidden, spin_splits
from oracle import refapi as R


def ccd_specs(occ_blocks: List[int], vir_blocks: List[int]):
    """(t, V, W) descriptions of the iteration's tensors."""
    cfg = LadderConfig("ccd", list(occ_blocks), list(vir_blocks))
    so, sv = spin_splits(occ_blocks), spin_splits(vir_blocks)
    w = BTSpec(dims=[cfg.o, cfg.v, cfg.v, cfg.o], splits=[so, sv, sv, so], part_pdims=[2, 2, 2, 2],
               part_forbidden=spin_forbidden([((0, 1), (2, 3))], 4))
    return cfg, cfg.t_spec(), cfg.v_spec(), w


def orbital_energies(o: int, v: int, seed: int) -> np.ndarray:
    """Occupied near -1, virtual near +1, per dimension of an (o,o,v,v) tensor."""
    rng = np.random.default_rng(seed)
    e_o = -1.0 - rng.random(o)
    e_v = 1.0 + rng.random(v)
    return np.concatenate([e_o, e_o, e_v, e_v])


class RefCCDIteration:
    def __init__(self, occ_blocks: List[int], vir_blocks: List[int], seed: int = 7):
        cfg, t_spec, v_spec, w_spec = ccd_specs(occ_blocks, vir_blocks)
        self.o, self.v = cfg.o, cfg.v
        self.t, self.V, self.W = R.RefBT(t_spec), R.RefBT(v_spec), R.RefBT(w_spec)
        self.t.fill_seeded(seed, 0.01)
        self.V.fill_seeded(seed + 1, 0.01)
        self.W.fill_seeded(seed + 2, 0.01)
        self.ladder = R.RefContract2(2, 2, 2, None, [(2, 2), (3, 3)], self.t, self.V, 1.0, 1.0, 0.5)
        self.ring = R.RefContract2(2, 2, 2, [0, 3, 1, 2], [(1, 0), (3, 2)], self.t, self.W, 1.0, 1.0, 1.0)
        self.L = self.ladder.make_result()
        self.G = self.ring.make_result()
        self.X = R.RefBT(permuted_spec(t_spec, (0, 2, 1, 3)))
        self.R = R.RefBT(t_spec)
        self.eps = orbital_energies(self.o, self.v, seed)
        self.energy = None
        self.flops = 2.0 * (self.ladder.cost()[0] + self.ring.cost()[0])

    def step(self):
        R.ref_copy(self.t, (0, 2, 1, 3), 1.0, self.X)
        self.ladder.perform(self.L)
        self.ring.perform(self.G)
        G = self.G
        R.ref_add([(self.L, None, 1.0), (G, None, 0.5), (G, (1, 0, 2, 3), -0.5), (G, (0, 1, 3, 2), -0.5),
                   (G, (1, 0, 3, 2), 0.5)], self.R)
        R.ref_denominator(self.R, self.eps, 2)
        self.energy = R.ref_dotprod(self.R, None, self.t, None)
        R.ref_copy(self.R, None, 1.0, self.t)

    def close(self):
        for x in (self.ladder, self.ring):
            x.close()
        for x in (self.L, self.G, self.X, self.R, self.t, self.V, self.W):
            x.close()
