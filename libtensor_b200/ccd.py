"""One coupled-cluster-doubles (CCD) amplitude iteration on the block-tensor
path, captured once as a CUDA graph and replayed:

    X  = P(0,2,1,3) t                                      (btod_copy)
    L  = 1/2 sum_cd t(i,j,c,d) V(a,b,c,d)                  (btod_contract2, ladder)
    G  = sum_kc t(i,k,a,c) W(k,b,c,j)                      (btod_contract2, ring)
    R  = L + 1/2 (G - P(ij) G - P(ab) G + P(ij)P(ab) G)    (btod_add)
    R /= e_i + e_j - e_a - e_b                             (denominator)
    E  = <R, t>                                            (btod_dotprod, on the device)
    t  = R                                                 (btod_copy, next iteration)

t is antisymmetric in (i,j) and (a,b), V in (a,b) and (c,d); all tensors are
spin-blocked (alpha blocks, then beta blocks) with spin-forbidden blocks zero.
The two contractions run in the requested arithmetic (plain FP64 or a
split-precision mode).  Every operation is prepared by one eager iteration
before the capture, so the graph holds kernel launches only.
"""
from __future__ import annotations

import ctypes as C
from typing import List

import numpy as np

from .core import (MODE_PLAIN_FP64, Context, block_tensor, btod_add, btod_contract2, btod_copy,
                   contraction2)
from .spec import BTSpec, LadderConfig, spin_forbidden, spin_splits
from ._capi import check, lib


class CCDIteration:
    def __init__(self, ctx: Context, occ_blocks: List[int], vir_blocks: List[int],
                 mode: int = MODE_PLAIN_FP64, nslices: int = 0, seed: int = 7):
        self.ctx, self.mode, self.nslices = ctx, mode, nslices
        cfg = LadderConfig("ccd", list(occ_blocks), list(vir_blocks))
        self.o, self.v = cfg.o, cfg.v
        so, sv = spin_splits(occ_blocks), spin_splits(vir_blocks)
        t_spec, v_spec = cfg.t_spec(), cfg.v_spec()
        w_spec = BTSpec(dims=[self.o, self.v, self.v, self.o], splits=[so, sv, sv, so], part_pdims=[2, 2, 2, 2],
                        part_forbidden=spin_forbidden([((0, 1), (2, 3))], 4))
        self.t = block_tensor(ctx, t_spec)
        self.V = block_tensor(ctx, v_spec)
        self.W = block_tensor(ctx, w_spec)
        self.t.fill_seeded(seed, 0.01)
        self.V.fill_seeded(seed + 1, 0.01)
        self.W.fill_seeded(seed + 2, 0.01)
        # ladder and ring contractions
        cl = contraction2(2, 2, 2).contract(2, 2).contract(3, 3)
        self.ladder = btod_contract2(cl, self.t, self.V, kc=0.5)
        cr = contraction2(2, 2, 2, [0, 3, 1, 2]).contract(1, 0).contract(3, 2)
        self.ring = btod_contract2(cr, self.t, self.W)
        self.L = self.ladder.make_result()
        self.G = self.ring.make_result()
        self.X = self.t.permuted((0, 2, 1, 3))
        self.R = block_tensor(ctx, t_spec)
        self.copy_x = btod_copy(self.t, (0, 2, 1, 3))
        self.combine = btod_add(self.L, None, 1.0)
        self.combine.add_op(self.G, None, 0.5)
        self.combine.add_op(self.G, (1, 0, 2, 3), -0.5)
        self.combine.add_op(self.G, (0, 1, 3, 2), -0.5)
        self.combine.add_op(self.G, (1, 0, 3, 2), 0.5)
        self.copy_back = btod_copy(self.R)
        # orbital energies: occupied near -1, virtual near +1 (|denominator| >= 2)
        rng = np.random.default_rng(seed)
        e_o = -1.0 - rng.random(self.o)
        e_v = 1.0 + rng.random(self.v)
        self.eps = np.concatenate([e_o, e_o, e_v, e_v])
        self.energy_dev = None
        self.graph = None
        self.flops = self.ladder.flops() + self.ring.flops()

    def _energy_buffer(self):
        import torch
        if self.energy_dev is None:
            self.energy_dev = torch.zeros(1, dtype=torch.float64, device=f"cuda:{self.ctx.device}")
        return self.energy_dev

    def step(self):
        """One iteration, enqueued on the context stream."""
        self.copy_x.perform(self.X)
        self.ladder.perform(self.L, mode=self.mode, nslices=self.nslices)
        self.ring.perform(self.G, mode=self.mode, nslices=self.nslices)
        self.combine.perform(self.R)
        self.R.denominator(self.eps, nocc=2)
        e = self._energy_buffer()
        check(lib().ltg_dotprod_async(self.R.h, None, self.t.h, None, C.c_void_p(e.data_ptr())))
        self.copy_back.perform(self.t)

    def capture(self):
        """Runs one eager iteration (prepares every plan), then captures one."""
        self.step()
        self.ctx.synchronize()
        self.ctx.graph_begin()
        try:
            self.step()
        finally:
            self.graph = self.ctx.graph_end()
        return self.graph

    def launch(self):
        self.graph.launch()

    def energy(self) -> float:
        self.ctx.synchronize()
        return float(self.energy_dev.item())

    def close(self):
        if self.graph is not None:
            self.graph.close()
            self.graph = None
        for x in (self.ladder, self.ring):
            x.close()
        for x in (self.X, self.L, self.G, self.R, self.t, self.V, self.W):
            x.close()


__all__ = ["CCDIteration"]
