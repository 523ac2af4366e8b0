"""Shared test helpers: seeded inputs on both sides (product library and the
reference compiled under oracle/_ref) and block-wise comparisons."""
import numpy as np

from libtensor_b200.core import block_tensor
from oracle import refapi as R


def seeded_pair(ctx, spec, seed, scale, zero=()):
    """Product tensor filled on the host with the seeded distribution, the
    reference tensor holding bit-identical canonical blocks, and the arena.
    Blocks listed in `zero` are zero blocks on both sides."""
    t = block_tensor(ctx, spec)
    arena = t.fill_seeded_host(seed, scale)
    zero = {tuple(z) for z in zero}
    if ctx.device >= 0:
        t.upload(arena)
    else:
        t.mark_nonzero()
    for z in zero:
        t.zero_block(z)
    r = R.RefBT(spec)
    for bidx, blk in t.blocks(arena):
        if tuple(bidx) in zero:
            blk[...] = 0.0
            continue
        r.set_block(bidx, blk)
    return t, r, arena


def block_errors(t, arena, ref, spec):
    """Per canonical block: (bidx, max|diff|, max|ref|) against the reference."""
    out = []
    for bidx, blk in t.blocks(arena):
        rb = ref.get_block(bidx, blk.shape)
        out.append((tuple(bidx), float(np.max(np.abs(blk - rb))) if blk.size else 0.0,
                    float(np.max(np.abs(rb))) if blk.size else 0.0))
    return out


def max_rel_block_error(errs, floor=1e-300):
    worst = 0.0
    for _, d, m in errs:
        if m > floor:
            worst = max(worst, d / m)
        elif d > 0:
            worst = max(worst, np.inf)
    return worst


def contraction_args(cfg):
    c = cfg.contraction
    return c["n"], c["m"], c["k"], c["permc"], c["pairs"]
