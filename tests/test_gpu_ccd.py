"""CCD iteration captured as one CUDA graph: the graph replay gives the same
bits as the eager sequence, and one iteration matches a dense numpy
restatement of the same algebra (contractions, antisymmetrising add,
denominator, energy)."""
import numpy as np
import pytest

from libtensor_b200.ccd import CCDIteration
from libtensor_b200.core import MODE_OZAKI_CRT, MODE_PLAIN_FP64, Context
from oracle import restate as X

pytestmark = pytest.mark.gpu

OCC, VIR = [3], [4, 3]


@pytest.fixture(scope="module")
def gctx():
    c = Context(0)
    yield c
    c.close()


@pytest.mark.parametrize("mode,nslices", [(MODE_PLAIN_FP64, 0), (MODE_OZAKI_CRT, 13)], ids=["fp64", "crt13"])
def test_graph_replay_matches_eager(gctx, mode, nslices):
    a = CCDIteration(gctx, OCC, VIR, mode, nslices)
    b = CCDIteration(gctx, OCC, VIR, mode, nslices)
    a.step()
    a.step()
    b.capture()          # one eager iteration, then the captured one (recorded, not run)
    b.launch()
    assert np.array_equal(a.t.download().view(np.uint64), b.t.download().view(np.uint64))
    assert a.energy() == b.energy()
    for _ in range(3):   # replays keep agreeing with eager steps
        a.step()
        b.launch()
    assert np.array_equal(a.t.download().view(np.uint64), b.t.download().view(np.uint64))
    a.close()
    b.close()


def test_one_iteration_matches_dense_algebra(gctx):
    it = CCDIteration(gctx, OCC, VIR, MODE_PLAIN_FP64, 0)
    t0 = X.seeded_dense(it.t.spec, 7, 0.01)
    V = X.seeded_dense(it.V.spec, 8, 0.01)
    W = X.seeded_dense(it.W.spec, 9, 0.01)
    it.step()
    L = 0.5 * np.einsum("ijcd,abcd->ijab", t0, V)
    G = np.einsum("ikac,kbcj->ijab", t0, W)
    R = L + 0.5 * (G - G.transpose(1, 0, 2, 3) - G.transpose(0, 1, 3, 2) + G.transpose(1, 0, 3, 2))
    o, v = it.o, it.v
    e = it.eps
    D = e[:o, None, None, None] + e[o:2 * o][None, :, None, None] - e[2 * o:2 * o + v][None, None, :, None] \
        - e[2 * o + v:][None, None, None, :]
    Rd = np.where(X.allowed_element_mask(it.t.spec), R / D, 0.0)
    got = it.t.download()                          # t <- R after the iteration
    worst = 0.0
    for bidx, blk in it.t.blocks(got):
        ref = X.block_view(it.t.spec, Rd, bidx)
        m = float(np.max(np.abs(ref))) if ref.size else 0.0
        if m > 0:
            worst = max(worst, float(np.max(np.abs(blk - ref))) / m)
    assert worst <= 1e-12, worst
    E = float(np.sum(Rd * t0))
    assert abs(it.energy() - E) <= 1e-12 * abs(E)
    it.close()


def test_iteration_at_full_size_matches_reference(gctx):
    """CCD iteration o=30 v=300 (blocks 15 / 50,50,50 per spin) against the
    same iteration on the reference built from its sources (btod_copy,
    btod_contract2 x 2, btod_add, the denominator, btod_dotprod; one
    operation after the other, oracle/ref_ccd.py):
      - the permuted copy X = P(0,2,1,3) t bit-identical;
      - plain FP64: new amplitudes within 1e-12 per block and the energy
        within 1e-12 relative;
      - both contractions in split precision (modular INT8, 13 moduli): the
        energy within 1e-11 relative of the plain FP64 iteration and of the
        reference."""
    from libtensor_b200 import spec as S
    from oracle import refapi as R
    from oracle.ref_ccd import RefCCDIteration
    if not R.available():
        pytest.skip("oracle/_ref not built")
    cfg = S.LADDER_CCD
    R.set_threads(__import__("os").cpu_count() or 1)
    ref = RefCCDIteration(cfg.occ_blocks, cfg.vir_blocks)
    ref.step()
    e_ref = ref.energy
    assert e_ref != 0.0
    energies = {}
    for mode, nslices in ((MODE_PLAIN_FP64, 0), (MODE_OZAKI_CRT, 13)):
        it = CCDIteration(gctx, cfg.occ_blocks, cfg.vir_blocks, mode, nslices)
        assert it.flops == ref.flops
        it.step()
        energies[mode] = it.energy()
        if mode == MODE_PLAIN_FP64:
            for bidx, blk in it.X.blocks(it.X.download()):
                want = ref.X.get_block(bidx, blk.shape)
                assert np.array_equal(blk.view(np.uint64), want.view(np.uint64)), bidx
            worst = 0.0
            for bidx, blk in it.t.blocks(it.t.download()):
                want = ref.t.get_block(bidx, blk.shape)
                m = float(np.max(np.abs(want))) if want.size else 0.0
                if m > 0:
                    worst = max(worst, float(np.max(np.abs(blk - want))) / m)
            assert worst <= 1e-12, worst
        it.close()
    ref.close()
    e64, e_split = energies[MODE_PLAIN_FP64], energies[MODE_OZAKI_CRT]
    assert abs(e64 - e_ref) <= 1e-12 * abs(e_ref), (e64, e_ref)
    assert abs(e_split - e64) <= 1e-11 * abs(e64), (e64, e_split)
    assert abs(e_split - e_ref) <= 1e-11 * abs(e_ref), (e_ref, e_split)
