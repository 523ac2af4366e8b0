"""Python face of the C ABI, named after the reference's operations.

    ctx = Context(0)
    t = block_tensor(ctx, spec); t.fill_seeded(seed)
    contr = contraction2(2, 2, 2); contr.contract(2, 2); contr.contract(3, 3)
    op = btod_contract2(contr, t, v, kc=0.5)
    r = op.make_result(); op.perform(r)            # r = 0.5 * contr(t, v)
    op.perform(r, 1.0)                             # r += ...
    btod_copy(t, perm, c).perform(u)
    btod_add(x, p1, c1).add_op(x, p2, c2).perform(y)
    e = btod_dotprod(a, None, b, None).calculate()

Every call goes through libltg.so; nothing here computes tensor data.
"""
from __future__ import annotations

import ctypes as C
from typing import List, Optional, Sequence

import numpy as np

from . import _capi
from ._capi import check, lib
from .spec import BTSpec

MODE_PLAIN_FP64 = _capi.MODE_PLAIN_FP64
MODE_OZAKI_BF16 = _capi.MODE_OZAKI_BF16
MODE_OZAKI_FP8 = _capi.MODE_OZAKI_FP8
MODE_OZAKI_INT8 = _capi.MODE_OZAKI_INT8
MODE_OZAKI_CRT = _capi.MODE_OZAKI_CRT


def _i32(vals):
    return (C.c_int32 * max(1, len(vals)))(*vals)


def _perm(p, n):
    return None if p is None else _i32(list(p))


class Context:
    """One device (device >= 0) or a host-only context (device = -1) for
    schedules and orbit queries without a GPU."""

    def __init__(self, device: int = 0):
        h = C.c_void_p()
        check(lib().ltg_ctx_create(device, C.byref(h)))
        self.h = h
        self.device = device

    def synchronize(self):
        check(lib().ltg_ctx_synchronize(self.h))

    def stream(self) -> int:
        s = C.c_void_p()
        check(lib().ltg_ctx_stream(self.h, C.byref(s)))
        return s.value or 0

    def launch_count(self) -> int:
        n = C.c_int64()
        check(lib().ltg_ctx_launch_count(self.h, C.byref(n)))
        return n.value

    KERNELS = ("contract_fp64", "oz_split", "oz_gemm", "transfer", "dot", "scale", "fill", "denominator",
               "oz_combine")

    def set_timing(self, enable: bool):
        """Per-kernel device timing with CUDA events (resets the totals)."""
        check(lib().ltg_ctx_set_timing(self.h, 1 if enable else 0))

    def kernel_times(self):
        """{kernel: (total ms, timed launches)} since timing was enabled."""
        k = len(self.KERNELS)
        ms = (C.c_double * k)()
        n = (C.c_int64 * k)()
        check(lib().ltg_ctx_kernel_times(self.h, ms, n))
        return {name: (ms[i], n[i]) for i, name in enumerate(self.KERNELS) if n[i]}

    def set_wait_limit(self, ns: int):
        """Limit of one pipeline wait inside the tcgen05 products kernels (ns;
        default 2e9).  A wait that runs out makes the call's kernel unwind and
        the next call or synchronize() raise LTG_ERR_TIMEOUT; 0 = no waiting."""
        check(lib().ltg_ctx_set_wait_limit(self.h, int(ns)))

    def wait_limit(self) -> int:
        v = C.c_uint64()
        check(lib().ltg_ctx_wait_limit(self.h, C.byref(v)))
        return v.value

    def set_host_threads(self, n: int):
        check(lib().ltg_ctx_set_host_threads(self.h, n))

    def close(self):
        if self.h:
            check(lib().ltg_ctx_destroy(self.h))
            self.h = None

    # graphs
    def graph_begin(self):
        check(lib().ltg_graph_begin(self.h))

    def graph_end(self) -> "Graph":
        g = C.c_void_p()
        check(lib().ltg_graph_end(self.h, C.byref(g)))
        return Graph(g)


class Graph:
    def __init__(self, h):
        self.h = h

    def launch(self):
        check(lib().ltg_graph_launch(self.h))

    def close(self):
        if self.h:
            check(lib().ltg_graph_destroy(self.h))
            self.h = None


class block_tensor:
    """Canonical blocks of a symmetric block tensor in one device arena."""

    def __init__(self, ctx: Context, spec: Optional[BTSpec] = None, _handle=None):
        self.ctx = ctx
        self.spec = spec
        if _handle is None:
            s = spec.to_ltg()
            h = C.c_void_p()
            check(lib().ltg_bt_create(ctx.h, C.byref(s), C.byref(h)))
            self.h = h
        else:
            self.h = _handle
        order, nb, ne = C.c_int32(), C.c_int64(), C.c_int64()
        check(lib().ltg_bt_info(self.h, C.byref(order), C.byref(nb), C.byref(ne)))
        self.order, self.nblocks, self.nelems = order.value, nb.value, ne.value
        self.abs_idx = np.zeros(max(1, self.nblocks), np.int64)
        self.offsets = np.zeros(max(1, self.nblocks), np.int64)
        self.sizes = np.zeros(max(1, self.nblocks), np.int64)
        check(lib().ltg_bt_blocks(self.h, self.abs_idx.ctypes.data_as(_capi.c_i64p),
                                  self.offsets.ctypes.data_as(_capi.c_i64p),
                                  self.sizes.ctypes.data_as(_capi.c_i64p)))
        self.abs_idx = self.abs_idx[:self.nblocks]
        self.offsets = self.offsets[:self.nblocks]
        self.sizes = self.sizes[:self.nblocks]
        bd = np.zeros(self.order, np.int64)
        check(lib().ltg_bt_bidims(self.h, bd.ctypes.data_as(_capi.c_i64p)))
        self.bidims = [int(x) for x in bd]

    def permuted(self, perm) -> "block_tensor":
        h = C.c_void_p()
        check(lib().ltg_bt_create_permuted(self.h, _i32(list(perm)), C.byref(h)))
        return block_tensor(self.ctx, None, _handle=h)

    def close(self):
        if getattr(self, "h", None):
            check(lib().ltg_bt_destroy(self.h))
            self.h = None

    # ----------------------------------------------------------- queries
    def block_index(self, aidx: int) -> List[int]:
        out, a = [], int(aidx)
        for d in reversed(self.bidims):
            out.append(a % d)
            a //= d
        return out[::-1]

    def abs_index(self, bidx: Sequence[int]) -> int:
        a = 0
        for d, b in zip(self.bidims, bidx):
            a = a * d + int(b)
        return a

    def nonzero(self) -> List[int]:
        n = C.c_int64()
        buf = np.zeros(max(1, self.nblocks), np.int64)
        check(lib().ltg_bt_nonzero(self.h, buf.ctypes.data_as(_capi.c_i64p), len(buf), C.byref(n)))
        return [int(x) for x in buf[:n.value]]

    def orbit(self, aidx: int):
        canon, coeff, allowed = C.c_int64(), C.c_double(), C.c_int32()
        perm = (C.c_int32 * self.order)()
        check(lib().ltg_bt_orbit(self.h, aidx, C.byref(canon), perm, C.byref(coeff), C.byref(allowed)))
        return canon.value, list(perm), coeff.value, bool(allowed.value)

    def block_dims(self, bidx) -> tuple:
        out = (C.c_int64 * self.order)()
        check(lib().ltg_bt_block_dims(self.h, (C.c_int64 * self.order)(*bidx), out))
        return tuple(int(x) for x in out)

    # ----------------------------------------------------------- data
    def upload(self, arena: np.ndarray):
        a = np.ascontiguousarray(arena, dtype=np.float64)
        assert a.size >= self.nelems
        check(lib().ltg_bt_upload(self.h, a.ctypes.data_as(_capi.c_dblp)))

    def download(self) -> np.ndarray:
        a = np.zeros(max(1, self.nelems), np.float64)
        check(lib().ltg_bt_download(self.h, a.ctypes.data_as(_capi.c_dblp)))
        return a[:self.nelems]

    def upload_async(self, ptr: int):
        check(lib().ltg_bt_upload_async(self.h, C.c_void_p(ptr)))

    def download_async(self, ptr: int):
        check(lib().ltg_bt_download_async(self.h, C.c_void_p(ptr)))

    def set_block(self, bidx, data: np.ndarray):
        b = np.ascontiguousarray(data, dtype=np.float64)
        check(lib().ltg_bt_upload_block(self.h, (C.c_int64 * self.order)(*bidx), b.ctypes.data_as(_capi.c_dblp)))

    def get_block(self, bidx, shape) -> np.ndarray:
        out = np.zeros(int(np.prod(shape)), np.float64)
        check(lib().ltg_bt_download_block(self.h, (C.c_int64 * self.order)(*bidx), out.ctypes.data_as(_capi.c_dblp)))
        return out.reshape(shape)

    def set_zero(self):
        check(lib().ltg_bt_set_zero(self.h))

    def mark_nonzero(self):
        check(lib().ltg_bt_mark_nonzero(self.h))

    def zero_block(self, bidx):
        check(lib().ltg_bt_zero_block(self.h, (C.c_int64 * self.order)(*bidx)))

    def fill_seeded(self, seed: int, scale: float = 1.0):
        check(lib().ltg_bt_fill_seeded(self.h, seed, scale))

    def fill_seeded_host(self, seed: int, scale: float = 1.0) -> np.ndarray:
        a = np.zeros(max(1, self.nelems), np.float64)
        check(lib().ltg_bt_fill_seeded_host(self.h, seed, scale, a.ctypes.data_as(_capi.c_dblp)))
        return a[:self.nelems]

    def device_ptr(self) -> int:
        p = C.c_void_p()
        check(lib().ltg_bt_device_ptr(self.h, C.byref(p)))
        return p.value or 0

    def scale(self, c: float):
        check(lib().ltg_scale(self.h, c))

    def denominator(self, eps: np.ndarray, nocc: int = 2):
        e = np.ascontiguousarray(eps, dtype=np.float64)
        check(lib().ltg_denominator(self.h, e.ctypes.data_as(_capi.c_dblp), nocc))

    def blocks(self, arena: np.ndarray):
        """Yields (block index, ndarray view) of every canonical block."""
        for s in range(self.nblocks):
            bidx = self.block_index(self.abs_idx[s])
            shape = self.block_dims(bidx)
            yield bidx, arena[self.offsets[s]:self.offsets[s] + self.sizes[s]].reshape(shape)


class contraction2:
    """contraction2<N,M,K>(permc) + contract(ia, ib) (libtensor/core/contraction2.h:48)."""

    def __init__(self, n: int, m: int, k: int, permc: Optional[Sequence[int]] = None):
        self.n, self.m, self.k = n, m, k
        self.permc = list(permc) if permc is not None else list(range(n + m))
        self.pairs = []

    def contract(self, ia: int, ib: int):
        self.pairs.append((ia, ib))
        return self


class btod_contract2:
    """btod_contract2<N,M,K>(contr, A, ka, B, kb, kc) (btod_contract2.h:29-140)."""

    def __init__(self, contr: contraction2, a: block_tensor, b: block_tensor,
                 ka: float = 1.0, kb: float = 1.0, kc: float = 1.0):
        self.contr, self.a, self.b = contr, a, b
        self.ka, self.kb, self.kc = ka, kb, kc
        h = C.c_void_p()
        pairs = [v for p in contr.pairs for v in p]
        check(lib().ltg_contract2_create(a.ctx.h, contr.n, contr.m, contr.k, _i32(contr.permc),
                                         _i32(pairs), a.h, b.h, C.byref(h)))
        self.h = h

    def close(self):
        if getattr(self, "h", None):
            check(lib().ltg_plan_destroy(self.h))
            self.h = None

    def get_schedule(self) -> List[int]:
        n = C.c_int64()
        check(lib().ltg_plan_schedule(self.h, None, 0, C.byref(n)))
        buf = np.zeros(max(1, n.value), np.int64)
        check(lib().ltg_plan_schedule(self.h, buf.ctypes.data_as(_capi.c_i64p), len(buf), C.byref(n)))
        return [int(x) for x in buf[:n.value]]

    def pairs(self, i: int):
        """Coalesced pairs of schedule entry i:
        [(aia, acia, perm_a, coeff_a, aib, acib, perm_b, coeff_b), ...]."""
        na, nb = self.contr.n + self.contr.k, self.contr.m + self.contr.k
        rec = 2 + na + 1 + 2 + nb + 1
        n = C.c_int64()
        check(lib().ltg_plan_pairs(self.h, i, None, 0, C.byref(n)))
        buf = np.zeros(max(1, n.value * rec), np.int64)
        check(lib().ltg_plan_pairs(self.h, i, buf.ctypes.data_as(_capi.c_i64p), len(buf), C.byref(n)))
        return decode_pairs(buf[:n.value * rec], na, nb)

    def flops(self) -> float:
        f = C.c_double()
        check(lib().ltg_plan_flops(self.h, C.byref(f)))
        return f.value

    def make_result(self) -> block_tensor:
        h = C.c_void_p()
        check(lib().ltg_contract2_make_result(self.h, C.byref(h)))
        return block_tensor(self.a.ctx, None, _handle=h)

    def make_symmetrized(self, symm: bool, idx=(), perm=None) -> block_tensor:
        """A tensor for the contraction symmetrized over an index pair (idx)
        or a unitary permutation (perm): ltg_contract2_make_symmetrized."""
        nidx, arr = _symm_args(self.contr.n + self.contr.m, idx, perm)
        h = C.c_void_p()
        check(lib().ltg_contract2_make_symmetrized(self.h, nidx, arr, 1 if symm else 0, C.byref(h)))
        return block_tensor(self.a.ctx, None, _handle=h)

    def perform_symmetrized(self, r: block_tensor, symm: bool, idx=(), perm=None, c: float = 1.0,
                            mode: int = 0, nslices: int = 0):
        """r = c (T + sign P(T)) with T this contraction (plain FP64, or the
        modular mode), both terms written by the kernel that forms T's
        elements straight into r (ltg_contract2_symmetrized; btod_symmetrize2
        over btod_contract2)."""
        nidx, arr = _symm_args(self.contr.n + self.contr.m, idx, perm)
        check(lib().ltg_contract2_symmetrized(self.h, r.h, mode, nslices, c, nidx, arr, 1 if symm else 0,
                                              self.ka, self.kb, self.kc))

    def set_tile(self, cfg: int):
        check(lib().ltg_contract2_set_tile(self.h, cfg))

    def set_split_k(self, k: int):
        """Plain FP64 mode: k chunks per output tile (0 automatic, 1 never, 2-4 always)."""
        check(lib().ltg_contract2_set_split_k(self.h, k))

    def set_fused_split(self, shape: int):
        """Modular mode: one-read split of row families in kernel shape 1 or 2,
        or 0 (default) for the exponent and residue passes."""
        check(lib().ltg_contract2_set_fused_split(self.h, int(shape)))

    def set_crt_bound(self, sampled: bool):
        """Modular mode: row exponents from sampled bounds checked by the
        residue pass (True, the default) or from an exact exponent pass."""
        check(lib().ltg_contract2_set_crt_bound(self.h, 1 if sampled else 0))

    def set_crt_stage(self, kblocks: int):
        """Modular mode: k blocks per pipeline stage of the products kernel."""
        check(lib().ltg_contract2_set_crt_stage(self.h, kblocks))

    def set_grouping(self, enable: bool):
        """Modular mode: grouped products of small C blocks (default on)."""
        check(lib().ltg_contract2_set_grouping(self.h, 1 if enable else 0))

    def set_crt_rows(self, rows: int):
        """Modular mode: rows of the products kernel's work items (128, 256; 0 default = 256)."""
        check(lib().ltg_contract2_set_crt_rows(self.h, rows))

    def group_info(self, c: block_tensor):
        """(groups, C blocks grouped, grouped-product flops, their blocks'
        algorithmic flops) of the modular mode for result c; host only."""
        ng, nb = C.c_int64(), C.c_int64()
        gf, bf = C.c_double(), C.c_double()
        check(lib().ltg_contract2_group_info(self.h, c.h, C.byref(ng), C.byref(nb), C.byref(gf), C.byref(bf)))
        return ng.value, nb.value, gf.value, bf.value

    def autotune(self, c: block_tensor, mode: int = MODE_PLAIN_FP64, nslices: int = 0, reps: int = 2):
        check(lib().ltg_contract2_autotune(self.h, c.h, mode, nslices, self.ka, self.kb, self.kc, reps))
        return self.tiles()

    def tiles(self):
        n = C.c_int64()
        check(lib().ltg_plan_tiles(self.h, None, None, None, 0, C.byref(n)))
        m = np.zeros(max(1, n.value), np.int64)
        nn = np.zeros(max(1, n.value), np.int64)
        cfg = np.zeros(max(1, n.value), np.int32)
        check(lib().ltg_plan_tiles(self.h, m.ctypes.data_as(_capi.c_i64p), nn.ctypes.data_as(_capi.c_i64p),
                                   cfg.ctypes.data_as(_capi.c_i32p), n.value, C.byref(n)))
        return {(int(a), int(b)): int(c) for a, b, c in zip(m[:n.value], nn[:n.value], cfg[:n.value])}

    def split_bytes(self, c: block_tensor, mode: int, nslices: int = 0, d: Optional[float] = None):
        """(bytes read, bytes written) by the split pass(es) of a split-precision mode."""
        r, w = C.c_int64(), C.c_int64()
        check(lib().ltg_contract2_split_bytes(self.h, c.h, mode, nslices, self.ka, self.kb, self.kc,
                                              0 if d is None else 1, 0.0 if d is None else d,
                                              C.byref(r), C.byref(w)))
        return r.value, w.value

    def perform(self, c: block_tensor, d: Optional[float] = None, mode: int = MODE_PLAIN_FP64,
                nslices: int = 0):
        check(lib().ltg_contract2(self.h, c.h, mode, nslices, self.ka, self.kb, self.kc,
                                  0 if d is None else 1, 0.0 if d is None else d))

    def export_tasks(self, c: block_tensor) -> np.ndarray:
        """Block-pair products of this contraction for result c, one row of
        LTG_TASK_WORDS int64 per product (coefficients without ka, kb, kc)."""
        n = C.c_int64()
        check(lib().ltg_plan_export_tasks(self.h, c.h, None, 0, C.byref(n)))
        buf = np.zeros((max(1, n.value), _capi.LTG_TASK_WORDS), np.int64)
        check(lib().ltg_plan_export_tasks(self.h, c.h, buf.ctypes.data_as(_capi.c_i64p), n.value, C.byref(n)))
        return buf[:n.value]


class contract2_task_plan:
    """A contraction given as a caller-built list of block-pair products over
    the arenas of a, b and the result (rows of LTG_TASK_WORDS int64, as
    btod_contract2.export_tasks writes them); plain FP64 mode only."""

    def __init__(self, a: block_tensor, b: block_tensor, tasks: np.ndarray,
                 ka: float = 1.0, kb: float = 1.0, kc: float = 1.0):
        self.a, self.b = a, b
        self.ka, self.kb, self.kc = ka, kb, kc
        t = np.ascontiguousarray(tasks, dtype=np.int64).reshape(-1, _capi.LTG_TASK_WORDS)
        h = C.c_void_p()
        check(lib().ltg_plan_contract2_upload(a.ctx.h, a.h, b.h, t.ctypes.data_as(_capi.c_i64p), len(t),
                                              C.byref(h)))
        self.h = h
        self.ntasks = len(t)

    def close(self):
        if getattr(self, "h", None):
            check(lib().ltg_plan_free(self.h))
            self.h = None

    def flops(self) -> float:
        f = C.c_double()
        check(lib().ltg_plan_flops(self.h, C.byref(f)))
        return f.value

    def perform(self, c: block_tensor, d: Optional[float] = None, mode: int = MODE_PLAIN_FP64):
        check(lib().ltg_contract2(self.h, c.h, mode, 0, self.ka, self.kb, self.kc,
                                  0 if d is None else 1, 0.0 if d is None else d))


def decode_pairs(buf, na, nb):
    rec = 2 + na + 1 + 2 + nb + 1
    out = []
    for k in range(len(buf) // rec):
        o = buf[k * rec:(k + 1) * rec]
        ca = float(np.frombuffer(np.int64(o[2 + na]).tobytes(), np.float64)[0])
        q = o[3 + na:]
        cb = float(np.frombuffer(np.int64(q[2 + nb]).tobytes(), np.float64)[0])
        out.append((int(o[0]), int(o[1]), tuple(int(x) for x in o[2:2 + na]), ca,
                    int(q[0]), int(q[1]), tuple(int(x) for x in q[2:2 + nb]), cb))
    return out


class btod_copy:
    """btod_copy<N>(A, perm, c).perform(B[, d]) (btod_copy.h:38-115)."""

    def __init__(self, a: block_tensor, perm: Optional[Sequence[int]] = None, c: float = 1.0):
        self.a, self.perm, self.c = a, perm, c

    def perform(self, b: block_tensor, d: Optional[float] = None):
        check(lib().ltg_copy(self.a.h, _perm(self.perm, self.a.order), self.c, b.h,
                             0 if d is None else 1, 0.0 if d is None else d))


class btod_add:
    """btod_add<N>(A, perm, c).add_op(...).perform(B[, d]) (btod_add.h:38-131)."""

    def __init__(self, a: block_tensor, perm: Optional[Sequence[int]] = None, c: float = 1.0):
        self.ops = [(a, perm, c)]

    def add_op(self, a: block_tensor, perm: Optional[Sequence[int]] = None, c: float = 1.0):
        self.ops.append((a, perm, c))
        return self

    def perform(self, b: block_tensor, d: Optional[float] = None):
        n = b.order
        hs = (C.c_void_p * len(self.ops))(*[o[0].h.value if isinstance(o[0].h, C.c_void_p) else o[0].h for o in self.ops])
        perms = []
        for _, p, _ in self.ops:
            perms += list(p) if p is not None else list(range(n))
        cs = (C.c_double * len(self.ops))(*[o[2] for o in self.ops])
        check(lib().ltg_add(len(self.ops), hs, _i32(perms), cs, b.h, 0 if d is None else 1,
                            0.0 if d is None else d))


class btod_dotprod:
    """btod_dotprod<N>(A, permA, B, permB).calculate() (btod_dotprod.h:35-70)."""

    def __init__(self, a: block_tensor, perma, b: block_tensor, permb):
        self.a, self.pa, self.b, self.pb = a, perma, b, permb

    def calculate(self) -> float:
        out = C.c_double()
        check(lib().ltg_dotprod(self.a.h, _perm(self.pa, self.a.order), self.b.h,
                                _perm(self.pb, self.b.order), C.byref(out)))
        return out.value


def _symm_args(n, idx, perm):
    if perm is not None:
        return -1, _i32(list(perm))
    return len(idx), _i32(list(idx))


class btod_symmetrize:
    """Symmetrizer of a tensor (btod_symmetrize2 / btod_symmetrize4,
    libtensor/block_tensor/btod_symmetrize2.h:19, btod_symmetrize4.h:27):
    B = sum over the group of sign * P(A) -- the exchange of two indexes
    (idx of length 2), a unitary permutation (perm), or the 24 permutations
    of four indexes (idx of length 4); sign +1 with symm, else the parity."""

    def __init__(self, a: block_tensor, symm: bool, idx=(), perm=None, c: float = 1.0):
        self.a, self.symm, self.c = a, symm, c
        self.nidx, self.idx = _symm_args(a.order if hasattr(a, "order") else len(a.bidims), idx, perm)

    def make_result(self) -> block_tensor:
        """A tensor with the symmetrized space (ltg_bt_create_symmetrized)."""
        h = C.c_void_p()
        check(lib().ltg_bt_create_symmetrized(self.a.h, self.nidx, self.idx, 1 if self.symm else 0, C.byref(h)))
        return block_tensor(self.a.ctx, None, _handle=h)

    def perform(self, b: block_tensor, d: Optional[float] = None):
        check(lib().ltg_symmetrize(self.a.h, self.c, self.nidx, self.idx, 1 if self.symm else 0, b.h,
                                   0 if d is None else 1, 0.0 if d is None else d))


class btod_contract3:
    """btod_contract3<N1,N2,N3,K1,K2>(contr1, contr2, A, B, C, kd)
    (libtensor/block_tensor/btod_contract3.h:36): D = kd * contr2(contr1(A, B), C),
    the intermediate AB formed in batches of B's non-zero canonical blocks,
    AB = sum_i A B_i (gen_bto_contract3_impl.h:51-260), each batch's
    intermediate kept on the device and contracted with C into D.  One batch
    (the default) forms the whole intermediate once; more batches bound its
    size by contracting A with a copy of B holding only that batch's blocks.
    The operations (and their schedules) are built on the first perform and
    reused."""

    def __init__(self, contr1: contraction2, contr2: contraction2, a: block_tensor, b: block_tensor,
                 c: block_tensor, kd: float = 1.0, batches: int = 1):
        if batches < 1:
            raise ValueError("batches must be >= 1")
        self.contr1, self.contr2 = contr1, contr2
        self.a, self.b, self.c, self.kd = a, b, c, kd
        self.batches = batches
        self._stages = None           # [(B_i, op1_i, AB, op2_i)]

    def _build(self):
        ctx = self.a.ctx
        nz = set(self.b.nonzero())
        slots = [s for s in range(self.b.nblocks) if int(self.b.abs_idx[s]) in nz]
        nb = max(1, min(self.batches, len(slots)))
        # batches of about equal size, canonical blocks in order
        sizes = [int(self.b.sizes[s]) for s in slots]
        total, acc, cut = sum(sizes), 0, [0]
        for i, x in enumerate(sizes):
            acc += x
            if len(cut) < nb and acc >= total * len(cut) / nb:
                cut.append(i + 1)
        cut.append(len(slots))
        self._stages = []
        ab = None
        for i in range(len(cut) - 1):
            if nb == 1:
                bi = self.b
            else:
                bi = self.b.permuted(list(range(self.b.order)))
                btod_copy(self.b).perform(bi)
                keep = set(slots[cut[i]:cut[i + 1]])
                for s in range(bi.nblocks):
                    if s not in keep:
                        bi.zero_block(bi.block_index(bi.abs_idx[s]))
            op1 = btod_contract2(self.contr1, self.a, bi)
            if ab is None:
                ab = op1.make_result()
            self._stages.append([bi, op1, ab, None])

    def perform(self, d: block_tensor, dd: Optional[float] = None, mode: int = MODE_PLAIN_FP64,
                nslices: int = 0):
        """D = kd (AB) C (assign), or D += dd kd (AB) C."""
        if self._stages is None:
            self._build()
        for i, st in enumerate(self._stages):
            bi, op1, ab, op2 = st
            op1.perform(ab, mode=mode, nslices=nslices)
            if op2 is None:
                # the second contraction's schedule follows AB's non-zero blocks
                op2 = st[3] = btod_contract2(self.contr2, ab, self.c, kc=self.kd)
            if i == 0 and dd is None:
                op2.perform(d, mode=mode, nslices=nslices)
            else:
                op2.perform(d, 1.0 if dd is None else dd, mode=mode, nslices=nslices)

    def make_result(self) -> block_tensor:
        if self._stages is None:
            self._build()
        # the result space does not depend on AB's non-zero blocks: a throwaway
        # operation gives it (the stages' own second operations are built after
        # AB is formed, so that their schedules see its blocks)
        tmp = btod_contract2(self.contr2, self._stages[0][2], self.c, kc=self.kd)
        try:
            return tmp.make_result()
        finally:
            tmp.close()

    def close(self):
        for bi, op1, ab, op2 in self._stages or []:
            op1.close()
            if op2 is not None:
                op2.close()
            if bi is not self.b:
                bi.close()
        if self._stages:
            self._stages[0][2].close()
        self._stages = None


class direct_block_tensor(block_tensor):
    """A block tensor holding an operation's result, computed when it is
    first read (libtensor/block_tensor/direct_block_tensor.h:22): as an
    operand of another operation it needs no separate perform.  The whole
    result is formed on the device at the first read (the reference forms
    each block when it is requested); refresh() forms it again at the next
    read, after the operation's inputs changed."""

    def __init__(self, op):
        t = op.make_result()
        self._op, self._t, self._ready = op, t, False
        self.ctx, self.spec = t.ctx, t.spec
        self.order, self.nblocks, self.nelems = t.order, t.nblocks, t.nelems
        self.abs_idx, self.offsets, self.sizes, self.bidims = t.abs_idx, t.offsets, t.sizes, t.bidims

    @property
    def h(self):
        if not self._ready:
            self._ready = True
            self._op.perform(self._t)
        return self._t.h

    def refresh(self):
        self._ready = False

    def close(self):
        if self._t is not None:
            self._t.close()
            self._t = None

