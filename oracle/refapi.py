"""ctypes wrapper of oracle/_ref/libltref.so -- the reference implementation
(libtensor) compiled from its own sources with oracle/ref_driver.C.

TEST INFRASTRUCTURE ONLY: imported by tests/, by __graft_entry__.smoke() as a
checker and by bench.py's CPU-baseline leg.  Product code never imports it.
"""
from __future__ import annotations

import ctypes as C
import os
from typing import List, Optional, Sequence

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
LIB_PATH = os.path.join(HERE, "_ref", "libltref.so")

_i64p = C.POINTER(C.c_int64)
_i32p = C.POINTER(C.c_int32)
_dblp = C.POINTER(C.c_double)
_vp = C.c_void_p

_SIGS = {
    "ref_last_error": (C.c_char_p, []),
    "ref_set_threads": (C.c_int, [C.c_int]),
    "ref_set_batch_size": (None, [C.c_int64]),
    "ref_bt_create": (_vp, [_i64p, C.c_int64]),
    "ref_bt_destroy": (None, [_vp]),
    "ref_bt_order": (C.c_int, [_vp]),
    "ref_bt_set_block": (C.c_int, [_vp, _i64p, _dblp, C.c_int64]),
    "ref_bt_get_block": (C.c_int, [_vp, _i64p, _dblp, C.c_int64]),
    "ref_bt_nonzero": (C.c_int64, [_vp, _i64p, C.c_int64]),
    "ref_bt_block_index_dims": (C.c_int, [_vp, _i64p]),
    "ref_bt_orbit": (C.c_int, [_vp, C.c_int64, _i64p, _i32p, _dblp, _i64p]),
    "ref_contract2_create": (_vp, [C.c_int, C.c_int, C.c_int, _i32p, _i32p, _vp, C.c_double, _vp,
                                   C.c_double, C.c_double]),
    "ref_contract2_destroy": (None, [_vp]),
    "ref_contract2_schedule": (C.c_int64, [_vp, _i64p, C.c_int64]),
    "ref_contract2_make_result": (_vp, [_vp]),
    "ref_contract2_result_bidims": (C.c_int, [_vp, _i64p]),
    "ref_contract2_perform": (C.c_int, [_vp, _vp, C.c_int, C.c_double]),
    "ref_contract2_clst": (C.c_int64, [_vp, C.c_int64, _i64p, C.c_int64]),
    "ref_contract2_cost": (C.c_int, [_vp, _i64p, _i64p]),
    "ref_denominator": (C.c_int, [_vp, _dblp, C.c_int]),
    "ref_symmetrize": (C.c_int, [_vp, C.c_double, C.c_int, _i32p, C.c_int, _vp, C.c_int, C.c_double]),
    "ref_contract2_symmetrize": (C.c_int, [_vp, C.c_int, _i32p, C.c_int, _vp, C.c_int, C.c_double]),
    "ref_bt_fill_seeded": (C.c_int, [_vp, C.c_uint64, C.c_double, C.c_int, _i32p, _i32p, C.c_int]),
    "ref_copy": (C.c_int, [_vp, _i32p, C.c_double, _vp, C.c_int, C.c_double]),
    "ref_add": (C.c_int, [C.c_int, C.POINTER(_vp), _i32p, _dblp, _vp, C.c_int, C.c_double]),
    "ref_dotprod": (C.c_int, [_vp, _i32p, _vp, _i32p, _dblp]),
}

_lib = None
DEFAULT_BATCH_SIZE = 1 << 24


def available() -> bool:
    return os.path.exists(LIB_PATH)


def lib():
    global _lib
    if _lib is None:
        # The bundled OpenBLAS finds its libgfortran/libquadmath next to it.
        names = os.listdir(os.path.dirname(LIB_PATH))
        for prefix in ("libquadmath-", "libgfortran-"):
            for f in sorted(names):
                if f.startswith(prefix):
                    C.CDLL(os.path.join(os.path.dirname(LIB_PATH), f), mode=C.RTLD_GLOBAL)
        L = C.CDLL(LIB_PATH)
        for n, (r, a) in _SIGS.items():
            f = getattr(L, n)
            f.restype = r
            f.argtypes = a
        _lib = L
        # The reference's default batch size 0 makes every batch one block
        # (core/impl/batching_policy_base.C:6 with
        # gen_bto_contract2_batching_policy.h:60-69), i.e. nA*nB*nC batch
        # iterations; one batch per operand is the intended use.
        L.ref_set_batch_size(DEFAULT_BATCH_SIZE)
    return _lib


def _err():
    return lib().ref_last_error().decode(errors="replace")


def _chk(st):
    if st != 0:
        raise RuntimeError("reference: " + _err())


def _i32(v):
    return (C.c_int32 * max(1, len(v)))(*v)


def set_threads(n: int):
    _chk(lib().ref_set_threads(n))


def set_batch_size(b: int):
    lib().ref_set_batch_size(b)


class RefBT:
    """block_tensor<N,double> of the reference with the symmetry of a BTSpec."""

    def __init__(self, spec=None, _handle=None):
        self.spec = spec
        if _handle is None:
            blob = spec.to_ref_blob()
            h = lib().ref_bt_create(blob.ctypes.data_as(_i64p), len(blob))
            if not h:
                raise RuntimeError("reference: " + _err())
            self.h = h
        else:
            self.h = _handle
        self.order = lib().ref_bt_order(self.h)
        bd = np.zeros(self.order, np.int64)
        _chk(lib().ref_bt_block_index_dims(self.h, bd.ctypes.data_as(_i64p)))
        self.bidims = [int(x) for x in bd]

    def close(self):
        if self.h:
            lib().ref_bt_destroy(self.h)
            self.h = None

    def block_index(self, aidx):
        out, a = [], int(aidx)
        for d in reversed(self.bidims):
            out.append(a % d)
            a //= d
        return out[::-1]

    def set_block(self, bidx, data):
        d = np.ascontiguousarray(data, np.float64)
        _chk(lib().ref_bt_set_block(self.h, (C.c_int64 * self.order)(*bidx), d.ctypes.data_as(_dblp), d.size))

    def get_block(self, bidx, shape):
        out = np.zeros(int(np.prod(shape)), np.float64)
        st = lib().ref_bt_get_block(self.h, (C.c_int64 * self.order)(*bidx), out.ctypes.data_as(_dblp), out.size)
        if st < 0:
            raise RuntimeError("reference: " + _err())
        return out.reshape(shape)

    def nonzero(self) -> List[int]:
        n = lib().ref_bt_nonzero(self.h, None, 0)
        buf = np.zeros(max(1, n), np.int64)
        lib().ref_bt_nonzero(self.h, buf.ctypes.data_as(_i64p), len(buf))
        return [int(x) for x in buf[:n]]

    def fill_seeded(self, seed: int, scale: float = 1.0, nthreads: Optional[int] = None):
        """Seeded, symmetrised test inputs in every canonical allowed block
        (the distribution of oracle/restate.seeded_dense, generated inside
        the reference library; bit-identical to the product's generator)."""
        from oracle.restate import perm_group
        n = self.order
        grp = perm_group(n, self.spec.perms)
        perms = _i32([v for p, _ in grp for v in p])
        signs = _i32([1 if c > 0 else -1 for _, c in grp])
        _chk(lib().ref_bt_fill_seeded(self.h, seed, scale, len(grp), perms, signs,
                                      nthreads or os.cpu_count() or 1))

    def orbit(self, aidx):
        canon, coeff, osz = C.c_int64(), C.c_double(), C.c_int64()
        perm = (C.c_int32 * self.order)()
        r = lib().ref_bt_orbit(self.h, aidx, C.byref(canon), perm, C.byref(coeff), C.byref(osz))
        if r < 0:
            raise RuntimeError("reference: " + _err())
        return canon.value, list(perm), coeff.value, bool(r), osz.value


class RefContract2:
    def __init__(self, n, m, k, permc, pairs, a: RefBT, b: RefBT, ka=1.0, kb=1.0, kc=1.0):
        self.n, self.m, self.k = n, m, k
        pc = list(permc) if permc is not None else list(range(n + m))
        pp = [v for p in pairs for v in p]
        h = lib().ref_contract2_create(n, m, k, _i32(pc), _i32(pp), a.h, ka, b.h, kb, kc)
        if not h:
            raise RuntimeError("reference: " + _err())
        self.h = h

    def close(self):
        if self.h:
            lib().ref_contract2_destroy(self.h)
            self.h = None

    def schedule(self) -> List[int]:
        n = lib().ref_contract2_schedule(self.h, None, 0)
        buf = np.zeros(max(1, n), np.int64)
        lib().ref_contract2_schedule(self.h, buf.ctypes.data_as(_i64p), len(buf))
        return [int(x) for x in buf[:n]]

    def pairs(self, cabs):
        na, nb = self.n + self.k, self.m + self.k
        rec = 2 + na + 1 + 2 + nb + 1
        cap = 1 << 16
        while True:
            buf = np.zeros(cap, np.int64)
            n = lib().ref_contract2_clst(self.h, cabs, buf.ctypes.data_as(_i64p), cap)
            if n < 0:
                raise RuntimeError("reference: " + _err())
            if n * rec <= cap:
                break
            cap = n * rec
        out = []
        for k in range(n):
            o = buf[k * rec:(k + 1) * rec]
            ca = float(np.frombuffer(np.int64(o[2 + na]).tobytes(), np.float64)[0])
            q = o[3 + na:]
            cb = float(np.frombuffer(np.int64(q[2 + nb]).tobytes(), np.float64)[0])
            out.append((int(o[0]), int(o[1]), tuple(int(x) for x in o[2:2 + na]), ca,
                        int(q[0]), int(q[1]), tuple(int(x) for x in q[2:2 + nb]), cb))
        return out

    def cost(self):
        """(exact, ref_cost): the schedule's work as the reference's task cost
        counts it -- sum over scheduled C blocks and coalesced pairs of
        K * |C block| -- without and with the reference's per-pair integer
        division by 1000.  2 * exact is the algorithmic FP64 flop count."""
        ex, rc = C.c_int64(), C.c_int64()
        _chk(lib().ref_contract2_cost(self.h, C.byref(ex), C.byref(rc)))
        return ex.value, rc.value

    def symmetrize(self, b: RefBT, symm: bool, idx=(), perm=None, d=None):
        """The contraction symmetrized (btod_symmetrize2/4 wrapping this
        btod_contract2) into b."""
        n, arr = _symm_args(idx, perm)
        _chk(lib().ref_contract2_symmetrize(self.h, n, arr, 1 if symm else 0, b.h, 0 if d is None else 1,
                                            0.0 if d is None else d))

    def make_result(self) -> RefBT:
        h = lib().ref_contract2_make_result(self.h)
        if not h:
            raise RuntimeError("reference: " + _err())
        return RefBT(None, _handle=h)

    def perform(self, c: RefBT, d: Optional[float] = None):
        _chk(lib().ref_contract2_perform(self.h, c.h, 0 if d is None else 1, 0.0 if d is None else d))


def ref_copy(a: RefBT, perm, c, b: RefBT, d=None):
    _chk(lib().ref_copy(a.h, None if perm is None else _i32(list(perm)), c, b.h,
                        0 if d is None else 1, 0.0 if d is None else d))


def ref_add(ops, b: RefBT, d=None):
    n = b.order
    hs = (C.c_void_p * len(ops))(*[o[0].h for o in ops])
    perms = []
    for _, p, _ in ops:
        perms += list(p) if p is not None else list(range(n))
    cs = (C.c_double * len(ops))(*[o[2] for o in ops])
    _chk(lib().ref_add(len(ops), hs, _i32(perms), cs, b.h, 0 if d is None else 1, 0.0 if d is None else d))


def _symm_args(idx, perm):
    if perm is not None:
        return -1, _i32(list(perm))
    return len(idx), _i32(list(idx))


def ref_symmetrize(a: RefBT, c, b: RefBT, symm: bool, idx=(), perm=None, d=None):
    """b = c (A + s P A) (btod_symmetrize2 over indexes idx[0], idx[1] or the
    unitary permutation perm) or the 24-term sum over four indexes idx
    (btod_symmetrize4); s = +1 symmetric, -1 antisymmetric (and the
    permutation's parity for four indexes)."""
    n, arr = _symm_args(idx, perm)
    _chk(lib().ref_symmetrize(a.h, c, n, arr, 1 if symm else 0, b.h, 0 if d is None else 1,
                              0.0 if d is None else d))


def ref_denominator(a: RefBT, eps: np.ndarray, nocc: int):
    """a /= (sum of eps over the first nocc dims - sum over the others), per
    element; eps holds each dimension's values one after the other."""
    e = np.ascontiguousarray(eps, np.float64)
    _chk(lib().ref_denominator(a.h, e.ctypes.data_as(_dblp), nocc))


def ref_dotprod(a: RefBT, pa, b: RefBT, pb) -> float:
    out = C.c_double()
    _chk(lib().ref_dotprod(a.h, None if pa is None else _i32(list(pa)), b.h,
                           None if pb is None else _i32(list(pb)), C.byref(out)))
    return out.value
