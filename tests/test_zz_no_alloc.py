"""GPU test of ltg_dot_noalloc, the allocation-free dot product.

Collected last (file name) so that it also runs after every other GPU test in
the same process; it must pass alone in a fresh process too.  The reference
value is the existing entry point ltg_dotprod on block tensors without
symmetry, where every block is canonical with orbit weight 1, so the full
tensor dot product equals the dot product of the two packed arenas.
"""
import ctypes as C

import numpy as np
import pytest

from libtensor_b200 import _capi
from libtensor_b200._capi import lib
from libtensor_b200.core import Context, block_tensor, btod_dotprod
from libtensor_b200.spec import BTSpec

pytestmark = pytest.mark.gpu

# Same bound as the dot-product parity tests: two FP64 sums of ~1e6 products
# in different orders.
REL_TOL = 1e-12
LTG_ERR_BAD_ARG = 1


def _last_error() -> str:
    return lib().ltg_last_error().decode(errors="replace")


def _noalloc_dot(x_ptr: int, y_ptr: int, n: int, stream: int):
    out = C.c_double(np.nan)
    st = lib().ltg_dot_noalloc(C.c_void_p(x_ptr), C.c_void_p(y_ptr), n, C.c_void_p(stream),
                               C.byref(out))
    return st, out.value


def _free_device_bytes() -> int:
    """Free memory of the current device (cudaMemGetInfo)."""
    import torch
    return int(torch.cuda.mem_get_info(0)[0])


def test_noalloc_dot_matches_dotprod():
    ctx = Context(0)
    try:
        spec = BTSpec(dims=[24, 30, 40, 44], splits=[[10], [15], [20, 30], [22]])
        a = block_tensor(ctx, spec)
        b = block_tensor(ctx, spec)
        a.fill_seeded(11, 1.0)
        b.fill_seeded(12, 1.0)
        n = a.nelems
        assert n == 24 * 30 * 40 * 44 and n % 65536 != 0   # several units and a ragged tail

        expected = btod_dotprod(a, None, b, None).calculate()
        host = float(np.dot(a.download(), b.download()))
        assert abs(expected - host) <= REL_TOL * abs(host)

        # The first call on a device loads the module (not allocation-free);
        # after it, repeated calls leave the device's free memory unchanged.
        st, _ = _noalloc_dot(a.device_ptr(), b.device_ptr(), n, ctx.stream())
        assert st == _capi.LTG_OK, _last_error()
        free_before = _free_device_bytes()

        results = []
        for _ in range(2):       # two calls in a row share the static array
            st, v = _noalloc_dot(a.device_ptr(), b.device_ptr(), n, ctx.stream())
            assert st == _capi.LTG_OK, _last_error()
            results.append(v)
        for _ in range(3):
            st, _ = _noalloc_dot(a.device_ptr(), b.device_ptr(), n, ctx.stream())
            assert st == _capi.LTG_OK
        assert _free_device_bytes() == free_before
        for v in results:
            assert abs(v - expected) <= REL_TOL * abs(expected), (v, expected)
        assert results[0] == results[1]          # fixed summation order

        # an element count below one unit and the empty case
        st, v = _noalloc_dot(a.device_ptr(), b.device_ptr(), 1000, ctx.stream())
        assert st == _capi.LTG_OK
        ref = float(np.dot(a.download()[:1000], b.download()[:1000]))
        assert abs(v - ref) <= REL_TOL * abs(ref)
        st, v = _noalloc_dot(a.device_ptr(), b.device_ptr(), 0, ctx.stream())
        assert st == _capi.LTG_OK and v == 0.0

        # more elements than the static array can serve: rejected on the host
        st, _ = _noalloc_dot(a.device_ptr(), b.device_ptr(), (1 << 30) + 1, ctx.stream())
        assert st == LTG_ERR_BAD_ARG
        assert "exceed the maximum" in _last_error()
    finally:
        ctx.close()
