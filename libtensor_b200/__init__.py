"""B200-native block-sparse tensor contraction path with libtensor's operator
surface: btod_contract2 / btod_add / btod_copy / btod_dotprod on symmetric
block tensors, computed by sm_100a kernels behind the C ABI of include/ltg.h."""
from .core import (  # noqa: F401
    Context, Graph, block_tensor, btod_add, btod_contract2, btod_copy, btod_dotprod,
    contraction2, MODE_OZAKI_BF16, MODE_OZAKI_FP8, MODE_OZAKI_INT8, MODE_PLAIN_FP64,
)
from .spec import BTSpec  # noqa: F401
