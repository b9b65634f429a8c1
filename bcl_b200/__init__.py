"""bcl_b200 — B200-native sparse tile multiply for BCL's SPMatrix / DMatrix.

The product path is the CUDA library libbclx.so (C ABI in include/bclx.h);
``bcl_b200.containers`` mirrors the reference's container API on top of it.
"""
__version__ = "0.1.0"


def __getattr__(name):
    # containers import torch; load them only when used
    if name in ("SPMatrix", "DMatrix", "BlockCustom", "gemm", "spgemm", "spgemm_plain", "spmm", "spmm_plain",
                "tile_accumulate", "context", "split_tiles"):
        from . import containers
        return getattr(containers, name)
    raise AttributeError(name)
