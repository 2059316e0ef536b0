"""hasteboots_b200: TFHE gate bootstrapping (HasteBoots' tfhe path) on B200 / sm_100a.

The compute lives in libhb_gpu.so (CUDA kernels behind the C ABI in include/hb_gpu.h); this
package is its Python host binding. Build with `python -m hasteboots_b200.build`.
"""

from ._lib import LIB_PATH, HbError, lib  # noqa: F401
