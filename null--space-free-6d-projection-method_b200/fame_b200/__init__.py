"""fame_b200 — B200 (sm_100a) eigensolver hot path of the 6D null-space-free
Maxwell projection method, behind the C ABI of include/fame.h.

The host layer mirrors the reference's MATLAB interface (applyMij_fft, the
mass handles, apply_V_blockdiag / solveV1_blockdiag, make_explicit_krinv_compact,
make_nested_krinv_instrumented, Lanczos, the Taylor / direct Yee-field
reconstruction).  All compute runs in libfame_b200.so; importing the package
fails if the library has not been built.
"""
from ._lib import FameError, LIB_PATH  # noqa: F401  (loads the library or raises)
from .core import *  # noqa: F401,F403
from . import configs  # noqa: F401
from .recon import *  # noqa: F401,F403
from . import grad  # noqa: F401
from .method_a import *  # noqa: F401,F403
from . import autotune  # noqa: F401
from . import results  # noqa: F401
