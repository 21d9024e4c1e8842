"""B200 engine for the MDFT energy-and-gradient path of dborgis/mdft-dev_general.

The compute lives in libmdft_b200.so (hand-written sm_100a CUDA behind the
C-ABI of include/mdft_b200.h); this package binds that library with ctypes
and provides the seeded synthetic inputs.
"""
from .engine import Engine, Mixture, MdftError, PREC_FP64, PREC_MIXED, library_path, solve_batch  # noqa: F401
from . import inputs  # noqa: F401
from . import synth  # noqa: F401
