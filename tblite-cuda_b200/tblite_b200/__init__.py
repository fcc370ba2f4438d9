"""tblite-b200: B200-native (sm_100a) GFN2-xTB singlepoint engine.

Python host-side mirror of the reference's xtb_singlepoint path; all compute
runs in the CUDA library lib/libtblite_b200.so through the C ABI of
include/tblite_b200.h.
"""
from .capi import (Batch, Calculator, DEFAULT_PARAMS, LIB_PATH, TBError, default_options,  # noqa: F401
                   load_library)
from . import geometry  # noqa: F401
