"""B200-native force engine for MDFF (drop-in for the reference's engforce).

The compute path is libmdff_gpu.so (hand-written sm_100a CUDA behind the C ABI
of include/mdff_gpu.h); this package is the Python host mirror of that ABI.
"""
from . import _abi  # noqa: F401
from .params import make_params, itype_of, charges_of  # noqa: F401
