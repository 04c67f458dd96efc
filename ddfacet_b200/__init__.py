"""B200-native DDFacet facet gridding/degridding hot path.

Host side in Python over a C ABI (libddfg.so, include/ddfg.h) of hand-written sm_100a kernels.
"""
__version__ = "0.1.0"
