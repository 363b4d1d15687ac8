"""B200 `cuda` engine for vfhe's RNS polynomial hot path.

The C ABI (include/vfhe_cuda.h) is the drop-in boundary; the Python modules here
mirror the reference's operator surface over it (arith, mlwe, fhe).
"""
