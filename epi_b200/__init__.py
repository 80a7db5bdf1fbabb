"""B200-native cell-mechanics step of the epi5_MT epidermis model.

The product is libepi_mech.so (hand-written sm_100a CUDA kernels behind the C
ABI in include/epi_mech.h). This package builds it (build.py), binds it for
tests and benchmarks (capi.py) and generates synthetic tissues in the
reference's cell-file layout (tissue.py).
"""
