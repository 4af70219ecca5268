"""B200-native drop-in for ``ccpi.reconstruction.parallelbeam.alg`` and
``ccpi.reconstruction.conebeam.alg`` (CCPi-Reconstruction's Python API for
its iterative CGLS / SIRT / MLEM / CGLS-Tikhonov / CGLS-TV solvers and the
Siddon projectors they drive).

All computation runs in ``libccpi_b200.so`` (hand-written sm_100a CUDA
kernels behind a C ABI, ``include/ccpi_b200.h``); these modules only
validate and marshal numpy arrays.  Importing a solver module without the
built library raises ImportError: there is no CPU fallback.
"""
