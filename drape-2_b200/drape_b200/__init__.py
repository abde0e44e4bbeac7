"""Host side of the B200 cloth-solver hot path: scene description, synthetic scenes, and the ctypes binding of the
C-ABI library (include/drape_cuda.h) with the reference's Solver interface on top."""
