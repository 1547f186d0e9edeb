"""B200 (sm_100a) implementation of DVIDE's rigid-body frictional-contact time
step (System::DoTimeStep: collision detection, the APGD cone-complementarity
solve, the half-implicit update).

- libdvide_b200.so: the CUDA kernels behind the C ABI of include/dvide.h
  (sources in csrc/); libdvide_cxx.so: the reference's C++ classes (System,
  Body, APGD, PGJ, PGS, CollisionDetector) over that ABI, include/dvide/*.h.
  Both are built in-tree by build.py (python -m dvide_b200.build).
- _native: the ctypes mirror of the C ABI (NativeScene, NativeBatch,
  NativeServer); it fails loudly when the library is missing.
- scenes, workloads: seeded synthetic scenes and the saved column states the
  tests and bench use.
- replicas: placement of independent scenes on ranks (one process per GPU).
- drivers/settle.cpp: a driver written against the C++ classes.
"""
