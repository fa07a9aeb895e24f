"""B200 (sm_100a) implementation of the static-exchange per-energy scattering path.

Modules:
  _lib     ctypes binding of libscatt_b200.so (C ABI in include/scatt_b200.h)
  solver   ScanSolver: upload a scan once, solve batches of energies
  synth    seeded synthetic molecular inputs of the benchmark shapes
"""
