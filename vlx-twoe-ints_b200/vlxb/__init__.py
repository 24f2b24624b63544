"""vlxb: B200-native (sm_100a) two-electron J/K engine.

Drop-in replacement, behind a C ABI (include/vlxb.h, libvlxb.so), for the
computeCoulombFock<ABCD> / computeExchangeFock<ABCD> kernels that
VeloxChem's vlx-twoe-ints generator emits.

  vlxb.basis   synthetic molecules, Cartesian s/p/d basis, densities
  vlxb.lists   reference-format input lists (prim_info, pair lists, Q, D)
  vlxb.fock    J/K builds through the C ABI (torch tensors as device buffers)
  vlxb.gradient  nuclear gradients of 1/2 Tr[D J] and 1/2 Tr[D K] on the device
  vlxb.build   nvcc build of libvlxb.so
"""
__version__ = "0.1.0"
