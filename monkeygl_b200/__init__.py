"""MonkeyGL-B200: MonkeyGL's volume ray-casting path (VR, MIP, surface, MPR,
CPR) as hand-written sm_100a CUDA behind a C ABI (include/monkeygl_b200.h).

Submodules:
  capi      ctypes binding of the C ABI (no fallback: the native library must be built)
  camera    MonkeyGL's FP32 camera / volume-factor setup
  phantom   seeded synthetic CT phantoms, transfer functions, CPR paths
  build     in-tree build of the native library
"""
__version__ = "0.1.0"
