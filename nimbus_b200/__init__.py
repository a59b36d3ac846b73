"""Nimbus-B200: a B200-native (sm_100a) CUDA backend for the Nimbus
dynamical-core hot path -- the Klemp-Wilhelmson split-explicit acoustic
substep loop and the conservative WENO5 scalar transport on the Arakawa
C-grid -- behind a C-ABI shared library (include/nimbus_cuda.h)."""
__version__ = "0.1.0"
