"""B200 (sm_100a) implementation of the ActFEMtide tidal forward path.

``actfemtide_b200.forward.Forward`` is the host API over the C ABI of
``libactfem_gpu.so`` (``include/afem.h``); ``actfemtide_b200.synth`` builds
seeded synthetic models; ``actfemtide_b200.build`` compiles the library.
"""
__all__ = ["forward", "synth", "capi", "build"]
