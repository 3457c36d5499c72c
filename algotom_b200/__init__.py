"""B200-native filtered back-projection with algotom's Python interface.

``algotom_b200.rec.reconstruction`` mirrors the FBP / BPF functions of
``algotom.rec.reconstruction`` (algotom 1.6.0); the compute runs in the
sm_100a kernels of ``algotom_b200/lib/libalgotom_b200.so`` (C ABI declared
in ``include/algotom_b200.h``).
"""
__version__ = "0.1.0"
