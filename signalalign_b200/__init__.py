"""B200-native engine for signalAlign's banded, anchored 3-state pair-HMM forward-backward.

The product is the C-ABI library libsa_b200.so (include/sa_b200.h): hand-written sm_100a kernels
plus the C++ host planner.  `signalalign_b200.api` is its Python mirror; `signalalign_b200.synth`
generates the seeded synthetic workloads of the benchmark.
"""
import os

PACKAGE_DIR = os.path.dirname(os.path.abspath(__file__))
LIB_PATH = os.path.join(PACKAGE_DIR, "libsa_b200.so")

__all__ = ["PACKAGE_DIR", "LIB_PATH"]
