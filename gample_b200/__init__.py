"""gample_b200: B200-native particle-in-cell step of gample (sm_100a CUDA).

The product is the C-ABI library libgample_b200.so (include/gample_gpu.h)
and the command-line driver gample_pic, both built from gample_b200/csrc by
gample_b200/Makefile. This package exposes the Python binding of the C ABI.
"""
import os
import subprocess

HERE = os.path.dirname(os.path.abspath(__file__))


def build(jobs=8):
    """Compile the CUDA library and driver in-tree (sm_100a)."""
    subprocess.run(["make", "-s", "-C", HERE, f"-j{jobs}"], check=True)


from . import capi  # noqa: E402
from .capi import Init, Sim, GampleError  # noqa: E402,F401
