"""qem4molly_b200 -- B200-native QEM (Quasi-Ewald Method) forces and energies.

The compute path is libqem.so (hand-written sm_100a CUDA behind the C-ABI of
include/qem.h).  This package binds it (ctypes), mirrors the reference's
interaction API (QEM_short, QEM_long, QEM_inter, Substrate_LJ, forces,
potential_energy) and wraps it as a torch.autograd.Function.
"""
from ._lib import (QEM_CUTOFF_PYTHON, QEM_DIR_MINIMAGE, QEM_FP32_FIX, QEM_FP64, QEM_MEM_DEVICE, QEM_MEM_HOST,
                   QEM_PAIR_PHYSICAL, QEM_PYTHON_MODE, QEM_RESAMPLE_KSET, QEM_STALE_NEIGHBORS, QEM_TERM_ALL,
                   QEM_TERM_LJ, QEM_TERM_LONG, QEM_TERM_SHORT, QemError, load)
from .api import QEM_inter, QEM_long, QEM_short, Engine, Substrate_LJ, System, forces, potential_energy

__all__ = ["Engine", "QEM_short", "QEM_long", "QEM_inter", "Substrate_LJ", "System", "forces",
           "potential_energy", "QemError", "load", "QEM_FP64", "QEM_FP32_FIX", "QEM_TERM_SHORT", "QEM_TERM_LONG",
           "QEM_TERM_LJ", "QEM_TERM_ALL", "QEM_MEM_HOST", "QEM_MEM_DEVICE", "QEM_CUTOFF_PYTHON",
           "QEM_DIR_MINIMAGE", "QEM_PAIR_PHYSICAL", "QEM_PYTHON_MODE", "QEM_STALE_NEIGHBORS", "QEM_RESAMPLE_KSET"]
