"""B200-native direct evaluation of the nodal-DG Boltzmann collision integral.

The compute path is libdgv_b200.so (hand-written sm_100a CUDA behind the C-ABI in
include/dgv_b200.h); this package is its host-side mirror.  Importing the
package loads the library and raises if it has not been built.
"""
from ._lib import DGVError, load as _load
from .solver import DGVSolver, collide_group

_load()

__all__ = ["DGVSolver", "DGVError", "collide_group"]
