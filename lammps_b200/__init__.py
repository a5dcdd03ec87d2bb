"""lammps_b200 -- B200-native short-range MD step (LJ + EAM) behind a C ABI.

The engine is ``lammps_b200/_lib/libb200md.so`` (CUDA, sm_100a), declared in
``include/b200md.h``.  This package is its host side for Python callers:
pair-style tables (``pair``), input generators (``inputs``, ``eam_synth``)
and the ``System`` driver; ``lammps/`` holds the LAMMPS package sources
(``pair_style lj/cut/b200``, ``eam/b200``, ``fix nve/b200``).
"""
from .pair import PairEAM, PairEAMAlloy, PairEAMFS, PairLJCut  # noqa: F401
from .system import System  # noqa: F401
from . import inputs  # noqa: F401

__all__ = ["System", "PairLJCut", "PairEAM", "PairEAMAlloy", "PairEAMFS", "inputs"]
