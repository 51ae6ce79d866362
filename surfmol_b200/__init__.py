"""surfmol_b200: B200-native multi-system UFF + GridFF FIRE relaxation (sm_100a CUDA).

Host interface: :class:`surfmol_b200.relax.RelaxMulti` over the C ABI declared in
include/surfmol_relax.h; synthetic workloads in :mod:`surfmol_b200.synth`.
"""
from .relax import (RelaxMulti, Topology, SmrError, fire_params, FIRE_DEFAULT, GRID_F32, GRID_F16, GRID_BF16,  # noqa: F401
                    MODE_BATCHED, MODE_PLAIN, ST_RUNNING, ST_CONVERGED, ST_MAXSTEPS, ST_NONFINITE)

__version__ = "0.1"
