"""B200-native Barnes-Hut step behind the Simulation backend interface of
PhivPap/n-body-2d.  The compute path is libnbody_b200.so (CUDA, sm_100a) with
the C ABI in include/nbody_b200.h; this package is its host side."""
from . import csvio, render, universes
from ._lib import (NB_FLAG_CPU_LAW, NB_FLAG_LEARNED, NB_FLAG_QUADRUPOLE, NB_MLP_PARAMS,
                   NB_MODE_ALLPAIRS, NB_MODE_FP64, NB_MODE_SPLIT, NB_STATIC_SORT_MAX_BODIES,
                   EXPORTS, LIB_PATH, NbError, NbParams, NbStats, NbView, load)
from .simulation import (BarnesHutB200, Bodies, NbContext, SimConfig, Simulation, State, Stats,
                         allpairs_accelerations, mlp_forward, mlp_loss_grad, mlp_train)

__all__ = [
    "csvio", "render", "universes",
    "NB_FLAG_CPU_LAW", "NB_FLAG_LEARNED", "NB_FLAG_QUADRUPOLE", "NB_MLP_PARAMS",
    "NB_MODE_ALLPAIRS", "NB_MODE_FP64", "NB_MODE_SPLIT", "NB_STATIC_SORT_MAX_BODIES",
    "EXPORTS", "LIB_PATH", "NbError", "NbParams", "NbStats", "NbView", "load",
    "BarnesHutB200", "Bodies", "NbContext", "SimConfig", "Simulation", "State", "Stats",
    "allpairs_accelerations", "mlp_forward", "mlp_loss_grad", "mlp_train",
]
