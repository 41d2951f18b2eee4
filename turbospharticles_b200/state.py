"""UniversalSimState: host-side SoA particle state crossing the backend boundary.

Mirrors `Sync::UniversalSimState` (source/simulation/sync/state_sim.h): fluid, boundary,
rigid-particle and rigid-body SoA vectors. `view()` exposes the arrays as a C
`tsp_state_view` without copying.
"""
from __future__ import annotations

import ctypes as C

import numpy as np

from .abi import TspStateView

FLUID_F32 = ["xPosF", "yPosF", "zPosF", "xVelF", "yVelF", "zVelF", "xVelPredF", "yVelPredF",
             "zVelPredF", "xAccPressF", "yAccPressF", "zAccPressF", "sourceTermF", "diagElemF",
             "pressureF", "densityF"]
BOUNDARY_F32 = ["xPosB", "yPosB", "zPosB", "volB", "psiB"]
RIGID_F32 = ["xPosRelR", "yPosRelR", "zPosRelR", "volR", "psiR", "xPosR", "yPosR", "zPosR"]
BODY_F32 = ["xCM", "yCM", "zCM", "xVelRB", "yVelRB", "zVelRB", "xOmegaRB", "yOmegaRB",
            "zOmegaRB", "xAngMomRB", "yAngMomRB", "zAngMomRB", "a00", "a01", "a02", "a10", "a11",
            "a12", "a20", "a21", "a22", "massRB", "massInvRB", "iBodyInv00", "iBodyInv01",
            "iBodyInv02", "iBodyInv10", "iBodyInv11", "iBodyInv12", "iBodyInv20", "iBodyInv21",
            "iBodyInv22"]


class UniversalSimState:
    def __init__(self, N_F=0, N_B=0, N_R=0, N_RB=0, rest_density=1000.0):
        self.N_F, self.N_B, self.N_R, self.N_RB = int(N_F), int(N_B), int(N_R), int(N_RB)
        self.step = 0
        self.time = 0.0
        self.idF = np.arange(self.N_F, dtype=np.uint64)
        for n in FLUID_F32:
            setattr(self, n, np.zeros(self.N_F, np.float32))
        self.densityF[:] = rest_density
        self.idB = np.arange(self.N_B, dtype=np.uint64)
        for n in BOUNDARY_F32:
            setattr(self, n, np.zeros(self.N_B, np.float32))
        self.idR = np.arange(self.N_R, dtype=np.uint64)
        self.bodyIdR = np.zeros(self.N_R, np.uint32)
        for n in RIGID_F32:
            setattr(self, n, np.zeros(self.N_R, np.float32))
        self.idRB = np.arange(self.N_RB, dtype=np.uint64)
        self.rigidParticleCountRB = np.zeros(self.N_RB, np.uint32)
        for n in BODY_F32:
            setattr(self, n, np.zeros(self.N_RB, np.float32))
        for n in ("a00", "a11", "a22"):
            getattr(self, n)[:] = 1.0

    def copy(self) -> "UniversalSimState":
        s = UniversalSimState.__new__(UniversalSimState)
        for k, v in self.__dict__.items():
            setattr(s, k, v.copy() if isinstance(v, np.ndarray) else v)
        return s

    def arrays(self):
        return {k: v for k, v in self.__dict__.items() if isinstance(v, np.ndarray)}

    def view(self) -> TspStateView:
        """C view onto these arrays (the arrays must stay alive while the view is used)."""
        v = TspStateView()
        v.N_F, v.N_B, v.N_R, v.N_RB = self.N_F, self.N_B, self.N_R, self.N_RB
        v.step, v.time = int(self.step), float(self.time)
        for name, ctype in TspStateView._fields_[6:]:
            arr = getattr(self, name, None)
            if arr is None or arr.size == 0:
                setattr(v, name, None)
                continue
            assert arr.flags["C_CONTIGUOUS"]
            setattr(v, name, arr.ctypes.data_as(ctype))
        return v

    def sync_counts_from(self, v: TspStateView):
        self.step, self.time = int(v.step), float(v.time)
