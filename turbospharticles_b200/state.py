"""UniversalSimState: host-side SoA particle state crossing the backend boundary.

Mirrors `Sync::UniversalSimState` (source/simulation/sync/state_sim.h): fluid, boundary,
rigid-particle and rigid-body SoA vectors. `view()` exposes the arrays as a C
`tsp_state_view` without copying.
"""
from __future__ import annotations

import ctypes as C

import numpy as np

from .abi import NO_MESH_ID, TspExportSnapshot, TspStateView

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


EXPORT_F32 = {"F": ["xPosF", "yPosF", "zPosF", "velMagF"], "B": ["xPosB", "yPosB", "zPosB", "volB"],
              "R": ["xPosR", "yPosR", "zPosR", "volR"]}


class ExportSnapshot:
    """Mirrors `Sync::ExportSnapshot` (source/simulation/sync/snapshots.h:37-66): the surface
    fluid particles (positions, velocity magnitudes), the boundary particles (positions,
    volumes, mesh flags) and the rigid particles (world positions, volumes, body indices) of
    one export. `rankF` stays empty outside distributed runs, as in the reference."""

    def __init__(self, N_F=0, N_B=0, N_R=0):
        self.simStep, self.simTime = 0, 0.0
        self.N_F, self.N_B, self.N_R = int(N_F), int(N_B), int(N_R)
        for pop, n in (("F", self.N_F), ("B", self.N_B), ("R", self.N_R)):
            for name in EXPORT_F32[pop]:
                setattr(self, name, np.zeros(n, np.float32))
        self.isMeshB = np.zeros(self.N_B, np.uint8)
        self.bodyIdR = np.zeros(self.N_R, np.uint32)
        self.rankF = np.zeros(0, np.uint16)

    @classmethod
    def pack(cls, packer, counts, params_c, include_b=True, mesh_id_begin_b=None):
        """Allocate full-size arrays for the backend's counts, let `packer(cparams, include_b,
        mesh_begin, view)` fill them, and trim each population to the exported count."""
        nF, nB, nR = counts
        snap = cls(nF, nB if include_b else 0, nR)
        v = TspExportSnapshot()
        for name, ctype in TspExportSnapshot._fields_[6:]:
            arr = getattr(snap, name)
            setattr(v, name, arr.ctypes.data_as(ctype) if arr.size else None)
        packer(C.byref(params_c), 1 if include_b else 0,
               NO_MESH_ID if mesh_id_begin_b is None else int(mesh_id_begin_b), C.byref(v))
        snap.simStep, snap.simTime = int(v.simStep), float(v.simTime)
        snap.N_F, snap.N_B, snap.N_R = int(v.N_F), int(v.N_B), int(v.N_R)
        for pop, n in (("F", snap.N_F), ("B", snap.N_B), ("R", snap.N_R)):
            for name in EXPORT_F32[pop]:
                setattr(snap, name, getattr(snap, name)[:n].copy())
        snap.isMeshB = snap.isMeshB[:snap.N_B].copy()
        snap.bodyIdR = snap.bodyIdR[:snap.N_R].copy()
        return snap
